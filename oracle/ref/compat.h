// compat.h -- force-included (nvcc -include) when the reference's CUDA kernel
// files are compiled as a test oracle.  TEST INFRASTRUCTURE ONLY.
//
// The reference binds file-scope legacy texture references
// (texture<T, dim, mode> globals + cudaBindTextureToArray), which CUDA 12
// removed.  This header maps each such global onto a managed struct holding
// the same settings and a texture object, so the reference sources compile
// unmodified and sample with the same unnormalised / border / linear texture
// state.  It also routes cudaMemcpyToArray through cudaMemcpyDefault, since
// the reference passes device pointers with cudaMemcpyHostToDevice.
#pragma once

#include <cuda_runtime.h>
#include <texture_indirect_functions.h>

#include <cstdio>   // the TF headers the reference includes provide these
#include <cstdlib>

template <class T, int Dim = 1, enum cudaTextureReadMode Mode = cudaReadModeElementType>
struct compat_texture {
    cudaTextureAddressMode addressMode[3];
    cudaTextureFilterMode filterMode;
    int normalized;
    cudaTextureObject_t obj;
};

// `texture<float, 3, cudaReadModeElementType> volume_as_texture;` becomes a
// managed (host- and device-visible) compat_texture global.
#define texture __managed__ compat_texture

template <class T, int D, enum cudaTextureReadMode M>
__device__ __forceinline__ T tex2D(const compat_texture<T, D, M> &t, float x, float y)
{
    return tex2D<T>(t.obj, x, y);
}

template <class T, int D, enum cudaTextureReadMode M>
__device__ __forceinline__ T tex3D(const compat_texture<T, D, M> &t, float x, float y, float z)
{
    return tex3D<T>(t.obj, x, y, z);
}

template <class T, int D, enum cudaTextureReadMode M>
__device__ __forceinline__ T tex2DLayered(const compat_texture<T, D, M> &t, float x, float y, int layer)
{
    return tex2DLayered<T>(t.obj, x, y, layer);
}

template <class T, int D, enum cudaTextureReadMode M>
static cudaError_t cudaBindTextureToArray(compat_texture<T, D, M> &t, cudaArray_const_t array,
                                          const cudaChannelFormatDesc &)
{
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = const_cast<cudaArray_t>(array);
    cudaTextureDesc td = {};
    for (int i = 0; i < 3; ++i) td.addressMode[i] = t.addressMode[i];
    td.filterMode = t.filterMode;
    td.readMode = M;
    td.normalizedCoords = t.normalized;
    // the previous launch may still read the old object; objects are leaked
    // on purpose (tiny) instead of being destroyed under a running kernel
    cudaTextureObject_t obj = 0;
    cudaError_t e = cudaCreateTextureObject(&obj, &res, &td, nullptr);
    if (e != cudaSuccess) return e;
    cudaDeviceSynchronize();
    t.obj = obj;
    return cudaSuccess;
}

template <class T, int D, enum cudaTextureReadMode M>
static cudaError_t cudaUnbindTexture(compat_texture<T, D, M> &)
{
    return cudaSuccess;
}

static cudaError_t compat_memcpy_to_array(cudaArray_t dst, size_t w_offset, size_t h_offset, const void *src,
                                          size_t count, cudaMemcpyKind)
{
    cudaChannelFormatDesc desc;
    cudaExtent ext;
    unsigned flags;
    cudaError_t e = cudaArrayGetInfo(&desc, &ext, &flags, dst);
    if (e != cudaSuccess) return e;
    const size_t elem = (desc.x + desc.y + desc.z + desc.w) / 8;
    const size_t row = ext.width * elem;
    const size_t rows = row ? count / row : 0;
    return cudaMemcpy2DToArray(dst, w_offset, h_offset, src, row, row, rows, cudaMemcpyDefault);
}
#define cudaMemcpyToArray compat_memcpy_to_array

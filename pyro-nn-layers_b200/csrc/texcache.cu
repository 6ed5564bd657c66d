// texcache.cu -- CUDA arrays and texture objects for the hardware_interp paths.
//
// Texture filtering needs the data in a CUDA array.  The reference allocates
// a fresh array, copies the whole input into it and frees it on every call
// (cone_projector_3D_CudaKernel_hardware_interp.cu.cc:221-243,258;
// cone_backprojector_3D_CudaKernel_hardware_interp.cu.cc:129-142,159).  Here the
// arrays are kept in a per-device cache keyed by kind/extent/texel format and
// handed out stream-aware: an entry is reused on the stream that used it last
// (stream order makes that safe) or on any stream once the event recorded
// after its last use has completed; otherwise a new entry is created.
// The copy into the array is a kernel writing through a surface object, so
// BF16 input can be widened on the way (the texture unit has no BF16 texel
// format; BF16 and FP16 storage both use FP16 texels, FP32 uses FP32 texels).
#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.h"

namespace pyronn {

struct CachedArray {
    int device;
    int kind;
    int w, h, d;
    bool half_texels;
    cudaArray_t array;
    cudaTextureObject_t tex;
    cudaSurfaceObject_t surf;
    cudaStream_t last_stream;
    cudaEvent_t done;
    bool busy;
};

namespace {

std::mutex g_mu;
std::vector<CachedArray *> g_entries;

template <typename T, bool HALF>
__global__ void fill_volume_kernel(const T *__restrict__ src, cudaSurfaceObject_t surf, int w, int h, int d)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int z = blockIdx.z;
    if (x >= w) return;
    const float v = load_as_float(src + ((size_t)z * h + y) * w + x);
    if (HALF)
        surf3Dwrite(__half_as_ushort(__float2half_rn(v)), surf, x * (int)sizeof(__half), y, z);
    else
        surf3Dwrite(v, surf, x * (int)sizeof(float), y, z);
}

template <typename T, bool HALF>
__global__ void fill_layered_kernel(const T *__restrict__ src, cudaSurfaceObject_t surf, int w, int h, int d)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int layer = blockIdx.z;
    if (x >= w) return;
    const float v = load_as_float(src + ((size_t)layer * h + y) * w + x);
    if (HALF)
        surf2DLayeredwrite(__half_as_ushort(__float2half_rn(v)), surf, x * (int)sizeof(__half), y, layer);
    else
        surf2DLayeredwrite(v, surf, x * (int)sizeof(float), y, layer);
}

template <typename T>
cudaError_t fill_typed(CachedArray *a, const void *src, cudaStream_t stream)
{
    // extents are bounded by the texture limits (<= 65535 in y and z)
    const dim3 block(128);
    const dim3 grid((a->w + 127) / 128, a->h, a->d);
    const T *s = (const T *)src;
    if (a->kind == ARRAY_VOLUME_3D) {
        if (a->half_texels)
            fill_volume_kernel<T, true><<<grid, block, 0, stream>>>(s, a->surf, a->w, a->h, a->d);
        else
            fill_volume_kernel<T, false><<<grid, block, 0, stream>>>(s, a->surf, a->w, a->h, a->d);
    } else {
        if (a->half_texels)
            fill_layered_kernel<T, true><<<grid, block, 0, stream>>>(s, a->surf, a->w, a->h, a->d);
        else
            fill_layered_kernel<T, false><<<grid, block, 0, stream>>>(s, a->surf, a->w, a->h, a->d);
    }
    return cudaGetLastError();
}

void destroy_entry(CachedArray *e)
{
    if (e->tex) cudaDestroyTextureObject(e->tex);
    if (e->surf) cudaDestroySurfaceObject(e->surf);
    if (e->array) cudaFreeArray(e->array);
    if (e->done) cudaEventDestroy(e->done);
    delete e;
}

cudaError_t create_entry(int device, int kind, int w, int h, int d, bool half_texels, CachedArray **out)
{
    CachedArray *e = new CachedArray();
    e->device = device;
    e->kind = kind;
    e->w = w;
    e->h = h;
    e->d = d;
    e->half_texels = half_texels;
    cudaChannelFormatDesc desc = half_texels ? cudaCreateChannelDescHalf() : cudaCreateChannelDesc<float>();
    const unsigned flags = cudaArraySurfaceLoadStore | (kind == ARRAY_SINOGRAM_LAYERED ? cudaArrayLayered : 0);
    cudaError_t err = cudaMalloc3DArray(&e->array, &desc, make_cudaExtent(w, h, d), flags);
    if (err != cudaSuccess) {
        delete e;
        return err;
    }
    cudaResourceDesc res = {};
    res.resType = cudaResourceTypeArray;
    res.res.array.array = e->array;
    cudaTextureDesc td = {};
    // border addressing, linear filtering, unnormalised coordinates: the
    // reference's texture settings (e.g. ..._hardware_interp.cu.cc:203-208)
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    err = cudaCreateTextureObject(&e->tex, &res, &td, nullptr);
    if (err == cudaSuccess) err = cudaCreateSurfaceObject(&e->surf, &res);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->done, cudaEventDisableTiming);
    if (err != cudaSuccess) {
        destroy_entry(e);
        return err;
    }
    *out = e;
    return cudaSuccess;
}

}  // namespace

cudaError_t array_acquire(int kind, int w, int h, int d, bool half_texels, cudaStream_t stream, CachedArray **out)
{
    int device = 0;
    cudaError_t err = cudaGetDevice(&device);
    if (err != cudaSuccess) return err;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        CachedArray *pick = nullptr;
        for (CachedArray *e : g_entries) {
            if (e->busy || e->device != device || e->kind != kind || e->w != w || e->h != h || e->d != d ||
                e->half_texels != half_texels)
                continue;
            if (e->last_stream == stream) {
                pick = e;
                break;
            }
            if (!pick && cudaEventQuery(e->done) == cudaSuccess) pick = e;
        }
        if (pick) {
            pick->busy = true;
            *out = pick;
            return cudaSuccess;
        }
    }
    CachedArray *e = nullptr;
    err = create_entry(device, kind, w, h, d, half_texels, &e);
    if (err != cudaSuccess) return err;
    e->busy = true;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        g_entries.push_back(e);
    }
    *out = e;
    return cudaSuccess;
}

cudaTextureObject_t array_texture(CachedArray *a)
{
    return a->tex;
}

cudaError_t array_fill(CachedArray *a, const void *src, int dtype, cudaStream_t stream)
{
    if (a->d > 65535) return cudaErrorInvalidValue;
    switch (dtype) {
    case PYRONN_FLOAT32: return fill_typed<float>(a, src, stream);
    case PYRONN_BFLOAT16: return fill_typed<__nv_bfloat16>(a, src, stream);
    case PYRONN_FLOAT16: return fill_typed<__half>(a, src, stream);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t array_release(CachedArray *a, cudaStream_t stream)
{
    cudaError_t err = cudaEventRecord(a->done, stream);
    std::lock_guard<std::mutex> lock(g_mu);
    a->last_stream = stream;
    a->busy = false;
    return err;
}

int array_cache_clear()
{
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return -1;
    cudaError_t err = cudaDeviceSynchronize();
    std::lock_guard<std::mutex> lock(g_mu);
    std::vector<CachedArray *> keep;
    int freed = 0;
    for (CachedArray *e : g_entries) {
        if (e->device == device && !e->busy) {
            destroy_entry(e);
            ++freed;
        } else {
            keep.push_back(e);
        }
    }
    g_entries.swap(keep);
    return err == cudaSuccess ? freed : -1;
}

}  // namespace pyronn

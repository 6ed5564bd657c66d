// cone_bp.cu -- voxel-driven cone-beam backprojector (ConeBackprojection3D).
//
// vol[z,y,x] = multiplier * sum_n interp(sino_n, u/w, v/w) / w^2 with
// (u, v, w) = P_n (x, y, z, 1) (cone_backprojector_3D_CudaKernel.cu.cc:84-118).
// The projection matrices are pre-multiplied in FP64 into voxel-index space
// (geometry.cu), so (u, v, w) is an affine function of the voxel index and
// each thread walks ZB voxels along z with one FMA per coordinate.
//
// Software interpolation keeps interp2D's `>` bounds
// (cone_backprojector_3D_CudaKernel.cu.cc:68-71): taps 0 <= x <= W,
// 0 <= y <= H are read from the flat sinogram (x == W is the next row's first
// texel, y == H the next view's first row); a tap past the end of the
// sinogram buffer -- undefined behaviour in the reference -- reads zero.
// Hardware interpolation samples a layered texture at (u + 0.5, v + 0.5, n)
// with border addressing, as cone_backprojector_3D_CudaKernel_hardware_interp.cu.cc:81,115-119.
#include "common.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int BP_BLOCK_X = 32;
constexpr int BP_BLOCK_Y = 4;
constexpr int BP_ZB = 8;  // voxels per thread along z

template <typename T>
__device__ __forceinline__ float interp2d_quirk(const T *__restrict__ sino, float u, float v, unsigned view_base,
                                                int W, int H, unsigned total)
{
    const float fu = floorf(u), fv = floorf(v);
    const float tx = u - fu, ty = v - fv;
    // comparisons on the float floors: no integer overflow for far-off
    // coordinates, and a NaN coordinate selects no tap
    const float fw = (float)W, fh = (float)H;
    const bool vx0 = fu >= 0.0f && fu <= fw;
    const bool vx1 = fu >= -1.0f && fu <= fw - 1.0f;
    const bool vy0 = fv >= 0.0f && fv <= fh;
    const bool vy1 = fv >= -1.0f && fv <= fh - 1.0f;
    // saturating conversions; the index is only used when its tap is valid
    const int x0 = __float2int_rz(fu), y0 = __float2int_rz(fv);
    const unsigned i00 = view_base + (unsigned)y0 * (unsigned)W + (unsigned)x0;
    const unsigned i01 = i00 + 1u;
    const unsigned i10 = i00 + (unsigned)W;
    const unsigned i11 = i10 + 1u;
    const float p00 = (vx0 && vy0 && i00 < total) ? load_as_float(sino + i00) : 0.0f;
    const float p01 = (vx1 && vy0 && i01 < total) ? load_as_float(sino + i01) : 0.0f;
    const float p10 = (vx0 && vy1 && i10 < total) ? load_as_float(sino + i10) : 0.0f;
    const float p11 = (vx1 && vy1 && i11 < total) ? load_as_float(sino + i11) : 0.0f;
    const float p0 = lerp_first<T>(p00, p01, tx);
    const float p1 = lerp_first<T>(p10, p11, tx);
    return lerp_ref(p0, p1, ty);
}

template <typename T, typename Tout, bool HW>
__global__ void __launch_bounds__(BP_BLOCK_X *BP_BLOCK_Y)
    cone_bp_kernel(const T *__restrict__ sino, Tout *__restrict__ vol, const ConeBpView *__restrict__ views,
                   const float *__restrict__ mult, int X, int Y, int Z, int W, int H, int n_proj, int geom_batch,
                   int batch_begin, cudaTextureObject_t tex)
{
    const int i = blockIdx.x * BP_BLOCK_X + threadIdx.x;
    const int j = blockIdx.y * BP_BLOCK_Y + threadIdx.y;
    const int zblocks = (Z + BP_ZB - 1) / BP_ZB;
    const int k0 = (blockIdx.z % zblocks) * BP_ZB;
    const int b = batch_begin + blockIdx.z / zblocks;
    if (i >= X || j >= Y) return;
    const int g = geom_batch == 1 ? 0 : b;
    const ConeBpView *pv = views + (size_t)g * n_proj;
    const T *sino_b = sino + (size_t)b * n_proj * H * W;
    const unsigned total = (unsigned)n_proj * (unsigned)H * (unsigned)W;

    float acc[BP_ZB];
#pragma unroll
    for (int z = 0; z < BP_ZB; ++z) acc[z] = 0.0f;

    const float fi = (float)i, fj = (float)j, fk = (float)k0;
    for (int n = 0; n < n_proj; ++n) {
        const float4 r0 = __ldg(&pv[n].row[0]);
        const float4 r1 = __ldg(&pv[n].row[1]);
        const float4 r2 = __ldg(&pv[n].row[2]);
        const float ub = fmaf(r0.x, fi, fmaf(r0.y, fj, fmaf(r0.z, fk, r0.w)));
        const float vb = fmaf(r1.x, fi, fmaf(r1.y, fj, fmaf(r1.z, fk, r1.w)));
        const float wb = fmaf(r2.x, fi, fmaf(r2.y, fj, fmaf(r2.z, fk, r2.w)));
        const unsigned view_base = (unsigned)n * (unsigned)H * (unsigned)W;
#pragma unroll
        for (int z = 0; z < BP_ZB; ++z) {
            const float fz = (float)z;
            const float un = fmaf(r0.z, fz, ub);
            const float vn = fmaf(r1.z, fz, vb);
            const float wn = fmaf(r2.z, fz, wb);
            const float rw = fast_rcp(wn);
            const float uu = un * rw, vv = vn * rw;
            float val;
            if (HW)
                val = tex2DLayered<float>(tex, uu + 0.5f, vv + 0.5f, n);
            else
                val = interp2d_quirk<T>(sino_b, uu, vv, view_base, W, H, total);
            acc[z] = fmaf(val * rw, rw, acc[z]);
        }
    }
    const float m = mult[g];
    Tout *vol_b = vol + (size_t)b * Z * Y * X;
#pragma unroll
    for (int z = 0; z < BP_ZB; ++z) {
        if (k0 + z < Z) store_from_float(vol_b + ((size_t)(k0 + z) * Y + j) * X + i, acc[z] * m);
    }
}

template <typename Tin, typename Tout>
cudaError_t launch_typed(const void *sinogram, void *volume, const Dims3D &d, int batch_begin, int batch_count,
                         const ConeBpView *views, const float *mult, cudaTextureObject_t tex, cudaStream_t stream)
{
    const dim3 block(BP_BLOCK_X, BP_BLOCK_Y, 1);
    const int zblocks = (d.vol_z + BP_ZB - 1) / BP_ZB;
    const int per_launch = (65535 / zblocks) > 0 ? (65535 / zblocks) : 1;
    for (int b0 = 0; b0 < batch_count; b0 += per_launch) {
        const int nb = (batch_count - b0) < per_launch ? (batch_count - b0) : per_launch;
        const dim3 grid((d.vol_x + BP_BLOCK_X - 1) / BP_BLOCK_X, (d.vol_y + BP_BLOCK_Y - 1) / BP_BLOCK_Y,
                        zblocks * nb);
        if (tex)  // the texture holds the data; the input pointer is not read
            cone_bp_kernel<float, Tout, true><<<grid, block, 0, stream>>>(
                nullptr, (Tout *)volume, views, mult, d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h, d.n_proj,
                d.geom_batch, batch_begin + b0, tex);
        else
            cone_bp_kernel<Tin, Tout, false><<<grid, block, 0, stream>>>(
                (const Tin *)sinogram, (Tout *)volume, views, mult, d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h,
                d.n_proj, d.geom_batch, batch_begin + b0, tex);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_cone_bp(const void *sinogram, void *volume, int in_dtype, int out_dtype, const Dims3D &d,
                           int batch_index, const ConeBpView *views, const float *mult, cudaTextureObject_t tex,
                           cudaStream_t stream)
{
    const int b0 = batch_index < 0 ? 0 : batch_index;
    const int nb = batch_index < 0 ? d.batch : 1;
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return launch_typed<Tin, Tout>(sinogram, volume, d, b0, nb, views, mult, tex, stream);
    });
}

}  // namespace pyronn

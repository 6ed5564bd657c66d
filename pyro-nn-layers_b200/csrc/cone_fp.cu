// cone_fp.cu -- ray-driven cone-beam forward projector (ConeProjection3D).
//
// One thread per detector ray, warps laid along detector-u so the sinogram
// writes coalesce.  Per ray, the direction, the box entry/exit parameters and
// the source are FP64 (long lever arms: the source sits ~1500 voxels from the
// grid); the march itself is FP32 with alpha advanced exactly as the reference
// does (`min_alpha += step_size` on a float, cone_projector_3D_CudaKernel.cu.cc:135-159),
// so sample positions match the reference's.
//
// Software interpolation (hardware_interp = false) reproduces interp3D of
// cone_projector_3D_CudaKernel.cu.cc:42-85: box [0, N], taps outside [0, N-1]
// read as zero, lerps in the reference's FMA form.  Hardware interpolation
// (hardware_interp = true) samples a 3D texture at p + 0.5 with border
// addressing and box [-0.5, N-0.5], as
// cone_projector_3D_CudaKernel_hardware_interp.cu.cc:43-142 does; its kernel
// runs the block order of the cell forward projector (cone_ray.cuh:
// neighbouring views of a detector tile together) with warps along detector
// u -- the texture's block-linear layout keeps x/y neighbours close, z
// neighbours far, so warps along v are 1.7x slower here -- and the counted
// march where the alpha sequence is exact.
#include <math_constants.h>

#include "common.cuh"
#include "cone_ray.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int FP_BLOCK_X = 32;
constexpr int FP_BLOCK_Y = 8;

template <typename T>
__device__ __forceinline__ float interp3d_sw(const T *__restrict__ vol, float x, float y, float z, int X, int Y,
                                             int Z)
{
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    const float tx = x - fx, ty = y - fy, tz = z - fz;
    const bool vx0 = (unsigned)x0 < (unsigned)X, vx1 = (unsigned)(x0 + 1) < (unsigned)X;
    const bool vy0 = (unsigned)y0 < (unsigned)Y, vy1 = (unsigned)(y0 + 1) < (unsigned)Y;
    const bool vz0 = (unsigned)z0 < (unsigned)Z, vz1 = (unsigned)(z0 + 1) < (unsigned)Z;
    const int sy = X, sz = X * Y;
    const int base = z0 * sz + y0 * sy + x0;
    const float p000 = (vz0 && vy0 && vx0) ? load_as_float(vol + base) : 0.0f;
    const float p001 = (vz0 && vy0 && vx1) ? load_as_float(vol + base + 1) : 0.0f;
    const float p010 = (vz0 && vy1 && vx0) ? load_as_float(vol + base + sy) : 0.0f;
    const float p011 = (vz0 && vy1 && vx1) ? load_as_float(vol + base + sy + 1) : 0.0f;
    const float p100 = (vz1 && vy0 && vx0) ? load_as_float(vol + base + sz) : 0.0f;
    const float p101 = (vz1 && vy0 && vx1) ? load_as_float(vol + base + sz + 1) : 0.0f;
    const float p110 = (vz1 && vy1 && vx0) ? load_as_float(vol + base + sz + sy) : 0.0f;
    const float p111 = (vz1 && vy1 && vx1) ? load_as_float(vol + base + sz + sy + 1) : 0.0f;
    const float p00 = lerp_first<T>(p000, p100, tz);
    const float p01 = lerp_first<T>(p001, p101, tz);
    const float p10 = lerp_first<T>(p010, p110, tz);
    const float p11 = lerp_first<T>(p011, p111, tz);
    const float p0 = lerp_ref(p00, p10, ty);
    const float p1 = lerp_ref(p01, p11, ty);
    return lerp_ref(p0, p1, tx);
}

template <typename T, bool HW>
struct Sampler {
    const T *vol;
    cudaTextureObject_t tex;
    int X, Y, Z;
    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        if (HW) return tex3D<float>(tex, x + 0.5f, y + 0.5f, z + 0.5f);
        return interp3d_sw<T>(vol, x, y, z, X, Y, Z);
    }
};

template <typename T, typename Tout, bool HW>
__global__ void __launch_bounds__(FP_BLOCK_X *FP_BLOCK_Y)
    cone_fp_kernel(const T *__restrict__ vol, Tout *__restrict__ sino, const ConeFpView *__restrict__ views,
                   const float *__restrict__ step_ptr, const float *__restrict__ spacing_ptr, int X, int Y, int Z,
                   int W, int H, int n_proj, int geom_batch, int batch_begin, cudaTextureObject_t tex)
{
    const int u = blockIdx.x * FP_BLOCK_X + threadIdx.x;
    const int v = blockIdx.y * FP_BLOCK_Y + threadIdx.y;
    const int p = blockIdx.z % n_proj;
    const int b = batch_begin + blockIdx.z / n_proj;
    if (u >= W || v >= H) return;
    const int g = geom_batch == 1 ? 0 : b;
    const float step = step_ptr[g];
    const ConeFpView &view = views[(size_t)g * n_proj + p];
    float pixel = 0.0f;
    if (in_footprint(view, u, v)) {
        const ConeRay ray = cone_ray_setup(view, u, v, X, Y, Z, HW ? -0.5 : 0.0, step, spacing_ptr[g * 3 + 2],
                                           spacing_ptr[g * 3 + 1], spacing_ptr[g * 3 + 0]);
        const Sampler<T, HW> sample{vol + (size_t)b * X * Y * Z, tex, X, Y, Z};
        pixel = cone_ray_march<false>(ray, step, sample);
    }
    store_from_float(sino + (((size_t)b * n_proj + p) * H + v) * (size_t)W + u, pixel);
}

static_assert(FP_BLOCK_X == 32 && FP_BLOCK_Y == 8, "the ray kernels index threads as 32 x 8");

struct TexSampler {
    cudaTextureObject_t tex;
    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        return tex3D<float>(tex, x + 0.5f, y + 0.5f, z + 0.5f);
    }
};

// hardware_interp forward of batch element b: grid ray_block_count blocks of
// 32 x 8 threads, a warp is 32 consecutive u
template <typename Tout>
__global__ void __launch_bounds__(256)
    cone_fp_tex_kernel(cudaTextureObject_t tex, Tout *__restrict__ sino, const ConeFpView *__restrict__ views,
                       const float *__restrict__ step_ptr, const float *__restrict__ spacing_ptr, int X, int Y,
                       int Z, int W, int H, int n_proj, int geom_batch, int b)
{
    const RayBlock rb = ray_block(blockIdx.x, W, H, n_proj);
    const int u = rb.tile_u * 32 + threadIdx.x, v = rb.tile_v * 32 + rb.sub * 8 + threadIdx.y;
    if (u >= W || v >= H) return;
    const int g = geom_batch == 1 ? 0 : b;
    const float step = step_ptr[g];
    const ConeFpView &view = views[(size_t)g * n_proj + rb.p];
    float pixel = 0.0f;
    if (in_footprint(view, u, v)) {
        const ConeRay ray = cone_ray_setup(view, u, v, X, Y, Z, -0.5, step, spacing_ptr[g * 3 + 2],
                                           spacing_ptr[g * 3 + 1], spacing_ptr[g * 3 + 0]);
        const TexSampler s{tex};
        const int n = exact_sample_count(ray, step);
        pixel = n > 0 ? march_counted_x2(ray, n, step, s) : march_x2(ray, step, s);
    }
    store_from_float(sino + (((size_t)b * n_proj + rb.p) * H + v) * (size_t)W + u, pixel);
}

template <typename Tin, typename Tout>
cudaError_t launch_typed(const void *volume, void *sinogram, const Dims3D &d, int batch_begin, int batch_count,
                         const ConeFpView *views, const float *step, const float *spacing, cudaTextureObject_t tex,
                         cudaStream_t stream)
{
    const dim3 block(FP_BLOCK_X, FP_BLOCK_Y, 1);  // 32 x 8, the layout both kernels index by
    if (tex && ray_blocks_fit(d.det_w, d.det_h, d.n_proj)) {  // the texture holds batch element batch_begin
        cone_fp_tex_kernel<Tout><<<ray_block_count(d.det_w, d.det_h, d.n_proj), block, 0, stream>>>(
            tex, (Tout *)sinogram, views, step, spacing, d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h, d.n_proj,
            d.geom_batch, batch_begin);
        return cudaGetLastError();
    }
    // grid.z covers (batch, view) pairs, at most 65535 per launch
    const int per_launch = (65535 / d.n_proj) > 0 ? (65535 / d.n_proj) : 1;
    for (int b0 = 0; b0 < batch_count; b0 += per_launch) {
        const int nb = (batch_count - b0) < per_launch ? (batch_count - b0) : per_launch;
        const dim3 grid((d.det_w + FP_BLOCK_X - 1) / FP_BLOCK_X, (d.det_h + FP_BLOCK_Y - 1) / FP_BLOCK_Y,
                        d.n_proj * nb);
        if (tex)  // the texture holds the data; the input pointer is not read
            cone_fp_kernel<float, Tout, true><<<grid, block, 0, stream>>>(
                nullptr, (Tout *)sinogram, views, step, spacing, d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h,
                d.n_proj, d.geom_batch, batch_begin + b0, tex);
        else
            cone_fp_kernel<Tin, Tout, false><<<grid, block, 0, stream>>>(
                (const Tin *)volume, (Tout *)sinogram, views, step, spacing, d.vol_x, d.vol_y, d.vol_z, d.det_w,
                d.det_h, d.n_proj, d.geom_batch, batch_begin + b0, tex);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

// With a texture (hardware_interp) the texture holds batch element
// batch_index only; without one every batch element runs in one launch
// (batch_index < 0).
cudaError_t launch_cone_fp(const void *volume, void *sinogram, int in_dtype, int out_dtype, const Dims3D &d,
                           int batch_index, const ConeFpView *views, const float *step, const float *spacing,
                           cudaTextureObject_t tex, cudaStream_t stream)
{
    const int b0 = batch_index < 0 ? 0 : batch_index;
    const int nb = batch_index < 0 ? d.batch : 1;
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return launch_typed<Tin, Tout>(volume, sinogram, d, b0, nb, views, step, spacing, tex, stream);
    });
}

}  // namespace pyronn

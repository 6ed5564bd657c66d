// cone_matched.cu -- matched cone backprojector: the exact transpose of the
// software-interpolation forward projector.
//
// The reference's backprojector (voxel-driven, bilinear on the detector,
// 1/w^2 weights, cone_backprojector_3D_CudaKernel.cu.cc:84-118) is not the
// transpose of its ray-driven projector, so <A x, y> != <x, A^T y>.  This
// kernel walks every ray with the forward projector's samples and weights
// (cone_ray.cuh, linear form) and scatters sino[ray] * weight * trilinear
// weight into the eight taps with FP32 atomics: the result is A^T y for the
// linear forward operator, which equals the reference forward projector on
// every ray whose line integral is > 0 (e.g. any non-negative volume).
#include "common.cuh"
#include "cone_ray.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int MB_X = 32;
constexpr int MB_Y = 8;

__device__ __forceinline__ void scatter_trilinear(float *__restrict__ vol, float x, float y, float z, float val,
                                                  int X, int Y, int Z)
{
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int x0 = (int)fx, y0 = (int)fy, z0 = (int)fz;
    const float tx = x - fx, ty = y - fy, tz = z - fz;
    // weights of lerp_ref(a, b, t) = a (1 - t) + b t
    const float wx[2] = {1.0f - tx, tx}, wy[2] = {1.0f - ty, ty}, wz[2] = {1.0f - tz, tz};
#pragma unroll
    for (int dz = 0; dz < 2; ++dz) {
        const int zz = z0 + dz;
        if ((unsigned)zz >= (unsigned)Z) continue;
#pragma unroll
        for (int dy = 0; dy < 2; ++dy) {
            const int yy = y0 + dy;
            if ((unsigned)yy >= (unsigned)Y) continue;
            const float wzy = val * wz[dz] * wy[dy];
#pragma unroll
            for (int dx = 0; dx < 2; ++dx) {
                const int xx = x0 + dx;
                if ((unsigned)xx >= (unsigned)X) continue;
                atomicAdd(vol + ((size_t)zz * Y + yy) * X + xx, wzy * wx[dx]);
            }
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(MB_X *MB_Y)
    cone_scatter_kernel(const T *__restrict__ sino, float *__restrict__ vol, const ConeFpView *__restrict__ views,
                        const float *__restrict__ step_ptr, const float *__restrict__ spacing_ptr, int X, int Y,
                        int Z, int W, int H, int n_proj, int geom_batch)
{
    const int u = blockIdx.x * MB_X + threadIdx.x;
    const int v = blockIdx.y * MB_Y + threadIdx.y;
    const int p = blockIdx.z % n_proj;
    const int b = blockIdx.z / n_proj;
    if (u >= W || v >= H) return;
    const float y = load_as_float(sino + (((size_t)b * n_proj + p) * H + v) * (size_t)W + u);
    if (y == 0.0f) return;
    const int g = geom_batch == 1 ? 0 : b;
    const float step = step_ptr[g];
    if (!in_footprint(views[(size_t)g * n_proj + p], u, v)) return;
    const ConeRay ray = cone_ray_setup(views[(size_t)g * n_proj + p], u, v, X, Y, Z, 0.0, step,
                                       spacing_ptr[g * 3 + 2], spacing_ptr[g * 3 + 1], spacing_ptr[g * 3 + 0]);
    float *vol_b = vol + (size_t)b * Z * Y * X;
    cone_ray_weights(ray, step, [&](float px, float py, float pz, float w) {
        scatter_trilinear(vol_b, px, py, pz, y * w, X, Y, Z);
    });
}

}  // namespace

cudaError_t launch_cone_scatter(const void *sinogram, float *volume, int in_dtype, const Dims3D &d,
                                const ConeFpView *views, const float *step, const float *spacing,
                                cudaStream_t stream)
{
    cudaError_t e = cudaMemsetAsync(volume, 0, sizeof(float) * (size_t)d.batch * d.vol_z * d.vol_y * d.vol_x, stream);
    if (e != cudaSuccess) return e;
    const dim3 block(MB_X, MB_Y);
    const dim3 grid((d.det_w + MB_X - 1) / MB_X, (d.det_h + MB_Y - 1) / MB_Y, d.n_proj * d.batch);
    if (grid.z > 65535) return cudaErrorInvalidConfiguration;
    switch (in_dtype) {
    case PYRONN_FLOAT32:
        cone_scatter_kernel<float><<<grid, block, 0, stream>>>((const float *)sinogram, volume, views, step, spacing,
                                                               d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h, d.n_proj,
                                                               d.geom_batch);
        break;
    case PYRONN_BFLOAT16:
        cone_scatter_kernel<__nv_bfloat16><<<grid, block, 0, stream>>>((const __nv_bfloat16 *)sinogram, volume, views,
                                                                       step, spacing, d.vol_x, d.vol_y, d.vol_z,
                                                                       d.det_w, d.det_h, d.n_proj, d.geom_batch);
        break;
    case PYRONN_FLOAT16:
        cone_scatter_kernel<__half><<<grid, block, 0, stream>>>((const __half *)sinogram, volume, views, step, spacing,
                                                                d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h, d.n_proj,
                                                                d.geom_batch);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace pyronn

// cone_fp_padded.cu -- software-interpolation cone forward projector over
// zero-padded, view-oriented copies of the volume.
//
// The reference gathers the 8 trilinear taps straight from the x-fastest
// volume with a bounds test per tap (cone_projector_3D_CudaKernel.cu.cc:42-85).
// A warp here is 32 rays of one detector row; at a given step their samples
// lie on a line perpendicular to the rays.  When the rays run mostly along x
// that line runs along y, so in an x-fastest layout every lane hits its own
// cache line.  The call therefore stages two copies of the volume in the
// workspace, both with a zero border (1 voxel below, 2 above, so the taps of
// any sample inside the box [0, N] need no bounds test):
//   * x-fastest [Z+3][Y+3][X+3]  -- used by views whose rays run mostly along y
//   * y-fastest [Z+3][X+3][Y+3]  -- used by views whose rays run mostly along x
// Sample positions, weights and the march are those of cone_fp.cu (FP64 ray
// set-up, FP32 alpha advanced as the reference does), so results are the same.
#include <math_constants.h>

#include "common.cuh"
#include "cone_ray.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int PB_X = 32;
constexpr int PB_Y = 8;
constexpr int PAD_TILE = 32;

// copies one batch element into both padded layouts; the border is written as
// zeros by the same kernel (every padded element is written exactly once)
template <typename T>
__global__ void __launch_bounds__(PAD_TILE *8) pad_volume_kernel(const T *__restrict__ src, T *__restrict__ xfast,
                                                                 T *__restrict__ yfast, int X, int Y, int Z)
{
    __shared__ T tile[PAD_TILE][PAD_TILE + 1];
    const int Xp = X + 3, Yp = Y + 3;
    const int zp = blockIdx.z;   // padded z
    const int z = zp - 1;        // source z
    const int x0 = blockIdx.x * PAD_TILE - 1, y0 = blockIdx.y * PAD_TILE - 1;  // padded tile origin - 1
    const bool zin = z >= 0 && z < Z;
    // load a tile (source coordinates x0.., y0..) and write the x-fastest copy
    for (int r = threadIdx.y; r < PAD_TILE; r += 8) {
        const int y = y0 + r, x = x0 + threadIdx.x;
        T v = T(0.0f);
        if (zin && y >= 0 && y < Y && x >= 0 && x < X) v = src[((size_t)z * Y + y) * X + x];
        tile[r][threadIdx.x] = v;
        const int xp = x + 1, yp = y + 1;
        if (xp < Xp && yp < Yp) xfast[((size_t)zp * Yp + yp) * Xp + xp] = v;
    }
    __syncthreads();
    // transposed write of the y-fastest copy
    for (int r = threadIdx.y; r < PAD_TILE; r += 8) {
        const int xp = x0 + r + 1, yp = y0 + threadIdx.x + 1;
        if (xp < Xp && yp < Yp) yfast[((size_t)zp * Xp + xp) * Yp + yp] = tile[threadIdx.x][r];
    }
}

template <typename T>
__device__ __forceinline__ float interp3d_padded(const T *__restrict__ vol, float x, float y, float z, float xmax,
                                                 float ymax, float zmax, int sx, int sy, int sz)
{
    // clamping to [-1, N + 0.999] keeps every tap inside the padded copy and
    // changes no value: outside [-1, N + 1) all taps are border zeros anyway
    x = fminf(fmaxf(x, -1.0f), xmax);
    y = fminf(fmaxf(y, -1.0f), ymax);
    z = fminf(fmaxf(z, -1.0f), zmax);
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const float tx = x - fx, ty = y - fy, tz = z - fz;
    const int base = ((int)fx + 1) * sx + ((int)fy + 1) * sy + ((int)fz + 1) * sz;
    const T *p = vol + base;
    const float p000 = load_as_float(p);
    const float p001 = load_as_float(p + sx);
    const float p010 = load_as_float(p + sy);
    const float p011 = load_as_float(p + sy + sx);
    const float p100 = load_as_float(p + sz);
    const float p101 = load_as_float(p + sz + sx);
    const float p110 = load_as_float(p + sz + sy);
    const float p111 = load_as_float(p + sz + sy + sx);
    const float p00 = lerp_ref(p000, p100, tz);
    const float p01 = lerp_ref(p001, p101, tz);
    const float p10 = lerp_ref(p010, p110, tz);
    const float p11 = lerp_ref(p011, p111, tz);
    return lerp_ref(lerp_ref(p00, p10, ty), lerp_ref(p01, p11, ty), tx);
}

template <typename T, typename Tout>
__global__ void __launch_bounds__(PB_X *PB_Y)
    cone_fp_padded_kernel(const T *__restrict__ xfast, const T *__restrict__ yfast, Tout *__restrict__ sino,
                          const ConeFpView *__restrict__ views, const float *__restrict__ step_ptr,
                          const float *__restrict__ spacing_ptr, int X, int Y, int Z, int W, int H, int n_proj,
                          int geom_batch, int b)
{
    const int u = blockIdx.x * PB_X + threadIdx.x;
    const int v = blockIdx.y * PB_Y + threadIdx.y;
    const int p = blockIdx.z;
    if (u >= W || v >= H) return;
    const int g = geom_batch == 1 ? 0 : b;
    const ConeFpView &view = views[(size_t)g * n_proj + p];
    const float step = step_ptr[g];
    const ConeRay ray = cone_ray_setup(view, u, v, X, Y, Z, 0.0, step, spacing_ptr[g * 3 + 2], spacing_ptr[g * 3 + 1],
                                       spacing_ptr[g * 3 + 0]);
    // layout of this view: rays mostly along x -> y-fastest copy
    const double cr0 = view.inv_ar[2] + 0.5 * (W - 1) * view.inv_ar[0] + 0.5 * (H - 1) * view.inv_ar[1];
    const double cr1 = view.inv_ar[5] + 0.5 * (W - 1) * view.inv_ar[3] + 0.5 * (H - 1) * view.inv_ar[4];
    const bool along_x = fabs(cr0) > fabs(cr1);
    const int Xp = X + 3, Yp = Y + 3;
    const int sx = along_x ? Yp : 1, sy = along_x ? 1 : Xp, sz = Xp * Yp;
    const T *vol = along_x ? yfast : xfast;
    const float xmax = (float)X + 0.999f, ymax = (float)Y + 0.999f, zmax = (float)Z + 0.999f;
    auto sample = [&](float x, float y, float z) {
        return interp3d_padded<T>(vol, x, y, z, xmax, ymax, zmax, sx, sy, sz);
    };
    const float pixel = cone_ray_march<false>(ray, step, sample);
    store_from_float(sino + (((size_t)b * n_proj + p) * H + v) * (size_t)W + u, pixel);
}

template <typename Tin, typename Tout>
cudaError_t launch_typed(const void *volume, void *sinogram, const Dims3D &d, const ConeFpView *views,
                         const float *step, const float *spacing, void *scratch, cudaStream_t stream)
{
    const size_t padded = (size_t)(d.vol_x + 3) * (d.vol_y + 3) * (d.vol_z + 3);
    Tin *xfast = (Tin *)scratch;
    Tin *yfast = xfast + padded;
    const dim3 pblock(PAD_TILE, 8);
    const dim3 pgrid((d.vol_x + 3 + PAD_TILE - 1) / PAD_TILE, (d.vol_y + 3 + PAD_TILE - 1) / PAD_TILE, d.vol_z + 3);
    const dim3 block(PB_X, PB_Y);
    const dim3 grid((d.det_w + PB_X - 1) / PB_X, (d.det_h + PB_Y - 1) / PB_Y, d.n_proj);
    for (int b = 0; b < d.batch; ++b) {
        const Tin *src = (const Tin *)volume + (size_t)b * d.vol_z * d.vol_y * d.vol_x;
        pad_volume_kernel<Tin><<<pgrid, pblock, 0, stream>>>(src, xfast, yfast, d.vol_x, d.vol_y, d.vol_z);
        cone_fp_padded_kernel<Tin, Tout><<<grid, block, 0, stream>>>(xfast, yfast, (Tout *)sinogram, views, step,
                                                                     spacing, d.vol_x, d.vol_y, d.vol_z, d.det_w,
                                                                     d.det_h, d.n_proj, d.geom_batch, b);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

size_t cone_fp_padded_scratch_bytes(int vol_z, int vol_y, int vol_x, int in_dtype)
{
    return 2 * (size_t)(vol_x + 3) * (vol_y + 3) * (vol_z + 3) * dtype_size(in_dtype);
}

bool cone_fp_padded_supported(const Dims3D &d)
{
    const long long padded = (long long)(d.vol_x + 3) * (d.vol_y + 3) * (d.vol_z + 3);
    return padded < (1LL << 31) - (1LL << 20) && d.n_proj <= 65535 && d.vol_z + 3 <= 65535;
}

cudaError_t launch_cone_fp_padded(const void *volume, void *sinogram, int in_dtype, int out_dtype, const Dims3D &d,
                                  const ConeFpView *views, const float *step, const float *spacing, void *scratch,
                                  cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return launch_typed<Tin, Tout>(volume, sinogram, d, views, step, spacing, scratch, stream);
    });
}

}  // namespace pyronn

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

// Trilinear interpolation from a padded copy.  FASTY selects the y-fastest
// layout; the tap along the fastest axis is then the next element (an
// immediate offset), the others are a row / a slice away.  `origin` points at
// padded (1, 1, 1), i.e. source voxel (0, 0, 0); any sample whose floor lies
// in [-1, N] keeps all its taps inside the padded copy.
template <typename T, bool FASTY>
struct PaddedSampler {
    const T *origin;
    int s_row, s_slice;  // element strides of the slow in-slice axis and of z

    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        const FloorFrac fx = floor_frac(x), fy = floor_frac(y), fz = floor_frac(z);
        const int fast = FASTY ? fy.i : fx.i, slow = FASTY ? fx.i : fy.i;
        const T *p = origin + (fz.i * s_slice + slow * s_row + fast);
        const T *q = p + s_slice;
        const float p000 = load_as_float(p), p_f = load_as_float(p + 1);
        const float p0s = load_as_float(p + s_row), p_fs = load_as_float(p + s_row + 1);
        const float p100 = load_as_float(q), q_f = load_as_float(q + 1);
        const float q0s = load_as_float(q + s_row), q_fs = load_as_float(q + s_row + 1);
        // the reference's order: lerp in z, then y, then x
        const float c00 = lerp_ref(p000, p100, fz.f), c_f = lerp_ref(p_f, q_f, fz.f);
        const float c_s = lerp_ref(p0s, q0s, fz.f), c_fs = lerp_ref(p_fs, q_fs, fz.f);
        if (FASTY) {  // fast = y, slow = x
            const float x0 = lerp_ref(c00, c_f, fy.f), x1 = lerp_ref(c_s, c_fs, fy.f);
            return lerp_ref(x0, x1, fx.f);
        } else {      // fast = x, slow = y
            const float y0 = lerp_ref(c00, c_s, fy.f), y1 = lerp_ref(c_f, c_fs, fy.f);
            return lerp_ref(y0, y1, fx.f);
        }
    }
};

// Generic clamped sample for rays whose end points are not proven inside the
// padded range: clamping to [-1, N + 0.999] changes no value (outside
// [-1, N + 1) all taps are border zeros) and keeps every tap in the copy.
template <typename T, bool FASTY>
struct ClampedSampler {
    PaddedSampler<T, FASTY> s;
    float xmax, ymax, zmax;
    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        return s(fminf(fmaxf(x, -1.0f), xmax), fminf(fmaxf(y, -1.0f), ymax), fminf(fmaxf(z, -1.0f), zmax));
    }
};

// The reference's march (cone_ray.cuh) with the main loop taking two
// samples per iteration, so the gathers of both are in flight together; the
// alpha sequence and the order of the additions are unchanged.
template <typename F>
__device__ __forceinline__ float march_x2(const ConeRay &ray, float step, const F &sample)
{
    if (!ray.hit) return 0.0f;
    float a = ray.a;
    float px = fmaf(a, ray.dx, ray.ox), py = fmaf(a, ray.dy, ray.oy), pz = fmaf(a, ray.dz, ray.oz);
    float pixel = 0.5f * sample(px, py, pz);
    a += step;
    int iter = 1;
    while (a < ray.am && iter < ray.max_iter) {
        const float a1 = a + step;
        if (a1 < ray.am && iter + 1 < ray.max_iter) {
            const float qx = fmaf(a, ray.dx, ray.ox), qy = fmaf(a, ray.dy, ray.oy), qz = fmaf(a, ray.dz, ray.oz);
            px = fmaf(a1, ray.dx, ray.ox);
            py = fmaf(a1, ray.dy, ray.oy);
            pz = fmaf(a1, ray.dz, ray.oz);
            const float v0 = sample(qx, qy, qz), v1 = sample(px, py, pz);
            pixel += v0;
            pixel += v1;
            a = a1 + step;
            iter += 2;
        } else {
            px = fmaf(a, ray.dx, ray.ox);
            py = fmaf(a, ray.dy, ray.oy);
            pz = fmaf(a, ray.dz, ray.oz);
            pixel += sample(px, py, pz);
            a += step;
            ++iter;
        }
    }
    pixel *= step;
    if (pixel > 0.0f) {
        const float last_val = sample(px, py, pz);
        pixel -= 0.5f * step * last_val;
        a -= step;
        const float last_step = ray.am - a;
        pixel += 0.5f * last_step * last_val;
        px = fmaf(ray.am, ray.dx, ray.ox);
        py = fmaf(ray.am, ray.dy, ray.oy);
        pz = fmaf(ray.am, ray.dz, ray.oz);
        pixel += 0.5f * last_step * sample(px, py, pz);
    }
    return pixel * ray.mm_scale;
}

// true when every point of the FP32 march lies in [-0.5, N + 0.5]: its end
// points do (the segment between is convex) -- checked once per ray
__device__ __forceinline__ bool march_inside(const ConeRay &r, int X, int Y, int Z)
{
    if (!r.hit) return true;
    const float x0 = fmaf(r.a, r.dx, r.ox), y0 = fmaf(r.a, r.dy, r.oy), z0 = fmaf(r.a, r.dz, r.oz);
    const float x1 = fmaf(r.am, r.dx, r.ox), y1 = fmaf(r.am, r.dy, r.oy), z1 = fmaf(r.am, r.dz, r.oz);
    const float lo = -0.5f;
    return fminf(x0, x1) >= lo && fminf(y0, y1) >= lo && fminf(z0, z1) >= lo && fmaxf(x0, x1) <= X + 0.5f &&
           fmaxf(y0, y1) <= Y + 0.5f && fmaxf(z0, z1) <= Z + 0.5f;
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
    // layout of this view (uniform per block): rays mostly along x -> y-fastest copy
    const double cr0 = view.inv_ar[2] + 0.5 * (W - 1) * view.inv_ar[0] + 0.5 * (H - 1) * view.inv_ar[1];
    const double cr1 = view.inv_ar[5] + 0.5 * (W - 1) * view.inv_ar[3] + 0.5 * (H - 1) * view.inv_ar[4];
    const bool along_x = fabs(cr0) > fabs(cr1);
    const int Xp = X + 3, Yp = Y + 3;
    const int s_slice = Xp * Yp;
    const bool inside = march_inside(ray, X, Y, Z);
    const float xmax = (float)X + 0.999f, ymax = (float)Y + 0.999f, zmax = (float)Z + 0.999f;
    float pixel;
    if (along_x) {
        const PaddedSampler<T, true> s{yfast + s_slice + Yp + 1, Yp, s_slice};
        pixel = inside ? march_x2(ray, step, s) : march_x2(ray, step, ClampedSampler<T, true>{s, xmax, ymax, zmax});
    } else {
        const PaddedSampler<T, false> s{xfast + s_slice + Xp + 1, Xp, s_slice};
        pixel = inside ? march_x2(ray, step, s) : march_x2(ray, step, ClampedSampler<T, false>{s, xmax, ymax, zmax});
    }
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

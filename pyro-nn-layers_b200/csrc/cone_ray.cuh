// cone_ray.cuh -- per-ray set-up and the trapezoid march of the cone-beam
// forward projector, shared by the projector kernels and by the matched
// (exact-adjoint) scatter backprojector.
//
// Set-up (FP64): direction = normalize(inv_ar (u, v, 1)) in voxel-index space,
// box entry/exit with the reference's slab tests
// (cone_projector_3D_CudaKernel.cu.cc:96-132; box [lo, N + lo], lo = 0 for
// software and -0.5 for hardware interpolation).
// March (FP32): alpha starts half a step in and advances by `step` in a float
// (:135-159); the sum is the trapezoid rule with the last segment corrected
// to the exit point (:160-179).  The reference applies that correction only
// when the running sum is > 0; `Linear` = true applies it always, which makes
// the operator linear (it differs only for rays whose sum is <= 0).
#pragma once

#include <math_constants.h>

#include "internal.h"

namespace pyronn {

struct ConeRay {
    float dx, dy, dz;  // unit direction (voxel-index space)
    float ox, oy, oz;  // source (voxel-index space)
    float a, am;       // first sample parameter (entry + step/2) and exit
    int max_iter;      // bound on the samples (guards a stagnating float alpha)
    bool hit;          // the ray has at least one sample
    float mm_scale;    // |direction (.) spacing|: index length -> mm (:217-219)
};

// Whether detector pixel (u, v) lies in the view's footprint of the volume
// box: rays outside it miss the box, so their set-up (FP64) is skipped and
// their value is the miss's, 0.
__device__ __forceinline__ bool in_footprint(const ConeFpView &view, int u, int v)
{
    const float fu = (float)u, fv = (float)v;
    return fu >= view.foot[0] && fu <= view.foot[1] && fv >= view.foot[2] && fv <= view.foot[3];
}

__device__ __forceinline__ ConeRay cone_ray_setup(const ConeFpView &view, int u, int v, int X, int Y, int Z,
                                                  double lo, float step, float spx, float spy, float spz)
{
    double r[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        r[k] = view.inv_ar[3 * k + 2] + (double)v * view.inv_ar[3 * k + 1] + (double)u * view.inv_ar[3 * k + 0];
    const double inv_len = 1.0 / sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
#pragma unroll
    for (int k = 0; k < 3; ++k) r[k] *= inv_len;
    const double n_dim[3] = {(double)X, (double)Y, (double)Z};
    double amin = 0.0, amax = CUDART_INF;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (r[k] != 0.0) {
            const double rc = 1.0 / r[k];
            const double a0 = (lo - view.src[k]) * rc;
            const double a1 = (n_dim[k] + lo - view.src[k]) * rc;
            if (k == 0) {
                amin = fmin(a0, a1);
                amax = fmax(a0, a1);
            } else {
                amin = fmax(amin, fmin(a0, a1));
                amax = fmin(amax, fmax(a0, a1));
            }
        }
    }
    ConeRay ray;
    ray.dx = (float)r[0];
    ray.dy = (float)r[1];
    ray.dz = (float)r[2];
    ray.ox = (float)view.src[0];
    ray.oy = (float)view.src[1];
    ray.oz = (float)view.src[2];
    float a = (float)amin;
    a += step * 0.5f;
    ray.a = a;
    ray.am = (float)amax;
    ray.hit = step > 0.0f && step < CUDART_INF_F && amin < amax && a < ray.am;
    const double bound = ray.hit ? ((double)ray.am - (double)a) / (double)step + 4.0 : 0.0;
    ray.max_iter = bound > 1.0e8 ? 100000000 : (int)bound;
    ray.mm_scale = sqrtf((ray.dx * spx) * (ray.dx * spx) + (ray.dy * spy) * (ray.dy * spy) +
                         (ray.dz * spz) * (ray.dz * spz));
    return ray;
}

// Block order of the ray-driven forward kernels.  The grid is one
// dimension; each 32 x 32 tile of detector rays of a view is four blocks of
// 256 threads (sub = 0..3).  Views go in chunks of VIEW_CHUNK; inside a chunk
// the tiles follow one another (u fastest), each with the chunk's views
// consecutive.  Rays of neighbouring views through one detector tile cross
// nearly the same voxels, so blocks resident together share their taps in L2
// instead of every view streaming the whole volume from DRAM.
#ifndef PYRONN_FP_VIEW_CHUNK
#define PYRONN_FP_VIEW_CHUNK 32
#endif
constexpr int VIEW_CHUNK = PYRONN_FP_VIEW_CHUNK;

struct RayBlock {
    int p;               // view
    int tile_u, tile_v;  // 32 x 32 ray tile
    int sub;             // quarter of the tile
};

__device__ __forceinline__ RayBlock ray_block(unsigned block, int W, int H, int n_proj)
{
    RayBlock rb;
    rb.sub = (int)(block & 3u);
    const unsigned combo = block >> 2;  // (tile, view) index in the block order
    const unsigned tiles_u = (W + 31) / 32, tiles = tiles_u * ((H + 31) / 32);
    const unsigned chunk = combo / (VIEW_CHUNK * tiles), rem = combo - chunk * VIEW_CHUNK * tiles;
    const unsigned chunk_views = min((unsigned)VIEW_CHUNK, (unsigned)n_proj - chunk * VIEW_CHUNK);
    const unsigned tile = rem / chunk_views;
    rb.p = (int)(chunk * VIEW_CHUNK + (rem - tile * chunk_views));
    rb.tile_v = (int)(tile / tiles_u);
    rb.tile_u = (int)(tile - (unsigned)rb.tile_v * tiles_u);
    return rb;
}

inline unsigned ray_block_count(int W, int H, int n_proj)
{
    return (unsigned)((W + 31) / 32) * (unsigned)((H + 31) / 32) * (unsigned)n_proj * 4u;
}

inline bool ray_blocks_fit(int W, int H, int n_proj)
{
    return (long long)((W + 31) / 32) * ((H + 31) / 32) * n_proj * 4 < (1LL << 31);
}

// Z-mode test of a view: the ray direction's derivative along detector v,
// inv_ar (0, 1, 0) in voxel-index space, points along z.
__device__ __forceinline__ bool view_is_z_mode(const ConeFpView &v)
{
    const double cx = v.inv_ar[1], cy = v.inv_ar[4], cz = v.inv_ar[7];
    return cz * cz >= 0.81 * (cx * cx + cy * cy + cz * cz);
}

// The march of cone_ray_march<false> with the main loop taking two
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

// march_x2 for a ray whose alpha sequence is exact (exact_sample_count
// gave n): the same samples in the same order, counted instead of compared.
template <typename F>
__device__ __forceinline__ float march_counted_x2(const ConeRay &ray, int n, float step, const F &sample)
{
    float a = ray.a;
    float px = fmaf(a, ray.dx, ray.ox), py = fmaf(a, ray.dy, ray.oy), pz = fmaf(a, ray.dz, ray.oz);
    float pixel = 0.5f * sample(px, py, pz);
    a += step;
    int k = 1;
    for (; k + 1 < n; k += 2) {
        const float a1 = a + step;
        const float qx = fmaf(a, ray.dx, ray.ox), qy = fmaf(a, ray.dy, ray.oy), qz = fmaf(a, ray.dz, ray.oz);
        px = fmaf(a1, ray.dx, ray.ox);
        py = fmaf(a1, ray.dy, ray.oy);
        pz = fmaf(a1, ray.dz, ray.oz);
        const float v0 = sample(qx, qy, qz), v1 = sample(px, py, pz);
        pixel += v0;
        pixel += v1;
        a = a1 + step;
    }
    if (k < n) {
        px = fmaf(a, ray.dx, ray.ox);
        py = fmaf(a, ray.dy, ray.oy);
        pz = fmaf(a, ray.dz, ray.oz);
        pixel += sample(px, py, pz);
        a += step;
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

// march_counted_x2 with U samples per iteration (their U cell loads in
// flight together): the same samples, alpha sequence and order of additions.
// The last sample's value is kept for the end correction instead of being
// interpolated again (same position, same value).
template <int U, typename F>
__device__ __forceinline__ float march_counted(const ConeRay &ray, int n, float step, const F &sample)
{
    float a = ray.a;
    float last = sample(fmaf(a, ray.dx, ray.ox), fmaf(a, ray.dy, ray.oy), fmaf(a, ray.dz, ray.oz));
    float pixel = 0.5f * last;
    a += step;
    int k = 1;
    for (; k + U - 1 < n; k += U) {
        float v[U];
#pragma unroll
        for (int j = 0; j < U; ++j) {
            v[j] = sample(fmaf(a, ray.dx, ray.ox), fmaf(a, ray.dy, ray.oy), fmaf(a, ray.dz, ray.oz));
            a += step;
        }
#pragma unroll
        for (int j = 0; j < U; ++j) pixel += v[j];
        last = v[U - 1];
    }
    for (; k < n; ++k) {
        last = sample(fmaf(a, ray.dx, ray.ox), fmaf(a, ray.dy, ray.oy), fmaf(a, ray.dz, ray.oz));
        pixel += last;
        a += step;
    }
    pixel *= step;
    if (pixel > 0.0f) {
        pixel -= 0.5f * step * last;
        a -= step;
        const float last_step = ray.am - a;
        pixel += 0.5f * last_step * last;
        pixel += 0.5f * last_step *
                 sample(fmaf(ray.am, ray.dx, ray.ox), fmaf(ray.am, ray.dy, ray.oy), fmaf(ray.am, ray.dz, ray.oz));
    }
    return pixel * ray.mm_scale;
}

// Number of samples of the march when its float alpha sequence is exact:
// step a multiple of ulp(a0) and every alpha up to the one after the last
// sample below the next power of two above a0, so each a += step adds
// exactly and a_k = a0 + k * step.  Then the count is the number of k >= 0
// with a0 + k * step < am (capped at max_iter like the checked loop),
// computed here in FP64; -1 when the sequence may round.
__device__ __forceinline__ int exact_sample_count(const ConeRay &ray, float step)
{
    const int bits = __float_as_int(ray.a);
    const int e = (bits >> 23) & 0xff;
    if (!ray.hit || bits <= 0 || e == 0 || e == 0xff || !(step > 0.0f)) return -1;
    const double ulp = ldexp(1.0, e - 150);  // 2^(exponent - 23)
    const double q = (double)step / ulp;    // exact (power-of-two divisor)
    if (q != floor(q) || q > 16777216.0) return -1;
    const double a0 = ray.a, st = step, am = ray.am, top = ldexp(1.0, e - 126);
    double k = fmax(1.0, ceil((am - a0) / st));
    // a0 + k * st is exact in FP64 (k < 2^31, 24-bit step): settle the
    // rounding of the division
    if (k > 1.0 && a0 + (k - 1.0) * st >= am) k -= 1.0;
    if (a0 + k * st < am) k += 1.0;
    if (!(a0 + (k - 1.0) * st < am) || !(a0 + k * st >= am) || a0 + k * st >= top) return -1;
    return k > (double)ray.max_iter ? ray.max_iter : (int)k;
}

// sum of one ray; sample(x, y, z) returns the interpolated value at a point
template <bool Linear, typename F>
__device__ __forceinline__ float cone_ray_march(const ConeRay &ray, float step, const F &sample)
{
    if (!ray.hit) return 0.0f;
    float a = ray.a;
    float px = fmaf(a, ray.dx, ray.ox), py = fmaf(a, ray.dy, ray.oy), pz = fmaf(a, ray.dz, ray.oz);
    float pixel = 0.5f * sample(px, py, pz);
    a += step;
    int iter = 1;
    while (a < ray.am && iter < ray.max_iter) {
        px = fmaf(a, ray.dx, ray.ox);
        py = fmaf(a, ray.dy, ray.oy);
        pz = fmaf(a, ray.dz, ray.oz);
        pixel += sample(px, py, pz);
        a += step;
        ++iter;
    }
    pixel *= step;
    if (Linear || pixel > 0.0f) {
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

// Visits every sample point of the linear march with the weight the sample
// carries in the (scaled) line integral: visit(x, y, z, weight).  The sum of
// weight * value over the visits equals cone_ray_march<true>.
template <typename F>
__device__ __forceinline__ void cone_ray_weights(const ConeRay &ray, float step, const F &visit)
{
    if (!ray.hit) return;
    float a = ray.a;
    const float s = ray.mm_scale;
    // the final sample's weight is only known at the end: hold it back
    float px = fmaf(a, ray.dx, ray.ox), py = fmaf(a, ray.dy, ray.oy), pz = fmaf(a, ray.dz, ray.oz);
    float w_held = 0.5f * step;
    a += step;
    int iter = 1;
    while (a < ray.am && iter < ray.max_iter) {
        visit(px, py, pz, w_held * s);
        px = fmaf(a, ray.dx, ray.ox);
        py = fmaf(a, ray.dy, ray.oy);
        pz = fmaf(a, ray.dz, ray.oz);
        w_held = step;
        a += step;
        ++iter;
    }
    a -= step;
    const float last_step = ray.am - a;
    // last sample: its march weight, minus the half step the correction
    // removes, plus half the last segment
    visit(px, py, pz, (w_held - 0.5f * step + 0.5f * last_step) * s);
    visit(fmaf(ray.am, ray.dx, ray.ox), fmaf(ray.am, ray.dy, ray.oy), fmaf(ray.am, ray.dz, ray.oz),
          0.5f * last_step * s);
}

}  // namespace pyronn

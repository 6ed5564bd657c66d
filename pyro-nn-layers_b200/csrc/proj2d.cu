// proj2d.cu -- 2D parallel-beam and fan-beam projector / backprojector.
//
// Forward (ParallelProjection2D / FanProjection2D): one thread per detector
// pixel, blockIdx.y = view, blockIdx.z = batch element; the ray march follows
// kernel_project2D (par_projector_2D_CudaKernel.cu.cc:28-102): box edges
// index_to_physical(0|N) - 0.5 in mm, first sample at the entry with weight
// 1/2, alpha advanced in a float, step 0.2 * min(spacing) mm, end correction
// only when the sum is > 0, result scaled by |ray (.) spacing| (:141).
// The reference samples a border/linear texture at index + 0.5; here the
// same bilinear interpolation is done with exact FP32 weights.
// Given a workspace, the call first writes two copies of the batch as
// bilinear CELLS -- cell (x, y) holds the four taps V(x + {0,1}, y + {0,1}),
// with zeros outside the slice, for floors x, y in [-2, N] -- one x-fastest
// and one y-fastest.  (The box starts half a millimetre below pixel 0: at
// index -1 for 0.5 mm pixels, where rounding puts some rays' first sample a
// hair below -1; the second border cell keeps every ray of such a view, and
// so every lane of its warps, on the unclamped path.)  The cells hold FP32
// taps for every storage type, so a sample is one 16-byte load with no bounds
// tests and no widening.  A warp's 32 threads are 32 neighbouring detector pixels, so at each
// step their samples lie along the detector direction: views whose rays run
// mostly along y read the x-fastest cells, the others the y-fastest ones, so
// the warp's loads stay on few cache lines.  Without a workspace the taps are
// read from the caller's slice with a bounds test each.  Taps are combined in
// the same order on every path, so the choice does not change a result.
//
// Launches with few rays (batch x views x detector pixels up to
// SEG2D_MAX_RAYS) march each ray with SEG2D threads over contiguous ranges of
// its samples, the range starts found in closed form on the same float alpha
// sequence.
//
// Backward (ParallelBackprojection2D / FanBackprojection2D): one thread per
// pixel, loop over views, linear interpolation along the detector row;
// launches of few pixels split each pixel's views over BP2_VSPLIT threads.
#include <math_constants.h>
#include <type_traits>

#include "common.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr float PI_REF = 3.14159265359f;  // par_backprojector_2D_CudaKernel.cu.cc:32
constexpr int FP2_BLOCK = 128;
constexpr int BP2_BLOCK_X = 32;
constexpr int BP2_BLOCK_Y = 8;
constexpr int BP2_CHUNK = BP2_BLOCK_X * BP2_BLOCK_Y;  // views per shared-memory table
constexpr int BP2_VSPLIT = 4;                          // view groups of a small slice's backprojection
constexpr long long BP2_SPLIT_MAX_PIXELS = 131072;     // pixels per launch up to which view groups are used

template <typename T>
__device__ __forceinline__ float interp2d_border(const T *__restrict__ img, float x, float y, int X, int Y)
{
    // sample positions stay inside the box (|x|, |y| << 2^22): exact FADD floor
    const FloorFrac ffx = floor_frac(x), ffy = floor_frac(y);
    const int x0 = ffx.i, y0 = ffy.i;
    const float tx = ffx.f, ty = ffy.f;
    const bool vx0 = (unsigned)x0 < (unsigned)X, vx1 = (unsigned)(x0 + 1) < (unsigned)X;
    const bool vy0 = (unsigned)y0 < (unsigned)Y, vy1 = (unsigned)(y0 + 1) < (unsigned)Y;
    const int base = y0 * X + x0;
    const float p00 = (vy0 && vx0) ? load_as_float(img + base) : 0.0f;
    const float p01 = (vy0 && vx1) ? load_as_float(img + base + 1) : 0.0f;
    const float p10 = (vy1 && vx0) ? load_as_float(img + base + X) : 0.0f;
    const float p11 = (vy1 && vx1) ? load_as_float(img + base + X + 1) : 0.0f;
    const float p0 = lerp_ref(p00, p01, tx);
    const float p1 = lerp_ref(p10, p11, tx);
    return lerp_ref(p0, p1, ty);
}

template <typename T>
struct BorderSampler {
    const T *img;
    int X, Y;
    __device__ __forceinline__ float operator()(float x, float y) const { return interp2d_border<T>(img, x, y, X, Y); }
};

// The four taps of a bilinear cell in the order V(x0,y0), V(x1,y0),
// V(x0,y1), V(x1,y1), widened to FP32 whatever the storage type: the
// forward is bound by instruction issue, not by bytes (the slices' cells sit
// in L2), and FP32 taps need no widening per sample (measured on the 64 x 512^2
// fan batch: FP16 cells 43.7 ms, FP32 cells 42.3 ms per forward).  Widening is
// exact, so 16-bit storage gives the FP32 result of the rounded input.
struct Cell2 {
    // the two x lerps of a cell: along y0 and along y1
    __device__ static void xlerp(const float4 *c, float t, float &x0, float &x1)
    {
        const float4 w = __ldg(c);
        x0 = lerp_ref(w.x, w.y, t), x1 = lerp_ref(w.z, w.w, t);
    }
    __device__ static float4 make(float a, float b, float c, float d) { return make_float4(a, b, c, d); }
};

// Bilinear interpolation from a cell copy; `origin` is the cell of floor
// (0, 0), (s_x, s_y) the cell strides.  Floors must lie in [-2, N].
struct CellSampler2 {
    const float4 *origin;
    unsigned s_x, s_y;
    unsigned bias;  // -FLOOR_BIAS * (s_x + s_y), modulo 2^32: the floors' bias folded into one offset

    __device__ CellSampler2(const float4 *o, int sx, int sy)
        : origin(o), s_x((unsigned)sx), s_y((unsigned)sy), bias(0u - (unsigned)FLOOR_BIAS * ((unsigned)sx + (unsigned)sy))
    {
    }

    __device__ __forceinline__ float operator()(float x, float y) const
    {
        const FloorFrac fx = floor_frac(x), fy = floor_frac(y);
        const unsigned idx = (unsigned)fx.bits * s_x + (unsigned)fy.bits * s_y + bias;
        float x0, x1;
        Cell2::xlerp(origin + (int)idx, fx.f, x0, x1);
        return lerp_ref(x0, x1, fy.f);
    }
};

// For rays whose march leaves [-1.5, N + 0.5]: positions clamped into it,
// which changes no tap weight that is not zero either way.
struct ClampedCellSampler2 {
    CellSampler2 s;
    float xmax, ymax;
    __device__ __forceinline__ float operator()(float x, float y) const
    {
        return s(fminf(fmaxf(x, -1.5f), xmax), fminf(fmaxf(y, -1.5f), ymax));
    }
};

// The iteration bound of march2d's loops.
__device__ __forceinline__ int march2d_max_iter(float a, float am, float step)
{
    const double bound = ((double)am - (double)a) / (double)step + 4.0;
    return bound > 1.0e8 ? 100000000 : (int)bound;
}

// The ray march of kernel_project2D (par_projector_2D_CudaKernel.cu.cc:58-102)
// at positions (bx + a gx, by + a gy) in index space, eight (then four, two,
// one) samples per iteration (their gathers overlap) with the same alpha
// sequence and order of additions as one at a time.
template <typename F>
__device__ __forceinline__ float march2d(float a, float am, float step, float gx, float bx, float gy, float by,
                                         const F &sample)
{
    const int max_iter = march2d_max_iter(a, am, step);
    float pixel = 0.0f, px = 0.0f, py = 0.0f;
    int iter = 0;
    if (a < am) {
        px = fmaf(a, gx, bx);
        py = fmaf(a, gy, by);
        pixel += 0.5f * sample(px, py);
        a += step;
        ++iter;
    }
    // eight samples per compare while the eighth alpha is still before the exit
    while (iter + 7 < max_iter) {
        const float a1 = a + step, a2 = a1 + step, a3 = a2 + step, a4 = a3 + step, a5 = a4 + step, a6 = a5 + step,
                    a7 = a6 + step;
        if (!(a7 < am)) break;
        const float v0 = sample(fmaf(a, gx, bx), fmaf(a, gy, by));
        const float v1 = sample(fmaf(a1, gx, bx), fmaf(a1, gy, by));
        const float v2 = sample(fmaf(a2, gx, bx), fmaf(a2, gy, by));
        const float v3 = sample(fmaf(a3, gx, bx), fmaf(a3, gy, by));
        const float v4 = sample(fmaf(a4, gx, bx), fmaf(a4, gy, by));
        const float v5 = sample(fmaf(a5, gx, bx), fmaf(a5, gy, by));
        const float v6 = sample(fmaf(a6, gx, bx), fmaf(a6, gy, by));
        px = fmaf(a7, gx, bx);
        py = fmaf(a7, gy, by);
        const float v7 = sample(px, py);
        pixel += v0;
        pixel += v1;
        pixel += v2;
        pixel += v3;
        pixel += v4;
        pixel += v5;
        pixel += v6;
        pixel += v7;
        a = a7 + step;
        iter += 8;
    }
    // four samples per compare while the fourth alpha is still before the
    // exit (the sequence never decreases, so the first three are too)
    while (iter + 3 < max_iter) {
        const float a1 = a + step, a2 = a1 + step, a3 = a2 + step;
        if (!(a3 < am)) break;
        const float v0 = sample(fmaf(a, gx, bx), fmaf(a, gy, by));
        const float v1 = sample(fmaf(a1, gx, bx), fmaf(a1, gy, by));
        const float v2 = sample(fmaf(a2, gx, bx), fmaf(a2, gy, by));
        px = fmaf(a3, gx, bx);
        py = fmaf(a3, gy, by);
        const float v3 = sample(px, py);
        pixel += v0;
        pixel += v1;
        pixel += v2;
        pixel += v3;
        a = a3 + step;
        iter += 4;
    }
    while (a < am && iter < max_iter) {
        const float a1 = a + step;
        if (a1 < am && iter + 1 < max_iter) {
            const float qx = fmaf(a, gx, bx), qy = fmaf(a, gy, by);
            px = fmaf(a1, gx, bx);
            py = fmaf(a1, gy, by);
            const float v0 = sample(qx, qy);
            const float v1 = sample(px, py);
            pixel += v0;
            pixel += v1;
            a = a1 + step;
            iter += 2;
        } else {
            px = fmaf(a, gx, bx);
            py = fmaf(a, gy, by);
            pixel += sample(px, py);
            a += step;
            ++iter;
        }
    }
    pixel *= step;
    if (pixel > 0.0f) {  // :88-100
        const float last_val = sample(px, py);
        pixel -= 0.5f * step * last_val;
        a -= step;
        const float last_step = am - a;
        pixel += 0.5f * last_step * last_val;
        px = fmaf(am, gx, bx);
        py = fmaf(am, gy, by);
        pixel += 0.5f * last_step * sample(px, py);
    }
    return pixel;
}

// Ray segments.  A launch with few rays (one 256^2 slice scanned over 180
// views by 367 pixels has 66 k) fills a fraction of the GPU's warp slots
// while each thread marches ~1800 samples in sequence.  Its rays are marched
// by SEG2D threads each, over contiguous ranges of the ray's samples; the
// ranges start at alphas found in closed form (alpha_advance), so every
// sample sits where the one-thread march puts it, and the block adds the
// ranges' sums in order before the end correction (a different order of FP32
// additions than one thread's: the results differ in the last bits).  A full
// launch does better with one thread per ray (measured on 256 such slices per
// call: 14.1 ms per forward against 17.4 ms with segments), so segments are
// used up to SEG2D_MAX_RAYS rays per launch (batch x views x pixels).
constexpr int SEG2D = 4;
constexpr long long SEG2D_MAX_RAYS = 150000;

// The alpha sequence of march2d: a_{k+1} = fl(a_k + step).  Moves (a, k)
// forward while k < kmax and a < am, as the one-at-a-time loop does, in
// closed form over runs of equal increments, in integer arithmetic on the
// floats' significands: inside the binade [2^e, 2^(e+1)) of a, a = M u with
// u = 2^(e-23) and M in [2^23, 2^24), every exact sum a_k + step lies at the
// same offset from the grid of multiples of u, so each step adds D u with
// D = round(step / u); a result equal to 2^(e+1) (M = 2^24) is also right
// (the sum lies within u/2 of it on either side's grid), and the step past it
// is one float addition.  Returns false -- sequence not followed -- for a or
// step not positive normal, a step below u/2 (the loop stalls) or a sum
// halfway between two grid values (round-to-even then alternates).
__device__ bool alpha_advance(float &a, int &k, int kmax, float am, float step)
{
    const int sb = __float_as_int(step), se = (sb >> 23) & 0xff;
    if (sb <= 0 || se == 0 || se == 0xff) return false;
    const unsigned ms = (unsigned)(sb & 0x7fffff) | 0x800000u;
    const int amb = __float_as_int(am), ae = (amb >> 23) & 0xff;
    for (int guard = 0; guard < 512 && k < kmax && a < am; ++guard) {
        const int bits = __float_as_int(a), be = (bits >> 23) & 0xff;
        if (bits <= 0 || be == 0 || be == 0xff) return false;
        const unsigned M = (unsigned)(bits & 0x7fffff) | 0x800000u;
        // D = round(step / u), step / u = ms 2^(se - be)
        const int sh = be - se;
        unsigned D;
        if (sh <= 0) {
            D = -sh >= 8 ? 0x2000000u : ms << -sh;
        } else {
            if (sh >= 26) return false;
            const unsigned rem = ms & ((1u << sh) - 1u), half = 1u << (sh - 1);
            if (rem == half) return false;
            D = (ms >> sh) + (rem > half ? 1u : 0u);
            if (D == 0u) return false;
        }
        // results a + j D u, j = 1..m, stay on this grid (M + j D <= 2^24)
        unsigned m = D > 0x1000000u ? 0u : (0x1000000u - M) / D;
        if (m == 0u) {
            a = __fadd_rn(a, step);
            ++k;
            continue;
        }
        // and the loop stops after the step from the last alpha below am
        // (am > a, so its binade is e or above; two or more above, it is out of reach)
        if (ae - be <= 1) {
            const unsigned am_u = ((unsigned)(amb & 0x7fffff) | 0x800000u) << (ae - be);  // am / u, exact
            m = min(m, (am_u - M + D - 1u) / D);
        }
        m = min(m, (unsigned)(kmax - k));
        a = __int_as_float((be << 23) + (int)(M + m * D) - 0x800000);  // M + m D = 2^24 gives 2^(e+1)
        k += (int)m;
    }
    return k >= kmax || !(a < am);
}

// Samples k0 .. k1 - 1 of march2d's ray, a = a_{k0} on entry and a_{k1} on
// return (the same float additions); sample 0 weighs 1/2.  Returns their sum
// in order and the last one's value in `last`.
template <typename F>
__device__ __forceinline__ float march2d_range(float &a, int k0, int k1, float step, float gx, float bx, float gy,
                                               float by, const F &sample, float &last)
{
    float sum = 0.0f;
    int k = k0;
    if (k == 0 && k < k1) {
        last = sample(fmaf(a, gx, bx), fmaf(a, gy, by));
        sum += 0.5f * last;
        a += step;
        ++k;
    }
    for (; k + 8 <= k1; k += 8) {
        const float a1 = a + step, a2 = a1 + step, a3 = a2 + step, a4 = a3 + step, a5 = a4 + step, a6 = a5 + step,
                    a7 = a6 + step;
        const float v0 = sample(fmaf(a, gx, bx), fmaf(a, gy, by));
        const float v1 = sample(fmaf(a1, gx, bx), fmaf(a1, gy, by));
        const float v2 = sample(fmaf(a2, gx, bx), fmaf(a2, gy, by));
        const float v3 = sample(fmaf(a3, gx, bx), fmaf(a3, gy, by));
        const float v4 = sample(fmaf(a4, gx, bx), fmaf(a4, gy, by));
        const float v5 = sample(fmaf(a5, gx, bx), fmaf(a5, gy, by));
        const float v6 = sample(fmaf(a6, gx, bx), fmaf(a6, gy, by));
        const float v7 = sample(fmaf(a7, gx, bx), fmaf(a7, gy, by));
        sum += v0;
        sum += v1;
        sum += v2;
        sum += v3;
        sum += v4;
        sum += v5;
        sum += v6;
        sum += v7;
        last = v7;
        a = a7 + step;
    }
    for (; k < k1; ++k) {
        last = sample(fmaf(a, gx, bx), fmaf(a, gy, by));
        sum += last;
        a += step;
    }
    return sum;
}

// One ray: SEG = 1, march2d's pixel.  SEG > 1: the sum of range `seg` of
// the ray's samples (n samples, counted by alpha_advance); the range holding
// the last sample also returns that sample's value, the value at the exit and
// the end correction's last step (am - fl(a_n - step), as march2d forms it).
// A sequence alpha_advance cannot follow is marched whole by range 0 (`whole`).
template <int SEG, typename F>
__device__ __forceinline__ float march_ray(float a, float am, float step, float gx, float bx, float gy, float by,
                                           const F &sample, int seg, float &last, float &end_val, float &last_step,
                                           bool &holds_last, bool &whole)
{
    if (SEG == 1) return march2d(a, am, step, gx, bx, gy, by, sample);
    float an = a;
    int n = 0;
    if (!alpha_advance(an, n, march2d_max_iter(a, am, step), am, step)) {
        whole = true;
        return seg == 0 ? march2d(a, am, step, gx, bx, gy, by, sample) : 0.0f;
    }
    const int k0 = (int)((long long)seg * n / SEG), k1 = (int)((long long)(seg + 1) * n / SEG);
    int k = 0;
    alpha_advance(a, k, k0, am, step);  // every alpha before k0 <= n - 1 is below am
    const float sum = march2d_range(a, k0, k1, step, gx, bx, gy, by, sample, last);
    if (k1 == n && k1 > k0) {
        holds_last = true;
        last_step = am - (a - step);
        end_val = sample(fmaf(am, gx, bx), fmaf(am, gy, by));
    }
    return sum;
}

// SEG = 1: one thread per detector pixel.  SEG > 1: FP2_BLOCK / SEG pixels
// per block, warp w of the block marching range w of their rays.
template <typename T, typename Tout, bool FAN, int SEG>
// (12 blocks per SM: 40 registers hold the eight-sample loop; the kernel is
// bound by the cell loads' latency, so more resident warps pay.  SEG > 1
// keeps a range's bookkeeping across the loop: 10 blocks, 48 registers.)
__global__ void __launch_bounds__(FP2_BLOCK, SEG == 1 ? 12 : 10)
    projection2d_kernel(const T *__restrict__ vol, const float4 *__restrict__ cells_x,
                        const float4 *__restrict__ cells_y, Tout *__restrict__ sino, Geom2D geo,
                        int X, int Y, int W, int n_proj, int geom_batch)
{
    constexpr int RAYS = FP2_BLOCK / SEG;  // rays per block
    static_assert(SEG == 1 || RAYS == 32, "a segment per warp");
    const int lane = threadIdx.x % RAYS, seg = threadIdx.x / RAYS;
    const int u = blockIdx.x * RAYS + lane;
    const int p = blockIdx.y;
    const int b = blockIdx.z;
    if (SEG == 1 && u >= W) return;
    const bool live = u < W;
    const int g = geom_batch == 1 ? 0 : b;
    const float sx = geo.volume_spacing[2 * g + 1], sy = geo.volume_spacing[2 * g + 0];
    const float ox = geo.volume_origin[2 * g + 1], oy = geo.volume_origin[2 * g + 0];
    const float ds = geo.detector_spacing[g], dorg = geo.detector_origin[g];
    const float2 ray_in = reinterpret_cast<const float2 *>(geo.rays)[(size_t)g * n_proj + p];
    const float uu = __fmaf_rn((float)u, ds, dorg);  // index_to_physical, helper_grid.h

    double srcx, srcy, rx, ry;
    if (!FAN) {
        // par_projector_2D_CudaKernel.cu.cc:120-132.  The virtual source point
        // is formed in FP32 as the reference forms it (ray * (-sid) + u_vec *
        // u, the second product fused) before the FP64 box test: a ray that
        // grazes the box -- along an axis with a 1e-17 cross component, say
        // -- enters or misses on that rounding, as in the reference.
        const float fx = (float)X, fy = (float)Y;
        const float sid =
            __fmul_rn(sqrtf(__fadd_rn(__fmul_rn(__fmul_rn(__fmul_rn(fx, sx), fx), sx),
                                      __fmul_rn(__fmul_rn(__fmul_rn(fy, sy), fy), sy))),
                      1.2f);
        rx = ray_in.x;
        ry = ray_in.y;
        srcx = (double)__fmaf_rn(-ray_in.y, uu, __fmul_rn(ray_in.x, -sid));
        srcy = (double)__fmaf_rn(ray_in.x, uu, __fmul_rn(ray_in.y, -sid));
    } else {
        // fan_projector_2D_CudaKernel.cu.cc:122-133
        const double sid = geo.sid[g], sdd = geo.sdd[g];
        srcx = ray_in.x * -sid;
        srcy = ray_in.y * -sid;
        const double lx = ray_in.x * sdd + (double)(-ray_in.y) * uu;
        const double ly = ray_in.y * sdd + (double)ray_in.x * uu;
        const double inv = 1.0 / sqrt(lx * lx + ly * ly);
        rx = lx * inv;
        ry = ly * inv;
    }

    // box in mm (the reference's -0.5 is in mm, :38-39,50-51), FP64
    double amin = 0.0, amax = CUDART_INF;
    if (rx != 0.0) {
        const double e0 = (double)ox - 0.5, e1 = (double)X * sx + ox - 0.5;
        const double rc = 1.0 / rx;
        const double a0 = (e0 - srcx) * rc, a1 = (e1 - srcx) * rc;
        amin = fmin(a0, a1);
        amax = fmax(a0, a1);
    }
    if (ry != 0.0) {
        const double e0 = (double)oy - 0.5, e1 = (double)Y * sy + oy - 0.5;
        const double rc = 1.0 / ry;
        const double a0 = (e0 - srcy) * rc, a1 = (e1 - srcy) * rc;
        amin = fmax(amin, fmin(a0, a1));
        amax = fmin(amax, fmax(a0, a1));
    }

    const float step = 0.2f * fminf(sx, sy);
    const float dx = (float)rx, dy = (float)ry;
    float pixel = 0.0f;                 // SEG > 1: this range's sum (or the whole ray's pixel, `whole`)
    float last = 0.0f, end_val = 0.0f;  // SEG > 1, the range holding the last sample: its value and
    float last_step = 0.0f;             // the end correction's sample and step
    bool holds_last = false, whole = false;
    if (live && step > 0.0f && amin < amax) {
        // sample positions in index space: idx = (src + a r - o) / s
        const float isx = 1.0f / sx, isy = 1.0f / sy;
        const float bx = (float)((srcx - ox) / sx), by = (float)((srcy - oy) / sy);
        const float gx = dx * isx, gy = dy * isy;
        const float a = (float)amin, am = (float)amax;
        if (cells_x) {
            // block-uniform layout choice: y-fastest cells when the view's
            // rays run mostly along x (fan: the central ray)
            const bool fast_y = fabsf(ray_in.x) > fabsf(ray_in.y);
            const size_t slice = (size_t)(X + 3) * (Y + 3);
            const CellSampler2 cs = fast_y ? CellSampler2(cells_y + b * slice + 2 * (Y + 3) + 2, Y + 3, 1)
                                           : CellSampler2(cells_x + b * slice + 2 * (X + 3) + 2, 1, X + 3);
            // every position of the march lies between its two end points
            const float x0 = fmaf(a, gx, bx), y0 = fmaf(a, gy, by), x1 = fmaf(am, gx, bx), y1 = fmaf(am, gy, by);
            const float xmax = (float)X + 0.5f, ymax = (float)Y + 0.5f;
            const bool inside = fminf(x0, x1) >= -1.5f && fminf(y0, y1) >= -1.5f && fmaxf(x0, x1) <= xmax &&
                                fmaxf(y0, y1) <= ymax;
            if (inside)
                pixel = march_ray<SEG>(a, am, step, gx, bx, gy, by, cs, seg, last, end_val, last_step, holds_last,
                                       whole);
            else
                pixel = march_ray<SEG>(a, am, step, gx, bx, gy, by, ClampedCellSampler2{cs, xmax, ymax}, seg, last,
                                       end_val, last_step, holds_last, whole);
        } else {
            pixel = march_ray<SEG>(a, am, step, gx, bx, gy, by, BorderSampler<T>{vol + (size_t)b * X * Y, X, Y},
                                   seg, last, end_val, last_step, holds_last, whole);
        }
    }
    if (SEG > 1) {
        // range sums in order, then march2d's scaling and end correction
        __shared__ float s_sum[SEG][RAYS];
        __shared__ float s_last[RAYS], s_end[RAYS], s_step[RAYS];
        __shared__ int s_whole[RAYS];
        s_sum[seg][lane] = pixel;
        if (holds_last) s_last[lane] = last, s_end[lane] = end_val, s_step[lane] = last_step;
        if (seg == 0) s_whole[lane] = whole;
        __syncthreads();
        if (seg != 0 || !live) return;
        if (!s_whole[lane]) {
            pixel = s_sum[0][lane];
#pragma unroll
            for (int r = 1; r < SEG; ++r) pixel += s_sum[r][lane];
            pixel *= step;
            if (pixel > 0.0f) {  // a sample exists: some range held the last one
                pixel -= 0.5f * step * s_last[lane];
                pixel += 0.5f * s_step[lane] * s_last[lane];
                pixel += 0.5f * s_step[lane] * s_end[lane];
            }
        }
    }
    pixel *= sqrtf((dx * sx) * (dx * sx) + (dy * sy) * (dy * sy));  // :141
    store_from_float(sino + ((size_t)b * n_proj + p) * W + u, pixel);
}

// Linear interpolation of a sinogram row at floor x0 with weight t, taps
// outside [0, W) zero: the reference's form for FP32; for 16-bit storage
// a + t (b - a) with b - a one mixed-precision subtraction (lerp_first's bits).
template <typename T>
struct RowTaps {
    __device__ static __forceinline__ float lerp(const T *row, int x0, int W, float t)
    {
        const unsigned short r0 = (unsigned)x0 < (unsigned)W ? __ldg(reinterpret_cast<const unsigned short *>(row + x0)) : 0;
        const unsigned short r1 =
            (unsigned)(x0 + 1) < (unsigned)W ? __ldg(reinterpret_cast<const unsigned short *>(row + x0 + 1)) : 0;
        if (std::is_same<T, __half>::value) {
            const float a = __half2float(__ushort_as_half(r0));
            return fmaf(t, sub_f32_f16<false>(r1, a), a);
        } else {
            const float a = __uint_as_float((unsigned)r0 << 16);
            return fmaf(t, sub_f32_bf16<false>(r1, a), a);
        }
    }
};
template <>
struct RowTaps<float> {
    __device__ static __forceinline__ float lerp(const float *row, int x0, int W, float t)
    {
        const float p0 = (unsigned)x0 < (unsigned)W ? __ldg(row + x0) : 0.0f;
        const float p1 = (unsigned)(x0 + 1) < (unsigned)W ? __ldg(row + x0 + 1) : 0.0f;
        return lerp_ref(p0, p1, t);
    }
};

// Detector index of pixel c for one fan view by the reference's own FP32
// steps: source r * (-SID), central point source + r * SDD, intersectLines2D
// (pixel, source, centre, centre + (-r.y, r.x)) and physical_to_index
// (fan_backprojector_2D_CudaKernel.cu.cc:47-59, helper_geometry_gpu.h:28-44),
// each operation rounded once.  Used for pixels near the source's depth,
// where the lines are nearly parallel and the reference's FP32 intersection
// differs from the exact one: its denominator below 1e-6 gives NaN, which the
// texture unit samples as coordinate 0 (measured on B200: half of the view's
// first texel, i.e. index -0.5); just above it, a far-off point.
__device__ __forceinline__ float fan_index_reference_steps(float cx, float cy, float rx, float ry, float sid, float sdd,
                                                        float dorg, float ds)
{
    const float srcx = __fmul_rn(rx, -sid), srcy = __fmul_rn(ry, -sid);
    const float cpx = __fadd_rn(srcx, __fmul_rn(rx, sdd)), cpy = __fadd_rn(srcy, __fmul_rn(ry, sdd));
    const float detx = -ry, dety = rx;
    const float p4x = __fadd_rn(cpx, detx), p4y = __fadd_rn(cpy, dety);
    const float a1 = __fsub_rn(cx, srcx), b1 = __fsub_rn(cpy, p4y);
    const float a2 = __fsub_rn(cy, srcy), b2 = __fsub_rn(cpx, p4x);
    const float dn = __fsub_rn(__fmul_rn(a1, b1), __fmul_rn(a2, b2));
    if (dn < 1.0e-6f && dn > -1.0e-6f) return -0.5f;
    const float x12 = __fsub_rn(__fmul_rn(cx, srcy), __fmul_rn(cy, srcx));
    const float x34 = __fsub_rn(__fmul_rn(cpx, p4y), __fmul_rn(cpy, p4x));
    const float x = __fdiv_rn(__fsub_rn(__fmul_rn(x12, b2), __fmul_rn(a1, x34)), dn);
    const float y = __fdiv_rn(__fsub_rn(__fmul_rn(x12, b1), __fmul_rn(a2, x34)), dn);
    const float s = __fadd_rn(__fmul_rn(x, detx), __fmul_rn(y, dety));
    return __fdiv_rn(__fsub_rn(s, dorg), ds);
}

// One thread per pixel, views in chunks of BP2_CHUNK whose per-view
// constants the block first puts in shared memory (one view per thread):
// parallel beam (-r.y, r.x) / detector spacing, fan beam (r.x, r.y, SID |r|^2,
// SDD |r|^2 / detector spacing), so a view costs each pixel one broadcast load.
// Fan beam: a geometry in which some view's source depth line comes within
// 2e-2 mm of the slice (the source inside or at the field) needs the
// reference's FP32 steps near that line (fan_index_reference_steps), which
// would cost the common case registers and occupancy; two instantiations are
// launched instead, NEAR_DEPTH = false and true, and each block checks the
// geometry first and leaves the work to the instantiation that matches it.
// VSPLIT > 1 (launches of few pixels, which leave most warp slots idle): the
// block's 8 thread rows are VSPLIT groups of 8 / VSPLIT pixel rows, group v
// summing part v of every chunk's views; the groups' sums are added in
// order at the end (the results differ from one thread's in the last bits).
template <typename T, typename Tout, bool FAN, bool NEAR_DEPTH, int VSPLIT>
__global__ void __launch_bounds__(BP2_BLOCK_X *BP2_BLOCK_Y)
    backprojection2d_kernel(const T *__restrict__ sino, Tout *__restrict__ vol, Geom2D geo, int X, int Y, int W,
                            int n_proj, int geom_batch)
{
    constexpr int ROWS = BP2_BLOCK_Y / VSPLIT;  // pixel rows per block
    __shared__ float4 tab[BP2_CHUNK];
    const int vg = threadIdx.y / ROWS;          // view group
    const int i = blockIdx.x * BP2_BLOCK_X + threadIdx.x;
    const int j = blockIdx.y * ROWS + threadIdx.y % ROWS;
    const int tid = threadIdx.y * BP2_BLOCK_X + threadIdx.x;
    const int b = blockIdx.z;
    const bool live = i < X && j < Y;
    const int g = geom_batch == 1 ? 0 : b;
    const float sx = geo.volume_spacing[2 * g + 1], sy = geo.volume_spacing[2 * g + 0];
    const float ox = geo.volume_origin[2 * g + 1], oy = geo.volume_origin[2 * g + 0];
    const float2 *rays = reinterpret_cast<const float2 *>(geo.rays) + (size_t)g * n_proj;
    float sid = 0.0f, sdd = 0.0f;
    if (FAN) {
        sid = geo.sid[g];
        sdd = geo.sdd[g];
        // a view's depth <c - src, r> is affine in the pixel centre c, so its
        // extremes over the slice are at the corners of the pixel-centre box
        const float x0 = ox, x1 = ox + (float)(X - 1) * sx, y0 = oy, y1 = oy + (float)(Y - 1) * sy;
        bool near = false;
        for (int n = tid; n < n_proj; n += BP2_BLOCK_X * BP2_BLOCK_Y) {
            const float2 r = __ldg(&rays[n]);
            const float base = sid * (r.x * r.x + r.y * r.y);
            const float d0 = fmaf(x0, r.x, fmaf(y0, r.y, base)), d1 = fmaf(x1, r.x, fmaf(y0, r.y, base));
            const float d2 = fmaf(x0, r.x, fmaf(y1, r.y, base)), d3 = fmaf(x1, r.x, fmaf(y1, r.y, base));
            near |= fminf(fminf(d0, d1), fminf(d2, d3)) < 2.0e-2f && fmaxf(fmaxf(d0, d1), fmaxf(d2, d3)) > -2.0e-2f;
        }
        if (__syncthreads_or(near) != NEAR_DEPTH) return;  // the other instantiation's block
    }
    const float ds = geo.detector_spacing[g], dorg = geo.detector_origin[g];
    const float ids = 1.0f / ds;
    const float sdo = dorg * ids;  // detector origin in pixels
    const float cx = (float)i * sx + ox, cy = (float)j * sy + oy;
    const T *sino_b = sino + (size_t)b * n_proj * W;
    float acc = 0.0f;
    for (int n0 = 0; n0 < n_proj; n0 += BP2_CHUNK) {
        const int cnt = min(BP2_CHUNK, n_proj - n0);
        __syncthreads();  // the previous chunk's constants are no longer read
        if (tid < cnt) {
            const float2 r = __ldg(&rays[n0 + tid]);
            if (FAN) {
                const float rr = r.x * r.x + r.y * r.y;
                tab[tid] = make_float4(r.x, r.y, sid * rr, sdd * rr * ids);
            } else {
                // detector direction (-r.y, r.x), par_backprojector_2D_CudaKernel.cu.cc:48-49
                tab[tid] = make_float4(-r.y * ids, r.x * ids, 0.0f, 0.0f);
            }
        }
        __syncthreads();
        if (!live) continue;
        const int kb = VSPLIT == 1 ? 0 : vg * cnt / VSPLIT, ke = VSPLIT == 1 ? cnt : (vg + 1) * cnt / VSPLIT;
        const T *row = sino_b + (size_t)(n0 + kb) * W;
#pragma unroll(NEAR_DEPTH ? 1 : 4)
        for (int k = kb; k < ke; ++k, row += W) {
            const float4 q = tab[k];
            float sidx, w = 1.0f;
            if (!FAN) {
                sidx = fmaf(cx, q.x, fmaf(cy, q.y, -sdo));  // (<c, d> - origin) / spacing, :51
            } else {
                // intersectLines2D(pixel, source, centre, centre + det) of
                // fan_backprojector_2D_CudaKernel.cu.cc:52-57 in closed form:
                // s = SDD |r|^2 <c, d> / (<c, r> + SID |r|^2), weight 1 / |c - src|^2
                const float cd = fmaf(cy, q.x, -cx * q.y);
                const float cr = fmaf(cx, q.x, cy * q.y);
                const float den = cr + q.z;  // <c - src, r>: the pixel's depth from the source
                sidx = fmaf(q.w * cd, fast_rcp(den), -sdo);
                // within 1e-2 mm of the source's depth, the reference's FP32 steps decide
                if (NEAR_DEPTH && fabsf(den) < 1.0e-2f)
                    sidx = fan_index_reference_steps(cx, cy, q.x, q.y, sid, sdd, dorg, ds);
                const float ex = fmaf(q.x, sid, cx), ey = fmaf(q.y, sid, cy);
                w = fast_rcp(fmaf(ex, ex, ey * ey));
            }
            // detector positions of pixels inside the field stay far below 2^22;
            // a pixel whose position is larger misses the row either way
            const float sc = fminf(fmaxf(sidx, -4.0f), (float)W + 4.0f);
            const FloorFrac ff = floor_frac(sc);
            acc = fmaf(RowTaps<T>::lerp(row, ff.i, W, ff.f), w, acc);
        }
    }
    if (VSPLIT > 1) {
        __shared__ float s_acc[VSPLIT][ROWS][BP2_BLOCK_X];
        s_acc[vg][threadIdx.y % ROWS][threadIdx.x] = acc;
        __syncthreads();
        if (vg != 0) return;
#pragma unroll
        for (int r = 1; r < VSPLIT; ++r) acc += s_acc[r][threadIdx.y][threadIdx.x];
    }
    if (!live) return;
    float out;
    if (!FAN)
        out = PI_REF * acc / (float)n_proj;  // :58
    else
        out = sid * sdd * PI_REF * acc / (float)n_proj;  // fan_backprojector_2D_CudaKernel.cu.cc:64
    store_from_float(vol + ((size_t)b * Y + j) * X + i, out);
}

// Both cell copies of the batch: cell (xc, yc), xc in [0, X+2], yc in
// [0, Y+2], has its low corner at pixel (xc-2, yc-2).  A block loads a 33 x 33
// tile along x and writes 32 x 32 cells x-fastest (along x) and y-fastest
// (along y); grid (ceil((X+3)/32), ceil((Y+3)/32), batch), block 32 x 8.
template <typename T>
__global__ void __launch_bounds__(256) pad_cells2d_kernel(const T *__restrict__ in,
                                                          float4 *__restrict__ cells_x,
                                                          float4 *__restrict__ cells_y, int X, int Y)
{
    __shared__ float tile[33][34];  // [y - (yc0-2)][x - (xc0-2)], widened
    const int Xc = X + 3, Yc = Y + 3;
    const int xc0 = blockIdx.x * 32, yc0 = blockIdx.y * 32;
    const T *img = in + (size_t)blockIdx.z * X * Y;
    for (int r = threadIdx.y; r < 33; r += 8) {
        const int y = yc0 - 2 + r;
        for (int c = threadIdx.x; c < 33; c += 32) {
            const int x = xc0 - 2 + c;
            float v = 0.0f;
            if (y >= 0 && y < Y && x >= 0 && x < X) v = load_as_float(img + (size_t)y * X + x);
            tile[r][c] = v;
        }
    }
    __syncthreads();
    const size_t slice = (size_t)blockIdx.z * Xc * Yc;
    for (int r = threadIdx.y; r < 32; r += 8) {
        {  // x-fastest: thread x along xc
            const int xc = xc0 + threadIdx.x, yc = yc0 + r;
            if (xc < Xc && yc < Yc)
                cells_x[slice + (size_t)yc * Xc + xc] = Cell2::make(
                    tile[r][threadIdx.x], tile[r][threadIdx.x + 1], tile[r + 1][threadIdx.x], tile[r + 1][threadIdx.x + 1]);
        }
        {  // y-fastest: thread x along yc
            const int yc = yc0 + threadIdx.x, xc = xc0 + r;
            if (xc < Xc && yc < Yc)
                cells_y[slice + (size_t)xc * Yc + yc] = Cell2::make(
                    tile[threadIdx.x][r], tile[threadIdx.x][r + 1], tile[threadIdx.x + 1][r], tile[threadIdx.x + 1][r + 1]);
        }
    }
}

template <typename Tin, typename Tout>
cudaError_t fp_typed(const void *volume, void *sinogram, bool fan, const Dims2D &d, const Geom2D &g,
                     void *workspace, cudaStream_t stream)
{
    using C = float4;
    C *cells_x = nullptr, *cells_y = nullptr;
    if (workspace) {
        const size_t n = (size_t)d.batch * (d.vol_x + 3) * (d.vol_y + 3);
        cells_x = (C *)workspace;
        cells_y = (C *)((char *)workspace + (n * sizeof(C) + 255) / 256 * 256);
        const dim3 tgrid((d.vol_x + 3 + 31) / 32, (d.vol_y + 3 + 31) / 32, d.batch);
        pad_cells2d_kernel<Tin><<<tgrid, dim3(32, 8), 0, stream>>>((const Tin *)volume, cells_x, cells_y, d.vol_x,
                                                                  d.vol_y);
    }
    // segments per ray for launches of few rays (see SEG2D)
    const bool segs = (long long)d.batch * d.n_proj * d.det_w <= SEG2D_MAX_RAYS;
    const int rays = segs ? FP2_BLOCK / SEG2D : FP2_BLOCK;
    const dim3 grid((d.det_w + rays - 1) / rays, d.n_proj, d.batch);
    auto launch = [&](auto kernel) {
        kernel<<<grid, FP2_BLOCK, 0, stream>>>((const Tin *)volume, cells_x, cells_y, (Tout *)sinogram, g, d.vol_x,
                                               d.vol_y, d.det_w, d.n_proj, d.geom_batch);
    };
    if (fan)
        segs ? launch(projection2d_kernel<Tin, Tout, true, SEG2D>) : launch(projection2d_kernel<Tin, Tout, true, 1>);
    else
        segs ? launch(projection2d_kernel<Tin, Tout, false, SEG2D>)
             : launch(projection2d_kernel<Tin, Tout, false, 1>);
    return cudaGetLastError();
}

template <typename Tin, typename Tout>
cudaError_t bp_typed(const void *sinogram, void *volume, bool fan, const Dims2D &d, const Geom2D &g,
                     cudaStream_t stream)
{
    const dim3 block(BP2_BLOCK_X, BP2_BLOCK_Y);
    // view groups for launches of few pixels (see VSPLIT; a full launch does
    // better without: 256 slices of 256^2, 2.48 ms against 2.87 ms)
    const bool split = (long long)d.batch * d.vol_x * d.vol_y <= BP2_SPLIT_MAX_PIXELS;
    const int rows = split ? BP2_BLOCK_Y / BP2_VSPLIT : BP2_BLOCK_Y;
    const dim3 grid((d.vol_x + BP2_BLOCK_X - 1) / BP2_BLOCK_X, (d.vol_y + rows - 1) / rows, d.batch);
    auto launch = [&](auto kernel) {
        kernel<<<grid, block, 0, stream>>>((const Tin *)sinogram, (Tout *)volume, g, d.vol_x, d.vol_y, d.det_w,
                                           d.n_proj, d.geom_batch);
    };
    if (fan) {
        // every block runs in exactly one of the two (see the kernel)
        if (split) {
            launch(backprojection2d_kernel<Tin, Tout, true, false, BP2_VSPLIT>);
            launch(backprojection2d_kernel<Tin, Tout, true, true, BP2_VSPLIT>);
        } else {
            launch(backprojection2d_kernel<Tin, Tout, true, false, 1>);
            launch(backprojection2d_kernel<Tin, Tout, true, true, 1>);
        }
    } else {
        split ? launch(backprojection2d_kernel<Tin, Tout, false, false, BP2_VSPLIT>)
              : launch(backprojection2d_kernel<Tin, Tout, false, false, 1>);
    }
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_projection2d(const void *volume, void *sinogram, int in_dtype, int out_dtype, bool fan,
                                const Dims2D &d, const Geom2D &g, void *workspace, cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return fp_typed<Tin, Tout>(volume, sinogram, fan, d, g, workspace, stream);
    });
}

cudaError_t launch_backprojection2d(const void *sinogram, void *volume, int in_dtype, int out_dtype, bool fan,
                                    const Dims2D &d, const Geom2D &g, cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return bp_typed<Tin, Tout>(sinogram, volume, fan, d, g, stream);
    });
}

}  // namespace pyronn

// cone_fp_padded.cu -- software-interpolation cone forward projector over
// zero-padded, view-oriented copies of the volume.
//
// The reference gathers the 8 trilinear taps straight from the x-fastest
// volume with a bounds test per tap (cone_projector_3D_CudaKernel.cu.cc:42-85).
// What makes a gather cheap is that the 32 samples a warp takes at one step
// fall on few cache lines.  Rays of one detector COLUMN (fixed u, varying v)
// sample at nearly the same (x, y) and at consecutive z whenever the
// detector's v axis runs along z -- true for every view of a circular
// trajectory.  Such views ("z mode") lay warps along v and read a z-fastest
// copy of trilinear CELLS: the element of cell (x, y, z) holds all eight taps
// V(x + {0,1}, y + {0,1}, z + {0,1}), so a sample is ONE 16-byte load (two
// for FP32) whose warp-wide footprint is a few consecutive lines.
// Other views ("xy mode") lay warps along u and read an x-fastest or a
// y-fastest copy, whichever fastest axis runs across their rays.
// All copies carry a zero border, so the taps of any sample inside the box
// [0, N] need no bounds test; they are
// written into the workspace per batch element, and a copy no view needs is
// skipped on the device.  Sample positions, weights and the march are those
// of cone_ray.cuh (FP64 ray set-up, FP32 alpha advanced as the reference
// does), so results match the direct path.
#include <math_constants.h>

#include <algorithm>
#include <type_traits>

#include "common.cuh"
#include "cone_ray.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int PB_X = 32;
constexpr int PB_Y = 8;
constexpr int PAD_TILE = 32;
constexpr size_t PAD_Z_BLOCKS = 16;  // z blocks of the xy-mode padded copy, each striding over planes
// workspace header words (after the error flag) set by classify_views_kernel
// (FLAG_WIDE, set by detect_wide_kernel: a 16-bit input holds magnitudes
// whose differences may not fit the storage type, so the cells keep their
// plain form and the rays take the FP32 y and x lerps)
enum { FLAG_NEED_XY = 1, FLAG_NEED_Z = 2, FLAG_WIDE = 3 };

__global__ void classify_views_kernel(const ConeFpView *__restrict__ views, int n, unsigned *__restrict__ flags)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    atomicOr(&flags[view_is_z_mode(views[t]) ? FLAG_NEED_Z : FLAG_NEED_XY], 1u);
}

// The eight taps of a trilinear cell, as (x0, x1) pairs in the order
// (y0 z0), (y0 z1), (y1 z0), (y1 z1): two float4 for FP32, four 32-bit words
// of two 16-bit values for BF16 / FP16 (x0 in the low half).  The 16-bit
// cells hold the z0 taps and, in place of the z1 taps, the half-differences
// (z1 - z0) / 2 rounded to the storage type (the halving keeps every FP16
// difference finite).  Their z lerp z0 + (2t) ((z1 - z0) / 2) takes 16-bit
// operands only: as one mixed-precision FMA and one mixed-precision addition
// of the z0 tap (sm_100 fma.f32.f16 / add.f32.f16, bf16 alike), or, in the
// packed form used unless the input's range forbids it, as a packed FMA on
// the (x0, x1) pair, followed by the pair's y lerp in packed form and the x
// lerp in FP32 (trilinear_packed); the packed form's cells hold their y1
// words as differences from the y0 words (make_ydiff), so the y difference
// of the pair is one FMA.  Roundings to the storage type happen only where
// neighbouring taps differ: the 512^3 forward's error against the FP64
// oracle stays the storage rounding's (FP16 2.65e-4), measured at 96.8 ms
// (widened taps, FP32 lerps) -> 90.0 ms (mixed z lerps) -> 83.0 ms (packed)
// -> 75.4 ms (other changes) -> 73.0 ms (y-difference cells).
struct alignas(16) CellF32 {
    float4 y0, y1;  // (x0 z0, x1 z0, x0 z1, x1 z1) at y0, then at y1
};

// z0 + t2 * hd for the z0 tap in word `a` and the half-difference in word
// `d` (the half selected by HI) and t2 = 2t in the storage type
template <bool BF16, bool HI>
__device__ __forceinline__ float lerp_half_diff(unsigned a, unsigned d, unsigned short t2)
{
    float p, z;
    if (BF16) {
        if (HI) {
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %2; fma.rn.f32.bf16 %0, %1, h, %3;}" : "=f"(p) : "h"(t2), "r"(d), "f"(0.0f));
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %1; add.rn.f32.bf16 %0, h, %2;}" : "=f"(z) : "r"(a), "f"(p));
        } else {
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %2; fma.rn.f32.bf16 %0, %1, l, %3;}" : "=f"(p) : "h"(t2), "r"(d), "f"(0.0f));
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %1; add.rn.f32.bf16 %0, l, %2;}" : "=f"(z) : "r"(a), "f"(p));
        }
    } else {
        if (HI) {
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %2; fma.rn.f32.f16 %0, %1, h, %3;}" : "=f"(p) : "h"(t2), "r"(d), "f"(0.0f));
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %1; add.rn.f32.f16 %0, h, %2;}" : "=f"(z) : "r"(a), "f"(p));
        } else {
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %2; fma.rn.f32.f16 %0, %1, l, %3;}" : "=f"(p) : "h"(t2), "r"(d), "f"(0.0f));
            asm("{.reg .b16 l, h; mov.b32 {l, h}, %1; add.rn.f32.f16 %0, l, %2;}" : "=f"(z) : "r"(a), "f"(p));
        }
    }
    return z;
}

template <typename T>
struct Cell;
template <>
struct Cell<float> {
    using type = CellF32;
    __device__ static void load(const CellF32 *c, float (&v)[8])
    {
        const float4 a = __ldg(&c->y0), b = __ldg(&c->y1);
        v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
    }
    // the four z lerps of a cell: z[0] = (x0 y0), z[1] = (x1 y0), z[2] = (x0 y1), z[3] = (x1 y1)
    __device__ static void zlerp(const CellF32 *c, float t, float (&z)[4])
    {
        float v[8];
        load(c, v);
        z[0] = lerp_ref(v[0], v[2], t), z[1] = lerp_ref(v[1], v[3], t);
        z[2] = lerp_ref(v[4], v[6], t), z[3] = lerp_ref(v[5], v[7], t);
    }
    __device__ static float trilinear(const CellF32 *c, float tz, float ty, float tx)
    {
        float zl[4];
        zlerp(c, tz, zl);
        return lerp_ref(lerp_ref(zl[0], zl[2], ty), lerp_ref(zl[1], zl[3], ty), tx);
    }
    __device__ static CellF32 make(const float (&v)[8])
    {
        CellF32 c;
        c.y0 = make_float4(v[0], v[1], v[2], v[3]);
        c.y1 = make_float4(v[4], v[5], v[6], v[7]);
        return c;
    }
};
// the 16-bit cells: words (z0 taps at y0, half-differences at y0, z0 taps
// at y1, half-differences at y1) -- or, for the packed lerps, the last two
// as their differences from the first two (make_ydiff)
template <typename T16>
struct Cell16 {
    static constexpr bool BF16 = std::is_same<T16, __nv_bfloat16>::value;
    using type = uint4;
    __device__ static void zlerp(const uint4 *c, float t, float (&z)[4])
    {
        const uint4 w = __ldg(c);
        unsigned short t2;
        if (BF16)
            asm("cvt.rn.bf16.f32 %0, %1;" : "=h"(t2) : "f"(t + t));
        else
            asm("cvt.rn.f16.f32 %0, %1;" : "=h"(t2) : "f"(t + t));
        z[0] = lerp_half_diff<BF16, false>(w.x, w.y, t2), z[1] = lerp_half_diff<BF16, true>(w.x, w.y, t2);
        z[2] = lerp_half_diff<BF16, false>(w.z, w.w, t2), z[3] = lerp_half_diff<BF16, true>(w.z, w.w, t2);
    }
    // FP32 y and x lerps of the four z lerps (inputs of any magnitude)
    __device__ static float trilinear(const uint4 *c, float tz, float ty, float tx)
    {
        float zl[4];
        zlerp(c, tz, zl);
        return lerp_ref(lerp_ref(zl[0], zl[2], ty), lerp_ref(zl[1], zl[3], ty), tx);
    }
    // Packed, on the y-difference cells (make_ydiff): the z lerp of the
    // (x0, x1) pair at y0 as one FMA on pairs of 16-bit values (z0 + (2t) hd,
    // one rounding), the pair's y difference -- z lerp at y1 minus z lerp at
    // y0 -- as one FMA on the cell's y-difference words (Dz0 + (2t) Dhd), the
    // y lerp as one FMA, the x lerp in FP32 on the pair widened (one widening,
    // one mixed-precision subtraction, one FMA): 7 instructions for the seven
    // lerps.  The differences must fit the storage type: used when every input
    // magnitude is below Wide16<T16>'s bound (FLAG_WIDE clear).
    // (tz2 = 2 tz, the z weight in half-voxel units).  Both weights are
    // rounded by one conversion into the two halves of a word and each packed
    // FMA takes its half replicated: 512^3 FP16 forward 77.3 -> 75.4 ms
    // against one conversion per weight (the same bits)
    __device__ static float trilinear_packed(const uint4 *c, float tz2f, float ty, float tx)
    {
        const uint4 w = __ldg(c);
        unsigned tz2, ty2, zy0, dy, yv;
        if (BF16) {
            asm("{.reg .b32 p; .reg .b16 l, h; cvt.rn.bf16x2.f32 p, %2, %3; mov.b32 {l, h}, p; mov.b32 %0, {l, l};"
                " mov.b32 %1, {h, h};}"
                : "=r"(tz2), "=r"(ty2) : "f"(ty), "f"(tz2f));
            asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(zy0) : "r"(tz2), "r"(w.y), "r"(w.x));
            asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(dy) : "r"(tz2), "r"(w.w), "r"(w.z));
            asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(yv) : "r"(ty2), "r"(dy), "r"(zy0));
            const float lo = __uint_as_float(yv << 16);
            return fmaf(tx, sub_f32_bf16<true>(yv, lo), lo);
        } else {
            asm("{.reg .b32 p; .reg .b16 l, h; cvt.rn.f16x2.f32 p, %2, %3; mov.b32 {l, h}, p; mov.b32 %0, {l, l};"
                " mov.b32 %1, {h, h};}"
                : "=r"(tz2), "=r"(ty2) : "f"(ty), "f"(tz2f));
            asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(zy0) : "r"(tz2), "r"(w.y), "r"(w.x));
            asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(dy) : "r"(tz2), "r"(w.w), "r"(w.z));
            asm("fma.rn.f16x2 %0, %1, %2, %3;" : "=r"(yv) : "r"(ty2), "r"(dy), "r"(zy0));
            const float lo = __half2float(__ushort_as_half((unsigned short)(yv & 0xFFFFu)));
            return fmaf(tx, sub_f32_f16<true>(yv, lo), lo);
        }
    }
    __device__ static unsigned short bits(__half v) { return __half_as_ushort(v); }
    __device__ static unsigned short bits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }
    __device__ static unsigned short half_diff(T16 z1, T16 z0)
    {
        // (z1 - z0) / 2: exact in FP32, one rounding to the storage type
        return bits(T16(0.5f * ((float)z1 - (float)z0)));
    }
    __device__ static uint4 make(const T16 (&v)[8])
    {
        const unsigned w0 = (unsigned)bits(v[0]) | ((unsigned)bits(v[1]) << 16);
        const unsigned w1 = (unsigned)half_diff(v[2], v[0]) | ((unsigned)half_diff(v[3], v[1]) << 16);
        const unsigned w2 = (unsigned)bits(v[4]) | ((unsigned)bits(v[5]) << 16);
        const unsigned w3 = (unsigned)half_diff(v[6], v[4]) | ((unsigned)half_diff(v[7], v[5]) << 16);
        return make_uint4(w0, w1, w2, w3);
    }
    __device__ static float value(unsigned short b)
    {
        if constexpr (BF16)
            return __bfloat162float(__ushort_as_bfloat16(b));
        else
            return __half2float(__ushort_as_half(b));
    }
    // b - a for each half of two words: exact in FP32, one rounding each
    __device__ static unsigned word_diff(unsigned b, unsigned a)
    {
        const unsigned short lo = bits(T16(value((unsigned short)b) - value((unsigned short)a)));
        const unsigned short hi = bits(T16(value((unsigned short)(b >> 16)) - value((unsigned short)(a >> 16))));
        return (unsigned)lo | ((unsigned)hi << 16);
    }
    // the packed lerps' cells: the y0 words of make, then the y1 words minus
    // the y0 words (z0 taps, half-differences), rounded to the storage type
    __device__ static uint4 make_ydiff(const T16 (&v)[8])
    {
        const uint4 c = make(v);
        return make_uint4(c.x, c.y, word_diff(c.z, c.x), word_diff(c.w, c.y));
    }
};
template <>
struct Cell<__nv_bfloat16> : Cell16<__nv_bfloat16> {
};
template <>
struct Cell<__half> : Cell16<__half> {
};
// Magnitudes above which the packed lerps' differences could leave the
// storage type's range.  FP16: below L = 32704 every stored difference is at
// most 2L and the y difference of two interpolated values, Dz0 + (2t) Dhd, at
// most 2L plus its roundings (under 2.5 ulp of 2L = 80): 65488, inside the
// largest finite value 65504.  FP32 input never takes the packed lerps.
template <typename T>
struct Wide16 {
    __device__ static bool exceeds(T) { return false; }
};
template <>
struct Wide16<__half> {
    __device__ static bool exceeds(__half v) { return fabsf(__half2float(v)) > 32704.0f; }
};
template <>
struct Wide16<__nv_bfloat16> {
    __device__ static bool exceeds(__nv_bfloat16 v) { return fabsf(__bfloat162float(v)) > 8.5e37f; }
};

// z-fastest cell copy: element [xc][yc][zc], xc in [0, X+1] (pitch s_x >=
// (Y+2) (Z+2), from cell_x_pitch), yc in [0, Y+1], zc in [0, Z+1], holds the
// cell whose low corner is voxel (xc-1, yc-1, zc-1)
// (V zero outside the volume), i.e. the taps of every floor in [-1, N].
// A block reads a 33 (x) x 33 (z) x (CELL_PLANES + 1) (y) tile along x --
// each plane once for its CELL_PLANES cell planes -- and writes 32 (z) x 32
// (x) x CELL_PLANES cells along z (at 512^3 the copy took 1.07 ms with one
// plane per block, 0.88 ms with four; the whole forward op 80.39 / 80.14 /
// 80.10 ms with one / four / eight).  Skipped when no view is in z mode.
constexpr int CELL_PLANES = 8;

// Sets FLAG_WIDE when a 16-bit input holds a magnitude beyond Wide16's bound:
// the cell copy then keeps the plain cells (z0 taps at y1, not differences)
// and the rays take FP32 y and x lerps.  One read of the volume before the
// copy, whose cell form depends on it.
template <typename T>
__global__ void __launch_bounds__(256) detect_wide_kernel(const T *__restrict__ src, size_t n,
                                                          unsigned *__restrict__ flags)
{
    if (!flags[FLAG_NEED_Z]) return;
    bool wide = false;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        wide |= Wide16<T>::exceeds(src[i]);
    if (__syncthreads_or(wide) && threadIdx.x == 0) atomicOr(&flags[FLAG_WIDE], 1u);
}

template <typename T>
__global__ void __launch_bounds__(PAD_TILE *8) pad_cells_kernel(const T *__restrict__ src,
                                                                 typename Cell<T>::type *__restrict__ dst, int X,
                                                                 int Y, int Z, int s_x, unsigned *__restrict__ flags)
{
    if (!flags[FLAG_NEED_Z]) return;
    // [y - (yc0-1)][z - (zc0-1)][x - (xc0-1)]
    __shared__ T tile[CELL_PLANES + 1][PAD_TILE + 1][PAD_TILE + 2];
    // 16-bit inputs within range take the packed lerps' y-difference cells
    const bool ydiff = sizeof(T) == 2 && !flags[FLAG_WIDE];
    const int Yc = Y + 2, Zc = Z + 2;
    const int xc0 = blockIdx.x * PAD_TILE, yc0 = blockIdx.y * CELL_PLANES, zc0 = blockIdx.z * PAD_TILE;
    for (int rr = threadIdx.y; rr < (CELL_PLANES + 1) * (PAD_TILE + 1); rr += 8) {
        const int dy = rr / (PAD_TILE + 1), r = rr % (PAD_TILE + 1);
        const int y = yc0 - 1 + dy, z = zc0 - 1 + r;
        const bool yz_in = y >= 0 && y < Y && z >= 0 && z < Z;
        for (int c = threadIdx.x; c < PAD_TILE + 1; c += PAD_TILE) {
            const int x = xc0 - 1 + c;
            T v = T(0.0f);
            if (yz_in && x >= 0 && x < X) v = src[((size_t)z * Y + y) * X + x];
            tile[dy][r][c] = v;
        }
    }
    __syncthreads();
    const int tz = threadIdx.x, zc = zc0 + tz;
    if (zc >= Zc) return;
#pragma unroll
    for (int pl = 0; pl < CELL_PLANES; ++pl) {
        const int yc = yc0 + pl;
        if (yc >= Yc) break;
#pragma unroll
        for (int k = 0; k < PAD_TILE / 8; ++k) {
            const int c = threadIdx.y + 8 * k, xc = xc0 + c;
            if (xc < X + 2) {
                const T v[8] = {tile[pl][tz][c],     tile[pl][tz][c + 1],     tile[pl][tz + 1][c],
                                tile[pl][tz + 1][c + 1], tile[pl + 1][tz][c], tile[pl + 1][tz][c + 1],
                                tile[pl + 1][tz + 1][c], tile[pl + 1][tz + 1][c + 1]};
                typename Cell<T>::type cell;
                if constexpr (sizeof(T) == 2)
                    cell = ydiff ? Cell<T>::make_ydiff(v) : Cell<T>::make(v);
                else
                    cell = Cell<T>::make(v);
                dst[(size_t)xc * s_x + (size_t)yc * Zc + zc] = cell;
            }
        }
    }
}

// copies one batch element into both padded layouts; the border is written as
// zeros by the same kernel (every padded element is written exactly once)
template <typename T>
__global__ void __launch_bounds__(PAD_TILE *8) pad_volume_kernel(const T *__restrict__ src, T *__restrict__ xfast,
                                                                 T *__restrict__ yfast, int X, int Y, int Z,
                                                                 const unsigned *__restrict__ flags)
{
    if (!flags[FLAG_NEED_XY]) return;
    __shared__ T tile[PAD_TILE][PAD_TILE + 1];
    const int Xp = X + 3, Yp = Y + 3, Zp = Z + 3;
    const int x0 = blockIdx.x * PAD_TILE - 1, y0 = blockIdx.y * PAD_TILE - 1;  // padded tile origin - 1
    // padded z planes strided over the grid's z blocks: a small grid, so a
    // call with no xy-mode view (every circular trajectory) costs one wave of
    // blocks that return at once
    for (int zp = blockIdx.z; zp < Zp; zp += gridDim.z) {
        const int z = zp - 1;  // source z
        const bool zin = z >= 0 && z < Z;
        __syncthreads();  // the previous plane's transposed reads are done
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
        const float c00 = lerp_first<T>(p000, p100, fz.f), c_f = lerp_first<T>(p_f, q_f, fz.f);
        const float c_s = lerp_first<T>(p0s, q0s, fz.f), c_fs = lerp_first<T>(p_fs, q_fs, fz.f);
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

// floor and fraction of z2 / 2 from z2 = 2 z (exact: scaling by two commutes
// with every rounding here): bits = floor(z) + FLOOR_BIAS_2Z, f = 2 (z - floor(z))
constexpr int FLOOR_BIAS_2Z = 0x4BC00000;  // bit pattern of 1.5 * 2^24
__device__ __forceinline__ FloorFrac floor_frac_2z(float z2)
{
    const float magic = 25165824.0f;  // 1.5 * 2^24: ulp 2, so the sum rounds down to an even integer
    const float y = __fadd_rd(z2, magic);
    FloorFrac r;
    r.bits = __float_as_int(y);
    r.i = r.bits - FLOOR_BIAS_2Z;
    r.f = __fadd_rn(z2, -__fadd_rn(y, -magic));
    return r;
}

// The cell index with the three floor biases folded in, FLOOR_BIAS (s_x +
// s_y) + z bias + index (mod 2^32), is the bias plus the index without
// wrapping when the x pitch s_x is chosen for it (cell_x_pitch): then the
// biased index addresses the copy through one unsigned 32 x 32 -> 64-bit
// multiply-add from a base that takes the bias back out.
__host__ __device__ inline unsigned cell_index_bias(unsigned s_x, unsigned s_y, bool z2)
{
    return (unsigned)FLOOR_BIAS * (s_x + s_y) + (unsigned)(z2 ? FLOOR_BIAS_2Z : FLOOR_BIAS);
}

// Trilinear interpolation from the cell copy: one cell load gives the eight
// taps.  The packed sampler takes z in half-voxel units (Z2): its floor then
// gives the doubled z weight the half-difference lerp multiplies by, with no
// doubling per sample.
template <typename T, bool PACKED>
struct CellSampler {
    using C = typename Cell<T>::type;
    static constexpr bool Z2 = PACKED;
    unsigned long long base;  // address of biased index 0 (modulo 2^64)
    unsigned s_y, s_x;        // cell strides of y and x (z is fastest)

    // `cells` is the copy's first cell, whose floor is (-1, -1, -1)
    __device__ CellSampler(const C *cells, int sy, int sx) : s_y((unsigned)sy), s_x((unsigned)sx)
    {
        const unsigned long long origin = (unsigned long long)s_x + s_y + 1;  // index of floor (0, 0, 0)
        base = (unsigned long long)cells + sizeof(C) * (origin - cell_index_bias(s_x, s_y, Z2));
    }

    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        const FloorFrac fx = floor_frac(x), fy = floor_frac(y), fz = Z2 ? floor_frac_2z(z) : floor_frac(z);
        const unsigned t = (unsigned)fx.bits * s_x + (unsigned)fy.bits * s_y + (unsigned)fz.bits;
        const C *c = (const C *)(base + (unsigned long long)t * sizeof(C));
        // the reference's order: lerp in z, then y, then x
        if constexpr (PACKED)
            return Cell<T>::trilinear_packed(c, fz.f, fy.f, fx.f);
        else
            return Cell<T>::trilinear(c, fz.f, fy.f, fx.f);
    }
};

template <typename T, bool PACKED>
struct ClampedCellSampler {
    CellSampler<T, PACKED> s;
    float xmax, ymax, zlo, zmax;  // z bounds in the sampler's z units
    __device__ __forceinline__ float operator()(float x, float y, float z) const
    {
        return s(fminf(fmaxf(x, -1.0f), xmax), fminf(fmaxf(y, -1.0f), ymax), fminf(fmaxf(z, zlo), zmax));
    }
};

// The march of one z-mode ray over the cell copy.
template <typename T, bool PACKED>
__device__ __forceinline__ float march_cells(const ConeRay &ray, float step, bool inside,
                                             const typename Cell<T>::type *cells, int Z, int s_x, float xmax,
                                             float ymax, float zmax)
{
    const CellSampler<T, PACKED> s(cells, Z + 2, s_x);
    const int n = inside ? exact_sample_count(ray, step) : -1;
    // samples per iteration: four for the 32-byte FP32 cells (whose loads
    // need twice the registers), seven for FP16 and six for BF16 cells
    // (measured on the 512^3 forward, the best of a sweep whose times follow
    // the compiler's schedule more than the count: FP16 4 / 5 / 6 / 7 / 8 per
    // iteration 82.3 / 80.3 / 79.0 / 77.2 / 77.4 ms; BF16 5 / 6 / 7 / 8 / 10:
    // 76.0 / 74.5 / 77.5 / 76.0 / 75.8 ms)
    constexpr int U = sizeof(T) == 4 ? 4 : (std::is_same<T, __half>::value ? 7 : 6);
    // the packed sampler's z in half-voxel units: the ray's z scaled by two
    // (fmaf(a, 2 dz, 2 oz) = 2 fmaf(a, dz, oz) exactly), clamps with it
    ConeRay r = ray;
    float zlo = -1.0f;
    if (CellSampler<T, PACKED>::Z2) r.dz *= 2.0f, r.oz *= 2.0f, zlo = -2.0f, zmax *= 2.0f;
    return n > 0    ? march_counted<U>(r, n, step, s)
           : inside ? march_x2(r, step, s)
                    : march_x2(r, step, ClampedCellSampler<T, PACKED>{s, xmax, ymax, zlo, zmax});
}

// Grid: one dimension, ray_block_count blocks in ray_block order (four
// blocks of 256 threads per 32 x 32 ray tile, neighbouring views of a tile
// consecutive, cone_ray.cuh).  z mode: a warp is 32 consecutive v at one u, and the
// block's 8 x 32 results go through shared memory so the sinogram rows are
// written 8 pixels at a time; xy mode: a warp is 32 consecutive u.
template <typename T, typename Tout>
// (4 blocks per SM: 64 registers hold the counted loop without spills, and
// 32 resident warps hide the cell loads better than 24 with 80 registers)
__global__ void __launch_bounds__(PB_X *PB_Y, 4)
    cone_fp_padded_kernel(const T *__restrict__ xfast, const T *__restrict__ yfast,
                          const typename Cell<T>::type *__restrict__ cells, Tout *__restrict__ sino,
                          const ConeFpView *__restrict__ views, const float *__restrict__ step_ptr,
                          const float *__restrict__ spacing_ptr, int X, int Y, int Z, int cell_sx, int W, int H,
                          int n_proj, int geom_batch, int b, const unsigned *__restrict__ flags)
{
    __shared__ float out_tile[PB_Y][PB_X + 1];
    const RayBlock rb = ray_block(blockIdx.x, W, H, n_proj);
    const int p = rb.p, sub = rb.sub, tile_u = rb.tile_u, tile_v = rb.tile_v;
    const int g = geom_batch == 1 ? 0 : b;
    const ConeFpView &view = views[(size_t)g * n_proj + p];
    const bool zmode = view_is_z_mode(view);
    int u, v;
    if (zmode) {
        u = tile_u * 32 + sub * PB_Y + threadIdx.y;
        v = tile_v * 32 + threadIdx.x;
    } else {
        u = tile_u * 32 + threadIdx.x;
        v = tile_v * 32 + sub * PB_Y + threadIdx.y;
    }
    const bool live = u < W && v < H;
    const float step = step_ptr[g];
    // 16-bit cells take the packed lerps unless the input's range forbids them
    const bool packed = sizeof(T) == 2 && !flags[FLAG_WIDE];
    float pixel = 0.0f;
    if (live && in_footprint(view, u, v)) {
        const ConeRay ray = cone_ray_setup(view, u, v, X, Y, Z, 0.0, step, spacing_ptr[g * 3 + 2],
                                           spacing_ptr[g * 3 + 1], spacing_ptr[g * 3 + 0]);
        const bool inside = march_inside(ray, X, Y, Z);
        const float xmax = (float)X + 0.999f, ymax = (float)Y + 0.999f, zmax = (float)Z + 0.999f;
        const int Xp = X + 3, Yp = Y + 3;
        if (zmode) {
            if (packed)
                pixel = march_cells<T, sizeof(T) == 2>(ray, step, inside, cells, Z, cell_sx, xmax, ymax, zmax);
            else
                pixel = march_cells<T, false>(ray, step, inside, cells, Z, cell_sx, xmax, ymax, zmax);
        } else {
            // rays mostly along x -> y-fastest copy
            const double cr0 = view.inv_ar[2] + 0.5 * (W - 1) * view.inv_ar[0] + 0.5 * (H - 1) * view.inv_ar[1];
            const double cr1 = view.inv_ar[5] + 0.5 * (W - 1) * view.inv_ar[3] + 0.5 * (H - 1) * view.inv_ar[4];
            const int s_slice = Xp * Yp;
            if (fabs(cr0) > fabs(cr1)) {
                const PaddedSampler<T, true> s{yfast + s_slice + Yp + 1, Yp, s_slice};
                pixel = inside ? march_x2(ray, step, s)
                               : march_x2(ray, step, ClampedSampler<T, true>{s, xmax, ymax, zmax});
            } else {
                const PaddedSampler<T, false> s{xfast + s_slice + Xp + 1, Xp, s_slice};
                pixel = inside ? march_x2(ray, step, s)
                               : march_x2(ray, step, ClampedSampler<T, false>{s, xmax, ymax, zmax});
            }
        }
    }
    Tout *out = sino + ((size_t)b * n_proj + p) * H * (size_t)W;
    if (!zmode) {
        if (live) store_from_float(out + (size_t)v * W + u, pixel);
        return;
    }
    // z mode: transpose the 8 (u) x 32 (v) results so each row is written as 8 pixels
    out_tile[threadIdx.y][threadIdx.x] = pixel;
    __syncthreads();
    const int t = threadIdx.y * PB_X + threadIdx.x;
    const int ov = tile_v * 32 + t / PB_Y, ou = tile_u * 32 + sub * PB_Y + t % PB_Y;
    if (ov < H && ou < W) store_from_float(out + (size_t)ov * W + ou, out_tile[t % PB_Y][t / PB_Y]);
}

size_t section_bytes(size_t n)
{
    return (n + 255) / 256 * 256;
}

// x pitch (in cells) of the cell copy: the least s_x >= (Y+2) (Z+2) for which
// the sampler's biased index, cell_index_bias + index, stays in [0, 2^32) for
// every index of the copy relative to floor (0, 0, 0) -- from -(s_x + s_y + 1)
// up to below (X+2) s_x -- under both z floors; 0 when none is found.  The
// bias moves by FLOOR_BIAS (mod 2^32) per unit of s_x, which steps through all
// 1024 multiples of 2^22, so a few units of padding suffice.
long long cell_x_pitch(int vol_x, int vol_y, int vol_z)
{
    const unsigned long long Xc = vol_x + 2, Yc = vol_y + 2, Zc = vol_z + 2;
    for (unsigned long long sx = Yc * Zc; sx < Yc * Zc + 2048 && Xc * sx < (1ULL << 31); ++sx) {
        bool ok = true;
        for (const bool z2 : {false, true}) {
            const unsigned long long bias = cell_index_bias((unsigned)sx, (unsigned)Zc, z2);
            ok = ok && bias >= sx + Zc + 1 && bias + Xc * sx <= (1ULL << 32);
        }
        if (ok) return (long long)sx;
    }
    return 0;
}

template <typename Tin, typename Tout>
cudaError_t launch_typed(const void *volume, void *sinogram, const Dims3D &d, const ConeFpView *views,
                         const float *step, const float *spacing, void *scratch, unsigned *flags, cudaStream_t stream)
{
    using CellT = typename Cell<Tin>::type;
    const size_t Xp = d.vol_x + 3, Yp = d.vol_y + 3, Zp = d.vol_z + 3;
    const size_t Xc = d.vol_x + 2, Yc = d.vol_y + 2, Zc = d.vol_z + 2;
    const long long cell_sx = cell_x_pitch(d.vol_x, d.vol_y, d.vol_z);
    if (cell_sx <= 0) return cudaErrorInvalidValue;
    char *base = (char *)scratch;
    Tin *xfast = (Tin *)base;
    Tin *yfast = (Tin *)(base + section_bytes(Xp * Yp * Zp * sizeof(Tin)));
    CellT *cells = (CellT *)(base + 2 * section_bytes(Xp * Yp * Zp * sizeof(Tin)));
    const int nviews = d.geom_batch * d.n_proj;
    classify_views_kernel<<<(nviews + 127) / 128, 128, 0, stream>>>(views, nviews, flags);
    const dim3 pblock(PAD_TILE, 8);
    const dim3 pgrid((unsigned)((Xp + PAD_TILE - 1) / PAD_TILE), (unsigned)((Yp + PAD_TILE - 1) / PAD_TILE),
                     (unsigned)std::min<size_t>(Zp, PAD_Z_BLOCKS));
    const dim3 cgrid((unsigned)((Xc + PAD_TILE - 1) / PAD_TILE), (unsigned)((Yc + CELL_PLANES - 1) / CELL_PLANES),
                     (unsigned)((Zc + PAD_TILE - 1) / PAD_TILE));
    const dim3 block(PB_X, PB_Y);
    const unsigned grid = ray_block_count(d.det_w, d.det_h, d.n_proj);
    for (int b = 0; b < d.batch; ++b) {
        const Tin *src = (const Tin *)volume + (size_t)b * d.vol_z * d.vol_y * d.vol_x;
        pad_volume_kernel<Tin><<<pgrid, pblock, 0, stream>>>(src, xfast, yfast, d.vol_x, d.vol_y, d.vol_z, flags);
        if constexpr (sizeof(Tin) == 2) {
            const size_t n = (size_t)d.vol_z * d.vol_y * d.vol_x;
            const unsigned wgrid = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
            detect_wide_kernel<Tin><<<wgrid, 256, 0, stream>>>(src, n, flags);
        }
        pad_cells_kernel<Tin><<<cgrid, pblock, 0, stream>>>(src, cells, d.vol_x, d.vol_y, d.vol_z, (int)cell_sx,
                                                             flags);
        cone_fp_padded_kernel<Tin, Tout><<<grid, block, 0, stream>>>(xfast, yfast, cells, (Tout *)sinogram, views,
                                                                     step, spacing, d.vol_x, d.vol_y, d.vol_z,
                                                                     (int)cell_sx, d.det_w, d.det_h, d.n_proj,
                                                                     d.geom_batch, b, flags);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

size_t cone_fp_padded_scratch_bytes(int vol_z, int vol_y, int vol_x, int in_dtype)
{
    const size_t e = dtype_size(in_dtype);
    const size_t padded = (size_t)(vol_x + 3) * (vol_y + 3) * (vol_z + 3);
    const size_t cells = (size_t)(vol_x + 2) * (size_t)cell_x_pitch(vol_x, vol_y, vol_z);
    return 2 * section_bytes(padded * e) + section_bytes(cells * 8 * e);
}

bool cone_fp_padded_supported(const Dims3D &d)
{
    const long long padded = (long long)(d.vol_x + 3) * (d.vol_y + 3) * (d.vol_z + 3);
    return padded < (1LL << 31) - (1LL << 20) && ray_blocks_fit(d.det_w, d.det_h, d.n_proj) &&
           d.vol_z + 3 <= 65535 && d.vol_y + 3 <= 65535 && cell_x_pitch(d.vol_x, d.vol_y, d.vol_z) > 0;
}

cudaError_t launch_cone_fp_padded(const void *volume, void *sinogram, int in_dtype, int out_dtype, const Dims3D &d,
                                  const ConeFpView *views, const float *step, const float *spacing, void *scratch,
                                  unsigned *flags, cudaStream_t stream)
{
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return launch_typed<Tin, Tout>(volume, sinogram, d, views, step, spacing, scratch, flags, stream);
    });
}

}  // namespace pyronn

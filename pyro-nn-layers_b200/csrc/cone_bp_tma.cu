// cone_bp_tma.cu -- voxel-driven cone backprojector with TMA-staged detector
// tiles (software interpolation, the reference's default hardware_interp=false
// path, cone_backprojector_3D_CudaKernel.cu.cc:84-118).
//
// Block = 256 threads = 32 (x) x 8 (y) voxels, each thread walks 16 voxels
// along z: a 32 x 8 x 16 voxel tile.  Views are processed in passes of
// BP_K views.  For every view of a pass one warp projects the 8 tile corners,
// takes the bounding box of the taps the tile can touch (+1 pixel margin), and
// one thread issues a 3D TMA load of a BW x BH detector box around it into
// shared memory; the next pass's boxes load while the current pass computes
// (two stages, one mbarrier per stage, bounded waits).
// A wait that gives up records DEVICE_ERROR_MBARRIER_TIMEOUT in the error
// word; the block then issues no further load and uses its barriers no more
// (a phase that did not complete must not see another arrival), finishes its
// passes on whatever the tiles hold, and before it exits waits (again
// bounded) for the two passes that can still have boxes in flight.  Its
// voxels are stored, invalid: the error word says so.
//
// Given room in the workspace, a 16-bit sinogram is first copied into a
// paired layout -- element u + 1 of a detector row holds taps u and u + 1 --
// and the boxes stage those 32-bit pairs: a lerp along u is then one shared-
// memory load instead of two, on the same taps with the same operations (the
// same bits).  512^3 workload: backprojection 32.5 -> 31.8 ms, the pairing
// pass (1.1 GB written) included.
//
// Exactness: the tap indices and weights are computed exactly as the direct
// path computes them (floor of u/w, frac), only the texel source differs.  TMA
// zero-fills out-of-range texels, which equals the reference's semantics for
// taps x < W and y < H; a (tile, view) whose box reaches column W or row H --
// where the reference's `>` bounds read the next row / next view -- or does
// not fit the box, or has a corner at w <= 0, is computed from global memory
// with the reference's tap rules instead.  A (tile, view) whose taps all lie
// outside the detector contributes zero and is skipped.
//
// Views whose u and w rows have a zero z coefficient -- every view of a
// circular trajectory about the z axis -- take a column loop: 1/w, w^-2, u,
// the u tap and its weight are then the same for the thread's 16 voxels and
// are computed once, and v steps along the column as one FMA from its value
// at the column base (within a few ulp of the general loop's per-voxel
// v = (P1 . x) / w).
#include <cuda.h>

#include <atomic>

#include "common.cuh"
#include "internal.h"
#include "tma.cuh"

namespace pyronn {

namespace {

constexpr int TB_X = 32;
constexpr int TB_Y = 8;
constexpr int TB_Z = 16;  // voxels per thread along z
constexpr int BP_K = 4;  // views per pass
constexpr int BOX_W = 72;  // 72-element rows shift banks between rows (64 would alias them)
constexpr int BOX_H = 24;
constexpr int BOX_ELEMS = BOX_W * BOX_H;
// Paired boxes (16-bit sinograms given a workspace for the paired copy):
// 32-bit elements (tap u, tap u + 1), 68-word rows (4 banks of shift per row)
constexpr int BOX_WP = 68;

// The staged box of a sinogram type: element type, row length, TMA x
// alignment (elements) and the paired copy's column offset (element u + 1
// holds taps u and u + 1; element 0 holds a zero tap -1 and tap 0).
template <typename T, bool PAIRED>
struct BoxLayout {
    using E = T;
    static constexpr int W = BOX_W, ALIGN = 16 / (int)sizeof(T), OFF = 0;
};
template <typename T>
struct BoxLayout<T, true> {
    using E = unsigned;
    static constexpr int W = BOX_WP, ALIGN = 4, OFF = 1;
};

enum ViewMode : int { MODE_SMEM = 0, MODE_GLOBAL = 1, MODE_SKIP = 2 };

struct ViewMeta {
    float4 row[3];  // voxel-index projection matrix rows
    float u0, v0;   // box origin (pixels), as floats
    int iu0, iv0;   // box origin, as ints
    int mode;
    int zconst;     // row[0].z == row[2].z == 0: u and w constant along z
    int pad[2];
};

// lerp along u of the taps p[0], p[1] in shared memory: the reference's form
// for FP32; for 16-bit taps a + t (b - a) with b - a one mixed-precision
// subtraction (no widening of b)
template <typename T>
__device__ __forceinline__ float smem_ulerp(const T *p, float t);
template <>
__device__ __forceinline__ float smem_ulerp<float>(const float *p, float t)
{
    return lerp_ref(p[0], p[1], t);
}
template <>
__device__ __forceinline__ float smem_ulerp<__half>(const __half *p, float t)
{
    const float a = __half2float(p[0]);
    return fmaf(t, sub_f32_f16<false>(__half_as_ushort(p[1]), a), a);
}
template <>
__device__ __forceinline__ float smem_ulerp<__nv_bfloat16>(const __nv_bfloat16 *p, float t)
{
    const float a = __bfloat162float(p[0]);
    return fmaf(t, sub_f32_bf16<false>(__bfloat16_as_ushort(p[1]), a), a);
}

// the same lerp on a paired element: tap u in the low half, tap u + 1 in the
// high half (the same operations, hence the same bits)
template <typename T>
__device__ __forceinline__ float pair_ulerp(unsigned w, float t);
template <>
__device__ __forceinline__ float pair_ulerp<__half>(unsigned w, float t)
{
    const float a = __half2float(__ushort_as_half((unsigned short)(w & 0xFFFFu)));
    return fmaf(t, sub_f32_f16<true>(w, a), a);
}
template <>
__device__ __forceinline__ float pair_ulerp<__nv_bfloat16>(unsigned w, float t)
{
    const float a = __uint_as_float(w << 16);
    return fmaf(t, sub_f32_bf16<true>(w, a), a);
}
template <typename T, bool PAIRED>
__device__ __forceinline__ float box_ulerp(const typename BoxLayout<T, PAIRED>::E *p, float t)
{
    if constexpr (PAIRED)
        return pair_ulerp<T>(*p, t);  // 16-bit sinograms only
    else
        return smem_ulerp(p, t);
}

// tap rules of interp2D, cone_backprojector_3D_CudaKernel.cu.cc:55-82
template <typename T>
__device__ __forceinline__ float interp_global(const T *__restrict__ sino, float u, float v, unsigned view_base, int W,
                                               int H, unsigned total)
{
    const float fu = floorf(u), fv = floorf(v);
    const float tx = u - fu, ty = v - fv;
    const float fw = (float)W, fh = (float)H;
    const bool vx0 = fu >= 0.0f && fu <= fw;
    const bool vx1 = fu >= -1.0f && fu <= fw - 1.0f;
    const bool vy0 = fv >= 0.0f && fv <= fh;
    const bool vy1 = fv >= -1.0f && fv <= fh - 1.0f;
    const int x0 = __float2int_rz(fu), y0 = __float2int_rz(fv);
    const unsigned i00 = view_base + (unsigned)y0 * (unsigned)W + (unsigned)x0;
    const unsigned i01 = i00 + 1u, i10 = i00 + (unsigned)W, i11 = i10 + 1u;
    const float p00 = (vx0 && vy0 && i00 < total) ? load_as_float(sino + i00) : 0.0f;
    const float p01 = (vx1 && vy0 && i01 < total) ? load_as_float(sino + i01) : 0.0f;
    const float p10 = (vx0 && vy1 && i10 < total) ? load_as_float(sino + i10) : 0.0f;
    const float p11 = (vx1 && vy1 && i11 < total) ? load_as_float(sino + i11) : 0.0f;
    return lerp_ref(lerp_first<T>(p00, p01, tx), lerp_first<T>(p10, p11, tx), ty);
}

// Resident blocks per SM the kernel is compiled for: the paired layout runs
// best at 4 (64 registers; 3 blocks with 80: 512^3 backprojection 31.8 vs
// 32.6 ms), the unpaired at the compiler's choice (80 registers, 3 blocks for
// 16-bit taps: 32.5 ms, against 33.1 ms forced to 4; 0 = no minimum)
#ifndef PYRONN_BP_MIN_BLOCKS
#define PYRONN_BP_MIN_BLOCKS(paired) ((paired) ? 4 : 0)
#endif

// Computes the metadata of one pass (warp 0 only): lane = k * 8 + corner.
template <typename T, bool PAIRED>
__device__ __forceinline__ void pass_meta(ViewMeta *meta, const ConeBpView *__restrict__ pv, int n_first, int n_proj,
                                          int i0, int j0, int k0, int W, int H)
{
    const int lane = threadIdx.x & 31;
    const int k = lane >> 3, c = lane & 7;
    const int n = n_first + k;
    const bool live = n < n_proj;
    float4 r0 = make_float4(0, 0, 0, 0), r1 = r0, r2 = make_float4(0, 0, 0, 1);
    if (live) {
        r0 = __ldg(&pv[n].row[0]);
        r1 = __ldg(&pv[n].row[1]);
        r2 = __ldg(&pv[n].row[2]);
    }
    const float ci = (float)(i0 + ((c & 1) ? TB_X - 1 : 0));
    const float cj = (float)(j0 + ((c & 2) ? TB_Y - 1 : 0));
    const float ck = (float)(k0 + ((c & 4) ? TB_Z - 1 : 0));
    const float un = fmaf(r0.x, ci, fmaf(r0.y, cj, fmaf(r0.z, ck, r0.w)));
    const float vn = fmaf(r1.x, ci, fmaf(r1.y, cj, fmaf(r1.z, ck, r1.w)));
    const float wn = fmaf(r2.x, ci, fmaf(r2.y, cj, fmaf(r2.z, ck, r2.w)));
    float u = un / wn, v = vn / wn;
    float umin = u, umax = u, vmin = v, vmax = v, wmin = wn;
    // a NaN corner makes the view take the global path
    bool finite = isfinite(u) && isfinite(v);
#pragma unroll
    for (int off = 1; off < 8; off <<= 1) {
        umin = fminf(umin, __shfl_xor_sync(0xffffffffu, umin, off));
        umax = fmaxf(umax, __shfl_xor_sync(0xffffffffu, umax, off));
        vmin = fminf(vmin, __shfl_xor_sync(0xffffffffu, vmin, off));
        vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, off));
        wmin = fminf(wmin, __shfl_xor_sync(0xffffffffu, wmin, off));
        finite = __shfl_xor_sync(0xffffffffu, (int)finite, off) && finite;
    }
    if (live && c == 0) {
        ViewMeta m;
        m.row[0] = r0;
        m.row[1] = r1;
        m.row[2] = r2;
        int mode = MODE_GLOBAL;
        int iu0 = 0, iv0 = 0;
        if (finite && wmin > 0.0f && fabsf(umin) < 1.0e6f && fabsf(umax) < 1.0e6f && fabsf(vmin) < 1.0e6f &&
            fabsf(vmax) < 1.0e6f) {
            // taps span [floor(u), floor(u) + 1]; one pixel of margin each side
            const int x_lo = (int)floorf(umin) - 1, x_hi = (int)floorf(umax) + 2;
            const int y_lo = (int)floorf(vmin) - 1, y_hi = (int)floorf(vmax) + 2;
            if (x_hi < 0 || y_hi < 0 || x_lo > W || y_lo > H) {
                mode = MODE_SKIP;  // every tap outside the detector and past the quirk row/column
            } else {
                // the box's first element, x = iu0 + OFF in the staged
                // layout, on the TMA alignment
                using L = BoxLayout<T, PAIRED>;
                const int a = L::ALIGN, xo = x_lo + L::OFF;
                iu0 = ((xo >= 0) ? (xo / a) * a : -(((-xo) + a - 1) / a) * a) - L::OFF;
                iv0 = y_lo;
                // elements up to x_hi (the unpaired box's taps) or x_hi - 1
                // (the paired element x_hi - 1 holds tap x_hi)
                const bool fits = (x_hi - L::OFF - iu0 + 1 <= L::W) && (y_hi - iv0 + 1 <= BOX_H);
                const bool clear_of_quirk = (x_hi <= W - 1) && (y_hi <= H - 1);
                if (fits && clear_of_quirk) mode = MODE_SMEM;
            }
        }
        m.u0 = (float)iu0;
        m.v0 = (float)iv0;
        m.iu0 = iu0;
        m.iv0 = iv0;
        m.mode = mode;
        m.zconst = (r0.z == 0.0f && r2.z == 0.0f) ? 1 : 0;
        meta[k] = m;
    }
}

template <typename T, typename Tout, bool PAIRED>
__global__ void __launch_bounds__(TB_X *TB_Y, PYRONN_BP_MIN_BLOCKS(PAIRED))
    cone_bp_tma_kernel(const __grid_constant__ CUtensorMap tmap, const T *__restrict__ sino, Tout *__restrict__ vol,
                       const ConeBpView *__restrict__ views, const float *__restrict__ mult, int X, int Y, int Z,
                       int W, int H, int n_proj, int geom_batch, unsigned *__restrict__ err,
                       int starve_last_pass)
{
    extern __shared__ __align__(128) unsigned char dyn_smem[];
    // TMA destinations must be 128-byte aligned: round the base up (the
    // launch reserves 128 spare bytes); every tile is a multiple of 128 bytes
    unsigned char *tile_base = dyn_smem + ((128u - (smem_addr(dyn_smem) & 127u)) & 127u);
    using E = typename BoxLayout<T, PAIRED>::E;
    constexpr int BW = BoxLayout<T, PAIRED>::W, BE = BW * BOX_H;
    E(*tiles)[BP_K][BE] = reinterpret_cast<E(*)[BP_K][BE]>(tile_base);  // [2][BP_K][BE]
    __shared__ __align__(16) ViewMeta meta[2][BP_K];
    __shared__ __align__(8) uint64_t full[2];
    __shared__ int s_failed;  // first pass whose wait gave up, n_pass if none (kept out of registers)

    const int tid = threadIdx.y * TB_X + threadIdx.x;
    const int warp = tid >> 5;
    const int i0 = blockIdx.x * TB_X, j0 = blockIdx.y * TB_Y;
    const int zblocks = (Z + TB_Z - 1) / TB_Z;
    const int k0 = (blockIdx.z % zblocks) * TB_Z;
    const int b = blockIdx.z / zblocks;
    const int i = i0 + threadIdx.x, j = j0 + threadIdx.y;
    const int g = geom_batch == 1 ? 0 : b;
    const ConeBpView *pv = views + (size_t)g * n_proj;
    const T *sino_b = sino + (size_t)b * n_proj * H * W;
    const unsigned total = (unsigned)n_proj * (unsigned)H * (unsigned)W;
    const int n_pass = (n_proj + BP_K - 1) / BP_K;
    constexpr unsigned TILE_BYTES = BE * sizeof(E);

    if (tid == 0) {
        mbar_init(&full[0], 1);
        mbar_init(&full[1], 1);
        fence_mbar_init();
        s_failed = n_pass;
    }
    // spin limit of the bounded waits: short for the starved test pass
#define PYRONN_BP_SPINS (starve_last_pass ? (1u << 12) : (1u << 22))
    // issues the TMA loads of pass p into stage s (one thread)
    auto issue = [&](int p, int s) {
        if (s_failed < n_pass) return;  // after a failed wait: no load, no arrival
        if (starve_last_pass && p == n_pass - 1) {
            // test hook: wait for bytes no copy will deliver, with no copy in flight
            mbar_arrive_expect_tx(&full[s], 16u);
            return;
        }
        int n_fast = 0;
#pragma unroll
        for (int k = 0; k < BP_K; ++k) n_fast += (p * BP_K + k < n_proj && meta[s][k].mode == MODE_SMEM);
        mbar_arrive_expect_tx(&full[s], n_fast * TILE_BYTES);
#pragma unroll
        for (int k = 0; k < BP_K; ++k) {
            const int n = p * BP_K + k;
            if (n < n_proj && meta[s][k].mode == MODE_SMEM)
                tma_load_3d(&tiles[s][k][0], &tmap, meta[s][k].iu0 + BoxLayout<T, PAIRED>::OFF, meta[s][k].iv0,
                            b * n_proj + n, &full[s]);
        }
    };
    if (warp == 0) {
        pass_meta<T, PAIRED>(meta[0], pv, 0, n_proj, i0, j0, k0, W, H);
        __syncwarp();
    }
    __syncthreads();
    if (tid == 0) issue(0, 0);

    float acc[TB_Z];
#pragma unroll
    for (int z = 0; z < TB_Z; ++z) acc[z] = 0.0f;
    const float fi = (float)i, fj = (float)j, fk = (float)k0;
    // a lerp reads elements idx and idx + 1 (one paired element)
    constexpr unsigned LAST = PAIRED ? 1 : 2;
    constexpr unsigned MAX_IDX = BE - BW - LAST, MAX_IDX2 = BE - 2 * BW - LAST;
    static_assert(TB_Z % 2 == 0, "the column loop takes voxels in pairs");

    for (int p = 0; p < n_pass; ++p) {
        const int cur = p & 1, nxt = cur ^ 1;
        __syncthreads();  // pass p-1 is done with stage nxt
        if (warp == 0 && p + 1 < n_pass) {
            pass_meta<T, PAIRED>(meta[nxt], pv, (p + 1) * BP_K, n_proj, i0, j0, k0, W, H);
            __syncwarp();
            if (tid == 0) issue(p + 1, nxt);
        }
        if (s_failed == n_pass && !mbar_wait_bounded(&full[cur], (p >> 1) & 1, err, PYRONN_BP_SPINS))
            atomicMin(&s_failed, p);
#pragma unroll 1
        for (int k = 0; k < BP_K; ++k) {
            const int n = p * BP_K + k;
            if (n >= n_proj) break;
            const ViewMeta &m = meta[cur][k];
            const int mode = m.mode;
            if (mode == MODE_SKIP) continue;
            const float4 r0 = m.row[0], r1 = m.row[1], r2 = m.row[2];
            const float ub = fmaf(r0.x, fi, fmaf(r0.y, fj, fmaf(r0.z, fk, r0.w)));
            const float vb = fmaf(r1.x, fi, fmaf(r1.y, fj, fmaf(r1.z, fk, r1.w)));
            const float wb = fmaf(r2.x, fi, fmaf(r2.y, fj, fmaf(r2.z, fk, r2.w)));
            if (mode == MODE_SMEM && m.zconst) {
                const E *tile = &tiles[cur][k][0];
                // fmaf(0, z, x) == x: these are the general loop's values at every z
                const float rw = fast_rcp(wb), rw2 = rw * rw;
                // floor and weight of u itself, the box origin subtracted
                // from the integer floor: the tap and weight do not depend on
                // where the box starts (paired and unpaired boxes align
                // differently, and u - u0 in floating point rounds when u0 < 0)
                const FloorFrac fu = floor_frac(__fmul_rn(ub, rw));
                const float tx = fu.f;
                // row of floor(lv) from its FloorFrac bits: the bias folded into one offset
                const unsigned col = (unsigned)(fu.i - m.iu0) - (unsigned)FLOOR_BIAS * (unsigned)BW;
                const float lv0 = fmaf(vb, rw, -m.v0), dlv = r1.z * rw;  // local v at z = 0, its step
                if (dlv >= 0.0f && dlv < 0.999f) {
                    // rows of voxels z and z + 1 differ by 0 or 1: the pair
                    // reads rows r, r + 1, r + 2 once (three u lerps for two
                    // voxels instead of four) and gives each voxel the same
                    // taps, hence the same bits, as the loop below
#pragma unroll
                    for (int z = 0; z < TB_Z; z += 2) {
                        const float la = fmaf((float)z, dlv, lv0), lb = fmaf((float)(z + 1), dlv, lv0);
                        const FloorFrac fa = floor_frac(la), fb = floor_frac(lb);
                        unsigned idx = (unsigned)fa.bits * (unsigned)BW + col;
                        idx = min(idx, MAX_IDX2);  // memory safety only: the margin keeps idx in range
                        const float p0 = box_ulerp<T, PAIRED>(tile + idx, tx);
                        const float p1 = box_ulerp<T, PAIRED>(tile + idx + BW, tx);
                        const float p2 = box_ulerp<T, PAIRED>(tile + idx + 2 * BW, tx);
                        acc[z] = fmaf(lerp_ref(p0, p1, fa.f), rw2, acc[z]);
                        const bool up = fb.bits != fa.bits;
                        acc[z + 1] = fmaf(lerp_ref(up ? p1 : p0, up ? p2 : p1, fb.f), rw2, acc[z + 1]);
                    }
                } else {
#pragma unroll
                    for (int z = 0; z < TB_Z; ++z) {
                        const float lv = fmaf((float)z, dlv, lv0);
                        const FloorFrac fv = floor_frac(lv);
                        unsigned idx = (unsigned)fv.bits * (unsigned)BW + col;
                        idx = min(idx, MAX_IDX);  // memory safety only: the margin keeps idx in range
                        const float val = lerp_ref(box_ulerp<T, PAIRED>(tile + idx, tx),
                                                   box_ulerp<T, PAIRED>(tile + idx + BW, tx), fv.f);
                        acc[z] = fmaf(val, rw2, acc[z]);
                    }
                }
            } else if (mode == MODE_SMEM) {
                const E *tile = &tiles[cur][k][0];
                const int iu0 = m.iu0, iv0 = m.iv0;
#pragma unroll
                for (int z = 0; z < TB_Z; ++z) {
                    const float fz = (float)z;
                    const float rw = fast_rcp(fmaf(r2.z, fz, wb));
                    // floors and weights of (u, v) themselves, the box origin
                    // subtracted from the integer floors (see the column loop)
                    const float uu = __fmul_rn(fmaf(r0.z, fz, ub), rw);
                    const float vv = __fmul_rn(fmaf(r1.z, fz, vb), rw);
                    const FloorFrac fu = floor_frac(uu), fv = floor_frac(vv);
                    const float tx = fu.f, ty = fv.f;
                    unsigned idx = (unsigned)((fv.i - iv0) * BW + (fu.i - iu0));
                    idx = min(idx, MAX_IDX);  // memory safety only: the margin keeps idx in range
                    const float val = lerp_ref(box_ulerp<T, PAIRED>(tile + idx, tx),
                                               box_ulerp<T, PAIRED>(tile + idx + BW, tx), ty);
                    acc[z] = fmaf(val * rw, rw, acc[z]);
                }
            } else {
                const unsigned view_base = (unsigned)n * (unsigned)H * (unsigned)W;
#pragma unroll
                for (int z = 0; z < TB_Z; ++z) {
                    const float fz = (float)z;
                    const float rw = fast_rcp(fmaf(r2.z, fz, wb));
                    const float uu = fmaf(r0.z, fz, ub) * rw, vv = fmaf(r1.z, fz, vb) * rw;
                    const float val = interp_global<T>(sino_b, uu, vv, view_base, W, H, total);
                    acc[z] = fmaf(val * rw, rw, acc[z]);
                }
            }
        }
    }
    __syncthreads();
    if (tid == 0 && s_failed < n_pass) {
        // boxes possibly still in flight: those of the pass waited for in
        // vain and of the pass issued before that wait; the CTA must not
        // exit while they can still write its shared memory
        const int q = s_failed;
        for (int r = q; r <= q + 1 && r < n_pass; ++r)
            mbar_wait_bounded(&full[r & 1], (r >> 1) & 1, nullptr, PYRONN_BP_SPINS);
    }
#undef PYRONN_BP_SPINS
    if (i < X && j < Y) {
        const float mv = mult[g];
        Tout *vol_b = vol + (size_t)b * Z * Y * X;
#pragma unroll
        for (int z = 0; z < TB_Z; ++z)
            if (k0 + z < Z) store_from_float(vol_b + ((size_t)(k0 + z) * Y + j) * X + i, acc[z] * mv);
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// looked up once per process (a function-local static initialises once, also
// when several host threads get here together)
EncodeTiledFn encode_fn()
{
    static const EncodeTiledFn fn = []() -> EncodeTiledFn {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return (EncodeTiledFn)p;
        return nullptr;
    }();
    return fn;
}

template <typename T>
CUtensorMapDataType tma_type();
template <>
CUtensorMapDataType tma_type<float>()
{
    return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
}
template <>
CUtensorMapDataType tma_type<__nv_bfloat16>()
{
    return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}
template <>
CUtensorMapDataType tma_type<__half>()
{
    return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
}

// The paired copy of a 16-bit sinogram: per detector row, element x holds
// taps x - 1 (low half) and x (high half), x in [0, Wp), Wp = W + 1 rounded
// up to 4 (16-byte rows), taps outside [0, W) zero.  Grid: x chunks of 256
// elements by rows (a row per blockIdx.y, strided).
template <typename T>
__global__ void __launch_bounds__(256)
    pair_sinogram_kernel(const T *__restrict__ sino, unsigned *__restrict__ paired, int W, int Wp, long long rows)
{
    const int x = blockIdx.x * 256 + threadIdx.x;
    if (x >= Wp) return;
    for (long long r = blockIdx.y; r < rows; r += gridDim.y) {
        const unsigned short *row = reinterpret_cast<const unsigned short *>(sino + r * W);
        const unsigned lo = (x >= 1 && x <= W) ? __ldg(row + x - 1) : 0u;
        const unsigned hi = (x < W) ? __ldg(row + x) : 0u;
        paired[r * Wp + x] = lo | (hi << 16);
    }
}

inline int paired_row(int W)
{
    return (W + 1 + 3) / 4 * 4;
}

template <typename Tin, typename Tout, bool PAIRED>
cudaError_t launch_kernel(const void *sinogram, const void *staged, void *volume, const Dims3D &d,
                          const ConeBpView *views, const float *mult, unsigned *err, int starve_last_pass,
                          cudaStream_t stream)
{
    EncodeTiledFn enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    using L = BoxLayout<Tin, PAIRED>;
    using E = typename L::E;
    const cuuint64_t row = PAIRED ? (cuuint64_t)paired_row(d.det_w) : (cuuint64_t)d.det_w;
    CUtensorMap map;
    const cuuint64_t dims[3] = {row, (cuuint64_t)d.det_h, (cuuint64_t)d.n_proj * d.batch};
    const cuuint64_t strides[2] = {row * sizeof(E), row * d.det_h * sizeof(E)};
    const cuuint32_t box[3] = {(cuuint32_t)L::W, BOX_H, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType type = PAIRED ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : tma_type<Tin>();
    CUresult r = enc(&map, type, 3, const_cast<void *>(staged), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return cudaErrorInvalidValue;
    const int zblocks = (d.vol_z + TB_Z - 1) / TB_Z;
    const dim3 block(TB_X, TB_Y, 1);
    const dim3 grid((d.vol_x + TB_X - 1) / TB_X, (d.vol_y + TB_Y - 1) / TB_Y, zblocks * d.batch);
    static_assert((BOX_ELEMS * sizeof(float)) % 128 == 0 && (BOX_ELEMS * 2) % 128 == 0 &&
                      (BOX_WP * BOX_H * 4) % 128 == 0,
                  "tile alignment");
    const size_t smem = 2 * BP_K * (size_t)L::W * BOX_H * sizeof(E) + 128;
    // set on every launch: the attribute belongs to the current device's copy
    // of the kernel, and the call is a cheap host-side update
    cudaError_t e = cudaFuncSetAttribute(cone_bp_tma_kernel<Tin, Tout, PAIRED>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    cone_bp_tma_kernel<Tin, Tout, PAIRED><<<grid, block, smem, stream>>>(
        map, (const Tin *)sinogram, (Tout *)volume, views, mult, d.vol_x, d.vol_y, d.vol_z, d.det_w, d.det_h, d.n_proj,
        d.geom_batch, err, starve_last_pass);
    return cudaGetLastError();
}

template <typename Tin, typename Tout>
cudaError_t launch_typed(const void *sinogram, void *volume, const Dims3D &d, const ConeBpView *views,
                         const float *mult, unsigned *err, int starve_last_pass, void *paired, cudaStream_t stream)
{
    if constexpr (sizeof(Tin) == 2) {
        if (paired) {
            const int Wp = paired_row(d.det_w);
            const long long rows = (long long)d.batch * d.n_proj * d.det_h;
            const dim3 pgrid((unsigned)((Wp + 255) / 256), (unsigned)(rows < 65535 ? rows : 65535));
            pair_sinogram_kernel<Tin><<<pgrid, 256, 0, stream>>>((const Tin *)sinogram, (unsigned *)paired, d.det_w,
                                                                 Wp, rows);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
            return launch_kernel<Tin, Tout, true>(sinogram, paired, volume, d, views, mult, err, starve_last_pass,
                                                  stream);
        }
    }
    return launch_kernel<Tin, Tout, false>(sinogram, sinogram, volume, d, views, mult, err, starve_last_pass, stream);
}

}  // namespace

// The TMA path needs 16-byte aligned sinogram rows and base, and a grid that
// fits one launch; the caller falls back to the direct kernel otherwise.
bool cone_bp_tma_supported(const void *sinogram, int in_dtype, const Dims3D &d)
{
    const size_t e = dtype_size(in_dtype);
    if (e == 0 || ((uintptr_t)sinogram % 16) != 0) return false;
    if (((size_t)d.det_w * e) % 16 != 0) return false;
    const long long zb = (d.vol_z + TB_Z - 1) / TB_Z;
    if (zb * d.batch > 65535 || (d.vol_y + TB_Y - 1) / TB_Y > 65535) return false;
    if ((long long)d.n_proj * d.batch >= (1LL << 31)) return false;
    return encode_fn() != nullptr;
}

namespace {
std::atomic<int> g_starve_last_pass{0};
}  // namespace

void cone_bp_tma_starve_last_pass(int enable)
{
    g_starve_last_pass.store(enable ? 1 : 0);
}

size_t cone_bp_tma_paired_bytes(int in_dtype, const Dims3D &d)
{
    // the pairing pass costs about a read and two writes of the sinogram and
    // saves a shared-memory load per tap pair: it pays when a detector pixel
    // serves many voxel updates (512^3 on 1024 x 768: 171, 31.8 against
    // 32.5 ms; 256^3 on 512^2: 64, 4.26 against 4.08 ms)
    if (dtype_size(in_dtype) != 2) return 0;
    if ((long long)d.vol_x * d.vol_y * d.vol_z < 100LL * d.det_h * d.det_w) return 0;
    return (size_t)d.batch * d.n_proj * d.det_h * (size_t)paired_row(d.det_w) * sizeof(unsigned);
}

cudaError_t launch_cone_bp_tma(const void *sinogram, void *volume, int in_dtype, int out_dtype, const Dims3D &d,
                               const ConeBpView *views, const float *mult, unsigned *err, void *paired,
                               cudaStream_t stream)
{
    const int starve = g_starve_last_pass.load();
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        return launch_typed<Tin, Tout>(sinogram, volume, d, views, mult, err, starve, paired, stream);
    });
}

}  // namespace pyronn

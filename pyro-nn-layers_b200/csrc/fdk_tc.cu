// fdk_tc.cu -- the FDK / FBP ramp filter on the tensor cores (tcgen05).
//
// The linear convolution of every detector row with the ramp kernel,
// q[r][j] = sum_k tau h[j - k] g[r][k], is a product with a Toeplitz matrix:
// Q^T = T G^T with T[j][k] = tau h[j - k].  A CTA computes a tile of 128
// outputs j (the MMA's M, one TMEM lane each) by 128 rows r (its N, one TMEM
// column each) and walks the row's inputs k in chunks of 32:
//   * 512 threads build the chunk's operands in shared memory in the
//     canonical K-major 128-byte-swizzled layout with 16-byte stores: T from
//     a tap table (a chunk of a Toeplitz matrix is a slice of the taps; four
//     shifted copies make every four taps one aligned 16-byte load), G from
//     the projections (loaded one chunk ahead) with the Feldkamp cosine
//     weights applied;
//   * one thread issues tcgen05.mma kind::tf32 (M 128, N 128, K 8) into FP32
//     accumulators in TMEM; two stages, each released by tcgen05.commit on
//     its mbarrier, let the next chunk be built while the MMAs run.
// FP32 accuracy from TF32 inputs: every operand is split into hi (rounded to
// its top 19 bits, exact in TF32) and lo = x - hi (exact in FP32, of either
// sign), and the accumulators take hi*hi + hi*lo + lo*hi (the 3xTF32 scheme;
// the dropped lo*lo term and lo's own TF32 rounding are below 2^-21
// relative).  The tensor core's accumulation is not an IEEE FP32 sum, and the
// ramp filter's output is a small difference of large partial sums, so the
// chunks rotate over four accumulators (each sums a quarter of the row) that
// the epilogue adds in FP32: the result stays within a few 1e-6 of the
// CUDA-core kernel's FP32 sums.
// Epilogue: each warp reads its 32 TMEM lanes (outputs j) 32 columns (rows)
// at a time; for a fixed row the warp's 32 lanes are 32 consecutive outputs,
// so the stores are coalesced without staging.
//
// No TMA and no multicast: every operand byte is written by the CTA's own
// threads.  Waits are bounded: a wait that gives up records
// DEVICE_ERROR_MBARRIER_TIMEOUT in g_fdk_error (read by pyronn_fdk_error); the
// thread then tries its later waits once each, thread 0 issues no more MMAs,
// every thread still walks every chunk (same barriers, no early exit; the
// operands it keeps writing may race with MMAs in flight, and the tile is
// not stored), a failed final wait is waited for again (bounded) before the
// TMEM is freed, and a warp with any failed wait stores nothing.  Skipping
// the operand writes after a failure instead cost 4 % of the filter's time.
#include <type_traits>

#include "common.cuh"
#include "fdk_taps.cuh"
#include "internal.h"
#include "tma.cuh"

namespace pyronn {

namespace {

constexpr int TC_M = 128;   // outputs j per tile (TMEM lanes)
constexpr int TC_N = 128;   // rows per tile (TMEM columns of one accumulator)
constexpr int NACC = 4;     // accumulators, chunk c adds into accumulator c % 4
constexpr int TC_K = 32;    // inputs per chunk: one 128-byte swizzle row of FP32
constexpr int TC_THREADS = 512;  // 16 warps: four per TMEM lane quadrant
constexpr uint32_t A_BYTES = TC_M * TC_K * 4;          // 16 KB
constexpr uint32_t B_BYTES = TC_N * TC_K * 4;          // 16 KB
constexpr uint32_t STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;  // hi and lo of both
constexpr uint32_t TMEM_COLS = TC_N * NACC;  // all 512 columns
constexpr int TC_MAX_WIDTH = 2048;  // two stages + four tap-table copies: at most 199 KB

// sticky device error word of the filter on this device (DeviceError codes)
__device__ unsigned g_fdk_error;

// instruction descriptor: D FP32, A and B TF32, both K-major, N = 128, M = 128
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TC_N >> 3) << 17) |
                           ((uint32_t)(TC_M >> 4) << 24);

// byte offset of element (row, col), col < 32, in a K-major tile of 32-bit
// elements with the 128-byte swizzle: rows of 128 bytes, groups of 8 rows
// 1024 bytes apart, the 16-byte chunk index XORed with the row within its group
__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t col)
{
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((((col >> 2) ^ (row & 7u)) << 4) | ((col & 3u) << 2));
}

// shared-memory matrix descriptor of such a tile (start address in 16-byte
// units, leading offset 1, stride 1024 bytes between 8-row groups, version 1,
// layout SWIZZLE_128B); the tile base is 1024-byte aligned
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
           ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// x split for 3xTF32: hi = x rounded (half away from zero) to 10 mantissa
// bits, so x - hi has either sign and at most half a TF32 unit
__device__ __forceinline__ float tf32_hi(float x)
{
    return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u);
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

// 32 lanes x 32 columns of 32-bit values from TMEM: lane l of the warp gets
// TMEM lane (taddr's lane + l), columns taddr's column .. + 31
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float cosine_weight(float sdd, float uu, float vv2)
{
    return sdd * rsqrtf(fmaf(sdd, sdd, fmaf(uu, uu, vv2)));
}

// four consecutive inputs as raw bits (loaded one chunk ahead, widened when
// the chunk is built, so the load latency overlaps a chunk's work)
template <typename T>
struct Quad {
    using raw = uint2;  // four 16-bit values
    __device__ static raw load(const T *p) { return __ldg(reinterpret_cast<const uint2 *>(p)); }
    __device__ static raw zero() { return make_uint2(0u, 0u); }
    __device__ static void widen(const raw &v, float (&x)[4])
    {
        if (std::is_same<T, __half>::value) {
            x[0] = __half2float(__ushort_as_half((unsigned short)(v.x & 0xFFFFu)));
            x[1] = __half2float(__ushort_as_half((unsigned short)(v.x >> 16)));
            x[2] = __half2float(__ushort_as_half((unsigned short)(v.y & 0xFFFFu)));
            x[3] = __half2float(__ushort_as_half((unsigned short)(v.y >> 16)));
        } else {
            x[0] = __uint_as_float(v.x << 16), x[1] = __uint_as_float(v.x & 0xFFFF0000u);
            x[2] = __uint_as_float(v.y << 16), x[3] = __uint_as_float(v.y & 0xFFFF0000u);
        }
    }
};
template <>
struct Quad<float> {
    using raw = float4;
    __device__ static raw load(const float *p) { return __ldg(reinterpret_cast<const float4 *>(p)); }
    __device__ static raw zero() { return make_float4(0.0f, 0.0f, 0.0f, 0.0f); }
    __device__ static void widen(const raw &v, float (&x)[4]) { x[0] = v.x, x[1] = v.y, x[2] = v.z, x[3] = v.w; }
};

__host__ __device__ inline int tap_copy_len(int Wk)
{
    return (Wk + TC_M - 1 + 3) / 4 * 4;
}

// grid (ceil(W / 128), ceil(rows / 128)) -- the output tiles of one block of
// rows run one after another, so its inputs are re-read from L2 -- 512
// threads, dynamic shared memory
// fdk_tc_smem_bytes(W); Wk = W rounded up to 32 (zero inputs beyond W);
// W a multiple of 4 and 16-byte aligned rows (vector loads of 4 inputs)
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(TC_THREADS, 1)
    fdk_filter_tc_kernel(const Tin *__restrict__ in, Tout *__restrict__ out, long long rows, int det_h, int W,
                         int Wk, float sdd, float dv, float du, float cv, float cu, int kind, int weight_output)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ uint64_t mma_done[2];  // stage s free again: its MMAs are done
    __shared__ uint32_t tmem_slot;
    __shared__ float vv2[TC_N];  // per row of the tile: (v - cv)^2 dv^2 of its detector row
    unsigned char *base = smem_raw + ((1024u - (smem_addr(smem_raw) & 1023u)) & 1023u);
    // the tile's taps tau h[m], m = j0 + jj - k over jj < 128, k < Wk, in
    // reverse order R[x] = tau h[j0 + 127 - x], x in [0, Wk + 127), so that
    // the four taps of a 16-byte chunk of the T tile (inputs k .. k + 3) are
    // R[x0 .. x0 + 3]; copy a holds R shifted by a (copy_a[i] = R[i + a]),
    // which makes every such quadruple one aligned 16-byte load
    const int ntaps = Wk + TC_M - 1, clen = tap_copy_len(Wk);
    float *cop_hi = reinterpret_cast<float *>(base + 2 * STAGE_BYTES);  // [4][clen]
    float *cop_lo = cop_hi + 4 * clen;                                  // [4][clen]

    const int tid = threadIdx.x, warp = tid >> 5;
    const long long r0 = (long long)blockIdx.y * TC_N;
    const int j0 = blockIdx.x * TC_M;
    for (int rr = tid; rr < TC_N; rr += TC_THREADS) {
        const long long row = r0 + rr;
        const float vv = row < rows ? ((float)(int)(row % det_h) - cv) * dv : 0.0f;
        vv2[rr] = vv * vv;
    }
    for (int x = tid; x < clen + 3; x += TC_THREADS) {
        const float h = x < ntaps ? fdk_tap(kind, j0 + TC_M - 1 - x, du) : 0.0f;
        const float hi = tf32_hi(h), lo = h - hi;
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            const int i = x - a;
            if (i >= 0 && i < clen) {
                cop_hi[a * clen + i] = hi;
                cop_lo[a * clen + i] = lo;
            }
        }
    }
    if (tid == 0) {
        mbar_init(&mma_done[0], 1);
        mbar_init(&mma_done[1], 1);
        fence_mbar_init();
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_d = tmem_slot;

    // this thread's two B chunks per K chunk: rows rr[i], inputs 4 q[i] .. + 3
    constexpr int BG = (TC_N * TC_K / 4) / TC_THREADS;
    int brr[BG], bq[BG];
    const Tin *bptr[BG];
    bool brow[BG];
    typename Quad<Tin>::raw bnext[BG];
#pragma unroll
    for (int i = 0; i < BG; ++i) {
        const int g = tid + i * TC_THREADS;
        brr[i] = g >> 3, bq[i] = g & 7;
        const long long row = r0 + brr[i];
        brow[i] = row < rows;
        bptr[i] = in + (brow[i] ? row : 0) * W + 4 * bq[i];
        bnext[i] = (brow[i] && 4 * bq[i] < W) ? Quad<Tin>::load(bptr[i]) : Quad<Tin>::zero();
    }
    const int nK = Wk / TC_K;
    bool failed = false;  // one of this thread's waits gave up
    for (int c = 0; c < nK; ++c) {
        const int s = c & 1;
        typename Quad<Tin>::raw bcur[BG];
#pragma unroll
        for (int i = 0; i < BG; ++i) {
            bcur[i] = bnext[i];
            const int kn = (c + 1) * TC_K + 4 * bq[i];
            if (c + 1 < nK) bnext[i] = (brow[i] && kn < W) ? Quad<Tin>::load(bptr[i] + (c + 1) * TC_K) : Quad<Tin>::zero();
        }
        unsigned char *st = base + s * STAGE_BYTES;
        // after a wait gave up the thread tries its later waits once each
        if (c >= 2 && !mbar_wait_bounded(&mma_done[s], ((c - 2) >> 1) & 1, &g_fdk_error, failed ? 1u : (1u << 22)))
            failed = true;
        const int k0 = c * TC_K;
        // 16-byte chunks: g = row * 8 + q, inputs k0 + 4q .. k0 + 4q + 3; a
        // warp covers 4 rows x 8 chunks (512 contiguous bytes when stored)
#pragma unroll
        for (int i = 0; i < (TC_M * TC_K / 4) / TC_THREADS; ++i) {
            // A = T chunk, row jj (output j0 + jj)
            const int g = tid + i * TC_THREADS, jj = g >> 3, q = g & 7;
            const int x0 = TC_M - 1 - jj + k0 + 4 * q, al = x0 & 3;
            const float4 hi = *reinterpret_cast<const float4 *>(cop_hi + al * clen + (x0 - al));
            const float4 lo = *reinterpret_cast<const float4 *>(cop_lo + al * clen + (x0 - al));
            const uint32_t off = sw128((uint32_t)jj, (uint32_t)(4 * q));
            *reinterpret_cast<float4 *>(st + off) = hi;
            *reinterpret_cast<float4 *>(st + A_BYTES + off) = lo;
        }
#pragma unroll
        for (int i = 0; i < BG; ++i) {
            // B = G chunk, row rr (detector row r0 + rr); W is a multiple of
            // 4, so a chunk's four inputs are all inside the row or all zero
            const int rr = brr[i], q = bq[i];
            const int k = k0 + 4 * q;
            float x[4];
            Quad<Tin>::widen(bcur[i], x);
            if (!weight_output && sdd > 0.0f) {
                const float v2 = vv2[rr];
#pragma unroll
                for (int e = 0; e < 4; ++e) x[e] *= cosine_weight(sdd, ((float)(k + e) - cu) * du, v2);
            }
            float4 hi, lo;
            hi.x = tf32_hi(x[0]), hi.y = tf32_hi(x[1]), hi.z = tf32_hi(x[2]), hi.w = tf32_hi(x[3]);
            lo.x = x[0] - hi.x, lo.y = x[1] - hi.y, lo.z = x[2] - hi.z, lo.w = x[3] - hi.w;
            const uint32_t off = sw128((uint32_t)rr, (uint32_t)(4 * q));
            *reinterpret_cast<float4 *>(st + 2 * A_BYTES + off) = hi;
            *reinterpret_cast<float4 *>(st + 2 * A_BYTES + B_BYTES + off) = lo;
        }
        // the stage's writes become visible to the tensor core's (async)
        // proxy; a CTA barrier, then one thread issues the chunk's MMAs
        // (per-warp mbarrier arrivals in place of the barrier measured slower:
        // 4.7 -> 5.4 ms on the 512^3 workload's rows)
        fence_proxy_async_smem();
        __syncthreads();
        if (tid == 0 && !failed) {
            tc_fence_after();
            const uint32_t a = smem_addr(st), b = smem_addr(st + 2 * A_BYTES);
            const uint32_t acc = tmem_d + (uint32_t)((c % NACC) * TC_N);
#pragma unroll
            for (int ks = 0; ks < TC_K / 8; ++ks) {
                const uint32_t ko = (uint32_t)ks * 32u;  // 8 TF32 values = 32 bytes along K
                const uint64_t ahi = sw128_desc(a + ko), alo = sw128_desc(a + A_BYTES + ko);
                const uint64_t bhi = sw128_desc(b + ko), blo = sw128_desc(b + B_BYTES + ko);
                umma_tf32(acc, ahi, bhi, (c >= NACC || ks != 0) ? 1u : 0u);
                umma_tf32(acc, ahi, blo, 1u);
                umma_tf32(acc, alo, bhi, 1u);
            }
            umma_commit(&mma_done[s]);
        }
    }
    // the last commit arrives once every MMA of the tile is done
    const bool done = !failed && mbar_wait_bounded(&mma_done[(nK - 1) & 1], ((nK - 1) >> 1) & 1, &g_fdk_error);
    // MMAs may still be in flight: thread 0 waits for them again (bounded)
    // before the barrier that precedes the TMEM's release
    if (!done && tid == 0) mbar_wait_bounded(&mma_done[(nK - 1) & 1], ((nK - 1) >> 1) & 1, nullptr);
    tc_fence_after();

    // epilogue: warp w reads TMEM lane quadrant w % 4 (outputs
    // j0 + 32 (w % 4) + lane) and 32-row block w / 4 of the columns, summing
    // the accumulators a chunk reached in FP32; for a fixed row the warp's
    // stores are 32 consecutive j
    const int lane = tid & 31, quad = warp & 3;
    const int j = j0 + 32 * quad + lane;
    const float uu = ((float)j - cu) * du;
    const int nacc = nK < NACC ? nK : NACC;
    if (__all_sync(0xffffffffu, done)) {  // warp-uniform: tcgen05.ld is .sync.aligned
        const int q = warp >> 2;
        float sum[32];
        for (int a = 0; a < nacc; ++a) {
            uint32_t v[32];
            tmem_ld32(tmem_d + ((uint32_t)(32 * quad) << 16) + (uint32_t)(a * TC_N + 32 * q), v);
#pragma unroll
            for (int e = 0; e < 32; ++e) sum[e] = a == 0 ? __uint_as_float(v[e]) : sum[e] + __uint_as_float(v[e]);
        }
        if (j < W) {
#pragma unroll
            for (int e = 0; e < 32; ++e) {
                const long long row = r0 + 32 * q + e;
                if (row < rows) {
                    float x = sum[e];
                    if (weight_output && sdd > 0.0f) x *= cosine_weight(sdd, uu, vv2[32 * q + e]);
                    store_from_float(out + row * W + j, x);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_d), "r"(TMEM_COLS) : "memory");
}

size_t fdk_tc_smem_bytes(int W)
{
    const int Wk = (W + TC_K - 1) / TC_K * TC_K;
    return 1024 + 2 * (size_t)STAGE_BYTES + 8 * sizeof(float) * (size_t)tap_copy_len(Wk);
}

}  // namespace

cudaError_t fdk_tc_error(cudaStream_t stream, unsigned *device_error)
{
    cudaError_t e = cudaMemcpyFromSymbolAsync(device_error, g_fdk_error, sizeof(unsigned), 0, cudaMemcpyDeviceToHost,
                                              stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e == cudaSuccess && *device_error != 0u) {
        const unsigned zero = 0u;
        e = cudaMemcpyToSymbolAsync(g_fdk_error, &zero, sizeof(unsigned), 0, cudaMemcpyHostToDevice, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    }
    return e;
}

bool fdk_tc_supported(long long rows, int W, const void *in, const void *out)
{
    return W >= 4 && W <= TC_MAX_WIDTH && W % 4 == 0 && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0 &&
           (rows + TC_N - 1) / TC_N <= 65535;
}

cudaError_t launch_fdk_filter_tc(const void *in, void *out, int in_dtype, int out_dtype, long long rows, int det_h,
                                 int W, float sdd, float dv, float du, float cv, float cu, int kind,
                                 int weight_output, cudaStream_t stream)
{
    const int Wk = (W + TC_K - 1) / TC_K * TC_K;
    const size_t smem = fdk_tc_smem_bytes(W);
    const long long row_tiles = (rows + TC_N - 1) / TC_N;
    if (row_tiles > 65535) return cudaErrorInvalidConfiguration;
    const dim3 grid((unsigned)((W + TC_M - 1) / TC_M), (unsigned)row_tiles);
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) -> cudaError_t {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        auto kernel = fdk_filter_tc_kernel<Tin, Tout>;
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kernel<<<grid, TC_THREADS, smem, stream>>>((const Tin *)in, (Tout *)out, rows, det_h, W, Wk, sdd, dv, du, cv,
                                                   cu, kind, weight_output);
        return cudaGetLastError();
    });
}

}  // namespace pyronn

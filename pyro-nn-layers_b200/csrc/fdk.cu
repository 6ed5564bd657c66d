// fdk.cu -- FDK / FBP pre-processing of projections: Feldkamp cosine
// weighting and discrete ramp filtering of every detector row.
//
// Not part of the reference's ops (the PYRO-NN package filters in Python);
// the algorithms are the published ones: cosine weight SDD / sqrt(SDD^2 +
// u^2 + v^2) of a flat detector (Feldkamp, Davis, Kress 1984) and the spatial
// Ram-Lak / Shepp-Logan kernels of Kak & Slaney (1988, ch. 3), convolved
// linearly along the row: q[j] = tau * sum_k h[j - k] g[k], tau the column
// pitch.  FP32 arithmetic, storage types as the projector ops.
//
// Kernel: direct convolution on the FP32 pipes.  A block holds `rows` whole
// detector rows and the taps in shared memory; each thread computes 16
// consecutive outputs of one row with a sliding window of 16 taps in
// registers: per input sample k, one tap load (the window's new element),
// one broadcast load of g[k] and 16 FMAs.  The taps sit in shared memory with
// one padding word per 16 (index i at i + i/16): the lanes' tap loads, 16
// taps apart, land 17 words apart, in 32 distinct banks, and the 16 loads of
// one window pass share one base address (immediate offsets).  Ram-Lak's
// even taps are zero except the centre: its loop takes the odd taps only
// (half the FMAs and tap loads) and adds the centre tap after.  Results are
// staged through shared memory so the rows are written coalesced.
#include "common.cuh"
#include "fdk_taps.cuh"
#include "internal.h"

namespace pyronn {

namespace {

constexpr int FB = 16;  // consecutive outputs per thread

__host__ __device__ inline int skew(int i)
{
    return i + (i >> 4);
}

__host__ __device__ inline int padded_width(int W)
{
    return (W + FB - 1) / FB * FB;
}

// taps m = -(Wp - 1) .. Wp + FB - 2 (the window can reach past the kernel's
// support, where it meets zero padding or outputs that are not stored)
__host__ __device__ inline int tap_count(int W)
{
    return 2 * padded_width(W) + FB - 2;
}

__host__ __device__ inline int tap_words(int W)
{
    return (skew(tap_count(W) - 1) + 1 + 3) / 4 * 4;
}

// ODD_ONLY: the Ram-Lak kernel, zero at every even offset but 0
template <typename Tin, typename Tout, bool ODD_ONLY>
__global__ void __launch_bounds__(256)
    fdk_filter_kernel(const Tin *in, Tout *out, long long rows, int det_h, int W,
                      float sdd, float dv, float du, float cv, float cu, int kind, int weight_output)
{
    extern __shared__ float smem[];
    const int Wp = padded_width(W);
    float *taps = smem;
    float *g = smem + tap_words(W);  // [blockDim.y][Wp]
    const int tid = threadIdx.y * blockDim.x + threadIdx.x, nthreads = blockDim.x * blockDim.y;

    // tau * h[m], in FP64, rounded once
    const int nt = tap_count(W);
    for (int i = tid; i < nt; i += nthreads) taps[skew(i)] = fdk_tap(kind, i - (Wp - 1), du);

    const long long row = (long long)blockIdx.x * blockDim.y + threadIdx.y;
    const bool live = row < rows;
    const int v = live ? (int)(row % det_h) : 0;
    const float vv = ((float)v - cv) * dv;
    float *gr = g + threadIdx.y * Wp;
    for (int k = threadIdx.x; k < Wp; k += blockDim.x) {
        float x = 0.0f;
        if (live && k < W) {
            x = load_as_float(in + row * W + k);
            if (!weight_output && sdd > 0.0f) {
                const float uu = ((float)k - cu) * du;
                x *= sdd * rsqrtf(fmaf(sdd, sdd, fmaf(uu, uu, vv * vv)));
            }
        }
        gr[k] = x;
    }
    __syncthreads();

    // outputs j0 .. j0 + FB - 1; every thread has one chunk (blockDim.x * FB >= W)
    const int j0 = threadIdx.x * FB;
    float acc[FB], win[FB];
#pragma unroll
    for (int a = 0; a < FB; ++a) acc[a] = 0.0f;
    if (j0 < Wp) {
        // window slot (m mod FB) holds tap m (at index m + Wp - 1); before the
        // first step slots 1 .. FB-1 hold m = j0 + 1 .. j0 + FB - 1.  Indices
        // j0 + Wp + [0, 14] share i >> 4, so they are one base plus a.
        const float *pre = taps + skew(j0 + Wp) - 1;
#pragma unroll
        for (int a = 1; a < FB; ++a)
            if (!ODD_ONLY || (a & 1)) win[a] = pre[a];
        for (int kk = 0; kk < Wp; kk += FB) {
            // this pass's new taps m = j0 - kk - r, indices j0 - kk + Wp - 1 - r,
            // r = 0 .. FB-1: one 16-aligned group, one base minus r
            const float *tb = taps + skew(j0 - kk + Wp - 1);
#pragma unroll
            for (int r = 0; r < FB; ++r) {
                // step k = kk + r needs taps m = j0 - k + a; the new one (a = 0,
                // parity of r) goes into slot (-r) mod FB
                if (!ODD_ONLY || (r & 1)) win[(FB - r) % FB] = tb[-r];
                const float gk = gr[kk + r];
#pragma unroll
                for (int a = 0; a < FB; ++a)
                    if (!ODD_ONLY || ((a - r) & 1)) acc[a] = fmaf(win[(a - r + FB) % FB], gk, acc[a]);
            }
        }
        if (ODD_ONLY) {  // the centre tap, m = 0
            const float h0 = taps[skew(Wp - 1)];
#pragma unroll
            for (int a = 0; a < FB; ++a) acc[a] = fmaf(h0, gr[j0 + a], acc[a]);
        }
    }
    __syncthreads();  // every thread is done with the row
    if (j0 < Wp) {
#pragma unroll
        for (int a = 0; a < FB; ++a) gr[j0 + a] = acc[a];
    }
    __syncthreads();
    if (!live) return;
    for (int k = threadIdx.x; k < W; k += blockDim.x) {
        float x = gr[k];
        if (weight_output && sdd > 0.0f) {
            const float uu = ((float)k - cu) * du;
            x *= sdd * rsqrtf(fmaf(sdd, sdd, fmaf(uu, uu, vv * vv)));
        }
        store_from_float(out + row * W + k, x);
    }
}

}  // namespace

// in and out may be the same buffer: a block reads its rows completely
// before it writes them, and no other block touches them
cudaError_t launch_fdk_filter(const void *in, void *out, int in_dtype, int out_dtype, long long rows, int det_h,
                              int W, float sdd, float dv, float du, float cv, float cu, int kind, int weight_output,
                              cudaStream_t stream)
{
    // the tensor-core kernel reads a row's inputs from every output tile of
    // it, so it needs distinct input and output buffers; in-place calls take
    // the CUDA-core kernel, which holds whole rows in shared memory
    const char *ib = (const char *)in, *ob = (const char *)out;
    const size_t n = (size_t)rows * (size_t)W;
    const bool overlap = ib < ob + n * dtype_size(out_dtype) && ob < ib + n * dtype_size(in_dtype);
    if (fdk_tc_supported(rows, W, in, out) && !overlap)
        return launch_fdk_filter_tc(in, out, in_dtype, out_dtype, rows, det_h, W, sdd, dv, du, cv, cu, kind,
                                    weight_output, stream);
    const int chunks = (W + FB - 1) / FB;
    const int tpr = (chunks + 31) / 32 * 32;  // threads per row, a warp multiple
    const int rpb = 256 / tpr > 0 ? 256 / tpr : 1;
    const size_t smem = ((size_t)tap_words(W) + (size_t)rpb * padded_width(W)) * sizeof(float);
    const long long blocks = (rows + rpb - 1) / rpb;
    return dispatch_dtypes(in_dtype, out_dtype, [&](auto tin, auto tout) -> cudaError_t {
        using Tin = typename decltype(tin)::type;
        using Tout = typename decltype(tout)::type;
        auto kernel = kind == 0 ? fdk_filter_kernel<Tin, Tout, true> : fdk_filter_kernel<Tin, Tout, false>;
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        kernel<<<(unsigned)blocks, dim3(tpr, rpb), smem, stream>>>((const Tin *)in, (Tout *)out, rows, det_h, W,
                                                                  sdd, dv, du, cv, cu, kind, weight_output);
        return cudaGetLastError();
    });
}

}  // namespace pyronn

using namespace pyronn;

extern "C" int pyronn_fdk_filter(const void *projections, void *filtered, int in_dtype, int out_dtype, int batch,
                                 int n_proj, int det_h, int det_w, double sdd, double det_spacing_v,
                                 double det_spacing_u, double principal_v, double principal_u, int filter,
                                 int weight_output, void *stream)
{
    const char *name = "fdk_filter";
    if (!projections || !filtered) return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "%s: null data pointer", name);
    if (in_dtype < 0 || in_dtype > 2 || out_dtype < 0 || out_dtype > 2)
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "%s: unknown dtype %d / %d", name, in_dtype, out_dtype);
    if (batch <= 0 || n_proj <= 0 || det_h <= 0 || det_w <= 0)
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "%s: sizes must be positive", name);
    if (det_w > PYRONN_FDK_MAX_WIDTH)
        return report_error(PYRONN_ERROR_UNSUPPORTED, "%s: detector rows of %d pixels exceed %d", name, det_w,
                            PYRONN_FDK_MAX_WIDTH);
    const long long rows = (long long)batch * n_proj * det_h;
    if (rows >= (1LL << 40)) return report_error(PYRONN_ERROR_UNSUPPORTED, "%s: too many rows", name);
    if (filter != PYRONN_FILTER_RAM_LAK && filter != PYRONN_FILTER_SHEPP_LOGAN)
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT, "%s: unknown filter %d", name, filter);
    if (!(det_spacing_u > 0.0 && det_spacing_u < 1.0e30) || !(det_spacing_v > 0.0 && det_spacing_v < 1.0e30) ||
        !(sdd >= 0.0 && sdd < 1.0e30) || !(principal_v == principal_v && principal_u == principal_u))
        return report_error(PYRONN_ERROR_INVALID_ARGUMENT,
                            "%s: detector spacings must be positive, SDD >= 0, the principal point finite", name);
    const cudaError_t e = launch_fdk_filter(projections, filtered, in_dtype, out_dtype, rows, det_h, det_w,
                                            (float)sdd, (float)det_spacing_v, (float)det_spacing_u,
                                            (float)principal_v, (float)principal_u, filter, weight_output ? 1 : 0,
                                            (cudaStream_t)stream);
    if (e != cudaSuccess) return report_cuda_error(e, name);
    return PYRONN_SUCCESS;
}

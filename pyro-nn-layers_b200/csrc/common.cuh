// common.cuh -- device helpers shared by the projector kernels.
//
// Storage types: float, __nv_bfloat16 and __half are loaded through the
// read-only path and widened to FP32; every sum is FP32.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyronn {

template <typename T>
__device__ __forceinline__ float load_as_float(const T *p);

template <>
__device__ __forceinline__ float load_as_float<float>(const float *p)
{
    return __ldg(p);
}

template <>
__device__ __forceinline__ float load_as_float<__nv_bfloat16>(const __nv_bfloat16 *p)
{
    return __bfloat162float(__ldg(p));
}

template <>
__device__ __forceinline__ float load_as_float<__half>(const __half *p)
{
    return __half2float(__ldg(p));
}

template <typename T>
__device__ __forceinline__ void store_from_float(T *p, float v);

template <>
__device__ __forceinline__ void store_from_float<float>(float *p, float v)
{
    *p = v;
}

template <>
__device__ __forceinline__ void store_from_float<__nv_bfloat16>(__nv_bfloat16 *p, float v)
{
    *p = __float2bfloat16_rn(v);
}

template <>
__device__ __forceinline__ void store_from_float<__half>(__half *p, float v)
{
    *p = __float2half_rn(v);
}

// Linear interpolation in the reference's FMA form,
// a * (1 - t) + b * t == fma(b, t, fma(a, -t, a))
// (cone_projector_3D_CudaKernel.cu.cc:74-82 uses the same expression).
__device__ __forceinline__ float lerp_ref(float a, float b, float t)
{
    return __fmaf_rn(b, t, __fmaf_rn(a, -t, a));
}

// f32(h) - c for the 16-bit value h in the low (HI = false) or high half of
// w: one mixed-precision instruction (PTX sub.f32.f16 / sub.f32.bf16, sm_100)
// in place of a widening conversion and an FP32 subtraction (same result
// up to FP32 subnormals, which this form does not flush).
template <bool HI>
__device__ __forceinline__ float sub_f32_f16(unsigned w, float c)
{
    float d;
    if (HI)
        asm("{.reg .b16 lo, hi; mov.b32 {lo, hi}, %1; sub.f32.f16 %0, hi, %2;}" : "=f"(d) : "r"(w), "f"(c));
    else
        asm("{.reg .b16 lo, hi; mov.b32 {lo, hi}, %1; sub.f32.f16 %0, lo, %2;}" : "=f"(d) : "r"(w), "f"(c));
    return d;
}
template <bool HI>
__device__ __forceinline__ float sub_f32_bf16(unsigned w, float c)
{
    float d;
    if (HI)
        asm("{.reg .b16 lo, hi; mov.b32 {lo, hi}, %1; sub.f32.bf16 %0, hi, %2;}" : "=f"(d) : "r"(w), "f"(c));
    else
        asm("{.reg .b16 lo, hi; mov.b32 {lo, hi}, %1; sub.f32.bf16 %0, lo, %2;}" : "=f"(d) : "r"(w), "f"(c));
    return d;
}

// The first-axis lerp of a storage type's taps, on values already widened to
// FP32: the reference's form for FP32 storage, a + t (b - a) for 16-bit
// storage -- the form the backprojectors and the 3D forward's direct and
// xy-mode paths compute with one mixed-precision subtraction (the forward's
// z-mode cells store half-differences instead: cone_fp_padded.cu).
template <typename T>
__device__ __forceinline__ float lerp_first(float a, float b, float t)
{
    return fmaf(t, b - a, a);
}
template <>
__device__ __forceinline__ float lerp_first<float>(float a, float b, float t)
{
    return lerp_ref(a, b, t);
}

template <typename T>
struct type_tag {
    using type = T;
};

// Calls f(type_tag<Tin>{}, type_tag<Tout>{}) for the storage types of the
// given pyronn_dtype_t codes (0 = float, 1 = bfloat16, 2 = half).
template <typename F>
cudaError_t dispatch_dtypes(int in_dtype, int out_dtype, F &&f)
{
    auto with_out = [&](auto tin) -> cudaError_t {
        switch (out_dtype) {
        case 0: return f(tin, type_tag<float>{});
        case 1: return f(tin, type_tag<__nv_bfloat16>{});
        case 2: return f(tin, type_tag<__half>{});
        default: return cudaErrorInvalidValue;
        }
    };
    switch (in_dtype) {
    case 0: return with_out(type_tag<float>{});
    case 1: return with_out(type_tag<__nv_bfloat16>{});
    case 2: return with_out(type_tag<__half>{});
    default: return cudaErrorInvalidValue;
    }
}

// floor and fraction without the conversion pipe: for |x| < 2^22,
// y = x + 1.5 * 2^23 rounded toward -inf lies in [2^23, 2^24), where the
// spacing of floats is 1, so y = 1.5 * 2^23 + floor(x) exactly and floor(x)
// is y's mantissa.  Three FADDs and an integer subtract instead of
// FRND + F2I; the fraction x - floor(x) is exact.
constexpr int FLOOR_BIAS = 0x4B400000;  // bit pattern of 1.5 * 2^23

struct FloorFrac {
    int i;     // floor(x)
    int bits;  // floor(x) + FLOOR_BIAS: callers that fold the bias elsewhere
    float f;   // x - floor(x), exact, in [0, 1)
};

__device__ __forceinline__ FloorFrac floor_frac(float x)
{
    const float magic = 12582912.0f;  // 1.5 * 2^23
    const float y = __fadd_rd(x, magic);
    FloorFrac r;
    r.bits = __float_as_int(y);
    r.i = r.bits - FLOOR_BIAS;
    r.f = __fadd_rn(x, -__fadd_rn(y, -magic));
    return r;
}

// Approximate reciprocal (one MUFU op, <= 1 ulp).
__device__ __forceinline__ float fast_rcp(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

}  // namespace pyronn

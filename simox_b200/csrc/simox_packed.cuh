// simox_packed.cuh -- packed FP32 arithmetic for the mixed-precision pair
// kernels on sm_100a.
//
// Blackwell issues FADD2 / FMUL2 / FFMA2: one instruction performs the same
// FP32 operation on two lanes of a register pair.  The pair kernels are bound
// by instruction issue, so each thread evaluates two list entries at once as
// the .x and .y halves of a v2 and every FP32 step of the pair function costs
// one issue slot for both.  Scalar coefficients are broadcast with bc(); the
// compiler feeds them from the constant bank without extra moves.
//
// The special functions are the hardware approximations (ex2.approx.ftz,
// rcp.approx.ftz, rsqrt.approx.ftz, PTX ISA), one per half.
#pragma once

#include <cuda_runtime.h>

namespace sx {

struct v2 {
    float2 v;
};

__device__ __forceinline__ v2 bc(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ v2 mk2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ v2 operator+(v2 a, v2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ v2 operator*(v2 a, v2 b) { return {__fmul2_rn(a.v, b.v)}; }
__device__ __forceinline__ v2 fma2(v2 a, v2 b, v2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
// a - b as one FFMA2 (b * -1 is exact, so this is the correctly rounded difference)
__device__ __forceinline__ v2 operator-(v2 a, v2 b) { return {__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v)}; }

__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ v2 ex2(v2 a) { return mk2(ex2_approx(a.v.x), ex2_approx(a.v.y)); }
__device__ __forceinline__ v2 rcp(v2 a) { return mk2(rcp_approx(a.v.x), rcp_approx(a.v.y)); }
__device__ __forceinline__ v2 rsqrt(v2 a) { return mk2(rsqrt_approx(a.v.x), rsqrt_approx(a.v.y)); }

// Compensated accumulation hi + lo += b (Knuth's TwoSum, exact error term).
__device__ __forceinline__ void two_sum2(v2& hi, v2& lo, v2 b) {
    const v2 s = hi + b;
    const v2 bp = s - hi;
    const v2 ap = s - bp;
    lo = lo + ((hi - ap) + (b - bp));
    hi = s;
}

// erfc(z) = t P(t) exp(-z^2), t = 1 / (1 + kErfcP z), z >= 0.  P is a degree-7
// polynomial fitted for this library (Lawson-iterated weighted least squares
// on 800 Chebyshev nodes of t, minimising the relative error of erfc) to
// scipy's erfcx(z)/t for z in [0, 4.5]: in exact arithmetic its relative error
// is below 4.2e-8 there; FP32 evaluation of t and P stays below 4e-7.  The
// Ewald pair term needs exp(-z^2) anyway, so erfc costs one reciprocal and
// seven FFMA on top of it.
constexpr float kErfcP = 0.4f;
__device__ __forceinline__ v2 erfc_poly(v2 t) {
    v2 p = fma2(t, bc(7.540615346e-02f), bc(-4.006163492e-01f));
    p = fma2(p, t, bc(6.982889910e-01f));
    p = fma2(p, t, bc(-3.912853263e-01f));
    p = fma2(p, t, bc(4.214142199e-01f));
    p = fma2(p, t, bc(1.342951894e-01f));
    p = fma2(p, t, bc(2.376611896e-01f));
    p = fma2(p, t, bc(2.248358903e-01f));
    return p;
}

// Per-thread asynchronous copies global -> shared (cp.async, PTX ISA): the
// partner records of later batches are in flight while a batch is computed,
// without holding registers.
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

}  // namespace sx

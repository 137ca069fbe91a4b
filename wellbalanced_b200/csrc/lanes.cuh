// Lane types of the float32 face arithmetic.
//
// `F2` holds two independent float32 lanes (the left and right states of a face, or two
// components) and advances them with the packed float32 instructions of sm_100 (add /
// sub / mul / fma on .f32x2: one instruction for both lanes). Comparisons give a lane
// mask `M2`; selects, min / max, absolute values and the special functions act on each
// lane.
//
// `L1` is one float32 lane with the same rounding: every add, subtract and multiply is
// rounded on its own (no implicit contraction into FMA) and every fused multiply-add is
// written as `fma`, so a value has the same bits in a lane of F2 and in L1, and the
// kernels that form the same face (the stage kernels, the refluxing kernel) agree on it.
#pragma once

#include <cuda_runtime.h>

namespace wb {

struct L1 {
  float v;
  L1() = default;
  __device__ __forceinline__ L1(float a) : v(a) {}
};

__device__ __forceinline__ L1 operator+(L1 a, L1 b) { return L1(__fadd_rn(a.v, b.v)); }
__device__ __forceinline__ L1 operator-(L1 a, L1 b) { return L1(__fsub_rn(a.v, b.v)); }
__device__ __forceinline__ L1 operator*(L1 a, L1 b) { return L1(__fmul_rn(a.v, b.v)); }
__device__ __forceinline__ L1 fma(L1 a, L1 b, L1 c) { return L1(__fmaf_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ bool operator>(L1 a, L1 b) { return a.v > b.v; }
__device__ __forceinline__ bool operator>=(L1 a, L1 b) { return a.v >= b.v; }
__device__ __forceinline__ bool operator<(L1 a, L1 b) { return a.v < b.v; }
__device__ __forceinline__ bool operator<=(L1 a, L1 b) { return a.v <= b.v; }
__device__ __forceinline__ L1 sel(bool m, L1 a, L1 b) { return m ? a : b; }
__device__ __forceinline__ L1 labs(L1 a) { return L1(fabsf(a.v)); }
__device__ __forceinline__ L1 lmin(L1 a, L1 b) { return L1(fminf(a.v, b.v)); }
__device__ __forceinline__ L1 lmax(L1 a, L1 b) { return L1(fmaxf(a.v, b.v)); }
__device__ __forceinline__ L1 lcopysign(L1 m, L1 s) { return L1(copysignf(m.v, s.v)); }
// reciprocal and reciprocal square root from the special-function unit (~1 ulp)
__device__ __forceinline__ L1 linv(L1 a) { return L1(__fdividef(1.0f, a.v)); }
__device__ __forceinline__ L1 lrsqrt(L1 a) { return L1(rsqrtf(a.v)); }
__device__ __forceinline__ bool any(bool m) { return m; }

struct M2 {
  bool x, y;
};
__device__ __forceinline__ M2 operator|(M2 a, M2 b) { return {a.x || b.x, a.y || b.y}; }
__device__ __forceinline__ M2 operator&(M2 a, M2 b) { return {a.x && b.x, a.y && b.y}; }
__device__ __forceinline__ M2 operator^(M2 a, M2 b) { return {a.x != b.x, a.y != b.y}; }
__device__ __forceinline__ M2 operator!(M2 a) { return {!a.x, !a.y}; }
__device__ __forceinline__ bool any(M2 m) { return m.x || m.y; }

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float a) : v(make_float2(a, a)) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ explicit F2(float2 a) : v(a) {}
};

__device__ __forceinline__ unsigned long long f2_bits(F2 a) {
  unsigned long long u;
  asm("mov.b64 %0, {%1, %2};" : "=l"(u) : "f"(a.v.x), "f"(a.v.y));
  return u;
}
__device__ __forceinline__ F2 f2_from_bits(unsigned long long u) {
  float x, y;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(u));
  return F2(x, y);
}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_bits(a)), "l"(f2_bits(b)));
  return f2_from_bits(d);
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
__device__ __forceinline__ M2 operator>(F2 a, F2 b) { return {a.v.x > b.v.x, a.v.y > b.v.y}; }
__device__ __forceinline__ M2 operator>=(F2 a, F2 b) { return {a.v.x >= b.v.x, a.v.y >= b.v.y}; }
__device__ __forceinline__ M2 operator<(F2 a, F2 b) { return {a.v.x < b.v.x, a.v.y < b.v.y}; }
__device__ __forceinline__ M2 operator<=(F2 a, F2 b) { return {a.v.x <= b.v.x, a.v.y <= b.v.y}; }
__device__ __forceinline__ F2 sel(M2 m, F2 a, F2 b) { return F2(m.x ? a.v.x : b.v.x, m.y ? a.v.y : b.v.y); }
__device__ __forceinline__ F2 labs(F2 a) { return F2(fabsf(a.v.x), fabsf(a.v.y)); }
__device__ __forceinline__ F2 lmin(F2 a, F2 b) { return F2(fminf(a.v.x, b.v.x), fminf(a.v.y, b.v.y)); }
__device__ __forceinline__ F2 lmax(F2 a, F2 b) { return F2(fmaxf(a.v.x, b.v.x), fmaxf(a.v.y, b.v.y)); }
__device__ __forceinline__ F2 lcopysign(F2 m, F2 s) { return F2(copysignf(m.v.x, s.v.x), copysignf(m.v.y, s.v.y)); }
__device__ __forceinline__ F2 linv(F2 a) { return F2(__fdividef(1.0f, a.v.x), __fdividef(1.0f, a.v.y)); }
__device__ __forceinline__ F2 lrsqrt(F2 a) { return F2(rsqrtf(a.v.x), rsqrtf(a.v.y)); }
// 0 - a (a negation for the packed type, kept identical in both lane types)
template <typename V>
__device__ __forceinline__ V lneg(V a) {
  return V(0.0f) - a;
}

}  // namespace wb

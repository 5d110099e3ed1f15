// Explicit-rounding arithmetic for the fused collisions, on one cell (F1) or
// on the two cells of a pair (F2, sm_100a packed float32).
//
// The pair kernels hold cells x and x + 1 of a row in one thread and apply
// the same operation sequence to both.  F2 holds the two cells' values of one
// quantity in a register pair, and its operators issue the packed float32
// instructions of sm_100a (fma.rn.f32x2, add.rn.f32x2, mul.rn.f32x2 through
// __ffma2_rn / __fadd2_rn / __fmul2_rn): one instruction does the operation
// for both cells, rounded per component exactly as the scalar instruction
// would.  Division, square root and the reciprocal have no packed form and run
// per component.
//
// A product a * b is kept unevaluated (a P value) until it meets an addition
// or a subtraction, where it becomes one fused multiply-add: the intrinsics are
// never contracted by the compiler, so the contraction of a scalar expression
// like a * b + c is made by the types.  Chains such as c0 * e0 + c1 * e1 +
// c2 * e2 become one multiply and two fused multiply-adds.
//
// F1 is the same type on one cell, with the scalar round-to-nearest
// intrinsics.  The single-cell kernels run the fused collisions on F1, so a
// cell gets bit for bit the same result whether a pair kernel or a
// single-cell kernel (the collide-only pass, the batched runner, the odd-nx
// fallback, the first AA step) updates it.
#pragma once

#include <type_traits>

#include <cuda_runtime.h>

// 1 / x as the IEEE division by default.  The hardware approximation
// (rcp.approx.ftz.f32, TLBM_FAST_RCP=1) saves a few instructions per cell, but
// with it the forced 512^3 MRT turbulence (constant-power linear forcing,
// tau 0.523) turned non-finite after about 950 steps, where the IEEE form
// runs its full 15-turnover spin-up.
#ifndef TLBM_FAST_RCP
#define TLBM_FAST_RCP 0
#endif

namespace tlbm {
// The types and their functions live in a namespace of their own: calls from
// the generic collision code find them by argument-dependent lookup, and they
// do not hide the scalar sqrt / fma of the global namespace.
namespace pk {

// 1 / x: the IEEE division, or with TLBM_FAST_RCP the hardware approximation
// (rcp.approx.ftz.f32, within 1 ulp)
__device__ __forceinline__ float rcp_approx(float x) {
#if TLBM_FAST_RCP
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
#else
  return 1.0f / x;
#endif
}

// the operations on one lane type: float (one cell) or float2 (two cells)
template <class V> struct Lane;
template <> struct Lane<float> {
  __host__ __device__ static constexpr float bcast(float c) { return c; }
  __device__ __forceinline__ static float mul(float a, float b) { return __fmul_rn(a, b); }
  __device__ __forceinline__ static float add(float a, float b) { return __fadd_rn(a, b); }
  __device__ __forceinline__ static float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  __device__ __forceinline__ static float neg(float a) { return -a; }
  __device__ __forceinline__ static float div(float a, float b) { return a / b; }
  __device__ __forceinline__ static float xdiv(float a, float b) { return __fdiv_rn(a, b); }
  __device__ __forceinline__ static float sqrt(float a) { return sqrtf(a); }
  __device__ __forceinline__ static float rcp(float a) { return rcp_approx(a); }
  __device__ __forceinline__ static float max(float a, float b) { return fmaxf(a, b); }
  __device__ __forceinline__ static float min(float a, float b) { return fminf(a, b); }
};
template <> struct Lane<float2> {
  __host__ __device__ static constexpr float2 bcast(float c) { return float2{c, c}; }
  __device__ __forceinline__ static float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
  __device__ __forceinline__ static float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
  __device__ __forceinline__ static float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
  __device__ __forceinline__ static float2 neg(float2 a) { return make_float2(-a.x, -a.y); }
  __device__ __forceinline__ static float2 div(float2 a, float2 b) { return make_float2(a.x / b.x, a.y / b.y); }
  __device__ __forceinline__ static float2 xdiv(float2 a, float2 b) {
    return make_float2(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y));
  }
  __device__ __forceinline__ static float2 sqrt(float2 a) { return make_float2(sqrtf(a.x), sqrtf(a.y)); }
  __device__ __forceinline__ static float2 rcp(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
  __device__ __forceinline__ static float2 max(float2 a, float2 b) {
    return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y));
  }
  __device__ __forceinline__ static float2 min(float2 a, float2 b) {
    return make_float2(fminf(a.x, b.x), fminf(a.y, b.y));
  }
};

template <class V> struct PV;

template <class V> struct FV {
  using Ln = Lane<V>;
  V v;
  FV() = default;
  __host__ __device__ __forceinline__ constexpr FV(V a) : v(a) {}
  // a scalar value broadcast to every lane (constants, uniform parameters)
  __host__ __device__ __forceinline__ explicit constexpr FV(double c) : v(Ln::bcast(float(c))) {}
  template <class W = V, typename std::enable_if<std::is_same<W, float2>::value, int>::type = 0>
  __host__ __device__ __forceinline__ explicit constexpr FV(float c) : v(Ln::bcast(c)) {}
  __host__ __device__ __forceinline__ explicit constexpr FV(int c) : v(Ln::bcast(float(c))) {}
  // the two cells of a pair
  template <class W = V, typename std::enable_if<std::is_same<W, float2>::value, int>::type = 0>
  __host__ __device__ __forceinline__ constexpr FV(float a, float b) : v{a, b} {}
  __device__ __forceinline__ FV(const PV<V>& p) : v(Ln::mul(p.x, p.y)) {}
  template <class W = V, typename std::enable_if<std::is_same<W, float2>::value, int>::type = 0>
  __host__ __device__ __forceinline__ float a() const { return v.x; }
  template <class W = V, typename std::enable_if<std::is_same<W, float2>::value, int>::type = 0>
  __host__ __device__ __forceinline__ float b() const { return v.y; }
};

// an unevaluated product x * y
template <class V> struct PV {
  V x, y;
};

using F1 = FV<float>;
using F2 = FV<float2>;
using P1 = PV<float>;
using P2 = PV<float2>;

template <class V> __device__ __forceinline__ PV<V> operator*(FV<V> a, FV<V> b) { return {a.v, b.v}; }
template <class V> __device__ __forceinline__ PV<V> operator*(const PV<V>& a, FV<V> b) { return {FV<V>(a).v, b.v}; }
template <class V> __device__ __forceinline__ PV<V> operator*(FV<V> a, const PV<V>& b) { return {a.v, FV<V>(b).v}; }
template <class V> __device__ __forceinline__ PV<V> operator*(const PV<V>& a, const PV<V>& b) {
  return {FV<V>(a).v, FV<V>(b).v};
}

template <class V> __device__ __forceinline__ FV<V> operator+(FV<V> a, FV<V> b) { return Lane<V>::add(a.v, b.v); }
template <class V> __device__ __forceinline__ FV<V> operator+(const PV<V>& p, FV<V> c) {
  return Lane<V>::fma(p.x, p.y, c.v);
}
template <class V> __device__ __forceinline__ FV<V> operator+(FV<V> c, const PV<V>& p) {
  return Lane<V>::fma(p.x, p.y, c.v);
}
template <class V> __device__ __forceinline__ FV<V> operator+(const PV<V>& p, const PV<V>& q) {
  return Lane<V>::fma(p.x, p.y, FV<V>(q).v);
}

// a - b as a + b * (-1): one instruction, exact like the subtraction
template <class V> __device__ __forceinline__ FV<V> operator-(FV<V> a, FV<V> b) {
  return Lane<V>::fma(b.v, Lane<V>::bcast(-1.0f), a.v);
}
template <class V> __device__ __forceinline__ FV<V> operator-(FV<V> c, const PV<V>& p) {
  return Lane<V>::fma(Lane<V>::neg(p.x), p.y, c.v);
}
template <class V> __device__ __forceinline__ FV<V> operator-(const PV<V>& p, FV<V> c) {
  return Lane<V>::fma(p.x, p.y, Lane<V>::neg(c.v));
}
template <class V> __device__ __forceinline__ FV<V> operator-(const PV<V>& p, const PV<V>& q) {
  return Lane<V>::fma(Lane<V>::neg(q.x), q.y, FV<V>(p).v);
}

template <class V> __device__ __forceinline__ FV<V> operator-(FV<V> a) {
  return Lane<V>::mul(a.v, Lane<V>::bcast(-1.0f));
}
template <class V> __device__ __forceinline__ PV<V> operator-(const PV<V>& p) { return {Lane<V>::neg(p.x), p.y}; }

template <class V> __device__ __forceinline__ FV<V> operator/(FV<V> a, FV<V> b) { return Lane<V>::div(a.v, b.v); }
template <class V> __device__ __forceinline__ FV<V> operator/(const PV<V>& a, FV<V> b) { return FV<V>(a) / b; }

template <class V> __device__ __forceinline__ FV<V>& operator+=(FV<V>& a, FV<V> b) { return a = a + b; }
template <class V> __device__ __forceinline__ FV<V>& operator+=(FV<V>& a, const PV<V>& p) { return a = a + p; }
template <class V> __device__ __forceinline__ FV<V>& operator-=(FV<V>& a, FV<V> b) { return a = a - b; }
template <class V> __device__ __forceinline__ FV<V>& operator-=(FV<V>& a, const PV<V>& p) { return a = a - p; }
template <class V> __device__ __forceinline__ FV<V>& operator*=(FV<V>& a, FV<V> b) { return a = FV<V>(a * b); }

// the lane type of an operand (FV or PV); no member for other types, so the
// fma below takes part only where an operand is one of these types
template <class T> struct LaneOf {};
template <class V> struct LaneOf<FV<V>> { using type = V; };
template <class V> struct LaneOf<PV<V>> { using type = V; };

// fma with any operand an unevaluated product: the product is rounded first,
// as the scalar code rounds a * b before the fused multiply-add that takes it
template <class A, class B, class C, class V = typename LaneOf<A>::type>
__device__ __forceinline__ FV<V> fma(const A& a, const B& b, const C& c) {
  return Lane<V>::fma(FV<V>(a).v, FV<V>(b).v, FV<V>(c).v);
}
template <class V> __device__ __forceinline__ FV<V> sqrt(FV<V> a) { return Lane<V>::sqrt(a.v); }
// the fast reciprocal of tlbm_collide.cuh, per lane
template <class V> __device__ __forceinline__ FV<V> rcp_fast(FV<V> a) { return Lane<V>::rcp(a.v); }

// per-lane max / min against a bound (the clamps of the collisions)
template <class V> __device__ __forceinline__ FV<V> clamp_lo(FV<V> a, FV<V> lo) { return Lane<V>::max(a.v, lo.v); }
template <class V> __device__ __forceinline__ FV<V> clamp_hi(FV<V> a, FV<V> hi) { return Lane<V>::min(a.v, hi.v); }

// reference-rounded operations (no contraction), per lane as __f*_rn
template <class V> __device__ __forceinline__ FV<V> xadd(FV<V> a, FV<V> b) { return Lane<V>::add(a.v, b.v); }
template <class V> __device__ __forceinline__ FV<V> xsub(FV<V> a, FV<V> b) {
  return Lane<V>::fma(b.v, Lane<V>::bcast(-1.0f), a.v);
}
template <class V> __device__ __forceinline__ FV<V> xmul(FV<V> a, FV<V> b) { return Lane<V>::mul(a.v, b.v); }
template <class V> __device__ __forceinline__ FV<V> xdiv(FV<V> a, FV<V> b) { return Lane<V>::xdiv(a.v, b.v); }

}  // namespace pk

using pk::F1;
using pk::F2;
using pk::P1;
using pk::P2;

}  // namespace tlbm

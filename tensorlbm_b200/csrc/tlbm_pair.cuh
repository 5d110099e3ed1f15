// Packed arithmetic on the two cells of a pair (sm_100a).
//
// The pair kernels hold cells x and x + 1 of a row in one thread and apply
// the same operation sequence to both.  F2 holds the two cells' values of one
// quantity in a register pair, and its operators issue the packed float32
// instructions of sm_100a (fma.rn.f32x2, add.rn.f32x2, mul.rn.f32x2 through
// __ffma2_rn / __fadd2_rn / __fmul2_rn): one instruction does the operation
// for both cells, rounded per component exactly as the scalar instruction
// would.  Division and square root have no packed form and run per component.
//
// A product a * b is kept unevaluated (P2) until it meets an addition or a
// subtraction, where it becomes one fused multiply-add: the packed intrinsics
// are never contracted by the compiler, so the contraction of a scalar
// expression like a * b + c is reproduced here by the types.  Chains such as
// c0 * e0 + c1 * e1 + c2 * e2 become one multiply and two fused multiply-adds.
#pragma once

#include <cuda_runtime.h>

namespace tlbm {

struct P2;

struct F2 {
  float2 v;
  F2() = default;
  __host__ __device__ __forceinline__ constexpr F2(float2 a) : v(a) {}
  __host__ __device__ __forceinline__ constexpr F2(float a, float b) : v{a, b} {}
  // a scalar value broadcast to both cells (constants, uniform parameters)
  __host__ __device__ __forceinline__ constexpr F2(double c) : v{float(c), float(c)} {}
  __host__ __device__ __forceinline__ constexpr F2(float c) : v{c, c} {}
  __host__ __device__ __forceinline__ constexpr F2(int c) : v{float(c), float(c)} {}
  __device__ __forceinline__ F2(const P2& p);
  __host__ __device__ __forceinline__ float a() const { return v.x; }
  __host__ __device__ __forceinline__ float b() const { return v.y; }
};

// an unevaluated product x * y
struct P2 {
  float2 x, y;
};

__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ F2::F2(const P2& p) : v(__fmul2_rn(p.x, p.y)) {}

__device__ __forceinline__ P2 operator*(F2 a, F2 b) { return {a.v, b.v}; }
__device__ __forceinline__ P2 operator*(const P2& a, F2 b) { return {F2(a).v, b.v}; }
__device__ __forceinline__ P2 operator*(F2 a, const P2& b) { return {a.v, F2(b).v}; }
__device__ __forceinline__ P2 operator*(const P2& a, const P2& b) { return {F2(a).v, F2(b).v}; }

__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return __fadd2_rn(a.v, b.v); }
__device__ __forceinline__ F2 operator+(const P2& p, F2 c) { return __ffma2_rn(p.x, p.y, c.v); }
__device__ __forceinline__ F2 operator+(F2 c, const P2& p) { return __ffma2_rn(p.x, p.y, c.v); }
__device__ __forceinline__ F2 operator+(const P2& p, const P2& q) { return __ffma2_rn(p.x, p.y, F2(q).v); }

// a - b as a + b * (-1): one instruction, exact like the scalar subtraction
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return __ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v); }
__device__ __forceinline__ F2 operator-(F2 c, const P2& p) { return __ffma2_rn(neg2(p.x), p.y, c.v); }
__device__ __forceinline__ F2 operator-(const P2& p, F2 c) { return __ffma2_rn(p.x, p.y, neg2(c.v)); }
__device__ __forceinline__ F2 operator-(const P2& p, const P2& q) { return __ffma2_rn(neg2(q.x), q.y, F2(p).v); }

__device__ __forceinline__ F2 operator-(F2 a) { return __fmul2_rn(a.v, make_float2(-1.0f, -1.0f)); }
__device__ __forceinline__ P2 operator-(const P2& p) { return {neg2(p.x), p.y}; }

__device__ __forceinline__ F2 operator/(F2 a, F2 b) { return F2(a.v.x / b.v.x, a.v.y / b.v.y); }
__device__ __forceinline__ F2 operator/(const P2& a, F2 b) { return F2(a) / b; }

__device__ __forceinline__ F2& operator+=(F2& a, F2 b) { return a = a + b; }
__device__ __forceinline__ F2& operator+=(F2& a, const P2& p) { return a = a + p; }
__device__ __forceinline__ F2& operator-=(F2& a, F2 b) { return a = a - b; }
__device__ __forceinline__ F2& operator-=(F2& a, const P2& p) { return a = a - p; }
__device__ __forceinline__ F2& operator*=(F2& a, F2 b) { return a = F2(a * b); }

__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return __ffma2_rn(a.v, b.v, c.v); }
__device__ __forceinline__ F2 sqrt(F2 a) { return F2(sqrtf(a.v.x), sqrtf(a.v.y)); }

// per-component max / min against a bound (the clamps of the collisions)
__device__ __forceinline__ F2 clamp_lo(F2 a, F2 lo) { return F2(fmaxf(a.v.x, lo.v.x), fmaxf(a.v.y, lo.v.y)); }
__device__ __forceinline__ F2 clamp_hi(F2 a, F2 hi) { return F2(fminf(a.v.x, hi.v.x), fminf(a.v.y, hi.v.y)); }

// reference-rounded operations (no contraction), per component as __f*_rn
__device__ __forceinline__ F2 xadd(F2 a, F2 b) { return __fadd2_rn(a.v, b.v); }
__device__ __forceinline__ F2 xsub(F2 a, F2 b) { return __ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v); }
__device__ __forceinline__ F2 xmul(F2 a, F2 b) { return __fmul2_rn(a.v, b.v); }
__device__ __forceinline__ F2 xdiv(F2 a, F2 b) { return F2(__fdiv_rn(a.v.x, b.v.x), __fdiv_rn(a.v.y, b.v.y)); }

}  // namespace tlbm

// Per-cell collision operators on populations held in registers.
//
// Every function here takes the Q populations of ONE cell in a register array
// and overwrites them with the post-collision populations.  Loops over q are
// fully unrolled, so q (and every lattice constant looked up with it) is a
// compile-time constant: terms with a zero velocity component are never
// emitted, and no work depends on data layout.
#pragma once

#include "tlbm_common.cuh"
#include "tlbm_pair.cuh"

namespace tlbm {

template <typename T> struct CollideParams {
  T tau, inv_tau;
  double inv_tau64;         // RN64(1 / float(tau)) for the exact BGK quotient
  MrtRates<T> mrt;          // s_nu = 1/tau unless a tau field overrides it per cell
  T omega_b, omega_odd, omega_even;
  T c_smag;
  T smag_coef;              // 18.0 * C_s**2 (turbulence.py:206)
  T smag_coef_cum;          // 18.0 * C_s * C_s (cumulant.py:1352), rounded differently in double
  T omega_b_minus_omega;    // omega_b - 1/tau formed in double, as a python scalar
  T keep_even;              // 1 - omega_even
  T tau_sq;                 // tau^2
  T tau_eff_max;            // max(1, tau + 0.5), turbulence.py:88-99
  T force_a;                // linear body force F = A rho u (exact-difference forcing); 0 = none
  bool cum_unit_rates;      // omega_b = omega_odd = omega_even = 1 (D3Q27 legacy cumulant fast path)
  T cm_s5, cm_s6;           // cascaded D3Q27 5th / 6th-order rates (omega_odd, omega_even are s_3, s_4)
  T tau_minus;              // TRT antisymmetric relaxation time
  double inv_tau_minus64;   // RN64(1 / float(tau_minus)) for the exact TRT quotient
  T rlbm_keep;              // 1 - 1/tau formed in float64 (regularised BGK)
};

// ---------------------------------------------------------------------------
// Reference-exact arithmetic.  TensorLBM evaluates its elementwise operators
// as separate torch kernels: every +, -, *, / is rounded on its own (no fused
// multiply-add) and divisions are IEEE divisions.  x* keep that rounding in
// device code (the compiler may not contract them), so the elementwise
// operators below reproduce the reference bit for bit.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// 1 / x for the fused-arithmetic collisions (no reference rounding order to
// keep): pk::rcp_approx (the IEEE division unless TLBM_FAST_RCP); float64
// keeps the division.
__device__ __forceinline__ float rcp_fast(float x) { return pk::rcp_approx(x); }
__device__ __forceinline__ double rcp_fast(double x) { return 1.0 / x; }

// a > lo ? a : lo and a < hi ? a : hi (F2 has per-component forms in tlbm_pair.cuh)
__device__ __forceinline__ float clamp_lo(float a, float lo) { return a > lo ? a : lo; }
__device__ __forceinline__ double clamp_lo(double a, double lo) { return a > lo ? a : lo; }
__device__ __forceinline__ float clamp_hi(float a, float hi) { return a < hi ? a : hi; }
__device__ __forceinline__ double clamp_hi(double a, double hi) { return a < hi ? a : hi; }

// sum of +-x, +-y, +-z terms for compile-time components a, b, c in {-1, 0, 1}
// (c_x u_x + c_y u_y + c_z u_z with exact integer products; only additions round)
template <typename T>
__device__ __forceinline__ T signed_sum(int a, int b, int c, T x, T y, T z) {
  T r = T(0);
  bool any = false;
  if (a != 0) { r = (a > 0) ? x : -x; any = true; }
  if (b != 0) { r = any ? ((b > 0) ? xadd(r, y) : xsub(r, y)) : ((b > 0) ? y : -y); any = true; }
  if (c != 0) { r = any ? ((c > 0) ? xadd(r, z) : xsub(r, z)) : ((c > 0) ? z : -z); any = true; }
  return r;
}

// torch's CPU sum over the direction axis of a (Q, ...) tensor accumulates
// directions 0..15 in order, directions 16..Q-1 in order, and adds the two
// partial sums (a 16-row cascade; measured bit for bit against torch 2.11).
// csum<L>(f, coeff) returns that sum of coeff(q) * f[q] for integer
// coefficients in {-1, 0, 1}; zero terms are skipped (adding a zero product
// does not change a non-zero sum).
template <class L, typename T, typename Coef>
__device__ __forceinline__ T csum(const T (&f)[L::Q], Coef coeff) {
  T head = T(0), tail = T(0);
  bool bh = false, bt = false;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    const int c = coeff(q);
    if (c == 0) continue;
    const T v = c > 0 ? f[q] : -f[q];
    if (q < 16) { head = bh ? xadd(head, v) : v; bh = true; }
    else { tail = bt ? xadd(tail, v) : v; bt = true; }
  }
  if (bh && bt) return xadd(tail, head);
  return bh ? head : tail;
}

struct OneCoef { __host__ __device__ constexpr int operator()(int) const { return 1; } };
template <class L> struct CxCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cx(q); } };
template <class L> struct CyCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cy(q); } };
template <class L> struct CzCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cz(q); } };

// rho = sum f, u = sum c f / max(rho, 1e-12): d2q9.py:61-74, d3q19.py:165-186,
// d3q27.py:395-420, in the reference's summation order and rounding.
template <class L, typename T>
__device__ __forceinline__ void macroscopic(const T (&f)[L::Q], T& rho, T& ux, T& uy, T& uz) {
  rho = csum<L>(f, OneCoef{});
  const T rs = rho > T(1e-12) ? rho : T(1e-12);
  ux = xdiv(csum<L>(f, CxCoef<L>{}), rs);
  uy = xdiv(csum<L>(f, CyCoef<L>{}), rs);
  uz = (L::DIM == 3) ? xdiv(csum<L>(f, CzCoef<L>{}), rs) : T(0);
}

// f_eq = w rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u.u): d2q9.py:39-58,
// d3q19.py:83-125, d3q27.py:353-392, evaluated as
// (w*rho) * (((1 + 3*cu) + (4.5*cu)*cu) - 1.5*usq), one rounding per operation.
template <class L, typename T>
__device__ __forceinline__ T usq_of(T ux, T uy, T uz) {
  return (L::DIM == 3) ? xadd(xadd(xmul(ux, ux), xmul(uy, uy)), xmul(uz, uz)) : xadd(xmul(ux, ux), xmul(uy, uy));
}

template <class L, typename T>
__device__ __forceinline__ T feq_q(int q, T rho, T ux, T uy, T uz, T usq) {
  const T wr = xmul(weight<L, T>(q), rho);
  if (L::cx(q) == 0 && L::cy(q) == 0 && L::cz(q) == 0) return xmul(wr, xsub(T(1), xmul(T(1.5), usq)));
  const T cu = signed_sum(L::cx(q), L::cy(q), L::cz(q), ux, uy, uz);
  const T inner = xsub(xadd(xadd(T(1), xmul(T(3), cu)), xmul(xmul(T(4.5), cu), cu)), xmul(T(1.5), usq));
  return xmul(wr, inner);
}

template <class L, typename T>
__device__ __forceinline__ void equilibrium(T rho, T ux, T uy, T uz, T (&fe)[L::Q]) {
  const T usq = usq_of<L>(ux, uy, uz);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fe[q] = feq_q<L>(q, rho, ux, uy, uz, usq);
}

// Correctly rounded a / b for a float32 divisor used many times, from one
// float64 reciprocal: RN32(RN64(a * RN64(1/b))).  The float64 product lies
// within 2^-52 (relative) of a/b.  A quotient of two float32 numbers is never
// a float32 rounding boundary (a boundary m has an odd 25-bit significand, so
// m*b cannot fit in 24 bits) and lies at least 2^-49 (relative) from every
// boundary, so the float64 product rounds to float32 exactly as a/b does.
// For float64 fields the division itself is used.
__device__ __forceinline__ float div_by(float a, float, double inv_b) { return __double2float_rn(__dmul_rn((double)a, inv_b)); }
__device__ __forceinline__ double div_by(double a, double b, double) { return __ddiv_rn(a, b); }

// Fused-arithmetic moments and equilibrium for the operators whose reference
// goes through BLAS matrix products (MRT, D3Q27 cumulants): same operators,
// rounding of a fused multiply-add pipeline, cheaper than the exact forms.
template <class L, typename T>
__device__ __forceinline__ void macroscopic_fused(const T (&f)[L::Q], T& rho, T& ux, T& uy, T& uz) {
  rho = f[0];
#pragma unroll
  for (int q = 1; q < L::Q; ++q) rho += f[q];
  T jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::cx(q) != 0) jx = (L::cx(q) > 0) ? jx + f[q] : jx - f[q];
    if (L::cy(q) != 0) jy = (L::cy(q) > 0) ? jy + f[q] : jy - f[q];
    if (L::cz(q) != 0) jz = (L::cz(q) > 0) ? jz + f[q] : jz - f[q];
  }
  const T ir = rcp_fast(clamp_lo(rho, T(1e-12)));
  ux = jx * ir;
  uy = jy * ir;
  uz = (L::DIM == 3) ? jz * ir : T(0);
}
template <class L, typename T>
__device__ __forceinline__ T feq_fused(int q, T rho, T ux, T uy, T uz, T usq) {
  const T wr = weight<L, T>(q) * rho;
  if (L::cx(q) == 0 && L::cy(q) == 0 && L::cz(q) == 0) return wr * (T(1) - T(1.5) * usq);
  T cu = T(0);
  if (L::cx(q) != 0) cu = (L::cx(q) > 0) ? cu + ux : cu - ux;
  if (L::cy(q) != 0) cu = (L::cy(q) > 0) ? cu + uy : cu - uy;
  if (L::cz(q) != 0) cu = (L::cz(q) > 0) ? cu + uz : cu - uz;
  return wr * (T(1) + cu * (T(3) + T(4.5) * cu) - T(1.5) * usq);
}
template <class L, typename T>
__device__ __forceinline__ T usq_fused(T ux, T uy, T uz) {
  return (L::DIM == 3) ? ux * ux + uy * uy + uz * uz : ux * ux + uy * uy;
}

// ---------------------------------------------------------------------------
// BGK: f - (f - feq)/tau (solver.py:67-71, solver3d.py:100-104, d3q27.py:423-437),
// bit-exact: (f - feq)/tau is the correctly rounded quotient, like torch's.
// ---------------------------------------------------------------------------
template <class L, typename T>
__device__ __forceinline__ void collide_bgk(T (&f)[L::Q], T tau, double inv_tau64) {
  T rho, ux, uy, uz;
  macroscopic<L>(f, rho, ux, uy, uz);
  const T usq = usq_of<L>(ux, uy, uz);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    const T fe = feq_q<L>(q, rho, ux, uy, uz, usq);
    f[q] = xsub(f[q], div_by(xsub(f[q], fe), tau, inv_tau64));
  }
}

// ---------------------------------------------------------------------------
// TRT (solver.py:440-486, solver3d.py:303-336, d3q27.py:438-480), bit-exact:
// f - (f+ - feq+)/tau_plus - (f- - feq-)/tau_minus with f+- = (f +- f_opp)/2
// formed one rounded operation at a time, like the torch expression.
// ---------------------------------------------------------------------------
template <class L, typename T>
__device__ __forceinline__ void collide_trt(T (&f)[L::Q], T tau_p, double inv_p64, T tau_m, double inv_m64) {
  T rho, ux, uy, uz;
  macroscopic<L>(f, rho, ux, uy, uz);
  const T usq = usq_of<L>(ux, uy, uz);
  T fe[L::Q], out[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fe[q] = feq_q<L>(q, rho, ux, uy, uz, usq);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    constexpr T half = T(0.5);
    const int o = L::opp(q);
    const T fp = xmul(half, xadd(f[q], f[o])), fm = xmul(half, xsub(f[q], f[o]));
    const T ep = xmul(half, xadd(fe[q], fe[o])), em = xmul(half, xsub(fe[q], fe[o]));
    out[q] = xsub(xsub(f[q], div_by(xsub(fp, ep), tau_p, inv_p64)), div_by(xsub(fm, em), tau_m, inv_m64));
  }
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = out[q];
}

// ---------------------------------------------------------------------------
// MRT: m* = m - S (m - m_eq), f = M^-1 m*  (solver.py:249-331, solver3d.py:107-160,
// d3q27.py:643-727), written as f -= M^-1 S M (f - feq) over the relaxed rows.
// ---------------------------------------------------------------------------
template <class L, typename T>
__device__ __forceinline__ void collide_mrt(T (&f)[L::Q], const MrtRates<T>& r) {
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fn[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fn[q] = f[q] - feq_fused<L>(q, rho, ux, uy, uz, usq);
  if constexpr (L::Q == 9) mrt_relax_d2q9<T>(f, fn, r);
  else if constexpr (L::Q == 19) mrt_relax_d3q19<T>(f, fn, r);
  else mrt_relax_d3q27<T>(f, fn, r);
}

// ---------------------------------------------------------------------------
// Second moment of the non-equilibrium part, Pi_ab = sum c_a c_b fneq
// ---------------------------------------------------------------------------
template <typename T> struct Pi6 { T xx, yy, zz, xy, xz, yz; };

template <class L> struct CxxCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cx(q) * L::cx(q); } };
template <class L> struct CyyCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cy(q) * L::cy(q); } };
template <class L> struct CzzCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cz(q) * L::cz(q); } };
template <class L> struct CxyCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cx(q) * L::cy(q); } };
template <class L> struct CxzCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cx(q) * L::cz(q); } };
template <class L> struct CyzCoef { __host__ __device__ constexpr int operator()(int q) const { return L::cy(q) * L::cz(q); } };

// (c_a c_b * fneq).sum(0) in the reference's summation order
template <class L, typename T>
__device__ __forceinline__ Pi6<T> neq_stress(const T (&fn)[L::Q]) {
  Pi6<T> p;
  p.xx = csum<L>(fn, CxxCoef<L>{});
  p.yy = csum<L>(fn, CyyCoef<L>{});
  p.xy = csum<L>(fn, CxyCoef<L>{});
  if constexpr (L::DIM == 3) {
    p.zz = csum<L>(fn, CzzCoef<L>{});
    p.xz = csum<L>(fn, CxzCoef<L>{});
    p.yz = csum<L>(fn, CyzCoef<L>{});
  } else {
    p.zz = p.xz = p.yz = T(0);
  }
  return p;
}

// |Pi|_F^2: pxx^2 + pyy^2 [+ pzz^2] + 2 (pxy^2 [+ pxz^2 + pyz^2])
template <class L, typename T>
__device__ __forceinline__ T stress_radicand(const Pi6<T>& p) {
  if constexpr (L::DIM == 3) {
    const T diag = xadd(xadd(xmul(p.xx, p.xx), xmul(p.yy, p.yy)), xmul(p.zz, p.zz));
    const T off = xadd(xadd(xmul(p.xy, p.xy), xmul(p.xz, p.xz)), xmul(p.yz, p.yz));
    return xadd(diag, xmul(T(2), off));
  } else {
    return xadd(xadd(xmul(p.xx, p.xx), xmul(p.yy, p.yy)), xmul(T(2), xmul(p.xy, p.xy)));
  }
}

// Hou-1994 tau_eff with the clamps of turbulence.py:183-208 (norm clamp of
// :128-140 / :170-181).
template <class L, typename T>
__device__ __forceinline__ T smagorinsky_tau(const Pi6<T>& p, T rho, const CollideParams<T>& cp) {
  T rad = stress_radicand<L>(p);
  rad = rad > T(1e-30) ? rad : T(1e-30);
  const T pi_norm = sqrt(rad);
  const T rs = rho > T(1e-12) ? rho : T(1e-12);
  T disc = xadd(cp.tau_sq, xdiv(xmul(cp.smag_coef, pi_norm), rs));
  disc = disc > T(0) ? disc : T(0);
  T te = xmul(T(0.5), xadd(cp.tau, sqrt(disc)));
  te = te < T(0.5001) ? T(0.5001) : te;
  te = te > cp.tau_eff_max ? cp.tau_eff_max : te;
  return te;
}

// BGK with per-cell Smagorinsky tau_eff, f - f_neq / tau_eff:
// turbulence.py:216-230 (D2Q9), :245-261 (D3Q19), :472-494 (D3Q27).
template <class L, typename T>
__device__ __forceinline__ void collide_smagorinsky(T (&f)[L::Q], const CollideParams<T>& cp) {
  T rho, ux, uy, uz;
  macroscopic<L>(f, rho, ux, uy, uz);
  const T usq = usq_of<L>(ux, uy, uz);
  T fn[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) fn[q] = xsub(f[q], feq_q<L>(q, rho, ux, uy, uz, usq));
  const Pi6<T> p = neq_stress<L>(fn);
  const T te = smagorinsky_tau<L>(p, rho, cp);
  const double inv_te = 1.0 / double(te);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = xsub(f[q], div_by(fn[q], te, inv_te));
}

// ---------------------------------------------------------------------------
// D3Q19 "cumulant": Hermite-regularised relaxation of the stress with a
// separate bulk rate and a damped higher-order remainder (cumulant.py:1159-1420),
// with the reference's evaluation order.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T hermite_contract(int a, int b, int c, T hxx, T hyy, T hzz, const Pi6<T>& s) {
  // h_xx s_xx + h_yy s_yy + h_zz s_zz + (2 h_xy) s_xy + (2 h_xz) s_xz + (2 h_yz) s_yz
  T r = xadd(xadd(xmul(hxx, s.xx), xmul(hyy, s.yy)), xmul(hzz, s.zz));
  if (a * b != 0) r = xadd(r, xmul(T(2 * a * b), s.xy));
  if (a * c != 0) r = xadd(r, xmul(T(2 * a * c), s.xz));
  if (b * c != 0) r = xadd(r, xmul(T(2 * b * c), s.yz));
  return r;
}

// ---------------------------------------------------------------------------
// Regularised BGK, Latt & Chopard 2006 (solver.py:338-392, solver3d.py:342-403,
// d3q27.py:481-540), bit-exact: Pi = sum c c (f - feq) in the reference's
// summation order, then per direction
//   f = feq + keep * ((4.5 w) * (h_xx Pi_xx + h_yy Pi_yy [+ h_zz Pi_zz]
//                                + (2 h_xy) Pi_xy [+ (2 h_xz) Pi_xz + (2 h_yz) Pi_yz]))
// with h_aa = c_a^2 - 1/3, h_ab = c_a c_b and keep = 1 - 1/tau (formed in
// float64, a Python scalar there), every operation rounded on its own.  The
// weights of the projection are the float32 ones for every field dtype (the
// reference's _w_on default, d3q19.py:75-80, d3q27.py:345-350), while the
// equilibrium keeps weight<L, T>.  A zero h_ab term is skipped: adding the
// zero product does not change the sum.
// ---------------------------------------------------------------------------
template <class L, typename T>
__device__ __forceinline__ void collide_rlbm(T (&f)[L::Q], T keep) {
  T rho, ux, uy, uz;
  macroscopic<L>(f, rho, ux, uy, uz);
  const T usq = usq_of<L>(ux, uy, uz);
  T fe[L::Q], fn[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    fe[q] = feq_q<L>(q, rho, ux, uy, uz, usq);
    fn[q] = xsub(f[q], fe[q]);
  }
  const Pi6<T> p = neq_stress<L>(fn);
  const T cs2 = T(1.0 / 3.0);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    const int a = L::cx(q), b = L::cy(q), c = L::cz(q);
    const T hxx = xsub(T(a * a), cs2), hyy = xsub(T(b * b), cs2);
    T r;
    if constexpr (L::DIM == 3) {
      r = hermite_contract(a, b, c, hxx, hyy, xsub(T(c * c), cs2), p);
    } else {
      r = xadd(xmul(hxx, p.xx), xmul(hyy, p.yy));
      if (a * b != 0) r = xadd(r, xmul(T(2 * a * b), p.xy));
    }
    f[q] = xadd(fe[q], xmul(keep, xmul(xmul(T(4.5), T(float(L::w(q)))), r)));
  }
}

template <typename T>
__device__ __forceinline__ void collide_cumulant_d3q19(T (&f)[19], const CollideParams<T>& cp) {
  using L = D3Q19;
  T rho, ux, uy, uz;
  macroscopic<L>(f, rho, ux, uy, uz);
  const T usq = usq_of<L>(ux, uy, uz);
  T fe[19], fn[19];
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    fe[q] = feq_q<L>(q, rho, ux, uy, uz, usq);
    fn[q] = xsub(f[q], fe[q]);
  }
  const Pi6<T> p = neq_stress<L>(fn);
  T omega = cp.inv_tau;
  T omb_minus_om = cp.omega_b_minus_omega;
  if (cp.c_smag > T(0)) {
    // cumulant.py:1349-1353: no norm or tau clamps on this path
    const T pn = sqrt(stress_radicand<L>(p));
    const T rs = rho > T(1e-12) ? rho : T(1e-12);
    const T te = xmul(T(0.5), xadd(cp.tau, sqrt(xadd(cp.tau_sq, xdiv(xmul(cp.smag_coef_cum, pn), rs)))));
    omega = xdiv(T(1), te);
    omb_minus_om = xsub(cp.omega_b, omega);
  }
  const T tr = xadd(xadd(p.xx, p.yy), p.zz);
  const T bulk = xdiv(xmul(omb_minus_om, tr), T(3));
  Pi6<T> s;
  s.xx = xsub(xsub(p.xx, xmul(omega, p.xx)), bulk);
  s.yy = xsub(xsub(p.yy, xmul(omega, p.yy)), bulk);
  s.zz = xsub(xsub(p.zz, xmul(omega, p.zz)), bulk);
  s.xy = xsub(p.xy, xmul(omega, p.xy));
  s.xz = xsub(p.xz, xmul(omega, p.xz));
  s.yz = xsub(p.yz, xmul(omega, p.yz));
  const T cs2 = T(1.0 / 3.0);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    const int a = L::cx(q), b = L::cy(q), c = L::cz(q);
    const T hxx = xsub(T(a * a), cs2), hyy = xsub(T(b * b), cs2), hzz = xsub(T(c * c), cs2);
    const T w45 = xmul(T(4.5), weight<L, T>(q));
    const T reg = xmul(w45, hermite_contract(a, b, c, hxx, hyy, hzz, s));
    const T ho = xsub(fn[q], xmul(w45, hermite_contract(a, b, c, hxx, hyy, hzz, p)));
    f[q] = xadd(xadd(fe[q], reg), xmul(cp.keep_even, ho));
  }
}

// ---------------------------------------------------------------------------
// D3Q27 cumulant operators.  Moments live in a 3x3x3 array g[a][b][c] indexed
// by the exponents of cx^a cy^b cz^c; because D3Q27 is the full tensor
// product {-1,0,1}^3, the raw-moment transform M (cumulant.py:904-919) factors
// into three 1-D transforms, and the central shift (cumulant.py:390-457) is
// the 1-D binomial shift along each axis.
// ---------------------------------------------------------------------------
template <typename T> using Cube = T[3][3][3];

// populations -> g[ix][iy][iz] with i = c + 1
template <typename T>
__device__ __forceinline__ void to_cube(const T (&f)[27], Cube<T>& g) {
#pragma unroll
  for (int q = 0; q < 27; ++q) g[D3Q27::cx(q) + 1][D3Q27::cy(q) + 1][D3Q27::cz(q) + 1] = f[q];
}
template <typename T>
__device__ __forceinline__ void from_cube(const Cube<T>& g, T (&f)[27]) {
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = g[D3Q27::cx(q) + 1][D3Q27::cy(q) + 1][D3Q27::cz(q) + 1];
}

// element accessor along an axis: axis 0 -> g[i][j][k], 1 -> g[j][i][k], 2 -> g[j][k][i]
template <int AX, typename T>
__device__ __forceinline__ T& at(Cube<T>& g, int i, int j, int k) {
  if constexpr (AX == 0) return g[i][j][k];
  else if constexpr (AX == 1) return g[j][i][k];
  else return g[j][k][i];
}

// values at c = -1, 0, +1 -> moments of degree 0, 1, 2 along AX
template <int AX, typename T>
__device__ __forceinline__ void raw_1d(Cube<T>& g) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T vm = at<AX>(g, 0, j, k), v0 = at<AX>(g, 1, j, k), vp = at<AX>(g, 2, j, k);
      at<AX>(g, 0, j, k) = vm + v0 + vp;
      at<AX>(g, 1, j, k) = vp - vm;
      at<AX>(g, 2, j, k) = vp + vm;
    }
}
template <int AX, typename T>
__device__ __forceinline__ void pop_1d(Cube<T>& g) {
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T m0 = at<AX>(g, 0, j, k), m1 = at<AX>(g, 1, j, k), m2 = at<AX>(g, 2, j, k);
      at<AX>(g, 0, j, k) = (m2 - m1) * T(0.5);
      at<AX>(g, 1, j, k) = m0 - m2;
      at<AX>(g, 2, j, k) = (m1 + m2) * T(0.5);
    }
}
// forward binomial shift (cumulant.py:390-412) and its inverse (:415-434)
template <int AX, typename T>
__device__ __forceinline__ void shift_1d(Cube<T>& g, T u) {
  const T tu = T(2) * u, uu = u * u;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T m0 = at<AX>(g, 0, j, k), m1 = at<AX>(g, 1, j, k), m2 = at<AX>(g, 2, j, k);
      at<AX>(g, 1, j, k) = m1 - u * m0;
      at<AX>(g, 2, j, k) = m2 - tu * m1 + uu * m0;
    }
}
template <int AX, typename T>
__device__ __forceinline__ void unshift_1d(Cube<T>& g, T u) {
  const T tu = T(2) * u, uu = u * u;
#pragma unroll
  for (int j = 0; j < 3; ++j)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const T m0 = at<AX>(g, 0, j, k), m1 = at<AX>(g, 1, j, k), m2 = at<AX>(g, 2, j, k);
      at<AX>(g, 1, j, k) = m1 + u * m0;
      at<AX>(g, 2, j, k) = m2 + tu * m1 + uu * m0;
    }
}

template <typename T>
__device__ __forceinline__ void central_moments(const T (&f)[27], T ux, T uy, T uz, Cube<T>& g) {
  to_cube(f, g);
  raw_1d<0>(g);
  raw_1d<1>(g);
  raw_1d<2>(g);
  shift_1d<0>(g, ux);
  shift_1d<1>(g, uy);
  shift_1d<2>(g, uz);
}
template <typename T>
__device__ __forceinline__ void populations(Cube<T>& g, T ux, T uy, T uz, T (&f)[27]) {
  unshift_1d<2>(g, uz);
  unshift_1d<1>(g, uy);
  unshift_1d<0>(g, ux);
  pop_1d<0>(g);
  pop_1d<1>(g);
  pop_1d<2>(g);
  from_cube(g, f);
}

// moment index k (cumulant.py:321-349 ordering) <-> cube exponents
__host__ __device__ constexpr int kdeg(int k, int axis) {
  constexpr int t[27][3] = {{0, 0, 0}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {2, 0, 0}, {0, 2, 0}, {0, 0, 2},
                            {1, 1, 0}, {1, 0, 1}, {0, 1, 1}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {0, 2, 1},
                            {1, 0, 2}, {0, 1, 2}, {1, 1, 1}, {2, 2, 0}, {2, 0, 2}, {0, 2, 2}, {2, 1, 1},
                            {1, 2, 1}, {1, 1, 2}, {2, 2, 1}, {2, 1, 2}, {1, 2, 2}, {2, 2, 2}};
  return t[k][axis];
}
template <typename T>
__device__ __forceinline__ void cube_to_k(const Cube<T>& g, T (&k)[27]) {
#pragma unroll
  for (int i = 0; i < 27; ++i) k[i] = g[kdeg(i, 0)][kdeg(i, 1)][kdeg(i, 2)];
}
template <typename T>
__device__ __forceinline__ void k_to_cube(const T (&k)[27], Cube<T>& g) {
#pragma unroll
  for (int i = 0; i < 27; ++i) g[kdeg(i, 0)][kdeg(i, 1)][kdeg(i, 2)] = k[i];
}

// Legacy pseudo-cumulant transform on central moments of f_neq
// (cumulant.py:470-577), in place.
template <typename T>
__device__ __forceinline__ void legacy_forward(T (&c)[27]) {
  const T k200 = c[4], k020 = c[5], k002 = c[6], k110 = c[7], k101 = c[8], k011 = c[9];
  c[17] = c[17] - k200 * k020 - T(2) * k110 * k110;
  c[18] = c[18] - k200 * k002 - T(2) * k101 * k101;
  c[19] = c[19] - k020 * k002 - T(2) * k011 * k011;
  c[20] = c[20] - k200 * k011 - T(2) * k101 * k110;
  c[21] = c[21] - k020 * k101 - T(2) * k110 * k011;
  c[22] = c[22] - k002 * k110 - T(2) * k101 * k011;
  c[23] = c[23] - k200 * c[13] - T(2) * k110 * c[16];
  c[24] = c[24] - k200 * c[15] - T(2) * k101 * c[16];
  c[25] = c[25] - k020 * c[14] - T(2) * k011 * c[16];
  c[26] = c[26] - k200 * c[19] - k020 * c[18] - k002 * c[17] -
          T(2) * (k110 * c[22] + k101 * c[21] + k011 * c[20]) + T(2) * k200 * k020 * k002 +
          T(4) * k110 * k101 * k011 + T(2) * k110 * k110 * k002 + T(2) * k101 * k101 * k020 +
          T(2) * k011 * k011 * k200;
}
// inverse (cumulant.py:580-651), in place
template <typename T>
__device__ __forceinline__ void legacy_inverse(T (&c)[27]) {
  const T c200 = c[4], c020 = c[5], c002 = c[6], c110 = c[7], c101 = c[8], c011 = c[9];
  const T c220 = c[17], c202 = c[18], c022 = c[19], c211 = c[20], c121 = c[21], c112 = c[22];
  c[17] = c220 + c200 * c020 + T(2) * c110 * c110;
  c[18] = c202 + c200 * c002 + T(2) * c101 * c101;
  c[19] = c022 + c020 * c002 + T(2) * c011 * c011;
  c[20] = c211 + c200 * c011 + T(2) * c101 * c110;
  c[21] = c121 + c020 * c101 + T(2) * c110 * c011;
  c[22] = c112 + c002 * c110 + T(2) * c101 * c011;
  c[23] = c[23] + c200 * c[13] + T(2) * c110 * c[16];
  c[24] = c[24] + c200 * c[15] + T(2) * c101 * c[16];
  c[25] = c[25] + c020 * c[14] + T(2) * c011 * c[16];
  c[26] = c[26] + c200 * c022 + c020 * c202 + c002 * c220 + T(2) * (c110 * c112 + c101 * c121 + c011 * c211) -
          T(2) * c200 * c020 * c002 - T(4) * c110 * c101 * c011 - T(2) * c110 * c110 * c002 -
          T(2) * c101 * c101 * c020 - T(2) * c011 * c011 * c200;
}

// ---------------------------------------------------------------------------
// Cascaded central-moment collision (cascaded_collision.py:445-576): central
// moments of f_neq, the second order split into trace (rate s_bulk) and
// deviator (1/tau), every higher order relaxed at its own rate, back to
// populations.  D3Q19 uses TensorLBM's 19-monomial basis (no corner
// monomials, so only the complete shift triples are shifted); D3Q27 the full
// 3x3x3 cube with the factorised transforms.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cascaded_relax_second(T& kxx, T& kyy, T& kzz, T& kxy, T& kxz, T& kyz, T om, T sb) {
  const T tr = kxx + kyy + kzz;
  const T trs = (T(1) - sb) * tr, ks = T(1) - om;
  const T tr3 = tr * T(1.0 / 3.0), trs3 = trs * T(1.0 / 3.0);
  kxx = ks * (kxx - tr3) + trs3;
  kyy = ks * (kyy - tr3) + trs3;
  kzz = ks * (kzz - tr3) + trs3;
  kxy = ks * kxy;
  kxz = ks * kxz;
  kyz = ks * kyz;
}

template <int AX, typename T>
__device__ __forceinline__ void cascaded19_shift(T (&m)[19], T u, bool inverse) {
  using B = CascadedD3Q19;
  constexpr int G = AX == 0 ? B::kGroupsX : (AX == 1 ? B::kGroupsY : B::kGroupsZ);
  const T tu = T(2) * u, uu = u * u;
#pragma unroll
  for (int k = 0; k < G; ++k) {
    const int i0 = AX == 0 ? B::group_x(k, 0) : (AX == 1 ? B::group_y(k, 0) : B::group_z(k, 0));
    const int i1 = AX == 0 ? B::group_x(k, 1) : (AX == 1 ? B::group_y(k, 1) : B::group_z(k, 1));
    const int i2 = AX == 0 ? B::group_x(k, 2) : (AX == 1 ? B::group_y(k, 2) : B::group_z(k, 2));
    const T m0 = m[i0], m1 = m[i1], m2 = m[i2];
    if (inverse) {
      m[i1] = m1 + u * m0;
      m[i2] = m2 + tu * m1 + uu * m0;
    } else {
      m[i1] = m1 - u * m0;
      m[i2] = m2 - tu * m1 + uu * m0;
    }
  }
}

template <typename T>
__device__ __forceinline__ void collide_cascaded_d3q19(T (&f)[19], const CollideParams<T>& cp) {
  using L = D3Q19;
  using B = CascadedD3Q19;
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fe[19], fn[19], m[19];
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    fe[q] = feq_fused<L>(q, rho, ux, uy, uz, usq);
    fn[q] = f[q] - fe[q];
  }
#pragma unroll
  for (int i = 0; i < 19; ++i) {
    T acc = T(0);
#pragma unroll
    for (int q = 0; q < 19; ++q) {
      if (B::M(i, q) == 1) acc += fn[q];
      else if (B::M(i, q) == -1) acc -= fn[q];
    }
    m[i] = acc;
  }
  cascaded19_shift<0>(m, ux, false);
  cascaded19_shift<1>(m, uy, false);
  cascaded19_shift<2>(m, uz, false);
  cascaded_relax_second(m[4], m[5], m[6], m[7], m[8], m[9], cp.inv_tau, cp.omega_b);
  const T k3 = T(1) - cp.omega_odd, k4 = T(1) - cp.omega_even;
#pragma unroll
  for (int i = 10; i < 16; ++i) m[i] = k3 * m[i];
#pragma unroll
  for (int i = 16; i < 19; ++i) m[i] = k4 * m[i];
  cascaded19_shift<2>(m, uz, true);
  cascaded19_shift<1>(m, uy, true);
  cascaded19_shift<0>(m, ux, true);
#pragma unroll
  for (int q = 0; q < 19; ++q) {
    T acc = T(0);
#pragma unroll
    for (int i = 0; i < 19; ++i)
      if (B::Minv(q, i) != 0.0) acc += T(B::Minv(q, i)) * m[i];
    f[q] = fe[q] + acc;
  }
}

template <typename T>
__device__ __forceinline__ void collide_cascaded_d3q27(T (&f)[27], const CollideParams<T>& cp) {
  using L = D3Q27;
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fe[27], fn[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    fe[q] = feq_fused<L>(q, rho, ux, uy, uz, usq);
    fn[q] = f[q] - fe[q];
  }
  Cube<T> g;
  central_moments(fn, ux, uy, uz, g);
  cascaded_relax_second(g[2][0][0], g[0][2][0], g[0][0][2], g[1][1][0], g[1][0][1], g[0][1][1], cp.inv_tau,
                        cp.omega_b);
  const T keep[7] = {T(1), T(1), T(1), T(1) - cp.omega_odd, T(1) - cp.omega_even, T(1) - cp.cm_s5,
                     T(1) - cp.cm_s6};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (a + b + c >= 3) g[a][b][c] = keep[a + b + c] * g[a][b][c];
  T fns[27];
  populations(g, ux, uy, uz, fns);
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = fe[q] + fns[q];
}

// D3Q27 legacy cumulant collision with omega_b = omega_odd = omega_even = 1
// (cumulant.py:935 defaults).  Those rates set every post-collision
// cumulant above second order to zero and leave no bulk part, so only the
// central moments of f_neq up to second order enter (restricted 1-D passes:
// an entry of total degree <= 2 only needs entries of total degree <= 2),
// and the back transform (cumulant.py:580-651) reduces to the products of
// the relaxed second-order cumulants at orders 4 and 6.  Same operator as
// the general path below; only which zero terms are formed differs.
template <typename T>
__device__ __forceinline__ void collide_cumulant_legacy_unit(T (&f)[27], T om) {
  using L = D3Q27;
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fe[27];
  Cube<T> g;
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    fe[q] = feq_fused<L>(q, rho, ux, uy, uz, usq);
    g[L::cx(q) + 1][L::cy(q) + 1][L::cz(q) + 1] = f[q] - fe[q];
  }
  // raw moments along x on all 9 lines
  raw_1d<0>(g);
  // along y: all degrees where x-degree 0, degrees 0-1 where 1, degree 0 where 2
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    T vm = g[0][0][k], v0 = g[0][1][k], vp = g[0][2][k];
    g[0][0][k] = vm + v0 + vp;
    g[0][1][k] = vp - vm;
    g[0][2][k] = vp + vm;
    vm = g[1][0][k], v0 = g[1][1][k], vp = g[1][2][k];
    g[1][0][k] = vm + v0 + vp;
    g[1][1][k] = vp - vm;
    g[2][0][k] = g[2][0][k] + g[2][1][k] + g[2][2][k];
  }
  // along z: the entries of total degree <= 2
  T m[3][3][3];
  {
    const T vm = g[0][0][0], v0 = g[0][0][1], vp = g[0][0][2];
    m[0][0][0] = vm + v0 + vp;
    m[0][0][1] = vp - vm;
    m[0][0][2] = vp + vm;
  }
  m[1][0][0] = g[1][0][0] + g[1][0][1] + g[1][0][2];
  m[1][0][1] = g[1][0][2] - g[1][0][0];
  m[0][1][0] = g[0][1][0] + g[0][1][1] + g[0][1][2];
  m[0][1][1] = g[0][1][2] - g[0][1][0];
  m[2][0][0] = g[2][0][0] + g[2][0][1] + g[2][0][2];
  m[1][1][0] = g[1][1][0] + g[1][1][1] + g[1][1][2];
  m[0][2][0] = g[0][2][0] + g[0][2][1] + g[0][2][2];
  // binomial shifts x, y, z (cumulant.py:390-412) on the same entries
  {
    const T tu = T(2) * ux, uu = ux * ux;
    const T a0 = m[0][0][0], a1 = m[1][0][0];
    m[1][0][0] = a1 - ux * a0;
    m[2][0][0] = m[2][0][0] - tu * a1 + uu * a0;
    m[1][1][0] = m[1][1][0] - ux * m[0][1][0];
    m[1][0][1] = m[1][0][1] - ux * m[0][0][1];
  }
  {
    const T tu = T(2) * uy, uu = uy * uy;
    const T a0 = m[0][0][0], a1 = m[0][1][0];
    m[0][1][0] = a1 - uy * a0;
    m[0][2][0] = m[0][2][0] - tu * a1 + uu * a0;
    m[1][1][0] = m[1][1][0] - uy * m[1][0][0];
    m[0][1][1] = m[0][1][1] - uy * m[0][0][1];
  }
  {
    const T tu = T(2) * uz, uu = uz * uz;
    const T a0 = m[0][0][0], a1 = m[0][0][1];
    m[0][0][1] = a1 - uz * a0;
    m[0][0][2] = m[0][0][2] - tu * a1 + uu * a0;
    m[1][0][1] = m[1][0][1] - uz * m[1][0][0];
    m[0][1][1] = m[0][1][1] - uz * m[0][1][0];
  }
  // relaxation: deviatoric second order by 1 - omega, bulk and orders >= 3 to zero
  const T ks = T(1) - om;
  const T tr = m[2][0][0] + m[0][2][0] + m[0][0][2];
  const T tr3 = tr * T(1.0 / 3.0);
  const T c200 = ks * (m[2][0][0] - tr3), c020 = ks * (m[0][2][0] - tr3), c002 = ks * (m[0][0][2] - tr3);
  const T c110 = ks * m[1][1][0], c101 = ks * m[1][0][1], c011 = ks * m[0][1][1];
  // central moments of the relaxed cumulants (cumulant.py:580-651 with zeros)
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int b = 0; b < 3; ++b)
#pragma unroll
      for (int c = 0; c < 3; ++c) g[a][b][c] = T(0);
  g[0][0][0] = m[0][0][0];
  g[1][0][0] = m[1][0][0];
  g[0][1][0] = m[0][1][0];
  g[0][0][1] = m[0][0][1];
  g[2][0][0] = c200;
  g[0][2][0] = c020;
  g[0][0][2] = c002;
  g[1][1][0] = c110;
  g[1][0][1] = c101;
  g[0][1][1] = c011;
  g[2][2][0] = c200 * c020 + T(2) * c110 * c110;
  g[2][0][2] = c200 * c002 + T(2) * c101 * c101;
  g[0][2][2] = c020 * c002 + T(2) * c011 * c011;
  g[2][1][1] = c200 * c011 + T(2) * c101 * c110;
  g[1][2][1] = c020 * c101 + T(2) * c110 * c011;
  g[1][1][2] = c002 * c110 + T(2) * c101 * c011;
  g[2][2][2] = -T(2) * c200 * c020 * c002 - T(4) * c110 * c101 * c011 - T(2) * c110 * c110 * c002 -
               T(2) * c101 * c101 * c020 - T(2) * c011 * c011 * c200;
  T fns[27];
  populations(g, ux, uy, uz, fns);
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = fe[q] + fns[q];
}

// D3Q27 legacy cumulant collision (cumulant.py:935-1047)
template <typename T>
__device__ __forceinline__ void collide_cumulant_legacy(T (&f)[27], const CollideParams<T>& cp) {
  using L = D3Q27;
  if (cp.cum_unit_rates) {
    collide_cumulant_legacy_unit(f, cp.inv_tau);
    return;
  }
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fe[27], fn[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) {
    fe[q] = feq_fused<L>(q, rho, ux, uy, uz, usq);
    fn[q] = f[q] - fe[q];
  }
  Cube<T> g;
  central_moments(fn, ux, uy, uz, g);
  T c[27];
  cube_to_k(g, c);
  legacy_forward(c);
  // relaxation (cumulant.py:654-740): trace / deviatoric split at 2nd order
  const T om = cp.inv_tau;
  const T tr = c[4] + c[5] + c[6];
  const T tr3 = tr * T(1.0 / 3.0);
  const T dxx = c[4] - tr3, dyy = c[5] - tr3, dzz = c[6] - tr3;
  const T trs = (T(1) - cp.omega_b) * tr;
  const T ks = T(1) - om;
  const T trs3 = trs * T(1.0 / 3.0);
  c[4] = ks * dxx + trs3;
  c[5] = ks * dyy + trs3;
  c[6] = ks * dzz + trs3;
  c[7] = ks * c[7];
  c[8] = ks * c[8];
  c[9] = ks * c[9];
  const T k3 = T(1) - cp.omega_odd, k4 = T(1) - cp.omega_even;
#pragma unroll
  for (int i = 10; i < 17; ++i) c[i] = k3 * c[i];
#pragma unroll
  for (int i = 17; i < 27; ++i) c[i] = k4 * c[i];
  legacy_inverse(c);
  k_to_cube(c, g);
  T fns[27];
  populations(g, ux, uy, uz, fns);
#pragma unroll
  for (int q = 0; q < 27; ++q) f[q] = fe[q] + fns[q];
}

// Geier-2015 cumulants of the full distribution (cumulant.py:674-815), using
// normalised central moments kt = k / rho.  Input/outputs in k ordering.
template <typename T>
__device__ __forceinline__ void geier_forward(T (&k)[27]) {
  const T rho = k[0];
  const T ir = rcp_fast(rho);
  T t[27];
#pragma unroll
  for (int i = 0; i < 27; ++i) t[i] = k[i] * ir;
  T c[27];
#pragma unroll
  for (int i = 0; i < 27; ++i) c[i] = t[i];
  c[17] = t[17] - (t[5] * t[4] + T(2) * t[7] * t[7]);
  c[18] = t[18] - (t[6] * t[4] + T(2) * t[8] * t[8]);
  c[19] = t[19] - (t[6] * t[5] + T(2) * t[9] * t[9]);
  c[20] = t[20] - (t[9] * t[4] + T(2) * t[8] * t[7]);
  c[21] = t[21] - (T(2) * t[9] * t[7] + t[5] * t[8]);
  c[22] = t[22] - (t[6] * t[7] + T(2) * t[9] * t[8]);
  c[23] = t[23] - (T(2) * t[9] * t[10] + t[5] * t[11] + t[13] * t[4] + T(2) * t[8] * t[12] + T(4) * t[7] * t[16]);
  c[24] = t[24] - (t[6] * t[10] + T(2) * t[9] * t[11] + t[15] * t[4] + T(4) * t[8] * t[16] + T(2) * t[14] * t[7]);
  c[25] = t[25] - (t[6] * t[12] + T(4) * t[9] * t[16] + T(2) * t[15] * t[7] + t[5] * t[14] + T(2) * t[13] * t[8]);
  c[26] = t[26] - (-T(2) * t[6] * t[5] * t[4] - T(4) * t[6] * t[7] * t[7] + t[6] * t[17] -
                   T(4) * t[9] * t[9] * t[4] - T(16) * t[9] * t[8] * t[7] + T(4) * t[9] * t[20] +
                   T(2) * t[15] * t[10] - T(4) * t[5] * t[8] * t[8] + t[5] * t[18] + T(2) * t[13] * t[11] +
                   t[19] * t[4] + T(4) * t[8] * t[21] + T(2) * t[14] * t[12] + T(4) * t[7] * t[22] +
                   T(4) * t[16] * t[16]);
#pragma unroll
  for (int i = 1; i < 27; ++i) k[i] = c[i] * rho;
  k[0] = rho;
}
template <typename T>
__device__ __forceinline__ void geier_inverse(T (&c)[27]) {
  const T rho = c[0];
  const T ir = rcp_fast(rho);
  T t[27];
#pragma unroll
  for (int i = 0; i < 27; ++i) t[i] = c[i] * ir;
  T k[27];
#pragma unroll
  for (int i = 0; i < 27; ++i) k[i] = t[i];
  k[17] = t[5] * t[4] + T(2) * t[7] * t[7] + t[17];
  k[18] = t[6] * t[4] + T(2) * t[8] * t[8] + t[18];
  k[19] = t[6] * t[5] + T(2) * t[9] * t[9] + t[19];
  k[20] = t[9] * t[4] + T(2) * t[8] * t[7] + t[20];
  k[21] = T(2) * t[9] * t[7] + t[5] * t[8] + t[21];
  k[22] = t[6] * t[7] + T(2) * t[9] * t[8] + t[22];
  k[23] = T(2) * t[9] * t[10] + t[5] * t[11] + t[13] * t[4] + T(2) * t[8] * t[12] + T(4) * t[7] * t[16] + t[23];
  k[24] = t[6] * t[10] + T(2) * t[9] * t[11] + t[15] * t[4] + T(4) * t[8] * t[16] + T(2) * t[14] * t[7] + t[24];
  k[25] = t[6] * t[12] + T(4) * t[9] * t[16] + T(2) * t[15] * t[7] + t[5] * t[14] + T(2) * t[13] * t[8] + t[25];
  k[26] = t[6] * t[5] * t[4] + T(2) * t[6] * t[7] * t[7] + t[6] * t[17] + T(2) * t[9] * t[9] * t[4] +
          T(8) * t[9] * t[8] * t[7] + T(4) * t[9] * t[20] + T(2) * t[15] * t[10] + T(2) * t[5] * t[8] * t[8] +
          t[5] * t[18] + T(2) * t[13] * t[11] + t[19] * t[4] + T(4) * t[8] * t[21] + T(2) * t[14] * t[12] +
          T(4) * t[7] * t[22] + T(4) * t[16] * t[16] + t[26];
#pragma unroll
  for (int i = 1; i < 27; ++i) c[i] = k[i] * rho;
  c[0] = rho;
}

// D3Q27 Geier cumulant collision (cumulant.py:1050-1156)
template <typename T>
__device__ __forceinline__ void collide_cumulant_geier(T (&f)[27], const CollideParams<T>& cp) {
  using L = D3Q27;
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fe[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) fe[q] = feq_fused<L>(q, rho, ux, uy, uz, usq);
  Cube<T> g;
  T c[27], ce[27];
  central_moments(fe, ux, uy, uz, g);
  cube_to_k(g, ce);
  geier_forward(ce);
  central_moments(f, ux, uy, uz, g);
  cube_to_k(g, c);
  geier_forward(c);
  const T om = cp.inv_tau;
  const T dxx = c[4] - ce[4], dyy = c[5] - ce[5], dzz = c[6] - ce[6];
  const T tr = dxx + dyy + dzz;
  const T tr3 = tr * T(1.0 / 3.0);
  c[4] = c[4] - (om * (dxx - tr3) + cp.omega_b * tr3);
  c[5] = c[5] - (om * (dyy - tr3) + cp.omega_b * tr3);
  c[6] = c[6] - (om * (dzz - tr3) + cp.omega_b * tr3);
  c[7] = c[7] - om * (c[7] - ce[7]);
  c[8] = c[8] - om * (c[8] - ce[8]);
  c[9] = c[9] - om * (c[9] - ce[9]);
#pragma unroll
  for (int i = 10; i < 17; ++i) c[i] = c[i] - cp.omega_odd * (c[i] - ce[i]);
#pragma unroll
  for (int i = 17; i < 27; ++i) c[i] = c[i] - cp.omega_even * (c[i] - ce[i]);
  geier_inverse(c);
  k_to_cube(c, g);
  populations(g, ux, uy, uz, f);
}

// ---------------------------------------------------------------------------
// Fused-arithmetic BGK and Smagorinsky for the half storage formats, whose
// populations are rounded to 11 / 8 bits on every store: there the
// reference's rounding order has no meaning, and fused multiply-adds save
// the instructions that the unfused exact forms cost.
// ---------------------------------------------------------------------------
template <class L, typename T>
__device__ __forceinline__ void collide_bgk_fast(T (&f)[L::Q], T inv_tau) {
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  // f' = (1 - om) f + om feq with feq_q = w rho (1 - 1.5 u.u + 4.5 cu^2 + 3 cu):
  // a direction and its opposite share cu up to sign, so om feq of the pair
  // is s +- d with s = om w rho (1 - 1.5 u.u + 4.5 cu^2), d = 3 om w rho cu
  const T om = inv_tau, keep = T(1) - inv_tau;
  const T orho = om * rho;
  const T obase = orho * (T(1) - T(1.5) * usq);
  f[0] = fma(f[0], keep, weight<L, T>(0) * obase);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::opp(q) < q) continue;
    const int qb = L::opp(q);
    T cu = T(0);
    if (L::cx(q) != 0) cu = (L::cx(q) > 0) ? cu + ux : cu - ux;
    if (L::cy(q) != 0) cu = (L::cy(q) > 0) ? cu + uy : cu - uy;
    if (L::cz(q) != 0) cu = (L::cz(q) > 0) ? cu + uz : cu - uz;
    const double w = L::w(q);
    const T sq = fma(T(T(4.5 * w) * orho) * cu, cu, T(T(w) * obase));
    const T k3 = T(T(3.0 * w) * orho), k3n = T(T(-3.0 * w) * orho);
    f[q] = fma(f[q], keep, fma(k3, cu, sq));
    f[qb] = fma(f[qb], keep, fma(k3n, cu, sq));
  }
}

// BGK on the stored deviations of the shifted half formats, G_q = s (f_q - w_q):
// with R = sum G (so rho = 1 + R / s) and B = om s rho,
//   s om (feq_q - w_q) = w_q (om R + B (3 cu + 4.5 cu^2 - 1.5 u.u)),
// so G'_q = (1 - om) G_q + that, without forming f.  Same operation count as
// collide_bgk_fast, and no shift or scale on the loads and stores around it.
template <class L, typename T>
__device__ __forceinline__ void collide_bgk_deviation(T (&g)[L::Q], T om, T s) {
  T R = g[0];
#pragma unroll
  for (int q = 1; q < L::Q; ++q) R += g[q];
  T jx = T(0), jy = T(0), jz = T(0);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::cx(q) != 0) jx = (L::cx(q) > 0) ? jx + g[q] : jx - g[q];
    if (L::cy(q) != 0) jy = (L::cy(q) > 0) ? jy + g[q] : jy - g[q];
    if (L::cz(q) != 0) jz = (L::cz(q) > 0) ? jz + g[q] : jz - g[q];
  }
  const T rho = fma(R, T(1) / s, T(1));
  const T srho = s * clamp_lo(rho, T(1e-12));
  const T irs = rcp_fast(srho);
  const T ux = jx * irs, uy = jy * irs, uz = (L::DIM == 3) ? jz * irs : T(0);
  const T usq = usq_fused<L>(ux, uy, uz);
  const T keep = T(1) - om;
  const T B = om * srho;
  const T base = fma(B, T(-1.5) * usq, om * R);
  g[0] = fma(g[0], keep, weight<L, T>(0) * base);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::opp(q) < q) continue;
    const int qb = L::opp(q);
    T cu = T(0);
    if (L::cx(q) != 0) cu = (L::cx(q) > 0) ? cu + ux : cu - ux;
    if (L::cy(q) != 0) cu = (L::cy(q) > 0) ? cu + uy : cu - uy;
    if (L::cz(q) != 0) cu = (L::cz(q) > 0) ? cu + uz : cu - uz;
    const double w = L::w(q);
    const T sq = fma(T(T(4.5 * w) * B) * cu, cu, T(T(w) * base));
    const T k3 = T(T(3.0 * w) * B), k3n = T(T(-3.0 * w) * B);
    g[q] = fma(g[q], keep, fma(k3, cu, sq));
    g[qb] = fma(g[qb], keep, fma(k3n, cu, sq));
  }
}

template <class L, typename T>
__device__ __forceinline__ void collide_smagorinsky_fast(T (&f)[L::Q], const CollideParams<T>& cp) {
  T rho, ux, uy, uz;
  macroscopic_fused<L>(f, rho, ux, uy, uz);
  const T usq = usq_fused<L>(ux, uy, uz);
  T fn[L::Q];
  T pxx = T(0), pyy = T(0), pzz = T(0), pxy = T(0), pxz = T(0), pyz = T(0);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    fn[q] = f[q] - feq_fused<L>(q, rho, ux, uy, uz, usq);
    if (L::cx(q) != 0) pxx += fn[q];
    if (L::cy(q) != 0) pyy += fn[q];
    if (L::cz(q) != 0) pzz += fn[q];
    if (L::cx(q) * L::cy(q) != 0) pxy += T(L::cx(q) * L::cy(q)) * fn[q];
    if (L::cx(q) * L::cz(q) != 0) pxz += T(L::cx(q) * L::cz(q)) * fn[q];
    if (L::cy(q) * L::cz(q) != 0) pyz += T(L::cy(q) * L::cz(q)) * fn[q];
  }
  T rad = pxx * pxx + pyy * pyy + T(2) * pxy * pxy;
  if constexpr (L::DIM == 3) rad += pzz * pzz + T(2) * (pxz * pxz + pyz * pyz);
  rad = clamp_lo(rad, T(1e-30));
  const T rs = clamp_lo(rho, T(1e-12));
  T disc = cp.tau_sq + cp.smag_coef * sqrt(rad) * rcp_fast(rs);
  disc = clamp_lo(disc, T(0));
  T te = T(0.5) * (cp.tau + sqrt(disc));
  te = clamp_hi(clamp_lo(te, T(0.5001)), cp.tau_eff_max);
  const T ninv = -rcp_fast(te);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = fma(fn[q], ninv, f[q]);
}

// ---------------------------------------------------------------------------
// dispatch (FAST: fused-arithmetic forms, used for the half storage formats)
// ---------------------------------------------------------------------------
template <class L, int COLL, typename T, bool FAST = false>
__device__ __forceinline__ void collide(T (&f)[L::Q], const CollideParams<T>& cp, T tau_cell, bool has_tau_cell) {
  if constexpr (COLL == TLBM_COLL_BGK && FAST) {
    collide_bgk_fast<L>(f, has_tau_cell ? rcp_fast(tau_cell) : cp.inv_tau);
  } else if constexpr (COLL == TLBM_COLL_SMAGORINSKY && FAST) {
    collide_smagorinsky_fast<L>(f, cp);
  } else if constexpr (COLL == TLBM_COLL_BGK) {
    if (has_tau_cell) collide_bgk<L>(f, tau_cell, 1.0 / double(tau_cell));
    else collide_bgk<L>(f, cp.tau, cp.inv_tau64);
  } else if constexpr (COLL == TLBM_COLL_MRT) {
    MrtRates<T> r = cp.mrt;
    if (has_tau_cell) r.s_nu = rcp_fast(tau_cell);
    collide_mrt<L>(f, r);
  } else if constexpr (COLL == TLBM_COLL_SMAGORINSKY) {
    collide_smagorinsky<L>(f, cp);
  } else if constexpr (COLL == TLBM_COLL_CASCADED) {
    if constexpr (L::Q == 19) collide_cascaded_d3q19(f, cp);
    else if constexpr (L::Q == 27) collide_cascaded_d3q27(f, cp);
  } else if constexpr (COLL == TLBM_COLL_TRT) {
    collide_trt<L>(f, cp.tau, cp.inv_tau64, cp.tau_minus, cp.inv_tau_minus64);
  } else if constexpr (COLL == TLBM_COLL_RLBM) {
    collide_rlbm<L>(f, cp.rlbm_keep);
  } else if constexpr (COLL == TLBM_COLL_CUMULANT_D3Q19) {
    static_assert(L::Q == 19, "D3Q19 only");
    collide_cumulant_d3q19(f, cp);
  } else if constexpr (COLL == TLBM_COLL_CUMULANT) {
    static_assert(L::Q == 27, "D3Q27 only");
    collide_cumulant_legacy(f, cp);
  } else if constexpr (COLL == TLBM_COLL_CUMULANT_GEIER) {
    static_assert(L::Q == 27, "D3Q27 only");
    collide_cumulant_geier(f, cp);
  }
}

// The parameters of the explicit-rounding types (F1 one cell, F2 a pair):
// every scalar broadcast to every lane.
template <class F>
__host__ __device__ __forceinline__ CollideParams<F> pack_params(const CollideParams<float>& c) {
  CollideParams<F> p;
  p.tau = F(c.tau);
  p.inv_tau = F(c.inv_tau);
  p.inv_tau64 = c.inv_tau64;
  p.mrt = {F(c.mrt.s_e), F(c.mrt.s_eps), F(c.mrt.s_q), F(c.mrt.s_nu), F(c.mrt.s_pi)};
  p.omega_b = F(c.omega_b);
  p.omega_odd = F(c.omega_odd);
  p.omega_even = F(c.omega_even);
  p.c_smag = F(c.c_smag);
  p.smag_coef = F(c.smag_coef);
  p.smag_coef_cum = F(c.smag_coef_cum);
  p.omega_b_minus_omega = F(c.omega_b_minus_omega);
  p.keep_even = F(c.keep_even);
  p.tau_sq = F(c.tau_sq);
  p.tau_eff_max = F(c.tau_eff_max);
  p.force_a = F(c.force_a);
  p.cum_unit_rates = c.cum_unit_rates;
  p.cm_s5 = F(c.cm_s5);
  p.cm_s6 = F(c.cm_s6);
  p.tau_minus = F(c.tau_minus);
  p.inv_tau_minus64 = c.inv_tau_minus64;
  p.rlbm_keep = F(c.rlbm_keep);
  return p;
}

// Collisions that run on the explicit-rounding types (F2 in the pair kernels,
// F1 in the single-cell kernels): the fused-arithmetic forms (no reference
// rounding order to keep), in float32.
template <class L, int COLL, bool FAST>
__host__ __device__ constexpr bool packed_collision() {
  return COLL == TLBM_COLL_MRT || (COLL == TLBM_COLL_BGK && FAST) || (COLL == TLBM_COLL_SMAGORINSKY && FAST) ||
         (L::Q == 27 && COLL == TLBM_COLL_CUMULANT);
}

template <typename T>
__host__ __device__ CollideParams<T> make_collide_params(double tau, double s_e, double s_eps, double s_q, double s_pi,
                                     double omega_b, double omega_odd, double omega_even, double c_smag) {
  CollideParams<T> cp;
  cp.tau = T(tau);
  cp.inv_tau = T(1.0 / tau);
  cp.inv_tau64 = 1.0 / double(T(tau));
  cp.mrt.s_e = T(s_e);
  cp.mrt.s_eps = T(s_eps);
  cp.mrt.s_q = T(s_q);
  cp.mrt.s_pi = T(s_pi < 0 ? s_e : s_pi);
  cp.mrt.s_nu = T(1.0 / tau);
  cp.omega_b = T(omega_b);
  cp.omega_odd = T(omega_odd);
  cp.omega_even = T(omega_even);
  cp.c_smag = T(c_smag);
  cp.smag_coef = T(18.0 * (c_smag * c_smag));
  cp.smag_coef_cum = T(18.0 * c_smag * c_smag);
  cp.omega_b_minus_omega = T(omega_b - 1.0 / tau);
  cp.keep_even = T(1.0 - omega_even);
  cp.cum_unit_rates = (omega_b == 1.0) && (omega_odd == 1.0) && (omega_even == 1.0);
  cp.cm_s5 = cp.omega_even;
  cp.cm_s6 = cp.omega_even;
  cp.tau_minus = cp.tau;
  cp.inv_tau_minus64 = cp.inv_tau64;
  cp.rlbm_keep = T(1.0 - 1.0 / tau);
  cp.tau_sq = T(tau * tau);
  cp.tau_eff_max = T(tau + 0.5 > 1.0 ? tau + 0.5 : 1.0);
  cp.force_a = T(0);
  return cp;
}

// TRT: tau_minus = 1/2 + Lambda / (tau_plus - 1/2) in float64 (a Python
// scalar in the reference), used as a scalar of the field's type
template <typename T>
__host__ __device__ void set_trt_rates(CollideParams<T>& cp, double tau_plus, double lambda_trt) {
  const double tm = 0.5 + lambda_trt / (tau_plus - 0.5);
  cp.tau_minus = T(tm);
  cp.inv_tau_minus64 = 1.0 / double(T(tm));
}

}  // namespace tlbm

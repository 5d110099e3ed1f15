// Boundary conditions on the post-stream populations of one cell (registers).
//
// These are the per-cell forms of TensorLBM's plane operators; the fused step
// kernel applies them to the cells of the plane they act on, the stand-alone
// entry points run them over the plane alone.
#pragma once

#include "tlbm_collide.cuh"

namespace tlbm {

// full-way bounce-back at a solid cell: f_q <- f_opp(q)
template <class L, typename T>
__device__ __forceinline__ void bounce_back(T (&f)[L::Q]) {
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::opp(q) > q) {
      const T t = f[q];
      f[q] = f[L::opp(q)];
      f[L::opp(q)] = t;
    }
  }
}

// Ladd moving-wall bounce-back (propeller_benchmark.py:221-270 for D3Q19,
// rotating_cylinder.py:140-192 for D2Q9): swap, then add
// 2 w_q rho (c_q . u_w) / c_s^2 with rho the density before the swap,
// evaluated as (((2 w) rho) cu) 3 like the reference, whose weights there are
// the float32 W tensors of d2q9.py / d3q19.py cast to the field dtype.
template <class L, typename T>
__device__ __forceinline__ void moving_wall_bounce_back(T (&f)[L::Q], T uwx, T uwy, T uwz) {
  const T rho = csum<L>(f, OneCoef{});
  bounce_back<L>(f);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    const T cu = signed_sum(L::cx(q), L::cy(q), L::cz(q), uwx, uwy, uwz);
    const T corr = xmul(xmul(xmul(xmul(T(2), T(float(L::w(q)))), rho), cu), T(3));
    f[q] = xadd(f[q], corr);
  }
}

// momentum carried by the post-stream populations of one cell: sum_q c_q f_q
template <class L, typename T>
__device__ __forceinline__ void cell_momentum(const T (&f)[L::Q], T& mx, T& my, T& mz) {
  mx = T(0); my = T(0); mz = T(0);
#pragma unroll
  for (int q = 1; q < L::Q; ++q) {
    if (L::cx(q) != 0) mx = (L::cx(q) > 0) ? mx + f[q] : mx - f[q];
    if (L::cy(q) != 0) my = (L::cy(q) > 0) ? my + f[q] : my - f[q];
    if (L::cz(q) != 0) mz = (L::cz(q) > 0) ? mz + f[q] : mz - f[q];
  }
}

// Parameters of the plane conditions, in compute type.
template <typename T> struct BcParams {
  T u_in, uy_in, uz_in;     // inlet velocity
  T one_minus_u;            // 1 - u_in, rounded once like the torch scalar
  T rho_out;
  T u_lid;
  // D2Q9 closed forms use python-side products with rho_out
  T two_thirds_rho_out, sixth_rho_out;
  T ff_u[3];                // far field: free-stream velocity of the lateral planes (= u_in)
  T ff_in[3];               // far field: velocity of the x = 0 plane (u_in + the inlet perturbation)
};

template <typename T>
__host__ __device__ BcParams<T> make_bc_params(double u_in0, double u_in1, double u_in2, double rho_out, double u_lid,
                                               const double* ff_inlet_du = nullptr) {
  BcParams<T> b;
  b.u_in = T(u_in0);
  b.uy_in = T(u_in1);
  b.uz_in = T(u_in2);
  b.one_minus_u = T(1.0 - u_in0);
  b.rho_out = T(rho_out);
  b.u_lid = T(u_lid);
  b.two_thirds_rho_out = T((2.0 / 3.0) * rho_out);
  b.sixth_rho_out = T((1.0 / 6.0) * rho_out);
  const double u[3] = {u_in0, u_in1, u_in2};
  for (int i = 0; i < 3; ++i) {
    b.ff_u[i] = T(u[i]);
    b.ff_in[i] = T(ff_inlet_du ? u[i] + ff_inlet_du[i] : u[i]);
  }
  return b;
}

// Free-stream far field (boundaries.py:199-220, boundaries3d.py:446-538,
// boundaries_d3q27.py:63-104): f = feq(1, u) of the lattice's equilibrium
// function, bit for bit (rho = 1 exactly).
template <class L, typename T>
__device__ __forceinline__ void far_field_feq(T (&f)[L::Q], T ux, T uy, T uz) {
  const T usq = usq_of<L>(ux, uy, uz);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) f[q] = feq_q<L>(q, T(1), ux, uy, uz, usq);
}

// Known population paired with unknown q by the x-face Zou/He conditions.
// D3Q19 pairs opposites (boundaries3d.py:14-19); TensorLBM's D3Q27 tables pair
// x-mirrors, e.g. 7 (1,1,0) with 8 (-1,1,0) (boundaries_d3q27.py:36-41), and
// the results follow that pairing.
template <class L>
__host__ __device__ constexpr int zh_partner(int q) {
  if constexpr (L::Q != 27) {
    return L::opp(q);
  } else {
    for (int k = 0; k < L::Q; ++k)
      if (L::cx(k) == -L::cx(q) && L::cy(k) == L::cy(q) && L::cz(k) == L::cz(q)) return k;
    return q;
  }
}

// --------------------------------------------------------------------------
// Zou/He velocity inlet at x = 0
// --------------------------------------------------------------------------
// D3Q19 / D3Q27: rho from mass + x-momentum balance, then non-equilibrium
// bounce-back f_k = feq_k - feq_p(k) + f_p(k) for every k with c_kx > 0, p the
// partner above (boundaries3d.py:205-266, boundaries_d3q27.py:107-176).
template <class L, typename T>
__device__ __forceinline__ void zou_he_inlet_3d(T (&f)[L::Q], T u, T uy, T uz, T one_minus_u) {
  T s0 = T(0), sn = T(0);
  bool b0 = false, bn = false;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    if (L::cx(q) == 0) { s0 = b0 ? s0 + f[q] : f[q]; b0 = true; }
    if (L::cx(q) < 0) { sn = bn ? sn + f[q] : f[q]; bn = true; }
  }
  const T rho = (s0 + T(2) * sn) / one_minus_u;
  const T usq = usq_of<L>(u, uy, uz);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    if (L::cx(q) > 0) {
      const int o = zh_partner<L>(q);
      f[q] = feq_q<L>(q, rho, u, uy, uz, usq) - feq_q<L>(o, rho, u, uy, uz, usq) + f[o];
    }
  }
}

// D3Q19 / D3Q27 pressure outlet at x = nx-1 (boundaries3d.py:269-321,
// boundaries_d3q27.py:179-240)
template <class L, typename T>
__device__ __forceinline__ void zou_he_outlet_3d(T (&f)[L::Q], T rho_out) {
  T s0 = T(0), sp = T(0);
  bool b0 = false, bp = false;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    if (L::cx(q) == 0) { s0 = b0 ? s0 + f[q] : f[q]; b0 = true; }
    if (L::cx(q) > 0) { sp = bp ? sp + f[q] : f[q]; bp = true; }
  }
  const T ux = T(-1) + (s0 + T(2) * sp) / rho_out;
  const T usq = ux * ux;  // uy = uz = 0
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    if (L::cx(q) < 0) {
      const int o = zh_partner<L>(q);
      f[q] = feq_q<L>(q, rho_out, ux, T(0), T(0), usq) - feq_q<L>(o, rho_out, ux, T(0), T(0), usq) + f[o];
    }
  }
}

// D2Q9 closed forms (boundaries.py:50-99, :102-125).  The inlet profile is a
// float32 tensor there, so 1 - u is formed in the field dtype.
template <typename T>
__device__ __forceinline__ void zou_he_inlet_d2q9(T (&f)[9], T u, T uy) {
  const T rho = xdiv(xadd(xadd(xadd(f[0], f[2]), f[4]), xmul(T(2), xadd(xadd(f[3], f[6]), f[7]))), xsub(T(1), u));
  const T h24 = xmul(T(0.5), xsub(f[2], f[4]));
  const T r6u = xmul(xmul(T(1.0 / 6.0), rho), u);
  const T r2uy = xmul(xmul(T(0.5), rho), uy);
  f[1] = xadd(f[3], xmul(xmul(T(2.0 / 3.0), rho), u));
  f[5] = xadd(xadd(xsub(f[7], h24), r6u), r2uy);
  f[8] = xsub(xadd(xadd(f[6], h24), r6u), r2uy);
}
template <typename T>
__device__ __forceinline__ void zou_he_outlet_d2q9(T (&f)[9], T rho_out, T two_thirds_rho_out, T sixth_rho_out) {
  const T s = xadd(xadd(xadd(f[0], f[2]), f[4]), xmul(T(2), xadd(xadd(f[1], f[5]), f[8])));
  const T ux = xadd(T(-1), xdiv(s, rho_out));
  const T h24 = xmul(T(0.5), xsub(f[2], f[4]));
  const T su = xmul(sixth_rho_out, ux);
  const T f1 = f[1], f5 = f[5], f8 = f[8];
  f[3] = xsub(f1, xmul(two_thirds_rho_out, ux));
  f[7] = xsub(xadd(f5, h24), su);
  f[6] = xsub(xsub(f8, h24), su);
}

// --------------------------------------------------------------------------
// Moving lid at y = ny-1
// --------------------------------------------------------------------------
// D2Q9: lid_driven_cavity.py:431-473
template <typename T>
__device__ __forceinline__ void moving_lid_d2q9(T (&f)[9], T u_lid) {
  const T rho = xadd(xadd(xadd(xadd(xadd(f[0], f[1]), xmul(T(2), f[2])), f[3]), xmul(T(2), f[5])), xmul(T(2), f[6]));
  const T h13 = xmul(T(0.5), xsub(f[1], f[3]));
  const T ru = xmul(xmul(T(0.5), rho), u_lid);
  const T f2 = f[2], f5 = f[5], f6 = f[6];
  f[4] = f2;
  f[7] = xsub(xadd(f5, h13), ru);
  f[8] = xadd(xsub(f6, h13), ru);
}
// D3Q19: boundaries3d.py:324-404 (uy = uz = 0)
template <typename T>
__device__ __forceinline__ void moving_lid_d3q19(T (&f)[19], T u_lid) {
  const T sum0 = f[0] + f[1] + f[2] + f[5] + f[6] + f[11] + f[12] + f[13] + f[14];
  const T sump = f[3] + f[7] + f[10] + f[15] + f[17];
  const T rho = sum0 + T(2) * sump;
  const T sx0 = f[1] - f[2] + f[11] - f[12] + f[13] - f[14];
  const T sxp = f[7] - f[10];
  const T dx = xsub(xmul(rho, u_lid), xadd(sx0, sxp));
  const T sz0 = f[5] - f[6] + f[11] - f[12] - f[13] + f[14];
  const T h = T(0.5) * (f[7] + f[10]);
  f[4] = f[3];
  f[8] = h - T(0.5) * dx;
  f[9] = h + T(0.5) * dx;
  f[16] = f[15] + T(0.5) * sz0;
  f[18] = f[17] - T(0.5) * sz0;
}

}  // namespace tlbm

// The fused time-step kernel: pull -> boundary conditions -> collision -> store.
//
// One thread owns one cell.  It gathers the Q populations that stream into
// its cell (f_in[q, x - c_q], periodic wrap on every axis exactly like
// torch.roll / the cached index gather of stream3d), applies the boundary
// conditions in TensorLBM's order, collides, and writes the Q results at its
// own cell.  Every population of f_in is read by exactly one thread, so the
// kernel moves 2*Q*sizeof(S) bytes per cell and nothing else except the flag
// byte.  Warps span consecutive x, so each direction is one coalesced
// 128-byte row access (shifted by one element for c_x = +-1).
#pragma once

#include <type_traits>

#include "tlbm_bc.cuh"
#include "tlbm_pair.cuh"

#ifndef TLBM_PACK
#define TLBM_PACK 1
#endif
#ifndef TLBM_MINB_MRT
#define TLBM_MINB_MRT 3
#endif
#ifndef TLBM_MINB_MRT_HALF
#define TLBM_MINB_MRT_HALF 3
#endif
#ifndef TLBM_MINB_BGK_HALF
#define TLBM_MINB_BGK_HALF 4
#endif
#ifndef TLBM_MINB_CUM
#define TLBM_MINB_CUM 2
#endif
#ifndef TLBM_MINB_AA_MRT
#define TLBM_MINB_AA_MRT 0
#endif

namespace tlbm {

// Warp-reduce one cell's momentum in float64 and add scale x it to
// force[0..2]: 2 for the full-way momentum exchange (each population of an
// obstacle cell is reflected), 1 for a ledger that already holds both halves
// of every link (Bouzidi).  Blocks are at least 32 wide in x, so a warp is 32
// consecutive x of one row.
template <typename T>
__device__ __forceinline__ void accumulate_force(double* force, bool any_in_warp, T mx, T my, T mz,
                                                 double scale = 2.0) {
  if (!any_in_warp) return;
  const double sx = warp_sum(double(mx)), sy = warp_sum(double(my)), sz = warp_sum(double(mz));
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(force + 0, scale * sx);
    atomicAdd(force + 1, scale * sy);
    atomicAdd(force + 2, scale * sz);
  }
}

// One domain as seen by the per-cell update.
template <typename SI, typename SO> struct Domain {
  const SI* fin;
  SO* fout;
  const uint8_t* flags;     // may be null
  const float* tau_field;   // may be null
  double* force;            // may be null
  unsigned int* status;     // may be null
  const void* wall_u;       // (DIM, n) wall velocity of TLBM_FLAG_MOVING cells, compute type; may be null
  const int32_t* link_row;  // TLBM_FLAG_CURVED cells: row in link_q; may be null
  const float* link_q;      // (rows, Q) BFL wall fractions (0 = no link); may be null
  int nx, ny, nz;
  long long plane, n;
  uint32_t bc;
};

// The value a Bouzidi link (x, d) sends back into x along -c_d
// (bfl_common.py:169-180): Pd = P_d(x), up = P_d(x - c_d) (the pulled value),
// Po = P_opp(x); every product and sum rounded on its own like the torch
// expression, q promoted to the populations' type.
template <typename T>
__device__ __forceinline__ T bfl_value(T q, T Pd, T up, T Po) {
  const T q2 = xmul(T(2), q);
  if (q < T(0.5)) return xadd(xmul(q2, Pd), xmul(xsub(T(1), q2), up));
  const T inv = xdiv(T(1), q2);
  return xadd(xmul(Pd, inv), xmul(xmul(xsub(q2, T(1)), inv), Po));
}

// Bouzidi links of a TLBM_FLAG_CURVED cell: after the pull, f[opp_d] of every
// link (x, d) becomes the link value; a direction and its opposite are done
// together, so every read (pulled values, the cell's own stored P) precedes
// the writes.  With a force buffer the ledger sum_links c_d (P_d + value) is
// added to (mx, my, mz) in float64 (bfl_d3q19.py:339-377).
template <class L, typename T, typename SI, typename SO>
__device__ __forceinline__ void curved_links(const Domain<SI, SO>& d, long long cell, T (&f)[L::Q], double& mx,
                                             double& my, double& mz) {
  const float* __restrict__ lq = d.link_q + (long long)__ldg(d.link_row + cell) * L::Q;
  const long long N = d.n;
  const bool ledger = d.force != nullptr;
#pragma unroll
  for (int a = 1; a < L::Q; ++a) {
    const int b = L::opp(a);
    if (b < a) continue;
    const float qa = __ldg(lq + a), qb = __ldg(lq + b);
    if (!(qa > 0.0f) && !(qb > 0.0f)) continue;
    const T pa = Storage<SI>::load(ldg(d.fin + (long long)a * N + cell), weight<L, T>(a));
    const T pb = Storage<SI>::load(ldg(d.fin + (long long)b * N + cell), weight<L, T>(b));
    const T ua = f[a], ub = f[b];
    if (qa > 0.0f) {
      const T v = bfl_value(T(qa), pa, ua, pb);
      f[b] = v;
      if (ledger) {
        const double s = double(xadd(pa, v));
        mx += L::cx(a) * s;
        my += L::cy(a) * s;
        mz += L::cz(a) * s;
      }
    }
    if (qb > 0.0f) {
      const T v = bfl_value(T(qb), pb, ub, pa);
      f[a] = v;
      if (ledger) {
        const double s = double(xadd(pb, v));
        mx += L::cx(b) * s;
        my += L::cy(b) * s;
        mz += L::cz(b) * s;
      }
    }
  }
}

// Boundary conditions of one cell after the pull, in TensorLBM's order:
// Zou/He inlet / outlet planes, the far field, full-way (or moving-wall)
// bounce-back or the Bouzidi links of a curved wall, lid.  (mx, my, mz)
// collect the BFL force.  kCurved = false compiles the Bouzidi links out (the
// two-cells-per-thread kernels, which never run with link tables), kFar =
// false the far field (all but the far-field instantiations of those
// kernels).  The far field's zero-gradient outlet is the caller's: the
// x = nx-1 cell holds the post-stream populations of x = nx-2 when it gets here.
template <class L, typename T, typename SI, typename SO, bool kCurved = true, bool kFar = kCurved>
__device__ __forceinline__ void apply_boundaries(const Domain<SI, SO>& d, int x, int y, int z, long long cell,
                                                 uint8_t fl, T (&f)[L::Q], const BcParams<T>& bp, double& mx,
                                                 double& my, double& mz) {
  constexpr int Q = L::Q;
  const long long N = d.n;
  // Zou/He inlet / outlet planes
  if ((d.bc & TLBM_BC_ZH_INLET) && x == 0) {
    if constexpr (Q == 9) zou_he_inlet_d2q9(f, bp.u_in, bp.uy_in);
    else zou_he_inlet_3d<L>(f, bp.u_in, bp.uy_in, bp.uz_in, bp.one_minus_u);
  }
  if ((d.bc & TLBM_BC_ZH_OUTLET) && x == d.nx - 1) {
    if constexpr (Q == 9) zou_he_outlet_d2q9(f, bp.rho_out, bp.two_thirds_rho_out, bp.sixth_rho_out);
    else zou_he_outlet_3d<L>(f, bp.rho_out);
  }
  // far field: inlet plane, then the lateral planes (which win on the edges
  // of the outlet plane)
  if (kFar && (d.bc & TLBM_BC_FAR_FIELD)) {
    if (x == 0) {
      far_field_feq<L>(f, bp.ff_in[0], bp.ff_in[1], bp.ff_in[2]);
    } else if (y == 0 || y == d.ny - 1 || ((d.bc & TLBM_BC_FAR_FIELD_Z) && (z == 0 || z == d.nz - 1))) {
      far_field_feq<L>(f, bp.ff_u[0], bp.ff_u[1], bp.ff_u[2]);
    }
  }
  // full-way bounce-back; Ladd moving wall where flagged.  A moving obstacle
  // cell that is also a wall cell has SOLID cleared (wall XOR obstacle): it
  // takes the wall swap first, then the moving-wall pass, as
  // bounce_back(wall) followed by moving_wall_bounce_back(obstacle).
  if ((fl & TLBM_FLAG_MOVING) && d.wall_u) {
    const T* uw = static_cast<const T*>(d.wall_u);
    if (!(fl & TLBM_FLAG_SOLID)) bounce_back<L>(f);
    moving_wall_bounce_back<L>(f, uw[cell], uw[N + cell], L::DIM == 3 ? uw[2 * N + cell] : T(0));
  } else if (fl & TLBM_FLAG_SOLID) {
    bounce_back<L>(f);
  }
  if constexpr (L::DIM == 3 && kCurved) {
    if ((fl & TLBM_FLAG_CURVED) && d.link_q) curved_links<L>(d, cell, f, mx, my, mz);
  }
  // moving lid
  if ((d.bc & TLBM_BC_LID) && y == d.ny - 1) {
    if constexpr (Q == 9) moving_lid_d2q9(f, bp.u_lid);
    else if constexpr (Q == 19) moving_lid_d3q19(f, bp.u_lid);
  }
}

template <class L, typename SI, typename SO, int COLL, bool FORCED, typename T>
__device__ __forceinline__ void relax_fluid(const Domain<SI, SO>& d, long long cell, T (&f)[L::Q],
                                            const CollideParams<T>& cp);

// Collision of one cell (or the reversal of a half-way wall cell), the
// optional exact-difference linear force, and the non-finite status bit.
template <class L, typename SI, typename SO, int COLL, bool FORCED, typename T>
__device__ __forceinline__ void relax(const Domain<SI, SO>& d, long long cell, uint8_t fl, T (&f)[L::Q],
                                      const CollideParams<T>& cp) {
  if constexpr (COLL != TLBM_COLL_NONE) {
    if (fl & TLBM_FLAG_HALFWAY) {
      // pre-stream half-way wall: keep the populations, reversed, uncollided
      bounce_back<L>(f);
    } else {
      relax_fluid<L, SI, SO, COLL, FORCED>(d, cell, f, cp);
    }
  }
}

// The collision of a fluid cell, the optional force and the status bit.
template <class L, typename SI, typename SO, int COLL, bool FORCED, typename T>
__device__ __forceinline__ void relax_fluid(const Domain<SI, SO>& d, long long cell, T (&f)[L::Q],
                                            const CollideParams<T>& cp) {
  constexpr int Q = L::Q;
  if constexpr (COLL != TLBM_COLL_NONE) {
    {
      const bool has_tau = d.tau_field != nullptr;
      const T tau_cell = has_tau ? T(d.tau_field[cell]) : T(0);
      if constexpr (FORCED) {
        // exact-difference forcing of F = A rho u: collide, then add
        // feq(rho, (1 + A) u) - feq(rho, u) with the pre-collision moments
        T rho, ux, uy, uz;
        macroscopic_fused<L>(f, rho, ux, uy, uz);
        collide<L, COLL, T, Storage<SI>::kFast>(f, cp, tau_cell, has_tau);
        const T k = T(1) + cp.force_a;
        const T usq = ux * ux + uy * uy + uz * uz;
        const T usq_k = usq * k * k;
#pragma unroll
        for (int q = 0; q < Q; ++q)
          f[q] += feq_fused<L>(q, rho, ux * k, uy * k, uz * k, usq_k) - feq_fused<L>(q, rho, ux, uy, uz, usq);
      } else if constexpr (std::is_same<T, float>::value && packed_collision<L, COLL, Storage<SI>::kFast>()) {
        // the explicit-rounding form of the pair kernels, on one cell: the
        // same result bit for bit as a pair kernel gives this cell
        F1 g[Q];
#pragma unroll
        for (int q = 0; q < Q; ++q) g[q] = F1(f[q]);
        collide<L, COLL, F1, Storage<SI>::kFast>(g, pack_params<F1>(cp), F1(tau_cell), has_tau);
#pragma unroll
        for (int q = 0; q < Q; ++q) f[q] = g[q].v;
      } else {
        collide<L, COLL, T, Storage<SI>::kFast>(f, cp, tau_cell, has_tau);
      }
      if (d.status) {
        const T r = f[0];
        if (!(r == r) || r - r != T(0)) atomicOr(d.status, 1u);
      }
    }
  }
}

// Periodic pull of cell (x, y, z): f[q] = f_in[q, (x, y, z) - c_q]
template <class L, typename SI, typename SO, typename T>
__device__ __forceinline__ void pull_cell(const Domain<SI, SO>& d, int x, int y, int z, T (&f)[L::Q]) {
  const long long N = d.n;
  const int xm = (x == 0) ? d.nx - 1 : x - 1;
  const int xp = (x == d.nx - 1) ? 0 : x + 1;
  const int ym = (y == 0) ? d.ny - 1 : y - 1;
  const int yp = (y == d.ny - 1) ? 0 : y + 1;
  const int zm = (z == 0) ? d.nz - 1 : z - 1;
  const int zp = (z == d.nz - 1) ? 0 : z + 1;
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    const int sx = L::cx(q) > 0 ? xm : (L::cx(q) < 0 ? xp : x);
    const int sy = L::cy(q) > 0 ? ym : (L::cy(q) < 0 ? yp : y);
    const int sz = L::cz(q) > 0 ? zm : (L::cz(q) < 0 ? zp : z);
    const long long src = (long long)sz * d.plane + (long long)sy * d.nx + sx;
    f[q] = Storage<SI>::load(ldg(d.fin + (long long)q * N + src), weight<L, T>(q));
  }
}

// The update of cell (x, y, z) of one domain.  Every thread of a warp must
// call it (inactive ones with active = false) because the force reduction is
// warp-wide.
// PULL = true : gather from neighbours, boundaries, collide (COLL may be NONE)
// PULL = false: local collide / format conversion only (no boundaries)
// FORCED: add the exact-difference linear force after the collision (a
// separate instantiation, so that the unforced kernels carry none of it)
template <class L, typename SI, typename SO, int COLL, bool PULL, bool FORCED = false>
__device__ __forceinline__ void cell_update(const Domain<SI, SO>& d, int x, int y, int z, bool active,
                                            const CollideParams<typename Storage<SI>::T>& cp,
                                            const BcParams<typename Storage<SI>::T>& bp) {
  using T = typename Storage<SI>::T;
  constexpr int Q = L::Q;
  const long long N = d.n;
  const long long cell = (long long)z * d.plane + (long long)y * d.nx + x;
  const SI* __restrict__ fin = d.fin;
  SO* __restrict__ fout = d.fout;

  T f[Q];
  uint8_t fl = 0;
  if (active) {
    if constexpr (PULL) {
      pull_cell<L>(d, x, y, z, f);
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) f[q] = Storage<SI>::load(fin[(long long)q * N + cell], weight<L, T>(q));
    }
    if (d.flags) fl = d.flags[cell];
  }

  if constexpr (PULL) {
    // momentum-exchange force sample (post-stream, pre-bounce-back)
    if (d.force) {
      const bool ob = active && (fl & TLBM_FLAG_OBSTACLE);
      T mx = T(0), my = T(0), mz = T(0);
      if (ob) cell_momentum<L>(f, mx, my, mz);
      accumulate_force(d.force, __any_sync(0xffffffffu, ob), mx, my, mz);
    }
    // far field: the outlet plane takes the post-stream populations of x = nx-2
    // (after the force sample, as far_field_bc_* follows compute_obstacle_forces)
    if ((d.bc & TLBM_BC_FAR_FIELD) && active && x == d.nx - 1) pull_cell<L>(d, d.nx - 2, y, z, f);
    // boundaries; the ledger of Bouzidi links is reduced on its own
    double bx = 0.0, by = 0.0, bz = 0.0;
    if (active) apply_boundaries<L>(d, x, y, z, cell, fl, f, bp, bx, by, bz);
    if (d.force && d.link_q)
      accumulate_force(d.force, __any_sync(0xffffffffu, active && (fl & TLBM_FLAG_CURVED)), bx, by, bz, 1.0);
  }

  if (!active) return;
  relax<L, SI, SO, COLL, FORCED>(d, cell, fl, f, cp);
  // random bits of the stochastic rounding of half storage: a hash of the
  // cell and of this step's value of f[0] (so they change every step without
  // a seed), spread over the directions by a second multiply
  uint32_t h = 0;
  if constexpr (Storage<SO>::kShifted) h = fmix32(uint32_t(cell) * 0x9E3779B9u ^ __float_as_uint(float(f[0])));
#pragma unroll
  for (int q = 0; q < Q; ++q)
    fout[(long long)q * N + cell] = Storage<SO>::store(f[q], weight<L, T>(q), (h ^ (uint32_t(q) * 0x9E3779B9u)) * 0x85EBCA6Bu);
}

template <class L, typename SI, typename SO, int COLL, bool PULL, bool FORCED = false>
__global__ void __launch_bounds__(256) k_step(StepParams p, CollideParams<typename Storage<SI>::T> cp,
                                              BcParams<typename Storage<SI>::T> bp) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = p.z0 + int(blockIdx.z);
  Domain<SI, SO> d;
  d.fin = static_cast<const SI*>(p.f_in);
  d.fout = static_cast<SO*>(p.f_out);
  d.flags = p.flags;
  d.tau_field = p.tau_field;
  d.force = p.force;
  d.status = p.status;
  d.wall_u = p.wall_velocity;
  d.link_row = p.link_row;
  d.link_q = p.link_q;
  d.nx = p.nx;
  d.ny = p.ny;
  d.nz = p.nz;
  d.plane = p.plane;
  d.n = p.n;
  d.bc = p.bc;
  cell_update<L, SI, SO, COLL, PULL, FORCED>(d, x, y, z, (x < p.nx) && (y < p.ny), cp, bp);
}

// base + i elements as one wide multiply-add (mad.wide.s32), instead of a
// sign extension and a two-word add per address
template <typename E>
__device__ __forceinline__ E* at_offset(E* base, int i) {
  E* r;
  asm("mad.wide.s32 %0, %1, %2, %3;" : "=l"(r) : "r"(i), "n"(int(sizeof(E))), "l"(base));
  return r;
}

// Pulls of the pair kernel: the compute value, or for the deviation-form BGK
// (RAW) the stored deviation itself.
template <bool RAW, typename S>
__device__ __forceinline__ typename Storage<S>::T pull_value(S v, typename Storage<S>::T w) {
  if constexpr (RAW) return Storage<S>::load_raw(v);
  else return Storage<S>::load(v, w);
}
template <bool RAW, typename S, typename T>
__device__ __forceinline__ void pull_pair(typename PairIO<S>::V v, T w, T& a, T& b) {
  if constexpr (RAW) PairIO<S>::split_raw(v, a, b);
  else PairIO<S>::split(v, w, a, b);
}

// Interior cells of a shifted half format with BGK: the collision on the
// stored deviations, the per-cell tau, the status bit.
template <class L, typename SI, typename SO, typename T>
__device__ __forceinline__ void relax_deviation(const Domain<SI, SO>& d, long long cell, T (&g)[L::Q],
                                                const CollideParams<T>& cp) {
  const T om = d.tau_field ? rcp_fast(T(d.tau_field[cell])) : cp.inv_tau;
  collide_bgk_deviation<L>(g, om, T(Storage<SI>::kRaw));
  if (d.status) {
    const T r = g[0];
    if (!(r == r) || r - r != T(0)) atomicOr(d.status, 1u);
  }
}

// Interior cells of a shifted half format with BGK, both cells of the pair in
// packed arithmetic.
template <class L, typename S>
__device__ __forceinline__ void relax_deviation_pair(const Domain<S, S>& d, long long cell, float (&ga)[L::Q],
                                                     float (&gb)[L::Q], const CollideParams<float>& cp) {
  F2 g[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) g[q] = F2(ga[q], gb[q]);
  const F2 om = d.tau_field ? rcp_fast(F2(d.tau_field[cell], d.tau_field[cell + 1])) : F2(cp.inv_tau);
  collide_bgk_deviation<L>(g, om, F2(Storage<S>::kRaw));
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    ga[q] = g[q].a();
    gb[q] = g[q].b();
  }
  if (d.status) {
    const float ra = ga[0], rb = gb[0];
    if (!(ra == ra) || ra - ra != 0.0f || !(rb == rb) || rb - rb != 0.0f) atomicOr(d.status, 1u);
  }
}

// The collision of two fluid cells of a pair in packed arithmetic (the
// collisions packed_collision() admits), with the per-cell tau and the
// status bit.
template <class L, typename S, int COLL>
__device__ __forceinline__ void relax_fluid_pair(const Domain<S, S>& d, long long cell, float (&fa)[L::Q],
                                                 float (&fb)[L::Q], const CollideParams<float>& cp) {
  F2 g[L::Q];
#pragma unroll
  for (int q = 0; q < L::Q; ++q) g[q] = F2(fa[q], fb[q]);
  const bool has_tau = d.tau_field != nullptr;
  const F2 tau_cell = has_tau ? F2(d.tau_field[cell], d.tau_field[cell + 1]) : F2(0.0f);
  collide<L, COLL, F2, Storage<S>::kFast>(g, pack_params<F2>(cp), tau_cell, has_tau);
#pragma unroll
  for (int q = 0; q < L::Q; ++q) {
    fa[q] = g[q].a();
    fb[q] = g[q].b();
  }
  if (d.status) {
    const float ra = fa[0], rb = fb[0];
    if (!(ra == ra) || ra - ra != 0.0f || !(rb == rb) || rb - rb != 0.0f) atomicOr(d.status, 1u);
  }
}

// The collisions of the two cells of a pair after their boundaries (the
// half-way reversal of a wall cell included): one packed collision when PACK
// and both are fluid cells, else one per cell.  The two-buffer and the AA pair
// kernels share it, so their results stay identical.
template <class L, typename S, int COLL, bool FORCED, bool PACK>
__device__ __forceinline__ void relax_two(const Domain<S, S>& d, long long c, uint8_t fla, uint8_t flb,
                                          typename Storage<S>::T (&fa)[L::Q], typename Storage<S>::T (&fb)[L::Q],
                                          const CollideParams<typename Storage<S>::T>& cp) {
  if constexpr (PACK && COLL != TLBM_COLL_NONE) {
    if (!((fla | flb) & TLBM_FLAG_HALFWAY)) {
      relax_fluid_pair<L, S, COLL>(d, c, fa, fb, cp);
      return;
    }
  }
  relax<L, S, S, COLL, FORCED>(d, c, fla, fa, cp);
  relax<L, S, S, COLL, FORCED>(d, c + 1, flb, fb, cp);
}

// relax_two for two fluid cells without flags (a warp that took no boundary code)
template <class L, typename S, int COLL, bool FORCED, bool PACK>
__device__ __forceinline__ void relax_interior_two(const Domain<S, S>& d, long long c,
                                                   typename Storage<S>::T (&fa)[L::Q],
                                                   typename Storage<S>::T (&fb)[L::Q],
                                                   const CollideParams<typename Storage<S>::T>& cp) {
  if constexpr (COLL == TLBM_COLL_NONE) {
    return;
  } else if constexpr (PACK) {
    relax_fluid_pair<L, S, COLL>(d, c, fa, fb, cp);
  } else {
    relax_fluid<L, S, S, COLL, FORCED>(d, c, fa, cp);
    relax_fluid<L, S, S, COLL, FORCED>(d, c + 1, fb, cp);
  }
}

// Far field in the far-field instantiation of the pair kernels: the outlet
// cell x + 1 = nx - 1 takes the post-stream populations of its pair partner
// x = nx - 2 (after the force sample, as far_field_bc_* follows
// compute_obstacle_forces).  Called in the boundary branch only.
template <class L, bool FAR, typename S, typename T>
__device__ __forceinline__ void far_field_outlet_pair(const Domain<S, S>& d, int x, T (&fa)[L::Q], T (&fb)[L::Q]) {
  if constexpr (FAR) {
    if (x + 2 == d.nx) {
#pragma unroll
      for (int q = 0; q < L::Q; ++q) fb[q] = fa[q];
    }
  }
}

// Pair kernels: interior warps skip the boundary code on a warp-uniform branch
// (2-9 % faster for the D3Q19 collisions and the half formats on the sphere
// channel).  The D3Q27 legacy cumulant ran 4 % slower that way; it and the
// other collisions that run at the 128-register cap (Geier cumulant,
// cascaded) keep the per-cell path.
template <class L, int COLL>
__host__ __device__ constexpr bool uniform_edge_branch() {
  return !(L::Q == 27 && (COLL == TLBM_COLL_CUMULANT || COLL == TLBM_COLL_CUMULANT_GEIER ||
                          COLL == TLBM_COLL_CASCADED));
}

// Two cells per thread: (x, y, z) and (x + 1, y, z) with x even.  The pull
// of a direction with c_x = 0 is one aligned vector load of both cells'
// values, every store is one vector store, and the index arithmetic (32-bit
// offsets from the cell; the wrap is folded into six per-thread deltas) is
// shared by the two cells.  Each cell then takes exactly the per-cell path
// of k_step (boundaries, collision, forcing, status), so the float32 and
// float64 results are those of k_step bit for bit.
// Requires nx even, (Q/2 + 2) n < 2^31 (32-bit offsets), and f_in / f_out
// aligned to two values.
template <typename S>
__device__ __forceinline__ Domain<S, S> pair_domain(const StepParams& p) {
  Domain<S, S> d;
  d.fin = static_cast<const S*>(p.f_in);
  d.fout = static_cast<S*>(p.f_out);
  d.flags = p.flags;
  d.tau_field = p.tau_field;
  d.force = p.force;
  d.status = p.status;
  d.wall_u = p.wall_velocity;
  d.link_row = p.link_row;
  d.link_q = p.link_q;
  d.nx = p.nx;
  d.ny = p.ny;
  d.nz = p.nz;
  d.plane = p.plane;
  d.n = p.n;
  d.bc = p.bc;
  return d;
}

// Shifted float16 storage with BGK: interior warps collide on the stored
// deviations (no shift or scale around the loads and stores).  Not bf16: it
// saves only an add per value there and took the kernel past 64 registers
// (3 instead of 4 blocks per SM, 7 % slower).
template <class L, typename S, int COLL, bool FORCED>
__host__ __device__ constexpr bool pair_deviation_form() {
  return std::is_same<S, __half>::value && COLL == TLBM_COLL_BGK && !FORCED && uniform_edge_branch<L, COLL>();
}

template <class L, typename S, int COLL, bool FORCED, bool FAR = false>
__device__ __forceinline__ void pair_finish(const Domain<S, S>& d, const CollideParams<typename Storage<S>::T>& cp,
                                            const BcParams<typename Storage<S>::T>& bp, int x, int y, int z, int c,
                                            bool active, typename Storage<S>::T (&fa)[L::Q],
                                            typename Storage<S>::T (&fb)[L::Q], uint32_t fl2);

// The pair update of cells (x, y, z) and (x + 1, y, z) of domain d (x even):
// the pull (periodic wrap on every axis) and pair_finish.  Every thread of a
// warp must call it, inactive ones with active = false.
template <class L, typename S, int COLL, bool FORCED = false, bool FAR = false>
__device__ __forceinline__ void pair_update(const Domain<S, S>& d, const CollideParams<typename Storage<S>::T>& cp,
                                            const BcParams<typename Storage<S>::T>& bp, int x, int y, int z,
                                            bool active) {
  using T = typename Storage<S>::T;
  using IO = PairIO<S>;
  using V = typename IO::V;
  constexpr int Q = L::Q;
  constexpr int MID = Q / 2;
  constexpr bool kDev = pair_deviation_form<L, S, COLL, FORCED>();
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int plane = nx * ny;
  const int N = int(d.n);
  const int c = z * plane + y * nx + x;

  T fa[Q], fb[Q];
  uint32_t fl2 = 0;
  if (active) {
    // offsets from cell c to the source rows (periodic wrap on every axis)
    const int dym = (y == 0) ? (ny - 1) * nx : -nx;
    const int dyp = (y == ny - 1) ? -(ny - 1) * nx : nx;
    const int dzm = (L::DIM == 3) ? ((z == 0) ? (nz - 1) * plane : -plane) : 0;
    const int dzp = (L::DIM == 3) ? ((z == nz - 1) ? -(nz - 1) * plane : plane) : 0;
    const int dxm = (x == 0) ? nx - 1 : -1;      // cell x pulls c_x = +1 from x - 1
    const int dxp = (x + 2 == nx) ? 2 - nx : 2;  // cell x + 1 pulls c_x = -1 from x + 2
    // every source is a 32-bit element offset from this cell's value in
    // direction MID: (q - MID) N (the same for all threads) plus the row and
    // x deltas, so that each address is one wide multiply-add
    const S* __restrict__ pin = at_offset(d.fin + (long long)MID * N, c);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int o = (q - MID) * N + (L::cy(q) > 0 ? dym : (L::cy(q) < 0 ? dyp : 0)) +
                    (L::cz(q) > 0 ? dzm : (L::cz(q) < 0 ? dzp : 0));
      const T w = weight<L, T>(q);
      if (L::cx(q) == 0) {
        pull_pair<kDev, S>(__ldg(reinterpret_cast<const V*>(at_offset(pin, o))), w, fa[q], fb[q]);
      } else if (L::cx(q) > 0) {
        const int ia = o + dxm;
        fa[q] = pull_value<kDev>(ldg(at_offset(pin, ia)), w);
        fb[q] = pull_value<kDev>(ldg(at_offset(pin, o)), w);
      } else {
        const int ia = o + 1, ib = o + dxp;
        fa[q] = pull_value<kDev>(ldg(at_offset(pin, ia)), w);
        fb[q] = pull_value<kDev>(ldg(at_offset(pin, ib)), w);
      }
    }
    if (d.flags) fl2 = __ldg(reinterpret_cast<const uint16_t*>(at_offset(d.flags, c)));
  }
  pair_finish<L, S, COLL, FORCED, FAR>(d, cp, bp, x, y, z, c, active, fa, fb, fl2);
}

template <class L, typename S, int COLL, bool FORCED = false, bool FAR = false>
__device__ __forceinline__ void step_x2(const StepParams& p, const CollideParams<typename Storage<S>::T>& cp,
                                        const BcParams<typename Storage<S>::T>& bp) {
  const int x = 2 * int(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = p.z0 + int(blockIdx.z);
  pair_update<L, S, COLL, FORCED, FAR>(pair_domain<S>(p), cp, bp, x, y, z, (x < p.nx) && (y < p.ny));
}

// The pair update after the pull: boundary conditions, drag sample,
// collisions and the stores of cells c and c + 1 (x even).  fa / fb hold the
// pulled values (the stored deviations for the deviation-form BGK), fl2 the
// two flag bytes.  Every thread of a warp must call it (the force reduction
// and the edge test are warp-wide).
template <class L, typename S, int COLL, bool FORCED, bool FAR>
__device__ __forceinline__ void pair_finish(const Domain<S, S>& d, const CollideParams<typename Storage<S>::T>& cp,
                                            const BcParams<typename Storage<S>::T>& bp, int x, int y, int z, int c,
                                            bool active, typename Storage<S>::T (&fa)[L::Q],
                                            typename Storage<S>::T (&fb)[L::Q], uint32_t fl2) {
  using T = typename Storage<S>::T;
  using IO = PairIO<S>;
  using V = typename IO::V;
  constexpr int Q = L::Q;
  constexpr int MID = Q / 2;
  constexpr bool kDev = pair_deviation_form<L, S, COLL, FORCED>();
  // both cells' collisions as one stream of packed float32 instructions
  constexpr bool kPack = TLBM_PACK && std::is_same<T, float>::value && !FORCED &&
                         (kDev || packed_collision<L, COLL, Storage<S>::kFast>());
  const int nx = d.nx, ny = d.ny;
  const int N = int(d.n);
  const uint8_t fla = uint8_t(fl2), flb = uint8_t(fl2 >> 8);
  // whether any lane of the warp has a flagged cell or sits on a plane with a
  // condition: warps of the interior then skip all boundary code on a
  // warp-uniform branch
  // (the far-field instantiation adds its planes: x = 0, the outlet pair, the
  // y planes and with TLBM_BC_FAR_FIELD_Z the z planes)
  bool far = false;
  if constexpr (FAR)
    far = x == 0 || x + 2 == nx || y == 0 || y == ny - 1 ||
          ((d.bc & TLBM_BC_FAR_FIELD_Z) && (z == 0 || z == d.nz - 1));
  const bool edge = __any_sync(0xffffffffu, active && (fl2 != 0 || far || ((d.bc & TLBM_BC_ZH_INLET) && x == 0) ||
                                                       ((d.bc & TLBM_BC_ZH_OUTLET) && x + 2 == nx) ||
                                                       ((d.bc & TLBM_BC_LID) && y == ny - 1)));
  if constexpr (kDev) {
    if (edge) {
      // the boundary code and the drag work on the populations themselves
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        fa[q] = fma(fa[q], T(1) / T(Storage<S>::kRaw), weight<L, T>(q));
        fb[q] = fma(fb[q], T(1) / T(Storage<S>::kRaw), weight<L, T>(q));
      }
    }
  }

  // momentum-exchange force sample (post-stream, pre-bounce-back)
  if (d.force) {
    const bool oa = active && (fla & TLBM_FLAG_OBSTACLE), ob = active && (flb & TLBM_FLAG_OBSTACLE);
    double mx = 0.0, my = 0.0, mz = 0.0;
    if (oa) {
      T ax, ay, az;
      cell_momentum<L>(fa, ax, ay, az);
      mx = double(ax), my = double(ay), mz = double(az);
    }
    if (ob) {
      T bx, by, bz;
      cell_momentum<L>(fb, bx, by, bz);
      mx += double(bx), my += double(by), mz += double(bz);
    }
    accumulate_force(d.force, __any_sync(0xffffffffu, oa || ob), mx, my, mz);
  }
  if (!active) return;
  if constexpr (!uniform_edge_branch<L, COLL>()) {
    double unused_x = 0.0, unused_y = 0.0, unused_z = 0.0;
    far_field_outlet_pair<L, FAR>(d, x, fa, fb);
    apply_boundaries<L, T, S, S, false, FAR>(d, x, y, z, (long long)c, fla, fa, bp, unused_x, unused_y, unused_z);
    apply_boundaries<L, T, S, S, false, FAR>(d, x + 1, y, z, (long long)c + 1, flb, fb, bp, unused_x, unused_y,
                                             unused_z);
    relax_two<L, S, COLL, FORCED, kPack>(d, (long long)c, fla, flb, fa, fb, cp);
  } else if constexpr (kDev) {
    bool keep_a = false, keep_b = false;   // half-way wall cells: reversed, not collided
    if (edge) {
      double unused_x = 0.0, unused_y = 0.0, unused_z = 0.0;
      far_field_outlet_pair<L, FAR>(d, x, fa, fb);
      apply_boundaries<L, T, S, S, false, FAR>(d, x, y, z, (long long)c, fla, fa, bp, unused_x, unused_y, unused_z);
      apply_boundaries<L, T, S, S, false, FAR>(d, x + 1, y, z, (long long)c + 1, flb, fb, bp, unused_x, unused_y,
                                               unused_z);
      if (fla & TLBM_FLAG_HALFWAY) {
        bounce_back<L>(fa);
        keep_a = true;
      }
      if (flb & TLBM_FLAG_HALFWAY) {
        bounce_back<L>(fb);
        keep_b = true;
      }
      if (!keep_a) relax_fluid<L, S, S, COLL, FORCED>(d, (long long)c, fa, cp);
      if (!keep_b) relax_fluid<L, S, S, COLL, FORCED>(d, (long long)c + 1, fb, cp);
#pragma unroll
      for (int q = 0; q < Q; ++q) {   // back to the stored deviations
        fa[q] = (fa[q] - weight<L, T>(q)) * T(Storage<S>::kRaw);
        fb[q] = (fb[q] - weight<L, T>(q)) * T(Storage<S>::kRaw);
      }
    } else if constexpr (kPack) {
      relax_deviation_pair<L>(d, (long long)c, fa, fb, cp);
    } else {
      relax_deviation<L>(d, (long long)c, fa, cp);
      relax_deviation<L>(d, (long long)c + 1, fb, cp);
    }
  } else if (edge) {
    double unused_x = 0.0, unused_y = 0.0, unused_z = 0.0;
    far_field_outlet_pair<L, FAR>(d, x, fa, fb);
    apply_boundaries<L, T, S, S, false, FAR>(d, x, y, z, (long long)c, fla, fa, bp, unused_x, unused_y, unused_z);
    apply_boundaries<L, T, S, S, false, FAR>(d, x + 1, y, z, (long long)c + 1, flb, fb, bp, unused_x, unused_y,
                                             unused_z);
    relax_two<L, S, COLL, FORCED, kPack>(d, (long long)c, fla, flb, fa, fb, cp);
  } else {
    relax_interior_two<L, S, COLL, FORCED, kPack>(d, (long long)c, fa, fb, cp);   // no flag in the warp
  }

  // one hash per pair of its index and of this step's f_0 values (so the bits
  // change every step without a seed); NaN / Inf convert exactly whatever the bits
  uint32_t h = 0;
  if constexpr (Storage<S>::kShifted)
    h = fmix32(uint32_t(c) * 0x9E3779B9u ^ __float_as_uint(float(fa[0])) ^
               (__float_as_uint(float(fb[0])) * 0x85EBCA6Bu));
  S* __restrict__ pout = at_offset(d.fout + (long long)MID * N, c);
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if constexpr (kDev)
      __stwb(reinterpret_cast<V*>(at_offset(pout, (q - MID) * N)), IO::join_raw(fa[q], fb[q], h, q));
    else
      __stwb(reinterpret_cast<V*>(at_offset(pout, (q - MID) * N)), IO::join(fa[q], fb[q], weight<L, T>(q), h, q));
  }
}

// Resident blocks of 256 threads per SM that the pair kernel is compiled for
// (the register cap __launch_bounds__ derives from it); 0 = no cap.
template <class L, typename S, int COLL>
__host__ __device__ constexpr int x2_min_blocks() {
  constexpr bool f64 = std::is_same<S, double>::value;
  constexpr bool shifted = std::is_same<S, __half>::value || std::is_same<S, __nv_bfloat16>::value;
  if (L::Q == 19 && COLL == TLBM_COLL_MRT && !f64) return shifted ? TLBM_MINB_MRT_HALF : TLBM_MINB_MRT;
  if (L::Q == 19 && COLL == TLBM_COLL_BGK && shifted) return TLBM_MINB_BGK_HALF;
  if (L::Q == 27 && COLL == TLBM_COLL_CUMULANT && !f64) return TLBM_MINB_CUM;
  return 0;
}

template <class L, typename S, int COLL, bool FORCED = false, bool FAR = false>
__global__ void __launch_bounds__(256) k_step_x2(StepParams p, CollideParams<typename Storage<S>::T> cp,
                                                 BcParams<typename Storage<S>::T> bp) {
  step_x2<L, S, COLL, FORCED, FAR>(p, cp, bp);
}

// The collisions with a far-field instantiation of the pair kernel (float32
// populations); other far-field steps run the one-cell kernel.
template <class L, typename S, int COLL>
__host__ __device__ constexpr bool far_pair() {
  return std::is_same<S, float>::value && (COLL == TLBM_COLL_BGK || COLL == TLBM_COLL_MRT || COLL == TLBM_COLL_TRT ||
                                          COLL == TLBM_COLL_RLBM || COLL == TLBM_COLL_SMAGORINSKY);
}
// the same kernel compiled for MINB resident blocks per SM
template <class L, typename S, int COLL, int MINB, bool FAR = false>
__global__ void __launch_bounds__(256, MINB) k_step_x2_capped(StepParams p, CollideParams<typename Storage<S>::T> cp,
                                                               BcParams<typename Storage<S>::T> bp) {
  step_x2<L, S, COLL, false, FAR>(p, cp, bp);
}

}  // namespace tlbm

#include "tlbm_rows.cuh"

namespace tlbm {

// Whether the pair kernel can run this step: no Bouzidi link tables, no far
// field unless far_ok (its own instantiation), nx even (pairs never straddle
// a row), offsets of +-(Q/2 + 1) n within 32 bits, and both population
// buffers (and the flags) aligned to two values.
template <class L, typename S>
inline bool pair_layout_ok(const StepParams& p, bool far_ok = false) {
  const auto al = [](const void* ptr, size_t a) { return (reinterpret_cast<uintptr_t>(ptr) % a) == 0; };
  return (p.nx % 2 == 0) && p.link_q == nullptr && (far_ok || !(p.bc & TLBM_BC_FAR_FIELD)) &&
         (long long)(L::Q / 2 + 2) * p.n < (1LL << 31) && al(p.f_in, 2 * sizeof(S)) && al(p.f_out, 2 * sizeof(S)) &&
         (p.flags == nullptr || al(p.flags, 2));
}

inline void step_launch_shape(int nx, int ny, int nz, dim3& grid, dim3& block) {
  int bx = 32;
  while (bx < nx && bx < 256) bx <<= 1;
  int by = 256 / bx;
  block = dim3(bx, by, 1);
  grid = dim3((nx + bx - 1) / bx, (ny + by - 1) / by, nz);
}

template <class L, typename SI, typename SO, int COLL, bool PULL, bool FORCED = false>
int launch_step(const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  using T = typename Storage<SI>::T;
  dim3 grid, block;
  step_launch_shape(p.nx, p.ny, p.z_count, grid, block);
  CollideParams<T> cp = make_collide_params<T>(d.tau, d.s_e, d.s_eps, d.s_q, d.s_pi, d.omega_b, d.omega_odd,
                                               d.omega_even, d.c_smag);
  cp.force_a = T(d.force_lin);
  if (d.collision == TLBM_COLL_TRT) set_trt_rates(cp, d.tau, d.lambda_trt);
  if (d.cm_s5 >= 0.0) cp.cm_s5 = T(d.cm_s5);
  if (d.cm_s6 >= 0.0) cp.cm_s6 = T(d.cm_s6);
  const BcParams<T> bp = make_bc_params<T>(d.u_in[0], d.u_in[1], d.u_in[2], d.rho_out, d.u_lid, d.ff_inlet_du);
  // the forced instantiations stay on one cell per thread: two cells with
  // the pre-collision moments held for the force need 121 registers (2 blocks
  // per SM) and ran slower than k_step (26.8 against 28.0 GLUPS, forced
  // Smagorinsky at 256^3)
  if constexpr (PULL && !FORCED && std::is_same<SI, SO>::value) {
    int st = TLBM_OK;
    if (launch_rows<L, SI, COLL>(p, cp, bp, s, st)) return st;
    if constexpr (far_pair<L, SI, COLL>()) {
      if ((p.bc & TLBM_BC_FAR_FIELD) && pair_layout_ok<L, SI>(p, true)) {
        step_launch_shape(p.nx / 2, p.ny, p.z_count, grid, block);
        constexpr int minb = x2_min_blocks<L, SI, COLL>();
        if constexpr (minb > 0) k_step_x2_capped<L, SI, COLL, minb, true><<<grid, block, 0, s>>>(p, cp, bp);
        else k_step_x2<L, SI, COLL, false, true><<<grid, block, 0, s>>>(p, cp, bp);
        return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
      }
    }
    if (pair_layout_ok<L, SI>(p)) {
      step_launch_shape(p.nx / 2, p.ny, p.z_count, grid, block);
      constexpr int minb = x2_min_blocks<L, SI, COLL>();
      if constexpr (minb > 0) k_step_x2_capped<L, SI, COLL, minb><<<grid, block, 0, s>>>(p, cp, bp);
      else k_step_x2<L, SI, COLL, FORCED><<<grid, block, 0, s>>>(p, cp, bp);
      return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
    }
  }
  k_step<L, SI, SO, COLL, PULL, FORCED><<<grid, block, 0, s>>>(p, cp, bp);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

}  // namespace tlbm

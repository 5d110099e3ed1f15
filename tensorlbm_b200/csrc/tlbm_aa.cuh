// AA-pattern (in-place) time step: one population buffer instead of two.
//
// Slot q of cell x holds, between steps, either the natural layout (the
// populations that streamed into x, not yet bounded: "after an odd step") or
// the swapped layout (slot opp(q) holds x's post-collision population q:
// "after an even step").  An even step reads a cell's own natural slots and
// writes its post-collision values to the opposite slots of the same cell;
// an odd step gathers population q from slot opp(q) of x - c_q and writes its
// result q to slot q of x + c_q.  In both, a thread writes exactly the Q
// locations it read (for odd steps: (x + c_q, q) = (x - c_j, opp j) with
// j = opp q), so the update is race-free in place.  Between the two memory
// patterns every cell takes the per-cell path of k_step (force sample,
// boundaries, collision, forcing, status).
//
// The two-buffer step keeps P_{n-1} to read out the TensorLBM-phase field
// S_n = BC(stream(P_{n-1})); one buffer cannot, so the AA pipeline runs one
// collision behind: the load stores S_0 as it is (layout "loaded"), the first
// launch collides it in place without boundaries (the two-buffer load pass),
// launch n >= 2 is the regular step from P_{n-2}, and the readout of the
// buffer after n launches is S_n, equal to the two-buffer field bit for bit.
// Launch n samples the force of step n - 1 (the readout samples step n).
#pragma once

#include "tlbm_step.cuh"

namespace tlbm {

// READ: 0 = the cell's own natural slots, 1 = gather from the neighbours'
// swapped slots.  WRITE: 0 = own slots, swapped; 1 = scatter to the
// neighbours' natural slots; 2 = own slots, natural.  BC: 1 = the force
// sample and the boundaries after the read; 0 = neither.
enum { kAaReadOwn = 0, kAaReadGather = 1 };
enum { kAaWriteSwapped = 0, kAaWriteScatter = 1, kAaWriteNatural = 2 };
enum { kAaNoBc = 0, kAaBc = 1 };

template <class L, typename SI, typename SO, int COLL, int READ, int WRITE, int BC, bool FORCED = false>
__global__ void __launch_bounds__(256) k_step_aa(StepParams p, CollideParams<typename Storage<SI>::T> cp,
                                                 BcParams<typename Storage<SI>::T> bp) {
  using T = typename Storage<SI>::T;
  constexpr int Q = L::Q;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool active = (x < p.nx) && (y < p.ny);
  Domain<SI, SO> d;
  d.fin = static_cast<const SI*>(p.f_in);
  d.fout = static_cast<SO*>(p.f_out);
  d.flags = p.flags;
  d.tau_field = p.tau_field;
  d.force = p.force;
  d.status = p.status;
  d.wall_u = p.wall_velocity;
  d.link_row = nullptr;
  d.link_q = nullptr;
  d.nx = p.nx;
  d.ny = p.ny;
  d.nz = p.nz;
  d.plane = p.plane;
  d.n = p.n;
  d.bc = p.bc;
  const long long N = d.n;
  const long long cell = (long long)z * d.plane + (long long)y * d.nx + x;
  // periodic neighbours x - c and x + c along each axis
  const int xm = (x == 0) ? d.nx - 1 : x - 1, xp = (x == d.nx - 1) ? 0 : x + 1;
  const int ym = (y == 0) ? d.ny - 1 : y - 1, yp = (y == d.ny - 1) ? 0 : y + 1;
  const int zm = (z == 0) ? d.nz - 1 : z - 1, zp = (z == d.nz - 1) ? 0 : z + 1;
  // cell index of x + sign * c_q
  const auto shifted = [&](int q, int sign) -> long long {
    const int cx = sign * L::cx(q), cy = sign * L::cy(q), cz = sign * L::cz(q);
    const int sx = cx > 0 ? xp : (cx < 0 ? xm : x);
    const int sy = cy > 0 ? yp : (cy < 0 ? ym : y);
    const int sz = cz > 0 ? zp : (cz < 0 ? zm : z);
    return (long long)sz * d.plane + (long long)sy * d.nx + sx;
  };

  T f[Q];
  uint8_t fl = 0;
  if (active) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const SI v = (READ == kAaReadOwn) ? d.fin[(long long)q * N + cell]
                                        : d.fin[(long long)L::opp(q) * N + shifted(q, -1)];
      f[q] = Storage<SI>::load(v, weight<L, T>(q));
    }
    if (d.flags) fl = d.flags[cell];
  }
  if constexpr (BC == kAaBc) {
    if (d.force) {
      const bool ob = active && (fl & TLBM_FLAG_OBSTACLE);
      T mx = T(0), my = T(0), mz = T(0);
      if (ob) cell_momentum<L>(f, mx, my, mz);
      accumulate_force(d.force, __any_sync(0xffffffffu, ob), mx, my, mz);
    }
    double ux = 0.0, uy = 0.0, uz = 0.0;  // no Bouzidi links in the AA pattern
    if (active) apply_boundaries<L, T, SI, SO, false>(d, x, y, z, cell, fl, f, bp, ux, uy, uz);
  }
  if (!active) return;
  relax<L, SI, SO, COLL, FORCED>(d, cell, fl, f, cp);
  uint32_t h = 0;
  if constexpr (Storage<SO>::kShifted) h = fmix32(uint32_t(cell) * 0x9E3779B9u ^ __float_as_uint(float(f[0])));
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const SO v = Storage<SO>::store(f[q], weight<L, T>(q), (h ^ (uint32_t(q) * 0x9E3779B9u)) * 0x85EBCA6Bu);
    if (WRITE == kAaWriteSwapped) d.fout[(long long)L::opp(q) * N + cell] = v;
    else if (WRITE == kAaWriteScatter) d.fout[(long long)q * N + shifted(q, 1)] = v;
    else d.fout[(long long)q * N + cell] = v;
  }
}

// The two AA steps with two cells per thread ((x, x + 1), x even), as the
// two-buffer pair kernel does it: 32-bit offsets from a base at direction
// Q/2, vector accesses where both cells' slots are adjacent (every access of
// an even step; the c_x = 0 directions of an odd step), two scalar accesses
// otherwise.  Same per-cell path and the same packed stochastic rounding as
// k_step_x2.  Requires what pair_layout_ok checks.
template <class L, typename S, int COLL, int READ, int WRITE, bool FORCED = false>
__device__ __forceinline__ void step_aa_x2(const StepParams& p, const CollideParams<typename Storage<S>::T>& cp,
                                           const BcParams<typename Storage<S>::T>& bp) {
  using T = typename Storage<S>::T;
  using IO = PairIO<S>;
  using V = typename IO::V;
  constexpr int Q = L::Q;
  constexpr int MID = Q / 2;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int x = 2 * int(blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  const bool active = (x < nx) && (y < ny);
  const int plane = nx * ny;
  const int N = int(p.n);
  const int c = z * plane + y * nx + x;
  Domain<S, S> d;
  d.fin = static_cast<const S*>(p.f_in);
  d.fout = static_cast<S*>(p.f_out);
  d.flags = p.flags;
  d.tau_field = p.tau_field;
  d.force = p.force;
  d.status = p.status;
  d.wall_u = p.wall_velocity;
  d.link_row = nullptr;
  d.link_q = nullptr;
  d.nx = nx;
  d.ny = ny;
  d.nz = nz;
  d.plane = p.plane;
  d.n = p.n;
  d.bc = p.bc;
  // row deltas to y -+ 1 and z -+ 1 (periodic) and the x deltas of the pair
  const int dym = (y == 0) ? (ny - 1) * nx : -nx;
  const int dyp = (y == ny - 1) ? -(ny - 1) * nx : nx;
  const int dzm = (L::DIM == 3) ? ((z == 0) ? (nz - 1) * plane : -plane) : 0;
  const int dzp = (L::DIM == 3) ? ((z == nz - 1) ? -(nz - 1) * plane : plane) : 0;
  const int dxm = (x == 0) ? nx - 1 : -1;      // x - 1
  const int dxp = (x + 2 == nx) ? 2 - nx : 2;  // x + 2
  // offset of the row of (x, y, z) + sign * c_q
  const auto row = [&](int q, int sign) -> int {
    const int cy = sign * L::cy(q), cz = sign * L::cz(q);
    return (cy > 0 ? dyp : (cy < 0 ? dym : 0)) + (cz > 0 ? dzp : (cz < 0 ? dzm : 0));
  };
  S* __restrict__ base = at_offset(d.fout + (long long)MID * N, c);  // f_in == f_out
  const S* __restrict__ rbase = base;

  T fa[Q], fb[Q];
  uint32_t fl2 = 0;
  if (active) {
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const T w = weight<L, T>(q);
      if (READ == kAaReadOwn) {
        IO::split(__ldg(reinterpret_cast<const V*>(at_offset(rbase, (q - MID) * N))), w, fa[q], fb[q]);
      } else {
        // population q of cell x comes from slot opp(q) of x - c_q
        const int o = (L::opp(q) - MID) * N + row(q, -1);
        if (L::cx(q) == 0) {
          IO::split(__ldg(reinterpret_cast<const V*>(at_offset(rbase, o))), w, fa[q], fb[q]);
        } else if (L::cx(q) > 0) {
          fa[q] = Storage<S>::load(ldg(at_offset(rbase, o + dxm)), w);
          fb[q] = Storage<S>::load(ldg(at_offset(rbase, o)), w);
        } else {
          fa[q] = Storage<S>::load(ldg(at_offset(rbase, o + 1)), w);
          fb[q] = Storage<S>::load(ldg(at_offset(rbase, o + dxp)), w);
        }
      }
    }
    if (d.flags) fl2 = __ldg(reinterpret_cast<const uint16_t*>(at_offset(d.flags, c)));
  }
  const uint8_t fla = uint8_t(fl2), flb = uint8_t(fl2 >> 8);
  // warp-uniform: does any lane need boundary code (a flag or a condition plane)
  const bool edge = __any_sync(0xffffffffu, active && (fl2 != 0 || ((p.bc & TLBM_BC_ZH_INLET) && x == 0) ||
                                                       ((p.bc & TLBM_BC_ZH_OUTLET) && x + 2 == nx) ||
                                                       ((p.bc & TLBM_BC_LID) && y == ny - 1)));
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
  // packed collisions exactly where the two-buffer pair kernel packs them
  constexpr bool kPack = TLBM_PACK && std::is_same<T, float>::value && !FORCED &&
                         packed_collision<L, COLL, Storage<S>::kFast>();
  if (!uniform_edge_branch<L, COLL>() || edge) {
    double unused_x = 0.0, unused_y = 0.0, unused_z = 0.0;
    apply_boundaries<L, T, S, S, false>(d, x, y, z, (long long)c, fla, fa, bp, unused_x, unused_y, unused_z);
    apply_boundaries<L, T, S, S, false>(d, x + 1, y, z, (long long)c + 1, flb, fb, bp, unused_x, unused_y, unused_z);
    relax_two<L, S, COLL, FORCED, kPack>(d, (long long)c, fla, flb, fa, fb, cp);
  } else {
    relax_interior_two<L, S, COLL, FORCED, kPack>(d, (long long)c, fa, fb, cp);
  }
  uint32_t h = 0;
  if constexpr (Storage<S>::kShifted)
    h = fmix32(uint32_t(c) * 0x9E3779B9u ^ __float_as_uint(float(fa[0])) ^
               (__float_as_uint(float(fb[0])) * 0x85EBCA6Bu));
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const V v = IO::join(fa[q], fb[q], weight<L, T>(q), h, q);
    if (WRITE == kAaWriteSwapped) {
      __stwb(reinterpret_cast<V*>(at_offset(base, (L::opp(q) - MID) * N)), v);
    } else {
      // population q of cell x goes to slot q of x + c_q
      const int o = (q - MID) * N + row(q, 1);
      if (L::cx(q) == 0) {
        __stwb(reinterpret_cast<V*>(at_offset(base, o)), v);
      } else {
        const S* parts = reinterpret_cast<const S*>(&v);
        if (L::cx(q) > 0) {
          *at_offset(base, o + 1) = parts[0];
          *at_offset(base, o + dxp) = parts[1];
        } else {
          *at_offset(base, o + dxm) = parts[0];
          *at_offset(base, o) = parts[1];
        }
      }
    }
  }
}

// Resident blocks per SM the AA pair kernel is compiled for: the caps of the
// two-buffer kernel, except the D3Q19 MRT (the AA addressing adds registers,
// and the capped form spilled and ran slower)
template <class L, typename S, int COLL>
__host__ __device__ constexpr int aa_x2_min_blocks() {
  return (L::Q == 19 && COLL == TLBM_COLL_MRT) ? TLBM_MINB_AA_MRT : x2_min_blocks<L, S, COLL>();
}

template <class L, typename S, int COLL, int READ, int WRITE, bool FORCED = false>
__global__ void __launch_bounds__(256) k_step_aa_x2(StepParams p, CollideParams<typename Storage<S>::T> cp,
                                                    BcParams<typename Storage<S>::T> bp) {
  step_aa_x2<L, S, COLL, READ, WRITE, FORCED>(p, cp, bp);
}
// the same kernel compiled for MINB resident blocks per SM (x2_min_blocks)
template <class L, typename S, int COLL, int READ, int WRITE, int MINB>
__global__ void __launch_bounds__(256, MINB) k_step_aa_x2_capped(StepParams p, CollideParams<typename Storage<S>::T> cp,
                                                                  BcParams<typename Storage<S>::T> bp) {
  step_aa_x2<L, S, COLL, READ, WRITE, false>(p, cp, bp);
}

template <class L, typename SI, typename SO, int COLL, int READ, int WRITE, int BC, bool FORCED = false>
int launch_aa(const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  using T = typename Storage<SI>::T;
  dim3 grid, block;
  step_launch_shape(p.nx, p.ny, p.nz, grid, block);
  CollideParams<T> cp = make_collide_params<T>(d.tau, d.s_e, d.s_eps, d.s_q, d.s_pi, d.omega_b, d.omega_odd,
                                               d.omega_even, d.c_smag);
  cp.force_a = T(d.force_lin);
  if (d.collision == TLBM_COLL_TRT) set_trt_rates(cp, d.tau, d.lambda_trt);
  if (d.cm_s5 >= 0.0) cp.cm_s5 = T(d.cm_s5);
  if (d.cm_s6 >= 0.0) cp.cm_s6 = T(d.cm_s6);
  const BcParams<T> bp = make_bc_params<T>(d.u_in[0], d.u_in[1], d.u_in[2], d.rho_out, d.u_lid);
  // the two unforced steps (boundaries, same storage, own-swapped or
  // gather-scatter) run two cells per thread when the layout allows it;
  // forced steps keep one cell per thread, as the two-buffer step does
  constexpr bool kStep = BC == kAaBc && !FORCED && std::is_same<SI, SO>::value && COLL != TLBM_COLL_NONE &&
                         ((READ == kAaReadOwn && WRITE == kAaWriteSwapped) ||
                          (READ == kAaReadGather && WRITE == kAaWriteScatter));
  if constexpr (kStep) {
    if (pair_layout_ok<L, SI>(p)) {
      step_launch_shape(p.nx / 2, p.ny, p.nz, grid, block);
      constexpr int minb = aa_x2_min_blocks<L, SI, COLL>();
      if constexpr (minb > 0) k_step_aa_x2_capped<L, SI, COLL, READ, WRITE, minb><<<grid, block, 0, s>>>(p, cp, bp);
      else k_step_aa_x2<L, SI, COLL, READ, WRITE, FORCED><<<grid, block, 0, s>>>(p, cp, bp);
      return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
    }
  }
  k_step_aa<L, SI, SO, COLL, READ, WRITE, BC, FORCED><<<grid, block, 0, s>>>(p, cp, bp);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

// mode: 0 even step, 1 odd step, 5 first step from the loaded layout (in
// place, S -> S); 2 load (the TensorLBM-phase S_0 in the compute type -> S,
// as it is); 3 / 4 / 6 the TensorLBM-phase field of a natural / swapped /
// loaded buffer (S -> compute type, into another buffer; with a force buffer
// the force sample of that state).
template <class L, typename S, int COLL, bool FORCED = false>
int dispatch_aa_mode(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  using T = typename Storage<S>::T;
  switch (mode) {
    case 0: return launch_aa<L, S, S, COLL, kAaReadOwn, kAaWriteSwapped, kAaBc, FORCED>(p, d, s);
    case 1: return launch_aa<L, S, S, COLL, kAaReadGather, kAaWriteScatter, kAaBc, FORCED>(p, d, s);
    case 5: return launch_aa<L, S, S, COLL, kAaReadOwn, kAaWriteSwapped, kAaNoBc, FORCED>(p, d, s);
    case 2:
      if constexpr (FORCED || COLL != TLBM_COLL_BGK) return TLBM_ERR_UNSUPPORTED;
      else return launch_aa<L, T, S, TLBM_COLL_NONE, kAaReadOwn, kAaWriteNatural, kAaNoBc>(p, d, s);
    case 3:
      if constexpr (FORCED || COLL != TLBM_COLL_BGK) return TLBM_ERR_UNSUPPORTED;
      else return launch_aa<L, S, T, TLBM_COLL_NONE, kAaReadOwn, kAaWriteNatural, kAaBc>(p, d, s);
    case 4:
      if constexpr (FORCED || COLL != TLBM_COLL_BGK) return TLBM_ERR_UNSUPPORTED;
      else return launch_aa<L, S, T, TLBM_COLL_NONE, kAaReadGather, kAaWriteNatural, kAaBc>(p, d, s);
    case 6:
      if constexpr (FORCED || COLL != TLBM_COLL_BGK) return TLBM_ERR_UNSUPPORTED;
      else return launch_aa<L, S, T, TLBM_COLL_NONE, kAaReadOwn, kAaWriteNatural, kAaNoBc>(p, d, s);
    default: return TLBM_ERR_ARG;
  }
}

template <class L, typename S>
int dispatch_aa_collision(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  // the load and the readouts (modes 2, 3, 4, 6) do not collide: one instantiation serves all collisions
  const bool steps = (mode == 0 || mode == 1 || mode == 5);
  const int coll = steps ? d.collision : TLBM_COLL_BGK;
  if (d.force_lin != 0.0 && steps) {
    if constexpr (!std::is_same<S, float>::value) return TLBM_ERR_DTYPE;
    else {
      switch (coll) {
        case TLBM_COLL_BGK: return dispatch_aa_mode<L, S, TLBM_COLL_BGK, true>(mode, p, d, s);
        case TLBM_COLL_MRT: return dispatch_aa_mode<L, S, TLBM_COLL_MRT, true>(mode, p, d, s);
        case TLBM_COLL_SMAGORINSKY: return dispatch_aa_mode<L, S, TLBM_COLL_SMAGORINSKY, true>(mode, p, d, s);
        default: return TLBM_ERR_UNSUPPORTED;
      }
    }
  }
  switch (coll) {
    case TLBM_COLL_BGK: return dispatch_aa_mode<L, S, TLBM_COLL_BGK>(mode, p, d, s);
    case TLBM_COLL_MRT: return dispatch_aa_mode<L, S, TLBM_COLL_MRT>(mode, p, d, s);
    case TLBM_COLL_TRT: return dispatch_aa_mode<L, S, TLBM_COLL_TRT>(mode, p, d, s);
    case TLBM_COLL_RLBM: return dispatch_aa_mode<L, S, TLBM_COLL_RLBM>(mode, p, d, s);
    case TLBM_COLL_SMAGORINSKY: return dispatch_aa_mode<L, S, TLBM_COLL_SMAGORINSKY>(mode, p, d, s);
    case TLBM_COLL_CUMULANT:
      if constexpr (L::Q == 27) return dispatch_aa_mode<L, S, TLBM_COLL_CUMULANT>(mode, p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    case TLBM_COLL_CASCADED:
      if constexpr (L::Q != 9) return dispatch_aa_mode<L, S, TLBM_COLL_CASCADED>(mode, p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    default: return TLBM_ERR_UNSUPPORTED;
  }
}

template <class L>
int dispatch_aa(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  switch (d.dtype) {
    case TLBM_F32: return dispatch_aa_collision<L, float>(mode, p, d, s);
    case TLBM_F16_SHIFTED: return dispatch_aa_collision<L, __half>(mode, p, d, s);
    case TLBM_BF16_SHIFTED: return dispatch_aa_collision<L, __nv_bfloat16>(mode, p, d, s);
    default: return TLBM_ERR_DTYPE;
  }
}

// defined in aa_d2q9.cu / aa_d3q19.cu / aa_d3q27.cu
int dispatch_aa_d2q9(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s);
int dispatch_aa_d3q19(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s);
int dispatch_aa_d3q27(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s);

}  // namespace tlbm

// Batched runner: many independent small domains advanced together.
//
// The domains (each its own (Q, ny, nx) block at f_offset in one packed
// population buffer, its flag bytes at cell_offset in one packed flag buffer)
// are cut into tiles of tile_x x tile_y cells.  A step is the fused per-cell
// update (cell_update, identical arithmetic to tlbm_step) over every tile, so
// each domain evolves exactly as it would alone.
//
// Two execution modes:
//  * tlbm_batch_step: one launch per step, grid = tiles (the caller replays a
//    CUDA graph of these launches);
//  * tlbm_batch_run: one persistent cooperative launch that runs nsteps steps,
//    each CTA striding over the tile list, with a grid barrier between steps
//    (launched with cudaLaunchKernelEx, so it can be captured in a CUDA graph).
//    The barrier spins a bounded number of times; on expiry the kernel records
//    TLBM_ERR_TIMEOUT in *status and every CTA returns.
#include <cooperative_groups.h>

#include "tlbm_step.cuh"

namespace tlbm {
namespace {

template <class L, typename T>
__device__ __forceinline__ void domain_params(const tlbm_batch_domain& dm, CollideParams<T>& cp, BcParams<T>& bp) {
  // per-domain relaxation time; the other MRT rates are TensorLBM's defaults
  // of the lattice (solver.py:249 collide_mrt, solver3d.py:107 collide_mrt3d)
  if constexpr (L::Q == 9) cp = make_collide_params<T>(dm.tau, 1.64, 1.54, 1.7, -1.0, 1.0, 1.0, 1.0, 0.0);
  else cp = make_collide_params<T>(dm.tau, 1.19, 1.4, 1.2, -1.0, 1.0, 1.0, 1.0, 0.0);
  bp = make_bc_params<T>(dm.u_in, 0.0, 0.0, dm.rho_out, dm.u_lid);
}

// dom_status (may be null): one status word per domain.  A domain whose word
// is non-zero (a non-finite density seen in an earlier tile or step) is
// retired: its tiles are skipped, and its state stays as it was when that
// happened.  Without it every domain is updated and the non-finite bit goes to
// the one status word.
//
// cells_per_thread 2: the tile's tile_x cells of a row run on tile_x / 2
// threads.  In a domain of even nx a thread takes the pair (x, x + 1) through
// the pair update of k_step_x2 (the same results bit for bit as one cell per
// thread); in a domain of odd nx it updates x and x + tile_x / 2 one after
// the other.  The choice is uniform over the tile.
template <class L, typename S, int COLL>
__device__ __forceinline__ void process_tile(const tlbm_batch_domain* __restrict__ doms, const int* __restrict__ tiles,
                                             long long t, const S* fin, S* fout, const uint8_t* flags,
                                             double* forces, unsigned int* status, unsigned int* dom_status,
                                             int cells_per_thread) {
  using T = typename Storage<S>::T;
  const int di = tiles[3 * t + 0];
  if (dom_status && *(volatile unsigned int*)(dom_status + di)) return;   // uniform over the tile
  const int x0 = tiles[3 * t + 1];
  const int row = tiles[3 * t + 2] + threadIdx.y;   // over the nz * ny rows of the domain
  const tlbm_batch_domain dm = doms[di];
  const int nz = dm.nz > 1 ? dm.nz : 1;
  const int y = row % dm.ny, z = row / dm.ny;
  CollideParams<T> cp;
  BcParams<T> bp;
  domain_params<L, T>(dm, cp, bp);
  Domain<S, S> d;
  d.fin = fin + dm.f_offset;
  d.fout = fout + dm.f_offset;
  d.flags = flags ? flags + dm.cell_offset : nullptr;
  d.tau_field = nullptr;
  d.force = forces ? forces + 3 * (long long)di : nullptr;
  d.status = dom_status ? dom_status + di : status;
  d.wall_u = nullptr;
  d.link_row = nullptr;
  d.link_q = nullptr;
  d.nx = dm.nx;
  d.ny = dm.ny;
  d.nz = nz;
  d.plane = (long long)dm.nx * dm.ny;
  d.n = d.plane * nz;
  d.bc = dm.bc;
  const bool row_ok = row < dm.ny * nz;
  if (cells_per_thread == 2) {
    if ((dm.nx & 1) == 0) {
      const int x = x0 + 2 * int(threadIdx.x);
      pair_update<L, S, COLL>(d, cp, bp, x, y, z, x < dm.nx && row_ok);
    } else {
      const int x = x0 + int(threadIdx.x);
      cell_update<L, S, S, COLL, true>(d, x, y, z, x < dm.nx && row_ok, cp, bp);
      const int x2 = x + int(blockDim.x);
      cell_update<L, S, S, COLL, true>(d, x2, y, z, x2 < dm.nx && row_ok, cp, bp);
    }
  } else {
    const int x = x0 + int(threadIdx.x);
    cell_update<L, S, S, COLL, true>(d, x, y, z, x < dm.nx && row_ok, cp, bp);
  }
}

template <class L, typename S, int COLL>
__global__ void __launch_bounds__(256) k_batch_step(const tlbm_batch_domain* doms, const int* tiles, long long ntiles,
                                                    const S* fin, S* fout, const uint8_t* flags, double* forces,
                                                    const int* force_slot, int ndomains, unsigned int* status,
                                                    unsigned int* dom_status, int cells_per_thread) {
  // with a slot counter, the forces of this step go to record *force_slot
  if (forces && force_slot) forces += 3LL * ndomains * (*force_slot);
  for (long long t = blockIdx.x; t < ntiles; t += gridDim.x)
    process_tile<L, S, COLL>(doms, tiles, t, fin, fout, flags, forces, status, dom_status, cells_per_thread);
}

// Grid barrier over a cooperative launch, bounded: sync[0] counts arrivals,
// sync[1] is the generation, sync[2] the error flag.  Returns false if the wait
// gave up (or another CTA already did); the caller then returns.
__device__ bool grid_barrier(unsigned int* sync, unsigned long long max_spins) {
  __syncthreads();
  __shared__ int ok;
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    volatile unsigned int* gen = sync + 1;
    volatile unsigned int* err = sync + 2;
    const unsigned int g = *gen;
    __threadfence();
    const unsigned int arrived = atomicAdd(sync, 1u);
    if (arrived == gridDim.x - 1) {
      sync[0] = 0u;
      __threadfence();
      atomicAdd(sync + 1, 1u);
    } else {
      unsigned long long spins = 0;
      while (*gen == g && *err == 0u) {
        if (++spins > max_spins) {
          atomicExch(sync + 2, 1u);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok = (*err == 0u);
  }
  __syncthreads();
  return ok != 0;
}

template <class L, typename S, int COLL>
__global__ void __launch_bounds__(256) k_batch_run(const tlbm_batch_domain* doms, const int* tiles, long long ntiles,
                                                   S* fa, S* fb, const uint8_t* flags, int nsteps, double* force_hist,
                                                   int ndomains, int record_every, unsigned int* sync,
                                                   unsigned int* status, unsigned long long max_spins,
                                                   unsigned int* dom_status, int cells_per_thread) {
  for (int s = 0; s < nsteps; ++s) {
    const S* fin = (s & 1) ? fb : fa;
    S* fout = (s & 1) ? fa : fb;
    double* forces = nullptr;
    if (force_hist && record_every > 0 && (s % record_every) == 0)
      forces = force_hist + 3 * (long long)ndomains * (s / record_every);
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x)
      process_tile<L, S, COLL>(doms, tiles, t, fin, fout, flags, forces, status, dom_status, cells_per_thread);
    if (!grid_barrier(sync, max_spins)) {
      if (threadIdx.x == 0 && threadIdx.y == 0 && blockIdx.x == 0) atomicOr(status, 2u);
      return;
    }
  }
}

template <class L, typename S, int COLL>
int launch_batch(const tlbm_batch_desc& b, const tlbm_batch_domain* doms, const int* tiles, long long ntiles,
                 const void* fin, void* fout, const uint8_t* flags, double* forces, const int* force_slot,
                 unsigned int* status, cudaStream_t s) {
  const int cpt = b.cells_per_thread == 2 ? 2 : 1;
  const dim3 block(b.tile_x / cpt, b.tile_y);
  const long long grid = ntiles < 0x7fffffffLL ? ntiles : 0x7fffffffLL;
  k_batch_step<L, S, COLL><<<(unsigned)grid, block, 0, s>>>(doms, tiles, ntiles, (const S*)fin, (S*)fout, flags,
                                                           forces, force_slot, b.ndomains, status,
                                                           b.domain_status, cpt);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

template <class L, typename S, int COLL>
int launch_batch_run(const tlbm_batch_desc& b, const tlbm_batch_domain* doms, const int* tiles, long long ntiles,
                     void* fa, void* fb, const uint8_t* flags, int nsteps, double* force_hist, int record_every,
                     unsigned int* sync, unsigned int* status, long long max_spins, cudaStream_t s) {
  const int cpt = b.cells_per_thread == 2 ? 2 : 1;
  const dim3 block(b.tile_x / cpt, b.tile_y);
  int dev = 0, sms = 0, per_sm = 0, coop = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return TLBM_ERR_LAUNCH;
  if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess || !coop)
    return TLBM_ERR_UNSUPPORTED;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return TLBM_ERR_LAUNCH;
  auto kern = k_batch_run<L, S, COLL>;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)(block.x * block.y), 0) != cudaSuccess)
    return TLBM_ERR_LAUNCH;
  if (per_sm < 1) return TLBM_ERR_UNSUPPORTED;
  if (b.ctas_per_sm > 0 && b.ctas_per_sm < per_sm) per_sm = b.ctas_per_sm;
  long long grid = (long long)sms * per_sm;
  if (grid > ntiles) grid = ntiles;
  if (grid < 1) return TLBM_OK;
  // cudaLaunchKernelEx with the cooperative attribute: the same guarantees as
  // cudaLaunchCooperativeKernel (every CTA resident at once), and the launch
  // can be captured into a CUDA graph
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, kern, doms, tiles, ntiles, (S*)fa, (S*)fb, flags, nsteps, force_hist, b.ndomains,
                         record_every, sync, status, (unsigned long long)max_spins, b.domain_status, cpt) !=
      cudaSuccess)
    return TLBM_ERR_LAUNCH;
  return TLBM_OK;
}

__global__ void k_advance_slot(int* slot) { slot[0] += 1; }

int check_batch(const tlbm_batch_desc* b, const tlbm_batch_domain* doms, const int* tiles, long long ntiles) {
  if (!b || !doms || !tiles) return TLBM_ERR_ARG;
  if (b->lattice != TLBM_D2Q9 && b->lattice != TLBM_D3Q19) return TLBM_ERR_UNSUPPORTED;
  if (b->dtype != TLBM_F32) return TLBM_ERR_DTYPE;
  if (b->collision != TLBM_COLL_BGK && b->collision != TLBM_COLL_MRT) return TLBM_ERR_UNSUPPORTED;
  if (b->cells_per_thread != 0 && b->cells_per_thread != 1 && b->cells_per_thread != 2) return TLBM_ERR_ARG;
  // threads of a CTA: tile_x / cells_per_thread (whole warps) x tile_y, at most 256
  const int cpt = b->cells_per_thread == 2 ? 2 : 1;
  if (b->tile_x < 32 * cpt || (b->tile_x % (32 * cpt)) != 0 || b->tile_y < 1 || (b->tile_x / cpt) * b->tile_y > 256)
    return TLBM_ERR_ARG;
  if (ntiles < 0 || b->ndomains < 1) return TLBM_ERR_SHAPE;
  return TLBM_OK;
}

}  // namespace
}  // namespace tlbm

using namespace tlbm;

extern "C" {

TLBM_API int tlbm_batch_step(const tlbm_batch_desc* b, const tlbm_batch_domain* domains, const int32_t* tiles,
                             int64_t ntiles, const void* f_in, void* f_out, const uint8_t* flags, double* forces,
                             const int32_t* force_slot, unsigned int* status, void* stream) {
  int st = check_batch(b, domains, tiles, ntiles);
  if (st != TLBM_OK) return st;
  if (!f_in || !f_out) return TLBM_ERR_ARG;
  if (f_in == f_out) return TLBM_ERR_ALIAS;
  if (ntiles == 0) return TLBM_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (b->lattice == TLBM_D3Q19) {
    if (b->collision == TLBM_COLL_BGK)
      return launch_batch<D3Q19, float, TLBM_COLL_BGK>(*b, domains, tiles, ntiles, f_in, f_out, flags, forces,
                                                       force_slot, status, s);
    return launch_batch<D3Q19, float, TLBM_COLL_MRT>(*b, domains, tiles, ntiles, f_in, f_out, flags, forces,
                                                     force_slot, status, s);
  }
  if (b->collision == TLBM_COLL_BGK)
    return launch_batch<D2Q9, float, TLBM_COLL_BGK>(*b, domains, tiles, ntiles, f_in, f_out, flags, forces,
                                                    force_slot, status, s);
  return launch_batch<D2Q9, float, TLBM_COLL_MRT>(*b, domains, tiles, ntiles, f_in, f_out, flags, forces,
                                                  force_slot, status, s);
}

TLBM_API int tlbm_batch_advance_slot(int32_t* slot, void* stream) {
  if (!slot) return TLBM_ERR_ARG;
  k_advance_slot<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(slot);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

TLBM_API int tlbm_batch_run(const tlbm_batch_desc* b, const tlbm_batch_domain* domains, const int32_t* tiles,
                            int64_t ntiles, void* f_a, void* f_b, const uint8_t* flags, int32_t nsteps,
                            double* force_history, int32_t record_every, unsigned int* sync, unsigned int* status,
                            int64_t max_spins, void* stream) {
  int st = check_batch(b, domains, tiles, ntiles);
  if (st != TLBM_OK) return st;
  if (!f_a || !f_b || !sync || !status) return TLBM_ERR_ARG;
  if (f_a == f_b) return TLBM_ERR_ALIAS;
  if (nsteps < 0 || max_spins < 1) return TLBM_ERR_ARG;
  if (ntiles == 0 || nsteps == 0) return TLBM_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (b->lattice == TLBM_D3Q19) {
    if (b->collision == TLBM_COLL_BGK)
      return launch_batch_run<D3Q19, float, TLBM_COLL_BGK>(*b, domains, tiles, ntiles, f_a, f_b, flags, nsteps,
                                                           force_history, record_every, sync, status, max_spins, s);
    return launch_batch_run<D3Q19, float, TLBM_COLL_MRT>(*b, domains, tiles, ntiles, f_a, f_b, flags, nsteps,
                                                         force_history, record_every, sync, status, max_spins, s);
  }
  if (b->collision == TLBM_COLL_BGK)
    return launch_batch_run<D2Q9, float, TLBM_COLL_BGK>(*b, domains, tiles, ntiles, f_a, f_b, flags, nsteps,
                                                        force_history, record_every, sync, status, max_spins, s);
  return launch_batch_run<D2Q9, float, TLBM_COLL_MRT>(*b, domains, tiles, ntiles, f_a, f_b, flags, nsteps,
                                                     force_history, record_every, sync, status, max_spins, s);
}

}  // extern "C"

// Row-staged pair kernel: the two-cells-per-thread update with its pulls
// served from shared memory that bulk asynchronous copies (TMA,
// cp.async.bulk) fill ahead of use.
//
// One CTA of nx / 2 threads owns whole x-rows (y, z), taken round robin:
// row blockIdx.x, blockIdx.x + gridDim.x, ...  For a row, direction q pulls
// from source row (y - c_y, z - c_z) of plane q; the x shift (with its
// periodic wrap) stays inside that row.  So one row of the pull is Q
// contiguous copies of nx values, issued by one thread into a ring of ST
// shared-memory stages, each completing on the stage's "full" mbarrier with
// its byte count.  Every warp reads its 64 cells' values from the stage,
// arrives on the stage's "empty" mbarrier, and then runs the same per-pair
// update as k_step_x2 (pair_finish: boundaries, drag, collisions, stores to
// global memory), so the results are those of k_step_x2 bit for bit.  The
// copy of row j + ST - 1 goes out as soon as row j - 1's stage is released,
// so ST - 1 rows of loads are in flight while a row is computed, and no
// register waits on global memory.
//
// Included by tlbm_step.cuh after the pair kernels.  Waits are bounded: a
// wait that gives up sets status bit 3, the CTA stops, and the issuing
// thread waits (bounded again) for its copies in flight before returning.
#pragma once

#include "tlbm_umma.cuh"

namespace tlbm {

int row_staging_enabled();   // runtime switch (capi.cu, tlbm_set_row_staging)

namespace rows {

constexpr int kMaxNx = 512;                   // nx / 2 threads per CTA, at most 256
constexpr uint32_t kMaxWait = 1u << 20;       // polls of an mbarrier before giving up
constexpr unsigned int kStatusTimeout = 8u;   // status bit 3
constexpr int kHeader = 128;                  // mbarriers in front of the stages

__device__ __forceinline__ void arrive_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mbar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void arrive(uint32_t mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
// one contiguous global -> shared copy of `bytes` (a multiple of 16, both
// addresses 16-byte aligned) that completes on mbar's transaction count
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t mbar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(mbar)
               : "memory");
}

// Stages of the ring: three for 2-byte storage, two otherwise.
template <class L, typename S, int COLL>
__host__ __device__ constexpr int stages() {
  return sizeof(S) == 2 ? 3 : 2;
}

template <class L, typename S, int COLL>
__host__ __device__ constexpr long long smem_bytes(int nx) {
  return kHeader + (long long)stages<L, S, COLL>() * L::Q * nx * (long long)sizeof(S);
}

// Resident CTAs per SM the kernel is compiled for (the register cap): the
// pair kernel's cap, but no more CTAs than the stages of a 512-cell row let
// fit in the SM's 228 KB of shared memory (1 KB reserved per CTA), so that no
// registers are given up for CTAs that could not be resident anyway.
template <class L, typename S, int COLL>
__host__ __device__ constexpr int min_blocks() {
  constexpr int by_smem = int((228LL * 1024) / (smem_bytes<L, S, COLL>(kMaxNx) + 1024));
  constexpr int by_regs = x2_min_blocks<L, S, COLL>();
  return by_regs < 1 ? 1 : (by_regs < by_smem ? by_regs : by_smem);
}

// The (lattice, storage, collision) triples that have a row-staged kernel.
template <class L, typename S, int COLL>
__host__ __device__ constexpr bool built() {
  constexpr bool st = std::is_same<S, __half>::value || std::is_same<S, __nv_bfloat16>::value ||
                      std::is_same<S, float>::value;
  return st && ((L::Q == 19 && (COLL == TLBM_COLL_BGK || COLL == TLBM_COLL_MRT)) ||
                (L::Q == 27 && COLL == TLBM_COLL_CUMULANT));
}

}  // namespace rows

template <class L, typename S, int COLL>
__device__ __forceinline__ void step_rows(const StepParams& p, const CollideParams<typename Storage<S>::T>& cp,
                                          const BcParams<typename Storage<S>::T>& bp) {
  using T = typename Storage<S>::T;
  using IO = PairIO<S>;
  using V = typename IO::V;
  constexpr int Q = L::Q;
  constexpr int ST = rows::stages<L, S, COLL>();
  constexpr bool kDev = pair_deviation_form<L, S, COLL, false>();
  extern __shared__ __align__(128) uint8_t smem[];
  const uint32_t full0 = umma::smem_addr(smem);          // ST mbarriers
  const uint32_t empty0 = full0 + 8u * ST;                // ST mbarriers
  const S* stage0 = reinterpret_cast<const S*>(smem + rows::kHeader);
  const uint32_t stage0_addr = full0 + rows::kHeader;

  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int plane = nx * ny;
  const int N = int(p.n);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int x = 2 * tid;
  const uint32_t row_bytes = uint32_t(nx) * uint32_t(sizeof(S));
  const int stage_elems = Q * nx;
  const long long R = (long long)ny * p.z_count;
  const long long G = gridDim.x;
  const long long count = (R - blockIdx.x + G - 1) / G;   // rows of this CTA (the grid is at most R)
  const Domain<S, S> d = pair_domain<S>(p);

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < ST; ++s) {
      umma::mbar_init(full0 + 8u * s, 1);
      umma::mbar_init(empty0 + 8u * s, blockDim.x / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // thread 0: the Q source rows of this CTA's j-th row into stage j % ST
  auto issue = [&](long long j) {
    const long long r = blockIdx.x + j * G;
    const int y = int(r % ny), z = p.z0 + int(r / ny);
    const int s = int(j % ST);
    const uint32_t fb = full0 + 8u * s;
    rows::arrive_expect_tx(fb, uint32_t(Q) * row_bytes);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      int ys = y - L::cy(q), zs = z - L::cz(q);
      ys = ys < 0 ? ny - 1 : (ys >= ny ? 0 : ys);
      zs = zs < 0 ? nz - 1 : (zs >= nz ? 0 : zs);
      const S* src = d.fin + (long long)q * N + (long long)zs * plane + (long long)ys * nx;
      rows::bulk_g2s(stage0_addr + uint32_t((s * stage_elems + q * nx) * int(sizeof(S))), src, row_bytes, fb);
    }
  };

  long long issued = 0;   // rows thread 0 has issued
  if (tid == 0)
    for (; issued < count && issued < ST - 1; ++issued) issue(issued);

  bool ok = true;
  long long j = 0;
  for (; j < count; ++j) {
    const long long r = blockIdx.x + j * G;
    const int y = int(r % ny), z = p.z0 + int(r / ny);
    const int s = int(j % ST);
    const bool got = umma::mbar_wait(full0 + 8u * s, uint32_t((j / ST) & 1), rows::kMaxWait);
    if (!__all_sync(0xffffffffu, got)) {
      ok = false;
      break;
    }
    const int wi = tid;   // word (pair) index in the row
    const S* st = stage0 + s * stage_elems;
    T fa[Q], fb[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const S* row = st + q * nx;
      const T w = weight<L, T>(q);
      if constexpr (sizeof(S) == 2) {
        // words of two values: cells (x, x + 1) are word wi
        const uint32_t* wr = reinterpret_cast<const uint32_t*>(row);
        const int nw = nx / 2;
        uint32_t v;
        if (L::cx(q) == 0) {
          v = wr[wi];
        } else if (L::cx(q) > 0) {   // cells pull x - 1, x
          v = __byte_perm(wr[wi == 0 ? nw - 1 : wi - 1], wr[wi], 0x5432);
        } else {                     // cells pull x + 1, x + 2
          v = __byte_perm(wr[wi], wr[wi == nw - 1 ? 0 : wi + 1], 0x5432);
        }
        pull_pair<kDev, S>(v, w, fa[q], fb[q]);
      } else {
        if (L::cx(q) == 0) {
          pull_pair<kDev, S>(*reinterpret_cast<const V*>(row + x), w, fa[q], fb[q]);
        } else if (L::cx(q) > 0) {
          fa[q] = pull_value<kDev>(row[x == 0 ? nx - 1 : x - 1], w);
          fb[q] = pull_value<kDev>(row[x], w);
        } else {
          fa[q] = pull_value<kDev>(row[x + 1], w);
          fb[q] = pull_value<kDev>(row[x + 2 == nx ? 0 : x + 2], w);
        }
      }
    }
    const int c = z * plane + y * nx + x;
    uint32_t fl2 = 0;
    if (d.flags) fl2 = __ldg(reinterpret_cast<const uint16_t*>(at_offset(d.flags, c)));
    __syncwarp();
    if (lane == 0) rows::arrive(empty0 + 8u * s);
    // refill the stage of row j - 1 with row j + ST - 1 once every warp has read it
    bool issued_ok = true;
    if (tid == 0 && issued < count) {
      if (j >= 1) {
        const long long jp = j - 1;
        issued_ok = umma::mbar_wait(empty0 + 8u * uint32_t(jp % ST), uint32_t((jp / ST) & 1), rows::kMaxWait);
      }
      if (issued_ok) issue(issued++);
    }
    pair_finish<L, S, COLL, false>(d, cp, bp, x, y, z, c, true, fa, fb, fl2);
    if (!__all_sync(0xffffffffu, issued_ok)) {
      ok = false;
      ++j;
      break;
    }
  }
  if (!ok) {
    if (lane == 0 && d.status) atomicOr(d.status, rows::kStatusTimeout);
    // the copies thread 0 issued and nobody consumed: wait for them (bounded)
    if (tid == 0)
      for (long long k = j; k < issued; ++k)
        umma::mbar_wait(full0 + 8u * uint32_t(k % ST), uint32_t((k / ST) & 1), rows::kMaxWait);
  }
}

template <class L, typename S, int COLL, int MINB>
__global__ void __launch_bounds__(rows::kMaxNx / 2, MINB) k_step_rows(StepParams p,
                                                                      CollideParams<typename Storage<S>::T> cp,
                                                                      BcParams<typename Storage<S>::T> bp) {
  step_rows<L, S, COLL>(p, cp, bp);
}

// Launch the row-staged kernel when it is built for (L, S, COLL), enabled, and
// the layout allows it: nx a multiple of 64 up to kMaxNx (whole warps, one
// word per thread, 16-byte row copies), 16-byte aligned population buffers
// (every source row then starts on a 16-byte boundary), the pair kernel's
// conditions, no Bouzidi links, and the stages fit in shared memory.  Returns
// true if it launched (st holds the launch status).
template <class L, typename S, int COLL>
bool launch_rows(const StepParams& p, const CollideParams<typename Storage<S>::T>& cp,
                 const BcParams<typename Storage<S>::T>& bp, cudaStream_t s, int& st) {
  if constexpr (!rows::built<L, S, COLL>()) {
    return false;
  } else {
    if (!row_staging_enabled()) return false;
    const auto al = [](const void* ptr, size_t a) { return (reinterpret_cast<uintptr_t>(ptr) % a) == 0; };
    if (p.nx % 64 != 0 || p.nx > rows::kMaxNx || p.link_q != nullptr || (p.bc & TLBM_BC_FAR_FIELD) ||
        p.z_count < 1 || p.ny < 1)
      return false;
    if (!al(p.f_in, 16) || !al(p.f_out, 2 * sizeof(S)) || (p.flags && !al(p.flags, 2))) return false;
    if ((long long)(L::Q / 2 + 2) * p.n >= (1LL << 31)) return false;
    const long long smem = rows::smem_bytes<L, S, COLL>(p.nx);
    constexpr long long kMaxSmem = rows::smem_bytes<L, S, COLL>(rows::kMaxNx);
    if (smem > 227 * 1024) return false;
    constexpr int minb = rows::min_blocks<L, S, COLL>();
    auto kern = k_step_rows<L, S, COLL, minb>;
    // per device: SM count and resident CTAs for each row length (the
    // function attributes are set on each device before its first launch)
    constexpr int kDevices = 64;
    static int sms_of[kDevices] = {};
    static int per_sm_of[kDevices][rows::kMaxNx / 64 + 1] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDevices) {
      cudaGetLastError();
      return false;
    }
    int& sms = sms_of[dev];
    if (sms <= 0) {
      int n = 0;
      if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kMaxSmem < 227 * 1024 ? kMaxSmem : 227 * 1024)) != cudaSuccess ||
          cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                               cudaSharedmemCarveoutMaxShared) != cudaSuccess) {
        cudaGetLastError();
        return false;
      }
      sms = n;
    }
    int& per_sm = per_sm_of[dev][p.nx / 64];
    if (per_sm == 0) {
      int nb = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, p.nx / 2, size_t(smem)) != cudaSuccess || nb < 1) {
        cudaGetLastError();
        return false;
      }
      per_sm = nb;
    }
    const long long R = (long long)p.ny * p.z_count;
    const long long g = (long long)sms * per_sm;
    const int grid = int(g < R ? g : R);
    kern<<<grid, p.nx / 2, size_t(smem), s>>>(p, cp, bp);
    st = cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
    return true;
  }
}

}  // namespace tlbm

// Eddy-viscosity MLP of the learned LES closure: feature map, packed model
// blob, and the tensor-core inference engine.
//
// Network: 9 invariant features -> 64 -> 64 -> 64 (SiLU) -> 1,
// nu_t = nu_scale * softplus(y), tau_eff = tau0 + 3 nu_t.  All four layers run
// on tcgen05 (bf16 operands from shared memory, fp32 accumulators in TMEM,
// M = 128 cells per MMA, K = 16 per instruction; N = 64 for the hidden layers,
// N = 16 for the output layer whose B tile holds w4 in row 0).  Between layers
// each thread turns its cell's accumulator row into the next A row:
// h = bf16(0.5 (acc + b)), SiLU = h + h tanh(h) in packed bf16x2 arithmetic.
//
// A CTA is HALVES independent halves of 128 rows (threads).  Each half has its
// own A tile, 64 TMEM columns, mbarrier and named barrier, so the halves drift
// apart and one half's MMA round trip overlaps the other halves' CUDA-core
// work; the weights are one shared-memory copy per CTA.
#pragma once

#include <cuda_bf16.h>

#include "tlbm_umma.cuh"

namespace tlbm {
namespace mlp {

constexpr int NF = 9;        // input features
constexpr int H = 64;        // hidden width
constexpr int HALF = 128;    // rows of one half (M of its MMAs)
constexpr int N_PARAMS = H * NF + H + H * H + H + H * H + H + H + 1;  // 9025, flat training vector

// ---- packed inference blob (global memory) --------------------------------
// [0, 24576): W1, W2, W3 as SW128 K-major bf16 64x64 tiles (W1 zero beyond column 9)
// [24576, 26624): w4 as a 16-row SW128 tile (row 0 = w4, rows 1..15 zero)
// [26624, ..): float block (biases b1..b3 stored halved)
constexpr int W_TILE_BYTES = H * H * 2;  // 8192
constexpr int W4_TILE_BYTES = 16 * 128;  // 2048
constexpr int OFF_W = 0;
constexpr int OFF_W4 = 3 * W_TILE_BYTES;             // 24576
constexpr int OFF_P = OFF_W4 + W4_TILE_BYTES;        // 26624
constexpr int P_HB1 = 0, P_HB2 = 64, P_HB3 = 128, P_W4 = 192, P_B4 = 256, P_NUS = 257, P_MEAN = 260,
              P_ISTD = P_MEAN + NF, P_LO = P_ISTD + NF, P_HI = P_LO + NF, P_COUNT = P_HI + NF;  // 296
constexpr int P_BYTES = ((P_COUNT * 4 + 127) / 128) * 128;                               // 1280
constexpr int BLOB_BYTES = OFF_P + P_BYTES;                                              // 27904

// ---- shared memory of one CTA (offsets from a 1024-byte aligned base) -------
constexpr int A_TILE_BYTES = HALF * 128;  // 16384: one half's activations
template <int HALVES>
struct Cta {
  static_assert(HALVES == 2 || HALVES == 4 || HALVES == 8, "the TMEM allocation must be a power of two");
  static constexpr int THREADS = HALF * HALVES;             // = cells per CTA pass
  static constexpr int SM_A = 0;                            // HALVES A tiles
  static constexpr int SM_W = SM_A + HALVES * A_TILE_BYTES;  // the blob
  static constexpr int SM_P = SM_W + OFF_P;                 // its float block
  static constexpr int SM_BAR = SM_P + P_BYTES;             // one mbarrier per half
  static constexpr int SM_SLOT = SM_BAR + 8 * HALVES;       // TMEM base address
  static constexpr int SM_FLAG = SM_SLOT + 4;               // one timeout flag per half
  static constexpr int SM_BYTES = SM_FLAG + 4 * HALVES + 1024;  // with alignment slack
  static constexpr uint32_t TMEM_COLS = 64u * HALVES;       // 64 accumulator columns per half
};
constexpr uint32_t MAX_WAIT = 1u << 16;          // mbarrier waits before giving up
constexpr uint32_t WAIT_HINT_NS = 20000;         // each may suspend the polling warp up to 20 us

// ---- features --------------------------------------------------------------
// Nine rotation- and Galilean-invariant inputs from the non-equilibrium
// stress Pi = (xx, yy, zz, xy, xz, yz), rho and the molecular tau:
//  0 m = |dev Pi|_F / rho   1 log(m + 1e-12)   2 Lode 3 sqrt(6) det(dev Pi) / |dev Pi|^3
//  3 tr Pi / rho            4 rho - 1           5 tau0
//  6 tau_s - tau0 with the Smagorinsky tau_s of C_s (turbulence.py:183-208)
//  7 m / tau0               8 sqrt(m)
template <typename T>
__host__ __device__ inline void features(T xx, T yy, T zz, T xy, T xz, T yz, T rho, T tau0, T c_s, T (&x)[NF]) {
  const T tr = xx + yy + zz;
  const T third = T(1) / T(3);
  const T dxx = xx - tr * third, dyy = yy - tr * third, dzz = zz - tr * third;
  const T n2 = dxx * dxx + dyy * dyy + dzz * dzz + T(2) * (xy * xy + xz * xz + yz * yz);
  const T nd = sqrt(n2);
  const T det = dxx * (dyy * dzz - yz * yz) - xy * (xy * dzz - yz * xz) + xz * (xy * yz - dyy * xz);
  T lode = T(0);
  if (nd > T(1e-20)) {
    lode = T(7.3484692283495345) * det / (nd * nd * nd);  // 3 sqrt(6)
    lode = lode > T(1) ? T(1) : (lode < T(-1) ? T(-1) : lode);
  }
  const T m = nd / rho;
  T full = xx * xx + yy * yy + zz * zz + T(2) * (xy * xy + xz * xz + yz * yz);
  full = full > T(1e-30) ? full : T(1e-30);
  T disc = tau0 * tau0 + T(18) * c_s * c_s * sqrt(full) / rho;
  disc = disc > T(0) ? disc : T(0);
  T tau_s = T(0.5) * (tau0 + sqrt(disc));
  const T tmax = tau0 + T(0.5) > T(1) ? tau0 + T(0.5) : T(1);
  tau_s = tau_s < T(0.5001) ? T(0.5001) : (tau_s > tmax ? tmax : tau_s);
  x[0] = m;
  x[1] = log(m + T(1e-12));
  x[2] = lode;
  x[3] = tr / rho;
  x[4] = rho - T(1);
  x[5] = tau0;
  x[6] = tau_s - tau0;
  x[7] = m / tau0;
  x[8] = sqrt(m);
}

__device__ __forceinline__ float softplus(float y) { return y > 20.0f ? y : log1pf(__expf(y)); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// SiLU of two pre-activations given as h = a/2 (already rounded to bf16x2):
// a sigmoid(a) = h + h tanh(h), with the hardware bf16x2 tanh and one bf16x2 fma
__device__ __forceinline__ uint32_t silu_half_bf16x2(uint32_t h) {
  uint32_t t, r;
  asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(h));
  asm("fma.rn.bf16x2 %0, %1, %2, %1;" : "=r"(r) : "r"(h), "r"(t));
  return r;
}

__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// The tensor-core pass of one half-CTA (128 threads, one row each).
template <int HALVES>
struct Engine {
  using C = Cta<HALVES>;
  uint8_t* sm;
  uint32_t tmem;   // this half's first accumulator column
  uint32_t mbar;   // this half's mbarrier
  uint32_t phase;
  int half;        // 0 or 1
  int lt;          // thread index within the half

  // CTA-wide: copy the blob to shared memory, allocate TMEM, initialise the mbarriers
  __device__ void setup(uint8_t* raw_smem, const uint8_t* __restrict__ blob) {
    sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw_smem) + 1023) & ~uintptr_t(1023));
    const int4* src = reinterpret_cast<const int4*>(blob);
    int4* dst = reinterpret_cast<int4*>(sm + C::SM_W);
    for (int i = threadIdx.x; i < (BLOB_BYTES / 16); i += blockDim.x) dst[i] = src[i];
    if (threadIdx.x < 32) umma::tmem_alloc(umma::smem_addr(sm + C::SM_SLOT), C::TMEM_COLS);
    if (threadIdx.x == 0) {
      for (int h = 0; h < HALVES; ++h) {
        umma::mbar_init(umma::smem_addr(sm + C::SM_BAR + 8 * h), 1);
        reinterpret_cast<volatile int*>(sm + C::SM_FLAG)[h] = 0;
      }
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    half = threadIdx.x / HALF;
    lt = threadIdx.x % HALF;
    tmem = *reinterpret_cast<volatile uint32_t*>(sm + C::SM_SLOT) + uint32_t(half * H);
    mbar = umma::smem_addr(sm + C::SM_BAR + 8 * half);
    phase = 0;
  }

  // CTA-wide
  __device__ void teardown() {
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
      umma::fence_after_sync();
      umma::tmem_dealloc(*reinterpret_cast<volatile uint32_t*>(sm + C::SM_SLOT), C::TMEM_COLS);
    }
  }

  __device__ const float* params() const { return reinterpret_cast<const float*>(sm + C::SM_P); }
  __device__ void sync_half() const { named_sync(1 + half, HALF); }

  // this thread's A row: 16-byte chunk c (8 bf16)
  __device__ void put_chunk(int c, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    uint8_t* a = sm + C::SM_A + half * A_TILE_BYTES + umma::sw128_offset(lt, c * 8);
    *reinterpret_cast<uint4*>(a) = make_uint4(w0, w1, w2, w3);
  }

  // D = A B^T over k_slices slices of 16 (B = the tile at blob offset b_off,
  // N = 64, or N = 16 for the output layer).  Warp 0 of the half issues and
  // polls the mbarrier; the half meets at its named barrier.  False on timeout.
  template <int N>
  __device__ bool mma(int b_off, int k_slices) {
    volatile int* flag = reinterpret_cast<volatile int*>(sm + C::SM_FLAG) + half;
    umma::fence_proxy_async_smem();
    umma::fence_before_sync();
    sync_half();
    if (lt < 32) {
      if (lt == 0) {
        umma::fence_after_sync();
        const uint32_t a0 = umma::smem_addr(sm + C::SM_A + half * A_TILE_BYTES);
        const uint32_t b0 = umma::smem_addr(sm + C::SM_W + b_off);
        for (int ks = 0; ks < k_slices; ++ks)
          umma::mma_bf16(tmem, umma::sw128_desc(a0 + 32u * ks), umma::sw128_desc(b0 + 32u * ks),
                         umma::IdescBf16<128, N>::value, ks > 0 ? 1u : 0u);
        umma::commit(mbar);
      }
      __syncwarp();
      const bool done = umma::mbar_wait_sleep(mbar, phase, MAX_WAIT, WAIT_HINT_NS);
      if (lt == 0 && !done) *flag = 1;
    }
    phase ^= 1u;
    sync_half();
    umma::fence_after_sync();
    return *flag == 0;
  }

  // TMEM address of this thread's row (lane) at this half's first column
  __device__ uint32_t row_taddr() const {
    const int w = threadIdx.x >> 5;
    return tmem + (uint32_t((w & 3) * 32) << 16);
  }

  // accumulator row -> bf16(0.5 (acc + b)) -> SiLU (bf16x2) -> next A row
  __device__ void hidden_to_a(const float* hb) {
    const uint32_t ta = row_taddr();
    // 16 accumulator columns at a time: fewer live registers beside the
    // populations the caller holds across the pass
#pragma unroll
    for (int part = 0; part < 4; ++part) {
      float v[16];
      umma::tmem_ld16(ta + uint32_t(16 * part), v);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const float4 b0 = *reinterpret_cast<const float4*>(hb + 16 * part + 8 * c);
        const float4 b1 = *reinterpret_cast<const float4*>(hb + 16 * part + 8 * c + 4);
        const float* u = v + 8 * c;
        // 0.5 acc + b/2 for two columns per packed fma.rn.f32x2 (each lane
        // rounded as fmaf would)
        const float2 half = make_float2(0.5f, 0.5f);
        const float2 h0 = __ffma2_rn(make_float2(u[0], u[1]), half, make_float2(b0.x, b0.y));
        const float2 h1 = __ffma2_rn(make_float2(u[2], u[3]), half, make_float2(b0.z, b0.w));
        const float2 h2 = __ffma2_rn(make_float2(u[4], u[5]), half, make_float2(b1.x, b1.y));
        const float2 h3 = __ffma2_rn(make_float2(u[6], u[7]), half, make_float2(b1.z, b1.w));
        put_chunk(2 * part + c, silu_half_bf16x2(pack_bf16x2(h0.x, h0.y)), silu_half_bf16x2(pack_bf16x2(h1.x, h1.y)),
                  silu_half_bf16x2(pack_bf16x2(h2.x, h2.y)), silu_half_bf16x2(pack_bf16x2(h3.x, h3.y)));
      }
    }
  }

  // Full pass of this half.  z: normalised features of this thread's row
  // (zeros for idle rows).  Returns y; ok false if a tensor-core wait gave up.
  __device__ float run(const float (&z)[NF], bool& ok) {
    const float* p = params();
    put_chunk(0, pack_bf16x2(z[0], z[1]), pack_bf16x2(z[2], z[3]), pack_bf16x2(z[4], z[5]), pack_bf16x2(z[6], z[7]));
    put_chunk(1, pack_bf16x2(z[8], 0.0f), 0u, 0u, 0u);
    ok = mma<H>(OFF_W, 1);
    hidden_to_a(p + P_HB1);
    ok = mma<H>(OFF_W + W_TILE_BYTES, H / 16) && ok;
    hidden_to_a(p + P_HB2);
    ok = mma<H>(OFF_W + 2 * W_TILE_BYTES, H / 16) && ok;
    hidden_to_a(p + P_HB3);
    ok = mma<16>(OFF_W4, H / 16) && ok;
    uint32_t r;
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x1.b32 {%0}, [%1];" : "=r"(r) : "r"(row_taddr()) : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    return __uint_as_float(r) + p[P_B4];
  }
};

// CTAs of a persistent tensor-core kernel (Cta<HALVES>::THREADS threads,
// Cta<HALVES>::SM_BYTES dynamic shared memory) that fit on one SM at once,
// from the device's limits and the kernel's register count; the TMEM columns
// bound it too.  (The occupancy query of the runtime plans for the default
// shared-memory split and answers 1.)
// Also returns the SM count.  0 on a runtime error.
template <int HALVES, typename Kernel>
inline int resident_ctas(Kernel kern, int& sms) {
  using C = Cta<HALVES>;
  int dev = 0, smem_sm = 0, reserved = 0, regs_sm = 0, threads_sm = 0;
  cudaFuncAttributes fa;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess)
    return 0;
  const int regs_warp = ((fa.numRegs * 32 + 255) / 256) * 256;  // allocation unit: 256 registers per warp
  int n = smem_sm / (C::SM_BYTES + reserved);
  const int by_regs = regs_sm / (regs_warp * (C::THREADS / 32));
  const int by_threads = threads_sm / C::THREADS;
  const int by_tmem = 512 / int(C::TMEM_COLS);
  n = n < by_regs ? n : by_regs;
  n = n < by_threads ? n : by_threads;
  n = n < by_tmem ? n : by_tmem;
  return n;
}

}  // namespace mlp
}  // namespace tlbm

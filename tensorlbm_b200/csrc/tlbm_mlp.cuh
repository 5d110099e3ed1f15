// Eddy-viscosity MLP of the learned LES closure: feature map, packed model
// blob, and the per-CTA tensor-core inference engine.
//
// Network: 9 invariant features -> 64 -> 64 -> 64 (SiLU) -> 1,
// nu_t = nu_scale * softplus(y), tau_eff = tau0 + 3 nu_t.  The three hidden
// layers run on tcgen05 (bf16 operands from shared memory, fp32 accumulators in
// TMEM, M = 128 cells per MMA, N = 64, K = 16 per instruction); the output layer
// and the activations run in fp32 on the CUDA cores, one cell per thread.
#pragma once

#include <cuda_bf16.h>

#include "tlbm_umma.cuh"

namespace tlbm {
namespace mlp {

constexpr int NF = 9;        // input features
constexpr int H = 64;        // hidden width
constexpr int TILE = 256;    // cells per CTA pass (two M = 128 MMA tiles)
constexpr int N_PARAMS = H * NF + H + H * H + H + H * H + H + H + 1;  // 9025, flat training vector

// ---- packed inference blob (global memory) --------------------------------
// [0, 24576): W1, W2, W3 as SW128 K-major bf16 64x64 tiles (W1 zero beyond column 9)
// [24576, ..): float block
constexpr int W_TILE_BYTES = H * H * 2;  // 8192
constexpr int OFF_W = 0;
constexpr int OFF_P = 3 * W_TILE_BYTES;  // 24576
constexpr int P_B1 = 0, P_B2 = 64, P_B3 = 128, P_W4 = 192, P_B4 = 256, P_NUS = 257, P_MEAN = 260,
              P_ISTD = P_MEAN + NF, P_LO = P_ISTD + NF, P_HI = P_LO + NF, P_COUNT = P_HI + NF;  // 296
constexpr int BLOB_BYTES = OFF_P + ((P_COUNT * 4 + 127) / 128) * 128;                    // 25856

// ---- shared memory of one CTA (offsets from a 1024-byte aligned base) -------
constexpr int SM_A = 0;                          // 2 x (128 rows x 128 B) activations
constexpr int SM_W = SM_A + 2 * 128 * 128;       // 32768: three weight tiles
constexpr int SM_P = SM_W + 3 * W_TILE_BYTES;    // 57344: float block
constexpr int SM_BAR = SM_P + ((P_COUNT * 4 + 127) / 128) * 128;  // 58624
constexpr int SM_SLOT = SM_BAR + 8;
constexpr int SM_FLAG = SM_SLOT + 4;
constexpr int SM_BYTES = SM_FLAG + 4 + 1024;     // with alignment slack
constexpr uint32_t TMEM_COLS = 128;              // two 64-column accumulators
constexpr uint32_t MAX_WAIT = 1u << 20;          // mbarrier polls before giving up

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

__device__ __forceinline__ float silu(float a) { return a / (1.0f + __expf(-a)); }
__device__ __forceinline__ float softplus(float y) { return y > 20.0f ? y : log1pf(__expf(y)); }

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// The tensor-core pass of one CTA over TILE rows (threads 0..TILE-1, one row each).
struct Engine {
  uint8_t* sm;
  uint32_t tmem;
  uint32_t mbar;
  uint32_t phase;

  // copy the blob to shared memory, allocate TMEM, initialise the mbarrier
  __device__ void setup(uint8_t* raw_smem, const uint8_t* __restrict__ blob) {
    sm = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(raw_smem) + 1023) & ~uintptr_t(1023));
    const int4* src = reinterpret_cast<const int4*>(blob);
    int4* dst = reinterpret_cast<int4*>(sm + SM_W);
    for (int i = threadIdx.x; i < (BLOB_BYTES / 16); i += blockDim.x) dst[i] = src[i];
    mbar = umma::smem_addr(sm + SM_BAR);
    if (threadIdx.x < 32) umma::tmem_alloc(umma::smem_addr(sm + SM_SLOT), TMEM_COLS);
    if (threadIdx.x == 0) {
      umma::mbar_init(mbar, 1);
      *reinterpret_cast<volatile int*>(sm + SM_FLAG) = 0;
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    tmem = *reinterpret_cast<volatile uint32_t*>(sm + SM_SLOT);
    phase = 0;
  }

  __device__ void teardown() {
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
      umma::fence_after_sync();
      umma::tmem_dealloc(tmem, TMEM_COLS);
    }
  }

  __device__ const float* params() const { return reinterpret_cast<const float*>(sm + SM_P); }

  // A row of this thread: 16-byte chunk c (8 bf16) <- w[0..3]
  __device__ void put_chunk(int c, uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3) {
    const int t = threadIdx.x;
    uint8_t* a = sm + SM_A + (t >> 7) * (128 * 128) + umma::sw128_offset(t & 127, c * 8);
    *reinterpret_cast<uint4*>(a) = make_uint4(w0, w1, w2, w3);
  }

  // issue D = A W_l^T over k_slices slices of 16, wait for it; false on timeout
  __device__ bool mma_layer(int l, int k_slices) {
    umma::fence_proxy_async_smem();
    umma::fence_before_sync();
    __syncthreads();
    if (threadIdx.x == 0) {
      umma::fence_after_sync();
      const uint32_t b0 = umma::smem_addr(sm + SM_W + l * W_TILE_BYTES);
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) {
        const uint32_t a0 = umma::smem_addr(sm + SM_A + mt * 128 * 128);
        for (int ks = 0; ks < k_slices; ++ks)
          umma::mma_bf16(tmem + uint32_t(mt * H), umma::sw128_desc(a0 + 32u * ks), umma::sw128_desc(b0 + 32u * ks),
                         umma::IdescBf16<128, H>::value, ks > 0 ? 1u : 0u);
      }
      umma::commit(mbar);
    }
    const bool ok = umma::mbar_wait(mbar, phase, MAX_WAIT);
    phase ^= 1u;
    umma::fence_after_sync();
    return ok;
  }

  // TMEM address of this thread's row, column 0 of its tile's accumulator
  __device__ uint32_t row_taddr() const {
    const int w = threadIdx.x >> 5;
    return tmem + (uint32_t((w & 3) * 32) << 16) + uint32_t((w >> 2) * H);
  }

  // accumulator -> bias -> SiLU -> bf16 -> next A row
  __device__ void hidden_to_a(const float* bias) {
    const uint32_t ta = row_taddr();
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float v[32];
      umma::tmem_ld32(ta + uint32_t(32 * half), v);
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        uint32_t w[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int k = 32 * half + 8 * c + 2 * j;
          w[j] = pack_bf16x2(silu(v[8 * c + 2 * j] + bias[k]), silu(v[8 * c + 2 * j + 1] + bias[k + 1]));
        }
        put_chunk(4 * half + c, w[0], w[1], w[2], w[3]);
      }
    }
  }

  // y = w4 . SiLU(acc + b3) + b4 for this thread's row
  __device__ float output_layer() const {
    const float* p = params();
    const uint32_t ta = row_taddr();
    float y = p[P_B4];
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float v[32];
      umma::tmem_ld32(ta + uint32_t(32 * half), v);
#pragma unroll
      for (int i = 0; i < 32; ++i) y = fmaf(silu(v[i] + p[P_B3 + 32 * half + i]), p[P_W4 + 32 * half + i], y);
    }
    return y;
  }

  // Full pass.  z: normalised features of this thread's row (zeros for idle
  // rows).  Returns y; *ok false if a tensor-core wait gave up.
  __device__ float run(const float (&z)[NF], bool& ok) {
    const float* p = params();
    put_chunk(0, pack_bf16x2(z[0], z[1]), pack_bf16x2(z[2], z[3]), pack_bf16x2(z[4], z[5]), pack_bf16x2(z[6], z[7]));
    put_chunk(1, pack_bf16x2(z[8], 0.0f), 0u, 0u, 0u);
    ok = mma_layer(0, 1);
    hidden_to_a(p + P_B1);
    ok = mma_layer(1, H / 16) && ok;
    hidden_to_a(p + P_B2);
    ok = mma_layer(2, H / 16) && ok;
    return output_layer();
  }
};

}  // namespace mlp
}  // namespace tlbm

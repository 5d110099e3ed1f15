// Fused D3Q19 LES step with the learned eddy-viscosity closure.
//
// Persistent kernel: each CTA loads the packed network once (shared memory),
// allocates 64 TMEM columns per half, then walks tiles of TLBM_LES_HALVES x 128
// consecutive cells as independent halves of 128 (see tlbm_mlp.cuh):
//   pull (periodic) -> rho, u -> Pi_neq = sum_q c c (f - feq) -> 9 features
//   -> tcgen05 MLP (three 64-wide layers and the output layer, bf16 x bf16 ->
//      fp32 in TMEM)
//   -> nu_t = nu_scale softplus(y), tau_eff = tau0 + 3 nu_t
//      (Smagorinsky tau_s where a feature leaves the training range)
//   -> BGK with tau_eff + exact-difference linear forcing -> store.
// The populations stay in registers across the tensor-core pass, so the
// kernel moves 2 x 19 x 4 bytes per cell like the plain fused step.
#include "tlbm_collide.cuh"
#include "tlbm_mlp.cuh"

// CTA shape: halves of 128 cells per CTA and CTAs per SM.  One CTA of eight
// halves (1024 threads, 64 registers, all 512 TMEM columns, one 28 KB copy of
// the weights) gives 32 warps per SM.  Measured on the forced-HIT step at
// 128^3 / 256^3: 9.50 / 10.03 GLUPS, against 8.85 / 9.43 for two CTAs of four
// halves and 8.51 / 8.81 for three CTAs of two halves (80 registers, 24 warps;
// their shared memory, 61.7 KB each, stops a fourth).  Reading the
// accumulators 16 columns at a time and 32-bit cell offsets then took the
// spills from 124 to 8 bytes per thread: 10.39 / 10.93 GLUPS.  Results are
// identical in every shape.
#ifndef TLBM_LES_HALVES
#define TLBM_LES_HALVES 8
#endif
#ifndef TLBM_LES_MINB
#define TLBM_LES_MINB 1
#endif

namespace tlbm {
namespace {

using LesCta = mlp::Cta<TLBM_LES_HALVES>;

struct LesStep {
  const float* fin;
  float* fout;
  int nx, ny, nz;
  int plane, n;  // n < 2^31: 32-bit cell offsets within a direction's plane
  float tau0, c_s, a_lin;
  const uint8_t* blob;
  float* tau_out;                // per-cell tau_eff, may be null
  unsigned int* fallback_count;  // cells that took the Smagorinsky fallback, may be null
  unsigned int* status;          // bit0 non-finite, bit2 tensor-core wait timeout; may be null
};

__global__ void __launch_bounds__(LesCta::THREADS, TLBM_LES_MINB) k_step_les(LesStep p) {
  using L = D3Q19;
  constexpr int Q = L::Q;
  constexpr int TILE = LesCta::THREADS;
  extern __shared__ uint8_t raw[];
  mlp::Engine<TLBM_LES_HALVES> e;
  e.setup(raw, p.blob);
  const float* P = e.params();
  const float tmax = p.tau0 + 0.5f > 1.0f ? p.tau0 + 0.5f : 1.0f;
  const int ntiles = int((p.n + (long long)TILE - 1) / TILE);
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int cell = t * TILE + int(threadIdx.x);  // < n + TILE <= 2^31 - 1 + 1024: checked on the host
    const bool active = cell < p.n;
    float f[Q];
    float z[mlp::NF];
    float rho = 1.0f, ux = 0.0f, uy = 0.0f, uz = 0.0f, tau_s = p.tau0;
    bool inrange = false;
    if (active) {
      const int x = int(cell % p.nx);
      const int y = int((cell / p.nx) % p.ny);
      const int zc = int(cell / p.plane);
      const int xm = x == 0 ? p.nx - 1 : x - 1, xp = x == p.nx - 1 ? 0 : x + 1;
      const int ym = y == 0 ? p.ny - 1 : y - 1, yp = y == p.ny - 1 ? 0 : y + 1;
      const int zm = zc == 0 ? p.nz - 1 : zc - 1, zp = zc == p.nz - 1 ? 0 : zc + 1;
      // direction q's plane starts n values after direction q-1's; within it
      // the source cell's offset fits 32 bits
      const float* fq = p.fin;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int sx = L::cx(q) > 0 ? xm : (L::cx(q) < 0 ? xp : x);
        const int sy = L::cy(q) > 0 ? ym : (L::cy(q) < 0 ? yp : y);
        const int sz = L::cz(q) > 0 ? zm : (L::cz(q) < 0 ? zp : zc);
        f[q] = __ldg(fq + (sz * p.plane + sy * p.nx + sx));
        fq += p.n;
      }
      macroscopic_fused<L>(f, rho, ux, uy, uz);
      const float usq = ux * ux + uy * uy + uz * uz;
      float pxx = 0.f, pyy = 0.f, pzz = 0.f, pxy = 0.f, pxz = 0.f, pyz = 0.f;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const float fn = f[q] - feq_fused<L>(q, rho, ux, uy, uz, usq);
        if (L::cx(q) != 0) pxx += fn;
        if (L::cy(q) != 0) pyy += fn;
        if (L::cz(q) != 0) pzz += fn;
        if (L::cx(q) * L::cy(q) != 0) pxy += float(L::cx(q) * L::cy(q)) * fn;
        if (L::cx(q) * L::cz(q) != 0) pxz += float(L::cx(q) * L::cz(q)) * fn;
        if (L::cy(q) * L::cz(q) != 0) pyz += float(L::cy(q) * L::cz(q)) * fn;
      }
      float feat[mlp::NF];
      mlp::features<float>(pxx, pyy, pzz, pxy, pxz, pyz, rho, p.tau0, p.c_s, feat);
      tau_s = feat[6] + p.tau0;
      inrange = true;
#pragma unroll
      for (int k = 0; k < mlp::NF; ++k) {
        inrange = inrange && feat[k] >= P[mlp::P_LO + k] && feat[k] <= P[mlp::P_HI + k];
        z[k] = (feat[k] - P[mlp::P_MEAN + k]) * P[mlp::P_ISTD + k];
      }
    } else {
#pragma unroll
      for (int q = 0; q < Q; ++q) f[q] = 0.0f;
#pragma unroll
      for (int k = 0; k < mlp::NF; ++k) z[k] = 0.0f;
    }
    bool ok = true;
    const float y = e.run(z, ok);
    if (active) {
      float tau = tau_s;
      if (inrange) {
        tau = p.tau0 + 3.0f * P[mlp::P_NUS] * mlp::softplus(y);
        tau = tau < 0.5001f ? 0.5001f : (tau > tmax ? tmax : tau);
      }
      const float inv = 1.0f / tau;
      const float usq = ux * ux + uy * uy + uz * uz;
      // exact-difference force term feq(rho, (1+A) u) - feq(rho, u)
      //   = w rho [3 A (c.u) + ((1+A)^2 - 1) (4.5 (c.u)^2 - 1.5 u^2)]
      const float a3 = 3.0f * p.a_lin;
      const float k2m1 = p.a_lin * (2.0f + p.a_lin);
      float* oq = p.fout;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        float cu = 0.0f;
        if (L::cx(q) != 0) cu = L::cx(q) > 0 ? cu + ux : cu - ux;
        if (L::cy(q) != 0) cu = L::cy(q) > 0 ? cu + uy : cu - uy;
        if (L::cz(q) != 0) cu = L::cz(q) > 0 ? cu + uz : cu - uz;
        const float wr = weight<L, float>(q) * rho;
        const float quad = fmaf(4.5f * cu, cu, -1.5f * usq);
        const float feq = wr * (1.0f + fmaf(3.0f, cu, quad));
        const float force = wr * fmaf(a3, cu, k2m1 * quad);
        oq[cell] = fmaf(feq - f[q], inv, f[q]) + force;
        oq += p.n;
      }
      if (p.tau_out) p.tau_out[cell] = tau;
      if (p.status && !(rho == rho && rho - rho == 0.0f)) atomicOr(p.status, 1u);
    }
    if (p.fallback_count) {
      const unsigned int fb = __ballot_sync(0xffffffffu, active && !inrange);
      if ((threadIdx.x & 31) == 0 && fb) atomicAdd(p.fallback_count, __popc(fb));
    }
    if (!ok) {  // uniform across the half
      if (e.lt == 0 && p.status) atomicOr(p.status, 4u);
      break;
    }
  }
  e.teardown();
}

int les_grid(long long n, int& grid) {
  static int per_sm = -1, sms = 0;
  if (per_sm < 0) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TLBM_ERR_LAUNCH;
    if (cudaFuncSetAttribute(k_step_les, cudaFuncAttributeMaxDynamicSharedMemorySize, LesCta::SM_BYTES) !=
        cudaSuccess)
      return TLBM_ERR_LAUNCH;
    // the largest shared-memory carveout, so that several CTAs fit per SM
    if (cudaFuncSetAttribute(k_step_les, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared) != cudaSuccess)
      return TLBM_ERR_LAUNCH;
    per_sm = mlp::resident_ctas<TLBM_LES_HALVES>(k_step_les, sms);
  }
  if (per_sm < 1) return TLBM_ERR_UNSUPPORTED;
  const long long ntiles = (n + LesCta::THREADS - 1) / LesCta::THREADS;
  const long long g = (long long)sms * per_sm;
  grid = int(g < ntiles ? g : ntiles);
  return TLBM_OK;
}

}  // namespace
}  // namespace tlbm

using namespace tlbm;

extern "C" {

TLBM_API int tlbm_les_step(int32_t nx, int32_t ny, int32_t nz, double tau0, double c_s, double force_lin,
                           const void* blob, const float* f_in, float* f_out, float* tau_out,
                           unsigned int* fallback_count, unsigned int* status, void* stream) {
  if (!blob || !f_in || !f_out) return TLBM_ERR_ARG;
  if (f_in == f_out) return TLBM_ERR_ALIAS;
  if (reinterpret_cast<uintptr_t>(blob) % 16) return TLBM_ERR_ARG;
  if (nx < 1 || ny < 1 || nz < 1) return TLBM_ERR_SHAPE;
  if (!(tau0 > 0.5) || !(force_lin > -1.0 && force_lin < 1.0) || !(c_s >= 0.0)) return TLBM_ERR_ARG;
  const long long n = (long long)nx * ny * nz;
  if (n + LesCta::THREADS > 0x7fffffffLL) return TLBM_ERR_TOO_LARGE;  // 32-bit cell offsets
  LesStep p;
  p.fin = f_in;
  p.fout = f_out;
  p.nx = nx;
  p.ny = ny;
  p.nz = nz;
  p.plane = nx * ny;
  p.n = int(n);
  p.tau0 = float(tau0);
  p.c_s = float(c_s);
  p.a_lin = float(force_lin);
  p.blob = static_cast<const uint8_t*>(blob);
  p.tau_out = tau_out;
  p.fallback_count = fallback_count;
  p.status = status;
  int grid = 0;
  const int st = les_grid(p.n, grid);
  if (st != TLBM_OK) return st;
  k_step_les<<<grid, LesCta::THREADS, LesCta::SM_BYTES, static_cast<cudaStream_t>(stream)>>>(p);
  return cudaGetLastError() == cudaSuccess ? TLBM_OK : TLBM_ERR_LAUNCH;
}

}  // extern "C"

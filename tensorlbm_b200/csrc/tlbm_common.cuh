// Shared device-side definitions: storage formats, parameter blocks, helpers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tlbm.h"
#include "generated/lattice_tables.cuh"
#include "generated/mrt_tables.cuh"

namespace tlbm {

// ---------------------------------------------------------------------------
// Storage formats.  A population is held in HBM as S and computed in T.
// Half-width formats store the deviation f_q - w_q from the rest state
// (rho = 1, u = 0): the deviation is ~1e-2 of f_q, so the 11-bit (fp16) or
// 8-bit (bf16) mantissa resolves f_q about 100x finer than storing f_q.
// ---------------------------------------------------------------------------
template <typename S> struct Storage;

template <> struct Storage<float> {
  using T = float;
  static constexpr bool kShifted = false;
  __device__ __forceinline__ static float load(float v, float) { return v; }
  __device__ __forceinline__ static float store(float v, float) { return v; }
};
template <> struct Storage<double> {
  using T = double;
  static constexpr bool kShifted = false;
  __device__ __forceinline__ static double load(double v, double) { return v; }
  __device__ __forceinline__ static double store(double v, double) { return v; }
};
template <> struct Storage<__half> {
  using T = float;
  static constexpr bool kShifted = true;
  __device__ __forceinline__ static float load(__half v, float w) { return __half2float(v) + w; }
  __device__ __forceinline__ static __half store(float v, float w) { return __float2half_rn(v - w); }
};
template <> struct Storage<__nv_bfloat16> {
  using T = float;
  static constexpr bool kShifted = true;
  __device__ __forceinline__ static float load(__nv_bfloat16 v, float w) { return __bfloat162float(v) + w; }
  __device__ __forceinline__ static __nv_bfloat16 store(float v, float w) { return __float2bfloat16_rn(v - w); }
};

// Lattice weight in compute type T.  TensorLBM's D2Q9 module keeps its weights
// as float32 even for float64 fields (tensorlbm/d2q9.py:22-25, 35-36), so a
// float64 D2Q9 computation uses the float32-rounded weights; D3Q19/D3Q27 cast
// the exact binary64 weights (tensorlbm/d3q19.py:58-80, d3q27.py:353-370).
template <class L, typename T>
__host__ __device__ __forceinline__ constexpr T weight(int q) {
  return (L::Q == 9) ? T(float(L::w(q))) : T(L::w(q));
}

// ---------------------------------------------------------------------------
// Parameter block of one fused step (host fills it, kernel reads it by value)
// ---------------------------------------------------------------------------
struct StepParams {
  const void* f_in;
  void* f_out;
  const uint8_t* flags;     // per cell, may be null
  const float* tau_field;   // per cell relaxation time, may be null
  double* force;            // [3] accumulated momentum-exchange force, may be null
  unsigned int* status;     // bit0: non-finite density seen, may be null
  const void* wall_velocity;  // (DIM, n) moving-wall velocity, compute type, may be null
  int nx, ny, nz;
  long long plane;          // nx*ny
  long long n;              // nx*ny*nz
  uint32_t bc;              // TLBM_BC_* bits
  // relaxation
  double tau, inv_tau;
  double s_e, s_eps, s_q, s_pi;
  double omega_b, omega_odd, omega_even;
  double c_smag;
  // boundaries
  double u_lid;
  double u_in[3];
  double rho_out;
};

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace tlbm

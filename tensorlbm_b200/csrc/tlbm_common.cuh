// Shared device-side definitions: storage formats, parameter blocks, helpers.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/tlbm.h"
#include "generated/lattice_tables.cuh"
#include "generated/cascaded_tables.cuh"
#include "generated/mrt_tables.cuh"

namespace tlbm {

// ---------------------------------------------------------------------------
// Storage formats.  A population is held in HBM as S and computed in T.
// Half-width formats store the deviation f_q - w_q from the rest state
// (rho = 1, u = 0): the deviation is ~1e-2 of f_q, so the 11-bit (fp16) or
// 8-bit (bf16) mantissa resolves f_q about 100x finer than storing f_q.
// ---------------------------------------------------------------------------
template <typename S> struct Storage;

// MurmurHash3's 32-bit finaliser (Appleby): a bijective mixer of the key bits
__device__ __forceinline__ uint32_t fmix32(uint32_t h) {
  h ^= h >> 16;
  h *= 0x85EBCA6Bu;
  h ^= h >> 13;
  h *= 0xC2B2AE35u;
  h ^= h >> 16;
  return h;
}

// Stochastic rounding of the float32 bit pattern to its `drop` low bits:
// add uniform random bits below the kept mantissa, then truncate the
// magnitude (round toward zero).  The result rounds up with probability equal
// to the dropped fraction, so it is unbiased; non-finite values pass unchanged.
template <int DROP>
__device__ __forceinline__ float stochastic_truncate_bits(float d, uint32_t r) {
  const uint32_t bits = __float_as_uint(d);
  uint32_t mag = bits & 0x7FFFFFFFu;
  if (mag < 0x7F800000u) mag += r >> (32 - DROP);
  return __uint_as_float((bits & 0x80000000u) | mag);
}

// store(v, w, r): r is 32 random bits for the stochastic rounding of the
// half formats (ignored by float and double).
template <> struct Storage<float> {
  using T = float;
  static constexpr bool kShifted = false;
  static constexpr bool kFast = false;   // exact (reference-rounded) collisions
  __device__ __forceinline__ static float load(float v, float) { return v; }
  __device__ __forceinline__ static float store(float v, float, uint32_t) { return v; }
};
template <> struct Storage<double> {
  using T = double;
  static constexpr bool kShifted = false;
  static constexpr bool kFast = false;
  __device__ __forceinline__ static double load(double v, double) { return v; }
  __device__ __forceinline__ static double store(double v, double, uint32_t) { return v; }
};
// float16: (f - w) * 2^14, stochastically rounded.  The scale keeps every
// deviation |f - w| > 4e-9 out of the subnormal range (|f - w| < 4 stays finite).
template <> struct Storage<__half> {
  using T = float;
  static constexpr bool kShifted = true;
  static constexpr bool kFast = true;    // fused-arithmetic collisions (no bit-exact target)
  static constexpr float kScale = 16384.0f;
  static constexpr float kRaw = kScale;   // stored value = kRaw (f - w)
  __device__ __forceinline__ static float load(__half v, float w) {
    return fmaf(__half2float(v), 1.0f / kScale, w);
  }
  __device__ __forceinline__ static float load_raw(__half v) { return __half2float(v); }
  __device__ __forceinline__ static __half store(float v, float w, uint32_t r) {
    return __float2half_rz(stochastic_truncate_bits<13>((v - w) * kScale, r));
  }
};
// bfloat16: f - w (float32 range), stochastically rounded
template <> struct Storage<__nv_bfloat16> {
  using T = float;
  static constexpr bool kShifted = true;
  static constexpr bool kFast = true;
  static constexpr float kRaw = 1.0f;      // stored value = f - w
  __device__ __forceinline__ static float load(__nv_bfloat16 v, float w) { return __bfloat162float(v) + w; }
  __device__ __forceinline__ static float load_raw(__nv_bfloat16 v) { return __bfloat162float(v); }
  __device__ __forceinline__ static __nv_bfloat16 store(float v, float w, uint32_t r) {
    return __float2bfloat16_rz(stochastic_truncate_bits<16>(v - w, r));
  }
};

// Plain half formats: f itself in float16 / bfloat16, rounded to nearest on
// store (the storage tiers of TensorLBM's Triton kernel).  Distinct types so
// that they do not collide with the shifted formats above.
struct f16_plain { __half h; };
struct bf16_plain { __nv_bfloat16 h; };
template <> struct Storage<f16_plain> {
  using T = float;
  static constexpr bool kShifted = false;
  static constexpr bool kFast = true;
  __device__ __forceinline__ static float load(f16_plain v, float) { return __half2float(v.h); }
  __device__ __forceinline__ static f16_plain store(float v, float, uint32_t) { return {__float2half_rn(v)}; }
};
template <> struct Storage<bf16_plain> {
  using T = float;
  static constexpr bool kShifted = false;
  static constexpr bool kFast = true;
  __device__ __forceinline__ static float load(bf16_plain v, float) { return __bfloat162float(v.h); }
  __device__ __forceinline__ static bf16_plain store(float v, float, uint32_t) { return {__float2bfloat16_rn(v)}; }
};

// read-only cached load of a storage element (the plain half structs go
// through their 16-bit pattern)
template <typename S>
__device__ __forceinline__ S ldg(const S* p) { return __ldg(p); }
template <>
__device__ __forceinline__ f16_plain ldg(const f16_plain* p) {
  const unsigned short b = __ldg(reinterpret_cast<const unsigned short*>(p));
  return {__ushort_as_half(b)};
}
template <>
__device__ __forceinline__ bf16_plain ldg(const bf16_plain* p) {
  const unsigned short b = __ldg(reinterpret_cast<const unsigned short*>(p));
  return {__ushort_as_bfloat16(b)};
}

// Two consecutive values of one direction (cells x and x + 1, x even) moved
// as one aligned vector.  split() converts to the compute type; join()
// converts back with the stochastic rounding of the half formats.  Their
// random bits come from one 32-bit hash h of the pair and an odd constant per
// direction q: p = h * M_q mod 2^32 is a bijection of h, so every bit field of
// p is uniform; p ^ (p >> 13) keeps the fields uniform and mixes the upper
// bits of p into the low field (the low k bits of p depend only on the low k
// bits of h).  The high word of h * M_q would not do: it is uniform on
// [0, M_q) only, which leaves its top bits biased for a small M_q.
__device__ __forceinline__ uint32_t direction_mix(int q) { return 0x9E3779B9u * uint32_t(2 * q + 1); }
__device__ __forceinline__ uint32_t pair_bits(uint32_t h, int q) {
  const uint32_t p = h * direction_mix(q);
  return p ^ (p >> 13);
}

// Stochastic rounding in hardware (sm_100a, PTX ISA 8.7):
// cvt.rs.{f16,bf16}x2.f32 d, a, b, rbits puts a in the upper half and b in the
// lower half of d; the f32 bits below the kept mantissa plus a field of rbits
// (f16: rbits[28:16] for a, rbits[12:0] for b; bf16: rbits[31:16] and
// rbits[15:0]) carry into the kept mantissa, then the rest is truncated: the
// magnitude rounds up with probability equal to the dropped fraction.
__device__ __forceinline__ uint32_t cvt_rs_f16x2(float lo, float hi, uint32_t rbits) {
  uint32_t r;
  asm("cvt.rs.f16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
  return r;
}
__device__ __forceinline__ uint32_t cvt_rs_bf16x2(float lo, float hi, uint32_t rbits) {
  uint32_t r;
  asm("cvt.rs.bf16x2.f32 %0, %1, %2, %3;" : "=r"(r) : "f"(hi), "f"(lo), "r"(rbits));
  return r;
}

template <typename S> struct PairIO;
template <> struct PairIO<float> {
  using V = float2;
  __device__ __forceinline__ static void split(V v, float, float& a, float& b) { a = v.x; b = v.y; }
  __device__ __forceinline__ static V join(float a, float b, float, uint32_t, int) { return make_float2(a, b); }
};
template <> struct PairIO<double> {
  using V = double2;
  __device__ __forceinline__ static void split(V v, double, double& a, double& b) { a = v.x; b = v.y; }
  __device__ __forceinline__ static V join(double a, double b, double, uint32_t, int) {
    return make_double2(a, b);
  }
};
template <> struct PairIO<__half> {
  using V = uint32_t;
  static constexpr float kScale = Storage<__half>::kScale;
  __device__ __forceinline__ static void split(V v, float w, float& a, float& b) {
    const float2 t = __half22float2(*reinterpret_cast<const __half2*>(&v));
    a = fmaf(t.x, 1.0f / kScale, w);
    b = fmaf(t.y, 1.0f / kScale, w);
  }
  // (v - w) * 2^14 rounded once (the scaling is exact), then stochastically
  // rounded to f16: the format of Storage::store
  __device__ __forceinline__ static V join(float a, float b, float w, uint32_t h, int q) {
    return cvt_rs_f16x2(fmaf(a, kScale, -w * kScale), fmaf(b, kScale, -w * kScale), pair_bits(h, q));
  }
  // the stored values themselves, (f - w) 2^14, without the shift
  __device__ __forceinline__ static void split_raw(V v, float& a, float& b) {
    const float2 t = __half22float2(*reinterpret_cast<const __half2*>(&v));
    a = t.x;
    b = t.y;
  }
  __device__ __forceinline__ static V join_raw(float a, float b, uint32_t h, int q) {
    return cvt_rs_f16x2(a, b, pair_bits(h, q));
  }
};
template <> struct PairIO<__nv_bfloat16> {
  using V = uint32_t;
  __device__ __forceinline__ static void split(V v, float w, float& a, float& b) {
    a = __uint_as_float(v << 16) + w;
    b = __uint_as_float(v & 0xFFFF0000u) + w;
  }
  __device__ __forceinline__ static V join(float a, float b, float w, uint32_t h, int q) {
    return cvt_rs_bf16x2(a - w, b - w, pair_bits(h, q));
  }
  __device__ __forceinline__ static void split_raw(V v, float& a, float& b) {
    a = __uint_as_float(v << 16);
    b = __uint_as_float(v & 0xFFFF0000u);
  }
  __device__ __forceinline__ static V join_raw(float a, float b, uint32_t h, int q) {
    return cvt_rs_bf16x2(a, b, pair_bits(h, q));
  }
};

template <> struct PairIO<f16_plain> {
  using V = uint32_t;
  __device__ __forceinline__ static void split(V v, float, float& a, float& b) {
    const float2 t = __half22float2(*reinterpret_cast<const __half2*>(&v));
    a = t.x;
    b = t.y;
  }
  __device__ __forceinline__ static V join(float a, float b, float, uint32_t, int) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const V*>(&h);
  }
};
template <> struct PairIO<bf16_plain> {
  using V = uint32_t;
  __device__ __forceinline__ static void split(V v, float, float& a, float& b) {
    a = __uint_as_float(v << 16);
    b = __uint_as_float(v & 0xFFFF0000u);
  }
  __device__ __forceinline__ static V join(float a, float b, float, uint32_t, int) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const V*>(&h);
  }
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
  const int32_t* link_row;  // CURVED cells: row in link_q, may be null
  const float* link_q;      // (rows, Q) BFL wall fractions, 0 = no link, may be null
  int nx, ny, nz;
  int z0, z_count;          // the step updates planes [z0, z0 + z_count) (periodic wrap over nz)
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

// Runtime (dtype, collision, mode) -> template instantiation for one lattice.
// Each lattice's translation unit instantiates dispatch_step<L> once, so the
// three lattices compile in parallel.
#pragma once

#include <type_traits>

#include "tlbm_step.cuh"

namespace tlbm {

// linear forcing: float32 populations, BGK / MRT / Smagorinsky
template <class L, typename S, bool PULL>
int dispatch_forced(const tlbm_desc& d, const StepParams& p, cudaStream_t s) {
  if constexpr (std::is_same<S, float>::value) {
    switch (d.collision) {
      case TLBM_COLL_BGK: return launch_step<L, S, S, TLBM_COLL_BGK, PULL, true>(p, d, s);
      case TLBM_COLL_MRT: return launch_step<L, S, S, TLBM_COLL_MRT, PULL, true>(p, d, s);
      case TLBM_COLL_SMAGORINSKY: return launch_step<L, S, S, TLBM_COLL_SMAGORINSKY, PULL, true>(p, d, s);
      default: return TLBM_ERR_UNSUPPORTED;
    }
  } else {
    return TLBM_ERR_DTYPE;
  }
}

template <class L, typename S, bool PULL>
int dispatch_collision(const tlbm_desc& d, const StepParams& p, cudaStream_t s) {
  if (d.force_lin != 0.0 && d.collision != TLBM_COLL_NONE) return dispatch_forced<L, S, PULL>(d, p, s);
  switch (d.collision) {
    case TLBM_COLL_NONE: return launch_step<L, S, S, TLBM_COLL_NONE, PULL>(p, d, s);
    case TLBM_COLL_BGK: return launch_step<L, S, S, TLBM_COLL_BGK, PULL>(p, d, s);
    case TLBM_COLL_MRT: return launch_step<L, S, S, TLBM_COLL_MRT, PULL>(p, d, s);
    case TLBM_COLL_SMAGORINSKY: return launch_step<L, S, S, TLBM_COLL_SMAGORINSKY, PULL>(p, d, s);
    case TLBM_COLL_TRT: return launch_step<L, S, S, TLBM_COLL_TRT, PULL>(p, d, s);
    case TLBM_COLL_RLBM: return launch_step<L, S, S, TLBM_COLL_RLBM, PULL>(p, d, s);
    case TLBM_COLL_CASCADED:
      if constexpr (L::Q != 9) return launch_step<L, S, S, TLBM_COLL_CASCADED, PULL>(p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    case TLBM_COLL_CUMULANT_D3Q19:
      if constexpr (L::Q == 19) return launch_step<L, S, S, TLBM_COLL_CUMULANT_D3Q19, PULL>(p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    case TLBM_COLL_CUMULANT:
      if constexpr (L::Q == 27) return launch_step<L, S, S, TLBM_COLL_CUMULANT, PULL>(p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    case TLBM_COLL_CUMULANT_GEIER:
      if constexpr (L::Q == 27) return launch_step<L, S, S, TLBM_COLL_CUMULANT_GEIER, PULL>(p, d, s);
      else return TLBM_ERR_UNSUPPORTED;
    default: return TLBM_ERR_UNSUPPORTED;
  }
}

// plain half storage (the drop-in for TensorLBM's Triton kernel): D3Q19
// stream and BGK only
template <class L, typename S, bool PULL>
int dispatch_plain(const tlbm_desc& d, const StepParams& p, cudaStream_t s) {
  if constexpr (L::Q == 19) {
    if (d.force_lin != 0.0) return TLBM_ERR_UNSUPPORTED;
    switch (d.collision) {
      case TLBM_COLL_NONE: return launch_step<L, S, S, TLBM_COLL_NONE, PULL>(p, d, s);
      case TLBM_COLL_BGK: return launch_step<L, S, S, TLBM_COLL_BGK, PULL>(p, d, s);
      default: return TLBM_ERR_UNSUPPORTED;
    }
  } else {
    return TLBM_ERR_UNSUPPORTED;
  }
}

template <class L, bool PULL>
int dispatch_same_dtype(const tlbm_desc& d, const StepParams& p, cudaStream_t s) {
  switch (d.dtype) {
    case TLBM_F16: return dispatch_plain<L, f16_plain, PULL>(d, p, s);
    case TLBM_BF16: return dispatch_plain<L, bf16_plain, PULL>(d, p, s);
    case TLBM_F32: return dispatch_collision<L, float, PULL>(d, p, s);
    case TLBM_F64: return dispatch_collision<L, double, PULL>(d, p, s);
    case TLBM_F16_SHIFTED: return dispatch_collision<L, __half, PULL>(d, p, s);
    case TLBM_BF16_SHIFTED: return dispatch_collision<L, __nv_bfloat16, PULL>(d, p, s);
    default: return TLBM_ERR_DTYPE;
  }
}

// Format conversions (collision NONE): shifted half <-> float32, float64 <-> float32.
template <class L, bool PULL>
int dispatch_convert(const tlbm_desc& d, int dtype_out, const StepParams& p, cudaStream_t s) {
  if (d.collision != TLBM_COLL_NONE) return TLBM_ERR_UNSUPPORTED;
  const int a = d.dtype, b = dtype_out;
  if (a == TLBM_F16_SHIFTED && b == TLBM_F32) return launch_step<L, __half, float, TLBM_COLL_NONE, PULL>(p, d, s);
  if (a == TLBM_BF16_SHIFTED && b == TLBM_F32) return launch_step<L, __nv_bfloat16, float, TLBM_COLL_NONE, PULL>(p, d, s);
  if (a == TLBM_F32 && b == TLBM_F16_SHIFTED) return launch_step<L, float, __half, TLBM_COLL_NONE, PULL>(p, d, s);
  if (a == TLBM_F32 && b == TLBM_BF16_SHIFTED) return launch_step<L, float, __nv_bfloat16, TLBM_COLL_NONE, PULL>(p, d, s);
  if (a == TLBM_F64 && b == TLBM_F32) return launch_step<L, double, float, TLBM_COLL_NONE, PULL>(p, d, s);
  if (a == TLBM_F32 && b == TLBM_F64) return launch_step<L, float, double, TLBM_COLL_NONE, PULL>(p, d, s);
  return TLBM_ERR_DTYPE;
}

template <class L>
int dispatch_step(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s) {
  if (dtype_out == d.dtype) return pull ? dispatch_same_dtype<L, true>(d, p, s) : dispatch_same_dtype<L, false>(d, p, s);
  return pull ? dispatch_convert<L, true>(d, dtype_out, p, s) : dispatch_convert<L, false>(d, dtype_out, p, s);
}

// defined in step_d2q9.cu / step_d3q19.cu / step_d3q27.cu
int dispatch_step_d2q9(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s);
int dispatch_step_d3q19(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s);
int dispatch_step_d3q27(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s);

}  // namespace tlbm

// Fused-step instantiations for D3Q19 (one translation unit per lattice).
#include "tlbm_dispatch.cuh"

namespace tlbm {
int dispatch_step_d3q19(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s) {
  return dispatch_step<D3Q19>(d, dtype_out, pull, p, s);
}
}  // namespace tlbm

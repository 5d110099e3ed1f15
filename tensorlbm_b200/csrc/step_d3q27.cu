// Fused-step instantiations for D3Q27 (one translation unit per lattice).
#include "tlbm_dispatch.cuh"

namespace tlbm {
int dispatch_step_d3q27(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s) {
  return dispatch_step<D3Q27>(d, dtype_out, pull, p, s);
}
}  // namespace tlbm

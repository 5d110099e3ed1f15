// Fused-step instantiations for D2Q9 (one translation unit per lattice).
#include "tlbm_dispatch.cuh"

namespace tlbm {
int dispatch_step_d2q9(const tlbm_desc& d, int dtype_out, bool pull, const StepParams& p, cudaStream_t s) {
  return dispatch_step<D2Q9>(d, dtype_out, pull, p, s);
}
}  // namespace tlbm

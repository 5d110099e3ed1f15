// AA-pattern instantiations for D3Q19 (one translation unit per lattice).
#include "tlbm_aa.cuh"

namespace tlbm {
int dispatch_aa_d3q19(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  return dispatch_aa<D3Q19>(mode, p, d, s);
}
}  // namespace tlbm

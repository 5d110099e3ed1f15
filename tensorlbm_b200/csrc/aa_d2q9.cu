// AA-pattern instantiations for D2Q9 (one translation unit per lattice).
#include "tlbm_aa.cuh"

namespace tlbm {
int dispatch_aa_d2q9(int mode, const StepParams& p, const tlbm_desc& d, cudaStream_t s) {
  return dispatch_aa<D2Q9>(mode, p, d, s);
}
}  // namespace tlbm

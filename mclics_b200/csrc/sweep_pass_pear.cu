// Colour-pass kernels of one potential (instantiations split across files so they compile in parallel).
#include "sweep_pass.cuh"

namespace mcl {

cudaError_t launch_pass_pear(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.flip == true && l.chiral == false && l.field == false) return launch_pass_gp<POT_PEAR, true, false, false>(m, a, l);
  if (l.flip == true && l.chiral == false && l.field == true) return launch_pass_gp<POT_PEAR, true, false, true>(m, a, l);
  return cudaErrorInvalidValue;  // combination not instantiated (flip without field, chirality outside GHRL)
}

}  // namespace mcl

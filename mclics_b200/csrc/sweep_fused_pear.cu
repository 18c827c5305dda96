// Fused sweep kernels of one potential (instantiations split across files so they compile in parallel).
#include "sweep_fused.cuh"

namespace mcl {

cudaError_t launch_fused_pear(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.flip == true && l.chiral == false && l.field == false) return launch_fused_gp<POT_PEAR, true, false, false>(m, a, l);
  if (l.flip == true && l.chiral == false && l.field == true) return launch_fused_gp<POT_PEAR, true, false, true>(m, a, l);
  return cudaErrorInvalidValue;  // combination not instantiated (flip without field, chirality outside GHRL)
}

}  // namespace mcl

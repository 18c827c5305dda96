// Colour-pass kernels of the GHRL potential with the chiral term (sigma != 0).
#include "sweep_pass.cuh"

namespace mcl {

cudaError_t launch_pass_ghrl_chiral(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.flip == false && l.field == false) return launch_pass_gp<POT_GHRL, false, true, false>(m, a, l);
  if (l.flip == false && l.field == true) return launch_pass_gp<POT_GHRL, false, true, true>(m, a, l);
  if (l.flip == true && l.field == true) return launch_pass_gp<POT_GHRL, true, true, true>(m, a, l);
  return cudaErrorInvalidValue;  // combination not instantiated (flip without field)
}

}  // namespace mcl

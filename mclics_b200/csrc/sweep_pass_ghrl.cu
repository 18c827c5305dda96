// Colour-pass kernels of the GHRL potential without the chiral term (instantiations split across files so
// they compile in parallel; the chiral ones are in sweep_pass_ghrl_chiral.cu).
#include "sweep_pass.cuh"

namespace mcl {

cudaError_t launch_pass_ghrl_chiral(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l);

cudaError_t launch_pass_ghrl(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.chiral) return launch_pass_ghrl_chiral(m, a, l);
  if (l.flip == false && l.field == false) return launch_pass_gp<POT_GHRL, false, false, false>(m, a, l);
  if (l.flip == false && l.field == true) return launch_pass_gp<POT_GHRL, false, false, true>(m, a, l);
  if (l.flip == true && l.field == true) return launch_pass_gp<POT_GHRL, true, false, true>(m, a, l);
  return cudaErrorInvalidValue;  // combination not instantiated (flip without field)
}

}  // namespace mcl

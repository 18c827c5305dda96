// Colour-pass kernels of one potential (instantiations split across files so they compile in parallel).
#include "sweep_pass.cuh"

namespace mcl {

cudaError_t launch_pass_ghrl(const ModelDev &m, const FusedArgs &a, const FusedLaunch &l) {
  if (l.flip == false && l.chiral == false && l.field == false) return launch_pass_gp<POT_GHRL, false, false, false>(m, a, l);
  if (l.flip == false && l.chiral == true && l.field == false) return launch_pass_gp<POT_GHRL, false, true, false>(m, a, l);
  if (l.flip == false && l.chiral == false && l.field == true) return launch_pass_gp<POT_GHRL, false, false, true>(m, a, l);
  if (l.flip == false && l.chiral == true && l.field == true) return launch_pass_gp<POT_GHRL, false, true, true>(m, a, l);
  if (l.flip == true && l.chiral == false && l.field == true) return launch_pass_gp<POT_GHRL, true, false, true>(m, a, l);
  if (l.flip == true && l.chiral == true && l.field == true) return launch_pass_gp<POT_GHRL, true, true, true>(m, a, l);
  return cudaErrorInvalidValue;  // combination not instantiated (flip without field, chirality outside GHRL)
}

}  // namespace mcl

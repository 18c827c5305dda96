// Fused two-colour tiled sweep (sweep_fused.cu): both colours of a sweep in one pass over HBM.
#pragma once
#include <utility>
#include <vector>

#include "engine.h"

namespace mcl {

bool fused_supported(const mcl_engine *e);
int fused_create(mcl_engine *e);
void fused_destroy(mcl_engine *e);
// One sweep (both colours, optional fused measurement), then the per-sweep finalisation.
int fused_sweep(mcl_engine *e, bool measure, cudaEvent_t ev0, cudaEvent_t ev1);

}  // namespace mcl

namespace mcl {
// Reads and clears the fused kernel's error word (synchronises); MCL_ERR_CUDA if a TMA wait timed out.
int fused_check_error(mcl_engine *e);
// The device address of that error word (null without the tiled sweep), and the report of a word read from it
// elsewhere: a non-zero word is cleared and turned into MCL_ERR_CUDA.
unsigned int *fused_error_word(mcl_engine *e);
int fused_report_error(mcl_engine *e, unsigned int word);
// Test hook: wait limit in ns (> 0 to change) and whether the first TMA load of every CTA is withheld.
void fused_set_test_hooks(mcl_engine *e, long long timeout_ns, int skip_first_load);
// Tile configuration: 0: fused, 64 x 14 tiles, 256 threads; 1: fused, 64 x 28, 512 threads; 2: colour passes,
// 64 x 16, 256 threads, 3 CTAs/SM; 3: colour passes, 64 x 16, 256 threads, 2 CTAs/SM; 4: colour passes, 32 x 16,
// 128 threads, 5 CTAs/SM.
int fused_set_cfg(mcl_engine *e, int cfg);
int fused_get_cfg(const mcl_engine *e, int *cfg, int *ty, int *seg, int *items);
// Tile configuration and planes per z segment (seg <= 0: the heuristic's choice); rebuilds the work items.
int fused_set_plan(mcl_engine *e, int cfg, int seg);
// Candidate (configuration, planes per segment) pairs for the autotuner, and the threads per CTA of a configuration.
void fused_plan_candidates(const mcl_engine *e, std::vector<std::pair<int, int>> &out);
int fused_threads(int cfg);
// Kernel launches of one sweep of the current plan, finalisation included (fused: 2, colour passes: 3).
int fused_launches_per_sweep(const mcl_engine *e);
// Z-slab support (colour-pass plans only): whether the plan runs colour passes; one colour pass without the
// finalisation; each replica's sums over its work items (kZslabSums doubles: energy, q[6], sum n[3], accepted
// rotations; zeros for the observables when measure = 0); the finalisation from such sums reduced over processes.
bool fused_is_pass_plan(const mcl_engine *e);
// Work items, tensor maps and partials of the learned colour passes' own plan (64 x 8 tiles), built at the first
// call; MCL_ERR_STATE without the tiled sweep.
int fused_learned_view(mcl_engine *e, LearnedPassView *v);
int fused_pass(mcl_engine *e, int colour, bool measure);
int fused_item_sums(mcl_engine *e, int measure, double *d_sums);
int fused_finalize_global(mcl_engine *e, const double *d_sums, int measure);
}  // namespace mcl

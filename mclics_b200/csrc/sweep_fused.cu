// Fused two-colour tiled sweep (placeholder until the tiled kernel lands: reports unsupported).
#include "fused.h"

namespace mcl {

bool fused_supported(const mcl_engine *) { return false; }
int fused_create(mcl_engine *) { return MCL_OK; }
void fused_destroy(mcl_engine *) {}
int fused_sweep(mcl_engine *, bool, cudaEvent_t, cudaEvent_t) { return fail(MCL_ERR_STATE, "fused sweep not available"); }

}  // namespace mcl

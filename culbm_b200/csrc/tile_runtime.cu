// Blocked (L2 temporal blocking) policies.  Placeholder until the tile engine
// lands: blocked configurations are rejected at create time.
#include "sim_internal.cuh"

namespace culbm {

bool is_blocked(const culbm_config& cfg) { return cfg.opt_policy != CULBM_OPT_NONE; }

culbm_status tiles_create(culbm_sim*)
{
    return fail(CULBM_ERR_UNSUPPORTED, "L2 temporal blocking is not built yet");
}
void tiles_destroy(culbm_sim*) {}
culbm_status tiles_upload_flags(culbm_sim*, const uint32_t*) { return CULBM_OK; }
culbm_status tiles_step(culbm_sim*, uint32_t) { return fail(CULBM_ERR_UNSUPPORTED, "no tile engine"); }

}  // namespace culbm

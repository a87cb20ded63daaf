// passes_mixed.cu -- mixed-precision passes (FP32 near field, P2M and L2P;
// compensated M2L).  Not enabled in this build yet: the entry points refuse
// the option instead of running something else.
#include "passes.cuh"

namespace kifmm {

void run_passes_mixed(kifmm_plan *) {
    KIFMM_REQUIRE(false, KIFMM_ERR_UNSUPPORTED, "mixed precision is not built yet");
}
void run_eval_sources_mixed(kifmm_plan *, int) {
    KIFMM_REQUIRE(false, KIFMM_ERR_UNSUPPORTED, "mixed precision is not built yet");
}
void run_eval_targets_mixed(kifmm_plan *, const double *, const double *, int64_t, int, double *) {
    KIFMM_REQUIRE(false, KIFMM_ERR_UNSUPPORTED, "mixed precision is not built yet");
}

}  // namespace kifmm

// m2l_tc.cu -- M2L on the tensor cores (tcgen05), compensated half-precision.
#include "passes.cuh"

namespace kifmm {

bool run_m2l_tensor(kifmm_plan *, const PassArgs &, int) {
    KIFMM_REQUIRE(false, KIFMM_ERR_UNSUPPORTED, "tensor-core M2L forms are not built yet");
    return false;
}

}  // namespace kifmm

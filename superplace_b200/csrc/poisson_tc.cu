// Split-BF16 tensor-core (tcgen05) Poisson path. Placeholder until the kernel lands:
// tc_supported() reports false, so SPG_POISSON_BF16X3 plans are refused with
// SPG_E_INVALID rather than silently running another path.
#include "common.cuh"
#include "poisson.h"

namespace spg {

bool tc_supported(int, int) { return false; }
void tc_plan_create(PoissonPlan&) {
    throw Error(SPG_E_INVALID, "Poisson: split-BF16 path unavailable");
}
void tc_plan_destroy(PoissonPlan&) {}
void tc_solve(PoissonPlan&, int, const float*, float*, float*, float*, cudaStream_t) {
    throw Error(SPG_E_INVALID, "Poisson: split-BF16 path unavailable");
}

}  // namespace spg

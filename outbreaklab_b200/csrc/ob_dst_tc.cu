// ob_dst_tc.cu — bf16x3 tensor-core sine transforms (tcgen05, TMEM accumulators) for the pressure solve.
#include "ob_poisson.cuh"

namespace ob {

int PoissonPlan::tc_create() {
  set_error("poisson: the bf16x3 tensor-core path is not available in this build");
  return OB_ERR_INVALID;
}
int PoissonPlan::tc_solve(const float*, float*, cudaStream_t) {
  set_error("poisson: the bf16x3 tensor-core path is not available in this build");
  return OB_ERR_INVALID;
}
void PoissonPlan::tc_destroy() {}

}  // namespace ob

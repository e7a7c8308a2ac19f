// One (velocity set, storage) instance of the fused step; the build compiles
// this file once per pair with -DLBM_Q=<13|15|19|27> -DLBM_S=<0|1|2>.
#include "lbm_step.cuh"

#if !defined(LBM_Q) || !defined(LBM_S)
#error "compile with -DLBM_Q=<q> -DLBM_S=<storage>"
#endif

namespace lbm {
template int run_step_qs<LBM_Q, LBM_S>(const StepArgs &, bool, int, int, cudaStream_t);
template int run_step_batch_qs<LBM_Q, LBM_S>(const StepArgs *, const unsigned *, int, unsigned,
                                             bool, int, cudaStream_t);
template int run_stats_qs<LBM_Q, LBM_S>(const StepArgs &, bool, unsigned long long *,
                                        cudaStream_t);
}  // namespace lbm

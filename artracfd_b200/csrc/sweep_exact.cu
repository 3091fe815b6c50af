// Stage kernels, exact FP64 form (reference operation order; build with --fmad=false).
#define ACFD_FORM 0
#define ACFD_NS form_exact
#include "sweep_impl.cuh"

namespace acfd {

int launch_stage_exact(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                       cudaStream_t st)
{
    return form_exact::launch_stage_impl(g, m, a, s, viscous, st);
}

int launch_weno_batch_exact(int scheme, const double *F, double *out, int count, cudaStream_t st)
{
    return form_exact::launch_weno_batch_impl(scheme, F, out, count, st);
}

int launch_fhat_batch_exact(const ModelParams &m, int s, const double *U, double *out, int count,
                            cudaStream_t st)
{
    return form_exact::launch_fhat_batch_impl(m, s, U, out, count, st);
}

}  // namespace acfd

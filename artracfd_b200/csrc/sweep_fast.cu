// Stage kernels, fast FP64 form (FMA-contracted).
#define ACFD_FORM 1
#define ACFD_NS form_fast
#include "sweep_impl.cuh"

namespace acfd {

int launch_stage_fast(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                       cudaStream_t st)
{
    return form_fast::launch_stage_impl(g, m, a, s, viscous, st);
}

int launch_weno_batch_fast(int scheme, const double *F, double *out, int count, cudaStream_t st)
{
    return form_fast::launch_weno_batch_impl(scheme, F, out, count, st);
}

int launch_fhat_batch_fast(const ModelParams &m, int s, const double *U, double *out, int count,
                            cudaStream_t st)
{
    return form_fast::launch_fhat_batch_impl(m, s, U, out, count, st);
}

}  // namespace acfd

#include "sweep_brick.cuh"

namespace acfd {

int launch_stage_brick_fast(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            cudaStream_t st)
{
    return form_fast::launch_brick_impl(g, m, a, s, viscous, st);
}

}  // namespace acfd

#include "sweep_march.cuh"

namespace acfd {

int launch_stage_march_fast(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            int target, cudaStream_t st)
{
    return form_fast::launch_march_impl(g, m, a, s, viscous, false, target, st);
}

}  // namespace acfd

#include "sweep_plane.cuh"

namespace acfd {

int launch_stage_plane_fast(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            const PlaneTile &pt, const CUtensorMap &map, cudaStream_t st)
{
    return form_fast::launch_plane_impl(g, m, a, s, viscous, false, pt, map, st);
}

}  // namespace acfd

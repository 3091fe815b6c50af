// Stage kernels, FP32 stencil form with FP64 accumulation.
#define ACFD_FORM 2
#define ACFD_NS form_fp32
#include "sweep_impl.cuh"

namespace acfd {

int launch_stage_fp32(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                       cudaStream_t st)
{
    return form_fp32::launch_stage_impl(g, m, a, s, viscous, st);
}

int launch_weno_batch_fp32(int scheme, const double *F, double *out, int count, cudaStream_t st)
{
    return form_fp32::launch_weno_batch_impl(scheme, F, out, count, st);
}

int launch_fhat_batch_fp32(const ModelParams &m, int s, const double *U, double *out, int count,
                            cudaStream_t st)
{
    return form_fp32::launch_fhat_batch_impl(m, s, U, out, count, st);
}

}  // namespace acfd

#include "sweep_brick.cuh"

namespace acfd {

int launch_stage_brick_fp32(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            cudaStream_t st)
{
    return form_fp32::launch_brick_impl(g, m, a, s, viscous, st);
}

}  // namespace acfd

namespace acfd {

int launch_stage_brick_hybrid(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                              cudaStream_t st)
{
    return form_fp32::launch_brick_hybrid_impl(g, m, a, s, viscous, st);
}

}  // namespace acfd

namespace acfd {

int launch_stage_batch(const BatchCase *cases, const CUtensorMap *maps, const long long *prefix, int ncase,
                       const StageCoefs &sc, const double *dts, unsigned long long *counter, int *status, int blocks,
                       int s, bool hybrid, cudaStream_t st)
{
    return form_fp32::launch_batch_impl(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, s, hybrid, st);
}

}  // namespace acfd

#include "sweep_march.cuh"

namespace acfd {

int launch_stage_march_fp32(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            bool hybrid, int target, cudaStream_t st)
{
    return form_fp32::launch_march_impl(g, m, a, s, viscous, hybrid, target, st);
}

}  // namespace acfd

#include "sweep_plane.cuh"

namespace acfd {

int launch_stage_plane_fp32(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                            bool hybrid, const PlaneTile &pt, const CUtensorMap &map, cudaStream_t st)
{
    return form_fp32::launch_plane_impl(g, m, a, s, viscous, hybrid, pt, map, st);
}

}  // namespace acfd

namespace acfd {

int launch_stage_plane_batch(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                             const long long *prefix, long long blocks, int ncase, const StageCoefs &sc,
                             const double *dts, int *status, int s, bool viscous, bool hybrid, int nthreads, int smem,
                             cudaStream_t st)
{
    return form_fp32::launch_plane_batch_impl(cases, planes, pmaps, prefix, blocks, ncase, sc, dts, status, s, viscous,
                                              hybrid, nthreads, smem, st);
}

int launch_stage_plane_persistent(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                  const long long *prefix, int ncase, const PersistStep &ps, const double *dts,
                                  const BatchLevel *levels, const int4 *pairs, const long long *pair_off,
                                  const long long *fill_pre, unsigned long long *queue, unsigned *done,
                                  unsigned *filled, int *abort, int *status, bool viscous, bool hybrid, int blocks,
                                  int nthreads, int smem, cudaStream_t st)
{
    return form_fp32::launch_plane_persistent_impl(cases, planes, pmaps, prefix, ncase, ps, dts, levels, pairs,
                                                   pair_off, fill_pre, queue, done, filled, abort, status, viscous,
                                                   hybrid, blocks, nthreads, smem, st);
}

int plane_persistent_occupancy(bool viscous, bool hybrid, int nthreads, int smem, int *blocks_per_sm)
{
    return form_fp32::plane_persistent_occupancy_impl(viscous, hybrid, nthreads, smem, blocks_per_sm);
}

}  // namespace acfd

// Domain ghost-node fill (boundary_treatment.c:28-192), CFL wave-speed
// maximum (solve.c:108-153), gravity source stage (source_term.c:21-39) and
// the reference-layout <-> device-layout conversion.
//
// Compiled with --fmad=false: the primitive/conservative maps and the
// method-of-images arithmetic are evaluated in the reference's order, so the
// filled ghost values are bitwise those of the reference.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "acfd_internal.cuh"
#include "fast_div.h"

namespace acfd {

namespace {

__device__ __forceinline__ long long node_of(const Grid &g, int i, int j, int k)
{
    return ((long long)k * g.n[1] + j) * g.pitch + i;
}

// loads bypass L1: in the fused ghost fill a value may have been written by
// another SM in the previous phase of the same launch
__device__ __forceinline__ void load5(const double *U, long long nn, long long id, double u[5])
{
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        u[v] = __ldcg(U + v * nn + id);
    }
}

__device__ __forceinline__ void store5(double *U, long long nn, long long id, const double u[5])
{
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        U[v * nn + id] = u[v];
    }
}

// MapPrimitive / MapConservative (cfd_commons.c:296-322)
__device__ __forceinline__ void to_primitive(double gamma, double gasR, const double U[5], double Uo[6])
{
    Uo[0] = U[0];
    Uo[1] = U[1] / U[0];
    Uo[2] = U[2] / U[0];
    Uo[3] = U[3] / U[0];
    Uo[4] = (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]) * (gamma - 1.0);
    Uo[5] = Uo[4] / (Uo[0] * gasR);
}

__device__ __forceinline__ void to_conservative(double gamma, const double Uo[6], double U[5])
{
    U[0] = Uo[0];
    U[1] = Uo[0] * Uo[1];
    U[2] = Uo[0] * Uo[2];
    U[3] = Uo[0] * Uo[3];
    U[4] = 0.5 * Uo[0] * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3]) + Uo[4] / (gamma - 1.0);
}

struct FaceJob {
    int lo[3];
    int ext[3];
    int N[3];
    int LN[3];
    int type;
    int r;
    long long count;
    double given[6];
};

struct FaceJobs {
    FaceJob job[2];
    int njob;
};

__device__ void fill_node(const Grid &g, const ModelParams &mp, const FaceJob &J, long long t, double *U);

__global__ void domain_fill(Grid g, ModelParams mp, FaceJobs jobs, double *U)
{
    pdl_wait();
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int q = 0;
    if (t >= jobs.job[0].count) {
        t -= jobs.job[0].count;
        q = 1;
        if (jobs.njob < 2 || t >= jobs.job[1].count) {
            return;
        }
    }
    fill_node(g, mp, jobs.job[q], t, U);
}

// All phases of one TreatBoundary in one cooperative launch: the blocks sweep
// the boxes of a phase, then meet at a grid barrier before the next phase.
constexpr int kMaxPhases = 16;
struct PhasePlan {
    FaceJobs phase[kMaxPhases];
    int nphase;
};

constexpr long long kBarrierSpinLimit = 1LL << 22;

// Grid barrier for co-resident blocks (cooperative launch).  bar[0] counts
// arrivals, bar[1] is the generation.  A block that waits longer than the
// spin limit records error 5 and returns false.
__device__ bool grid_barrier(unsigned *bar, unsigned nblocks, int *status)
{
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        ok = 1;
        volatile unsigned *gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        if (atomicAdd(bar, 1u) == nblocks - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            long long it = 0;
            while (*gen == g0) {
                if (++it > kBarrierSpinLimit) {
                    atomicExch(status, 5);
                    ok = 0;
                    break;
                }
                __nanosleep(20);
            }
        }
        __threadfence();
    }
    __syncthreads();
    return ok != 0;
}

__global__ void __launch_bounds__(1024) domain_fill_fused(Grid g, ModelParams mp, PhasePlan plan, double *U,
                                                          unsigned *bar, int *status)
{
    const long long nthreads = (long long)gridDim.x * blockDim.x;
    for (int ph = 0; ph < plan.nphase; ++ph) {
        const FaceJobs &jobs = plan.phase[ph];
        const long long total = jobs.job[0].count + (jobs.njob > 1 ? jobs.job[1].count : 0);
        for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += nthreads) {
            if (t < jobs.job[0].count) {
                fill_node(g, mp, jobs.job[0], t, U);
            } else {
                fill_node(g, mp, jobs.job[1], t - jobs.job[0].count, U);
            }
        }
        if (ph + 1 < plan.nphase) {
            __threadfence();
            if (!grid_barrier(bar, gridDim.x, status)) {
                return;
            }
        }
    }
}

// method of images of a wall ghost node from its boundary point O and image
// node I (boundary_treatment.c:105-115 with DoMethodOfImage,
// immersed_boundary.c:341-356)
__device__ __forceinline__ void image_ghost(const ModelParams &mp, const double UO[5], const double UI[5],
                                            double Ut[5])
{
    double UoO[6], UoI[6], UoG[6];
    to_primitive(mp.gamma, mp.gasR, UO, UoO);
    to_primitive(mp.gamma, mp.gasR, UI, UoI);
    UoG[1] = UoO[1] + UoO[1] - UoI[1];
    UoG[2] = UoO[2] + UoO[2] - UoI[2];
    UoG[3] = UoO[3] + UoO[3] - UoI[3];
    UoG[4] = UoI[4];
    UoG[5] = UoI[5];
    UoG[0] = UoG[4] / (UoG[5] * mp.gasR);
    to_conservative(mp.gamma, UoG, Ut);
}

// slip (type 2) or no-slip (type 3) wall boundary node from its inner
// neighbour h (boundary_treatment.c:148-177); given5 < 0: adiabatic
__device__ __forceinline__ void wall_node(const ModelParams &mp, int type, const int N[3], double given5,
                                          const double Uh[5], double Ut[5])
{
    double Uoh[6], UoO[6];
    to_primitive(mp.gamma, mp.gasR, Uh, Uoh);
    if (type == 2) {
        UoO[1] = (double)(!N[0]) * Uoh[1];
        UoO[2] = (double)(!N[1]) * Uoh[2];
        UoO[3] = (double)(!N[2]) * Uoh[3];
    } else {
        UoO[1] = 0.0;
        UoO[2] = 0.0;
        UoO[3] = 0.0;
    }
    UoO[4] = Uoh[4];
    UoO[5] = (0.0 > given5) ? Uoh[5] : given5;
    UoO[0] = UoO[4] / (UoO[5] * mp.gasR);
    to_conservative(mp.gamma, UoO, Ut);
}

__device__ void fill_node(const Grid &g, const ModelParams &mp, const FaceJob &J, long long t, double *U)
{
    const int i = J.lo[0] + (int)(t % J.ext[0]);
    const long long rest = t / J.ext[0];
    const int j = J.lo[1] + (int)(rest % J.ext[1]);
    const int k = J.lo[2] + (int)(rest / J.ext[1]);
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    const int *N = J.N;
    const int r = J.r;
    double Ut[5];
    if (r != 0) {
        // ghost layer r
        if (J.type == 2 || J.type == 3) {
            double UO[5], UI[5];
            load5(U, nn, node_of(g, i - r * N[0], j - r * N[1], k - r * N[2]), UO);
            load5(U, nn, node_of(g, i - 2 * r * N[0], j - 2 * r * N[1], k - 2 * r * N[2]), UI);
            image_ghost(mp, UO, UI, Ut);
        } else if (J.type == 4) {
            load5(U, nn, node_of(g, i - J.LN[0], j - J.LN[1], k - J.LN[2]), Ut);
        } else {
            load5(U, nn, node_of(g, i - N[0], j - N[1], k - N[2]), Ut);
        }
        store5(U, nn, id, Ut);
        return;
    }
    // physical boundary node
    switch (J.type) {
        case 0:  // inflow
            to_conservative(mp.gamma, J.given, Ut);
            break;
        case 1:  // outflow
            load5(U, nn, node_of(g, i - N[0], j - N[1], k - N[2]), Ut);
            break;
        case 2:  // slip wall
        case 3: {  // no-slip wall
            double Uh[5];
            load5(U, nn, node_of(g, i - N[0], j - N[1], k - N[2]), Uh);
            wall_node(mp, J.type, N, J.given[5], Uh, Ut);
            break;
        }
        default:  // periodic: the boundary plane is computed like an interior node
            return;
    }
    store5(U, nn, id, Ut);
}

// debug mode: count the non-finite values of one level (all nodes, all five
// variables; padding and never-written nodes hold finite values)
__global__ void finite_scan(const double *__restrict__ U, long long count, int *word)
{
    int bad = 0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        bad += !isfinite(U[t]);
    }
    bad = __reduce_add_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad > 0) {
        atomicAdd(word, bad);
    }
}

// CFL: per-direction max of |u_s| + sqrt(gamma*gasR*T) over PIN nodes with
// did == 0 (the max is order independent, so the result is the reference's)
__device__ __forceinline__ double vmax_of(double a, double b)
{
    return (a < b) ? b : a;  // NaN in b never replaces a, as in solve.c:145
}

// The maximum of the wave speeds over the computed fluid nodes, per sweep
// direction, in one launch: each block reduces its nodes and writes its three
// partial maxima and a non-finite flag; the last block to finish (a counter
// after the partials, zero between launches) combines all blocks' partials
// with the whole block and writes out[0..3].  Every partial maximum starts
// from 0 and a NaN never replaces a value (vmax_of), so no NaN enters and the
// maximum does not depend on the order of combination.
// div_x, div_y: division by the PIN extents along x and y (32-bit path).
__global__ void cfl_partial(Grid g, ModelParams mp, const double *U, const int *did, double *part, double *out,
                            FastDiv div_x, FastDiv div_y)
{
    pdl_wait();
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long total = (long long)Lx * Ly * Lz;
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    bool bad = false;  // a fluid node whose wave speed is not finite
    // the node type and the state are loaded together (one memory round
    // trip, not two); a node that is not a fluid node is passed over after
    auto visit = [&](long long id) {
        const int d = did[id];
        double Uc[5], Uo[6];
        load5(U, g.nn, id, Uc);
        if (d != 0) {
            return;
        }
        to_primitive(mp.gamma, mp.gasR, Uc, Uo);
        const double c = sqrt(mp.gamma * mp.gasR * Uo[5]);
        const double v0 = fabs(Uo[1]) + c, v1 = fabs(Uo[2]) + c, v2 = fabs(Uo[3]) + c;
        m0 = vmax_of(m0, v0);
        m1 = vmax_of(m1, v1);
        m2 = vmax_of(m2, v2);
        // the maximum passes over a NaN as the reference's does; it is
        // reported beside it (a blown-up or corrupted state)
        bad = bad || !isfinite(v0 + v1 + v2);
    };
    if (total < (long long)INT32_MAX / 2 && g.nn < (long long)INT32_MAX) {
        // 32-bit work indices: 64-bit divisions would cost more than the loads
        const int tot = (int)total, sy = g.pitch, sz = g.pitch * g.n[1];
        const int stride = (int)(gridDim.x * blockDim.x);
        auto node = [&](int t) {
            const int rest = (int)fast_div((uint32_t)t, div_x);
            const int kk = (int)fast_div((uint32_t)rest, div_y);
            return (long long)((g.lo[2] + kk) * sz + (g.lo[1] + rest - kk * Ly) * sy + g.lo[0] + t - rest * Lx);
        };
        // two nodes an iteration: both nodes' loads in flight at once
        int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
        for (; t + stride < tot; t += 2 * stride) {
            const long long a = node(t), b = node(t + stride);
            visit(a);
            visit(b);
        }
        if (t < tot) visit(node(t));
    } else {
        for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
             t += (long long)gridDim.x * blockDim.x) {
            const int i = g.lo[0] + (int)(t % Lx);
            const long long rest = t / Lx;
            const int j = g.lo[1] + (int)(rest % Ly);
            const int k = g.lo[2] + (int)(rest / Ly);
            visit(node_of(g, i, j, k));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        m0 = vmax_of(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = vmax_of(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = vmax_of(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    __shared__ double sm[4][32];
    __shared__ bool last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    if (lane == 0) {
        sm[0][warp] = m0;
        sm[1][warp] = m1;
        sm[2][warp] = m2;
    }
    const int any_bad = __syncthreads_or(bad);
    if (threadIdx.x < 3) {
        double m = 0.0;
        for (int w = 0; w < nw; ++w) {
            m = vmax_of(m, sm[threadIdx.x][w]);
        }
        part[3 * blockIdx.x + threadIdx.x] = m;
    }
    if (threadIdx.x == 3) {
        part[3 * gridDim.x + blockIdx.x] = any_bad ? 1.0 : 0.0;
    }
    if (threadIdx.x < 4) {
        __threadfence();  // the partials before the count
    }
    __syncthreads();
    unsigned *count = reinterpret_cast<unsigned *>(part + 4 * gridDim.x);
    if (threadIdx.x == 0) {
        last = atomicAdd(count, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) {
        return;
    }
    // the last block: every block's partials (written by other SMs: read
    // through L2)
    double r[3] = {0.0, 0.0, 0.0};
    double nbad = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            r[q] = vmax_of(r[q], __ldcg(part + 3 * b + q));
        }
        nbad += __ldcg(part + 3 * gridDim.x + b);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int q = 0; q < 3; ++q) {
            r[q] = vmax_of(r[q], __shfl_xor_sync(0xffffffffu, r[q], o));
        }
        nbad += __shfl_xor_sync(0xffffffffu, nbad, o);
    }
    __syncthreads();  // sm is reused
    if (lane == 0) {
        sm[0][warp] = r[0];
        sm[1][warp] = r[1];
        sm[2][warp] = r[2];
        sm[3][warp] = nbad;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < nw; ++w) {
            v = threadIdx.x < 3 ? vmax_of(v, sm[threadIdx.x][w]) : v + sm[3][w];
        }
        // out[3]: blocks that met a fluid node with a non-finite wave speed
        out[threadIdx.x] = v;
    }
    if (threadIdx.x == 0) {
        *count = 0u;  // for the next launch (stream order)
    }
}

// gravity source stage: LLLU with p = PHI (fluid_dynamics.c:177-214)
__global__ void stage_phi(Grid g, ModelParams mp, StageArgs a)
{
    pdl_wait();
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long total = (long long)Lx * Ly * Lz;
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) {
        return;
    }
    const int i = g.lo[0] + (int)(t % Lx);
    const long long rest = t / Lx;
    const int j = g.lo[1] + (int)(rest % Ly);
    const int k = g.lo[2] + (int)(rest / Ly);
    const long long id = node_of(g, i, j, k);
    if (a.did[id] != 0) {
        return;
    }
    const double dt = a.dt_scale * a.dt[0];
    double Phi[5];
    if (mp.sState == 0) {
        for (int v = 0; v < 5; ++v) Phi[v] = 0.0;
    } else {
        double Un[5];
        load5(a.Un, g.nn, id, Un);
        const double V[3] = {Un[1] / Un[0], Un[2] / Un[0], Un[3] / Un[0]};
        const double fb[3] = {Un[0] * mp.g[0], Un[0] * mp.g[1], Un[0] * mp.g[2]};
        Phi[0] = 0.0;
        Phi[1] = fb[0];
        Phi[2] = fb[1];
        Phi[3] = fb[2];
        Phi[4] = fb[0] * V[0] + fb[1] * V[1] + fb[2] * V[2];
    }
    for (int v = 0; v < 5; ++v) {
        const long long q = v * g.nn + id;
        a.Um[q] = a.coeA * a.Uo[q] + a.coeB * (a.Un[q] + dt * Phi[v]);
    }
}

// reference node records (AoS, 136 B) <-> device planes
__global__ void scatter_nodes(Grid g, const acfd_node_t *staged, double *U, int *flags, unsigned mask)
{
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) {
        return;
    }
    const int i = (int)(t % g.n[0]);
    const long long rest = t / g.n[0];
    const int j = (int)(rest % g.n[1]);
    const int k = (int)(rest / g.n[1]);
    const long long id = node_of(g, i, j, k);
    const acfd_node_t &nd = staged[t];
    for (int l = 0; l < kLevels; ++l) {
        if (mask & (1u << l)) {
            for (int v = 0; v < kVars; ++v) {
                U[((long long)l * kVars + v) * g.nn + id] = nd.U[l][v];
            }
        }
    }
    if (mask & ACFD_SYNC_FLAGS) {
        flags[id] = nd.did;
        flags[g.nn + id] = nd.fid;
        flags[2 * g.nn + id] = nd.lid;
        flags[3 * g.nn + id] = nd.gst;
    }
}

__global__ void gather_nodes(Grid g, const double *U, const int *flags, acfd_node_t *staged, unsigned mask)
{
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total) {
        return;
    }
    const int i = (int)(t % g.n[0]);
    const long long rest = t / g.n[0];
    const int j = (int)(rest % g.n[1]);
    const int k = (int)(rest / g.n[1]);
    const long long id = node_of(g, i, j, k);
    acfd_node_t &nd = staged[t];
    for (int l = 0; l < kLevels; ++l) {
        if (mask & (1u << l)) {
            for (int v = 0; v < kVars; ++v) {
                nd.U[l][v] = U[((long long)l * kVars + v) * g.nn + id];
            }
        }
    }
    if (mask & ACFD_SYNC_FLAGS) {
        nd.did = flags[id];
        nd.fid = flags[g.nn + id];
        nd.lid = flags[2 * g.nn + id];
        nd.gst = flags[3 * g.nn + id];
    }
}

unsigned blocks_for(long long n, int bs)
{
    return (unsigned)((n + bs - 1) / bs);
}

}  // namespace

// U[dst] = U[src], all five variables: the five loads are issued before the
// first store (U is both read and written, so a store may not be moved above
// a later load; loads issued first keep five requests in flight)
__device__ __forceinline__ void copy_node(double *U, long long nn, long long dst, long long src)
{
    double u[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        u[v] = U[v * nn + src];
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        U[v * nn + dst] = u[v];
    }
}

// Ghost fill of a case whose faces are all copies (periodic, outflow): every
// changed node takes the value of one unchanged node, so the ordered faces
// collapse into one gather (pairs: destination, source node index)
__global__ void ghost_gather(long long nn, const int2 *__restrict__ pairs, int count, double *U)
{
    pdl_wait();
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < count; t += gridDim.x * blockDim.x) {
        const int2 q = pairs[t];
        copy_node(U, nn, q.x, q.y);
    }
}

int launch_ghost_gather(const Grid &g, const int2 *pairs, int count, double *U, cudaStream_t st)
{
    if (count <= 0) {
        return ACFD_OK;
    }
    const int blocks = (int)blocks_for(count, 256);
    cudaError_t e = launch_k(ghost_gather, dim3(blocks), dim3(256), 0, st, g.nn, pairs, count, U);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "ghost_gather launch");
}

// Ghost fill as one launch of formulas (see build_bc_program): the first
// nchunk blocks copy one run of nodes each; then a thread per remaining copy
// (U[dst] = U[src]) and a thread per postfix program -- LOAD pushes a node's
// five values, INFLOW the given inflow state,
// WALL replaces the top with the wall formula of a boundary node, IMAGE
// replaces the top two (boundary point O, image node I) with the image
// ghost -- and store the result.  No node a program or pair reads is written
// by the launch, so the threads need no ordering among themselves.
__global__ void __launch_bounds__(256) ghost_program(long long nn, const int4 *__restrict__ tasks, int ntask,
                                                     const int2 *__restrict__ single, int nsingle,
                                                     const int4 *__restrict__ progs, int nprog,
                                                     const int2 *__restrict__ ops, GhostFaces F, ModelParams mp,
                                                     double *U)
{
    pdl_wait();
    if ((int)blockIdx.x < ntask) {
        // a run of copies, up to four per thread in flight: their twenty
        // loads before their stores
        const int4 c = tasks[blockIdx.x];
        for (int q0 = threadIdx.x; q0 < c.z; q0 += 4 * blockDim.x) {
            long long d[4];
            double u[4][5];
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const int q = q0 + r * (int)blockDim.x;
                d[r] = q < c.z ? (long long)c.x + q : -1;
                // a copy outside the level is dropped (the tasks cover exactly
                // the fill's copies: tests/test_host.py)
                if (d[r] >= nn || d[r] + c.y < 0 || d[r] + c.y >= nn) d[r] = -1;
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (d[r] >= 0) {
#pragma unroll
                    for (int v = 0; v < 5; ++v) u[r][v] = U[v * nn + d[r] + c.y];
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                if (d[r] >= 0) {
#pragma unroll
                    for (int v = 0; v < 5; ++v) U[v * nn + d[r]] = u[r][v];
                }
            }
        }
        return;
    }
    const int t = ((int)blockIdx.x - ntask) * blockDim.x + threadIdx.x;
    if (t < nsingle) {
        const int2 q = single[t];
        copy_node(U, nn, q.x, q.y);
        return;
    }
    if (t >= nsingle + nprog) {
        return;
    }
    const int4 pr = progs[t - nsingle];  // dst, first op, op count
    double st[kGhostStack][5];
    int sp = 0;
    for (int o = 0; o < pr.z; ++o) {
        const int2 op = ops[pr.y + o];
        const int code = op.x & 7, face = op.x >> 3;
        if (code == kGhostLoad) {
            load5(U, nn, op.y, st[sp]);
            ++sp;
        } else if (code == kGhostInflow) {
            to_conservative(mp.gamma, F.given[face], st[sp]);
            ++sp;
        } else if (code == kGhostWall) {
            double Ut[5];
            wall_node(mp, F.type[face], F.N[face], F.given[face][5], st[sp - 1], Ut);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                st[sp - 1][v] = Ut[v];
            }
        } else {  // kGhostImage
            double Ut[5];
            image_ghost(mp, st[sp - 2], st[sp - 1], Ut);
            --sp;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                st[sp - 1][v] = Ut[v];
            }
        }
    }
    store5(U, nn, pr.x, st[0]);
}

int launch_ghost_program(const Grid &g, const ModelParams &m, const GhostFaces &F, const int4 *tasks, int ntask,
                         const int2 *single, int nsingle, const int4 *progs, int nprog, const int2 *ops, double *U,
                         cudaStream_t st)
{
    const long long rest = (long long)nsingle + nprog;
    const long long blocks = ntask + (rest + 255) / 256;
    if (blocks <= 0) {
        return ACFD_OK;
    }
    cudaError_t e = launch_k(ghost_program, dim3((unsigned)blocks), dim3(256), 0, st, g.nn, tasks, ntask, single,
                             nsingle, progs, nprog, ops, F, m, U);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "ghost_program launch");
}

// ghost fill of all cases of a batch in one launch (copy-only cases, see
// ghost_gather)
__global__ void batch_ghost_gather(const BatchLevel *__restrict__ cases, const int4 *__restrict__ pairs,
                                   long long count, int tn)
{
    pdl_wait();
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < count;
         t += (long long)gridDim.x * blockDim.x) {
        const int4 q = pairs[t];
        const BatchLevel c = cases[q.x];
        copy_node(c.U + (long long)tn * 5 * c.nn, c.nn, q.y, q.z);
    }
}

int launch_batch_gather(const BatchLevel *cases, const int4 *pairs, long long count, int tn, cudaStream_t st)
{
    if (count <= 0) {
        return ACFD_OK;
    }
    const long long want = (count + 255) / 256;
    const unsigned blocks = (unsigned)(want < 148 * 64 ? want : 148 * 64);
    cudaError_t e = launch_k(batch_ghost_gather, dim3(blocks), dim3(256), 0, st, cases, pairs, count, tn);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "batch_ghost_gather launch");
}

// per-case dt of a batch, in the order of the reference's expression
__global__ void batch_dt(const double *const *vmax, const double *d, const double *cfl, double *dts, int ncase)
{
    pdl_wait();
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncase) {
        return;
    }
    const double *v = vmax[c];
    const double a = d[3 * c + 1] / v[1];
    const double b = d[3 * c + 2] / v[2];
    const double inner = (a < b) ? a : b;
    const double x = d[3 * c] / v[0];
    dts[c] = cfl[c] * ((x < inner) ? x : inner);
}

int launch_batch_dt(const double *const *vmax, const double *d, const double *cfl, double *dts, int ncase,
                    cudaStream_t st)
{
    cudaError_t e = launch_k(batch_dt, dim3((ncase + 127) / 128), dim3(128), 0, st, vmax, d, cfl, dts, ncase);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "batch_dt launch");
}

int launch_domain_boundary(const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                           const FaceBox *boxes, int nbox, double *U, cudaStream_t st)
{
    if (nbox < 1 || nbox > 2) {
        set_error("domain boundary group of %d faces", nbox);
        return ACFD_ERR_ARG;
    }
    FaceJobs jobs;
    jobs.njob = nbox;
    long long total = 0;
    for (int q = 0; q < nbox; ++q) {
        FaceJob &J = jobs.job[q];
        const FaceBox &b = boxes[q];
        const int p = b.face;
        for (int s = 0; s < 3; ++s) {
            J.lo[s] = b.box[s][0];
            J.ext[s] = b.box[s][1] - b.box[s][0];
            J.N[s] = part.N[p][s];
            J.LN[s] = part.m[s] * part.N[p][s];
        }
        J.type = part.typeBC[p];
        J.r = b.r;
        J.count = (long long)J.ext[0] * J.ext[1] * J.ext[2];
        for (int v = 0; v < 6; ++v) {
            J.given[v] = part.varBC[p][v];
        }
        total += J.count;
    }
    if (nbox == 1) {
        jobs.job[1] = jobs.job[0];
        jobs.job[1].count = 0;
    }
    if (total == 0) {
        return ACFD_OK;
    }
    cudaError_t e = launch_k(domain_fill, dim3(blocks_for(total, 256)), dim3(256), 0, st, g, m, jobs, U);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "domain_fill launch");
}

static int fill_jobs(const acfd_partition_t &part, const FaceBox *boxes, int nbox, FaceJobs &jobs)
{
    jobs.njob = nbox;
    for (int q = 0; q < nbox; ++q) {
        FaceJob &J = jobs.job[q];
        const FaceBox &b = boxes[q];
        const int p = b.face;
        for (int s = 0; s < 3; ++s) {
            J.lo[s] = b.box[s][0];
            J.ext[s] = b.box[s][1] - b.box[s][0];
            J.N[s] = part.N[p][s];
            J.LN[s] = part.m[s] * part.N[p][s];
        }
        J.type = part.typeBC[p];
        J.r = b.r;
        J.count = (long long)J.ext[0] * J.ext[1] * J.ext[2];
        for (int v = 0; v < 6; ++v) {
            J.given[v] = part.varBC[p][v];
        }
    }
    if (nbox == 1) {
        jobs.job[1] = jobs.job[0];
        jobs.job[1].count = 0;
    }
    return ACFD_OK;
}

int launch_domain_boundary_fused(const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                                 const FaceBox *const *groups, const int *sizes, int ngroups, double *U,
                                 unsigned *bar, int *status, cudaStream_t st)
{
    if (ngroups <= 0) {
        return ACFD_OK;
    }
    if (ngroups > kMaxPhases) {
        set_error("fused ghost fill: %d phases (at most %d)", ngroups, kMaxPhases);
        return ACFD_ERR_ARG;
    }
    PhasePlan plan;
    plan.nphase = ngroups;
    for (int q = 0; q < ngroups; ++q) {
        if (sizes[q] < 1 || sizes[q] > 2) {
            set_error("fused ghost fill: phase of %d faces", sizes[q]);
            return ACFD_ERR_ARG;
        }
        fill_jobs(part, groups[q], sizes[q], plan.phase[q]);
    }
    // every block must be resident at once for the grid barrier
    static int blocks_per_sm[64] = {0};
    static int sms[64] = {0};
    int dev = 0;
    ACFD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("device ordinal %d", dev);
        return ACFD_ERR_ARG;
    }
    // few large blocks: the barrier cost grows with the number of arriving
    // blocks (ACFD_BC_BLOCKS overrides the default of 64 x 1024 threads)
    static int nb_env = -1;
    if (nb_env < 0) {
        const char *e = getenv("ACFD_BC_BLOCKS");
        nb_env = e ? atoi(e) : 64;
    }
    if (!blocks_per_sm[dev]) {
        ACFD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm[dev], domain_fill_fused, 1024, 0));
        ACFD_CUDA(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
        if (blocks_per_sm[dev] < 1) {
            set_error("fused ghost fill cannot be resident");
            return ACFD_ERR_CUDA;
        }
    }
    const unsigned nblocks = (unsigned)std::max(1, std::min(nb_env, sms[dev] * blocks_per_sm[dev]));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(1024);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    ACFD_CUDA(cudaLaunchKernelEx(&cfg, domain_fill_fused, g, m, plan, U, bar, status));
    return ACFD_OK;
}

int launch_cfl(const Grid &g, const ModelParams &m, const double *U, const int *did, double *partials,
               double *out, cudaStream_t st)
{
    const FastDiv div_x = make_fast_div((uint32_t)std::max(1, g.hi[0] - g.lo[0]));
    const FastDiv div_y = make_fast_div((uint32_t)std::max(1, g.hi[1] - g.lo[1]));
    cudaError_t e = launch_k(cfl_partial, dim3(kCflBlocks), dim3(256), 0, st, g, m, U, did, partials, out, div_x,
                             div_y);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "cfl launch");
}

// Arrays transposed between two grids whose axes 0 and 1 are exchanged:
// element (a, b, k) of src -- index (k * nb + b) * src_pitch + a, a < na the
// fast axis -- goes to index (k * na + a) * dst_pitch + b of dst, for each of
// NV variables; with swap_uv variables 1 and 2 (the x and y momenta) trade
// places, so that a transposed state is the same flow with the axes renamed.
// 32 x 32 tiles through shared memory, both sides coalesced; one block moves
// the tile of every variable, so that a thread has 4 * NV loads in flight
// before the barrier (one variable per block leaves HBM half idle).
template <typename T, int NV>
__global__ void __launch_bounds__(256) transpose_xy(const T *__restrict__ src, long long src_nn, int src_pitch,
                                                    T *__restrict__ dst, long long dst_nn, int dst_pitch, int na,
                                                    int nb, bool swap_uv)
{
    pdl_wait();
    __shared__ T tile[NV][32][33];
    const int k = (int)blockIdx.z;
    const int a0 = blockIdx.x * 32, b0 = blockIdx.y * 32;
    {
        const int a = a0 + threadIdx.x;
#pragma unroll
        for (int v = 0; v < NV; ++v) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = threadIdx.y + 8 * i, b = b0 + r;
                if (a < na && b < nb) tile[v][r][threadIdx.x] = src[v * src_nn + ((long long)k * nb + b) * src_pitch + a];
            }
        }
    }
    __syncthreads();
    const int b = b0 + threadIdx.x;
#pragma unroll
    for (int v = 0; v < NV; ++v) {
        const int vd = swap_uv ? (v == 1 ? 2 : (v == 2 ? 1 : v)) : v;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int r = threadIdx.y + 8 * i, a = a0 + r;
            if (a < na && b < nb) dst[vd * dst_nn + ((long long)k * na + a) * dst_pitch + b] = tile[v][threadIdx.x][r];
        }
    }
}

template <typename T, int NV>
static int launch_transpose(const T *src, const Grid &gs, T *dst, const Grid &gd, bool swap_uv, cudaStream_t st)
{
    if (gs.n[0] != gd.n[1] || gs.n[1] != gd.n[0] || gs.n[2] != gd.n[2] || gs.n[2] > 65535) {
        set_error("transpose: grids (%d, %d, %d) and (%d, %d, %d) are not each other's transpose", gs.n[0], gs.n[1],
                  gs.n[2], gd.n[0], gd.n[1], gd.n[2]);
        return ACFD_ERR_ARG;
    }
    const dim3 grid((unsigned)((gs.n[0] + 31) / 32), (unsigned)((gs.n[1] + 31) / 32), (unsigned)gs.n[2]);
    cudaError_t e = launch_k(transpose_xy<T, NV>, grid, dim3(32, 8), 0, st, src, gs.nn, gs.pitch, dst, gd.nn,
                             gd.pitch, gs.n[0], gs.n[1], swap_uv);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "transpose launch");
}

int launch_transpose_state(const double *src, const Grid &gs, double *dst, const Grid &gd, cudaStream_t st)
{
    return launch_transpose<double, 5>(src, gs, dst, gd, true, st);
}

int launch_transpose_int(const int *src, const Grid &gs, int *dst, const Grid &gd, cudaStream_t st)
{
    return launch_transpose<int, 1>(src, gs, dst, gd, false, st);
}

int launch_transpose_u8(const uint8_t *src, const Grid &gs, uint8_t *dst, const Grid &gd, cudaStream_t st)
{
    return launch_transpose<uint8_t, 1>(src, gs, dst, gd, false, st);
}

int launch_finite_scan(const double *U, long long count, int *word, cudaStream_t st)
{
    const unsigned blocks = (unsigned)std::min<long long>(blocks_for(count, 256), 148LL * 8);
    finite_scan<<<blocks, 256, 0, st>>>(U, count, word);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "finite_scan launch");
}

int launch_stage_phi(const Grid &g, const ModelParams &m, const StageArgs &a, cudaStream_t st)
{
    const long long total = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    if (total <= 0) {
        return ACFD_OK;
    }
    cudaError_t e = launch_k(stage_phi, dim3(blocks_for(total, 256)), dim3(256), 0, st, g, m, a);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_phi launch");
}

int launch_scatter_nodes(const Grid &g, const acfd_node_t *staged, double *U, int *flags, unsigned mask,
                         cudaStream_t st)
{
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    scatter_nodes<<<blocks_for(total, 256), 256, 0, st>>>(g, staged, U, flags, mask);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "scatter_nodes launch");
}

int launch_gather_nodes(const Grid &g, const double *U, const int *flags, acfd_node_t *staged, unsigned mask,
                        cudaStream_t st)
{
    const long long total = (long long)g.n[0] * g.n[1] * g.n[2];
    gather_nodes<<<blocks_for(total, 256), 256, 0, st>>>(g, U, flags, staged, mask);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "gather_nodes launch");
}

}  // namespace acfd

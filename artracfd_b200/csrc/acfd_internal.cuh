// Internal declarations of libacfd_gpu (not part of the C ABI).
//
// Device layout of one case ("structure of arrays", FP64 state):
//   U[level][var][node]   level in {TO,TN,TM}, var in rho,rho*u,rho*v,rho*w,rho*eT
//   node = (k * n[Y] + j) * pitch + i        pitch = n[X] rounded up to 8 doubles
//   did, fid, lid, gst    int32 planes with the same node index
// so that each variable of each level is a 3D array whose x-rows start on a
// 64-byte boundary and whose accesses along x are fully coalesced.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "acfd.h"
#include "launch.cuh"

namespace acfd {

constexpr int kLevels = 3;
constexpr int kVars = 5;

// Everything a stage kernel needs about the grid and the model, passed by
// value (fits in kernel parameter space).
struct Grid {
    int n[3];         // nodes per dimension (with ghosts)
    int pitch;        // padded x extent
    long long nn;     // nodes per plane = n[Z]*n[Y]*pitch
    int lo[3], hi[3]; // PIN range [lo, hi)
    double dd[3];     // reciprocal mesh sizes
};

struct ModelParams {
    double gamma, gasR, cv, refMu, refT;
    double g[3];
    int sScheme, jacobMean, fluxSplit, multidim, sState, ibmLayer;
};

// Arguments of one LLLU stage.
struct StageArgs {
    const double *Uo;     // level to (read at the node itself)
    const double *Un;     // level tn (stencil level)
    double *Um;           // level tm (written; may alias Uo)
    const int *did;
    const double *dt;     // device scalar: step dt
    double dt_scale;      // this sweep uses dt_scale * (*dt) (0.5 for Strang halves)
    double coeA, coeB;
    int accumulate;       // operator-by-operator Y/Z: Um += coeB*r*Phi
    int to, tn, tm;       // level indices (the brick kernels address U through a tensor map)
    const CUtensorMap *maps;  // host array: TMA map of the whole state per (sweep axis, tile variant)
    const CUtensorMap *omaps; // host array: node-update box maps of the persistent FP32 kernel (or null)
    int var[3];               // tile variant of each sweep axis (brick_geometry.cuh)
    int *status;          // device error word of the case
    const uint8_t *flags; // hybrid form: sensor flags [3][node] (1 = full WENO5)
    long long wait_limit; // polls of a plane-march wait for a TMA plane or a free ring slot
};

// polls of a bounded device wait before it gives up (kernels then write their
// status word and leave; the wait for a block's own copies in flight before
// it ends always uses this default)
constexpr long long kWaitLimitDefault = 1LL << 22;

// one case of a batch (batch.cu), as the batched kernels see it
struct BatchCase {
    Grid g;
    ModelParams mp;
    double *U;              // the case's state (3 levels x 5 variables)
    const int *did;
    const uint8_t *flags;   // sensor flags [3][nn] or null
    int tiles[3][3];        // tile counts (x, y, z) of the stage kernel of each sweep axis
};

// RK coefficients and levels of one stage, common to all cases of a batch
struct StageCoefs {
    double coeA, coeB, dt_scale;
    int to, tn, tm;
};

int launch_stage_batch(const BatchCase *cases, const CUtensorMap *maps, const long long *prefix, int ncase,
                       const StageCoefs &sc, const double *dts, unsigned long long *counter, int *status, int blocks,
                       int s, bool hybrid, cudaStream_t st);

// state of one case of a batch, as the batched ghost fill and time step see it
struct BatchLevel {
    double *U;       // the case's state (3 levels x 5 variables x nn)
    long long nn;    // nodes per variable plane
};
// ghost fill of every case of a batch at level tn: pairs (case, dst, src, 0)
int launch_batch_gather(const BatchLevel *cases, const int4 *pairs, long long count, int tn, cudaStream_t st);
// time step of every case from its CFL maximum (ComputeTimeStep, solve.c:152):
// dt = cfl * min(d0/v0, min(d1/v1, d2/v2)) with vmax[c] the case's three maxima
// and d the mesh sizes (3 per case)
int launch_batch_dt(const double *const *vmax, const double *d, const double *cfl, double *dts, int ncase,
                    cudaStream_t st);

// Plane-march stage kernels (Y/Z sweeps): geometry of one launch, computed on
// the host and passed by value.  A block owns WX consecutive x by NR rows of
// the other transverse axis over one segment of the sweep axis; a producer
// warp streams halo'd planes of U[tn] into a ring of kPlaneSlots slots.
constexpr int kPlaneSlots = 6;
constexpr int kPlaneMaxThreads = 256;
constexpr int kPlaneSmemMax = 112 * 1024;  // two blocks per SM (228 KB, 1 KB reserved per block)
// hybrid form: per consumer warp, the WENO5 inputs of kCoopSlots flagged
// interfaces (2 sides x 5 fields x 5 points, FP32) shared out over the warp
constexpr int kCoopSlots = 6;
constexpr int kCoopBytes = kCoopSlots * 50 * 4;

// bytes of one ring slot: a TMA destination in shared memory starts on a
// 128-byte boundary, so the slot stride is rounded up to it
__host__ __device__ inline int plane_slot_bytes(int BXp, int BC)
{
    return (BXp * BC * 5 * 8 + 127) & ~127;
}

// shared memory of a plane-march block: the ring, the X sweep's double-
// buffered interface fluxes (nflux interfaces, five values of at most 8
// bytes), the hybrid form's per-warp WENO buffers of the ncw consumer warps
// and the full/empty barriers
__host__ __device__ inline int plane_flux_bytes(int nflux)
{
    return (2 * nflux * 5 * 8 + 127) & ~127;
}

__host__ __device__ inline int plane_smem_total(int BXp, int BC, int nflux, int ncw)
{
    return kPlaneSlots * plane_slot_bytes(BXp, BC) + plane_flux_bytes(nflux) + ncw * kCoopBytes +
           2 * kPlaneSlots * 8;
}

struct PlaneTile {
    int WX, NR;    // tile: nodes updated along x and rows of the row axis
    int TR;        // consumer threads per row (WX; WX + 1 interfaces on X sweeps)
    int ntx, ntc;  // tiles along x and along the rows
    int nseg;      // segments of each line (with shares: the chunks of the chunk-major plane order)
    int nblk;      // blocks of a launch: tiles x segments, or (share) equal shares of all tiles' planes
    int share;     // 1 = a block marches an equal share of the tiles' planes, chunk-major
    int BXp, BC;   // plane box: x extent (even, covers the x halo) and rows with halo
    int ncw;       // consumer warps (the producer is warp ncw)
    int swap;      // Y/Z kernel: 1 = a Z sweep run with axes 1 and 2 exchanged
    long long st, rs;  // Y/Z kernel: node strides along the line and along the rows
};

// Tile geometry of the plane march of sweep s.  Y and Z sweeps march along s
// with rows along the other transverse axis; X sweeps march along y with rows
// along z and an x halo of three nodes (the WENO5 stencil).  `waves` scales
// the number of blocks (segments of the march axis, each at least 8 planes).
inline PlaneTile plane_tile(const Grid &g, int s, bool visc, int waves, int sms, bool share = false)
{
    PlaneTile pt = {};
    const int T2 = (s == 1) ? 2 : (s == 2 ? 1 : 2);  // row axis
    const int M = (s == 0) ? 1 : s;                    // march axis
    const int Lx = g.hi[0] - g.lo[0], Lt = g.hi[T2] - g.lo[T2], Ls = g.hi[M] - g.lo[M];
    const int hv = visc ? 1 : 0;
    const int hx = (s == 0) ? 3 : hv;  // x halo
    pt.ntx = (Lx + 63) / 64;
    if (pt.ntx < 1) pt.ntx = 1;
    pt.WX = (Lx + pt.ntx - 1) / pt.ntx;
    if (pt.WX < 1) pt.WX = 1;
    pt.TR = (s == 0) ? pt.WX + 1 : pt.WX;
    pt.NR = (kPlaneMaxThreads - 32) / pt.TR;
    if (pt.NR > Lt) pt.NR = Lt;
    if (pt.NR < 1) pt.NR = 1;
    pt.BXp = (pt.WX + 2 * hx + 2) & ~1;
    // the ring of kPlaneSlots planes (and the X sweep's flux exchange) must fit
    while (pt.NR > 1 && plane_smem_total(pt.BXp, pt.NR + 2 * hv, s == 0 ? pt.TR * pt.NR : 0,
                                         (pt.TR * pt.NR + 31) / 32) > kPlaneSmemMax) {
        --pt.NR;
    }
    pt.ntc = (Lt + pt.NR - 1) / pt.NR;
    pt.ncw = (pt.TR * pt.NR + 31) / 32;
    pt.BC = pt.NR + 2 * hv;
    const long long tiles = (long long)pt.ntx * pt.ntc;
    const long long target = (long long)waves * 2 * sms;
    long long nseg = (target + tiles - 1) / tiles;
    const int cap = Ls / 8 > 1 ? Ls / 8 : 1;
    if (nseg > cap) nseg = cap;
    if (nseg < 1) nseg = 1;
    pt.nseg = (int)nseg;
    pt.share = share ? 1 : 0;
    if (!pt.share) {
        pt.nblk = (int)(tiles * nseg);
    } else {
        // every block the same number of planes (at least 8): no partial
        // last wave, one fill of the ring per item; the lines are cut into
        // about one chunk per block of a tile (the chunk-major order of the
        // shares)
        long long nb = std::min<long long>(target, tiles * Ls / 8);
        pt.nblk = (int)std::max<long long>(1, nb);
        long long nch = (pt.nblk + tiles / 2) / tiles;
        if (nch > cap) nch = cap;
        if (nch < 1) nch = 1;
        pt.nseg = (int)nch;
    }
    return pt;
}

inline int plane_smem_bytes(const PlaneTile &pt, int s)
{
    return plane_smem_total(pt.BXp, pt.BC, s == 0 ? pt.TR * pt.NR : 0, pt.ncw);
}

// plane-march geometry of one case and sweep axis of a batch: the kernel's
// grid descriptor (axes 1 and 2 exchanged for a Z sweep) and the plane tile
struct BatchPlane {
    Grid gk;
    PlaneTile pt;
};
// plane-march stage of a batch: block b of the launch runs block
// b - prefix[c] of case c (prefix[c] <= b < prefix[c+1]) with the case's plane
// map pmaps[3c+s]; nthreads and smem are the largest over the cases
int launch_stage_plane_batch(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                             const long long *prefix, long long blocks, int ncase, const StageCoefs &sc,
                             const double *dts, int *status, int s, bool viscous, bool hybrid, int nthreads, int smem,
                             cudaStream_t st);

// Persistent batch step: the RK stages of one directional half step of every
// case in one launch (six launches per time step, one per sweep of the
// Strang schedule, so that a kernel holds the block body of one sweep axis
// only).  Work items, in order: for each stage k of the launch, the plane
// blocks of every case (case order) and then the ghost-fill items of every
// case (its copy pairs in chunks of kFillChunk).  A plane block of stage
// k > 0 of case c waits until every fill item of stage k-1 of case c is
// done; a fill item of stage k of case c waits until all plane blocks of
// stage k of case c are done (per-case counters, no grid-wide barrier).
// Items are taken from a queue in order, so every item a block waits for was
// taken earlier by a running block.
constexpr int kMaxStepStages = 18;
constexpr long long kFillChunk = 16384;  // copy pairs of one ghost-fill item
struct PersistStep {
    int nk;                               // stages of this launch
    int k0;                               // step-wide index of its first stage (counters are per step)
    int s_of[kMaxStepStages];             // sweep axis of stage k
    StageCoefs sc[kMaxStepStages];
    long long kbase[kMaxStepStages + 1];  // first item of stage k
    long long ntile[3];                   // plane blocks of one stage along axis s, all cases
    long long nfill;                      // ghost-fill items of one stage, all cases
};
// queue: one counter; done, filled: [nk][ncase] (zero at launch); abort: one
// word set by a block whose wait gave up (status code 7), after which every
// block leaves; pairs: (case, dst, src) copy pairs of the ghost fill, case
// by case, pair_off[c] .. pair_off[c + 1] those of case c; fill_pre[c]: the
// first fill item of case c within a stage (fill_pre[ncase] = ps.nfill)
int launch_stage_plane_persistent(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                  const long long *prefix, int ncase, const PersistStep &ps, const double *dts,
                                  const BatchLevel *levels, const int4 *pairs, const long long *pair_off,
                                  const long long *fill_pre, unsigned long long *queue, unsigned *done,
                                  unsigned *filled, int *abort, int *status, bool viscous, bool hybrid, int blocks,
                                  int nthreads, int smem, cudaStream_t st);
// resident blocks per SM of the persistent batch kernel
int plane_persistent_occupancy(bool viscous, bool hybrid, int nthreads, int smem, int *blocks_per_sm);

// learned sensor (sensor.cu)
// Flags of the PIN nodes (the caller sets the others to 1 once); rho_p:
// scratch of nn float2 (density and pressure of every node)
int launch_sensor_flags(const Grid &g, const ModelParams &m, const double *U, const int *did, const float *params,
                        float logit_threshold, float2 *rho_p, uint8_t *flags, unsigned long long *count,
                        cudaStream_t st);
int launch_sensor_features(const Grid &g, const ModelParams &m, const double *U, const int *did, int s, float *feat,
                           float *dep, cudaStream_t st);
int sensor_param_count();

// ---------------------------------------------------------------------------
// error state (per host thread)
// ---------------------------------------------------------------------------
void set_error(const char *fmt, ...);
int cuda_status(cudaError_t e, const char *what);

#define ACFD_CUDA(call)                                           \
    do {                                                          \
        cudaError_t e__ = (call);                                 \
        if (e__ != cudaSuccess) return acfd::cuda_status(e__, #call); \
    } while (0)

// ---------------------------------------------------------------------------
// kernel launchers (one translation unit per arithmetic form)
// ---------------------------------------------------------------------------
// FP64, reference operation order, compiled with --fmad=false
int launch_stage_exact(const Grid &g, const ModelParams &m, const StageArgs &a, int s,
                       bool viscous, cudaStream_t st);
// FP64, reassociated with FMA
int launch_stage_fast(const Grid &g, const ModelParams &m, const StageArgs &a, int s,
                      bool viscous, cudaStream_t st);
// FP32 stencil arithmetic with FP64 accumulation
int launch_stage_fp32(const Grid &g, const ModelParams &m, const StageArgs &a, int s,
                      bool viscous, cudaStream_t st);
// gravity source stage
int launch_stage_phi(const Grid &g, const ModelParams &m, const StageArgs &a, cudaStream_t st);

// per-point twins
int launch_weno_batch(int scheme, int mode, const double *F, double *Fhat, int count,
                      cudaStream_t st);
int launch_fhat_batch(const ModelParams &m, int s, int mode, const double *U, double *F,
                      int count, cudaStream_t st);

// domain ghost fill: one launch per group of independent face boxes
struct FaceBox {
    int box[3][2];
    int face;  // 1..6
    int r;     // layer
};
int launch_domain_boundary(const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                           const FaceBox *boxes, int nbox, double *U, cudaStream_t st);
// ghost fill as one gather: U[dst] = U[src] for every (dst, src) pair, all
// five variables of the level U
int launch_ghost_gather(const Grid &g, const int2 *pairs, int count, double *U, cudaStream_t st);
// one level of the state (five variables, the x and y momenta exchanged),
// an int array or a byte array transposed from grid gs to grid gd, whose axes
// 0 and 1 are those of gs exchanged (every node, ghosts included)
int launch_transpose_state(const double *src, const Grid &gs, double *dst, const Grid &gd, cudaStream_t st);
int launch_transpose_int(const int *src, const Grid &gs, int *dst, const Grid &gd, cudaStream_t st);
int launch_transpose_u8(const uint8_t *src, const Grid &gs, uint8_t *dst, const Grid &gd, cudaStream_t st);
// debug mode: add the count of non-finite values among U[0, count) to *word
int launch_finite_scan(const double *U, long long count, int *word, cudaStream_t st);
// ghost fill as one launch of formulas: per-face constants of the programs
// (type, outward normal, given primitive state of faces 1..6), op codes
// (low 3 bits; the face in the bits above), the value-stack depth
struct GhostFaces {
    int type[7];
    int N[7][3];
    double given[7][6];
};
constexpr int kGhostLoad = 0;    // push U[arg]
constexpr int kGhostInflow = 1;  // push the given inflow state of the face
constexpr int kGhostWall = 2;    // top := wall boundary node from the top (its inner neighbour)
constexpr int kGhostImage = 3;   // (O, I) := image ghost of boundary point O and image node I
constexpr int kGhostStack = 6;
constexpr int kGhostMaxOps = 32;
// tasks: runs of copies, a block each -- (first destination, source offset,
// length <= 2048, 0); single: the other copies (dst, src); progs: (dst,
// first op, op count, 0); ops: (code | face << 3, node)
int launch_ghost_program(const Grid &g, const ModelParams &m, const GhostFaces &F, const int4 *tasks, int ntask,
                         const int2 *single, int nsingle, const int4 *progs, int nprog, const int2 *ops, double *U,
                         cudaStream_t st);
// all groups of one TreatBoundary in one cooperative launch with grid barriers;
// bar: two device words (arrival count, generation), zero at first use
int launch_domain_boundary_fused(const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                                 const FaceBox *const *groups, const int *sizes, int ngroups, double *U,
                                 unsigned *bar, int *status, cudaStream_t st);

// CFL wave-speed maximum, one launch: partials (kCflPartials doubles: four
// per block, then a completion counter that must be zero when the buffer is
// allocated) and out[4]: the three maxima and the count of blocks that met a
// non-finite wave speed
constexpr int kCflBlocks = 1184;  // 148 SMs x 8 blocks of 256 threads: enough warps to hide the loads
constexpr int kCflPartials = 4 * kCflBlocks + 1;
int launch_cfl(const Grid &g, const ModelParams &m, const double *U, const int *did,
               double *partials, double *out, cudaStream_t st);

// layout conversion between the reference node records and the device planes
int launch_scatter_nodes(const Grid &g, const acfd_node_t *staged, double *U, int *flags,
                         unsigned mask, cudaStream_t st);
int launch_gather_nodes(const Grid &g, const double *U, const int *flags, acfd_node_t *staged,
                        unsigned mask, cudaStream_t st);

}  // namespace acfd

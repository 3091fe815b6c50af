// C ABI of libacfd_gpu (include/acfd.h): case life cycle, host <-> device
// coherence, and the schedule of one fluid time step
// (EvolveFluidDynamics -> DiscretizeTime -> RungeKutta2/3 -> LLLU +
// TreatBoundary, fluid_dynamics.c:55-148, boundary_treatment.c:28-65).
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>

#include <unistd.h>
#include <unordered_map>
#include <vector>

#include <cudaTypedefs.h>

#include "acfd_internal.cuh"
#include "ghost_tasks.h"
#include "brick_geometry.cuh"

namespace acfd {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char *what)
{
    set_error("%s: %s (%s)", what, cudaGetErrorString(e), cudaGetErrorName(e));
    // a failed call that leaves the context usable (an allocation that did
    // not fit, an invalid argument) also sets the runtime's last error: clear
    // it, or the next launch check of this thread would report it again
    (void)cudaGetLastError();
    return (e == cudaErrorMemoryAllocation) ? ACFD_ERR_NOMEM : ACFD_ERR_CUDA;
}

int launch_stage_exact(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_fast(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_fp32(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_brick_fast(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_brick_fp32(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_brick_hybrid(const Grid &, const ModelParams &, const StageArgs &, int, bool, cudaStream_t);
int launch_stage_march_fast(const Grid &, const ModelParams &, const StageArgs &, int, bool, int, cudaStream_t);
int launch_stage_march_fp32(const Grid &, const ModelParams &, const StageArgs &, int, bool, bool, int,
                            cudaStream_t);
int launch_stage_plane_fast(const Grid &, const ModelParams &, const StageArgs &, int, bool, const PlaneTile &,
                            const CUtensorMap &, cudaStream_t);
int launch_stage_plane_fp32(const Grid &, const ModelParams &, const StageArgs &, int, bool, bool,
                            const PlaneTile &, const CUtensorMap &, cudaStream_t);
int launch_weno_batch_exact(int, const double *, double *, int, cudaStream_t);
int launch_weno_batch_fast(int, const double *, double *, int, cudaStream_t);
int launch_weno_batch_fp32(int, const double *, double *, int, cudaStream_t);
int launch_fhat_batch_exact(const ModelParams &, int, const double *, double *, int, cudaStream_t);
int launch_fhat_batch_fast(const ModelParams &, int, const double *, double *, int, cudaStream_t);
int launch_fhat_batch_fp32(const ModelParams &, int, const double *, double *, int, cudaStream_t);

// IB (ib.cu)
struct IbState;
int ib_create(IbState **out);
void ib_destroy(IbState *ib);
int ib_upload(IbState *ib, const acfd_polyhedron_t *poly, int totN, const acfd_partition_t &part,
              cudaStream_t st, bool *relayout);
int ib_treat_launches(const IbState *ib, const acfd_partition_t &part);
int ib_flags_changed(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                     const int *flags, cudaStream_t st);
int ib_surface_force(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                     const double *U, const int *flags, double *force, cudaStream_t st);
int ib_collision_scan(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                      const int *flags, int *counts, int *gid, int *N, cudaStream_t st);
int ib_count(const IbState *ib);
int ib_compute_geometric_field(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                               double *U, int *flags, cudaStream_t st);
int ib_treat(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part, double *U,
             int *flags, int tn, cudaStream_t st);
int ib_check(IbState *ib, cudaStream_t st);
int ib_transform(IbState *ib, int n, const double O[3], const double scale[3], const double angle[3],
                 const double offset[3], double centroid[3], double inertia[9], double box[6], cudaStream_t st);
int ib_fetch(IbState *ib, int n, double *v, double *Nf, double *Ne, double *Nv, cudaStream_t st);

bool pdl_enabled()
{
    static const bool on = [] {
        const char *e = getenv("ACFD_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}

// Stage-kernel variants: the brick tile shapes (0 .. kTileVariants-1), the
// line-march kernels and the plane-march kernels, each launched with 1, 2 or
// 4 waves; the plane march twice: lines cut into equal segments per tile,
// then equal shares of all tiles' planes per block
constexpr int kMarchVariants = 3;
constexpr int kMarchWaves[kMarchVariants] = {1, 2, 4};
constexpr int kPlaneVariants = 6;
constexpr int kPlaneWaves[kPlaneVariants] = {1, 2, 4, 1, 2, 4};
constexpr bool kPlaneShare[kPlaneVariants] = {false, false, false, true, true, true};
constexpr int kPlaneFirst = kTileVariants + kMarchVariants;
constexpr int kStageVariants = kPlaneFirst + kPlaneVariants;
static_assert(ACFD_BRICK_VARIANTS == kTileVariants && ACFD_STAGE_VARIANTS == kStageVariants &&
                  ACFD_PLANE_VARIANT == kPlaneFirst,
              "stage-variant numbering of the C ABI");

__global__ void set_scalar(double *p, double v)
{
    pdl_wait();
    *p = v;
}

}  // namespace acfd

using namespace acfd;

// one piece of a profiled step (acfd_profile_step)
struct StepPiece {
    int kind, axis, stage;
    cudaEvent_t e0, e1;
};

struct acfd_case {
    acfd_partition_t part;
    acfd_model_t model;
    Grid grid;
    ModelParams mp;
    int device = 0;
    int mode = ACFD_FP64;
    double *U = nullptr;       // [3][5][nn]
    int *flags = nullptr;      // [4][nn]
    double *d_dt = nullptr;    // device scalar dt of the current step
    double *cfl_part = nullptr;
    double *cfl_out = nullptr;
    double *h_cfl = nullptr;   // pinned
    acfd_node_t *staging = nullptr;
    // asynchronous snapshot of the node records (output and checkpoints)
    acfd_node_t *snap_dev = nullptr;   // device copy in the node layout
    acfd_node_t *snap_host = nullptr;  // pinned host copy
    cudaStream_t snap_stream = nullptr;
    cudaEvent_t snap_gathered = nullptr, snap_copied = nullptr;
    bool snap_pending = false;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<std::vector<FaceBox>> bc_groups;  // ordered, each group independent inside
    IbState *ib = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    int graph_mode = -1;
    long long launches = 0;        // kernels launched by this case (graph replays included)
    long long graph_kernels = 0;   // kernels in the captured step graph
    int *dstatus = nullptr;        // device error word (TMA wait time-outs)
    CUtensorMap maps[3 * kTileVariants];  // state tensor maps of the brick kernels per (axis, tile variant)
    bool maps_ok = false;
    // stage-kernel variant of each sweep axis per arithmetic form (acfd_autotune,
    // acfd_set_tiles): brick tile shapes, then line-march launch sizes
    int tile_var[4][3] = {{0, 0, 0},
                          {0, 0, 0},
                          {0, kPlaneFirst + 2, kPlaneFirst + 2},
                          {0, kPlaneFirst + 2, kPlaneFirst + 2}};
    int sms = 148;                 // SM count of the case's device
    CUtensorMap pmaps[3];          // plane-march state maps per sweep axis
    int pbox[3][2] = {{0, 0}, {0, 0}, {0, 0}};  // their box: x extent and rows
    bool pmaps_ok = false;
    bool plain_kernels = false;    // use the global-memory stage kernels instead of the bricks
    bool bc_multi = false;         // one launch per ghost-fill phase instead of the fused launch
    unsigned *bcbar = nullptr;     // grid-barrier words of the fused ghost fill
    int2 *bc_pairs = nullptr;      // ghost fill as one launch: copies (dst, src) -- base of the allocation
    int bc_npairs = 0;
    int4 *bc_progs = nullptr;      // ... and formula programs (dst, first op, op count)
    int bc_nprog = 0;
    int4 *bc_tasks = nullptr;      // the copies in runs (launch_ghost_program) ...
    int bc_ntask = 0;
    int2 *bc_single = nullptr;     // ... and the others
    int bc_nsingle = 0;
    int2 *bc_ops = nullptr;
    GhostFaces bc_faces;
    bool bc_gather = false;        // the one-launch fill replaces the ordered launches
    std::vector<int2> bc_copies;   // host copy of the copies of a copy-only fill
    // The X half steps as Y sweeps of the transposed state (build_xt): xg is
    // the grid with axes 0 and 1 exchanged, xU its three levels, xdid the
    // node types on it, xfl the sensor's x flags as the flags of its axis 1
    // ([2][xg.nn], slot 1), xmap the plane map of its Y sweep (box xbox), and
    // the copy-only fill remapped to it (x_tasks, x_single).
    bool xt_ok = false;
    bool xt_all_forms = false;     // the transposed X sweep for the fast FP64 form too
    Grid xg = {};
    double *xU = nullptr;
    int *xdid = nullptr;
    uint8_t *xfl = nullptr;
    CUtensorMap xmap;
    int xbox[2] = {0, 0};
    int4 *x_tasks = nullptr;
    int x_ntask = 0;
    int2 *x_single = nullptr;
    int x_nsingle = 0;
    long long wait_limit = kWaitLimitDefault;  // polls of a plane-march wait (acfd_set_wait_limit)
    std::vector<StepPiece> *prof = nullptr;     // pieces of a step being profiled (acfd_profile_step)
    // ACFD_DEBUG=1: every stage and ghost fill is followed by a scan of its
    // level for non-finite values, checked at once (no step graphs)
    bool debug = false;
    int *dbg_word = nullptr;
    std::vector<const FaceBox *> bc_ptrs;
    std::vector<int> bc_sizes;
    // learned sensor of the hybrid form
    float *sensor_params = nullptr;          // device, acfd_mlp_param_count() floats
    uint8_t *sensor_flags = nullptr;         // device, [3][nn]
    float2 *sensor_rp = nullptr;             // device, [nn] (rho, p) scratch of the flag pass
    unsigned long long *sensor_count = nullptr;
    float sensor_logit = 0.0f;               // flag where the logit exceeds this
    bool sensor_ok = false;
};

namespace {

bool viscous(const acfd_case *cs)
{
    return cs->model.refMu > 0.0;
}

// 5-D tensor map of the whole state U[level][var][z][y][x] with the brick of
// sweep axis s as its box (cuTensorMapEncodeTiled through the runtime's driver
// entry point, so the library needs no -lcuda)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
            set_error("cuTensorMapEncodeTiled not available from the driver");
            return nullptr;
        }
        encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }
    return encode;
}

// map of the whole state of a case with the given box (x, y, z), five
// variables, one level
int encode_box_map(const Grid &g, double *U, const int b[3], CUtensorMap *out)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) {
        return ACFD_ERR_CUDA;
    }
    const cuuint64_t dims[5] = {(cuuint64_t)g.pitch, (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 5, 3};
    const cuuint64_t strides[4] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.pitch * g.n[1] * 8,
                                   (cuuint64_t)g.nn * 8, (cuuint64_t)g.nn * 5 * 8};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const cuuint32_t box[5] = {(cuuint32_t)b[0], (cuuint32_t)b[1], (cuuint32_t)b[2], 5, 1};
    CUresult r = encode(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, U, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d) for box %d x %d x %d", (int)r, b[0], b[1], b[2]);
        return ACFD_ERR_CUDA;
    }
    return ACFD_OK;
}

int encode_state_maps(acfd_case *cs)
{
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) {
        return ACFD_ERR_CUDA;
    }
    const Grid &g = cs->grid;
    const cuuint64_t dims[5] = {(cuuint64_t)g.pitch, (cuuint64_t)g.n[1], (cuuint64_t)g.n[2], 5, 3};
    const cuuint64_t strides[4] = {(cuuint64_t)g.pitch * 8, (cuuint64_t)g.pitch * g.n[1] * 8,
                                   (cuuint64_t)g.nn * 8, (cuuint64_t)g.nn * 5 * 8};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    for (int s = 0; s < 3; ++s) {
        for (int var = 0; var < kTileVariants; ++var) {
            int b[3];
            brick_box(s, viscous(cs), var, b);
            const cuuint32_t box[5] = {(cuuint32_t)b[0], (cuuint32_t)b[1], (cuuint32_t)b[2], 5, 1};
            CUresult r = encode(&cs->maps[s * kTileVariants + var], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, cs->U, dims,
                                strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
            if (r != CUDA_SUCCESS) {
                set_error("cuTensorMapEncodeTiled failed (%d) for sweep axis %d, tile variant %d", (int)r, s, var);
                return ACFD_ERR_CUDA;
            }
        }
    }
    cs->maps_ok = true;
    // plane-march maps: one plane of the tile with its halo, five variables
    for (int s = 0; s < 3; ++s) {
        const PlaneTile pt = plane_tile(g, s, viscous(cs), 1, cs->sms);
        // X and Y sweeps load a y-plane (rows along z), Z sweeps a z-plane
        // (rows along y)
        const cuuint32_t box[5] = {(cuuint32_t)pt.BXp, (cuuint32_t)(s == 2 ? pt.BC : 1),
                                   (cuuint32_t)(s == 2 ? 1 : pt.BC), 5, 1};
        cs->pbox[s][0] = pt.BXp;
        cs->pbox[s][1] = pt.BC;
        if (pt.BXp > 256 || pt.BC > 256) {
            return ACFD_OK;  // no plane maps for this grid
        }
        CUresult r = encode(&cs->pmaps[s], CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, cs->U, dims, strides, box, estr,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) {
            set_error("cuTensorMapEncodeTiled failed (%d) for the plane map of axis %d", (int)r, s);
            return ACFD_ERR_CUDA;
        }
    }
    cs->pmaps_ok = true;
    return ACFD_OK;
}

// read and clear the device error word
int check_device_status(acfd_case *cs)
{
    int h = 0;
    ACFD_CUDA(cudaMemcpyAsync(&h, cs->dstatus, sizeof(int), cudaMemcpyDeviceToHost, cs->stream));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    if (h != 0) {
        cudaMemsetAsync(cs->dstatus, 0, sizeof(int), cs->stream);
        set_error("stage kernel reported device error %d (TMA load not completed within its wait limit)", h);
        return ACFD_ERR_DEVICE;
    }
    return ACFD_OK;
}

double *level(acfd_case *cs, int l)
{
    return cs->U + (long long)l * kVars * cs->grid.nn;
}

// ordered ghost-fill plan: layer r = 0..max(ng), faces W,E,S,N,F,B; the two
// faces normal to one axis never read each other's box, so they form one
// launch (boundary_treatment.c:51-63)
void build_bc_plan(acfd_case *cs)
{
    const acfd_partition_t &p = cs->part;
    const int R = std::max(p.ng[0], std::max(p.ng[1], p.ng[2]));
    cs->bc_groups.clear();
    for (int r = 0; r <= R; ++r) {
        for (int axis = 0; axis < 3; ++axis) {
            std::vector<FaceBox> group;
            for (int side = 0; side < 2; ++side) {
                const int face = 1 + 2 * axis + side;
                FaceBox b;
                b.face = face;
                b.r = r;
                bool empty = false;
                for (int s = 0; s < 3; ++s) {
                    const int N = p.N[face][s];
                    const int w = std::min(r, p.ng[s]);
                    b.box[s][0] = p.ns[face][s][0] + w * (N - !N);
                    b.box[s][1] = p.ns[face][s][1] + w * (N + !N) - (p.ng[s] < r) * (!!N);
                    if (b.box[s][0] >= b.box[s][1]) {
                        empty = true;
                    }
                }
                // periodic boundary planes (r == 0) need no treatment
                if (!empty && !(r == 0 && p.typeBC[face] == 4)) {
                    group.push_back(b);
                }
            }
            if (!group.empty()) {
                cs->bc_groups.push_back(group);
            }
        }
    }
    cs->bc_ptrs.clear();
    cs->bc_sizes.clear();
    for (const auto &grp : cs->bc_groups) {
        cs->bc_ptrs.push_back(grp.data());
        cs->bc_sizes.push_back((int)grp.size());
    }
}

// Ghost fill as one launch.  The reference fills the faces in order, layer
// by layer (boundary_treatment.c:51-63), and every write is one of: a copy of
// another node (outflow, periodic, the outer layers of inflow), the given
// inflow state (inflow boundary node), the wall formula of a boundary node
// from its inner neighbour (slip / no-slip wall, :148-177) or the method of
// images of a wall ghost node from its boundary point and image node
// (:105-115).  Replaying the ordered fill on formulas instead of values gives,
// for every node the fill changes, one formula over values from before the
// fill (a write that reads a node changed earlier in the fill takes that
// node's formula).  When no node that a final formula reads is itself changed
// by the fill, one launch evaluating every formula reproduces the ordered
// fill bit for bit: the operations and their order are the reference's.  Pure
// copies are kept as (destination, source) pairs, the other formulas as short
// postfix programs.  Returns false (keep the ordered launches) when a formula
// reads a changed node, a program is longer than kGhostMaxOps, or the node
// count does not fit 32-bit indices.
namespace {

struct GhostExpr {
    int op, a, b, face;  // a, b: references (>= 0 expression, < 0 LOAD of node -ref-1)
    bool operator==(const GhostExpr &o) const { return op == o.op && a == o.a && b == o.b && face == o.face; }
};
struct GhostExprHash {
    size_t operator()(const GhostExpr &e) const
    {
        unsigned long long h = (unsigned long long)(unsigned)e.a * 0x9E3779B97F4A7C15ULL;
        h ^= ((unsigned long long)(unsigned)e.b + 0x632BE59BD9B4E019ULL) * 0xC2B2AE3D27D4EB4FULL;
        h ^= (unsigned long long)(e.op * 8 + e.face) * 0x165667B19E3779F9ULL;
        return (size_t)(h ^ (h >> 29));
    }
};

}  // namespace

bool build_bc_program(acfd_case *cs)
{
    const acfd_partition_t &p = cs->part;
    const Grid &g = cs->grid;
    if (g.nn * 5 > (long long)INT32_MAX) {
        return false;
    }
    const int kUnset = INT32_MIN;
    std::vector<int> def((size_t)g.nn, kUnset);
    std::vector<GhostExpr> ex;
    std::unordered_map<GhostExpr, int, GhostExprHash> memo;
    auto make = [&](const GhostExpr &e) {
        auto it = memo.find(e);
        if (it != memo.end()) {
            return it->second;
        }
        const int id = (int)ex.size();
        ex.push_back(e);
        memo.emplace(e, id);
        return id;
    };
    auto ref_of = [&](long long q) { return def[(size_t)q] != kUnset ? def[(size_t)q] : -(int)q - 1; };
    auto idx = [&](int i, int j, int k) { return ((long long)k * g.n[1] + j) * g.pitch + i; };
    auto inside = [&](int i, int j, int k) {
        return i >= 0 && j >= 0 && k >= 0 && i < g.n[0] && j < g.n[1] && k < g.n[2];
    };
    for (const auto &grp : cs->bc_groups) {
        for (const FaceBox &b : grp) {
            const int face = b.face, r = b.r, type = p.typeBC[face];
            const int *N = p.N[face];
            for (int k = b.box[2][0]; k < b.box[2][1]; ++k) {
                for (int j = b.box[1][0]; j < b.box[1][1]; ++j) {
                    for (int i = b.box[0][0]; i < b.box[0][1]; ++i) {
                        const long long q = idx(i, j, k);
                        int e;
                        if (r != 0) {
                            if (type == 2 || type == 3) {
                                const int oi = i - r * N[0], oj = j - r * N[1], ok = k - r * N[2];
                                const int ii = i - 2 * r * N[0], ij = j - 2 * r * N[1], ik = k - 2 * r * N[2];
                                if (!inside(oi, oj, ok) || !inside(ii, ij, ik)) return false;
                                e = make(GhostExpr{kGhostImage, ref_of(idx(oi, oj, ok)), ref_of(idx(ii, ij, ik)), 0});
                            } else {
                                const int per = (type == 4);
                                const int si = i - (per ? p.m[0] * N[0] : N[0]);
                                const int sj = j - (per ? p.m[1] * N[1] : N[1]);
                                const int sk = k - (per ? p.m[2] * N[2] : N[2]);
                                if (!inside(si, sj, sk)) return false;
                                e = ref_of(idx(si, sj, sk));
                            }
                        } else if (type == 0) {
                            e = make(GhostExpr{kGhostInflow, 0, 0, face});
                        } else if (type == 1 || type == 2 || type == 3) {
                            const int si = i - N[0], sj = j - N[1], sk = k - N[2];
                            if (!inside(si, sj, sk)) return false;
                            e = ref_of(idx(si, sj, sk));
                            if (type != 1) {
                                e = make(GhostExpr{kGhostWall, e, 0, face});
                            }
                        } else {
                            continue;  // periodic boundary plane: computed like an interior node
                        }
                        def[(size_t)q] = e;
                    }
                }
            }
        }
    }
    // final formulas: copies and programs; no node a formula reads may change
    std::vector<int2> pairs;
    std::vector<int4> progs;
    std::vector<int2> ops;
    std::vector<char> changed((size_t)g.nn, 0);
    for (long long q = 0; q < g.nn; ++q) {
        const int d = def[(size_t)q];
        if (d != kUnset && d != -(int)q - 1) {
            changed[(size_t)q] = 1;
        }
    }
    std::vector<int> first((size_t)ex.size(), -1), count((size_t)ex.size(), 0), depth((size_t)ex.size(), 0);
    bool ok = true;
    // postfix flattening of expression e into ops (memoized: a shared
    // sub-formula is copied, not referenced)
    std::vector<int2> tmp;
    auto emit = [&](auto &&self, int ref, std::vector<int2> &out, int &dep) -> void {
        if (!ok) return;
        if (ref < 0) {
            const int node = -ref - 1;
            if (changed[(size_t)node]) ok = false;
            out.push_back(make_int2(kGhostLoad, node));
            dep = 1;
            return;
        }
        const GhostExpr &e = ex[(size_t)ref];
        if (e.op == kGhostInflow) {
            out.push_back(make_int2(kGhostInflow | (e.face << 3), 0));
            dep = 1;
        } else if (e.op == kGhostWall) {
            int d0 = 0;
            self(self, e.a, out, d0);
            out.push_back(make_int2(kGhostWall | (e.face << 3), 0));
            dep = d0;
        } else {
            int d0 = 0, d1 = 0;
            self(self, e.a, out, d0);
            self(self, e.b, out, d1);
            out.push_back(make_int2(kGhostImage, 0));
            dep = std::max(d0, d1 + 1);
        }
    };
    for (long long q = 0; q < g.nn && ok; ++q) {
        if (!changed[(size_t)q]) continue;
        const int d = def[(size_t)q];
        if (d < 0) {
            const int src = -d - 1;
            if (changed[(size_t)src]) ok = false;
            pairs.push_back(make_int2((int)q, src));
            continue;
        }
        if (first[(size_t)d] < 0) {
            tmp.clear();
            int dep = 0;
            emit(emit, d, tmp, dep);
            if ((int)tmp.size() > kGhostMaxOps || dep > kGhostStack) ok = false;
            first[(size_t)d] = (int)ops.size();
            count[(size_t)d] = (int)tmp.size();
            ops.insert(ops.end(), tmp.begin(), tmp.end());
        }
        progs.push_back(make_int4((int)q, first[(size_t)d], count[(size_t)d], 0));
    }
    if (!ok || (pairs.empty() && progs.empty())) {
        return false;
    }
    for (int f = 0; f < 7; ++f) {
        cs->bc_faces.type[f] = p.typeBC[f];
        for (int s = 0; s < 3; ++s) cs->bc_faces.N[f][s] = p.N[f][s];
        for (int v = 0; v < 6; ++v) cs->bc_faces.given[f][v] = p.varBC[f][v];
    }
    // the copies as tasks (runs, a block each, no index loads) and single
    // copies (ghost_tasks.h)
    std::vector<int4> tasks;
    std::vector<int2> single;
    ghost_copy_tasks(pairs, tasks, single);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t b_pairs = pairs.size() * sizeof(int2), b_progs = progs.size() * sizeof(int4);
    const size_t b_ops = ops.size() * sizeof(int2), b_tasks = tasks.size() * sizeof(int4);
    const size_t off_progs = al(b_pairs), off_ops = off_progs + al(b_progs), off_tasks = off_ops + al(b_ops);
    const size_t off_single = off_tasks + al(b_tasks);
    const size_t total = off_single + single.size() * sizeof(int2);
    char *base = nullptr;
    if (cudaMalloc(&base, total) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    bool copied = cudaMemcpy(base, pairs.data(), b_pairs, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(base + off_progs, progs.data(), b_progs, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(base + off_ops, ops.data(), b_ops, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(base + off_tasks, tasks.data(), b_tasks, cudaMemcpyHostToDevice) == cudaSuccess &&
                  cudaMemcpy(base + off_single, single.data(), single.size() * sizeof(int2),
                             cudaMemcpyHostToDevice) == cudaSuccess;
    if (!copied) {
        cudaGetLastError();
        cudaFree(base);
        return false;
    }
    cs->bc_pairs = reinterpret_cast<int2 *>(base);
    cs->bc_npairs = (int)pairs.size();
    cs->bc_progs = reinterpret_cast<int4 *>(base + off_progs);
    cs->bc_nprog = (int)progs.size();
    cs->bc_ops = reinterpret_cast<int2 *>(base + off_ops);
    cs->bc_tasks = reinterpret_cast<int4 *>(base + off_tasks);
    cs->bc_ntask = (int)tasks.size();
    if (progs.empty()) {
        cs->bc_copies = pairs;
    }
    cs->bc_single = reinterpret_cast<int2 *>(base + off_single);
    cs->bc_nsingle = (int)single.size();
    return true;
}

// The X half steps of a step run as Y sweeps of the transposed state: the
// plane march along y reaches a higher rate than the X sweep's (a stencil
// window in registers instead of a stencil gathered from the plane, no
// barrier per row), so U[TO] is transposed (x and y exchanged, with the x and
// y momenta) before the first X half step of a run of them and back after the
// last; the stages between run on the transposed levels with the copy-only
// fill remapped to the transposed node indices.  Only for a fill of copies
// (whose transpose is the fill of the transposed grid); ACFD_X_TRANSPOSE=0
// keeps the X sweep, ACFD_X_TRANSPOSE=all offers the path to the fast FP64
// form too.
void build_xt(acfd_case *cs);

// the transposed levels and their fill freed; the X half steps stay on the
// X sweep
void release_xt(acfd_case *cs)
{
    cudaFree(cs->xU);
    cudaFree(cs->xdid);
    cudaFree(cs->xfl);
    cudaFree(cs->x_tasks);
    cs->xU = nullptr;
    cs->xdid = nullptr;
    cs->xfl = nullptr;
    cs->x_tasks = nullptr;
    cs->x_single = nullptr;
    cs->x_ntask = cs->x_nsingle = 0;
    cs->xt_ok = false;
}

void build_xt(acfd_case *cs)
{
    const char *env = getenv("ACFD_X_TRANSPOSE");
    cs->xt_all_forms = env && strcmp(env, "all") == 0;
    if ((env && env[0] == '0') || !cs->bc_gather || cs->bc_nprog != 0 || cs->bc_copies.empty() || !cs->pmaps_ok ||
        cs->model.multidim != 0) {
        return;
    }
    const Grid &g = cs->grid;
    Grid xg = g;
    xg.n[0] = g.n[1];
    xg.n[1] = g.n[0];
    xg.lo[0] = g.lo[1];
    xg.lo[1] = g.lo[0];
    xg.hi[0] = g.hi[1];
    xg.hi[1] = g.hi[0];
    xg.dd[0] = g.dd[1];
    xg.dd[1] = g.dd[0];
    xg.pitch = (xg.n[0] + 7) & ~7;
    xg.nn = (long long)xg.pitch * xg.n[1] * xg.n[2];
    if (xg.nn * 5 > (long long)INT32_MAX || (long long)g.n[2] * 5 > 65535) return;
    const PlaneTile pt = plane_tile(xg, 1, viscous(cs), 1, cs->sms);
    if (pt.BXp > 256 || pt.BC > 256) return;
    // the copies on the transposed node indices, in destination order
    const std::vector<int2> xc = transposed_copies_of(cs->bc_copies, g.pitch, g.n[0], g.n[1], xg.pitch);
    std::vector<int4> tasks;
    std::vector<int2> single;
    ghost_copy_tasks(xc, tasks, single);
    const size_t b_tasks = (tasks.size() * sizeof(int4) + 255) / 256 * 256;
    char *prog = nullptr;
    if (cudaMalloc(&cs->xU, sizeof(double) * kLevels * kVars * (size_t)xg.nn) != cudaSuccess ||
        cudaMalloc(&cs->xdid, sizeof(int) * (size_t)xg.nn) != cudaSuccess ||
        cudaMalloc(&cs->xfl, 2 * (size_t)xg.nn) != cudaSuccess ||
        cudaMemset(cs->xfl, 0, 2 * (size_t)xg.nn) != cudaSuccess ||
        cudaMalloc(&prog, b_tasks + single.size() * sizeof(int2) + 16) != cudaSuccess ||
        cudaMemcpy(prog, tasks.data(), tasks.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(prog + b_tasks, single.data(), single.size() * sizeof(int2), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        cudaGetLastError();
        cudaFree(prog);
        return;  // the X sweep stays (acfd_finalize frees what was allocated)
    }
    cs->x_tasks = reinterpret_cast<int4 *>(prog);
    cs->x_ntask = (int)tasks.size();
    cs->x_single = reinterpret_cast<int2 *>(prog + b_tasks);
    cs->x_nsingle = (int)single.size();
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return;
    const cuuint64_t dims[5] = {(cuuint64_t)xg.pitch, (cuuint64_t)xg.n[1], (cuuint64_t)xg.n[2], 5, 3};
    const cuuint64_t strides[4] = {(cuuint64_t)xg.pitch * 8, (cuuint64_t)xg.pitch * xg.n[1] * 8,
                                   (cuuint64_t)xg.nn * 8, (cuuint64_t)xg.nn * 5 * 8};
    const cuuint32_t estr[5] = {1, 1, 1, 1, 1};
    const cuuint32_t box[5] = {(cuuint32_t)pt.BXp, 1, (cuuint32_t)pt.BC, 5, 1};
    if (encode(&cs->xmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, cs->xU, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
        return;
    }
    cs->xbox[0] = pt.BXp;
    cs->xbox[1] = pt.BC;
    cs->xg = xg;
    if (launch_transpose_int(cs->flags, g, cs->xdid, xg, cs->stream) != ACFD_OK) return;
    cs->xt_ok = true;
}

int debug_scan(acfd_case *cs, int l, const char *what, int s);
static int treat_boundary_fill(acfd_case *cs, int tn);

int treat_boundary(acfd_case *cs, int tn)
{
    const int st = treat_boundary_fill(cs, tn);
    return st != ACFD_OK ? st : debug_scan(cs, tn, "ghost fill", -1);
}

// TreatBoundary (boundary_treatment.c:28-65): the bodies' ghost nodes, then
// the domain's ghost shells
static int treat_boundary_fill(acfd_case *cs, int tn)
{
    if (cs->ib && ib_count(cs->ib) > 0) {
        cs->launches += ib_treat_launches(cs->ib, cs->part);
        int st = ib_treat(cs->ib, cs->grid, cs->mp, cs->part, cs->U, cs->flags, tn, cs->stream);
        if (st != ACFD_OK) {
            return st;
        }
    }
    double *U = level(cs, tn);
    if (cs->bc_gather) {
        ++cs->launches;
        return launch_ghost_program(cs->grid, cs->mp, cs->bc_faces, cs->bc_tasks, cs->bc_ntask, cs->bc_single,
                                    cs->bc_nsingle, cs->bc_progs, cs->bc_nprog, cs->bc_ops, U, cs->stream);
    }
    if (!cs->bc_multi) {
        if (cs->bc_groups.empty()) {
            return ACFD_OK;
        }
        ++cs->launches;
        return launch_domain_boundary_fused(cs->grid, cs->mp, cs->part, cs->bc_ptrs.data(), cs->bc_sizes.data(),
                                            (int)cs->bc_groups.size(), U, cs->bcbar, cs->dstatus, cs->stream);
    }
    for (const auto &grp : cs->bc_groups) {
        int st = launch_domain_boundary(cs->grid, cs->mp, cs->part, grp.data(), (int)grp.size(), U, cs->stream);
        if (st != ACFD_OK) {
            return st;
        }
        ++cs->launches;
    }
    return ACFD_OK;
}

// debug mode: scan level l for non-finite values and report `what`
int debug_scan(acfd_case *cs, int l, const char *what, int s)
{
    if (!cs->debug) {
        return ACFD_OK;
    }
    const int st = launch_finite_scan(level(cs, l), (long long)kVars * cs->grid.nn, cs->dbg_word, cs->stream);
    if (st != ACFD_OK) {
        return st;
    }
    int h = 0;
    ACFD_CUDA(cudaMemcpyAsync(&h, cs->dbg_word, sizeof(int), cudaMemcpyDeviceToHost, cs->stream));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    if (h != 0) {
        ACFD_CUDA(cudaMemsetAsync(cs->dbg_word, 0, sizeof(int), cs->stream));
        set_error("ACFD_DEBUG: %d values of U[%d] not finite after the %s of sweep axis %d", h, l, what, s);
        return ACFD_ERR_DEVICE;
    }
    return ACFD_OK;
}

int stage(acfd_case *cs, double dt_scale, double coeA, double coeB, int to, int tn, int tm, int p)
{
    StageArgs a;
    a.Uo = level(cs, to);
    a.Un = level(cs, tn);
    a.Um = level(cs, tm);
    a.did = cs->flags;
    a.dt = cs->d_dt;
    a.dt_scale = dt_scale;
    a.coeA = coeA;
    a.coeB = coeB;
    a.accumulate = 0;
    a.to = to;
    a.tn = tn;
    a.tm = tm;
    a.maps = cs->maps;
    a.omaps = nullptr;
    a.status = cs->dstatus;
    a.flags = cs->sensor_flags;
    a.wait_limit = cs->wait_limit;
    for (int s = 0; s < 3; ++s) {
        const int v = cs->tile_var[cs->mode][s];
        a.var[s] = v < kTileVariants ? v : 0;
    }
    if (p == ACFD_PHI) {
        ++cs->launches;
        return launch_stage_phi(cs->grid, cs->mp, a, cs->stream);
    }
    int s0 = p, s1 = p + 1;
    if (p == ACFD_DIMS) {
        s0 = 0;
        s1 = 3;
    }
    const bool visc = viscous(cs);
    // the stencil of the first and last interface of a line must stay inside
    // the node array (a sweep along a collapsed axis has no ghost layers)
    const int half = (cs->model.sScheme == 1) ? 3 : 2;
    for (int s = s0; s < s1; ++s) {
        const Grid &g = cs->grid;
        if (g.lo[s] - half < 0 || g.hi[s] - 1 + half > g.n[s] - 1) {
            set_error("sweep along axis %d needs %d ghost layers (nodes %d, PIN [%d,%d))", s, half, g.n[s],
                      g.lo[s], g.hi[s]);
            return ACFD_ERR_ARG;
        }
        if (visc) {
            for (int t = 0; t < 3; ++t) {
                if (t != s && (g.lo[t] < 1 || g.hi[t] > g.n[t] - 1)) {
                    set_error("viscous sweep needs one node beyond PIN on axis %d", t);
                    return ACFD_ERR_ARG;
                }
            }
        }
    }
    for (int s = s0; s < s1; ++s) {
        a.accumulate = (cs->model.multidim == 1 && s != 0) ? 1 : 0;
        int st;
        const int var = cs->tile_var[cs->mode][s];
        const bool plane_v = !cs->plain_kernels && var >= kPlaneFirst && var < kStageVariants;
        const bool plane = plane_v && cs->pmaps_ok;
        const bool march = !cs->plain_kernels && !plane && var >= kTileVariants && var < kStageVariants;
        const bool brick = !march && !plane && cs->maps_ok && !cs->plain_kernels;
        // march launch size: waves x SMs x resident warps per SM (two blocks of
        // eight warps in the FP32 forms, one in FP64)
        const int waves = plane_v ? kPlaneWaves[var - kPlaneFirst] : march ? kMarchWaves[var - kTileVariants] : 1;
        const int target32 = waves * cs->sms * 16, target64 = waves * cs->sms * 8;
        PlaneTile pt = {};
        if (plane) {
            pt = plane_tile(cs->grid, s, visc, waves, cs->sms, kPlaneShare[var - kPlaneFirst]);
            if (pt.BXp != cs->pbox[s][0] || pt.BC != cs->pbox[s][1]) {
                set_error("plane tile (%d x %d) does not match the encoded box (%d x %d) of axis %d", pt.BXp, pt.BC,
                          cs->pbox[s][0], cs->pbox[s][1], s);
                return ACFD_ERR_STATE;
            }
        }
        switch (cs->mode) {
            case ACFD_FP64_EXACT: st = launch_stage_exact(cs->grid, cs->mp, a, s, visc, cs->stream); break;
            case ACFD_FP64:
                st = plane   ? launch_stage_plane_fast(cs->grid, cs->mp, a, s, visc, pt, cs->pmaps[s], cs->stream)
                     : march ? launch_stage_march_fast(cs->grid, cs->mp, a, s, visc, target64, cs->stream)
                     : brick ? launch_stage_brick_fast(cs->grid, cs->mp, a, s, visc, cs->stream)
                             : launch_stage_fast(cs->grid, cs->mp, a, s, visc, cs->stream);
                break;
            case ACFD_FP32_HYBRID:
                st = plane   ? launch_stage_plane_fp32(cs->grid, cs->mp, a, s, visc, true, pt, cs->pmaps[s],
                                                       cs->stream)
                     : march ? launch_stage_march_fp32(cs->grid, cs->mp, a, s, visc, true, target32, cs->stream)
                     : brick ? launch_stage_brick_hybrid(cs->grid, cs->mp, a, s, visc, cs->stream)
                             : launch_stage_fp32(cs->grid, cs->mp, a, s, visc, cs->stream);
                break;
            default:
                st = plane   ? launch_stage_plane_fp32(cs->grid, cs->mp, a, s, visc, false, pt, cs->pmaps[s],
                                                       cs->stream)
                     : march ? launch_stage_march_fp32(cs->grid, cs->mp, a, s, visc, false, target32, cs->stream)
                     : brick ? launch_stage_brick_fp32(cs->grid, cs->mp, a, s, visc, cs->stream)
                             : launch_stage_fp32(cs->grid, cs->mp, a, s, visc, cs->stream);
                break;
        }
        if (st != ACFD_OK) {
            return st;
        }
        ++cs->launches;
        if ((st = debug_scan(cs, tm, "stage", s)) != ACFD_OK) {
            return st;
        }
    }
    return ACFD_OK;
}

#define TRY(x)                      \
    do {                            \
        int st__ = (x);             \
        if (st__ != ACFD_OK) return st__; \
    } while (0)

// DiscretizeTime (fluid_dynamics.c:121-148) with dt = dt_scale * step dt
// events around one piece of a step while a profile is taken (the end
// event is recorded when the piece's scope closes)
struct Piece {
    acfd_case *cs;
    cudaEvent_t e1 = nullptr;
    Piece(acfd_case *c, int kind, int axis, int stage) : cs(c)
    {
        if (!cs->prof) return;
        StepPiece p = {kind, axis, stage, nullptr, nullptr};
        if (cudaEventCreate(&p.e0) != cudaSuccess) return;
        if (cudaEventCreate(&p.e1) != cudaSuccess) {
            cudaEventDestroy(p.e0);
            return;
        }
        cudaEventRecord(p.e0, cs->stream);
        cs->prof->push_back(p);
        e1 = p.e1;
    }
    ~Piece()
    {
        if (e1) cudaEventRecord(e1, cs->stream);
    }
};

// the RK stages of DiscretizeTime (fluid_dynamics.c:121-148): coefficients
// of U[to] and of the updated U[tn], and the levels
struct RkStage {
    double coeA, coeB;
    int to, tn, tm;
};
const RkStage kRk2[2] = {{0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN}, {1.0 / 2.0, 1.0 / 2.0, ACFD_TO, ACFD_TN, ACFD_TO}};
const RkStage kRk3[3] = {{0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN},
                         {3.0 / 4.0, 1.0 / 4.0, ACFD_TO, ACFD_TN, ACFD_TM},
                         {1.0 / 3.0, 2.0 / 3.0, ACFD_TO, ACFD_TM, ACFD_TO}};

int discretize(acfd_case *cs, double dt_scale, int s)
{
    const RkStage *rk = cs->model.tScheme == 0 ? kRk2 : kRk3;
    const int n = cs->model.tScheme == 0 ? 2 : 3;
    for (int q = 0; q < n; ++q) {
        {
            Piece p(cs, ACFD_PIECE_STAGE, s, q);
            TRY(stage(cs, dt_scale, rk[q].coeA, rk[q].coeB, rk[q].to, rk[q].tn, rk[q].tm, s));
        }
        Piece p(cs, ACFD_PIECE_FILL, s, q);
        TRY(treat_boundary(cs, rk[q].tm));
    }
    return ACFD_OK;
}

// the X half steps may run as Y sweeps of the transposed state (build_xt):
// the FP32 forms, whose X sweep is slower than the Y sweep by more than the
// two transposes of U[TO] cost (the fast FP64 form's is not: TGV 128^3, 12 us
// a stage, 72 us a step, against 80 us of transposes), no bodies (whose ghost
// values follow the fill), no debug scans
bool xt_eligible(const acfd_case *cs)
{
    const bool form = cs->mode == ACFD_FP32_HYBRID || cs->mode == ACFD_FP32_BULK ||
                      (cs->xt_all_forms && cs->mode != ACFD_FP64_EXACT);
    return cs->xt_ok && !cs->debug && !cs->plain_kernels && form && !(cs->ib && ib_count(cs->ib) > 0);
}

// ... and do, when the X sweep's variant is a plane march (acfd_autotune
// picks one for an eligible case); a brick or line variant keeps the X sweep
bool use_xt(const acfd_case *cs)
{
    const int v = cs->tile_var[cs->mode][0];
    return xt_eligible(cs) && v >= kPlaneFirst && v < kStageVariants;
}

// one LLLU stage along x on the transposed levels: the Y plane march of xg
// with the X sweep's variant
int stage_xt(acfd_case *cs, double dt_scale, double coeA, double coeB, int to, int tn, int tm)
{
    const long long lv = (long long)kVars * cs->xg.nn;
    StageArgs a;
    a.Uo = cs->xU + to * lv;
    a.Un = cs->xU + tn * lv;
    a.Um = cs->xU + tm * lv;
    a.did = cs->xdid;
    a.dt = cs->d_dt;
    a.dt_scale = dt_scale;
    a.coeA = coeA;
    a.coeB = coeB;
    a.accumulate = 0;
    a.to = to;
    a.tn = tn;
    a.tm = tm;
    a.maps = nullptr;
    a.omaps = nullptr;
    a.var[0] = a.var[1] = a.var[2] = 0;
    a.status = cs->dstatus;
    a.flags = cs->xfl;
    a.wait_limit = cs->wait_limit;
    const int var = cs->tile_var[cs->mode][0];
    if (var < kPlaneFirst || var >= kStageVariants) {
        set_error("transposed X sweep: variant %d is not a plane march", var);
        return ACFD_ERR_STATE;
    }
    const int waves = kPlaneWaves[var - kPlaneFirst];
    const bool share = kPlaneShare[var - kPlaneFirst];
    const bool visc = viscous(cs);
    const PlaneTile pt = plane_tile(cs->xg, 1, visc, waves, cs->sms, share);
    if (pt.BXp != cs->xbox[0] || pt.BC != cs->xbox[1]) {
        set_error("transposed plane tile (%d x %d) does not match its box (%d x %d)", pt.BXp, pt.BC, cs->xbox[0],
                  cs->xbox[1]);
        return ACFD_ERR_STATE;
    }
    int st;
    switch (cs->mode) {
        case ACFD_FP64: st = launch_stage_plane_fast(cs->xg, cs->mp, a, 1, visc, pt, cs->xmap, cs->stream); break;
        case ACFD_FP32_HYBRID:
            st = launch_stage_plane_fp32(cs->xg, cs->mp, a, 1, visc, true, pt, cs->xmap, cs->stream);
            break;
        default: st = launch_stage_plane_fp32(cs->xg, cs->mp, a, 1, visc, false, pt, cs->xmap, cs->stream); break;
    }
    ++cs->launches;
    return st;
}

int fill_xt(acfd_case *cs, int tn)
{
    ++cs->launches;
    return launch_ghost_program(cs->xg, cs->mp, cs->bc_faces, cs->x_tasks, cs->x_ntask, cs->x_single,
                                cs->x_nsingle, nullptr, 0, nullptr, cs->xU + (long long)tn * kVars * cs->xg.nn,
                                cs->stream);
}

// DiscretizeTime along x on the transposed levels (the stages of discretize)
int discretize_xt(acfd_case *cs, double dt_scale)
{
    const RkStage *rk = cs->model.tScheme == 0 ? kRk2 : kRk3;
    const int n = cs->model.tScheme == 0 ? 2 : 3;
    for (int q = 0; q < n; ++q) {
        {
            Piece p(cs, ACFD_PIECE_STAGE_XT, ACFD_X, q);
            TRY(stage_xt(cs, dt_scale, rk[q].coeA, rk[q].coeB, rk[q].to, rk[q].tn, rk[q].tm));
        }
        Piece p(cs, ACFD_PIECE_FILL, ACFD_X, q);
        TRY(fill_xt(cs, rk[q].tm));
    }
    return ACFD_OK;
}

// U[TO] (every node, ghosts included) to and from the transposed levels
int xt_transpose(acfd_case *cs, bool into)
{
    Piece p(cs, ACFD_PIECE_TRANSPOSE, -1, 0);
    ++cs->launches;
    return into ? launch_transpose_state(level(cs, ACFD_TO), cs->grid, cs->xU, cs->xg, cs->stream)
                : launch_transpose_state(cs->xU, cs->xg, level(cs, ACFD_TO), cs->grid, cs->stream);
}

// EvolveFluidDynamics (fluid_dynamics.c:55-116); the step dt is in d_dt
int evolve(acfd_case *cs)
{
    static const int kOrder[9][6] = {
        {2, 1, 0, 0, 1, 2}, {2, 1, 1, 2, -1, -1}, {2, 0, 0, 2, -1, -1}, {1, 0, 0, 1, -1, -1},
        {-1, -1, -1, -1, -1, -1}, {2, 2, -1, -1, -1, -1}, {-1, -1, -1, -1, -1, -1},
        {1, 1, -1, -1, -1, -1}, {0, 0, -1, -1, -1, -1}};
    if (cs->mode == ACFD_FP32_HYBRID) {
        // sensor flags from U[TO], fixed for the whole step: the flags are
        // dilated by one node in the sweep, which covers the motion of a
        // feature during a step at CFL < 1
        Piece p(cs, ACFD_PIECE_SENSOR, -1, 0);
        TRY(launch_sensor_flags(cs->grid, cs->mp, cs->U, cs->flags, cs->sensor_params, cs->sensor_logit,
                                cs->sensor_rp, cs->sensor_flags, nullptr, cs->stream));
        cs->launches += 2;
    }
    const bool xt = use_xt(cs);
    if (xt && cs->mode == ACFD_FP32_HYBRID) {
        // the x flags as the flags of the transposed grid's axis 1
        Piece p(cs, ACFD_PIECE_TRANSPOSE, -1, 0);
        TRY(launch_transpose_u8(cs->sensor_flags, cs->grid, cs->xfl + cs->xg.nn, cs->xg, cs->stream));
        ++cs->launches;
    }
    if (cs->model.sState != 0) {
        TRY(discretize(cs, 0.5, ACFD_PHI));
    }
    if (cs->model.multidim == 0) {
        const int c = cs->part.collapse;
        if (c >= 0 && c < 9) {
            for (int n = 0; n < 6 && kOrder[c][n] >= 0; ++n) {
                const int ax = kOrder[c][n];
                if (ax == ACFD_X && xt) {
                    // a run of X half steps on the transposed state
                    if (n == 0 || kOrder[c][n - 1] != ACFD_X) TRY(xt_transpose(cs, true));
                    TRY(discretize_xt(cs, 0.5));
                    if (n + 1 >= 6 || kOrder[c][n + 1] != ACFD_X) TRY(xt_transpose(cs, false));
                } else {
                    TRY(discretize(cs, 0.5, ax));
                }
            }
        }
    } else if (cs->model.multidim == 1) {
        TRY(discretize(cs, 0.5, ACFD_DIMS));
        TRY(discretize(cs, 0.5, ACFD_DIMS));
    }
    if (cs->model.sState != 0) {
        TRY(discretize(cs, 0.5, ACFD_PHI));
    }
    return ACFD_OK;
}

int set_dt(acfd_case *cs, double dt)
{
    cudaError_t e = launch_k(set_scalar, dim3(1), dim3(1), 0, cs->stream, cs->d_dt, dt);
    ++cs->launches;
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "set_scalar launch");
}

void release_graph(acfd_case *cs)
{
    if (cs->graph_exec) {
        cudaGraphExecDestroy(cs->graph_exec);
        cs->graph_exec = nullptr;
    }
    if (cs->graph) {
        cudaGraphDestroy(cs->graph);
        cs->graph = nullptr;
    }
    cs->graph_mode = -1;
}

int check_case(const acfd_case *cs)
{
    if (!cs) {
        set_error("null case handle");
        return ACFD_ERR_ARG;
    }
    return ACFD_OK;
}

// ---- host <-> device copies of the node array --------------------------
// The node array of a caller is pageable memory; the runtime copies such
// memory through its own small pinned buffers at a fraction of PCIe speed.
// Instead the array goes through four pinned bounce chunks of 16 MB, filled
// and drained by several host threads while the others are in flight (on
// TGV 128^3, 335 MB: 7.9 / 7.5 ms up / down against 8.5 / 7.6 ms with two
// chunks of 32 MB; eight of 8 MB took 12.7 / 10.9 ms).  The chunks are
// shared by every case of the process (one copy at a time).
constexpr size_t kPinChunk = (size_t)16 << 20;
constexpr int kPinSlots = 4;

struct PinnedBounce {
    std::mutex lock;
    unsigned char *buf = nullptr;  // kPinSlots x kPinChunk, pinned and portable
};

// completion events of the chunks, on the calling thread's device
struct ChunkEvents {
    cudaEvent_t done[kPinSlots] = {};
    cudaError_t create()
    {
        cudaError_t e = cudaSuccess;
        for (int q = 0; q < kPinSlots && e == cudaSuccess; ++q) {
            e = cudaEventCreateWithFlags(&done[q], cudaEventDisableTiming);
        }
        return e;
    }
    ~ChunkEvents()
    {
        for (int q = 0; q < kPinSlots; ++q) {
            if (done[q]) {
                cudaEventSynchronize(done[q]);
                cudaEventDestroy(done[q]);
            }
        }
    }
};

PinnedBounce &bounce()
{
    static PinnedBounce b;
    return b;
}

// Host threads for the bounce copies, created once per process and reused
// (spawning threads for every chunk cost about as much as the copy): a copy
// is cut into parts that the workers and the calling thread take in turn.
// Used under the bounce lock, one copy at a time.  A process forked after
// the pool started (whose child has no workers) builds its own pool.
class CopyPool {
public:
    static CopyPool &get()
    {
        static std::mutex m;
        static CopyPool *pool = nullptr;
        std::lock_guard<std::mutex> g(m);
        if (!pool || pool->pid_ != getpid()) {
            pool = new CopyPool();  // a pool inherited across fork is left alone
        }
        return *pool;
    }
    void copy(void *dst, const void *src, size_t bytes)
    {
        const size_t kPart = (size_t)1 << 20;
        const size_t nparts = (bytes + kPart - 1) / kPart;
        if (workers_.empty() || nparts < 2) {
            memcpy(dst, src, bytes);
            return;
        }
        {
            std::lock_guard<std::mutex> g(m_);
            dst_ = (char *)dst;
            src_ = (const char *)src;
            bytes_ = bytes;
            part_ = kPart;
            nparts_ = nparts;
            next_.store(0);
            busy_ = (unsigned)workers_.size();
            ++gen_;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&] { return busy_ == 0; });
    }

private:
    CopyPool() : pid_(getpid())
    {
        unsigned T = std::thread::hardware_concurrency();
        T = std::min<unsigned>(T == 0 ? 1u : T, 16u);
        for (unsigned t = 1; t < T; ++t) {
            workers_.emplace_back([this] { loop(); });
            workers_.back().detach();  // the pool lives for the process
        }
    }
    void work()
    {
        for (size_t p = next_.fetch_add(1); p < nparts_; p = next_.fetch_add(1)) {
            const size_t off = p * part_;
            memcpy(dst_ + off, src_ + off, std::min(part_, bytes_ - off));
        }
    }
    void loop()
    {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
            }
            work();
            std::lock_guard<std::mutex> g(m_);
            if (--busy_ == 0) done_.notify_one();
        }
    }
    pid_t pid_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    unsigned long long gen_ = 0;
    unsigned busy_ = 0;
    char *dst_ = nullptr;
    const char *src_ = nullptr;
    size_t bytes_ = 0, part_ = 0, nparts_ = 0;
    std::atomic<size_t> next_{0};
};

void parallel_memcpy(void *dst, const void *src, size_t bytes)
{
    CopyPool::get().copy(dst, src, bytes);
}

int ensure_bounce(PinnedBounce &b)
{
    if (b.buf) return ACFD_OK;
    ACFD_CUDA(cudaHostAlloc(&b.buf, kPinSlots * kPinChunk, cudaHostAllocPortable));
    return ACFD_OK;
}

// host array -> device buffer, on the case's stream (returns with the copies
// queued; the bounce chunks are free again when the stream reaches them)
int upload_host(acfd_case *cs, void *dev, const void *host, size_t bytes)
{
    PinnedBounce &b = bounce();
    std::lock_guard<std::mutex> guard(b.lock);
    TRY(ensure_bounce(b));
    ChunkEvents ev;
    ACFD_CUDA(ev.create());
    int c = 0;
    const size_t K = kPinChunk;
    const int S = kPinSlots;
    for (size_t off = 0; off < bytes; off += K, ++c) {
        const size_t len = std::min(K, bytes - off);
        unsigned char *slot = b.buf + (size_t)(c % S) * K;
        ACFD_CUDA(cudaEventSynchronize(ev.done[c % S]));  // the copy that last read this chunk
        parallel_memcpy(slot, (const char *)host + off, len);
        ACFD_CUDA(cudaMemcpyAsync((char *)dev + off, slot, len, cudaMemcpyHostToDevice, cs->stream));
        ACFD_CUDA(cudaEventRecord(ev.done[c % S], cs->stream));
    }
    // the chunks must not be refilled by another case before these copies
    // ran: the events are waited for when they go out of scope, under the lock
    return ACFD_OK;
}

// device buffer -> host array (waits for the case's stream)
int download_host(acfd_case *cs, void *host, const void *dev, size_t bytes)
{
    PinnedBounce &b = bounce();
    std::lock_guard<std::mutex> guard(b.lock);
    TRY(ensure_bounce(b));
    ChunkEvents ev;
    ACFD_CUDA(ev.create());
    const size_t K = kPinChunk;
    const size_t S = kPinSlots;
    const size_t n = (bytes + K - 1) / K;
    auto issue = [&](size_t c) -> int {
        const size_t off = c * K, len = std::min(K, bytes - off);
        ACFD_CUDA(cudaMemcpyAsync(b.buf + (c % S) * K, (const char *)dev + off, len, cudaMemcpyDeviceToHost,
                                  cs->stream));
        ACFD_CUDA(cudaEventRecord(ev.done[c % S], cs->stream));
        return ACFD_OK;
    };
    for (size_t c = 0; c < n && c < S; ++c) TRY(issue(c));
    for (size_t c = 0; c < n; ++c) {
        ACFD_CUDA(cudaEventSynchronize(ev.done[c % S]));
        const size_t off = c * K, len = std::min(K, bytes - off);
        parallel_memcpy((char *)host + off, b.buf + (c % S) * K, len);
        if (c + S < n) TRY(issue(c + S));
    }
    return ACFD_OK;
}

int ensure_staging(acfd_case *cs)
{
    if (cs->staging) {
        return ACFD_OK;
    }
    const size_t total = (size_t)cs->grid.n[0] * cs->grid.n[1] * cs->grid.n[2];
    ACFD_CUDA(cudaMalloc(&cs->staging, total * sizeof(acfd_node_t)));
    return ACFD_OK;
}

}  // namespace

extern "C" {

int acfd_abi_version(void)
{
    return ACFD_ABI_VERSION;
}

int acfd_last_error(char *buf, size_t len)
{
    if (!buf || len == 0) {
        return ACFD_ERR_ARG;
    }
    snprintf(buf, len, "%s", g_err);
    return ACFD_OK;
}

int acfd_init(const acfd_partition_t *part, const acfd_model_t *model, acfd_case_t **out)
{
    if (!part || !model || !out) {
        set_error("acfd_init: null argument");
        return ACFD_ERR_ARG;
    }
    *out = nullptr;
    for (int s = 0; s < 3; ++s) {
        if (part->n[s] < 3 || part->ns[0][s][0] < 0 || part->ns[0][s][1] > part->n[s]) {
            set_error("acfd_init: invalid node counts/ranges on axis %d", s);
            return ACFD_ERR_ARG;
        }
    }
    if (model->sScheme != 0 && model->sScheme != 1) {
        set_error("acfd_init: sScheme %d not supported", model->sScheme);
        return ACFD_ERR_ARG;
    }
    if (model->tScheme != 0 && model->tScheme != 1) {
        set_error("acfd_init: tScheme %d not supported", model->tScheme);
        return ACFD_ERR_ARG;
    }
    acfd_case *cs = new acfd_case();
    cs->part = *part;
    cs->model = *model;
    ACFD_CUDA(cudaGetDevice(&cs->device));
    ACFD_CUDA(cudaDeviceGetAttribute(&cs->sms, cudaDevAttrMultiProcessorCount, cs->device));
    Grid &g = cs->grid;
    for (int s = 0; s < 3; ++s) {
        g.n[s] = part->n[s];
        g.lo[s] = part->ns[0][s][0];
        g.hi[s] = part->ns[0][s][1];
        g.dd[s] = part->dd[s];
    }
    g.pitch = (part->n[0] + 7) & ~7;
    g.nn = (long long)g.pitch * g.n[1] * g.n[2];
    ModelParams &m = cs->mp;
    m.gamma = model->gamma;
    m.gasR = model->gasR;
    m.cv = model->cv;
    m.refMu = model->refMu;
    m.refT = model->refT;
    for (int s = 0; s < 3; ++s) m.g[s] = model->g[s];
    m.sScheme = model->sScheme;
    m.jacobMean = model->jacobMean;
    m.fluxSplit = model->fluxSplit;
    m.multidim = model->multidim;
    m.sState = model->sState;
    m.ibmLayer = model->ibmLayer;
    int st = ACFD_OK;
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&cs->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        st = cuda_status(e, "cudaStreamCreate");
        delete cs;
        return st;
    }
    cs->own_stream = true;
    const size_t ubytes = sizeof(double) * kLevels * kVars * (size_t)g.nn;
    const size_t fbytes = sizeof(int) * 4 * (size_t)g.nn;
    if ((e = cudaMalloc(&cs->U, ubytes)) != cudaSuccess ||
        (e = cudaMalloc(&cs->flags, fbytes)) != cudaSuccess ||
        (e = cudaMalloc(&cs->d_dt, sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&cs->cfl_part, sizeof(double) * kCflPartials)) != cudaSuccess ||
        (e = cudaMemset(cs->cfl_part, 0, sizeof(double) * kCflPartials)) != cudaSuccess ||
        (e = cudaMalloc(&cs->cfl_out, sizeof(double) * 4)) != cudaSuccess ||
        (e = cudaMallocHost(&cs->h_cfl, sizeof(double) * 4)) != cudaSuccess ||
        (e = cudaMalloc(&cs->dstatus, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&cs->bcbar, 2 * sizeof(unsigned))) != cudaSuccess) {
        st = cuda_status(e, "acfd_init allocation");
        acfd_finalize(cs);
        return st;
    }
    // padding and never-written nodes: flags -1 (outside PIN), U zero
    cudaMemsetAsync(cs->U, 0, ubytes, cs->stream);
    cudaMemsetAsync(cs->flags, 0xff, fbytes, cs->stream);
    cudaMemsetAsync(cs->dstatus, 0, sizeof(int), cs->stream);
    cudaMemsetAsync(cs->bcbar, 0, 2 * sizeof(unsigned), cs->stream);
    // one launch per ghost-fill phase by default: measured faster on B200 than
    // the single cooperative launch with grid barriers (ACFD_BC_FUSED=1)
    cs->bc_multi = (getenv("ACFD_BC_FUSED") == nullptr);
    if ((st = encode_state_maps(cs)) != ACFD_OK) {
        acfd_finalize(cs);
        return st;
    }
    if (getenv("ACFD_PLAIN_KERNELS")) {
        cs->plain_kernels = true;
    }
    {
        const char *dbg = getenv("ACFD_DEBUG");
        if (dbg && atoi(dbg) != 0) {
            if ((e = cudaMalloc(&cs->dbg_word, sizeof(int))) != cudaSuccess ||
                (e = cudaMemsetAsync(cs->dbg_word, 0, sizeof(int), cs->stream)) != cudaSuccess) {
                st = cuda_status(e, "acfd_init (debug word)");
                acfd_finalize(cs);
                return st;
            }
            cs->debug = true;
        }
    }
    if ((st = ib_create(&cs->ib)) != ACFD_OK) {
        acfd_finalize(cs);
        return st;
    }
    build_bc_plan(cs);
    // the ordered per-phase launches stay available for comparison
    // (ACFD_BC_PHASES=1 in the environment)
    if (!getenv("ACFD_BC_PHASES") && !getenv("ACFD_BC_FUSED")) {
        if ((e = cudaStreamSynchronize(cs->stream)) != cudaSuccess) {
            st = cuda_status(e, "acfd_init");
            acfd_finalize(cs);
            return st;
        }
        cs->bc_gather = build_bc_program(cs);
        build_xt(cs);
    }
    if ((e = cudaStreamSynchronize(cs->stream)) != cudaSuccess) {
        st = cuda_status(e, "acfd_init");
        acfd_finalize(cs);
        return st;
    }
    *out = cs;
    return ACFD_OK;
}

int acfd_finalize(acfd_case_t *cs)
{
    if (!cs) {
        return ACFD_OK;
    }
    if (cs->stream) {
        cudaStreamSynchronize(cs->stream);
    }
    release_graph(cs);
    if (cs->ib) ib_destroy(cs->ib);
    cudaFree(cs->U);
    cudaFree(cs->flags);
    cudaFree(cs->d_dt);
    cudaFree(cs->cfl_part);
    cudaFree(cs->cfl_out);
    cudaFree(cs->dstatus);
    cudaFree(cs->bcbar);
    cudaFree(cs->bc_pairs);
    release_xt(cs);
    cudaFree(cs->dbg_word);
    cudaFree(cs->sensor_params);
    cudaFree(cs->sensor_flags);
    cudaFree(cs->sensor_rp);
    cudaFree(cs->sensor_count);
    cudaFree(cs->staging);
    if (cs->snap_pending && cs->snap_copied) cudaEventSynchronize(cs->snap_copied);
    cudaFree(cs->snap_dev);
    if (cs->snap_host) cudaFreeHost(cs->snap_host);
    if (cs->snap_gathered) cudaEventDestroy(cs->snap_gathered);
    if (cs->snap_copied) cudaEventDestroy(cs->snap_copied);
    if (cs->snap_stream) cudaStreamDestroy(cs->snap_stream);
    if (cs->h_cfl) cudaFreeHost(cs->h_cfl);
    if (cs->own_stream && cs->stream) cudaStreamDestroy(cs->stream);
    delete cs;
    return ACFD_OK;
}

int acfd_set_stream(acfd_case_t *cs, void *stream)
{
    TRY(check_case(cs));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    if (cs->own_stream) {
        cudaStreamDestroy(cs->stream);
        cs->own_stream = false;
    }
    if (stream) {
        cs->stream = (cudaStream_t)stream;
    } else {
        ACFD_CUDA(cudaStreamCreateWithFlags(&cs->stream, cudaStreamNonBlocking));
        cs->own_stream = true;
    }
    release_graph(cs);
    return ACFD_OK;
}

int acfd_set_precision(acfd_case_t *cs, int mode)
{
    TRY(check_case(cs));
    if (mode < ACFD_FP64_EXACT || mode > ACFD_FP32_HYBRID) {
        set_error("acfd_set_precision: unknown mode %d", mode);
        return ACFD_ERR_ARG;
    }
    if (mode == ACFD_FP32_HYBRID && !cs->sensor_ok) {
        set_error("acfd_set_precision: the hybrid form needs a loaded sensor (acfd_sensor_load)");
        return ACFD_ERR_STATE;
    }
    if (mode != cs->mode) {
        release_graph(cs);
    }
    cs->mode = mode;
    return ACFD_OK;
}

int acfd_sync_to_device(acfd_case_t *cs, const acfd_node_t *node, unsigned mask)
{
    TRY(check_case(cs));
    if (!node) {
        set_error("acfd_sync_to_device: null node array");
        return ACFD_ERR_ARG;
    }
    TRY(ensure_staging(cs));
    const size_t total = (size_t)cs->grid.n[0] * cs->grid.n[1] * cs->grid.n[2];
    TRY(upload_host(cs, cs->staging, node, total * sizeof(acfd_node_t)));
    TRY(launch_scatter_nodes(cs->grid, cs->staging, cs->U, cs->flags, mask, cs->stream));
    if (mask & ACFD_SYNC_FLAGS) {
        TRY(ib_flags_changed(cs->ib, cs->grid, cs->mp, cs->part, cs->flags, cs->stream));
        if (cs->xt_ok) {
            TRY(launch_transpose_int(cs->flags, cs->grid, cs->xdid, cs->xg, cs->stream));  // the node types
        }
    }
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    return ACFD_OK;
}

int acfd_sync_to_host(acfd_case_t *cs, acfd_node_t *node, unsigned mask)
{
    TRY(check_case(cs));
    if (!node) {
        set_error("acfd_sync_to_host: null node array");
        return ACFD_ERR_ARG;
    }
    TRY(ensure_staging(cs));
    const size_t total = (size_t)cs->grid.n[0] * cs->grid.n[1] * cs->grid.n[2];
    // keep host members that are not selected: start from the host copy
    if ((mask & ACFD_SYNC_ALL) != ACFD_SYNC_ALL) {
        TRY(upload_host(cs, cs->staging, node, total * sizeof(acfd_node_t)));
    }
    TRY(launch_gather_nodes(cs->grid, cs->U, cs->flags, cs->staging, mask, cs->stream));
    TRY(download_host(cs, node, cs->staging, total * sizeof(acfd_node_t)));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    TRY(check_device_status(cs));
    return ib_check(cs->ib, cs->stream);
}

int acfd_device_state(acfd_case_t *cs, double **U, int **flags, int *pitch, size_t *plane)
{
    TRY(check_case(cs));
    if (U) *U = cs->U;
    if (flags) *flags = cs->flags;
    if (pitch) *pitch = cs->grid.pitch;
    if (plane) *plane = (size_t)cs->grid.nn;
    return ACFD_OK;
}

int acfd_cfl(acfd_case_t *cs, double vmax[3])
{
    TRY(check_case(cs));
    if (!vmax) {
        set_error("acfd_cfl: null output");
        return ACFD_ERR_ARG;
    }
    TRY(launch_cfl(cs->grid, cs->mp, cs->U, cs->flags, cs->cfl_part, cs->cfl_out, cs->stream));
    ++cs->launches;
    ACFD_CUDA(cudaMemcpyAsync(cs->h_cfl, cs->cfl_out, 4 * sizeof(double), cudaMemcpyDeviceToHost, cs->stream));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    for (int s = 0; s < 3; ++s) {
        vmax[s] = cs->h_cfl[s];
    }
    if (cs->h_cfl[3] != 0.0) {
        set_error("acfd_cfl: a fluid node of U[TO] has a non-finite wave speed (NaN or Inf in the state); "
                  "the maxima exclude it");
        return ACFD_ERR_DEVICE;
    }
    TRY(check_device_status(cs));
    return ib_check(cs->ib, cs->stream);
}

int acfd_evolve_fluid(acfd_case_t *cs, double dt)
{
    TRY(check_case(cs));
    TRY(set_dt(cs, dt));
    TRY(evolve(cs));
    return ACFD_OK;
}

int acfd_profile_step(acfd_case_t *cs, double dt, int cap, int *kind, int *axis, int *stage, float *ms, int *count)
{
    TRY(check_case(cs));
    if (cap < 0 || !count || (cap > 0 && (!kind || !axis || !stage || !ms))) {
        set_error("acfd_profile_step: bad output arrays");
        return ACFD_ERR_ARG;
    }
    std::vector<StepPiece> pieces;
    cs->prof = &pieces;
    int st = set_dt(cs, dt);
    if (st == ACFD_OK) st = evolve(cs);
    cs->prof = nullptr;
    const cudaError_t e = cudaStreamSynchronize(cs->stream);
    *count = (int)pieces.size();
    for (size_t i = 0; i < pieces.size(); ++i) {
        float t = 0.0f;
        if (st == ACFD_OK && e == cudaSuccess) cudaEventElapsedTime(&t, pieces[i].e0, pieces[i].e1);
        if ((int)i < cap) {
            kind[i] = pieces[i].kind;
            axis[i] = pieces[i].axis;
            stage[i] = pieces[i].stage;
            ms[i] = t;
        }
        cudaEventDestroy(pieces[i].e0);
        cudaEventDestroy(pieces[i].e1);
    }
    TRY(st);
    if (e != cudaSuccess) return cuda_status(e, "acfd_profile_step");
    return check_device_status(cs);
}

int acfd_evolve_fluid_graph(acfd_case_t *cs, double dt)
{
    TRY(check_case(cs));
    if (cs->debug) {
        return acfd_evolve_fluid(cs, dt);  // the per-stage checks synchronize: no capture
    }
    TRY(set_dt(cs, dt));
    if (!cs->graph_exec || cs->graph_mode != cs->mode) {
        release_graph(cs);
        ACFD_CUDA(cudaStreamBeginCapture(cs->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = cs->launches;
        int st = evolve(cs);
        cs->graph_kernels = cs->launches - before;
        cs->launches = before;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs->stream, &graph);
        if (st != ACFD_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) {
            return cuda_status(e, "cudaStreamEndCapture");
        }
        cs->graph = graph;
        ACFD_CUDA(cudaGraphInstantiate(&cs->graph_exec, cs->graph, 0));
        cs->graph_mode = cs->mode;
    }
    ACFD_CUDA(cudaGraphLaunch(cs->graph_exec, cs->stream));
    cs->launches += cs->graph_kernels;
    return ACFD_OK;
}

int acfd_autotune(acfd_case_t *cs, int tiles[3])
{
    TRY(check_case(cs));
    int *var_of = cs->tile_var[cs->mode];
    if (cs->mode == ACFD_FP64_EXACT || cs->plain_kernels) {
        for (int s = 0; s < 3; ++s) {
            if (tiles) tiles[s] = var_of[s];
        }
        return ACFD_OK;  // the exact form has no tile choice
    }
    cudaEvent_t e0, e1;
    ACFD_CUDA(cudaEventCreate(&e0));
    ACFD_CUDA(cudaEventCreate(&e1));
    int st = set_dt(cs, 0.0);
    if (st == ACFD_OK && cs->mode == ACFD_FP32_HYBRID) {
        // the flags of the current state, as a step would use them
        st = launch_sensor_flags(cs->grid, cs->mp, cs->U, cs->flags, cs->sensor_params, cs->sensor_logit,
                                 cs->sensor_rp, cs->sensor_flags, nullptr, cs->stream);
    }
    const int half = (cs->model.sScheme == 1) ? 3 : 2;
    for (int s = 0; s < 3 && st == ACFD_OK; ++s) {
        const Grid &g = cs->grid;
        if (g.lo[s] - half < 0 || g.hi[s] - 1 + half > g.n[s] - 1) {
            continue;  // no sweep along a collapsed axis
        }
        // an X sweep that may run transposed is timed as it would run: the
        // plane-march variants of the Y sweep over the transposed state
        const bool xt = s == 0 && xt_eligible(cs);
        if (xt) {
            st = xt_transpose(cs, true);
            if (st == ACFD_OK && cs->mode == ACFD_FP32_HYBRID) {
                st = launch_transpose_u8(cs->sensor_flags, cs->grid, cs->xfl + cs->xg.nn, cs->xg, cs->stream);
            }
        }
        auto run = [&](double coeA, double coeB, int tn, int tm) {
            return xt ? stage_xt(cs, 1.0, coeA, coeB, ACFD_TO, tn, tm)
                      : stage(cs, 1.0, coeA, coeB, ACFD_TO, tn, tm, s);
        };
        float best = 1e30f;
        int best_var = var_of[s];
        for (int var = xt ? kPlaneFirst : (cs->maps_ok ? 0 : kTileVariants); var < kStageVariants && st == ACFD_OK;
             ++var) {
            var_of[s] = var;
            // RK stage 1 (U[TO] -> U[TN]) then the timed RK stage 2 (U[TO],
            // U[TN] -> U[TM]), which reads two levels like stages 2 and 3 of
            // every step; both levels written are overwritten by every step
            st = run(0.0, 1.0, ACFD_TO, ACFD_TN);
            if (st == ACFD_OK) st = run(0.75, 0.25, ACFD_TN, ACFD_TM);  // warm-up
            float total = 0.0f;
            for (int rep = 0; rep < 3 && st == ACFD_OK; ++rep) {
                cudaEventRecord(e0, cs->stream);
                st = run(0.75, 0.25, ACFD_TN, ACFD_TM);
                cudaEventRecord(e1, cs->stream);
                cudaEventSynchronize(e1);
                float ms = 0.0f;
                cudaEventElapsedTime(&ms, e0, e1);
                total += ms;
            }
            if (st == ACFD_OK && total < best) {
                best = total;
                best_var = var;
            }
        }
        var_of[s] = best_var;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st != ACFD_OK) {
        return st;
    }
    release_graph(cs);
    TRY(check_device_status(cs));
    for (int s = 0; s < 3; ++s) {
        if (tiles) tiles[s] = var_of[s];
    }
    return ACFD_OK;
}

int acfd_set_tiles(acfd_case_t *cs, const int tiles[3])
{
    TRY(check_case(cs));
    if (!tiles) {
        set_error("acfd_set_tiles: null tiles");
        return ACFD_ERR_ARG;
    }
    for (int s = 0; s < 3; ++s) {
        if (tiles[s] < 0 || tiles[s] >= kStageVariants || (tiles[s] < kTileVariants && !cs->maps_ok)) {
            set_error("acfd_set_tiles: variant %d of axis %d not available", tiles[s], s);
            return ACFD_ERR_ARG;
        }
    }
    for (int s = 0; s < 3; ++s) {
        cs->tile_var[cs->mode][s] = tiles[s];
    }
    release_graph(cs);
    return ACFD_OK;
}

int acfd_set_wait_limit(acfd_case_t *cs, long long polls)
{
    TRY(check_case(cs));
    cs->wait_limit = polls < 0 ? kWaitLimitDefault : polls;
    release_graph(cs);  // a captured step holds the limit of its stage launches
    return ACFD_OK;
}

int acfd_sensor_load(acfd_case_t *cs, const float *params, float threshold)
{
    TRY(check_case(cs));
    if (!params || !(threshold > 0.0f) || !(threshold < 1.0f)) {
        set_error("acfd_sensor_load: parameters and a threshold in (0,1) are required");
        return ACFD_ERR_ARG;
    }
    const int np = sensor_param_count();
    if (!cs->sensor_params) {
        ACFD_CUDA(cudaMalloc(&cs->sensor_params, sizeof(float) * np));
        ACFD_CUDA(cudaMalloc(&cs->sensor_flags, (size_t)3 * cs->grid.nn));
        ACFD_CUDA(cudaMalloc(&cs->sensor_rp, sizeof(float2) * cs->grid.nn));
        ACFD_CUDA(cudaMalloc(&cs->sensor_count, sizeof(unsigned long long)));
    }
    ACFD_CUDA(cudaMemcpyAsync(cs->sensor_params, params, sizeof(float) * np, cudaMemcpyHostToDevice, cs->stream));
    ACFD_CUDA(cudaMemsetAsync(cs->sensor_flags, 1, (size_t)3 * cs->grid.nn, cs->stream));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    cs->sensor_logit = logf(threshold / (1.0f - threshold));
    cs->sensor_ok = true;
    release_graph(cs);
    return ACFD_OK;
}

int acfd_sensor_load_file(acfd_case_t *cs, const char *path)
{
    TRY(check_case(cs));
    if (!path) {
        set_error("acfd_sensor_load_file: null path");
        return ACFD_ERR_ARG;
    }
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        set_error("acfd_sensor_load_file: cannot open %s", path);
        return ACFD_ERR_IO;
    }
    char magic[8];
    int32_t count = 0;
    float threshold = 0.0f;
    const int np = sensor_param_count();
    std::vector<float> params((size_t)np);
    const bool ok = fread(magic, 1, 8, fp) == 8 && memcmp(magic, "ACFDSNS1", 8) == 0 &&
                    fread(&count, sizeof(count), 1, fp) == 1 && count == np &&
                    fread(&threshold, sizeof(threshold), 1, fp) == 1 &&
                    fread(params.data(), sizeof(float), (size_t)np, fp) == (size_t)np;
    fclose(fp);
    if (!ok) {
        set_error("acfd_sensor_load_file: %s is not a sensor file of %d parameters", path, np);
        return ACFD_ERR_IO;
    }
    return acfd_sensor_load(cs, params.data(), threshold);
}

int acfd_sensor_update(acfd_case_t *cs, unsigned long long *flagged)
{
    TRY(check_case(cs));
    if (!cs->sensor_ok) {
        set_error("acfd_sensor_update: no sensor loaded");
        return ACFD_ERR_STATE;
    }
    ACFD_CUDA(cudaMemsetAsync(cs->sensor_count, 0, sizeof(unsigned long long), cs->stream));
    TRY(launch_sensor_flags(cs->grid, cs->mp, cs->U, cs->flags, cs->sensor_params, cs->sensor_logit,
                            cs->sensor_rp, cs->sensor_flags, cs->sensor_count, cs->stream));
    cs->launches += 2;
    if (flagged) {
        ACFD_CUDA(cudaMemcpyAsync(flagged, cs->sensor_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                  cs->stream));
        ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    }
    return ACFD_OK;
}

int acfd_sensor_flags(acfd_case_t *cs, const unsigned char **flags)
{
    TRY(check_case(cs));
    if (!flags) {
        set_error("acfd_sensor_flags: null output");
        return ACFD_ERR_ARG;
    }
    if (!cs->sensor_ok) {
        set_error("acfd_sensor_flags: no sensor loaded");
        return ACFD_ERR_STATE;
    }
    *flags = cs->sensor_flags;
    return ACFD_OK;
}

int acfd_sensor_features(acfd_case_t *cs, int s, float *features, float *departure)
{
    TRY(check_case(cs));
    if (s < 0 || s > 2 || !features || !departure) {
        set_error("acfd_sensor_features: bad arguments");
        return ACFD_ERR_ARG;
    }
    if (cs->model.sScheme != 1) {
        set_error("acfd_sensor_features: the sensor is defined for WENO5");
        return ACFD_ERR_ARG;
    }
    TRY(launch_sensor_features(cs->grid, cs->mp, cs->U, cs->flags, s, features, departure, cs->stream));
    ++cs->launches;
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    return ACFD_OK;
}

int acfd_synchronize(acfd_case_t *cs)
{
    TRY(check_case(cs));
    ACFD_CUDA(cudaStreamSynchronize(cs->stream));
    TRY(check_device_status(cs));
    return ib_check(cs->ib, cs->stream);
}

int acfd_stats(acfd_case_t *cs, long long *launches)
{
    TRY(check_case(cs));
    if (launches) *launches = cs->launches;
    return ACFD_OK;
}

int acfd_discretize_time(acfd_case_t *cs, double dt, int s)
{
    TRY(check_case(cs));
    if (s < 0 || s > ACFD_PHI) {
        set_error("acfd_discretize_time: operator %d", s);
        return ACFD_ERR_ARG;
    }
    TRY(set_dt(cs, dt));
    return discretize(cs, 1.0, s);
}

int acfd_lllu(acfd_case_t *cs, double dt, double coeA, double coeB, int to, int tn, int tm, int s)
{
    TRY(check_case(cs));
    if (to < 0 || to > 2 || tn < 0 || tn > 2 || tm < 0 || tm > 2 || s < 0 || s > ACFD_PHI || tn == tm) {
        set_error("acfd_lllu: bad levels/operator");
        return ACFD_ERR_ARG;
    }
    TRY(set_dt(cs, dt));
    return stage(cs, 1.0, coeA, coeB, to, tn, tm, s);
}

int acfd_treat_boundary(acfd_case_t *cs, int tn)
{
    TRY(check_case(cs));
    if (tn < 0 || tn > 2) {
        set_error("acfd_treat_boundary: level %d", tn);
        return ACFD_ERR_ARG;
    }
    return treat_boundary(cs, tn);
}

int acfd_geo_upload(acfd_case_t *cs, const acfd_polyhedron_t *poly, int totN)
{
    TRY(check_case(cs));
    if (totN < 0 || (totN > 0 && !poly)) {
        set_error("acfd_geo_upload: bad body list");
        return ACFD_ERR_ARG;
    }
    // bodies change the node types through their treatment: the X half steps
    // stay on the X sweep from now on
    const bool leave_xt = totN > 0 && cs->xt_ok;
    if (totN > 0) cs->xt_ok = false;
    bool relayout = true;
    TRY(ib_upload(cs->ib, poly, totN, cs->part, cs->stream, &relayout));
    // bodies moved in place keep every device pointer and launch shape of a
    // captured step; a new body list does not
    if (relayout || leave_xt) release_graph(cs);
    return ACFD_OK;
}

int acfd_transform_polyhedron(acfd_case_t *cs, int n, const double O[3], const double scale[3],
                              const double angle[3], const double offset[3], double centroid[3],
                              double inertia[9], double box[6])
{
    TRY(check_case(cs));
    if (!O || !scale || !angle || !offset || !centroid || !inertia || !box) {
        set_error("acfd_transform_polyhedron: null argument");
        return ACFD_ERR_ARG;
    }
    return ib_transform(cs->ib, n, O, scale, angle, offset, centroid, inertia, box, cs->stream);
}

int acfd_geo_fetch(acfd_case_t *cs, int n, double *v, double *Nf, double *Ne, double *Nv)
{
    TRY(check_case(cs));
    return ib_fetch(cs->ib, n, v, Nf, Ne, Nv, cs->stream);
}

int acfd_compute_geometric_field(acfd_case_t *cs)
{
    TRY(check_case(cs));
    return ib_compute_geometric_field(cs->ib, cs->grid, cs->mp, cs->part, cs->U, cs->flags, cs->stream);
}

int acfd_treat_ib(acfd_case_t *cs, int tn)
{
    TRY(check_case(cs));
    if (tn < 0 || tn > 2) {
        set_error("acfd_treat_ib: level %d", tn);
        return ACFD_ERR_ARG;
    }
    return ib_treat(cs->ib, cs->grid, cs->mp, cs->part, cs->U, cs->flags, tn, cs->stream);
}

// ---- snapshots and FP64 checkpoints ------------------------------------
// File layout of a checkpoint (little-endian): a 64-byte header, the
// caller's block, then the node records of every node (ghosts included) in
// the reference's Node layout, so that the state round-trips bit for bit.
struct CheckpointHeader {
    char magic[8];        // "ACFDCKP1"
    int32_t version;      // 1
    int32_t node_bytes;   // sizeof(acfd_node_t)
    int32_t n[3];         // allocated nodes per axis
    int32_t pad;
    int64_t count;        // n[0] * n[1] * n[2]
    int64_t user_bytes;   // size of the caller's block
    int64_t reserved[2];
};
static_assert(sizeof(CheckpointHeader) == 64, "checkpoint header layout");
static const char kCheckpointMagic[8] = {'A', 'C', 'F', 'D', 'C', 'K', 'P', '1'};

static size_t node_count(const acfd_case *cs)
{
    return (size_t)cs->grid.n[0] * cs->grid.n[1] * cs->grid.n[2];
}

int acfd_snapshot_begin(acfd_case_t *cs)
{
    TRY(check_case(cs));
    const size_t total = node_count(cs);
    if (!cs->snap_dev) {
        ACFD_CUDA(cudaMalloc(&cs->snap_dev, total * sizeof(acfd_node_t)));
        ACFD_CUDA(cudaMallocHost(&cs->snap_host, total * sizeof(acfd_node_t)));
        ACFD_CUDA(cudaStreamCreateWithFlags(&cs->snap_stream, cudaStreamNonBlocking));
        ACFD_CUDA(cudaEventCreateWithFlags(&cs->snap_gathered, cudaEventDisableTiming));
        ACFD_CUDA(cudaEventCreateWithFlags(&cs->snap_copied, cudaEventDisableTiming));
    }
    if (cs->snap_pending) {
        // the previous snapshot's copy still reads snap_dev
        ACFD_CUDA(cudaStreamWaitEvent(cs->stream, cs->snap_copied, 0));
    }
    // the state as the case's stream has it now: node records on the device,
    // then copied to pinned memory on a stream of their own, overlapping the
    // work queued on the case's stream after this call
    TRY(launch_gather_nodes(cs->grid, cs->U, cs->flags, cs->snap_dev, ACFD_SYNC_ALL, cs->stream));
    ACFD_CUDA(cudaEventRecord(cs->snap_gathered, cs->stream));
    ACFD_CUDA(cudaStreamWaitEvent(cs->snap_stream, cs->snap_gathered, 0));
    ACFD_CUDA(cudaMemcpyAsync(cs->snap_host, cs->snap_dev, total * sizeof(acfd_node_t), cudaMemcpyDeviceToHost,
                              cs->snap_stream));
    ACFD_CUDA(cudaEventRecord(cs->snap_copied, cs->snap_stream));
    cs->snap_pending = true;
    return ACFD_OK;
}

static int snapshot_wait(acfd_case *cs, const char *who)
{
    if (!cs->snap_pending) {
        set_error("%s: no snapshot taken (acfd_snapshot_begin)", who);
        return ACFD_ERR_STATE;
    }
    ACFD_CUDA(cudaEventSynchronize(cs->snap_copied));
    return ACFD_OK;
}

int acfd_snapshot_nodes(acfd_case_t *cs, acfd_node_t *node)
{
    TRY(check_case(cs));
    if (!node) {
        set_error("acfd_snapshot_nodes: null node array");
        return ACFD_ERR_ARG;
    }
    TRY(snapshot_wait(cs, "acfd_snapshot_nodes"));
    memcpy(node, cs->snap_host, node_count(cs) * sizeof(acfd_node_t));
    return ACFD_OK;
}

static int write_checkpoint(const acfd_case *cs, const char *path, const void *user, size_t user_bytes,
                            const acfd_node_t *nodes)
{
    if (!path || (user_bytes && !user)) {
        set_error("checkpoint: null path or user block");
        return ACFD_ERR_ARG;
    }
    CheckpointHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, kCheckpointMagic, 8);
    h.version = 1;
    h.node_bytes = (int32_t)sizeof(acfd_node_t);
    for (int s = 0; s < 3; ++s) h.n[s] = cs->grid.n[s];
    h.count = (int64_t)node_count(cs);
    h.user_bytes = (int64_t)user_bytes;
    FILE *fp = fopen(path, "wb");
    if (!fp) {
        set_error("checkpoint: cannot open %s for writing", path);
        return ACFD_ERR_IO;
    }
    bool ok = fwrite(&h, sizeof(h), 1, fp) == 1;
    if (ok && user_bytes) ok = fwrite(user, 1, user_bytes, fp) == user_bytes;
    if (ok) ok = fwrite(nodes, sizeof(acfd_node_t), (size_t)h.count, fp) == (size_t)h.count;
    ok = (fclose(fp) == 0) && ok;
    if (!ok) {
        set_error("checkpoint: writing %s failed", path);
        return ACFD_ERR_IO;
    }
    return ACFD_OK;
}

int acfd_snapshot_save(acfd_case_t *cs, const char *path, const void *user, size_t user_bytes)
{
    TRY(check_case(cs));
    TRY(snapshot_wait(cs, "acfd_snapshot_save"));
    return write_checkpoint(cs, path, user, user_bytes, cs->snap_host);
}

int acfd_checkpoint_save(acfd_case_t *cs, const char *path, const void *user, size_t user_bytes)
{
    TRY(acfd_snapshot_begin(cs));
    return acfd_snapshot_save(cs, path, user, user_bytes);
}

int acfd_checkpoint_load(acfd_case_t *cs, const char *path, void *user, size_t user_cap, size_t *user_bytes)
{
    TRY(check_case(cs));
    if (!path) {
        set_error("acfd_checkpoint_load: null path");
        return ACFD_ERR_ARG;
    }
    FILE *fp = fopen(path, "rb");
    if (!fp) {
        set_error("acfd_checkpoint_load: cannot open %s", path);
        return ACFD_ERR_IO;
    }
    CheckpointHeader h;
    int st = ACFD_OK;
    if (fread(&h, sizeof(h), 1, fp) != 1 || memcmp(h.magic, kCheckpointMagic, 8) != 0 || h.version != 1 ||
        h.node_bytes != (int32_t)sizeof(acfd_node_t)) {
        set_error("acfd_checkpoint_load: %s is not a version-1 checkpoint", path);
        st = ACFD_ERR_IO;
    } else if (h.n[0] != cs->grid.n[0] || h.n[1] != cs->grid.n[1] || h.n[2] != cs->grid.n[2] ||
               h.count != (int64_t)node_count(cs)) {
        set_error("acfd_checkpoint_load: %s holds %d x %d x %d nodes, the case %d x %d x %d", path, h.n[0], h.n[1],
                  h.n[2], cs->grid.n[0], cs->grid.n[1], cs->grid.n[2]);
        st = ACFD_ERR_ARG;
    } else if (h.user_bytes < 0 || (size_t)h.user_bytes > user_cap || (h.user_bytes && !user)) {
        set_error("acfd_checkpoint_load: user block of %lld bytes, room for %zu", (long long)h.user_bytes, user_cap);
        st = ACFD_ERR_ARG;
    }
    if (user_bytes) *user_bytes = (st == ACFD_OK || st == ACFD_ERR_ARG) ? (size_t)std::max<int64_t>(0, h.user_bytes) : 0;
    if (st == ACFD_OK && h.user_bytes && fread(user, 1, (size_t)h.user_bytes, fp) != (size_t)h.user_bytes) {
        set_error("acfd_checkpoint_load: %s is truncated", path);
        st = ACFD_ERR_IO;
    }
    std::vector<acfd_node_t> nodes;
    if (st == ACFD_OK) {
        nodes.resize((size_t)h.count);
        if (fread(nodes.data(), sizeof(acfd_node_t), nodes.size(), fp) != nodes.size()) {
            set_error("acfd_checkpoint_load: %s is truncated", path);
            st = ACFD_ERR_IO;
        }
    }
    fclose(fp);
    if (st != ACFD_OK) return st;
    return acfd_sync_to_device(cs, nodes.data(), ACFD_SYNC_ALL);
}

int acfd_integrate_surface_force(acfd_case_t *cs, double *force)
{
    TRY(check_case(cs));
    if (!force) {
        set_error("acfd_integrate_surface_force: null output");
        return ACFD_ERR_ARG;
    }
    return ib_surface_force(cs->ib, cs->grid, cs->mp, cs->part, level(cs, ACFD_TO), cs->flags, force, cs->stream);
}

int acfd_collision_scan(acfd_case_t *cs, int *counts, int *gid, int *N)
{
    TRY(check_case(cs));
    if (!counts || !gid || !N) {
        set_error("acfd_collision_scan: null output");
        return ACFD_ERR_ARG;
    }
    return ib_collision_scan(cs->ib, cs->grid, cs->mp, cs->part, cs->flags, counts, gid, N, cs->stream);
}

static ModelParams params_of(const acfd_model_t *model)
{
    ModelParams m;
    memset(&m, 0, sizeof(m));
    m.gamma = model->gamma;
    m.gasR = model->gasR;
    m.cv = model->cv;
    m.refMu = model->refMu;
    m.refT = model->refT;
    m.sScheme = model->sScheme;
    m.jacobMean = model->jacobMean;
    m.fluxSplit = model->fluxSplit;
    m.multidim = model->multidim;
    m.ibmLayer = model->ibmLayer;
    return m;
}

int acfd_weno_batch(int scheme, int mode, const double *F, double *Fhat, int count)
{
    if (!F || !Fhat || count < 0 || (scheme != 0 && scheme != 1)) {
        set_error("acfd_weno_batch: bad arguments");
        return ACFD_ERR_ARG;
    }
    double *dF = nullptr, *dO = nullptr;
    ACFD_CUDA(cudaMalloc(&dF, sizeof(double) * 25 * (size_t)(count ? count : 1)));
    cudaError_t e = cudaMalloc(&dO, sizeof(double) * 5 * (size_t)(count ? count : 1));
    if (e != cudaSuccess) {
        cudaFree(dF);
        return cuda_status(e, "cudaMalloc");
    }
    int st = ACFD_OK;
    if ((e = cudaMemcpy(dF, F, sizeof(double) * 25 * (size_t)count, cudaMemcpyHostToDevice)) != cudaSuccess) {
        st = cuda_status(e, "cudaMemcpy");
    }
    if (st == ACFD_OK) {
        st = (mode == ACFD_FP64_EXACT) ? launch_weno_batch_exact(scheme, dF, dO, count, 0)
             : (mode == ACFD_FP64)     ? launch_weno_batch_fast(scheme, dF, dO, count, 0)
                                       : launch_weno_batch_fp32(scheme, dF, dO, count, 0);
    }
    if (st == ACFD_OK && (e = cudaMemcpy(Fhat, dO, sizeof(double) * 5 * (size_t)count, cudaMemcpyDeviceToHost)) != cudaSuccess) {
        st = cuda_status(e, "cudaMemcpy");
    }
    cudaFree(dF);
    cudaFree(dO);
    return st;
}

int acfd_fhat_batch(const acfd_model_t *model, int s, int mode, const double *Ust, double *Fhat, int count)
{
    if (!model || !Ust || !Fhat || count < 0 || s < 0 || s > 2) {
        set_error("acfd_fhat_batch: bad arguments");
        return ACFD_ERR_ARG;
    }
    const ModelParams m = params_of(model);
    double *dU = nullptr, *dO = nullptr;
    ACFD_CUDA(cudaMalloc(&dU, sizeof(double) * 30 * (size_t)(count ? count : 1)));
    cudaError_t e = cudaMalloc(&dO, sizeof(double) * 5 * (size_t)(count ? count : 1));
    if (e != cudaSuccess) {
        cudaFree(dU);
        return cuda_status(e, "cudaMalloc");
    }
    int st = ACFD_OK;
    if ((e = cudaMemcpy(dU, Ust, sizeof(double) * 30 * (size_t)count, cudaMemcpyHostToDevice)) != cudaSuccess) {
        st = cuda_status(e, "cudaMemcpy");
    }
    if (st == ACFD_OK) {
        st = (mode == ACFD_FP64_EXACT) ? launch_fhat_batch_exact(m, s, dU, dO, count, 0)
             : (mode == ACFD_FP64)     ? launch_fhat_batch_fast(m, s, dU, dO, count, 0)
                                       : launch_fhat_batch_fp32(m, s, dU, dO, count, 0);
    }
    if (st == ACFD_OK && (e = cudaMemcpy(Fhat, dO, sizeof(double) * 5 * (size_t)count, cudaMemcpyDeviceToHost)) != cudaSuccess) {
        st = cuda_status(e, "cudaMemcpy");
    }
    cudaFree(dU);
    cudaFree(dO);
    return st;
}

}  // extern "C"

// ===========================================================================
// Batch of independent cases: one persistent stage launch per RK stage for
// all cases (ComputeTimeStep, EvolveFluidDynamics of every case, advanced
// together; no reference counterpart for the batching itself)
// ===========================================================================
struct acfd_batch {
    std::vector<acfd_case *> cases;
    int mode = ACFD_FP32_BULK;
    int tScheme = 1;
    cudaStream_t stream = nullptr;
    bool own_stream = true;
    int sms = 148;
    int blocks = 0;                        // persistent blocks of the stage launch
    BatchCase *d_cases = nullptr;          // [ncase]
    CUtensorMap *d_maps = nullptr;         // [ncase][3] brick maps (viscous geometry, variant 0)
    long long *d_prefix = nullptr;         // [3][ncase + 1] prefix sums of the tiles per sweep axis
    double *d_dts = nullptr;               // [ncase] step dt of each case
    double *d_cfl = nullptr;               // [ncase] CFL number of each case
    double *d_mesh = nullptr;              // [ncase][3] mesh sizes
    const double **d_vmax = nullptr;       // [ncase] the cases' CFL maxima (device pointers)
    unsigned long long *d_counter = nullptr;  // work counters, one per stage launch of a step
    int *d_status = nullptr;
    BatchLevel *d_levels = nullptr;        // [ncase]
    int4 *d_pairs = nullptr;               // ghost gather of the copy-only cases
    long long npairs = 0;
    std::vector<int> ordered_fill;         // cases whose ghosts need the ordered fill
    // plane-march stage kernels (all cases viscous or all inviscid, plane maps present)
    bool plane_ok = false, plane = false, visc = false;
    BatchPlane *d_planes = nullptr;        // [ncase][3]
    CUtensorMap *d_pmaps = nullptr;        // [ncase][3]
    long long *d_pprefix = nullptr;        // [3][ncase + 1] prefix sums of the plane blocks per sweep axis
    long long pblocks[3] = {0, 0, 0};
    int pthreads[3] = {0, 0, 0}, psmem[3] = {0, 0, 0};
    // persistent step (plane march, copy-only ghost fills): all stages of a
    // time step of every case in one launch (stage_plane_persistent)
    bool persist_ok = false, persist = false;
    int persist_blocks = 0, persist_threads = 0, persist_smem = 0;
    unsigned long long *d_queue = nullptr;
    unsigned *d_done = nullptr, *d_filled = nullptr;  // [kMaxStepStages][ncase]
    int *d_abort = nullptr;
    long long *d_pair_off = nullptr;                  // [ncase + 1]
    long long *d_fill_pre = nullptr;                  // [ncase + 1] first fill item of each case
    long long nfill = 0;                              // fill items of one stage
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_mode = -1;
    long long graph_kernels = 0;
    long long launches = 0;
};

namespace {

constexpr int kBatchStagesPerStep = 18;  // 6 directional half steps x 3 RK stages (3D, RK3)

void batch_release_graph(acfd_batch *b)
{
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
    b->graph_mode = -1;
}

// one time step of every case: CFL maxima, dt on the device, sensor flags
// (hybrid), then the Strang schedule Z,Y,X,X,Y,Z of RK stages, each one
// persistent launch over all cases followed by the ghost fill
int batch_step(acfd_batch *b)
{
    const int ncase = (int)b->cases.size();
    for (acfd_case *cs : b->cases) {
        TRY(launch_cfl(cs->grid, cs->mp, cs->U, cs->flags, cs->cfl_part, cs->cfl_out, b->stream));
        ++b->launches;
    }
    TRY(launch_batch_dt(b->d_vmax, b->d_mesh, b->d_cfl, b->d_dts, ncase, b->stream));
    ++b->launches;
    const bool hybrid = (b->mode == ACFD_FP32_HYBRID);
    if (hybrid) {
        for (acfd_case *cs : b->cases) {
            TRY(launch_sensor_flags(cs->grid, cs->mp, cs->U, cs->flags, cs->sensor_params, cs->sensor_logit,
                                    cs->sensor_rp, cs->sensor_flags, nullptr, b->stream));
            b->launches += 2;
        }
    }
    static const int order[6] = {2, 1, 0, 0, 1, 2};
    struct Coef {
        double a, c;
        int to, tn, tm;
    };
    static const Coef rk3[3] = {{0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN},
                                {3.0 / 4.0, 1.0 / 4.0, ACFD_TO, ACFD_TN, ACFD_TM},
                                {1.0 / 3.0, 2.0 / 3.0, ACFD_TO, ACFD_TM, ACFD_TO}};
    static const Coef rk2[2] = {{0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN}, {1.0 / 2.0, 1.0 / 2.0, ACFD_TO, ACFD_TN, ACFD_TO}};
    const Coef *rk = b->tScheme == 1 ? rk3 : rk2;
    const int nstage = b->tScheme == 1 ? 3 : 2;
    if (b->persist && b->plane) {
        // one persistent launch per directional half step: its RK stages and
        // ghost fills of every case, linked by per-case counters (indexed by
        // the step-wide stage, cleared once per step)
        const size_t nflag = (size_t)kMaxStepStages * ncase;
        ACFD_CUDA(cudaMemsetAsync(b->d_done, 0, sizeof(unsigned) * nflag, b->stream));
        ACFD_CUDA(cudaMemsetAsync(b->d_filled, 0, sizeof(unsigned) * nflag, b->stream));
        ACFD_CUDA(cudaMemsetAsync(b->d_abort, 0, sizeof(int), b->stream));
        for (int h = 0; h < 6; ++h) {
            const int s = order[h];
            PersistStep ps;
            memset(&ps, 0, sizeof(ps));
            ps.nk = nstage;
            ps.k0 = h * nstage;
            ps.kbase[0] = 0;
            for (int a = 0; a < 3; ++a) {
                ps.ntile[a] = b->pblocks[a];
            }
            ps.nfill = b->nfill;
            for (int q = 0; q < nstage; ++q) {
                ps.s_of[q] = s;
                ps.sc[q].coeA = rk[q].a;
                ps.sc[q].coeB = rk[q].c;
                ps.sc[q].dt_scale = 0.5;
                ps.sc[q].to = rk[q].to;
                ps.sc[q].tn = rk[q].tn;
                ps.sc[q].tm = rk[q].tm;
                ps.kbase[q + 1] = ps.kbase[q] + b->pblocks[s] + b->nfill;
            }
            ACFD_CUDA(cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned long long), b->stream));
            TRY(launch_stage_plane_persistent(b->d_cases, b->d_planes, b->d_pmaps, b->d_pprefix, ncase, ps,
                                              b->d_dts, b->d_levels, b->d_pairs, b->d_pair_off, b->d_fill_pre,
                                              b->d_queue, b->d_done, b->d_filled, b->d_abort, b->d_status, b->visc,
                                              hybrid, b->persist_blocks, b->persist_threads, b->persist_smem,
                                              b->stream));
            ++b->launches;
        }
        return ACFD_OK;
    }
    ACFD_CUDA(cudaMemsetAsync(b->d_counter, 0, sizeof(unsigned long long) * kBatchStagesPerStep, b->stream));
    int launch = 0;
    for (int h = 0; h < 6; ++h) {
        const int s = order[h];
        for (int q = 0; q < nstage; ++q) {
            StageCoefs sc;
            sc.coeA = rk[q].a;
            sc.coeB = rk[q].c;
            sc.dt_scale = 0.5;
            sc.to = rk[q].to;
            sc.tn = rk[q].tn;
            sc.tm = rk[q].tm;
            if (b->plane) {
                TRY(launch_stage_plane_batch(b->d_cases, b->d_planes, b->d_pmaps, b->d_pprefix + (long long)s * (ncase + 1),
                                             b->pblocks[s], ncase, sc, b->d_dts, b->d_status, s, b->visc, hybrid,
                                             b->pthreads[s], b->psmem[s], b->stream));
            } else {
                TRY(launch_stage_batch(b->d_cases, b->d_maps, b->d_prefix + (long long)s * (ncase + 1), ncase, sc,
                                       b->d_dts, b->d_counter + launch, b->d_status, b->blocks, s, hybrid,
                                       b->stream));
            }
            ++launch;
            ++b->launches;
            if (b->npairs > 0) {
                TRY(launch_batch_gather(b->d_levels, b->d_pairs, b->npairs, sc.tm, b->stream));
                ++b->launches;
            }
            for (int c : b->ordered_fill) {
                acfd_case *cs = b->cases[c];
                const cudaStream_t keep = cs->stream;
                cs->stream = b->stream;
                const long long l0 = cs->launches;
                const int st = treat_boundary(cs, sc.tm);
                b->launches += cs->launches - l0;
                cs->stream = keep;
                TRY(st);
            }
        }
    }
    return ACFD_OK;
}

int batch_check(const acfd_batch *b)
{
    if (!b) {
        set_error("null batch handle");
        return ACFD_ERR_ARG;
    }
    return ACFD_OK;
}

}  // namespace

extern "C" {

int acfd_batch_init(int ncase, const acfd_partition_t *parts, const acfd_model_t *models, acfd_batch_t **out)
{
    if (ncase < 1 || !parts || !models || !out) {
        set_error("acfd_batch_init: bad arguments");
        return ACFD_ERR_ARG;
    }
    *out = nullptr;
    for (int c = 0; c < ncase; ++c) {
        const acfd_model_t &m = models[c];
        const acfd_partition_t &p = parts[c];
        if (m.sScheme != 1 || m.multidim != 0 || m.sState != 0 || p.collapse != 0 || m.tScheme != models[0].tScheme) {
            set_error("acfd_batch_init: case %d: the batch advances 3D cases with WENO5, the split scheme, no "
                      "gravity and one common RK scheme", c);
            return ACFD_ERR_ARG;
        }
    }
    acfd_batch *b = new acfd_batch();
    b->tScheme = models[0].tScheme;
    int st = ACFD_OK;
    cudaError_t e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess || (e = cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess) {
        st = cuda_status(e, "acfd_batch_init");
        delete b;
        return st;
    }
    for (int c = 0; c < ncase && st == ACFD_OK; ++c) {
        acfd_case *cs = nullptr;
        st = acfd_init(&parts[c], &models[c], &cs);
        if (st == ACFD_OK) {
            // the batch kernels sweep x directly: a batch case holds no
            // transposed levels
            release_xt(cs);
            b->cases.push_back(cs);
        }
    }
    std::vector<BatchCase> hc(ncase);
    std::vector<CUtensorMap> hm((size_t)ncase * 3);
    std::vector<long long> prefix((size_t)3 * (ncase + 1), 0);
    std::vector<double> mesh((size_t)ncase * 3);
    std::vector<const double *> vmax(ncase);
    std::vector<BatchLevel> lv(ncase);
    std::vector<int4> pairs;
    for (int c = 0; c < ncase && st == ACFD_OK; ++c) {
        acfd_case *cs = b->cases[c];
        BatchCase &C = hc[c];
        C.g = cs->grid;
        C.mp = cs->mp;
        C.U = cs->U;
        C.did = cs->flags;
        C.flags = nullptr;
        const int L[3] = {cs->grid.hi[0] - cs->grid.lo[0], cs->grid.hi[1] - cs->grid.lo[1],
                          cs->grid.hi[2] - cs->grid.lo[2]};
        for (int s = 0; s < 3 && st == ACFD_OK; ++s) {
            int box[3], step[3];
            brick_box(s, true, 0, box);
            brick_step(s, true, 0, step);
            for (int a = 0; a < 3; ++a) {
                C.tiles[s][a] = (L[a] + step[a] - 1) / step[a];
            }
            st = encode_box_map(cs->grid, cs->U, box, &hm[(size_t)c * 3 + s]);
            prefix[(size_t)s * (ncase + 1) + c + 1] =
                prefix[(size_t)s * (ncase + 1) + c] + (long long)C.tiles[s][0] * C.tiles[s][1] * C.tiles[s][2];
        }
        for (int s = 0; s < 3; ++s) {
            mesh[(size_t)c * 3 + s] = cs->part.d[s];
        }
        vmax[c] = cs->cfl_out;
        lv[c].U = cs->U;
        lv[c].nn = cs->grid.nn;
        if (cs->bc_gather && cs->bc_nprog == 0) {
            std::vector<int2> hp(cs->bc_npairs);
            if ((e = cudaMemcpy(hp.data(), cs->bc_pairs, sizeof(int2) * hp.size(), cudaMemcpyDeviceToHost)) !=
                cudaSuccess) {
                st = cuda_status(e, "acfd_batch_init");
            }
            for (const int2 &q : hp) {
                pairs.push_back(make_int4(c, q.x, q.y, 0));
            }
        } else {
            b->ordered_fill.push_back(c);
        }
    }
    // persistent stage launch: two resident blocks of the viscous bricks per SM
    b->blocks = 2 * b->sms;
    // plane-march launches: one launch per stage over the plane blocks of all cases
    std::vector<BatchPlane> hp((size_t)ncase * 3);
    std::vector<CUtensorMap> hpm((size_t)ncase * 3);
    std::vector<long long> pprefix((size_t)3 * (ncase + 1), 0);
    if (st == ACFD_OK) {
        b->visc = viscous(b->cases[0]);
        b->plane_ok = true;
        for (int c = 0; c < ncase && b->plane_ok; ++c) {
            acfd_case *cs = b->cases[c];
            if (!cs->pmaps_ok || viscous(cs) != b->visc) {
                b->plane_ok = false;
                break;
            }
            for (int s = 0; s < 3; ++s) {
                BatchPlane &P = hp[(size_t)c * 3 + s];
                P.pt = plane_tile(cs->grid, s, b->visc, 1, b->sms);
                P.gk = cs->grid;
                const long long sy = (long long)cs->grid.pitch, sz = (long long)cs->grid.pitch * cs->grid.n[1];
                if (s == 1) {
                    P.pt.swap = 0;
                    P.pt.st = sy;
                    P.pt.rs = sz;
                } else if (s == 2) {
                    // the Z sweep as a Y sweep of the grid with axes 1 and 2 exchanged
                    P.pt.swap = 1;
                    P.pt.st = sz;
                    P.pt.rs = sy;
                    std::swap(P.gk.n[1], P.gk.n[2]);
                    std::swap(P.gk.lo[1], P.gk.lo[2]);
                    std::swap(P.gk.hi[1], P.gk.hi[2]);
                    std::swap(P.gk.dd[1], P.gk.dd[2]);
                }
                if (P.pt.BXp != cs->pbox[s][0] || P.pt.BC != cs->pbox[s][1]) {
                    b->plane_ok = false;
                }
                hpm[(size_t)c * 3 + s] = cs->pmaps[s];
                const long long nb = P.pt.nblk;
                pprefix[(size_t)s * (ncase + 1) + c + 1] = pprefix[(size_t)s * (ncase + 1) + c] + nb;
                b->pthreads[s] = std::max(b->pthreads[s], (P.pt.ncw + 1) * 32);
                b->psmem[s] = std::max(b->psmem[s], plane_smem_bytes(P.pt, s));
            }
        }
        for (int s = 0; s < 3; ++s) {
            b->pblocks[s] = pprefix[(size_t)s * (ncase + 1) + ncase];
        }
        if (b->plane_ok) {
            if ((e = cudaMalloc(&b->d_planes, sizeof(BatchPlane) * hp.size())) != cudaSuccess ||
                (e = cudaMalloc(&b->d_pmaps, sizeof(CUtensorMap) * hpm.size())) != cudaSuccess ||
                (e = cudaMalloc(&b->d_pprefix, sizeof(long long) * pprefix.size())) != cudaSuccess ||
                (e = cudaMemcpy(b->d_planes, hp.data(), sizeof(BatchPlane) * hp.size(), cudaMemcpyHostToDevice)) !=
                    cudaSuccess ||
                (e = cudaMemcpy(b->d_pmaps, hpm.data(), sizeof(CUtensorMap) * hpm.size(), cudaMemcpyHostToDevice)) !=
                    cudaSuccess ||
                (e = cudaMemcpy(b->d_pprefix, pprefix.data(), sizeof(long long) * pprefix.size(),
                                cudaMemcpyHostToDevice)) != cudaSuccess) {
                st = cuda_status(e, "acfd_batch_init (plane maps)");
            }
        }
        b->plane = b->plane_ok;
    }
    const size_t nbytes[] = {sizeof(BatchCase) * ncase, sizeof(CUtensorMap) * 3 * ncase,
                             sizeof(long long) * prefix.size(), sizeof(double) * ncase, sizeof(double) * ncase,
                             sizeof(double) * mesh.size(), sizeof(double *) * ncase,
                             sizeof(unsigned long long) * kBatchStagesPerStep, sizeof(int),
                             sizeof(BatchLevel) * ncase, sizeof(int4) * (pairs.size() ? pairs.size() : 1)};
    void **ptrs[] = {(void **)&b->d_cases, (void **)&b->d_maps, (void **)&b->d_prefix, (void **)&b->d_dts,
                     (void **)&b->d_cfl, (void **)&b->d_mesh, (void **)&b->d_vmax, (void **)&b->d_counter,
                     (void **)&b->d_status, (void **)&b->d_levels, (void **)&b->d_pairs};
    for (int q = 0; q < 11 && st == ACFD_OK; ++q) {
        if ((e = cudaMalloc(ptrs[q], nbytes[q])) != cudaSuccess) {
            st = cuda_status(e, "acfd_batch_init allocation");
        }
    }
    if (st == ACFD_OK) {
        b->npairs = (long long)pairs.size();
        const void *src[] = {hc.data(), hm.data(), prefix.data(), nullptr, nullptr, mesh.data(), vmax.data(),
                             nullptr, nullptr, lv.data(), pairs.data()};
        for (int q = 0; q < 11 && st == ACFD_OK; ++q) {
            if (src[q] && nbytes[q] && (q != 10 || b->npairs > 0)) {
                if ((e = cudaMemcpy(*ptrs[q], src[q], nbytes[q], cudaMemcpyHostToDevice)) != cudaSuccess) {
                    st = cuda_status(e, "acfd_batch_init copy");
                }
            }
        }
        if (st == ACFD_OK && (e = cudaMemset(b->d_status, 0, sizeof(int))) != cudaSuccess) {
            st = cuda_status(e, "acfd_batch_init");
        }
    }
    // persistent step: plane maps for every case and copy-only ghost fills
    if (st == ACFD_OK && b->plane_ok && b->ordered_fill.empty()) {
        std::vector<long long> off((size_t)ncase + 1, 0);
        for (const int4 &q : pairs) {
            ++off[(size_t)q.x + 1];
        }
        for (int c = 0; c < ncase; ++c) {
            off[(size_t)c + 1] += off[(size_t)c];
        }
        // the copy pairs of a case's ghost fill in items of kFillChunk pairs
        std::vector<long long> fpre((size_t)ncase + 1, 0);
        for (int c = 0; c < ncase; ++c) {
            const long long np = off[(size_t)c + 1] - off[(size_t)c];
            fpre[(size_t)c + 1] = fpre[(size_t)c] + (np + kFillChunk - 1) / kFillChunk;
        }
        b->persist_threads = std::max(b->pthreads[0], std::max(b->pthreads[1], b->pthreads[2]));
        b->persist_smem = std::max(b->psmem[0], std::max(b->psmem[1], b->psmem[2]));
        int bps = 0;
        const size_t nflag = (size_t)kMaxStepStages * ncase;
        if (plane_persistent_occupancy(b->visc, true, b->persist_threads, b->persist_smem, &bps) == ACFD_OK &&
            bps >= 1 && (e = cudaMalloc(&b->d_queue, sizeof(unsigned long long))) == cudaSuccess &&
            (e = cudaMalloc(&b->d_done, sizeof(unsigned) * nflag)) == cudaSuccess &&
            (e = cudaMalloc(&b->d_filled, sizeof(unsigned) * nflag)) == cudaSuccess &&
            (e = cudaMalloc(&b->d_abort, sizeof(int))) == cudaSuccess &&
            (e = cudaMalloc(&b->d_pair_off, sizeof(long long) * off.size())) == cudaSuccess &&
            (e = cudaMemcpy(b->d_pair_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice)) ==
                cudaSuccess &&
            (e = cudaMalloc(&b->d_fill_pre, sizeof(long long) * fpre.size())) == cudaSuccess &&
            (e = cudaMemcpy(b->d_fill_pre, fpre.data(), sizeof(long long) * fpre.size(), cudaMemcpyHostToDevice)) ==
                cudaSuccess) {
            b->nfill = fpre[(size_t)ncase];
            b->persist_blocks = bps * b->sms;
            b->persist_ok = true;
            // available (acfd_batch_set_kernel), not the default: measured
            // 811 against 878 Mcell-steps/s for one launch per RK stage on the
            // 48-case batch
            b->persist = false;
        } else {
            cudaGetLastError();  // keep the per-stage launches
        }
    }
    if (st != ACFD_OK) {
        acfd_batch_finalize(b);
        return st;
    }
    for (acfd_case *cs : b->cases) {
        cs->mode = ACFD_FP32_BULK;
    }
    *out = b;
    return ACFD_OK;
}

int acfd_batch_finalize(acfd_batch_t *b)
{
    if (!b) {
        return ACFD_OK;
    }
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_release_graph(b);
    for (acfd_case *cs : b->cases) {
        acfd_finalize(cs);
    }
    cudaFree(b->d_cases);
    cudaFree(b->d_maps);
    cudaFree(b->d_prefix);
    cudaFree(b->d_dts);
    cudaFree(b->d_cfl);
    cudaFree(b->d_mesh);
    cudaFree(b->d_vmax);
    cudaFree(b->d_counter);
    cudaFree(b->d_status);
    cudaFree(b->d_levels);
    cudaFree(b->d_pairs);
    cudaFree(b->d_planes);
    cudaFree(b->d_pmaps);
    cudaFree(b->d_pprefix);
    cudaFree(b->d_queue);
    cudaFree(b->d_done);
    cudaFree(b->d_filled);
    cudaFree(b->d_abort);
    cudaFree(b->d_pair_off);
    cudaFree(b->d_fill_pre);
    if (b->stream && b->own_stream) cudaStreamDestroy(b->stream);
    delete b;
    return ACFD_OK;
}

int acfd_batch_case(acfd_batch_t *b, int c, acfd_case_t **cs)
{
    TRY(batch_check(b));
    if (c < 0 || c >= (int)b->cases.size() || !cs) {
        set_error("acfd_batch_case: case %d of %d", c, (int)b->cases.size());
        return ACFD_ERR_ARG;
    }
    *cs = b->cases[c];
    return ACFD_OK;
}

int acfd_batch_set_precision(acfd_batch_t *b, int mode)
{
    TRY(batch_check(b));
    if (mode != ACFD_FP32_BULK && mode != ACFD_FP32_HYBRID) {
        set_error("acfd_batch_set_precision: the batch runs ACFD_FP32_BULK or ACFD_FP32_HYBRID, not %d", mode);
        return ACFD_ERR_ARG;
    }
    std::vector<BatchCase> hc(b->cases.size());
    ACFD_CUDA(cudaMemcpy(hc.data(), b->d_cases, sizeof(BatchCase) * hc.size(), cudaMemcpyDeviceToHost));
    for (size_t c = 0; c < b->cases.size(); ++c) {
        acfd_case *cs = b->cases[c];
        if (mode == ACFD_FP32_HYBRID && !cs->sensor_ok) {
            set_error("acfd_batch_set_precision: case %d has no sensor (acfd_batch_sensor_load)", (int)c);
            return ACFD_ERR_STATE;
        }
        cs->mode = mode;
        hc[c].flags = (mode == ACFD_FP32_HYBRID) ? cs->sensor_flags : nullptr;
    }
    ACFD_CUDA(cudaMemcpy(b->d_cases, hc.data(), sizeof(BatchCase) * hc.size(), cudaMemcpyHostToDevice));
    if (mode != b->mode) {
        batch_release_graph(b);
    }
    b->mode = mode;
    return ACFD_OK;
}

int acfd_batch_sensor_load(acfd_batch_t *b, const float *params, float threshold)
{
    TRY(batch_check(b));
    for (acfd_case *cs : b->cases) {
        TRY(acfd_sensor_load(cs, params, threshold));
    }
    batch_release_graph(b);
    return ACFD_OK;
}

int acfd_batch_advance(acfd_batch_t *b, const double *cfl, int steps, double *dts)
{
    TRY(batch_check(b));
    const int ncase = (int)b->cases.size();
    if (!cfl || steps < 0) {
        set_error("acfd_batch_advance: bad arguments");
        return ACFD_ERR_ARG;
    }
    ACFD_CUDA(cudaMemcpyAsync(b->d_cfl, cfl, sizeof(double) * ncase, cudaMemcpyHostToDevice, b->stream));
    if (!b->exec || b->graph_mode != b->mode) {
        batch_release_graph(b);
        ACFD_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const long long before = b->launches;
        int st = batch_step(b);
        b->graph_kernels = b->launches - before;
        b->launches = before;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (st != ACFD_OK) {
            if (graph) cudaGraphDestroy(graph);
            return st;
        }
        if (e != cudaSuccess) {
            return cuda_status(e, "cudaStreamEndCapture");
        }
        b->graph = graph;
        ACFD_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
        b->graph_mode = b->mode;
    }
    for (int k = 0; k < steps; ++k) {
        ACFD_CUDA(cudaGraphLaunch(b->exec, b->stream));
        b->launches += b->graph_kernels;
        if (dts) {
            ACFD_CUDA(cudaMemcpyAsync(dts + (size_t)k * ncase, b->d_dts, sizeof(double) * ncase,
                                      cudaMemcpyDeviceToHost, b->stream));
        }
    }
    ACFD_CUDA(cudaStreamSynchronize(b->stream));
    int status = 0;
    ACFD_CUDA(cudaMemcpy(&status, b->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (status != 0) {
        cudaMemset(b->d_status, 0, sizeof(int));
        set_error("batch stage: device wait gave up (code %d)", status);
        return ACFD_ERR_DEVICE;
    }
    for (acfd_case *cs : b->cases) {
        TRY(check_device_status(cs));
    }
    return ACFD_OK;
}

int acfd_batch_set_kernel(acfd_batch_t *b, int kernel)
{
    TRY(batch_check(b));
    if (kernel != ACFD_BATCH_BRICK && kernel != ACFD_BATCH_PLANE && kernel != ACFD_BATCH_PERSISTENT) {
        set_error("acfd_batch_set_kernel: unknown kernel %d", kernel);
        return ACFD_ERR_ARG;
    }
    if (kernel != ACFD_BATCH_BRICK && !b->plane_ok) {
        set_error("acfd_batch_set_kernel: the plane-march batch needs all cases viscous or all inviscid");
        return ACFD_ERR_STATE;
    }
    if (kernel == ACFD_BATCH_PERSISTENT && !b->persist_ok) {
        set_error("acfd_batch_set_kernel: the persistent step needs copy-only ghost fills in every case");
        return ACFD_ERR_STATE;
    }
    b->plane = (kernel != ACFD_BATCH_BRICK);
    b->persist = (kernel == ACFD_BATCH_PERSISTENT);
    batch_release_graph(b);
    return ACFD_OK;
}

int acfd_batch_set_stream(acfd_batch_t *b, void *stream)
{
    TRY(batch_check(b));
    if (!stream) {
        set_error("acfd_batch_set_stream: null stream");
        return ACFD_ERR_ARG;
    }
    ACFD_CUDA(cudaStreamSynchronize(b->stream));
    ACFD_CUDA(cudaStreamDestroy(b->stream));
    b->stream = static_cast<cudaStream_t>(stream);
    b->own_stream = false;
    batch_release_graph(b);
    return ACFD_OK;
}

int acfd_batch_stats(acfd_batch_t *b, long long *launches)
{
    TRY(batch_check(b));
    if (launches) *launches = b->launches;
    return ACFD_OK;
}

}  // extern "C"

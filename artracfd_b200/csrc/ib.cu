// Immersed boundaries on the device: node mapping (ComputeGeometricField,
// immersed_boundary.c:65-264, with the point-in-polyhedron test of
// computational_geometry.c:463-783), the ghost-node reconstruction
// (TreatImmersedBoundary, immersed_boundary.c:270-487) and the node scans of
// the rigid-body step (IntegrateSurfaceForce and the contact search of
// ApplyCollision, solid_dynamics.c:51-171, 213-357).
//
// Compiled with --fmad=false and written in the reference's evaluation
// order: node flags (did, fid, lid, gst), image-point node indices and IDW
// stencils are bit-exact, ghost values bitwise up to the order-free parts.
//
// Parallel structure:
//  * domain mapping: one launch per body in body order (first body wins, as
//    the reference's body loop); a block stages the body's facets
//    (v0, e01, e02 per facet) in shared memory and a warp scans them for a
//    node, 32 facets at a time;
//  * interfacial field: newly uncovered nodes are marked first, so that the
//    reconstruction reads only nodes that stay fluid (the reference's TYPEF
//    selection) and never a value written in the same pass;
//  * ghost layers: the ghost nodes of all bodies are listed once per
//    treatment, then one launch per layer (layer r reads fluid nodes or
//    layer r-1 only; bodies do not read each other) gives each listed node of
//    the layer a warp, whose lanes share the inverse-distance searches;
//  * rigid-body step: surface-force terms per ghost node of layer 2 with the
//    sums taken in the reference's node order by one warp per body, and the
//    contact scan of the collision step with atomics that keep the order in
//    which the reference's node loop meets each contact.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <vector>

#include "acfd_internal.cuh"
#include "flux_math.cuh"

namespace acfd {

struct DevBody {
    int faceN, edgeN, vertN, state;
    double r, O[3], V[3], W[3], T, cf, area;
    double box[3][2];
    const int *f;
    const double *Nf;
    const int *e;
    const double *Ne;
    const double *v;
    const double *Nv;
    const double *tri;  // faceN x 9: v0, e01, e02
};

// node boxes of up to 8 bodies (body0 ..), flattened in (k, j, i) order
struct BoxList {
    int lo[8][3];
    int ext[8][3];
    long long start[9];
    int body0;
    int nb;
};

// box extremes of a block of vertices: (min x, max x, min y, ...) with the
// index of the vertex that gave each
struct BoxPart {
    double v[6];
    int i[6];
};
constexpr int kMotionBlocks = 148;

struct IbState {
    std::vector<DevBody> host;
    DevBody *dev = nullptr;
    std::vector<void *> buffers;
    unsigned char *joined = nullptr;
    long long joined_n = 0;
    int *status = nullptr;  // device error word
    int count = 0;
    int4 *ghosts = nullptr;  // ghost list of a boundary treatment
    int *nghost = nullptr;
    int ghost_cap = 0;
    BoxList *groups = nullptr;  // device: node boxes of the bodies, 8 per entry
    int ngroups = 0;
    // surface-force integration and collision scan (allocated on first use)
    double *sf_terms = nullptr;        // [box node][10]: Fp, Fv, Tt, p of ghost nodes of layer 2
    unsigned char *sf_valid = nullptr; // [box node]: 1 = ghost node of layer 2 of the box's body
    long long sf_cap = 0;
    long long *sf_off = nullptr;       // [totN + 1] box offsets
    int *sf_lid = nullptr;             // [totN] interfacial nodes of layer 2
    double *sf_force = nullptr;        // [totN][9]
    unsigned long long *col_key = nullptr;  // [totN][totN] first meeting (node order x path length + path index)
    int *col_N = nullptr;              // [totN][totN][3] summed path offsets
    int col_n = 0;
    BoxPart *motion_part = nullptr;  // [kMotionBlocks] box extremes of a surface motion
    // the ghost lists hold the ghost nodes of the current flags: rebuilt by
    // every writer of the flags (the geometric field, an upload of node
    // records), so that a boundary treatment, captured step graphs included,
    // only reads them
    bool lists_valid = false;
};

namespace {

constexpr int kIbR = 2;  // IDW search radius of the reconstruction (immersed_boundary.c:27)
constexpr int kTypeD = -1, kTypeF = -2;

struct IbGrid {
    Grid g;
    int ng[3];
    double dmin[3];  // domain minimum
    double d[3];
    double tinyL;
    int gl;
    int ibmLayer;
    int pathSep[4];
    int path[30][3];
};

__device__ __forceinline__ long long node_of(const Grid &g, int i, int j, int k)
{
    return ((long long)k * g.n[1] + j) * g.pitch + i;
}

__host__ __device__ __forceinline__ double dot3(const double *a, const double *b)
{
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ double dist2(const double *a, const double *b)
{
    const double v[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    return dot3(v, v);
}

__device__ __forceinline__ bool in_pin(const Grid &g, int k, int j, int i)
{
    return (g.lo[2] <= k) && (g.hi[2] > k) && (g.lo[1] <= j) && (g.hi[1] > j) && (g.lo[0] <= i) && (g.hi[0] > i);
}

__device__ __forceinline__ int map_node(double s, double smin, double dds, int ng)
{
    return (int)((s - smin) * dds + 0.5) + ng;
}

__device__ __forceinline__ double map_point(int n, double smin, double ds, int ng)
{
    return smin + (n - ng) * ds;
}

__device__ __forceinline__ void node_point(const IbGrid &G, int k, int j, int i, double p[3])
{
    p[0] = map_point(i, G.dmin[0], G.d[0], G.ng[0]);
    p[1] = map_point(j, G.dmin[1], G.d[1], G.ng[1]);
    p[2] = map_point(k, G.dmin[2], G.d[2], G.ng[2]);
}

__host__ __device__ inline int confine(int n, int lo, int hi)
{
    const int a = (lo > n) ? lo : n;
    return (hi - 1 < a) ? hi - 1 : a;
}

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

// Eberly's point-triangle distance (computational_geometry.c:511-688)
__device__ double point_triangle(const double p[3], const double v0[3], const double e01[3], const double e02[3],
                                 double para[3])
{
    const double D[3] = {v0[0] - p[0], v0[1] - p[1], v0[2] - p[2]};
    const double a = dot3(e01, e01), b = dot3(e01, e02), c = dot3(e02, e02);
    const double d = dot3(e01, D), e = dot3(e02, D), f = dot3(D, D);
    const double det = a * c - b * b;
    double s = b * e - c * d;
    double t = b * d - a * e;
    double q;
    if (s + t <= det) {
        if (s < 0.0) {
            if (t < 0.0) {
                if (d < 0.0) {
                    t = 0.0;
                    if (-d >= a) { s = 1.0; q = a + 2.0 * d + f; }
                    else { s = -d / a; q = d * s + f; }
                } else {
                    s = 0.0;
                    if (e >= 0.0) { t = 0.0; q = f; }
                    else if (-e >= c) { t = 1.0; q = c + 2.0 * e + f; }
                    else { t = -e / c; q = e * t + f; }
                }
            } else {
                s = 0.0;
                if (e >= 0.0) { t = 0.0; q = f; }
                else if (-e >= c) { t = 1.0; q = c + 2.0 * e + f; }
                else { t = -e / c; q = e * t + f; }
            }
        } else if (t < 0.0) {
            t = 0.0;
            if (d >= 0.0) { s = 0.0; q = f; }
            else if (-d >= a) { s = 1.0; q = a + 2.0 * d + f; }
            else { s = -d / a; q = d * s + f; }
        } else {
            s = s / det;
            t = t / det;
            q = s * (a * s + b * t + 2.0 * d) + t * (b * s + c * t + 2.0 * e) + f;
        }
    } else if (s < 0.0) {
        const double t0 = b + d, t1 = c + e;
        if (t1 > t0) {
            const double num = t1 - t0, den = a - 2.0 * b + c;
            if (num >= den) { s = 1.0; t = 0.0; q = a + 2.0 * d + f; }
            else {
                s = num / den;
                t = 1.0 - s;
                q = s * (a * s + b * t + 2.0 * d) + t * (b * s + c * t + 2.0 * e) + f;
            }
        } else {
            s = 0.0;
            if (t1 <= 0.0) { t = 1.0; q = c + 2.0 * e + f; }
            else if (e >= 0.0) { t = 0.0; q = f; }
            else { t = -e / c; q = e * t + f; }
        }
    } else if (t < 0.0) {
        const double t0 = b + e, t1 = a + d;
        if (t1 > t0) {
            const double num = t1 - t0, den = a - 2.0 * b + c;
            if (num >= den) { t = 1.0; s = 0.0; q = c + 2.0 * e + f; }
            else {
                t = num / den;
                s = 1.0 - t;
                q = s * (a * s + b * t + 2.0 * d) + t * (b * s + c * t + 2.0 * e) + f;
            }
        } else {
            t = 0.0;
            if (t1 <= 0.0) { s = 1.0; q = a + 2.0 * d + f; }
            else if (d >= 0.0) { s = 0.0; q = f; }
            else { s = -d / a; q = d * s + f; }
        }
    } else {
        const double num = c + e - b - d;
        if (num <= 0.0) { s = 0.0; t = 1.0; q = c + 2.0 * e + f; }
        else {
            const double den = a - 2.0 * b + c;
            if (num >= den) { s = 1.0; t = 0.0; q = a + 2.0 * d + f; }
            else {
                s = num / den;
                t = 1.0 - s;
                q = s * (a * s + b * t + 2.0 * d) + t * (b * s + c * t + 2.0 * e) + f;
            }
        }
    }
    para[0] = 1.0 - s - t;
    para[1] = s;
    para[2] = t;
    return (0.0 > q) ? 0.0 : q;
}

__device__ int find_edge(const DevBody &B, int v0, int v1)
{
    const int hi = (v0 > v1) ? v0 : v1, lo = (v0 > v1) ? v1 : v0;
    int a = 0, b = B.edgeN - 1;
    while (a <= b) {
        const int m = (a + b) / 2;
        const int *e = B.e + 4 * m;
        if (hi == e[0] && lo == e[1]) {
            return m;
        }
        if ((hi > e[0]) || ((hi == e[0]) && (lo > e[1]))) {
            a = m + 1;
        } else {
            b = m - 1;
        }
    }
    return -1;
}

// closest point on facet fid and its pseudo-normal (computational_geometry.c:689-761)
__device__ bool closest_on_facet(const double p[3], int fid, const DevBody &B, double pi[3], double N[3])
{
    const double *T = B.tri + 9 * (long long)fid;
    const double v0[3] = {T[0], T[1], T[2]};
    const double e01[3] = {T[3], T[4], T[5]};
    const double e02[3] = {T[6], T[7], T[8]};
    const int *fv = B.f + 3 * (long long)fid;
    double para[3];
    point_triangle(p, v0, e01, e02, para);
    const double *nrm = nullptr;
    if (0.0 == para[1]) {
        if (0.0 == para[2]) {
            nrm = B.Nv + 3 * fv[0];
            for (int s = 0; s < 3; ++s) pi[s] = v0[s];
        } else if (1.0 == para[2]) {
            nrm = B.Nv + 3 * fv[2];
            for (int s = 0; s < 3; ++s) pi[s] = B.v[3 * fv[2] + s];
        } else {
            const int e = find_edge(B, fv[0], fv[2]);
            if (e < 0) return false;
            nrm = B.Ne + 3 * e;
            for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[2] * e02[s];
        }
    } else if (1.0 == para[1]) {
        nrm = B.Nv + 3 * fv[1];
        for (int s = 0; s < 3; ++s) pi[s] = B.v[3 * fv[1] + s];
    } else if (0.0 == para[2]) {
        const int e = find_edge(B, fv[0], fv[1]);
        if (e < 0) return false;
        nrm = B.Ne + 3 * e;
        for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s];
    } else if (0.0 == para[0]) {
        const int e = find_edge(B, fv[1], fv[2]);
        if (e < 0) return false;
        nrm = B.Ne + 3 * e;
        for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s] + para[2] * e02[s];
    } else {
        nrm = B.Nf + 3 * (long long)fid;
        for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s] + para[2] * e02[s];
    }
    for (int s = 0; s < 3; ++s) N[s] = nrm[s];
    return true;
}

// boundary point pi, image point pm and normal N (computational_geometry.c:762-783)
__device__ bool surface_data(const double p[3], int fid, const DevBody &B, double pi[3], double pm[3], double N[3])
{
    if (0 >= B.faceN) {
        N[0] = p[0] - B.O[0];
        N[1] = p[1] - B.O[1];
        N[2] = p[2] - B.O[2];
        double dist = sqrt(dot3(N, N));
        for (int s = 0; s < 3; ++s) N[s] = N[s] / dist;
        dist = B.r - dist;
        for (int s = 0; s < 3; ++s) pi[s] = p[s] + dist * N[s];
    } else if (!closest_on_facet(p, fid, B, pi, N)) {
        return false;
    }
    for (int s = 0; s < 3; ++s) pm[s] = pi[s] + pi[s] - p[s];
    return true;
}

__device__ __forceinline__ void add_weighted(const double Uoh[6], double tiny, double w, double &wsum, double Uo[6])
{
    if (tiny > w) w = tiny;
    w = 1.0 / w;
    for (int n = 0; n < 6; ++n) Uo[n] = Uo[n] + Uoh[n] * w;
    wsum = wsum + w;
}

// inverse distance weighting (immersed_boundary.c:413-473); type TYPED: fluid
// nodes, TYPEF: fluid nodes that were fluid before this mapping (not joined),
// r >= 1: nodes of body did in ghost layer r
__device__ double idw(const IbGrid &G, const ModelParams &mp, const double *U, const int *flags,
                      const unsigned char *joined, const int c[3], const double p[3], int h, int type, int did,
                      double Uo[6], int *status)
{
    const Grid &g = G.g;
    const long long nn = g.nn;
    const int *fdid = flags;
    const int *fgst = flags + 3 * nn;
    double wsum = 0.0;
    for (int n = 0; n < 6; ++n) Uo[n] = 0.0;
    const int rmax = g.n[0] + g.n[1] + g.n[2];
    for (int r = h, tally = 0; 0 == tally; ++r) {
        if (r > rmax) {
            atomicExch(status, 1);  // no qualifying node: the reference would not terminate
            break;
        }
        for (int kh = -r; kh <= r; ++kh) {
            for (int jh = -r; jh <= r; ++jh) {
                for (int ih = -r; ih <= r; ++ih) {
                    const int i = c[0] + ih, j = c[1] + jh, k = c[2] + kh;
                    if (!in_pin(g, k, j, i)) continue;
                    const long long id = node_of(g, i, j, k);
                    if (did != fdid[id]) continue;
                    if (type == kTypeF) {
                        if (joined[id]) continue;
                    } else if (type != kTypeD) {
                        if (type != fgst[id]) continue;
                    }
                    ++tally;
                    double ph[3], Uh[5], Uoh[6];
                    node_point(G, k, j, i, ph);
                    for (int v = 0; v < 5; ++v) Uh[v] = U[v * nn + id];
                    to_primitive(mp.gamma, mp.gasR, Uh, Uoh);
                    add_weighted(Uoh, G.tinyL, dist2(p, ph), wsum, Uo);
                }
            }
        }
    }
    return wsum;
}

__device__ void orthogonal_space(const double N[3], double Ta[3], double Tb[3])
{
    int mark = 2;
    if (fabs(N[mark]) > fabs(N[1])) mark = 1;
    if (fabs(N[mark]) > fabs(N[0])) mark = 0;
    if (0 == mark) {
        Ta[0] = 0.0; Ta[1] = -N[2]; Ta[2] = N[1];
    } else if (1 == mark) {
        Ta[0] = N[2]; Ta[1] = 0.0; Ta[2] = -N[0];
    } else {
        Ta[0] = -N[1]; Ta[1] = N[0]; Ta[2] = 0.0;
    }
    const double nrm = sqrt(dot3(Ta, Ta));
    for (int s = 0; s < 3; ++s) Ta[s] = Ta[s] / nrm;
    Tb[0] = Ta[1] * N[2] - Ta[2] * N[1];
    Tb[1] = Ta[2] * N[0] - Ta[0] * N[2];
    Tb[2] = Ta[0] * N[1] - Ta[1] * N[0];
}

// ---------------------------------------------------------------------------
// ghost layer r of every body (immersed_boundary.c:294-338)
// ---------------------------------------------------------------------------

// Ghost lists: every ghost node of layers 1..gl of every body, as
// (i, j, k, body | layer << 24), in the list of its layer (cap entries each).
// The flags do not change during a boundary treatment and a node belongs to
// one body only, so a node is listed once; the order of a list is free
// (nodes of one layer are independent).
__global__ void ib_list(IbGrid G, const BoxList *groups, int gidx, const int *flags, int4 *ghosts, int *nghost,
                        int cap, int *status)
{
    const BoxList &bl = groups[gidx];
    const long long total = bl.start[bl.nb];
    for (long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x; t0 < total;
         t0 += (long long)gridDim.x * blockDim.x) {
        long long t = t0;
        int q = 0;
        while (t >= bl.start[q + 1]) ++q;
        t -= bl.start[q];
        const int n = bl.body0 + q;
        const int i = bl.lo[q][0] + (int)(t % bl.ext[q][0]);
        const long long rest = t / bl.ext[q][0];
        const int j = bl.lo[q][1] + (int)(rest % bl.ext[q][1]);
        const int k = bl.lo[q][2] + (int)(rest / bl.ext[q][1]);
        const Grid &g = G.g;
        const long long id = node_of(g, i, j, k);
        const int gst = flags[3 * g.nn + id];
        if (gst < 1 || gst > G.gl || n + 1 != flags[id]) continue;
        const int slot = atomicAdd(nghost + gst - 1, 1);
        if (slot >= cap) {
            atomicExch(status, 4);
            continue;
        }
        ghosts[(long long)(gst - 1) * cap + slot] = make_int4(i, j, k, n | (gst << 24));
    }
}

constexpr int kGhostWarps = 4;    // warps per block of ib_ghost
constexpr int kIdwBatch = 4;      // candidates per lane evaluated before the ordered sum

// Inverse distance weighting by one warp (the candidates of the serial
// version's k, j, i loop order, 32 x kIdwBatch at a time).  Every lane
// evaluates candidates and writes w and Uoh[n] * w to the warp's shared
// scratch; lanes 0..6 then add them in candidate order, each lane one sum
// (Uo[0..5], wsum), so every sum takes exactly the serial version's
// additions in the same order.  All lanes return the same values.
__device__ double idw_warp(const IbGrid &G, const ModelParams &mp, const double *U, const int *flags,
                           const int c[3], const double p[3], int h, int type, int did, double Uo[6],
                           double (*sp)[8], int *status)
{
    const Grid &g = G.g;
    const long long nn = g.nn;
    const int *fdid = flags;
    const int *fgst = flags + 3 * nn;
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    const int rmax = g.n[0] + g.n[1] + g.n[2];
    bool failed = false;
    for (int r = h, tally = 0; 0 == tally; ++r) {
        if (r > rmax) {
            failed = true;  // no qualifying node: the reference would not terminate
            break;
        }
        const long long side = 2 * r + 1;
        const long long total = side * side * side;
        for (long long base = 0; base < total; base += 32 * kIdwBatch) {
            bool qual[kIdwBatch];
            long long ids[kIdwBatch];
            int cc[kIdwBatch][3];
#pragma unroll
            for (int b = 0; b < kIdwBatch; ++b) {
                const long long cand = base + 32 * b + lane;
                qual[b] = false;
                ids[b] = 0;
                cc[b][0] = cc[b][1] = cc[b][2] = 0;
                if (cand < total) {
                    const int ih = (int)(cand % side) - r;
                    const long long rest = cand / side;
                    const int jh = (int)(rest % side) - r;
                    const int kh = (int)(rest / side) - r;
                    const int i = c[0] + ih, j = c[1] + jh, k = c[2] + kh;
                    cc[b][0] = i;
                    cc[b][1] = j;
                    cc[b][2] = k;
                    if (in_pin(g, k, j, i)) {
                        ids[b] = node_of(g, i, j, k);
                        qual[b] = true;
                    }
                }
            }
#pragma unroll
            for (int b = 0; b < kIdwBatch; ++b) {
                if (qual[b]) {
                    const long long id = ids[b];
                    bool ok = (did == fdid[id]);
                    if (ok && type != kTypeD) ok = (type == fgst[id]);
                    qual[b] = ok;
                }
            }
            unsigned mask[kIdwBatch];
#pragma unroll
            for (int b = 0; b < kIdwBatch; ++b) {
                if (qual[b]) {
                    const long long id = ids[b];
                    double ph[3], Uh[5], Uoh[6];
                    node_point(G, cc[b][2], cc[b][1], cc[b][0], ph);
                    for (int v = 0; v < 5; ++v) Uh[v] = U[v * nn + id];
                    to_primitive(mp.gamma, mp.gasR, Uh, Uoh);
                    double w = dist2(p, ph);
                    if (G.tinyL > w) w = G.tinyL;
                    w = 1.0 / w;
                    double *row = sp[32 * b + lane];
                    for (int v = 0; v < 6; ++v) row[v] = Uoh[v] * w;
                    row[6] = w;
                }
                mask[b] = __ballot_sync(0xffffffffu, qual[b]);
                tally += __popc(mask[b]);
            }
            __syncwarp();
            if (lane < 7) {
#pragma unroll
                for (int b = 0; b < kIdwBatch; ++b) {
                    for (unsigned m = mask[b]; m; m &= m - 1) acc = acc + sp[32 * b + __ffs(m) - 1][lane];
                }
            }
            __syncwarp();
        }
    }
    if (failed && lane == 0) atomicExch(status, 1);
    for (int n = 0; n < 6; ++n) Uo[n] = __shfl_sync(0xffffffffu, acc, n);
    return __shfl_sync(0xffffffffu, acc, 6);
}

// ghost layer r of every body (immersed_boundary.c:294-338), one warp per
// listed ghost node; the scalar parts run redundantly in all lanes of the
// warp, the searches of the reconstruction are shared out over the lanes
__global__ void __launch_bounds__(kGhostWarps * 32) ib_ghost(IbGrid G, ModelParams mp, const DevBody *bodies,
                                                             const int4 *ghosts, const int *nghost, int cap,
                                                             double *U, const int *flags, int tn, int r,
                                                             int *status)
{
    __shared__ double scratch[kGhostWarps][32 * kIdwBatch][8];
    const int lane = threadIdx.x & 31;
    double (*sp)[8] = scratch[threadIdx.x >> 5];
    const int count = min(nghost[r - 1], cap);  // an overflowing list has set the status
    ghosts += (long long)(r - 1) * cap;
    const Grid &g = G.g;
    const long long nn = g.nn;
    double *Ut = U + (long long)tn * 5 * nn;
    for (int e = blockIdx.x * kGhostWarps + (threadIdx.x >> 5); e < count; e += gridDim.x * kGhostWarps) {
        const int4 q = ghosts[e];
        if ((q.w >> 24) != r) continue;
        const int n = q.w & 0xffffff;
        const int i = q.x, j = q.y, k = q.z;
        const long long id = node_of(g, i, j, k);
        const DevBody &B = bodies[n];
        double pG[3], UoG[6];
        node_point(G, k, j, i, pG);
        if (G.ibmLayer >= r) {
            double pO[3], pI[3], N[3], UoO[6], UoI[6];
            const int fid = flags[nn + id];
            if (B.faceN > 0 && (fid < 0 || fid >= B.faceN)) {
                if (lane == 0) atomicExch(status, 3);  // ghost node without a valid closest facet
                continue;
            }
            if (!surface_data(pG, fid, B, pO, pI, N)) {
                if (lane == 0) atomicExch(status, 2);
                continue;
            }
            const int cI[3] = {map_node(pI[0], G.dmin[0], g.dd[0], G.ng[0]),
                               map_node(pI[1], G.dmin[1], g.dd[1], G.ng[1]),
                               map_node(pI[2], G.dmin[2], g.dd[2], G.ng[2])};
            // ReconstructFlow (immersed_boundary.c:357-412)
            double wsum = idw_warp(G, mp, Ut, flags, cI, pI, kIbR, kTypeD, 0, UoI, sp, status);
            const double w = 1.0 / wsum;
            const double rr[3] = {pO[0] - B.O[0], pO[1] - B.O[1], pO[2] - B.O[2]};
            double Vs[3];
            Vs[0] = B.W[1] * rr[2] - B.W[2] * rr[1];
            Vs[1] = B.W[2] * rr[0] - B.W[0] * rr[2];
            Vs[2] = B.W[0] * rr[1] - B.W[1] * rr[0];
            Vs[0] = B.V[0] + Vs[0];
            Vs[1] = B.V[1] + Vs[1];
            Vs[2] = B.V[2] + Vs[2];
            if (0.0 < B.cf) {
                UoO[1] = Vs[0];
                UoO[2] = Vs[1];
                UoO[3] = Vs[2];
            } else {
                const double V[3] = {UoI[1] * w, UoI[2] * w, UoI[3] * w};
                double Ta[3], Tb[3], rhs[3];
                orthogonal_space(N, Ta, Tb);
                rhs[0] = dot3(Vs, N);
                rhs[1] = dot3(V, Ta);
                rhs[2] = dot3(V, Tb);
                for (int s = 0; s < 3; ++s) UoO[s + 1] = N[s] * rhs[0] + Ta[s] * rhs[1] + Tb[s] * rhs[2];
            }
            UoO[4] = UoI[4] * w;
            UoO[5] = (0.0 > B.T) ? UoI[5] * w : B.T;
            add_weighted(UoO, G.tinyL, dist2(pI, pO), wsum, UoI);
            for (int v = 0; v < 6; ++v) UoI[v] = UoI[v] / wsum;
            // method of images
            UoG[1] = UoO[1] + UoO[1] - UoI[1];
            UoG[2] = UoO[2] + UoO[2] - UoI[2];
            UoG[3] = UoO[3] + UoO[3] - UoI[3];
            UoG[4] = UoI[4];
            UoG[5] = UoI[5];
        } else {
            const int cG[3] = {i, j, k};
            const double ws = idw_warp(G, mp, Ut, flags, cG, pG, 1, r - 1, n + 1, UoG, sp, status);
            for (int v = 0; v < 6; ++v) UoG[v] = UoG[v] / ws;
        }
        UoG[0] = UoG[4] / (UoG[5] * mp.gasR);
        double Uc[5];
        to_conservative(mp.gamma, UoG, Uc);
        double mine = Uc[0];
#pragma unroll
        for (int v = 1; v < 5; ++v) mine = (lane == v) ? Uc[v] : mine;
        if (lane < 5) Ut[lane * nn + id] = mine;
    }
}

// ---------------------------------------------------------------------------
// surface forces and contacts of the rigid-body step
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cross3(const double a[3], const double b[3], double c[3])
{
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

// Per-node terms of IntegrateSurfaceForce (solid_dynamics.c:86-146): a ghost
// node of layer 2 of body n gets Fp = p N, the shear force Fv of no-slip
// viscous bodies, the torque r x (Fp + Fv) and its pressure p, stored at its
// position in the body's node box (the reference's k, j, i loop order) for
// the ordered sums of sf_sum; interfacial nodes of layer 2 are counted.
__global__ void sf_terms(IbGrid G, ModelParams mp, const DevBody *bodies, BoxList bl, long long off0,
                         const double *U, const int *flags, double *terms, unsigned char *valid, int *lidN,
                         int *status)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bl.start[bl.nb]) return;
    const long long slot = off0 + t;
    int q = 0;
    while (t >= bl.start[q + 1]) ++q;
    t -= bl.start[q];
    const int n = bl.body0 + q;
    const int i = bl.lo[q][0] + (int)(t % bl.ext[q][0]);
    const long long rest = t / bl.ext[q][0];
    const int j = bl.lo[q][1] + (int)(rest % bl.ext[q][1]);
    const int k = bl.lo[q][2] + (int)(rest / bl.ext[q][1]);
    const Grid &g = G.g;
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    const DevBody &B = bodies[n];
    valid[slot] = 0;
    if (0 < B.state) return;
    const int did = flags[id];
    if (2 == flags[2 * nn + id] && n + 1 == did) atomicAdd(lidN + n, 1);
    if (2 != flags[3 * nn + id] || n + 1 != did) return;
    double pG[3], pO[3], pI[3], N[3];
    node_point(G, k, j, i, pG);
    const int fid = flags[nn + id];
    if (B.faceN > 0 && (fid < 0 || fid >= B.faceN)) {
        atomicExch(status, 3);
        return;
    }
    if (!surface_data(pG, fid, B, pO, pI, N)) {
        atomicExch(status, 2);
        return;
    }
    const double r[3] = {pO[0] - B.O[0], pO[1] - B.O[1], pO[2] - B.O[2]};
    double Uh[5], Uo[6];
    for (int v = 0; v < 5; ++v) Uh[v] = U[v * nn + id];
    to_primitive(mp.gamma, mp.gasR, Uh, Uo);
    double Fp[3], Fv[3], Fs[3], Tt[3];
    for (int s = 0; s < 3; ++s) Fp[s] = Uo[4] * N[s];
    if (0.0 < mp.refMu && 0.0 < B.cf) {
        const double mu = mp.refMu * exact::sutherland(Uo[5] * mp.refT);
        double V[3];
        cross3(B.W, r, V);
        V[0] = Uo[1] - (B.V[0] + V[0]);
        V[1] = Uo[2] - (B.V[1] + V[1]);
        V[2] = Uo[3] - (B.V[2] + V[2]);
        const double Vn = dot3(V, N);
        for (int s = 0; s < 3; ++s) Fv[s] = mu * (V[s] - Vn * N[s]) / sqrt(dist2(pG, pO));
    } else {
        Fv[0] = Fv[1] = Fv[2] = 0.0;
    }
    for (int s = 0; s < 3; ++s) Fs[s] = Fp[s] + Fv[s];
    cross3(r, Fs, Tt);
    double *row = terms + 10 * slot;
    for (int s = 0; s < 3; ++s) {
        row[s] = Fp[s];
        row[3 + s] = Fv[s];
        row[6 + s] = Tt[s];
    }
    row[9] = Uo[4];
    valid[slot] = 1;
}

// Ordered sums and calibration of IntegrateSurfaceForce (solid_dynamics.c:
// 139-168), one warp (block) per body: the warp walks the body's node box 128
// nodes at a time, stages the terms of the ghost nodes among them in shared
// memory, and lanes 0..8 add Fp, Fv, Tt and lanes 9, 10 the pressure offset
// sums of the variance test, each over the ghost nodes in box order.
constexpr int kSumChunks = 4;
__global__ void __launch_bounds__(32) sf_sum(const DevBody *bodies, const long long *off, const double *terms,
                                             const unsigned char *valid, const int *lidN, double *force)
{
    __shared__ double rows[32 * kSumChunks][10];
    const int lane = threadIdx.x;
    const int n = blockIdx.x;
    const DevBody &B = bodies[n];
    if (0 < B.state) return;
    const long long a = off[n], b = off[n + 1];
    double acc = 0.0, p0 = 0.0;
    int gstN = 0;
    for (long long base = a; base < b; base += 32 * kSumChunks) {
        unsigned mask[kSumChunks];
#pragma unroll
        for (int c = 0; c < kSumChunks; ++c) {
            const long long t = base + 32 * c + lane;
            const bool v = (t < b) && valid[t];
            if (v) {
#pragma unroll
                for (int q = 0; q < 10; ++q) rows[32 * c + lane][q] = terms[10 * t + q];
            }
            mask[c] = __ballot_sync(0xffffffffu, v);
        }
        __syncwarp();
#pragma unroll
        for (int c = 0; c < kSumChunks; ++c) {
            if (!mask[c]) continue;
            if (0 == gstN) p0 = rows[32 * c + __ffs(mask[c]) - 1][9];
            gstN += __popc(mask[c]);
            if (lane < 11) {
                for (unsigned m = mask[c]; m; m &= m - 1) {
                    const double *row = rows[32 * c + __ffs(m) - 1];
                    if (lane < 9) {
                        acc = acc + row[lane];
                    } else if (lane == 9) {
                        acc = acc + row[9] - p0;
                    } else {
                        acc = acc + (row[9] - p0) * (row[9] - p0);
                    }
                }
            }
        }
        __syncwarp();
    }
    const double f1 = __shfl_sync(0xffffffffu, acc, 9);
    const double f2 = __shfl_sync(0xffffffffu, acc, 10);
    if (lane >= 9) return;
    const int lid = lidN[n];
    double out = 0.0;
    if (0 != lid && 0 != gstN) {
        const double percent = (double)FLT_EPSILON * (double)FLT_EPSILON;
        double ds = B.area / lid;
        const double var = (f2 - f1 * f1 / gstN) / gstN;
        const double mean = f1 / gstN + p0;
        if (percent * mean * mean > var) ds = 0.0;
        out = -acc * ds;
    }
    force[9 * n + lane] = out;
}

// Contact scan of ApplyCollision (solid_dynamics.c:242-256, 327-357): every
// interfacial node of layer 1 of a moving body p looks along the collision
// search path; a node of another body q there makes q a contact of p, with
// the path offset added to their line of impact.  The order of the
// reference's contact list (first meeting in node order, then path order) is
// kept as the smallest key node x path length + path index.
__global__ void col_scan(IbGrid G, const DevBody *bodies, BoxList bl, const int *flags, int totN,
                         unsigned long long *key, int *cN, int *status)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= bl.start[bl.nb]) return;
    int q = 0;
    while (t >= bl.start[q + 1]) ++q;
    t -= bl.start[q];
    const int p = bl.body0 + q;
    if (1 == bodies[p].state) return;
    const int i = bl.lo[q][0] + (int)(t % bl.ext[q][0]);
    const long long rest = t / bl.ext[q][0];
    const int j = bl.lo[q][1] + (int)(rest % bl.ext[q][1]);
    const int k = bl.lo[q][2] + (int)(rest / bl.ext[q][1]);
    const Grid &g = G.g;
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    if (1 != flags[2 * nn + id] || p + 1 != flags[id]) return;
    const int end = G.pathSep[1];
    for (int c = 0; c < end; ++c) {
        const int kh = k + G.path[c][2], jh = j + G.path[c][1], ih = i + G.path[c][0];
        if (!in_pin(g, kh, jh, ih)) continue;
        const int d = flags[node_of(g, ih, jh, kh)];
        if (0 == d || p + 1 == d) continue;
        if (d < 0 || d > totN) {
            atomicExch(status, 5);
            continue;
        }
        const long long slot = (long long)p * totN + (d - 1);
        atomicMin(key + slot, (unsigned long long)t * end + c);
        for (int s = 0; s < 3; ++s) atomicAdd(cN + 3 * slot + s, G.path[c][s]);
    }
}

// ---------------------------------------------------------------------------
// node mapping
// ---------------------------------------------------------------------------
__global__ void map_init(Grid g, const DevBody *bodies, int *flags)
{
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Lx * Ly * Lz) return;
    const int i = g.lo[0] + (int)(t % Lx);
    const long long rest = t / Lx;
    const int j = g.lo[1] + (int)(rest % Ly);
    const int k = g.lo[2] + (int)(rest / Ly);
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    const int did = flags[id];
    flags[3 * nn + id] = did;  // keep the old domain field in gst
    if (did == 0) {
        flags[nn + id] = 0;
        return;
    }
    if (bodies[did - 1].state == 1) return;
    if (flags[2 * nn + id] > 0) flags[id] = 0;
}

constexpr int kMapThreads = 256;
constexpr int kMaxSmemFacets = 2048;  // 9 doubles each: 144 KB

__global__ void __launch_bounds__(kMapThreads) map_body(IbGrid G, const DevBody *bodies, int n, BoxList bl,
                                                        int *flags, int *status)
{
    extern __shared__ double stri[];
    const DevBody &B = bodies[n];
    const bool staged = (B.faceN > 0) && (B.faceN <= kMaxSmemFacets);
    if (staged) {
        for (int q = threadIdx.x; q < 9 * B.faceN; q += blockDim.x) stri[q] = B.tri[q];
        __syncthreads();
    }
    const double *tri = staged ? stri : B.tri;
    const int lane = threadIdx.x & 31;
    const long long warps = (long long)gridDim.x * (blockDim.x >> 5);
    const Grid &g = G.g;
    const long long nn = g.nn;
    // one warp per node of the body's box
    for (long long t = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); t < bl.start[1];
         t += warps) {
        const int i = bl.lo[0][0] + (int)(t % bl.ext[0][0]);
        const long long rest = t / bl.ext[0][0];
        const int j = bl.lo[0][1] + (int)(rest % bl.ext[0][1]);
        const int k = bl.lo[0][2] + (int)(rest / bl.ext[0][1]);
        const long long id = node_of(g, i, j, k);
        if (0 != flags[id]) continue;
        double p[3];
        node_point(G, k, j, i, p);
        if (0 >= B.faceN) {
            if (lane == 0 && B.r * B.r >= dist2(B.O, p)) {
                flags[id] = n + 1;
                flags[nn + id] = 0;
            }
            continue;
        }
        // nearest facet, first minimum wins (computational_geometry.c:463-494):
        // each lane keeps the first minimum of its facets f = lane (mod 32),
        // the warp takes the smallest distance and, among equal ones, the
        // smallest facet index
        double best = FLT_MAX;
        int cid = 0;
        for (int f = lane; f < B.faceN; f += 32) {
            const double *T = tri + 9 * f;
            const double v0[3] = {T[0], T[1], T[2]};
            const double e01[3] = {T[3], T[4], T[5]};
            const double e02[3] = {T[6], T[7], T[8]};
            double para[3];
            const double q = point_triangle(p, v0, e01, e02, para);
            if (best > q) {
                best = q;
                cid = f;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(0xffffffffu, best, o);
            const int oc = __shfl_xor_sync(0xffffffffu, cid, o);
            if (ob < best || (ob == best && oc < cid)) {
                best = ob;
                cid = oc;
            }
        }
        double pi[3], N[3];
        if (!closest_on_facet(p, cid, B, pi, N)) {
            if (lane == 0) atomicExch(status, 2);
            continue;
        }
        pi[0] = p[0] - pi[0];
        pi[1] = p[1] - pi[1];
        pi[2] = p[2] - pi[2];
        if (lane == 0 && !(0.0 < dot3(pi, N))) {
            flags[id] = n + 1;
            flags[nn + id] = cid;
        }
    }
}

__device__ __forceinline__ int layer_of(const IbGrid &G, int q)
{
    for (int r = 1; r <= G.gl; ++r) {
        if (G.pathSep[r] > q) return r;
    }
    return 0;
}

// interfacial layer, ghost layer and the joined mark (SetInterfacialField)
__global__ void map_interface(IbGrid G, int *flags, unsigned char *joined)
{
    const Grid &g = G.g;
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Lx * Ly * Lz) return;
    const int i = g.lo[0] + (int)(t % Lx);
    const long long rest = t / Lx;
    const int j = g.lo[1] + (int)(rest % Ly);
    const int k = g.lo[2] + (int)(rest / Ly);
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    const int did = flags[id];
    joined[id] = (flags[3 * nn + id] != did && did == 0) ? 1 : 0;
    int lid = 0, gst = 0;
    if (did != 0) {
        for (int q = 0; q < G.pathSep[0]; ++q) {
            const int kh = k + G.path[q][2], jh = j + G.path[q][1], ih = i + G.path[q][0];
            if (!in_pin(g, kh, jh, ih)) continue;
            if (did != flags[node_of(g, ih, jh, kh)]) {
                lid = layer_of(G, q);
                break;
            }
        }
        if (lid > 0) {
            for (int q = 0; q < G.pathSep[0]; ++q) {
                const int kh = k + G.path[q][2], jh = j + G.path[q][1], ih = i + G.path[q][0];
                if (!in_pin(g, kh, jh, ih)) continue;
                if (0 == flags[node_of(g, ih, jh, kh)]) {
                    gst = layer_of(G, q);
                    break;
                }
            }
        }
    }
    flags[2 * nn + id] = lid;
    flags[3 * nn + id] = gst;
}

// refill newly uncovered fluid nodes from fluid nodes that stayed fluid
__global__ void map_refill(IbGrid G, ModelParams mp, double *U, int *flags, const unsigned char *joined, int *status)
{
    const Grid &g = G.g;
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Lx * Ly * Lz) return;
    const int i = g.lo[0] + (int)(t % Lx);
    const long long rest = t / Lx;
    const int j = g.lo[1] + (int)(rest % Ly);
    const int k = g.lo[2] + (int)(rest / Ly);
    const long long nn = g.nn;
    const long long id = node_of(g, i, j, k);
    if (!joined[id]) return;
    const int c[3] = {i, j, k};
    double p[3], Uo[6];
    node_point(G, k, j, i, p);
    const double ws = idw(G, mp, U, flags, joined, c, p, kIbR, kTypeF, 0, Uo, status);
    for (int v = 0; v < 6; ++v) Uo[v] = Uo[v] / ws;
    Uo[0] = Uo[4] / (Uo[5] * mp.gasR);
    double Uc[5];
    to_conservative(mp.gamma, Uo, Uc);
    for (int v = 0; v < 5; ++v) U[v * nn + id] = Uc[v];
    flags[nn + id] = -1;
}

// facet table v0, e01, e02 (BuildTriangle, computational_geometry.c:449-462)
__global__ void build_tri(const int *f, const double *v, double *tri, int faceN)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= faceN) return;
    for (int s = 0; s < 3; ++s) {
        const double v0 = v[3 * f[3 * q + 0] + s];
        const double v1 = v[3 * f[3 * q + 1] + s];
        const double v2 = v[3 * f[3 * q + 2] + s];
        tri[9 * q + s] = v0;
        tri[9 * q + 3 + s] = v1 - v0;
        tri[9 * q + 6 + s] = v2 - v0;
    }
}

// ---- surface motion (TransformPolyhedron, computational_geometry.c:162-246) ----
// rot is the point rotation matrix of the angles; a point is moved relative
// to the reference point O: shifted to it, scaled, rotated, offset and
// shifted back, each product and sum rounded on its own in the reference's
// order (this unit is compiled without contraction).  Normals are rotated.
struct SurfaceMotion {
    double rot[3][3];
    double O[3], scale[3], offset[3];
};

__host__ __device__ inline void move_point(const SurfaceMotion &M, double p[3])
{
    double t[3];
    for (int s = 0; s < 3; ++s) t[s] = (p[s] - M.O[s]) * M.scale[s];
    for (int s = 0; s < 3; ++s) p[s] = dot3(M.rot[s], t) + M.offset[s] + M.O[s];
}

// The reference updates the box vertex by vertex with box = (box < v) ? box : v
// (and > for the maximum), starting from FLT_MAX and FLT_MIN: the result is
// the extreme value, and among equal values (+0 and -0) the last one in
// vertex order.  Extremes are therefore reduced as (value, vertex index)
// pairs, the larger index winning ties; the start values carry index -1.
__host__ __device__ inline void take_lo(double &v, int &i, double x, int j)
{
    if (x < v || (x == v && j > i)) {
        v = x;
        i = j;
    }
}

__host__ __device__ inline void take_hi(double &v, int &i, double x, int j)
{
    if (x > v || (x == v && j > i)) {
        v = x;
        i = j;
    }
}

constexpr int kMotionThreads = 256;

__global__ void __launch_bounds__(kMotionThreads) move_surface(SurfaceMotion M, double *v, double *Nf, double *Ne,
                                                               double *Nv, int vertN, int faceN, int edgeN,
                                                               BoxPart *part)
{
    double lo[3], hi[3];
    int loi[3], hii[3];
    for (int s = 0; s < 3; ++s) {
        lo[s] = FLT_MAX;
        hi[s] = FLT_MIN;
        loi[s] = -1;
        hii[s] = -1;
    }
    const long long total = 2LL * vertN + faceN + edgeN;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (long long)gridDim.x * blockDim.x) {
        if (q < vertN) {
            double p[3] = {v[3 * q], v[3 * q + 1], v[3 * q + 2]};
            move_point(M, p);
            for (int s = 0; s < 3; ++s) {
                v[3 * q + s] = p[s];
                take_lo(lo[s], loi[s], p[s], (int)q);
                take_hi(hi[s], hii[s], p[s], (int)q);
            }
        } else {
            long long k = q - vertN;
            double *N;
            if (k < faceN) {
                N = Nf + 3 * k;
            } else if ((k -= faceN) < edgeN) {
                N = Ne + 3 * k;
            } else {
                N = Nv + 3 * (k - edgeN);
            }
            const double t[3] = {N[0], N[1], N[2]};
            for (int s = 0; s < 3; ++s) N[s] = dot3(M.rot[s], t);
        }
    }
    // block extremes: lanes, then warps
    for (int off = 16; off > 0; off >>= 1) {
        for (int s = 0; s < 3; ++s) {
            const double a = __shfl_down_sync(0xffffffffu, lo[s], off);
            const int ai = __shfl_down_sync(0xffffffffu, loi[s], off);
            const double b = __shfl_down_sync(0xffffffffu, hi[s], off);
            const int bi = __shfl_down_sync(0xffffffffu, hii[s], off);
            take_lo(lo[s], loi[s], a, ai);
            take_hi(hi[s], hii[s], b, bi);
        }
    }
    __shared__ BoxPart warps[kMotionThreads / 32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        for (int s = 0; s < 3; ++s) {
            warps[warp].v[2 * s] = lo[s];
            warps[warp].i[2 * s] = loi[s];
            warps[warp].v[2 * s + 1] = hi[s];
            warps[warp].i[2 * s + 1] = hii[s];
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        BoxPart r = warps[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
            for (int s = 0; s < 3; ++s) {
                take_lo(r.v[2 * s], r.i[2 * s], warps[w].v[2 * s], warps[w].i[2 * s]);
                take_hi(r.v[2 * s + 1], r.i[2 * s + 1], warps[w].v[2 * s + 1], warps[w].i[2 * s + 1]);
            }
        }
        part[blockIdx.x] = r;
    }
}

IbGrid make_ibgrid(const Grid &g, const acfd_partition_t &part, int ibmLayer)
{
    IbGrid G;
    G.g = g;
    for (int s = 0; s < 3; ++s) {
        G.ng[s] = part.ng[s];
        G.dmin[s] = part.domain[s][0];
        G.d[s] = part.d[s];
    }
    G.tinyL = part.tinyL;
    G.gl = part.gl;
    G.ibmLayer = ibmLayer;
    for (int q = 0; q < 4; ++q) G.pathSep[q] = part.pathSep[q];
    for (int q = 0; q < 30; ++q)
        for (int s = 0; s < 3; ++s) G.path[q][s] = part.path[q][s];
    return G;
}

// node box of a body confined to PIN (immersed_boundary.c:151-154)
void body_box(const acfd_partition_t &part, const DevBody &B, int lo[3], int ext[3])
{
    for (int s = 0; s < 3; ++s) {
        const int nlo = part.ns[0][s][0], nhi = part.ns[0][s][1];
        const int a = confine((int)((B.box[s][0] - part.domain[s][0]) * part.dd[s] + 0.5) + part.ng[s], nlo, nhi);
        const int b = confine((int)((B.box[s][1] - part.domain[s][0]) * part.dd[s] + 0.5) + part.ng[s], nlo, nhi) + 1;
        lo[s] = a;
        ext[s] = std::max(0, b - a);
    }
}

int read_status(IbState *ib, cudaStream_t st)
{
    int h = 0;
    ACFD_CUDA(cudaMemcpyAsync(&h, ib->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    ACFD_CUDA(cudaStreamSynchronize(st));
    if (h == 1) {
        set_error("immersed boundary: no qualifying node for inverse distance weighting");
        return ACFD_ERR_DEVICE;
    }
    if (h == 2) {
        set_error("immersed boundary: edge of the closest facet not found in the edge list");
        return ACFD_ERR_NOT_FOUND;
    }
    if (h == 3) {
        set_error("immersed boundary: ghost node with a closest-facet id outside the body's facets");
        return ACFD_ERR_DEVICE;
    }
    if (h == 4) {
        set_error("immersed boundary: ghost list overflow");
        return ACFD_ERR_DEVICE;
    }
    if (h == 5) {
        set_error("collision scan: node with a body id outside the body list");
        return ACFD_ERR_DEVICE;
    }
    return ACFD_OK;
}

unsigned blocks_for(long long n, int bs)
{
    return (unsigned)((n + bs - 1) / bs);
}

}  // namespace

int ib_create(IbState **out)
{
    IbState *ib = new IbState();
    cudaError_t e = cudaMalloc(&ib->status, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(ib->status, 0, sizeof(int));
    if (e != cudaSuccess) {
        delete ib;
        return cuda_status(e, "ib_create");
    }
    *out = ib;
    return ACFD_OK;
}

static void ib_release_geometry(IbState *ib)
{
    for (void *p : ib->buffers) cudaFree(p);
    ib->buffers.clear();
    cudaFree(ib->dev);
    ib->dev = nullptr;
    ib->host.clear();
    ib->count = 0;
    ib->ghosts = nullptr;
    ib->nghost = nullptr;
    ib->ghost_cap = 0;
    cudaFree(ib->groups);
    ib->groups = nullptr;
    ib->ngroups = 0;
}

static void ib_release_solid(IbState *ib)
{
    cudaFree(ib->sf_terms);
    cudaFree(ib->sf_valid);
    cudaFree(ib->sf_off);
    cudaFree(ib->sf_lid);
    cudaFree(ib->sf_force);
    cudaFree(ib->col_key);
    cudaFree(ib->col_N);
    cudaFree(ib->motion_part);
    ib->motion_part = nullptr;
    ib->sf_terms = nullptr;
    ib->sf_valid = nullptr;
    ib->sf_off = nullptr;
    ib->sf_lid = nullptr;
    ib->sf_force = nullptr;
    ib->col_key = nullptr;
    ib->col_N = nullptr;
    ib->sf_cap = 0;
    ib->col_n = 0;
}

void ib_destroy(IbState *ib)
{
    if (!ib) return;
    ib_release_geometry(ib);
    ib_release_solid(ib);
    cudaFree(ib->joined);
    cudaFree(ib->status);
    delete ib;
}

int ib_count(const IbState *ib)
{
    return ib ? ib->count : 0;
}

static void body_scalars(DevBody &B, const acfd_polyhedron_t &P)
{
    B.faceN = P.faceN;
    B.edgeN = P.edgeN;
    B.vertN = P.vertN;
    B.state = P.state;
    B.r = P.r;
    B.T = P.T;
    B.cf = P.cf;
    B.area = P.area;
    for (int s = 0; s < 3; ++s) {
        B.O[s] = P.O[s];
        B.V[s] = P.V[s];
        B.W[s] = P.W[s];
        B.box[s][0] = P.box[s][0];
        B.box[s][1] = P.box[s][1];
    }
}

static int boxes_of(IbState *ib, const acfd_partition_t &part, int n0, BoxList &bl);

// the per-layer ghost capacity the bodies' node boxes need
static long long ghost_need(const IbState *ib, const acfd_partition_t &part)
{
    long long cap = 0;
    for (int n = 0; n < ib->count; ++n) {
        int lo[3], ext[3];
        body_box(part, ib->host[n], lo, ext);
        cap += (long long)ext[0] * ext[1] * ext[2];
    }
    long long pin = 1;
    for (int s = 0; s < 3; ++s) pin *= std::max(0, part.ns[0][s][1] - part.ns[0][s][0]);
    return std::max(1LL, std::min(cap, pin));
}

// the node boxes of all bodies to the device (the ghost list reads them there,
// so that a captured step stays valid while the bodies move)
static int upload_groups(IbState *ib, const acfd_partition_t &part, cudaStream_t st)
{
    std::vector<BoxList> h((size_t)ib->ngroups);
    for (int g = 0; g < ib->ngroups; ++g) boxes_of(ib, part, 8 * g, h[(size_t)g]);
    ACFD_CUDA(cudaMemcpyAsync(ib->groups, h.data(), sizeof(BoxList) * h.size(), cudaMemcpyHostToDevice, st));
    return ACFD_OK;
}

// A triangulated body given without vertices and normals keeps the surface
// it has on the device (moved there by acfd_transform_polyhedron); its face
// and edge lists are kept too.
static bool keeps_surface(const acfd_polyhedron_t &P)
{
    return P.faceN > 0 && !P.v && !P.Nv && !P.Nf && !P.Ne;
}

// A moved body list of the same bodies (same counts of faces, edges and
// vertices) whose ghost lists still fit: new positions, velocities and
// surfaces go into the device buffers in place, in stream order, so that
// the device pointers and launch shapes of a captured step stay valid.
static int update_in_place(IbState *ib, const acfd_polyhedron_t *poly, int totN, const acfd_partition_t &part,
                           cudaStream_t st, bool *done)
{
    *done = false;
    if (totN != ib->count || !ib->dev || !ib->groups) return ACFD_OK;
    for (int n = 0; n < totN; ++n) {
        const DevBody &B = ib->host[n];
        if (B.faceN != poly[n].faceN || B.edgeN != poly[n].edgeN || B.vertN != poly[n].vertN) return ACFD_OK;
        if (poly[n].faceN > 0 && !keeps_surface(poly[n]) &&
            (!poly[n].f || !poly[n].Nf || !poly[n].e || !poly[n].Ne || !poly[n].v || !poly[n].Nv)) {
            return ACFD_OK;
        }
    }
    std::vector<DevBody> prev = ib->host;
    for (int n = 0; n < totN; ++n) body_scalars(ib->host[n], poly[n]);
    if (ghost_need(ib, part) > ib->ghost_cap) {
        ib->host = prev;
        return ACFD_OK;
    }
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t &P = poly[n];
        const DevBody &B = ib->host[n];
        if (P.faceN <= 0 || keeps_surface(P)) continue;
        auto put = [&](const void *dst, const void *src, size_t bytes) {
            return cudaMemcpyAsync(const_cast<void *>(dst), src, bytes, cudaMemcpyHostToDevice, st);
        };
        cudaError_t e = put(B.f, P.f, sizeof(int) * 3 * P.faceN);
        if (e == cudaSuccess) e = put(B.Nf, P.Nf, sizeof(double) * 3 * P.faceN);
        if (e == cudaSuccess) e = put(B.e, P.e, sizeof(int) * 4 * P.edgeN);
        if (e == cudaSuccess) e = put(B.Ne, P.Ne, sizeof(double) * 3 * P.edgeN);
        if (e == cudaSuccess) e = put(B.v, P.v, sizeof(double) * 3 * P.vertN);
        if (e == cudaSuccess) e = put(B.Nv, P.Nv, sizeof(double) * 3 * P.vertN);
        if (e != cudaSuccess) return cuda_status(e, "acfd_geo_upload");
        build_tri<<<blocks_for(P.faceN, 128), 128, 0, st>>>(B.f, B.v, const_cast<double *>(B.tri), P.faceN);
        ACFD_CUDA(cudaGetLastError());
    }
    ACFD_CUDA(cudaMemcpyAsync(ib->dev, ib->host.data(), sizeof(DevBody) * totN, cudaMemcpyHostToDevice, st));
    int rc = upload_groups(ib, part, st);
    if (rc != ACFD_OK) return rc;
    *done = true;
    return ACFD_OK;
}

int ib_upload(IbState *ib, const acfd_polyhedron_t *poly, int totN, const acfd_partition_t &part, cudaStream_t st,
              bool *relayout)
{
    *relayout = true;
    ib->lists_valid = false;  // new boxes: the next geometric field (or treatment) lists the ghosts
    if (totN > 0) {
        bool done = false;
        const int rc = update_in_place(ib, poly, totN, part, st, &done);
        if (rc != ACFD_OK) return rc;
        if (done) {
            *relayout = false;
            return ACFD_OK;
        }
    }
    ACFD_CUDA(cudaStreamSynchronize(st));
    // bodies that keep their device surface through a new layout: the
    // surface comes back to the host first and is uploaded with the list
    std::vector<acfd_polyhedron_t> listed;
    std::vector<std::vector<double>> reals;
    std::vector<std::vector<int>> ints;
    for (int n = 0; n < totN; ++n) {
        if (!keeps_surface(poly[n])) continue;
        if (n >= ib->count || ib->host[n].faceN != poly[n].faceN || ib->host[n].edgeN != poly[n].edgeN ||
            ib->host[n].vertN != poly[n].vertN || !ib->host[n].v) {
            set_error("acfd_geo_upload: body %d has no surface on the device to keep", n);
            return ACFD_ERR_ARG;
        }
        if (listed.empty()) listed.assign(poly, poly + totN);
        const DevBody &B = ib->host[n];
        acfd_polyhedron_t &P = listed[n];
        const size_t sizes[4] = {3 * (size_t)B.vertN, 3 * (size_t)B.vertN, 3 * (size_t)B.faceN, 3 * (size_t)B.edgeN};
        const double *from[4] = {B.v, B.Nv, B.Nf, B.Ne};
        const double **to[4] = {&P.v, &P.Nv, &P.Nf, &P.Ne};
        for (int a = 0; a < 4; ++a) {
            reals.emplace_back(sizes[a]);
            ACFD_CUDA(cudaMemcpy(reals.back().data(), from[a], sizeof(double) * sizes[a], cudaMemcpyDeviceToHost));
            *to[a] = reals.back().data();
        }
        ints.emplace_back(3 * (size_t)B.faceN);
        ACFD_CUDA(cudaMemcpy(ints.back().data(), B.f, sizeof(int) * 3 * B.faceN, cudaMemcpyDeviceToHost));
        P.f = ints.back().data();
        ints.emplace_back(4 * (size_t)B.edgeN);
        ACFD_CUDA(cudaMemcpy(ints.back().data(), B.e, sizeof(int) * 4 * B.edgeN, cudaMemcpyDeviceToHost));
        P.e = ints.back().data();
    }
    if (!listed.empty()) poly = listed.data();
    ib_release_geometry(ib);
    if (totN == 0) return ACFD_OK;
    ib->host.resize(totN);
    auto dcopy = [&](const void *src, size_t bytes, void **dst) -> int {
        *dst = nullptr;
        if (bytes == 0) return ACFD_OK;
        if (!src) {
            set_error("acfd_geo_upload: missing geometry array");
            return ACFD_ERR_ARG;
        }
        ACFD_CUDA(cudaMalloc(dst, bytes));
        ib->buffers.push_back(*dst);
        ACFD_CUDA(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        return ACFD_OK;
    };
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t &P = poly[n];
        DevBody &B = ib->host[n];
        body_scalars(B, P);
        B.f = nullptr; B.Nf = nullptr; B.e = nullptr; B.Ne = nullptr; B.v = nullptr; B.Nv = nullptr; B.tri = nullptr;
        if (P.faceN > 0) {
            void *f, *Nf, *e, *Ne, *v, *Nv, *tri;
            int st2;
            if ((st2 = dcopy(P.f, sizeof(int) * 3 * P.faceN, &f)) != ACFD_OK) return st2;
            if ((st2 = dcopy(P.Nf, sizeof(double) * 3 * P.faceN, &Nf)) != ACFD_OK) return st2;
            if ((st2 = dcopy(P.e, sizeof(int) * 4 * P.edgeN, &e)) != ACFD_OK) return st2;
            if ((st2 = dcopy(P.Ne, sizeof(double) * 3 * P.edgeN, &Ne)) != ACFD_OK) return st2;
            if ((st2 = dcopy(P.v, sizeof(double) * 3 * P.vertN, &v)) != ACFD_OK) return st2;
            if ((st2 = dcopy(P.Nv, sizeof(double) * 3 * P.vertN, &Nv)) != ACFD_OK) return st2;
            ACFD_CUDA(cudaMalloc(&tri, sizeof(double) * 9 * P.faceN));
            ib->buffers.push_back(tri);
            build_tri<<<blocks_for(P.faceN, 128), 128>>>((const int *)f, (const double *)v, (double *)tri, P.faceN);
            ACFD_CUDA(cudaGetLastError());
            B.f = (const int *)f;
            B.Nf = (const double *)Nf;
            B.e = (const int *)e;
            B.Ne = (const double *)Ne;
            B.v = (const double *)v;
            B.Nv = (const double *)Nv;
            B.tri = (const double *)tri;
        }
    }
    ACFD_CUDA(cudaMalloc(&ib->dev, sizeof(DevBody) * totN));
    ACFD_CUDA(cudaMemcpy(ib->dev, ib->host.data(), sizeof(DevBody) * totN, cudaMemcpyHostToDevice));
    // ghost lists, one per layer: a node is listed at most once, so the
    // smaller of the bodies' node boxes and the computed nodes bounds each
    if (totN >= (1 << 24) || part.gl >= 128) {
        set_error("immersed boundary: %d bodies, %d ghost layers (at most %d, 127)", totN, part.gl, (1 << 24) - 1);
        return ACFD_ERR_ARG;
    }
    ib->count = totN;
    long long pin = 1;
    for (int s = 0; s < 3; ++s) pin *= std::max(0, part.ns[0][s][1] - part.ns[0][s][0]);
    // a margin for bodies that move into larger boxes (kept in place then)
    long long cap = ghost_need(ib, part);
    cap = std::max(1LL, std::min(cap + cap / 4 + 64, pin));
    if (cap > INT_MAX) {
        set_error("immersed boundary: ghost list of %lld nodes", cap);
        return ACFD_ERR_ARG;
    }
    void *gl_buf = nullptr, *cnt = nullptr;
    const int layers = std::max(1, part.gl);
    ACFD_CUDA(cudaMalloc(&gl_buf, sizeof(int4) * (size_t)cap * layers));
    ib->buffers.push_back(gl_buf);
    ACFD_CUDA(cudaMalloc(&cnt, sizeof(int) * layers));
    ib->buffers.push_back(cnt);
    ib->ghosts = (int4 *)gl_buf;
    ib->nghost = (int *)cnt;
    ib->ghost_cap = (int)cap;
    ib->ngroups = (totN + 7) / 8;
    ACFD_CUDA(cudaMalloc(&ib->groups, sizeof(BoxList) * ib->ngroups));
    ACFD_CUDA(cudaDeviceSynchronize());
    int rc = upload_groups(ib, part, st);
    if (rc != ACFD_OK) return rc;
    ACFD_CUDA(cudaStreamSynchronize(st));
    return ACFD_OK;
}

static int boxes_of(IbState *ib, const acfd_partition_t &part, int n0, BoxList &bl)
{
    bl.body0 = n0;
    bl.nb = std::min(8, ib->count - n0);
    bl.start[0] = 0;
    for (int q = 0; q < bl.nb; ++q) {
        body_box(part, ib->host[n0 + q], bl.lo[q], bl.ext[q]);
        bl.start[q + 1] = bl.start[q] + (long long)bl.ext[q][0] * bl.ext[q][1] * bl.ext[q][2];
    }
    return ACFD_OK;
}

// the ghost lists of every body from the current flags
static int build_lists(IbState *ib, const IbGrid &G, const acfd_partition_t &part, const int *flags,
                       cudaStream_t st)
{
    ACFD_CUDA(cudaMemsetAsync(ib->nghost, 0, sizeof(int) * part.gl, st));
    // the boxes come from device memory and the grid is fixed (grid-stride)
    const unsigned lblocks = (unsigned)std::min<long long>(blocks_for(ib->ghost_cap, 256), 148LL * 4);
    for (int gi = 0; gi < ib->ngroups; ++gi) {
        ib_list<<<lblocks, 256, 0, st>>>(G, ib->groups, gi, flags, ib->ghosts, ib->nghost, ib->ghost_cap,
                                         ib->status);
        ACFD_CUDA(cudaGetLastError());
    }
    ib->lists_valid = true;
    return ACFD_OK;
}

int ib_flags_changed(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                     const int *flags, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    ib->lists_valid = false;
    if (part.gl < 1) return ACFD_OK;
    return build_lists(ib, make_ibgrid(g, part, m.ibmLayer), part, flags, st);
}

int ib_treat(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part, double *U, int *flags,
             int tn, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    const IbGrid G = make_ibgrid(g, part, m.ibmLayer);
    if (part.gl < 1) return ACFD_OK;
    if (!ib->lists_valid) {
        const int rc = build_lists(ib, G, part, flags, st);
        if (rc != ACFD_OK) return rc;
    }
    // one warp per listed node, at most a few waves of resident warps
    const unsigned blocks = (unsigned)std::min<long long>(blocks_for(ib->ghost_cap, kGhostWarps), 148LL * 12);
    for (int r = 1; r <= part.gl; ++r) {
        ib_ghost<<<blocks, kGhostWarps * 32, 0, st>>>(G, m, ib->dev, ib->ghosts, ib->nghost, ib->ghost_cap, U, flags,
                                                      tn, r, ib->status);
        ACFD_CUDA(cudaGetLastError());
    }
    return ACFD_OK;
}

int ib_treat_launches(const IbState *ib, const acfd_partition_t &part)
{
    if (!ib || ib->count == 0) return 0;
    return (ib->lists_valid ? 0 : (ib->count + 7) / 8) + part.gl;
}

// node boxes of all bodies, their offsets and the scratch of the surface
// force and contact scans (allocated once per body list)
static int solid_scratch(IbState *ib, const acfd_partition_t &part, std::vector<long long> &off)
{
    const int totN = ib->count;
    off.assign(totN + 1, 0);
    for (int n = 0; n < totN; ++n) {
        int lo[3], ext[3];
        body_box(part, ib->host[n], lo, ext);
        off[n + 1] = off[n] + (long long)ext[0] * ext[1] * ext[2];
    }
    // kept across body uploads (moving bodies are uploaded every half step);
    // grown with a margin when the boxes outgrow it
    if (!ib->sf_off || ib->col_n != totN || off[totN] > ib->sf_cap) {
        ib_release_solid(ib);
        const long long cap = std::max(1LL, off[totN] + off[totN] / 4);
        ACFD_CUDA(cudaMalloc(&ib->sf_terms, sizeof(double) * 10 * (size_t)cap));
        ACFD_CUDA(cudaMalloc(&ib->sf_valid, (size_t)cap));
        ACFD_CUDA(cudaMalloc(&ib->sf_off, sizeof(long long) * (totN + 1)));
        ACFD_CUDA(cudaMalloc(&ib->sf_lid, sizeof(int) * totN));
        ACFD_CUDA(cudaMalloc(&ib->sf_force, sizeof(double) * 9 * totN));
        ACFD_CUDA(cudaMalloc(&ib->col_key, sizeof(unsigned long long) * totN * totN));
        ACFD_CUDA(cudaMalloc(&ib->col_N, sizeof(int) * 3 * totN * totN));
        ib->sf_cap = cap;
        ib->col_n = totN;
    }
    return ACFD_OK;
}

int ib_surface_force(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                     const double *U, const int *flags, double *force, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    std::vector<long long> off;
    int rc = solid_scratch(ib, part, off);
    if (rc != ACFD_OK) return rc;
    const int totN = ib->count;
    const IbGrid G = make_ibgrid(g, part, m.ibmLayer);
    ACFD_CUDA(cudaMemcpyAsync(ib->sf_off, off.data(), sizeof(long long) * (totN + 1), cudaMemcpyHostToDevice, st));
    ACFD_CUDA(cudaMemsetAsync(ib->sf_lid, 0, sizeof(int) * totN, st));
    for (int n0 = 0; n0 < totN; n0 += 8) {
        BoxList bl;
        boxes_of(ib, part, n0, bl);
        const long long total = bl.start[bl.nb];
        if (total == 0) continue;
        sf_terms<<<blocks_for(total, 128), 128, 0, st>>>(G, m, ib->dev, bl, off[n0], U, flags, ib->sf_terms,
                                                         ib->sf_valid, ib->sf_lid, ib->status);
        ACFD_CUDA(cudaGetLastError());
    }
    sf_sum<<<totN, 32, 0, st>>>(ib->dev, ib->sf_off, ib->sf_terms, ib->sf_valid, ib->sf_lid, ib->sf_force);
    ACFD_CUDA(cudaGetLastError());
    std::vector<double> h((size_t)9 * totN);
    ACFD_CUDA(cudaMemcpyAsync(h.data(), ib->sf_force, sizeof(double) * 9 * totN, cudaMemcpyDeviceToHost, st));
    rc = read_status(ib, st);  // synchronizes the stream
    if (rc != ACFD_OK) return rc;
    for (int n = 0; n < totN; ++n) {
        if (0 < ib->host[n].state) continue;  // rows of bodies without surface force stay as they are
        for (int c = 0; c < 9; ++c) force[9 * n + c] = h[(size_t)9 * n + c];
    }
    return ACFD_OK;
}

int ib_collision_scan(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                      const int *flags, int *counts, int *gid, int *N, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    std::vector<long long> off;
    int rc = solid_scratch(ib, part, off);
    if (rc != ACFD_OK) return rc;
    const int totN = ib->count;
    const IbGrid G = make_ibgrid(g, part, m.ibmLayer);
    const size_t pairs = (size_t)totN * totN;
    ACFD_CUDA(cudaMemsetAsync(ib->col_key, 0xff, sizeof(unsigned long long) * pairs, st));
    ACFD_CUDA(cudaMemsetAsync(ib->col_N, 0, sizeof(int) * 3 * pairs, st));
    for (int n0 = 0; n0 < totN; n0 += 8) {
        BoxList bl;
        boxes_of(ib, part, n0, bl);
        const long long total = bl.start[bl.nb];
        if (total == 0) continue;
        col_scan<<<blocks_for(total, 128), 128, 0, st>>>(G, ib->dev, bl, flags, totN, ib->col_key, ib->col_N,
                                                         ib->status);
        ACFD_CUDA(cudaGetLastError());
    }
    std::vector<unsigned long long> key(pairs);
    std::vector<int> cn(3 * pairs);
    ACFD_CUDA(cudaMemcpyAsync(key.data(), ib->col_key, sizeof(unsigned long long) * pairs, cudaMemcpyDeviceToHost,
                              st));
    ACFD_CUDA(cudaMemcpyAsync(cn.data(), ib->col_N, sizeof(int) * 3 * pairs, cudaMemcpyDeviceToHost, st));
    rc = read_status(ib, st);
    if (rc != ACFD_OK) return rc;
    for (int p = 0; p < totN; ++p) {
        std::vector<std::pair<unsigned long long, int>> met;
        for (int q = 0; q < totN; ++q) {
            const unsigned long long k = key[(size_t)p * totN + q];
            if (k != ~0ULL) met.emplace_back(k, q);
        }
        std::sort(met.begin(), met.end());
        counts[p] = (int)met.size();
        for (size_t c = 0; c < met.size(); ++c) {
            const size_t slot = (size_t)p * totN + met[c].second;
            gid[(size_t)p * totN + c] = met[c].second + 1;
            for (int s = 0; s < 3; ++s) N[3 * ((size_t)p * totN + c) + s] = cn[3 * slot + s];
        }
    }
    return ACFD_OK;
}

// TransformPolyhedron (computational_geometry.c:162-208) of body n: its
// device surface is moved (move_surface, then the facet table), and the
// reference point O, the centroid, the inertia tensor and the box follow on
// the host in the reference's order.  The host part uses the C library's
// sin, cos and sqrt, as the reference does.
int ib_transform(IbState *ib, int n, const double O[3], const double scale[3], const double angle[3],
                 const double offset[3], double centroid[3], double inertia[9], double box[6], cudaStream_t st)
{
    if (!ib || n < 0 || n >= ib->count) {
        set_error("acfd_transform_polyhedron: body %d of %d", n, ib ? ib->count : 0);
        return ACFD_ERR_ARG;
    }
    const DevBody &B = ib->host[n];
    if (B.faceN <= 0 || !B.v) {
        set_error("acfd_transform_polyhedron: body %d is not triangulated", n);
        return ACFD_ERR_ARG;
    }
    SurfaceMotion M;
    for (int s = 0; s < 3; ++s) {
        M.O[s] = O[s];
        M.scale[s] = scale[s];
        M.offset[s] = offset[s];
    }
    const double Sx = sin(angle[0]), Sy = sin(angle[1]), Sz = sin(angle[2]);
    const double Cx = cos(angle[0]), Cy = cos(angle[1]), Cz = cos(angle[2]);
    // rotation about x, then y, then z (the reference's point rotation matrix)
    const double R[3][3] = {{Cy * Cz, -Cx * Sz + Sx * Sy * Cz, Sx * Sz + Cx * Sy * Cz},
                            {Cy * Sz, Cx * Cz + Sx * Sy * Sz, -Sx * Cz + Cx * Sy * Sz},
                            {-Sy, Sx * Cy, Cx * Cy}};
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) M.rot[a][b] = R[a][b];
    if (!ib->motion_part) ACFD_CUDA(cudaMalloc(&ib->motion_part, sizeof(BoxPart) * kMotionBlocks));
    const long long total = 2LL * B.vertN + B.faceN + B.edgeN;
    const int nblk = (int)std::min<long long>(kMotionBlocks, (total + kMotionThreads - 1) / kMotionThreads);
    move_surface<<<nblk, kMotionThreads, 0, st>>>(M, const_cast<double *>(B.v), const_cast<double *>(B.Nf),
                                                  const_cast<double *>(B.Ne), const_cast<double *>(B.Nv), B.vertN,
                                                  B.faceN, B.edgeN, ib->motion_part);
    ACFD_CUDA(cudaGetLastError());
    build_tri<<<blocks_for(B.faceN, 128), 128, 0, st>>>(B.f, B.v, const_cast<double *>(B.tri), B.faceN);
    ACFD_CUDA(cudaGetLastError());
    std::vector<BoxPart> part((size_t)nblk);
    ACFD_CUDA(cudaMemcpyAsync(part.data(), ib->motion_part, sizeof(BoxPart) * nblk, cudaMemcpyDeviceToHost, st));
    ACFD_CUDA(cudaStreamSynchronize(st));
    BoxPart r;
    for (int s = 0; s < 3; ++s) {
        r.v[2 * s] = FLT_MAX;
        r.v[2 * s + 1] = FLT_MIN;
        r.i[2 * s] = r.i[2 * s + 1] = -1;
    }
    for (const BoxPart &p : part) {
        for (int s = 0; s < 3; ++s) {
            take_lo(r.v[2 * s], r.i[2 * s], p.v[2 * s], p.i[2 * s]);
            take_hi(r.v[2 * s + 1], r.i[2 * s + 1], p.v[2 * s + 1], p.i[2 * s + 1]);
        }
    }
    // inertia tensor: moments about the six axes xx, yy, zz, xy, yz, zx seen
    // in the rotated frame
    const double num = 1.0 / sqrt(2.0);
    const double axe[6][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0},
                              {num, num, 0.0}, {0.0, num, num}, {num, 0.0, num}};
    const double inv[3][3] = {{R[0][0], R[1][0], R[2][0]}, {R[0][1], R[1][1], R[2][1]}, {R[0][2], R[1][2], R[2][2]}};
    const double *I = inertia;  // rows xx xy xz / yx yy yz / zx zy zz
    double m[6];
    for (int q = 0; q < 6; ++q) {
        const double ax = dot3(inv[0], axe[q]), ay = dot3(inv[1], axe[q]), az = dot3(inv[2], axe[q]);
        m[q] = I[0] * ax * ax + I[4] * ay * ay + I[8] * az * az + 2.0 * I[1] * ax * ay + 2.0 * I[5] * ay * az +
               2.0 * I[6] * az * ax;
    }
    const double It[9] = {m[0], -m[3], -m[5], -m[3], m[1], -m[4], -m[5], -m[4], m[2]};
    for (int q = 0; q < 9; ++q) inertia[q] = It[q];
    // the centroid last, entering the box after the vertices
    double c[3] = {centroid[0], centroid[1], centroid[2]};
    move_point(M, c);
    for (int s = 0; s < 3; ++s) {
        centroid[s] = c[s];
        box[2 * s] = (r.v[2 * s] < c[s]) ? r.v[2 * s] : c[s];
        box[2 * s + 1] = (r.v[2 * s + 1] > c[s]) ? r.v[2 * s + 1] : c[s];
    }
    return ACFD_OK;
}

// the device surface of body n to the host (null outputs are skipped)
int ib_fetch(IbState *ib, int n, double *v, double *Nf, double *Ne, double *Nv, cudaStream_t st)
{
    if (!ib || n < 0 || n >= ib->count) {
        set_error("acfd_geo_fetch: body %d of %d", n, ib ? ib->count : 0);
        return ACFD_ERR_ARG;
    }
    const DevBody &B = ib->host[n];
    if (B.faceN <= 0 || !B.v) {
        set_error("acfd_geo_fetch: body %d is not triangulated", n);
        return ACFD_ERR_ARG;
    }
    const double *from[4] = {B.v, B.Nf, B.Ne, B.Nv};
    double *to[4] = {v, Nf, Ne, Nv};
    const int rows[4] = {B.vertN, B.faceN, B.edgeN, B.vertN};
    for (int a = 0; a < 4; ++a) {
        if (!to[a]) continue;
        ACFD_CUDA(cudaMemcpyAsync(to[a], from[a], sizeof(double) * 3 * rows[a], cudaMemcpyDeviceToHost, st));
    }
    ACFD_CUDA(cudaStreamSynchronize(st));
    return ACFD_OK;
}

int ib_check(IbState *ib, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    return read_status(ib, st);
}

int ib_compute_geometric_field(IbState *ib, const Grid &g, const ModelParams &m, const acfd_partition_t &part,
                               double *U, int *flags, cudaStream_t st)
{
    if (!ib || ib->count == 0) return ACFD_OK;
    const IbGrid G = make_ibgrid(g, part, m.ibmLayer);
    if (ib->joined_n < g.nn) {
        cudaFree(ib->joined);
        ib->joined = nullptr;
        ACFD_CUDA(cudaMalloc(&ib->joined, (size_t)g.nn));
        ib->joined_n = g.nn;
    }
    const long long pin = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    map_init<<<blocks_for(pin, 256), 256, 0, st>>>(g, ib->dev, flags);
    ACFD_CUDA(cudaGetLastError());
    static bool attr_set = false;
    if (!attr_set) {
        ACFD_CUDA(cudaFuncSetAttribute(map_body, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double) * 9 * kMaxSmemFacets)));
        attr_set = true;
    }
    for (int n = 0; n < ib->count; ++n) {
        const DevBody &B = ib->host[n];
        if (B.state == 1) continue;
        BoxList bl;
        bl.body0 = n;
        bl.nb = 1;
        body_box(part, B, bl.lo[0], bl.ext[0]);
        bl.start[0] = 0;
        bl.start[1] = (long long)bl.ext[0][0] * bl.ext[0][1] * bl.ext[0][2];
        if (bl.start[1] == 0) continue;
        const size_t smem = (B.faceN > 0 && B.faceN <= kMaxSmemFacets) ? sizeof(double) * 9 * B.faceN : 0;
        // a warp per node, at most two resident blocks per SM (staged facets)
        const long long want = (bl.start[1] + kMapThreads / 32 - 1) / (kMapThreads / 32);
        const unsigned blocks = (unsigned)std::min<long long>(want, 2LL * 148);
        map_body<<<blocks, kMapThreads, smem, st>>>(G, ib->dev, n, bl, flags, ib->status);
        ACFD_CUDA(cudaGetLastError());
    }
    map_interface<<<blocks_for(pin, 256), 256, 0, st>>>(G, flags, ib->joined);
    ACFD_CUDA(cudaGetLastError());
    map_refill<<<blocks_for(pin, 128), 128, 0, st>>>(G, m, U, flags, ib->joined, ib->status);
    ACFD_CUDA(cudaGetLastError());
    if (part.gl >= 1) {
        const int rc = build_lists(ib, G, part, flags, st);
        if (rc != ACFD_OK) return rc;
    }
    return read_status(ib, st);
}

}  // namespace acfd

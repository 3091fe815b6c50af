// Plane-march stage kernels (fast FP64, FP32 and hybrid forms).
//
// Y and Z sweeps:
// A block owns a tile of grid lines along the sweep axis s: WX consecutive x
// by NR consecutive rows of the other transverse axis, over one segment of
// the line.  It walks the segment plane by plane:
//  * a producer warp streams the planes of U[tn] (the tile plus a one-node
//    halo in x and in the rows, all five variables) into a ring of
//    kPlaneSlots shared-memory slots with TMA copies, two planes ahead of the
//    consumers (full/empty mbarrier pair per slot);
//  * every consumer thread walks one line: its stencil window (nodes p-2..p+3
//    of interface p+1/2) lives in registers and gains one node per plane, the
//    transverse differences of the viscous flux come from the halo'd plane
//    in shared memory, and the node update reads U[tn] of its node from the
//    ring.
// Every plane of U[tn] crosses from L2 once per tile (halo included), and the
// loads run ahead of the arithmetic without holding registers.  The direct
// loads of other levels (U[to] at the node) go to L2 (__ldcg): a block of the
// persistent batch kernel may read a level that another SM rewrote since this
// SM last cached it in L1.
//
// Included after sweep_march.cuh by sweep_fast.cu and sweep_fp32.cu.
#pragma once

#include <utility>

#include "sweep_march.cuh"

namespace acfd {
namespace ACFD_NS {

constexpr long long kPlaneWaitLimit = kWaitLimitDefault;

// Items of a plane-march block (both kernels march along y, or along z with
// the axes exchanged, over tiles of x by rows).  With shares (SHARE) a block
// marches positions [w, r1) of the list of all tiles' lines in chunk-major
// order: the lines are cut into pt.nseg chunks, and chunk c of every tile
// comes before chunk c+1 of any tile, so that blocks of neighbouring tiles
// march the same planes at the same time (their halo rows are shared in L2)
// while every block of the launch gets the same number of planes.  A share
// that crosses the end of a (chunk, tile) piece is two items, marched one
// after the other through the same ring.  Without shares a block marches
// segment blk / tiles of tile blk % tiles.  Returns false when the block has
// no item left; otherwise the item's tile T and planes [p0, p1) counted from
// the first computed node of the march axis, and w moves past the item.
template <bool SHARE>
__device__ __forceinline__ bool plane_next_item(const PlaneTile &pt, int Ls, long long tiles, int blk, long long r1,
                                                long long &w, long long &T, int &p0, int &p1)
{
    if (w >= r1) return false;
    const int nch = pt.nseg;
    auto plo = [&](int c) { return (int)((long long)c * Ls / nch); };  // first plane of chunk c
    if constexpr (SHARE) {
        int c = (int)((w / tiles) * nch / Ls);
        while (c + 1 < nch && tiles * plo(c + 1) <= w) ++c;
        while (c > 0 && tiles * plo(c) > w) --c;
        const int len = plo(c + 1) - plo(c);
        const long long rel = w - tiles * plo(c);
        T = rel / len;
        const int o = (int)(rel - T * len);
        const int n = (int)((r1 - w < (long long)(len - o)) ? r1 - w : (long long)(len - o));
        p0 = plo(c) + o;
        p1 = p0 + n;
        w += n;
    } else {
        T = blk % tiles;
        const int seg = (int)(blk / tiles);
        p0 = plo(seg);
        p1 = plo(seg + 1);
        w = r1;
    }
    return true;
}

// the first and one past the last list position of block blk's share
__device__ __forceinline__ void plane_share(const PlaneTile &pt, int Ls, long long tiles, int blk, long long &r0,
                                           long long &r1)
{
    const long long work = tiles * Ls;
    r0 = (long long)blk * work / pt.nblk;
    r1 = (long long)(blk + 1) * work / pt.nblk;
}

// One instantiation serves both axes: the kernel is written for the Y sweep
// (S = 1, rows along z).  A Z sweep runs it on a grid descriptor with axes 1
// and 2 exchanged (pt.swap = 1): the line and row strides come from pt, the
// momentum components rho*v and rho*w trade places in every read of the
// planes and of U[to] and in every write of U[tm], and the TMA coordinates of
// a plane are (x, row, position) instead of (x, position, row).
//
// The block body is a device function of the block's index within the launch
// (blk) so that the batched kernel runs the same code for a block of any case;
// warps beyond the case's producer warp (a batch launch sized for its largest
// tile) leave after the barrier set-up.
template <int NP, bool VISC, bool HYB, bool SHARE = false>
__device__ __forceinline__ void plane_yz_block(const Grid &g, const ModelParams &mp, const StageArgs &a,
                                               const PlaneTile &pt, const CUtensorMap *mapp, int blk,
                                               unsigned char *smem)
{
    constexpr int S = 1;
    constexpr int T2 = 2;
    constexpr int H = NP / 2;
    constexpr int hv = VISC ? 1 : 0;
    constexpr int NS = kPlaneSlots;
    constexpr unsigned kAll = 0xffffffffu;
    const int pe = pt.BXp * pt.BC;  // elements of one variable in a plane
    const int plane_bytes = pe * 5 * 8;
    const int slot_doubles = plane_slot_bytes(pt.BXp, pt.BC) / 8;  // 128-byte aligned slots
    double *ring = reinterpret_cast<double *>(smem);
    Real *coop = reinterpret_cast<Real *>(smem + (size_t)NS * slot_doubles * 8);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)NS * slot_doubles * 8 + (size_t)pt.ncw * kCoopBytes);
    uint64_t *empty = full + NS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NS; ++q) {
            tma::mbar_init(full + q, 1);
            tma::mbar_init(empty + q, pt.ncw);
        }
    }
    __syncthreads();
    pdl_wait();
    if (warp > pt.ncw) {
        return;
    }

    // the items of the block (plane_next_item); the plane sequence q of the
    // ring runs on from one item to the next
    const int Ls = g.hi[S] - g.lo[S];
    const long long tiles = (long long)pt.ntx * pt.ntc;
    long long r0 = 0, r1 = 1;
    if constexpr (SHARE) {
        plane_share(pt, Ls, tiles, blk, r0, r1);
        if (r1 <= r0) return;
    }
    // the item at list position w: tile origin, planes [p0, p1); w moves past it
    auto next_item = [&](long long &w, int &x0, int &c0, int &p0, int &p1) {
        long long T;
        if (!plane_next_item<SHARE>(pt, Ls, tiles, blk, r1, w, T, p0, p1)) return false;
        p0 += g.lo[S];
        p1 += g.lo[S];
        x0 = g.lo[0] + (int)(T % pt.ntx) * pt.WX;
        c0 = g.lo[T2] + (int)(T / pt.ntx) * pt.NR;
        return true;
    };

    if (warp == pt.ncw) {
        // producer: plane q of the block's sequence into slot q % NS
        if (lane == 0) {
            int q = 0, issued = 0;
            bool ok = true;
            long long w = r0;
            int x0, c0, p0, p1;
            while (ok && next_item(w, x0, c0, p0, p1)) {
                const int xs = (x0 - hv) & ~1, cs = c0 - hv;
                const int NQ = p1 - p0 + 2 * H;  // planes p0-H .. p1+H-1
                for (int ql = 0; ql < NQ; ++ql, ++q) {
                    const int slot = q % NS;
                    if (q >= NS && !tma::mbar_wait_bounded(empty + slot, ((q / NS) - 1) & 1, a.status, 5,
                                                           a.wait_limit)) {
                        ok = false;
                        break;
                    }
                    tma::mbar_expect_tx(full + slot, plane_bytes);
                    const int pos = p0 - H + ql;
                    double *dst = ring + (size_t)slot * slot_doubles;
                    if (!pt.swap) {
                        tma::load_5d(dst, mapp, xs, pos, cs, 0, a.tn, full + slot);
                    } else {
                        tma::load_5d(dst, mapp, xs, cs, pos, 0, a.tn, full + slot);
                    }
                    issued = q + 1;
                }
            }
            // the block must not end with copies in flight
            for (int qq = issued - NS > 0 ? issued - NS : 0; qq < issued; ++qq) {
                tma::mbar_wait_bounded(full + qq % NS, (qq / NS) & 1, a.status, 5, kPlaneWaitLimit);
            }
        }
        return;
    }

    int qbase = 0;  // first plane of the item in the block's sequence
    long long wi = r0;
    int x0, c0, p0, p1;
    while (next_item(wi, x0, c0, p0, p1)) {
        const int xs = (x0 - hv) & ~1;
        const int NQ = p1 - p0 + 2 * H;

        // consumer thread: line (i, c)
        const int t = threadIdx.x;
        const int xl = t % pt.WX, rl = t / pt.WX;
        const int i = x0 + xl, c = c0 + rl;
        const bool active = (rl < pt.NR) && (i < g.hi[0]) && (c < g.hi[T2]);
        // element of (i, c) in a plane (inactive threads: the tile's first node,
        // whose halo neighbours exist)
        const int e0 = active ? (rl + hv) * pt.BXp + (i - xs) : hv * pt.BXp + (x0 - xs);
        const long long nn = g.nn;
        const long long st = pt.st;                      // node stride along the line
        const long long base = (long long)c * pt.rs + i;  // node (i, c) at position 0
        // variable v of the kernel's frame is variable vg(v) of the state
        const int o2 = pt.swap ? 3 : 2, o3 = pt.swap ? 2 : 3;
        auto vg = [&](int v) { return v == 2 ? o2 : (v == 3 ? o3 : v); };
        const Real cvinv = Real(1.0 / mp.cv);
        const bool same_o = (a.Uo == a.Un);
        const double rdt = (a.dt_scale * a.dt[0]) * g.dd[S];
        // plane q of the item is plane qbase + q of the block's sequence
        auto plane = [&](int q) { return ring + (size_t)((qbase + q) % NS) * slot_doubles; };
        auto wait_plane = [&](int q) {
            const int qq = qbase + q;
            const bool ok = tma::mbar_wait_bounded(full + qq % NS, (qq / NS) & 1, a.status, 5, a.wait_limit);
            return __all_sync(kAll, ok);
        };
        auto release = [&](int q) {
            __syncwarp();
            if (lane == 0) tma::mbar_arrive(empty + (qbase + q) % NS);
        };
        auto node_of_plane = [&](const double *P, Real w[5]) {
    #pragma unroll
            for (int v = 0; v < 5; ++v) w[v] = Real(P[vg(v) * pe + e0]);
        };
        // transverse differences at the plane's node from its halo neighbours:
        // axis 0 (x, element stride 1) and axis T2 (rows, element stride BXp)
        auto tdiff = [&](const double *P, Real (&D)[2][2]) {
    #pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int tax = q == 0 ? 0 : T2;
                const int es = q == 0 ? 1 : pt.BXp;
                const int ep = e0 + es, em = e0 - es;
                const Real rp = fast::rcp<Real>(Real(P[ep])), rm = fast::rcp<Real>(Real(P[em]));
                const int ot = vg(1 + tax) * pe, os = vg(1 + S) * pe;
                const Real tp = Real(P[ot + ep]), tm = Real(P[ot + em]);
                const Real sp = Real(P[os + ep]), sm = Real(P[os + em]);
                D[q][0] = fast::diff_prod(tp, rp, tm, rm);
                D[q][1] = fast::diff_prod(sp, rp, sm, rm);
            }
        };

        // A wait that gave up ends the block's march.  The FP64 form marks it
        // and leaves at the end of the item, so that the march loop keeps a
        // single exit (measured: FP64 stages 4% faster); the FP32 forms leave
        // at once (measured: hybrid step 0.8% faster than with the mark).
        constexpr bool kMarkFailure = sizeof(Real) == sizeof(double);
        bool failed = false;
        Real W[NP][5];
    #pragma unroll
        for (int m = 0; m < NP - 1; ++m) {
            if constexpr (kMarkFailure) {
                if (!failed && !wait_plane(m)) failed = true;
            } else {
                if (!wait_plane(m)) return;
            }
            node_of_plane(plane(failed ? 0 : m), W[m]);
        }
        Real Pc[4] = {Real(0), Real(0), Real(0), Real(0)};
        Real Dc[2][2] = {{Real(0), Real(0)}, {Real(0), Real(0)}};
        if (VISC) {
            march_prims(W[H - 1], cvinv, Pc);
            tdiff(plane(failed ? 0 : H - 1), Dc);
        }
        for (int q = 0; q < H; ++q) {
            release(q);  // nodes p0-H .. p0-1 have no update
        }
        const uint8_t *__restrict__ fl = HYB ? a.flags + (long long)(pt.swap ? 2 : 1) * nn : nullptr;
        unsigned fw = 0;
        unsigned fl_ahead = 0;  // flag of node p+2, loaded one plane ahead of its use
        if (HYB && active) {
            fw = (unsigned)fl[base + (long long)(p0 - 2) * st] | ((unsigned)fl[base + (long long)(p0 - 1) * st] << 1) |
                 ((unsigned)fl[base + (long long)p0 * st] << 2);
            fl_ahead = fl[base + (long long)(p0 + 1) * st];
        }
        Real Fl[5];
        for (int p = p0 - 1; p < p1 && !failed; ++p) {
            const int qf = p - p0 + 2 * H;  // front node p+H
            const int q0 = p - p0 + H;      // node p
            const long long id = base + (long long)p * st;
            int did = 1;
            double uo[5];
            if (active && p >= p0) {
                did = a.did[id];
                if (!same_o && !a.accumulate) {
    #pragma unroll
                    for (int v = 0; v < 5; ++v) uo[v] = __ldcg(a.Uo + vg(v) * nn + id);
                }
            }
            bool full_w = true;
            if (HYB) {
                fw |= fl_ahead << 3;
                if (active) fl_ahead = fl[id + 3 * st];  // node p+3 <= p1+2, inside the march's planes
                full_w = (fw != 0u);
            }
            if (!wait_plane(qf)) {
                if constexpr (kMarkFailure) {
                    failed = true;
                    break;
                } else {
                    return;
                }
            }
            node_of_plane(plane(qf), W[NP - 1]);
            Real Pn[4], Dn[2][2];
            if (VISC) {
                march_prims(W[H], cvinv, Pn);
                tdiff(plane(q0 + 1), Dn);
            }
            Real F[5];
            if constexpr (HYB && NP == 6) {
                march_flux_coop<S>(mp, W, full_w, F, coop + (size_t)warp * (kCoopBytes / sizeof(Real)));
            } else {
                march_flux<S, NP, HYB>(mp, W, full_w, F);
            }
            if (VISC) {
                march_visc<S>(g, mp, Pc, Pn, Dc, Dn, F);
            }
            if (p >= p0) {
                if (active && did == 0) {
                    const double *P = plane(q0);
    #pragma unroll
                    for (int v = 0; v < 5; ++v) {
                        const double phi = double(Fl[v]) - double(F[v]);
                        const long long qv = vg(v) * nn + id;
                        const double un = P[vg(v) * pe + e0];
                        if (a.accumulate) {
                            a.Um[qv] = __ldcg(a.Um + qv) + a.coeB * rdt * phi;
                        } else {
                            a.Um[qv] = a.coeA * (same_o ? un : uo[v]) + a.coeB * (un + rdt * phi);
                        }
                    }
                }
                release(q0);
            }
    #pragma unroll
            for (int v = 0; v < 5; ++v) Fl[v] = F[v];
    #pragma unroll
            for (int m = 0; m < NP - 1; ++m) {
    #pragma unroll
                for (int v = 0; v < 5; ++v) W[m][v] = W[m + 1][v];
            }
            if (VISC) {
    #pragma unroll
                for (int q = 0; q < 4; ++q) Pc[q] = Pn[q];
    #pragma unroll
                for (int q = 0; q < 2; ++q) {
                    Dc[q][0] = Dn[q][0];
                    Dc[q][1] = Dn[q][1];
                }
            }
            fw >>= 1;
        }
        if constexpr (SHARE) {
            // planes p1 .. p1+H-1 were read for the last time: free their slots
            // for the next item's planes
            for (int q = NQ - H; q < NQ && !failed; ++q) {
                release(q);
            }
        }
        if (failed) return;
        qbase += NQ;
    }
}

template <int NP, bool VISC, bool HYB, bool SHARE>
__global__ void __launch_bounds__(kPlaneMaxThreads, sizeof(Real) == sizeof(float) ? 2 : 1)
stage_plane_yz(Grid g, ModelParams mp, StageArgs a, PlaneTile pt, const __grid_constant__ CUtensorMap map)
{
    extern __shared__ __align__(128) unsigned char smem[];
    plane_yz_block<NP, VISC, HYB, SHARE>(g, mp, a, pt, &map, (int)blockIdx.x, smem);
}

// ---------------------------------------------------------------------------
// X sweep: the block marches along y over a tile of WX nodes along x by NR
// z-rows.  Each consumer thread owns one interface of its row (WX + 1 per
// row, the first one only feeds its right neighbour): the x stencil comes
// from the plane in shared memory (x halo of three nodes), the viscous
// y differences from the neighbouring planes of the ring and the z
// differences from the neighbouring rows of the plane.  Interface fluxes go
// to the node on their right through a double-buffered shared array, one
// named barrier of the consumer warps per plane.
// ---------------------------------------------------------------------------

// the item of an X-sweep block at list position w (plane_next_item): tile
// origin (x0, c0) and rows [j0, j1) along y; w moves past it
template <bool SHARE>
__device__ __forceinline__ bool plane_x_item(const Grid &g, const PlaneTile &pt, long long tiles, int blk,
                                             long long r1, long long &w, int &x0, int &c0, int &j0, int &j1)
{
    long long T;
    if (!plane_next_item<SHARE>(pt, g.hi[1] - g.lo[1], tiles, blk, r1, w, T, j0, j1)) return false;
    j0 += g.lo[1];
    j1 += g.lo[1];
    x0 = g.lo[0] + (int)(T % pt.ntx) * pt.WX;
    c0 = g.lo[2] + (int)(T / pt.ntx) * pt.NR;
    return true;
}

// producer lane of an X-sweep block: the planes of rows j0-hv .. j1-1+hv of
// every item, plane q of the block's sequence into ring slot q % NS; the
// block does not end with copies in flight
template <int H, int hv, int NS, bool SHARE>
__device__ __forceinline__ void plane_x_produce(const Grid &g, const StageArgs &a, const PlaneTile &pt,
                                                const CUtensorMap *mapp, int blk, long long r0, long long r1,
                                                double *ring, uint64_t *full, uint64_t *empty)
{
    const int plane_bytes = pt.BXp * pt.BC * 5 * 8;
    const int slot_doubles = plane_slot_bytes(pt.BXp, pt.BC) / 8;
    const long long tiles = (long long)pt.ntx * pt.ntc;
    int q = 0, issued = 0;
    bool ok = true;
    long long w = r0;
    int x0, c0, j0, j1;
    while (ok && plane_x_item<SHARE>(g, pt, tiles, blk, r1, w, x0, c0, j0, j1)) {
        const int xs = (x0 - H) & ~1, cs = c0 - hv;
        const int NQ = j1 - j0 + 2 * hv;  // rows j0-hv .. j1-1+hv
        for (int ql = 0; ql < NQ; ++ql, ++q) {
            const int slot = q % NS;
            if (q >= NS && !tma::mbar_wait_bounded(empty + slot, ((q / NS) - 1) & 1, a.status, 5, a.wait_limit)) {
                ok = false;
                break;
            }
            tma::mbar_expect_tx(full + slot, plane_bytes);
            tma::load_5d(ring + (size_t)slot * slot_doubles, mapp, xs, j0 - hv + ql, cs, 0, a.tn, full + slot);
            issued = q + 1;
        }
    }
    for (int qq = issued - NS > 0 ? issued - NS : 0; qq < issued; ++qq) {
        tma::mbar_wait_bounded(full + qq % NS, (qq / NS) & 1, a.status, 5, kPlaneWaitLimit);
    }
}

// named barrier 1 of the nbar consumer threads, or-reducing `abort`: the
// consumer warps leave together when a wait of one of them gave up
__device__ __forceinline__ bool consumers_barrier_or(bool abort, unsigned nbar)
{
    unsigned any;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 q, %1, 0;\n\t"
        "bar.red.or.pred p, 1, %2, q;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(any)
        : "r"((unsigned)abort), "r"(nbar)
        : "memory");
    return any != 0u;
}

template <int NP, bool VISC, bool HYB, bool SHARE = false>
__device__ __forceinline__ void plane_x_block(const Grid &g, const ModelParams &mp, const StageArgs &a,
                                              const PlaneTile &pt, const CUtensorMap *mapp, int blk,
                                              unsigned char *smem)
{
    constexpr int H = NP / 2;
    constexpr int hv = VISC ? 1 : 0;
    constexpr int NS = kPlaneSlots;
    constexpr unsigned kAll = 0xffffffffu;
    const int pe = pt.BXp * pt.BC;
    const int slot_doubles = plane_slot_bytes(pt.BXp, pt.BC) / 8;
    const int nflux = pt.TR * pt.NR;
    double *ring = reinterpret_cast<double *>(smem);
    Real *sF = reinterpret_cast<Real *>(smem + (size_t)NS * slot_doubles * 8);
    Real *coop = reinterpret_cast<Real *>(smem + (size_t)NS * slot_doubles * 8 + plane_flux_bytes(nflux));
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + (size_t)NS * slot_doubles * 8 + plane_flux_bytes(nflux) +
                                                  (size_t)pt.ncw * kCoopBytes);
    uint64_t *empty = full + NS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int q = 0; q < NS; ++q) {
            tma::mbar_init(full + q, 1);
            tma::mbar_init(empty + q, pt.ncw);
        }
    }
    __syncthreads();
    pdl_wait();
    if (warp > pt.ncw) {
        return;
    }
    // the items of the block (plane_x_item); the plane sequence q of the
    // ring runs on from item to item
    const long long tiles = (long long)pt.ntx * pt.ntc;
    long long r0 = 0, r1 = 1;
    if constexpr (SHARE) {
        plane_share(pt, g.hi[1] - g.lo[1], tiles, blk, r0, r1);
        if (r1 <= r0) return;
    }
    if (warp == pt.ncw) {
        if (lane == 0) plane_x_produce<H, hv, NS, SHARE>(g, a, pt, mapp, blk, r0, r1, ring, full, empty);
        return;
    }

    const unsigned nbar = (unsigned)pt.ncw * 32u;
    int qbase = 0;  // first plane of the item in the block's sequence
    int buf = 0;    // flux buffer of the row
    long long wi = r0;
    int x0, c0, j0, j1;
    while (plane_x_item<SHARE>(g, pt, tiles, blk, r1, wi, x0, c0, j0, j1)) {
        const int xs = (x0 - H) & ~1;
        const int NQ = j1 - j0 + 2 * hv;

        // consumer thread: interface xi+1/2 of z-row c
        const int t = threadIdx.x;
        const int xl = t % pt.TR, rl = t / pt.TR;
        const int xi = x0 - 1 + xl;
        const int c = c0 + rl;
        const bool row_ok = (rl < pt.NR) && (c < g.hi[2]);
        const bool active = row_ok && (xi < g.hi[0]);          // interface computed
        const bool upd = active && xl >= 1;                      // node xi updated
        // element of node xi in a plane (inactive threads: the tile's first node)
        const int e0 = active ? (rl + hv) * pt.BXp + (xi - xs) : hv * pt.BXp + (x0 - xs);
        const long long nn = g.nn;
        const long long sy = (long long)g.pitch, sz = (long long)g.pitch * g.n[1];
        const long long xz = (long long)c * sz + xi;
        const Real cvinv = Real(1.0 / mp.cv);
        const bool same_o = (a.Uo == a.Un);
        const double rdt = (a.dt_scale * a.dt[0]) * g.dd[0];
        const uint8_t *__restrict__ fl = a.flags;  // sweep 0 flags
        // plane q of the item is plane qbase + q of the block's sequence
        auto plane = [&](int q) { return ring + (size_t)((qbase + q) % NS) * slot_doubles; };
        auto wait_plane = [&](int q) {
            const int qq = qbase + q;
            const bool ok = tma::mbar_wait_bounded(full + qq % NS, (qq / NS) & 1, a.status, 5, a.wait_limit);
            return __all_sync(kAll, ok);
        };
        auto release = [&](int q) {
            __syncwarp();
            if (lane == 0) tma::mbar_arrive(empty + (qbase + q) % NS);
        };
        bool ok = true;
        for (int q = 0; q < 2 * hv; ++q) {
            ok = ok && wait_plane(q);  // rows j0-1 and j0 (viscous)
        }
        // sensor flags of the interface's nodes xi-1 .. xi+2 and the did of node
        // xi, loaded one row ahead of their use
        auto row_flags = [&](long long idr) {
            return (unsigned)(fl[idr - 1] | fl[idr] | fl[idr + 1] | fl[idr + 2]);
        };
        unsigned fl_n = (HYB && active) ? row_flags(xz + (long long)j0 * sy) : 1u;
        int did_n = upd ? a.did[xz + (long long)j0 * sy] : 1;
        for (int j = j0; j < j1; ++j) {
            const int q = j - j0 + hv;  // plane of row j
            const long long id = xz + (long long)j * sy;
            const int did = did_n;
            const unsigned fl_j = fl_n;
            if (j + 1 < j1) {
                if (upd) did_n = a.did[id + sy];
                if (HYB && active) fl_n = row_flags(id + sy);
            }
            double uo[5];
            if (upd && !same_o && !a.accumulate) {
    #pragma unroll
                for (int v = 0; v < 5; ++v) uo[v] = __ldcg(a.Uo + v * nn + id);
            }
            const bool full_w = !HYB || fl_j != 0u;
            ok = ok && wait_plane(q + hv);  // row j+1 (viscous) or j
            const double *P = plane(ok ? q : 0);
            Real W[NP][5];
    #pragma unroll
            for (int m = 0; m < NP; ++m) {
    #pragma unroll
                for (int v = 0; v < 5; ++v) W[m][v] = Real(P[v * pe + e0 - (H - 1) + m]);
            }
            Real F[5];
            if constexpr (HYB && NP == 6) {
                march_flux_coop<0>(mp, W, full_w, F, coop + (size_t)warp * (kCoopBytes / sizeof(Real)));
            } else {
                march_flux<0, NP, HYB>(mp, W, full_w, F);
            }
            if (VISC) {
                Real Pc[4], Pn[4], Dc[2][2], Dn[2][2];
                march_prims(W[H - 1], cvinv, Pc);
                march_prims(W[H], cvinv, Pn);
                const double *Pm = plane(q - 1), *Pp = plane(q + 1);
    #pragma unroll
                for (int side = 0; side < 2; ++side) {
                    const int e = e0 + side;
                    Real(&D)[2][2] = side ? Dn : Dc;
                    // y: planes j+1 and j-1 (v and u)
                    {
                        const Real rp = fast::rcp<Real>(Real(Pp[e])), rm = fast::rcp<Real>(Real(Pm[e]));
                        D[0][0] = fast::diff_prod(Real(Pp[2 * pe + e]), rp, Real(Pm[2 * pe + e]), rm);
                        D[0][1] = fast::diff_prod(Real(Pp[pe + e]), rp, Real(Pm[pe + e]), rm);
                    }
                    // z: rows c+1 and c-1 of plane j (w and u)
                    {
                        const int ep = e + pt.BXp, em = e - pt.BXp;
                        const Real rp = fast::rcp<Real>(Real(P[ep])), rm = fast::rcp<Real>(Real(P[em]));
                        D[1][0] = fast::diff_prod(Real(P[3 * pe + ep]), rp, Real(P[3 * pe + em]), rm);
                        D[1][1] = fast::diff_prod(Real(P[pe + ep]), rp, Real(P[pe + em]), rm);
                    }
                }
                march_visc<0>(g, mp, Pc, Pn, Dc, Dn, F);
            }
            Real *sFb = sF + (size_t)buf * nflux * 5;
            if (active) {
    #pragma unroll
                for (int v = 0; v < 5; ++v) sFb[v * nflux + t] = F[v];
            }
            if (consumers_barrier_or(!ok, nbar)) {
                return;
            }
            if (upd && did == 0) {
    #pragma unroll
                for (int v = 0; v < 5; ++v) {
                    const double phi = double(sFb[v * nflux + t - 1]) - double(F[v]);
                    const long long qv = v * nn + id;
                    const double un = P[v * pe + e0];
                    if (a.accumulate) {
                        a.Um[qv] = __ldcg(a.Um + qv) + a.coeB * rdt * phi;
                    } else {
                        a.Um[qv] = a.coeA * (same_o ? un : uo[v]) + a.coeB * (un + rdt * phi);
                    }
                }
            }
            // the plane of row j-1 (viscous) or j is read for the last time
            release(q - hv);
            buf ^= 1;
        }
        if constexpr (SHARE) {
            // rows j1-1 and j1 (viscous) were read for the last time: free their
            // slots for the next item's planes
            for (int q = NQ - 2 * hv; q < NQ; ++q) {
                release(q);
            }
        }
        qbase += NQ;
    }
}


template <int NP, bool VISC, bool HYB, bool SHARE>
__global__ void __launch_bounds__(kPlaneMaxThreads, sizeof(Real) == sizeof(float) ? 2 : 1)
stage_plane_x(Grid g, ModelParams mp, StageArgs a, PlaneTile pt, const __grid_constant__ CUtensorMap map)
{
    extern __shared__ __align__(128) unsigned char smem[];
    plane_x_block<NP, VISC, HYB, SHARE>(g, mp, a, pt, &map, (int)blockIdx.x, smem);
}

template <int NP, bool VISC, bool HYB, bool SHARE>
static int launch_plane_x(const Grid &g, const ModelParams &m, const StageArgs &a, const PlaneTile &pt,
                          const CUtensorMap &map, cudaStream_t st)
{
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    const int smem = plane_smem_bytes(pt, 0);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_plane_x<NP, VISC, HYB, SHARE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             kPlaneSmemMax);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_plane_x)");
        configured[dev] = true;
    }
    if (smem > kPlaneSmemMax) {
        set_error("plane tile needs %d bytes of shared memory", smem);
        return ACFD_ERR_ARG;
    }
    const unsigned blocks = (unsigned)pt.nblk;
    cudaError_t e = launch_k(stage_plane_x<NP, VISC, HYB, SHARE>, dim3(blocks), dim3((pt.ncw + 1) * 32), smem, st, g, m, a,
                             pt, map);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_plane_x launch");
}

template <int NP, bool VISC, bool HYB, bool SHARE>
static int launch_plane_yz(const Grid &g, const ModelParams &m, const StageArgs &a, int s, const PlaneTile &pt0,
                           const CUtensorMap &map, cudaStream_t st)
{
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    const int smem = plane_smem_bytes(pt0, s);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_plane_yz<NP, VISC, HYB, SHARE>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kPlaneSmemMax);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_plane_yz)");
        configured[dev] = true;
    }
    if (smem > kPlaneSmemMax) {
        set_error("plane tile needs %d bytes of shared memory", smem);
        return ACFD_ERR_ARG;
    }
    PlaneTile pt = pt0;
    Grid gk = g;
    const long long sy = (long long)g.pitch, sz = (long long)g.pitch * g.n[1];
    if (s == 1) {
        pt.swap = 0;
        pt.st = sy;
        pt.rs = sz;
    } else {
        // the Z sweep as a Y sweep of the grid with axes 1 and 2 exchanged
        pt.swap = 1;
        pt.st = sz;
        pt.rs = sy;
        std::swap(gk.n[1], gk.n[2]);
        std::swap(gk.lo[1], gk.lo[2]);
        std::swap(gk.hi[1], gk.hi[2]);
        std::swap(gk.dd[1], gk.dd[2]);
    }
    const unsigned blocks = (unsigned)pt.nblk;
    cudaError_t e = launch_k(stage_plane_yz<NP, VISC, HYB, SHARE>, dim3(blocks), dim3((pt.ncw + 1) * 32), smem, st, gk,
                             m, a, pt, map);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_plane_yz launch");
}

template <int NP, bool VISC, bool HYB>
static int launch_plane_s(const Grid &g, const ModelParams &m, const StageArgs &a, int s, const PlaneTile &pt,
                          const CUtensorMap &map, cudaStream_t st)
{
    if (s == 0) {
        return pt.share ? launch_plane_x<NP, VISC, HYB, true>(g, m, a, pt, map, st)
                        : launch_plane_x<NP, VISC, HYB, false>(g, m, a, pt, map, st);
    }
    return pt.share ? launch_plane_yz<NP, VISC, HYB, true>(g, m, a, s, pt, map, st)
                    : launch_plane_yz<NP, VISC, HYB, false>(g, m, a, s, pt, map, st);
}

// `map` is the state map with box (BXp, 1, BC) (X and Y sweeps) or
// (BXp, BC, 1) (Z sweep), five variables, one level
static int launch_plane_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                             bool hybrid, const PlaneTile &pt, const CUtensorMap &map, cudaStream_t st)
{
    if (g.hi[0] <= g.lo[0] || g.hi[1] <= g.lo[1] || g.hi[2] <= g.lo[2]) {
        return ACFD_OK;
    }
    if (m.sScheme == 1) {
        if constexpr (sizeof(Real) == sizeof(float)) {
            if (hybrid && a.flags) {
                return viscous ? launch_plane_s<6, true, true>(g, m, a, s, pt, map, st)
                               : launch_plane_s<6, false, true>(g, m, a, s, pt, map, st);
            }
        }
        return viscous ? launch_plane_s<6, true, false>(g, m, a, s, pt, map, st)
                       : launch_plane_s<6, false, false>(g, m, a, s, pt, map, st);
    }
    return viscous ? launch_plane_s<4, true, false>(g, m, a, s, pt, map, st)
                   : launch_plane_s<4, false, false>(g, m, a, s, pt, map, st);
}

#if ACFD_FORM == 2
// ---------------------------------------------------------------------------
// batch: one launch covers the plane-march blocks of every case
// ---------------------------------------------------------------------------
template <int NP, bool VISC, bool HYB, bool XS>
__global__ void __launch_bounds__(kPlaneMaxThreads, 2)
stage_plane_batch(const BatchCase *__restrict__ cases, const BatchPlane *__restrict__ planes,
                  const CUtensorMap *pmaps, const long long *__restrict__ prefix, int ncase, StageCoefs sc,
                  const double *dts, int *status, int s)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const long long item = blockIdx.x;
    int lo = 0, hi = ncase - 1;  // the case whose blocks contain this one
    while (lo < hi) {
        const int mid = (lo + hi + 1) / 2;
        if (prefix[mid] <= item) lo = mid; else hi = mid - 1;
    }
    const BatchCase &C = cases[lo];
    const BatchPlane &P = planes[3 * lo + s];
    StageArgs a;
    const long long lv = 5LL * C.g.nn;
    a.Uo = C.U + sc.to * lv;
    a.Un = C.U + sc.tn * lv;
    a.Um = C.U + sc.tm * lv;
    a.did = C.did;
    a.dt = dts + lo;
    a.dt_scale = sc.dt_scale;
    a.coeA = sc.coeA;
    a.coeB = sc.coeB;
    a.accumulate = 0;
    a.to = sc.to;
    a.tn = sc.tn;
    a.tm = sc.tm;
    a.maps = nullptr;
    a.omaps = nullptr;
    a.var[0] = a.var[1] = a.var[2] = 0;
    a.status = status;
    a.flags = C.flags;
    a.wait_limit = kWaitLimitDefault;
    const int blk = (int)(item - prefix[lo]);
    if (XS) {
        plane_x_block<NP, VISC, HYB>(P.gk, C.mp, a, P.pt, pmaps + 3 * lo + s, blk, smem);
    } else {
        plane_yz_block<NP, VISC, HYB>(P.gk, C.mp, a, P.pt, pmaps + 3 * lo + s, blk, smem);
    }
}

template <bool VISC, bool HYB, bool XS>
static int launch_plane_batch_one(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                  const long long *prefix, long long blocks, int ncase, const StageCoefs &sc,
                                  const double *dts, int *status, int s, int nthreads, int smem, cudaStream_t st)
{
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_plane_batch<6, VISC, HYB, XS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kPlaneSmemMax);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_plane_batch)");
        configured[dev] = true;
    }
    cudaError_t e = launch_k(stage_plane_batch<6, VISC, HYB, XS>, dim3((unsigned)blocks), dim3(nthreads), smem, st,
                             cases, planes, pmaps, prefix, ncase, sc, dts, status, s);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_plane_batch launch");
}

static int launch_plane_batch_impl(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                   const long long *prefix, long long blocks, int ncase, const StageCoefs &sc,
                                   const double *dts, int *status, int s, bool viscous, bool hybrid, int nthreads,
                                   int smem, cudaStream_t st)
{
    if (blocks <= 0) {
        return ACFD_OK;
    }
    if (smem > kPlaneSmemMax || nthreads > kPlaneMaxThreads) {
        set_error("batch plane launch: %d threads, %d bytes of shared memory", nthreads, smem);
        return ACFD_ERR_ARG;
    }
#define ACFD_PB(V_, H_)                                                                                        \
    return (s == 0) ? launch_plane_batch_one<V_, H_, true>(cases, planes, pmaps, prefix, blocks, ncase, sc, dts, \
                                                           status, s, nthreads, smem, st)                       \
                    : launch_plane_batch_one<V_, H_, false>(cases, planes, pmaps, prefix, blocks, ncase, sc, dts, \
                                                            status, s, nthreads, smem, st);
    if (viscous) {
        if (hybrid) { ACFD_PB(true, true) } else { ACFD_PB(true, false) }
    } else {
        if (hybrid) { ACFD_PB(false, true) } else { ACFD_PB(false, false) }
    }
#undef ACFD_PB
}
// ---------------------------------------------------------------------------
// persistent batch step (see PersistStep)
// ---------------------------------------------------------------------------
constexpr long long kPersistWaitLimit = 1LL << 24;  // polls of 64+ ns: about a second or more

// bounded wait until *word >= want (acquire); false when it gave up (status 7,
// abort set) or another block aborted
__device__ __forceinline__ bool persist_wait(const unsigned *word, unsigned want, int *abort, int *status)
{
    for (long long it = 0; it < kPersistWaitLimit; ++it) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(word) : "memory");
        if (v >= want) {
            return true;
        }
        if (*reinterpret_cast<volatile int *>(abort) != 0) {
            return false;
        }
        __nanosleep(64);
    }
    atomicExch(status, 7);
    atomicExch(abort, 1);
    return false;
}

// the full/empty barriers of a plane block of sweep axis s (the layout of
// plane_yz_block and plane_x_block)
__device__ __forceinline__ uint64_t *plane_barriers(const PlaneTile &pt, int s, unsigned char *smem)
{
    const int slot_bytes = plane_slot_bytes(pt.BXp, pt.BC);
    const int nflux = (s == 0) ? pt.TR * pt.NR : 0;
    return reinterpret_cast<uint64_t *>(smem + (size_t)kPlaneSlots * slot_bytes + plane_flux_bytes(nflux) +
                                        (size_t)pt.ncw * kCoopBytes);
}

template <bool VISC, bool HYB, bool XS>
__global__ void __launch_bounds__(kPlaneMaxThreads, 2)
stage_plane_persistent(const BatchCase *__restrict__ cases, const BatchPlane *__restrict__ planes,
                       const CUtensorMap *pmaps, const long long *__restrict__ prefix, int ncase, PersistStep ps,
                       const double *dts, const BatchLevel *__restrict__ levels, const int4 *__restrict__ pairs,
                       const long long *__restrict__ pair_off, const long long *__restrict__ fill_pre,
                       unsigned long long *queue, unsigned *done, unsigned *filled, int *abort, int *status)
{
    extern __shared__ __align__(128) unsigned char smem[];
    // the decoded item, shared by the block; nothing of the loop stays in
    // registers across the item's block body (whose register budget is that
    // of the single-case kernel)
    __shared__ int s_k, s_c, s_blk, s_ok;  // s_blk < 0: fill chunk -s_blk-1 of case s_c
    for (;;) {
        if (threadIdx.x == 0) {
            const long long total = ps.kbase[ps.nk];
            const long long it = (*reinterpret_cast<volatile int *>(abort) != 0)
                                     ? total : (long long)atomicAdd(queue, 1ULL);
            int ok = it < total;
            if (ok) {
                int k = 0;
                while (it >= ps.kbase[k + 1]) ++k;
                const int s = ps.s_of[k];
                const long long local = it - ps.kbase[k];
                const long long *pre = prefix + (long long)s * (ncase + 1);
                int c = 0;
                if (local < ps.ntile[s]) {
                    int hi = ncase - 1;  // the case whose blocks contain this one
                    while (c < hi) {
                        const int mid = (c + hi + 1) / 2;
                        if (pre[mid] <= local) c = mid; else hi = mid - 1;
                    }
                    s_blk = (int)(local - pre[c]);
                    // the fill of the stage before (step-wide index; the first
                    // stage of a launch finds it done by the launch before)
                    const int kg = ps.k0 + k;
                    ok = (kg == 0) || persist_wait(filled + (long long)(kg - 1) * ncase + c,
                                                   (unsigned)(fill_pre[c + 1] - fill_pre[c]), abort, status);
                } else {
                    const long long f = local - ps.ntile[s];
                    int hi = ncase - 1;
                    while (c < hi) {
                        const int mid = (c + hi + 1) / 2;
                        if (fill_pre[mid] <= f) c = mid; else hi = mid - 1;
                    }
                    s_blk = -(int)(f - fill_pre[c]) - 1;
                    ok = persist_wait(done + (long long)(ps.k0 + k) * ncase + c, (unsigned)(pre[c + 1] - pre[c]),
                                      abort, status);
                }
                s_k = k;
                s_c = c;
            }
            s_ok = ok;
        }
        __syncthreads();
        if (!s_ok) {
            break;
        }
        if (s_blk >= 0) {
            // the planes this block's TMA copies read were written by other
            // blocks' ordinary stores
            asm volatile("fence.proxy.async.global;" ::: "memory");
            const int k = s_k, c = s_c, s = ps.s_of[k];
            const BatchCase &C = cases[c];
            const BatchPlane &P = planes[3 * c + s];
            const StageCoefs &sc = ps.sc[k];
            StageArgs a;
            const long long lv = 5LL * C.g.nn;
            a.Uo = C.U + sc.to * lv;
            a.Un = C.U + sc.tn * lv;
            a.Um = C.U + sc.tm * lv;
            a.did = C.did;
            a.dt = dts + c;
            a.dt_scale = sc.dt_scale;
            a.coeA = sc.coeA;
            a.coeB = sc.coeB;
            a.accumulate = 0;
            a.to = sc.to;
            a.tn = sc.tn;
            a.tm = sc.tm;
            a.maps = nullptr;
            a.omaps = nullptr;
            a.var[0] = a.var[1] = a.var[2] = 0;
            a.status = status;
            a.flags = C.flags;
            a.wait_limit = kWaitLimitDefault;
            if constexpr (XS) {
                plane_x_block<6, VISC, HYB>(P.gk, C.mp, a, P.pt, pmaps + 3 * c + s, s_blk, smem);
            } else {
                plane_yz_block<6, VISC, HYB>(P.gk, C.mp, a, P.pt, pmaps + 3 * c + s, s_blk, smem);
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                // the item's barriers are idle (its copies were waited for):
                // invalidate them before the next item initialises its own
                const int c2 = s_c, s2 = ps.s_of[s_k];
                uint64_t *bars = plane_barriers(planes[3 * c2 + s2].pt, s2, smem);
                for (int q = 0; q < 2 * kPlaneSlots; ++q) {
                    tma::mbar_inval(bars + q);
                }
                __threadfence();
                atomicAdd(done + (long long)(ps.k0 + s_k) * ncase + c2, 1u);
            }
        } else {
            // fill chunk of case c: its copy pairs, reading through L2
            const int k = s_k, c = s_c;
            const BatchLevel L = levels[c];
            double *U = L.U + (long long)ps.sc[k].tm * 5 * L.nn;
            const long long t0 = pair_off[c] + (long long)(-s_blk - 1) * kFillChunk;
            const long long t1 = min(pair_off[c + 1], t0 + kFillChunk);
            for (long long t = t0 + threadIdx.x; t < t1; t += blockDim.x) {
                const int4 q = pairs[t];
                double u[5];
#pragma unroll
                for (int v = 0; v < 5; ++v) u[v] = __ldcg(U + v * L.nn + q.z);
#pragma unroll
                for (int v = 0; v < 5; ++v) U[v * L.nn + q.y] = u[v];
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                __threadfence();
                atomicAdd(filled + (long long)(ps.k0 + s_k) * ncase + s_c, 1u);
            }
        }
        __syncthreads();  // the shared item is read by all before thread 0 takes the next
    }
}

template <bool VISC, bool HYB, bool XS>
static int launch_plane_persistent_one(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                       const long long *prefix, int ncase, const PersistStep &ps, const double *dts,
                                       const BatchLevel *levels, const int4 *pairs, const long long *pair_off,
                                       const long long *fill_pre, unsigned long long *queue, unsigned *done,
                                       unsigned *filled, int *abort, int *status, int blocks, int nthreads, int smem,
                                       cudaStream_t st)
{
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_plane_persistent<VISC, HYB, XS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kPlaneSmemMax);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_plane_persistent)");
        configured[dev] = true;
    }
    cudaError_t e = launch_k(stage_plane_persistent<VISC, HYB, XS>, dim3((unsigned)blocks), dim3(nthreads), smem, st,
                             cases, planes, pmaps, prefix, ncase, ps, dts, levels, pairs, pair_off, fill_pre, queue,
                             done, filled, abort, status);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_plane_persistent launch");
}

static int launch_plane_persistent_impl(const BatchCase *cases, const BatchPlane *planes, const CUtensorMap *pmaps,
                                        const long long *prefix, int ncase, const PersistStep &ps, const double *dts,
                                        const BatchLevel *levels, const int4 *pairs, const long long *pair_off,
                                        const long long *fill_pre, unsigned long long *queue, unsigned *done,
                                        unsigned *filled, int *abort, int *status, bool viscous, bool hybrid,
                                        int blocks, int nthreads, int smem, cudaStream_t st)
{
    if (smem > kPlaneSmemMax || nthreads > kPlaneMaxThreads || ps.nk < 1 || ps.nk > kMaxStepStages) {
        set_error("persistent batch launch: %d threads, %d bytes of shared memory, %d stages", nthreads, smem, ps.nk);
        return ACFD_ERR_ARG;
    }
#define ACFD_PP(V_, H_)                                                                                            \
    return (ps.s_of[0] == 0)                                                                                       \
               ? launch_plane_persistent_one<V_, H_, true>(cases, planes, pmaps, prefix, ncase, ps, dts, levels,     \
                                                           pairs, pair_off, fill_pre, queue, done, filled, abort,    \
                                                           status, blocks, nthreads, smem, st)                       \
               : launch_plane_persistent_one<V_, H_, false>(cases, planes, pmaps, prefix, ncase, ps, dts, levels,    \
                                                            pairs, pair_off, fill_pre, queue, done, filled, abort,   \
                                                            status, blocks, nthreads, smem, st);
    if (viscous) {
        if (hybrid) { ACFD_PP(true, true) } else { ACFD_PP(true, false) }
    } else {
        if (hybrid) { ACFD_PP(false, true) } else { ACFD_PP(false, false) }
    }
#undef ACFD_PP
}

static int plane_persistent_occupancy_impl(bool viscous, bool hybrid, int nthreads, int smem, int *blocks_per_sm)
{
    // the smaller of the X and Y/Z kernels' resident blocks
    const void *fns[2] = {viscous ? (hybrid ? (const void *)stage_plane_persistent<true, true, true>
                                            : (const void *)stage_plane_persistent<true, false, true>)
                                  : (hybrid ? (const void *)stage_plane_persistent<false, true, true>
                                            : (const void *)stage_plane_persistent<false, false, true>),
                          viscous ? (hybrid ? (const void *)stage_plane_persistent<true, true, false>
                                            : (const void *)stage_plane_persistent<true, false, false>)
                                  : (hybrid ? (const void *)stage_plane_persistent<false, true, false>
                                            : (const void *)stage_plane_persistent<false, false, false>)};
    *blocks_per_sm = 1 << 30;
    for (const void *fn : fns) {
        int b = 0;
        cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, kPlaneSmemMax);
        if (e == cudaSuccess) {
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, fn, nthreads, smem);
        }
        if (e != cudaSuccess) {
            return cuda_status(e, "persistent batch occupancy");
        }
        *blocks_per_sm = std::min(*blocks_per_sm, b);
    }
    return ACFD_OK;
}
#endif

}  // namespace ACFD_NS
}  // namespace acfd

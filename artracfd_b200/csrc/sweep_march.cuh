// Line-march stage kernels (fast FP64, FP32 and hybrid forms).
//
// One LLLU stage (fluid_dynamics.c:157-274) with every value a thread needs
// kept in registers: no shared-memory brick, no block barrier.
//
//  * Y and Z sweeps (stage_march_yz): one thread per segment of a grid line
//    along the sweep axis s, consecutive threads on consecutive x (coalesced
//    loads).  The thread walks its segment interface by interface with the
//    stencil (nodes p-2..p+3 of interface p+1/2 for WENO5) in a register
//    window: each step loads one new node, computes one interface flux and
//    updates the node left of it with the flux carried from the step before.
//  * X sweeps (stage_march_x): a warp holds 32 consecutive nodes of one
//    x-line; the stencil comes from the neighbouring lanes by warp shuffles,
//    so a warp computes the interfaces of its lanes 2..28 and updates its
//    lanes 3..28 (26 nodes).  The warp walks its segment of y-rows.
//
// Viscous flux: the transverse derivatives at an interface are averages of
// the central differences at its two nodes (diffusive_flux.c:58-312), so a
// thread computes the differences once per node from its transverse
// neighbours and carries them to the next interface.  X sweeps take the y
// differences from the rows they walk through.
//
// Hybrid form: interface p+1/2 uses full WENO5 when the sensor flag of any of
// the nodes p-1..p+2 is set (flags of ghost nodes are always set); otherwise
// the linear-weight limit.
//
// Included after sweep_brick.cuh (IfaceState, back_project) by sweep_fast.cu
// and sweep_fp32.cu.
#pragma once

#include "sweep_brick.cuh"

namespace acfd {
namespace ACFD_NS {

constexpr int kMarchThreads = 256;
// resident blocks per SM the register allocation must allow (128 registers
// per thread at 2)
constexpr int kMarchMinBlocks = 2;

__device__ __forceinline__ void march_load(const double *__restrict__ U, long long nn, long long id, Real w[5])
{
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        w[v] = Real(__ldg(U + v * nn + id));
    }
}

// velocity and temperature of a node; the fused operations are written out
// so that every inlined copy rounds alike (fast::diff_prod)
__device__ __forceinline__ void march_prims(const Real w[5], Real cvinv, Real P[4])
{
    const Real ir = fast::rcp<Real>(w[0]);
    P[0] = w[1] * ir;
    P[1] = w[2] * ir;
    P[2] = w[3] * ir;
    const Real vv = fma(P[2], P[2], fma(P[1], P[1], P[0] * P[0]));
    P[3] = fma(Real(-0.5), vv, w[4] * ir) * cvinv;
}

// the two transverse axes of sweep S, in increasing order
template <int S>
struct Transverse {
    static constexpr int t0 = (S == 0) ? 1 : 0;
    static constexpr int t1 = (S == 2) ? 1 : 2;
};

// Roe (or arithmetic) interface state from the two nodes of the interface
template <int S>
__device__ __forceinline__ IfaceState<Real> march_state(const ModelParams &mp, const Real UL[5], const Real UR[5])
{
    IfaceState<Real> is;
    const Real gamma = Real(mp.gamma);
    Real Uo[6];
    fast::interface_state<Real>(mp.jacobMean, gamma, UL, UR, Uo);
    is.V[0] = Uo[1];
    is.V[1] = Uo[2];
    is.V[2] = Uo[3];
    is.hT = Uo[4];
    is.cs = Uo[5];
    is.qk = Real(0.5) * (is.V[0] * is.V[0] + is.V[1] * is.V[1] + is.V[2] * is.V[2]);
    is.d = fast::rcp<Real>(Real(2) * is.cs);
    is.b = (gamma - Real(1)) * (Real(2) * is.d * is.d);
    is.b2 = Real(2) * is.b;
    Real lam[5];
    lam[0] = is.V[S] - is.cs;
    lam[1] = lam[2] = lam[3] = is.V[S];
    lam[4] = is.V[S] + is.cs;
    if (mp.fluxSplit == 0) {
        const Real ls = fabs(is.V[S]) + is.cs;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            is.lp[r] = Real(0.5) * (lam[r] + ls);
            is.ln[r] = Real(0.5) * (lam[r] - ls);
        }
    } else {
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            const Real sr = sqrt(lam[r] * lam[r] + Real(1.0e-6));
            is.lp[r] = Real(0.5) * (lam[r] + sr);
            is.ln[r] = Real(0.5) * (lam[r] - sr);
        }
    }
    return is;
}

// characteristic split fluxes with WENO5 (NP = 6) or WENO3 (NP = 4) on every
// field; W[m] holds node p-(NP/2-1)+m of interface p+1/2
template <int S, int NP>
__device__ __forceinline__ void march_weno(const IfaceState<Real> &is, const Real (&W)[NP][5], Real G[5])
{
    Real A[NP], Bv[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        A[m] = is.qk * W[m][0] - is.V[0] * W[m][1] - is.V[1] * W[m][2] - is.V[2] * W[m][3] + W[m][4];
        Bv[m] = is.V[S] * W[m][0] - W[m][S + 1];
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        Real C[NP];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            if (r == 0) {
                C[m] = is.b * A[m] + is.d * Bv[m];
            } else if (r == 4) {
                C[m] = is.b * A[m] - is.d * Bv[m];
            } else if (r == S + 1) {
                C[m] = W[m][0] - is.b2 * A[m];
            } else {
                C[m] = W[m][r] - is.b2 * is.V[r - 1] * A[m];
            }
        }
        const Real lp = is.lp[r], ln = is.ln[r];
        Real hp, hn;
        if constexpr (NP == 6 && sizeof(Real) == sizeof(double)) {
            hp = fast::weno5_pair<Real>(C, lp, ln);
            hn = Real(0);
        } else if constexpr (NP == 6) {
            hp = fast::weno5<Real>(lp * C[0], lp * C[1], lp * C[2], lp * C[3], lp * C[4]);
            hn = fast::weno5<Real>(ln * C[5], ln * C[4], ln * C[3], ln * C[2], ln * C[1]);
        } else {
            hp = fast::weno3<Real>(lp * C[0], lp * C[1], lp * C[2]);
            hn = fast::weno3<Real>(ln * C[3], ln * C[2], ln * C[1]);
        }
        G[r] = hp + hn;
    }
}

// WENO5 with the linear weights: reconstruct the two upwind states and
// project them with the interface's left eigenvectors
template <int S>
__device__ __forceinline__ void march_linear(const IfaceState<Real> &is, const Real (&W)[6][5], Real G[5])
{
    Real up[5], um[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        up[v] = fast::upwind5<Real>(W[0][v], W[1][v], W[2][v], W[3][v], W[4][v]);
        um[v] = fast::upwind5<Real>(W[5][v], W[4][v], W[3][v], W[2][v], W[1][v]);
    }
    Real wp[5], wm[5];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const Real *u = side ? um : up;
        Real *w = side ? wm : wp;
        const Real A = is.qk * u[0] - is.V[0] * u[1] - is.V[1] * u[2] - is.V[2] * u[3] + u[4];
        const Real Bs = is.V[S] * u[0] - u[S + 1];
        w[0] = is.b * A + is.d * Bs;
        w[4] = is.b * A - is.d * Bs;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            w[t + 1] = (t == S) ? u[0] - is.b2 * A : u[t + 1] - is.b2 * is.V[t] * A;
        }
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        G[r] = is.lp[r] * wp[r] + is.ln[r] * wm[r];
    }
}

// Central viscous flux of interface p+1/2, subtracted from F.  Pc, Pn:
// velocity and temperature at nodes p and p+1; Dc, Dn: per transverse axis
// (increasing order) the central differences v_t(n+e_t)-v_t(n-e_t) and
// v_S(n+e_t)-v_S(n-e_t) at those nodes.
template <int S>
__device__ __forceinline__ void march_visc(const Grid &g, const ModelParams &mp, const Real Pc[4], const Real Pn[4],
                                           const Real (&Dc)[2][2], const Real (&Dn)[2][2], Real F[5])
{
    typedef Transverse<S> TR;
    const Real ddS = Real(g.dd[S]);
    Real gS[3];  // d(v_a)/ds
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        gS[v] = (Pn[v] - Pc[v]) * ddS;
    }
    const Real dd0 = Real(0.25) * Real(g.dd[TR::t0]);
    const Real dd1 = Real(0.25) * Real(g.dd[TR::t1]);
    const Real g00 = (Dc[0][0] + Dn[0][0]) * dd0;  // d(v_t0)/d t0
    const Real gS0 = (Dc[0][1] + Dn[0][1]) * dd0;  // d(v_S)/d t0
    const Real g11 = (Dc[1][0] + Dn[1][0]) * dd1;  // d(v_t1)/d t1
    const Real gS1 = (Dc[1][1] + Dn[1][1]) * dd1;  // d(v_S)/d t1
    const Real Tc = Pc[3], Tp = Pn[3];
    const Real Th = Real(0.5) * (Tc + Tp);
    const Real Ts = Th * Real(mp.refT);
    const Real mu = Real(mp.refMu) * (Real(1.458e-6) * Ts * sqrt(Ts) * fast::rcp<Real>(Ts + Real(110.4)));
    const Real heatK = Real(mp.gamma * mp.cv / 0.71) * mu;
    const Real divV = gS[S] + g00 + g11;
    Real tau[3];
    tau[S] = mu * (Real(2) * gS[S] - Real(2.0 / 3.0) * divV);
    tau[TR::t0] = mu * (gS0 + gS[TR::t0]);
    tau[TR::t1] = mu * (gS1 + gS[TR::t1]);
    Real e5 = heatK * (Tp - Tc) * ddS;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const Real vh = Real(0.5) * (Pc[v] + Pn[v]);
        F[v + 1] -= tau[v];
        e5 += tau[v] * vh;
    }
    F[4] -= e5;
}

// transverse differences of a node from direct loads of its neighbours
// along axis t (v_t and v_S), written to D[0..1]
template <int S, int t>
__device__ __forceinline__ void march_tdiff(const double *__restrict__ U, long long nn, long long id, long long st,
                                            Real D[2])
{
    const long long qp = id + st, qm = id - st;
    const Real rp = fast::rcp<Real>(Real(__ldg(U + qp)));
    const Real rm = fast::rcp<Real>(Real(__ldg(U + qm)));
    const Real tp = Real(__ldg(U + (1 + t) * nn + qp)), tm = Real(__ldg(U + (1 + t) * nn + qm));
    const Real sp = Real(__ldg(U + (1 + S) * nn + qp)), sm = Real(__ldg(U + (1 + S) * nn + qm));
    D[0] = fast::diff_prod(tp, rp, tm, rm);
    D[1] = fast::diff_prod(sp, rp, sm, rm);
}

// interface flux (convective minus viscous is added by the caller)
template <int S, int NP, bool HYB>
__device__ __forceinline__ void march_flux(const ModelParams &mp, const Real (&W)[NP][5], bool full, Real F[5])
{
    constexpr int H = NP / 2;
    const IfaceState<Real> is = march_state<S>(mp, W[H - 1], W[H]);
    Real G[5];
    if constexpr (HYB && NP == 6) {
        if (full) {
            march_weno<S, NP>(is, W, G);
        } else {
            march_linear<S>(is, W, G);
        }
    } else {
        march_weno<S, NP>(is, W, G);
    }
    back_project<S>(is, G, F);
}

// The hybrid interface flux with the full WENO5 branch shared out over the
// warp.  The flagged lanes (full) need ten WENO5 evaluations each (five characteristic fields, two
// sides).  Taken lane by lane, a warp with one flagged lane runs all ten for
// that lane alone; here the flagged lanes write their WENO5 inputs to the
// warp's buffer (kCoopSlots interfaces per round) and every lane of the warp
// evaluates some of them, so a warp with k flagged lanes spends about
// ceil(k / kCoopSlots) * ceil(10 kCoopSlots / 32) WENO5 passes instead of
// ten; the other lanes then take the linear-weight flux.  A warp with more
// than 16 flagged lanes takes the lane-by-lane branch.
// The arithmetic of each evaluation is that of march_weno.  All 32 lanes of
// the warp must call this together (plane-march kernels: every consumer lane
// runs the same march).
template <int S>
__device__ __forceinline__ void march_flux_coop(const ModelParams &mp, const Real (&W)[6][5], bool full, Real F[5],
                                                Real *wbuf)
{
    constexpr unsigned kAll = 0xffffffffu;
    const IfaceState<Real> is = march_state<S>(mp, W[2], W[3]);
    Real G[5];
    unsigned fm = __ballot_sync(kAll, full);
    if (__popc(fm) > 16) {
        if (full) {
            march_weno<S, 6>(is, W, G);
        } else {
            march_linear<S>(is, W, G);
        }
    } else {
        const int lane = threadIdx.x & 31;
        while (fm) {
            // this round: the lowest kCoopSlots flagged lanes
            unsigned rest = fm;
#pragma unroll
            for (int k = 0; k < kCoopSlots; ++k) rest &= rest - 1;
            const unsigned chunk = fm & ~rest;
            fm = rest;
            const bool mine = (chunk >> lane) & 1u;
            const int slot = __popc(chunk & ((1u << lane) - 1u));
            if (mine) {
                Real A[6], Bv[6];
#pragma unroll
                for (int m = 0; m < 6; ++m) {
                    A[m] = is.qk * W[m][0] - is.V[0] * W[m][1] - is.V[1] * W[m][2] - is.V[2] * W[m][3] + W[m][4];
                    Bv[m] = is.V[S] * W[m][0] - W[m][S + 1];
                }
                Real *o = wbuf + slot * 50;
#pragma unroll
                for (int r = 0; r < 5; ++r) {
                    Real C[6];
#pragma unroll
                    for (int m = 0; m < 6; ++m) {
                        if (r == 0) {
                            C[m] = is.b * A[m] + is.d * Bv[m];
                        } else if (r == 4) {
                            C[m] = is.b * A[m] - is.d * Bv[m];
                        } else if (r == S + 1) {
                            C[m] = W[m][0] - is.b2 * A[m];
                        } else {
                            C[m] = W[m][r] - is.b2 * is.V[r - 1] * A[m];
                        }
                    }
                    const Real lp = is.lp[r], ln = is.ln[r];
#pragma unroll
                    for (int m = 0; m < 5; ++m) {
                        o[(2 * r) * 5 + m] = lp * C[m];
                        o[(2 * r + 1) * 5 + m] = ln * C[5 - m];
                    }
                }
            }
            __syncwarp();
            // task t = slot * 10 + 2 * field + side reads inputs [5t, 5t+5)
            // and leaves its result in the first of them
            const int ntask = __popc(chunk) * 10;
            for (int t = lane; t < ntask; t += 32) {
                Real *f = wbuf + t * 5;
                f[0] = fast::weno5<Real>(f[0], f[1], f[2], f[3], f[4]);
            }
            __syncwarp();
            if (mine) {
                const Real *o = wbuf + slot * 50;
#pragma unroll
                for (int r = 0; r < 5; ++r) {
                    G[r] = o[(2 * r) * 5] + o[(2 * r + 1) * 5];
                }
            }
            __syncwarp();
        }
        if (!full) {
            march_linear<S>(is, W, G);
        }
    }
    back_project<S>(is, G, F);
}

// node update from the fluxes of its left and right interfaces
__device__ __forceinline__ void march_update(const StageArgs &a, long long nn, long long id, double rdt,
                                             const Real Fl[5], const Real Fr[5], bool same_o)
{
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const double phi = double(Fl[v]) - double(Fr[v]);
        const long long q = v * nn + id;
        if (a.accumulate) {
            a.Um[q] = a.Um[q] + a.coeB * rdt * phi;
        } else {
            const double un = __ldg(a.Un + q);
            const double uo = same_o ? un : a.Uo[q];
            a.Um[q] = a.coeA * uo + a.coeB * (un + rdt * phi);
        }
    }
}

// ---------------------------------------------------------------------------
// Y and Z sweeps: a thread per line segment
// ---------------------------------------------------------------------------
template <int S, int NP, bool VISC, bool HYB>
__global__ void __launch_bounds__(kMarchThreads, kMarchMinBlocks)
stage_march_yz(Grid g, ModelParams mp, StageArgs a, int nseg)
{
    static_assert(S == 1 || S == 2, "march along y or z");
    constexpr int T2 = (S == 1) ? 2 : 1;  // transverse axis other than x
    constexpr int H = NP / 2;
    pdl_wait();
    const int Lx = g.hi[0] - g.lo[0], Lt = g.hi[T2] - g.lo[T2], Ls = g.hi[S] - g.lo[S];
    const long long nlines = (long long)Lx * Lt;
    const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int seg = (int)(gid / nlines);
    if (seg >= nseg) {
        return;
    }
    const long long line = gid - (long long)seg * nlines;
    const int i = g.lo[0] + (int)(line % Lx);
    const int c = g.lo[T2] + (int)(line / Lx);
    const int p0 = g.lo[S] + (int)((long long)seg * Ls / nseg);
    const int p1 = g.lo[S] + (int)((long long)(seg + 1) * Ls / nseg);
    const long long nn = g.nn;
    const long long sx = (long long)g.pitch;                 // stride along y
    const long long sz = (long long)g.pitch * g.n[1];        // stride along z
    const long long st = (S == 1) ? sx : sz;                 // stride along s
    const long long base = (S == 1) ? (long long)c * sz + i : (long long)c * sx + i;
    const double *__restrict__ Un = a.Un;
    const Real cvinv = Real(1.0 / mp.cv);
    const bool same_o = (a.Uo == a.Un);
    const double rdt = (a.dt_scale * a.dt[0]) * g.dd[S];

    Real W[NP][5];
#pragma unroll
    for (int m = 0; m < NP - 1; ++m) {
        march_load(Un, nn, base + (long long)(p0 - H + m) * st, W[m]);
    }
    Real Pc[4] = {Real(0), Real(0), Real(0), Real(0)};
    Real Dc[2][2] = {{Real(0), Real(0)}, {Real(0), Real(0)}};
    if (VISC) {
        const long long id = base + (long long)(p0 - 1) * st;
        march_prims(W[H - 1], cvinv, Pc);
        march_tdiff<S, 0>(Un, nn, id, 1, Dc[0]);
        march_tdiff<S, T2>(Un, nn, id, (T2 == 1) ? sx : sz, Dc[1]);
    }
    const uint8_t *__restrict__ fl = HYB ? a.flags + (long long)S * nn : nullptr;
    unsigned fw = 0;  // sensor flags of nodes p-1, p, p+1 (bits 0..2)
    if (HYB) {
        fw = (unsigned)fl[base + (long long)(p0 - 2) * st] | ((unsigned)fl[base + (long long)(p0 - 1) * st] << 1) |
             ((unsigned)fl[base + (long long)p0 * st] << 2);
    }
    Real Fl[5];
    for (int p = p0 - 1; p < p1; ++p) {
        const long long id = base + (long long)p * st;
        march_load(Un, nn, id + (long long)H * st, W[NP - 1]);
        bool full = true;
        if (HYB) {
            fw |= (unsigned)fl[id + 2 * st] << 3;
            full = (fw != 0u);
        }
        Real Pn[4], Dn[2][2];
        if (VISC) {
            march_prims(W[H], cvinv, Pn);
            march_tdiff<S, 0>(Un, nn, id + st, 1, Dn[0]);
            march_tdiff<S, T2>(Un, nn, id + st, (T2 == 1) ? sx : sz, Dn[1]);
        }
        Real F[5];
        march_flux<S, NP, HYB>(mp, W, full, F);
        if (VISC) {
            march_visc<S>(g, mp, Pc, Pn, Dc, Dn, F);
        }
        if (p >= p0 && a.did[id] == 0) {
            march_update(a, nn, id, rdt, Fl, F, same_o);
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            Fl[v] = F[v];
        }
#pragma unroll
        for (int m = 0; m < NP - 1; ++m) {
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                W[m][v] = W[m + 1][v];
            }
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
}

// ---------------------------------------------------------------------------
// X sweeps: a warp per 32 consecutive nodes of an x-line, walking y-rows
// ---------------------------------------------------------------------------
template <int NP, bool VISC, bool HYB>
__global__ void __launch_bounds__(kMarchThreads, kMarchMinBlocks)
stage_march_x(Grid g, ModelParams mp, StageArgs a, int nwx, int nseg)
{
    constexpr int H = NP / 2;
    constexpr int UW = 32 - NP;  // nodes updated per warp
    constexpr unsigned kAll = 0xffffffffu;
    pdl_wait();
    const int lane = threadIdx.x & 31;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const int wx = (int)(gw % nwx);
    const long long rest = gw / nwx;
    const int kq = (int)(rest % Lz);
    const int seg = (int)(rest / Lz);
    if (seg >= nseg) {
        return;  // the whole warp
    }
    const int k = g.lo[2] + kq;
    const int x = g.lo[0] - H + UW * wx + lane;
    const int j0 = g.lo[1] + (int)((long long)seg * Ly / nseg);
    const int j1 = g.lo[1] + (int)((long long)(seg + 1) * Ly / nseg);
    const bool need = x < g.hi[0] + H;                         // node read by an interface of the warp
    const bool upd_lane = lane >= H && lane < H + UW && x < g.hi[0];
    const long long nn = g.nn;
    const long long sy = (long long)g.pitch, sz = (long long)g.pitch * g.n[1];
    const long long xk = (long long)k * sz + (need ? x : g.lo[0]);
    const double *__restrict__ Un = a.Un;
    const Real cvinv = Real(1.0 / mp.cv);
    const bool same_o = (a.Uo == a.Un);
    const double rdt = (a.dt_scale * a.dt[0]) * g.dd[0];
    const uint8_t *__restrict__ fl = a.flags;  // sweep 0 flags

    // row values of this lane's node: current row j (Wc), next row (Wn)
    Real Wc[5];
    march_load(Un, nn, xk + (long long)j0 * sy, Wc);
    Real Pc[4] = {Real(0), Real(0), Real(0), Real(0)};
    Real Pm[2] = {Real(0), Real(0)};  // u, v of row j-1
    if (VISC) {
        Real w[5], P[4];
        march_load(Un, nn, xk + (long long)(j0 - 1) * sy, w);
        march_prims(w, cvinv, P);
        Pm[0] = P[0];
        Pm[1] = P[1];
        march_prims(Wc, cvinv, Pc);
    }
    for (int j = j0; j < j1; ++j) {
        const long long id = xk + (long long)j * sy;
        Real Wn[5];
        if (VISC || j + 1 < j1) {
            march_load(Un, nn, id + sy, Wn);
        }
        bool full = true;
        if (HYB) {
            const unsigned own = need ? (unsigned)fl[id] : 1u;
            const unsigned mask = __ballot_sync(kAll, own != 0u);
            // flags of lanes lane-1 .. lane+2
            const unsigned win = (lane >= 1) ? (mask >> (lane - 1)) : (mask << 1);
            full = (win & 0xFu) != 0u;
        }
        // stencil from the neighbouring lanes
        Real W[NP][5];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                W[m][v] = (m == H - 1) ? Wc[v] : __shfl_sync(kAll, Wc[v], lane - (H - 1) + m);
            }
        }
        Real F[5];
        march_flux<0, NP, HYB>(mp, W, full, F);
        Real Pp[4];
        if (VISC) {
            march_prims(Wn, cvinv, Pp);
            Real D[2][2];
            D[0][0] = Pp[1] - Pm[1];  // v(j+1) - v(j-1)
            D[0][1] = Pp[0] - Pm[0];  // u(j+1) - u(j-1)
            march_tdiff<0, 2>(Un, nn, id, sz, D[1]);
            Real Pn[4], Dn[2][2];
#pragma unroll
            for (int q = 0; q < 4; ++q) Pn[q] = __shfl_sync(kAll, Pc[q], lane + 1);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                Dn[q][0] = __shfl_sync(kAll, D[q][0], lane + 1);
                Dn[q][1] = __shfl_sync(kAll, D[q][1], lane + 1);
            }
            march_visc<0>(g, mp, Pc, Pn, D, Dn, F);
        }
        Real Fl[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            Fl[v] = __shfl_sync(kAll, F[v], lane - 1);
        }
        if (upd_lane && a.did[id] == 0) {
            march_update(a, nn, id, rdt, Fl, F, same_o);
        }
        if (VISC) {
            Pm[0] = Pc[0];
            Pm[1] = Pc[1];
#pragma unroll
            for (int q = 0; q < 4; ++q) Pc[q] = Pp[q];
        }
        if (VISC || j + 1 < j1) {
#pragma unroll
            for (int v = 0; v < 5; ++v) Wc[v] = Wn[v];
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// segments per line so that about `target` warps are launched
inline int march_segments(long long warps_per_segment, int len, int target)
{
    long long n = (target + warps_per_segment - 1) / warps_per_segment;
    if (n < 1) n = 1;
    const int cap = len / 4 > 1 ? len / 4 : 1;
    return (int)(n < cap ? n : cap);
}

template <int NP, bool VISC, bool HYB>
static int launch_march_s(const Grid &g, const ModelParams &m, const StageArgs &a, int s, int target,
                          cudaStream_t st)
{
    const int L[3] = {g.hi[0] - g.lo[0], g.hi[1] - g.lo[1], g.hi[2] - g.lo[2]};
    cudaError_t e;
    if (s == 0) {
        const int nwx = (L[0] + (32 - NP) - 1) / (32 - NP);
        const int nseg = march_segments((long long)nwx * L[2], L[1], target);
        const long long warps = (long long)nwx * L[2] * nseg;
        const long long blocks = (warps * 32 + kMarchThreads - 1) / kMarchThreads;
        e = launch_k(stage_march_x<NP, VISC, HYB>, dim3((unsigned)blocks), dim3(kMarchThreads), 0, st, g, m, a,
                     nwx, nseg);
    } else {
        const int T2 = (s == 1) ? 2 : 1;
        const long long lines = (long long)L[0] * L[T2];
        const int nseg = march_segments((lines + 31) / 32, L[s], target);
        const long long blocks = (lines * nseg + kMarchThreads - 1) / kMarchThreads;
        if (s == 1) {
            e = launch_k(stage_march_yz<1, NP, VISC, HYB>, dim3((unsigned)blocks), dim3(kMarchThreads), 0, st, g, m,
                         a, nseg);
        } else {
            e = launch_k(stage_march_yz<2, NP, VISC, HYB>, dim3((unsigned)blocks), dim3(kMarchThreads), 0, st, g, m,
                         a, nseg);
        }
    }
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_march launch");
}

// hybrid: the sensor form (WENO5 and flags present); otherwise every
// interface is reconstructed with full WENO
static int launch_march_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                             bool hybrid, int target, cudaStream_t st)
{
    if (g.hi[0] <= g.lo[0] || g.hi[1] <= g.lo[1] || g.hi[2] <= g.lo[2]) {
        return ACFD_OK;
    }
    if (m.sScheme == 1) {
        if constexpr (sizeof(Real) == sizeof(float)) {
            if (hybrid && a.flags) {
                return viscous ? launch_march_s<6, true, true>(g, m, a, s, target, st)
                               : launch_march_s<6, false, true>(g, m, a, s, target, st);
            }
        }
        return viscous ? launch_march_s<6, true, false>(g, m, a, s, target, st)
                       : launch_march_s<6, false, false>(g, m, a, s, target, st);
    }
    return viscous ? launch_march_s<4, true, false>(g, m, a, s, target, st)
                   : launch_march_s<4, false, false>(g, m, a, s, target, st);
}

}  // namespace ACFD_NS
}  // namespace acfd

// Stage kernel with shared-memory bricks (fast FP64 and FP32 forms).
//
// One block = one tile of interfaces (brick_geometry.cuh).  Thread 0 loads the
// tile's brick of U[tn] (five variables, stencil and viscous halos) with a
// single 5-D TMA copy; while it is in flight every thread reads its node
// flags.  Then, all from shared memory:
//   A. (viscous) per brick node: u, v, w, T, computed once and reused by the
//      ten interfaces that read each node;
//   B. per interface: Roe state, characteristic projection field by field
//      (W = L*U through A = q*U0 - V.U[1..3] + U4 and B = V_s*U0 - U_{s+1}),
//      WENO on the split fluxes, back projection, viscous flux;
//   C. per fluid node: U[tm] = coeA*U[to] + coeB*(U[tn] + r*(G_left - G_right)).
// Included after sweep_impl.cuh by sweep_fast.cu and sweep_fp32.cu.
#pragma once

#include "brick_geometry.cuh"
#include "tma.cuh"

namespace acfd {
namespace ACFD_NS {

constexpr long long kTmaWaitLimit = 1LL << 22;
constexpr int kBrickThreads = 256;

template <int S, bool VISC, int VAR>
struct BrickLayout {
    typedef Brick<S, VISC, VAR> B;
    static constexpr int nodes = B::BX * B::BY * B::BZ;
    static constexpr int u_bytes = 5 * nodes * 8;
    static constexpr int p_bytes = VISC ? 4 * nodes * (int)sizeof(Real) : 0;
    // FP32 form: a copy of the brick converted once, read by the interfaces
    static constexpr bool conv = sizeof(Real) != sizeof(double);
    static constexpr int r_bytes = conv ? 5 * nodes * (int)sizeof(Real) : 0;
    static constexpr int f_bytes = 5 * kBrickThreads * (int)sizeof(Real);
    static constexpr int p_off = (u_bytes + 127) / 128 * 128;
    static constexpr int r_off = (p_off + p_bytes + 127) / 128 * 128;
    static constexpr int f_off = (r_off + r_bytes + 127) / 128 * 128;
    // U[to] (or U[tm] when accumulating) of the nodes the block updates
    static constexpr int o_bytes = 5 * kBrickThreads * 8;
    static constexpr int o_off = (f_off + f_bytes + 127) / 128 * 128;
    // hybrid form: queue of the interfaces reconstructed with full WENO5
    static constexpr int q_off = o_off + o_bytes;
    static constexpr int q_bytes = (kBrickThreads + 4) * 4;
    static constexpr int bar_off = (q_off + q_bytes + 15) / 16 * 16;
    static constexpr int total = bar_off + 16;
};

// Roe (or arithmetic) state of an interface and the factors of its
// characteristic projection and flux splitting.
template <typename Real>
struct IfaceState {
    Real V[3], hT, cs, qk, d, b, b2;
    Real lp[5], ln[5];  // split eigenvalues
};

// interface between brick nodes c and c + bs (sR: the brick, NN nodes per variable)
template <int S, int NN>
__device__ __forceinline__ IfaceState<Real> iface_state(const ModelParams &mp, const Real *sR, int c, int bs)
{
    IfaceState<Real> is;
    const Real gamma = Real(mp.gamma);
    Real UL[5], UR[5], Uo[6];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        UL[v] = sR[v * NN + c];
        UR[v] = sR[v * NN + c + bs];
    }
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

// Characteristic split fluxes G of the interface with WENO5 (NP = 6) or WENO3
// (NP = 4) on every field, the projection W = L*U taken field by field
// through the two scalars A = q*U0 - V.U[1..3] + U4 and B = V_s*U0 - U_{s+1}.
template <int S, int NP, int NN>
__device__ __forceinline__ void conv_weno(const IfaceState<Real> &is, const Real *sR, int c, int bs, Real G[5])
{
    constexpr int first = -(NP / 2 - 1);
    Real A[NP], Bv[NP];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const int p = c + (first + m) * bs;
        const Real u0 = sR[p], u1 = sR[NN + p], u2 = sR[2 * NN + p];
        const Real u3 = sR[3 * NN + p], u4 = sR[4 * NN + p];
        A[m] = is.qk * u0 - is.V[0] * u1 - is.V[1] * u2 - is.V[2] * u3 + u4;
        const Real us = (S == 0) ? u1 : (S == 1 ? u2 : u3);
        Bv[m] = is.V[S] * u0 - us;
    }
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        Real W[NP];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            const int p = c + (first + m) * bs;
            if (r == 0) {
                W[m] = is.b * A[m] + is.d * Bv[m];
            } else if (r == 4) {
                W[m] = is.b * A[m] - is.d * Bv[m];
            } else if (r == S + 1) {
                W[m] = sR[p] - is.b2 * A[m];
            } else {
                W[m] = sR[r * NN + p] - is.b2 * is.V[r - 1] * A[m];
            }
        }
        const Real lp = is.lp[r], ln = is.ln[r];
        Real hp, hn;
        if constexpr (NP == 6 && sizeof(Real) == sizeof(double)) {
            hp = fast::weno5_pair<Real>(W, lp, ln);
            hn = Real(0);
        } else if constexpr (NP == 6) {
            hp = fast::weno5<Real>(lp * W[0], lp * W[1], lp * W[2], lp * W[3], lp * W[4]);
            hn = fast::weno5<Real>(ln * W[5], ln * W[4], ln * W[3], ln * W[2], ln * W[1]);
        } else {
            hp = fast::weno3<Real>(lp * W[0], lp * W[1], lp * W[2]);
            hn = fast::weno3<Real>(ln * W[3], ln * W[2], ln * W[1]);
        }
        G[r] = hp + hn;
    }
}

// Smooth interface (hybrid form): WENO5 with the linear weights.  The linear
// reconstruction commutes with the frozen projection, so the split fluxes
// need the projection of two reconstructed vectors only.
template <int S, int NN>
__device__ __forceinline__ void conv_linear(const IfaceState<Real> &is, const Real *sR, int c, int bs, Real G[5])
{
    Real up[5], um[5];
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        const Real *P = sR + v * NN + c;
        up[v] = fast::upwind5<Real>(P[-2 * bs], P[-bs], P[0], P[bs], P[2 * bs]);
        um[v] = fast::upwind5<Real>(P[3 * bs], P[2 * bs], P[bs], P[0], P[-bs]);
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

// back projection F = R*G of the split characteristic fluxes
template <int S>
__device__ __forceinline__ void back_project(const IfaceState<Real> &is, const Real G[5], Real F[5])
{
    const Real *V = is.V;
    F[0] = G[0] + G[S + 1] + G[4];
    Real e4 = is.hT * (G[0] + G[4]) + V[S] * is.cs * (G[4] - G[0]) + (V[S] * V[S] - is.qk) * G[S + 1];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t == S) {
            F[t + 1] = V[S] * (G[0] + G[S + 1] + G[4]) + is.cs * (G[4] - G[0]);
        } else {
            F[t + 1] = V[t] * (G[0] + G[4]) + G[t + 1];
            e4 += V[t] * G[t + 1];
        }
    }
    F[4] = e4;
}

// central viscous flux of the interface from the brick primitives u, v, w, T
// (sP), subtracted from F
template <int S, typename B, int NN>
__device__ __forceinline__ void visc_flux(const Grid &g, const ModelParams &mp, const Real *sP, int c, int bs,
                                          Real F[5])
{
    const int pn = c + bs;
    Real grad[3][3];
    const Real ddS = Real(g.dd[S]);
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        grad[v][S] = (sP[v * NN + pn] - sP[v * NN + c]) * ddS;
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t == S) continue;
        const int bt = (t == 0) ? 1 : (t == 1 ? B::BX : B::BX * B::BY);
        const Real ddt = Real(0.25) * Real(g.dd[t]);
#pragma unroll
        for (int v = 0; v < 3; ++v) {
            const Real *P = sP + v * NN;
            grad[v][t] = (P[c + bt] + P[pn + bt] - P[c - bt] - P[pn - bt]) * ddt;
        }
    }
    const Real Tc = sP[3 * NN + c], Tp = sP[3 * NN + pn];
    const Real Th = Real(0.5) * (Tc + Tp);
    const Real Ts = Th * Real(mp.refT);
    const Real mu = Real(mp.refMu) * (Real(1.458e-6) * Ts * sqrt(Ts) * fast::rcp<Real>(Ts + Real(110.4)));
    const Real heatK = Real(mp.gamma * mp.cv / 0.71) * mu;
    const Real divV = grad[0][0] + grad[1][1] + grad[2][2];
    Real tau[3];
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        tau[v] = (v == S) ? mu * (Real(2) * grad[S][S] - Real(2.0 / 3.0) * divV) : mu * (grad[S][v] + grad[v][S]);
    }
    Real e5 = heatK * (Tp - Tc) * ddS;
#pragma unroll
    for (int v = 0; v < 3; ++v) {
        const Real vh = Real(0.5) * (sP[v * NN + c] + sP[v * NN + pn]);
        F[v + 1] -= tau[v];
        e5 += tau[v] * vh;
    }
    F[4] -= e5;
}

// One tile of interfaces (tile indices tbx, tby, tbz of the case's tiling):
// the body shared by the per-case kernel and the persistent batched kernel.
// The caller has initialised the block's mbarrier; `parity` is the phase this
// tile's load completes.  Returns false when the load did not complete within
// the wait limit (the block must then stop).
template <int S, int NP, bool VISC, bool HYB, int VAR>
__device__ __forceinline__ bool brick_tile(const Grid &g, const ModelParams &mp, const StageArgs &a,
                                           const CUtensorMap *map, int tbx, int tby, int tbz, unsigned char *smem,
                                           uint32_t parity)
{
    typedef Brick<S, VISC, VAR> B;
    typedef BrickLayout<S, VISC, VAR> LY;
    double *sU = reinterpret_cast<double *>(smem);
    Real *sP = reinterpret_cast<Real *>(smem + LY::p_off);
    // the brick in the arithmetic type: the FP64 brick itself, or its FP32 copy
    Real *sR = LY::conv ? reinterpret_cast<Real *>(smem + LY::r_off) : reinterpret_cast<Real *>(sU);
    Real *sF = reinterpret_cast<Real *>(smem + LY::f_off);
    double *sO = reinterpret_cast<double *>(smem + LY::o_off);
    int *sQ = reinterpret_cast<int *>(smem + LY::q_off);
    int *sQn = sQ + kBrickThreads;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + LY::bar_off);
    const bool visc_on = VISC && (mp.refMu > 0.0);

    const int tid = threadIdx.x + B::TX * (threadIdx.y + B::TY * threadIdx.z);
    // tile origin (first updated node) and brick origin
    const int i0 = g.lo[0] + tbx * B::SX;
    const int j0 = g.lo[1] + tby * B::SY;
    const int k0 = g.lo[2] + tbz * B::SZ;
    const int xs = (i0 - B::HX) & ~1;
    const int ys = j0 - B::HY;
    const int zs = k0 - B::HZ;

    __syncthreads();  // every thread is done with the previous tile's shared data
    if (tid == 0) {
        *sQn = 0;
        tma::mbar_expect_tx(bar, LY::u_bytes);
        tma::load_5d(sU, map, xs, ys, zs, 0, a.tn, bar);
    }

    // this thread's interface: between node (i,j,k) and (i,j,k) + e_S
    const int i = i0 + (S == 0 ? (int)threadIdx.x - 1 : (int)threadIdx.x);
    const int j = j0 + (S == 1 ? (int)threadIdx.y - 1 : (int)threadIdx.y);
    const int k = k0 + (S == 2 ? (int)threadIdx.z - 1 : (int)threadIdx.z);
    const int sl = (S == 0) ? threadIdx.x : (S == 1 ? threadIdx.y : threadIdx.z);  // local index along s
    const int q = (S == 0 ? i : (S == 1 ? j : k)) - g.lo[S];                   // PIN position along s
    const int Ls = g.hi[S] - g.lo[S];
    bool inside = (i < g.hi[0]) && (j < g.hi[1]) && (k < g.hi[2]);
    if (S != 0) inside = inside && (i >= g.lo[0]);
    if (S != 1) inside = inside && (j >= g.lo[1]);
    if (S != 2) inside = inside && (k >= g.lo[2]);
    inside = inside && (q >= -1) && (q <= Ls - 1);
    const long long st = (S == 0) ? 1LL : (S == 1 ? (long long)g.pitch : (long long)g.pitch * g.n[1]);
    const long long node = ((long long)k * g.n[1] + j) * g.pitch + i;
    bool fl_left = false, fl_right = false;
    if (inside) {
        fl_left = (q >= 0) && (a.did[node] == 0);
        fl_right = (q + 1 < Ls) && (a.did[node + st] == 0);
    }
    // everything else from global memory is read while the brick is in
    // flight: the sensor flags of the interface's stencil (hybrid form), the
    // step and the node-update operand U[to] (U[tm] when accumulating)
    bool full_own = true;
    if (HYB && NP == 6 && (fl_left || fl_right)) {
        const uint8_t *fl = a.flags + (long long)S * g.nn;
        full_own = (fl[node - st] | fl[node] | fl[node + st] | fl[node + 2 * st]) != 0;
    }
    const bool upd = fl_left && sl >= 1;  // the first interface of each line only feeds its right neighbour
    const bool need_o = a.accumulate || (a.to != a.tn);
    if (upd && need_o) {
        const double *src = a.accumulate ? a.Um : a.Uo;
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            sO[v * kBrickThreads + tid] = __ldcs(src + v * g.nn + node);
        }
    }
    const double rdt = (a.dt_scale * a.dt[0]) * g.dd[S];

    const bool ok = tma::mbar_wait_bounded(bar, parity, a.status, 4, kTmaWaitLimit);
    if (!__syncthreads_and(ok)) {
        // time-out: give the copy a second bounded chance to land, then leave
        if (tid == 0) {
            for (long long it = 0; it < kTmaWaitLimit && !tma::mbar_try_wait(bar, parity); ++it) {
            }
        }
        __syncthreads();
        return false;
    }

    // brick index of node (x, y, z), variable v
    auto bidx = [&](int x, int y, int z) { return ((z - zs) * B::BY + (y - ys)) * B::BX + (x - xs); };

    // A. per brick node: the FP32 copy (FP32 form) and the primitives u, v, w,
    // T (viscous cases)
    if (LY::conv || visc_on) {
        const Real cvinv = Real(1.0 / mp.cv);
        for (int n = tid; n < LY::nodes; n += kBrickThreads) {
            Real uc[5];
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                uc[v] = Real(sU[v * LY::nodes + n]);
                if (LY::conv) sR[v * LY::nodes + n] = uc[v];
            }
            if (!visc_on) continue;
            const Real r = uc[0];
            const Real ir = fast::rcp<Real>(r);
            const Real u = uc[1] * ir;
            const Real v = uc[2] * ir;
            const Real w = uc[3] * ir;
            const Real e = uc[4] * ir;
            sP[n] = u;
            sP[LY::nodes + n] = v;
            sP[2 * LY::nodes + n] = w;
            sP[3 * LY::nodes + n] = (e - Real(0.5) * (u * u + v * v + w * w)) * cvinv;
        }
        __syncthreads();
    }

    // B. interface flux.  Hybrid form: an interface whose stencil carries a
    // sensor flag is queued; after the others, the block's first threads
    // reconstruct the queued interfaces with full WENO5, so that a few flags
    // cost a few lanes instead of whole warps.
    const int bs = (S == 0) ? 1 : (S == 1 ? B::BX : B::BX * B::BY);  // brick stride along s
    if (fl_left || fl_right) {
        const int c = bidx(i, j, k);  // node i of the interface
        const IfaceState<Real> is = iface_state<S, LY::nodes>(mp, sR, c, bs);
        Real F[5];
        const bool defer = HYB && NP == 6 && full_own;
        if (defer) {
#pragma unroll
            for (int v = 0; v < 5; ++v) F[v] = Real(0);
            const int slot = atomicAdd(sQn, 1);
            sQ[slot] = tid;
        } else {
            Real G[5];
            if (HYB && NP == 6) {
                conv_linear<S, LY::nodes>(is, sR, c, bs, G);
            } else {
                conv_weno<S, NP, LY::nodes>(is, sR, c, bs, G);
            }
            back_project<S>(is, G, F);
        }
        if (visc_on) {
            visc_flux<S, B, LY::nodes>(g, mp, sP, c, bs, F);
        }
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            sF[v * kBrickThreads + tid] = F[v];
        }
    }
    if (HYB && NP == 6) {
        __syncthreads();
        const int nq = *sQn;
        if (tid < nq) {
            const int lt = sQ[tid];
            const int tx = lt % B::TX, ty = (lt / B::TX) % B::TY, tz = lt / (B::TX * B::TY);
            const int c = bidx(i0 + tx - (S == 0), j0 + ty - (S == 1), k0 + tz - (S == 2));
            const IfaceState<Real> is = iface_state<S, LY::nodes>(mp, sR, c, bs);
            Real G[5], F[5];
            conv_weno<S, NP, LY::nodes>(is, sR, c, bs, G);
            back_project<S>(is, G, F);
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                sF[v * kBrickThreads + lt] += F[v];
            }
        }
    }
    __syncthreads();

    // C. node update
    if (upd) {
        const int lt = tid - ((S == 0) ? 1 : (S == 1 ? B::TX : B::TX * B::TY));
        const int c = bidx(i, j, k);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double phi = double(sF[v * kBrickThreads + lt]) - double(sF[v * kBrickThreads + tid]);
            const long long qv = v * g.nn + node;
            const double un = sU[v * LY::nodes + c];
            if (a.accumulate) {
                a.Um[qv] = sO[v * kBrickThreads + tid] + a.coeB * rdt * phi;
            } else {
                const double uo = need_o ? sO[v * kBrickThreads + tid] : un;
                a.Um[qv] = a.coeA * uo + a.coeB * (un + rdt * phi);
            }
        }
    }
    return true;
}

// one tile per block
template <int S, int NP, bool VISC, bool HYB, int VAR>
__global__ void __launch_bounds__(kBrickThreads, 2)
stage_brick(Grid g, ModelParams mp, StageArgs a, const __grid_constant__ CUtensorMap map)
{
    typedef BrickLayout<S, VISC, VAR> LY;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + LY::bar_off);
    if (threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0) {
        tma::mbar_init(bar, 1);
    }
    __syncthreads();
    pdl_wait();
    brick_tile<S, NP, VISC, HYB, VAR>(g, mp, a, &map, blockIdx.x, blockIdx.y, blockIdx.z, smem, 0);
}

template <int S, int NP, bool VISC, bool HYB, int VAR>
static int launch_brick_one(const Grid &g, const ModelParams &m, const StageArgs &a, cudaStream_t st)
{
    typedef Brick<S, VISC, VAR> B;
    typedef BrickLayout<S, VISC, VAR> LY;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_brick<S, NP, VISC, HYB, VAR>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, LY::total);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_brick)");
        configured[dev] = true;
    }
    const int L0 = g.hi[0] - g.lo[0], L1 = g.hi[1] - g.lo[1], L2 = g.hi[2] - g.lo[2];
    dim3 grid((L0 + B::SX - 1) / B::SX, (L1 + B::SY - 1) / B::SY, (L2 + B::SZ - 1) / B::SZ);
    dim3 block(B::TX, B::TY, B::TZ);
    cudaError_t e = launch_k(stage_brick<S, NP, VISC, HYB, VAR>, grid, block, LY::total, st, g, m, a,
                             a.maps[S * kTileVariants + VAR]);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_brick launch");
}

template <int S, int NP, bool VISC, bool HYB>
static int launch_brick_var(const Grid &g, const ModelParams &m, const StageArgs &a, cudaStream_t st)
{
    if (a.var[S] == 1) return launch_brick_one<S, NP, VISC, HYB, 1>(g, m, a, st);
    return launch_brick_one<S, NP, VISC, HYB, 0>(g, m, a, st);
}

template <int NP, bool VISC, bool HYB>
static int launch_brick_np(const Grid &g, const ModelParams &m, const StageArgs &a, int s, cudaStream_t st)
{
    if (s == 0) return launch_brick_var<0, NP, VISC, HYB>(g, m, a, st);
    if (s == 1) return launch_brick_var<1, NP, VISC, HYB>(g, m, a, st);
    return launch_brick_var<2, NP, VISC, HYB>(g, m, a, st);
}

static int launch_brick_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                             cudaStream_t st)
{
    if (g.hi[0] <= g.lo[0] || g.hi[1] <= g.lo[1] || g.hi[2] <= g.lo[2]) {
        return ACFD_OK;
    }
    if (m.sScheme == 1) {
        return viscous ? launch_brick_np<6, true, false>(g, m, a, s, st)
                       : launch_brick_np<6, false, false>(g, m, a, s, st);
    }
    return viscous ? launch_brick_np<4, true, false>(g, m, a, s, st) : launch_brick_np<4, false, false>(g, m, a, s, st);
}

#if ACFD_FORM == 2
// ---------------------------------------------------------------------------
// persistent stage kernel of a batch of independent cases: resident blocks
// pull (case, tile) work items from a counter until every tile of every case
// is done.  Viscous brick geometry for all cases (inviscid ones skip the
// viscous part at run time).
// ---------------------------------------------------------------------------
template <int S, bool HYB>
__global__ void __launch_bounds__(kBrickThreads, 2)
stage_batch(const BatchCase *cases, const CUtensorMap *maps, const long long *prefix, int ncase, StageCoefs sc,
            const double *dts, unsigned long long *counter, int *status)
{
    typedef BrickLayout<S, true, 0> LY;
    typedef Brick<S, true, 0> B;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + LY::bar_off);
    __shared__ long long item_s;
    const int tid = threadIdx.x + B::TX * (threadIdx.y + B::TY * threadIdx.z);
    if (tid == 0) {
        tma::mbar_init(bar, 1);
    }
    __syncthreads();
    pdl_wait();
    const long long total = prefix[ncase];
    uint32_t parity = 0;
    for (;;) {
        if (tid == 0) {
            item_s = (long long)atomicAdd(counter, 1ULL);
        }
        __syncthreads();
        const long long item = item_s;
        if (item >= total) {
            break;
        }
        int lo = 0, hi = ncase - 1;  // the case whose tiles contain item
        while (lo < hi) {
            const int mid = (lo + hi + 1) / 2;
            if (prefix[mid] <= item) lo = mid; else hi = mid - 1;
        }
        const BatchCase &C = cases[lo];
        const long long t = item - prefix[lo];
        const int nx = C.tiles[S][0], ny = C.tiles[S][1];
        const int tx = (int)(t % nx);
        const int ty = (int)((t / nx) % ny);
        const int tz = (int)(t / ((long long)nx * ny));
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
        if (!brick_tile<S, 6, true, HYB, 0>(C.g, C.mp, a, maps + 3 * lo + S, tx, ty, tz, smem, parity)) {
            break;
        }
        parity ^= 1u;
    }
}

template <int S, bool HYB>
static int launch_batch_one(const BatchCase *cases, const CUtensorMap *maps, const long long *prefix, int ncase,
                            const StageCoefs &sc, const double *dts, unsigned long long *counter, int *status,
                            int blocks, cudaStream_t st)
{
    typedef Brick<S, true, 0> B;
    typedef BrickLayout<S, true, 0> LY;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_batch<S, HYB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             LY::total);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_batch)");
        configured[dev] = true;
    }
    cudaError_t e = launch_k(stage_batch<S, HYB>, dim3(blocks), dim3(B::TX, B::TY, B::TZ), LY::total, st, cases,
                             maps, prefix, ncase, sc, dts, counter, status);
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_batch launch");
}

static int launch_batch_impl(const BatchCase *cases, const CUtensorMap *maps, const long long *prefix, int ncase,
                             const StageCoefs &sc, const double *dts, unsigned long long *counter, int *status,
                             int blocks, int s, bool hybrid, cudaStream_t st)
{
    if (hybrid) {
        if (s == 0) return launch_batch_one<0, true>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
        if (s == 1) return launch_batch_one<1, true>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
        return launch_batch_one<2, true>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
    }
    if (s == 0) return launch_batch_one<0, false>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
    if (s == 1) return launch_batch_one<1, false>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
    return launch_batch_one<2, false>(cases, maps, prefix, ncase, sc, dts, counter, status, blocks, st);
}

// hybrid form (WENO5 only): interfaces the sensor did not flag use the
// linear-weight limit
static int launch_brick_hybrid_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                                    cudaStream_t st)
{
    if (g.hi[0] <= g.lo[0] || g.hi[1] <= g.lo[1] || g.hi[2] <= g.lo[2]) {
        return ACFD_OK;
    }
    if (m.sScheme != 1 || !a.flags) {
        return launch_brick_impl(g, m, a, s, viscous, st);
    }
    return viscous ? launch_brick_np<6, true, true>(g, m, a, s, st) : launch_brick_np<6, false, true>(g, m, a, s, st);
}
#endif

}  // namespace ACFD_NS
}  // namespace acfd

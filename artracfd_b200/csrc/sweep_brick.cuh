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

template <int S, bool VISC>
struct BrickLayout {
    typedef Brick<S, VISC> B;
    static constexpr int nodes = B::BX * B::BY * B::BZ;
    static constexpr int u_bytes = 5 * nodes * 8;
    static constexpr int p_bytes = VISC ? 4 * nodes * (int)sizeof(Real) : 0;
    static constexpr int f_bytes = 5 * kBrickThreads * (int)sizeof(Real);
    static constexpr int p_off = (u_bytes + 127) / 128 * 128;
    static constexpr int f_off = (p_off + p_bytes + 127) / 128 * 128;
    static constexpr int bar_off = (f_off + f_bytes + 15) / 16 * 16;
    static constexpr int total = bar_off + 16;
};

template <int S, int NP, bool VISC>
__global__ void __launch_bounds__(kBrickThreads, 2)
stage_brick(Grid g, ModelParams mp, StageArgs a, const __grid_constant__ CUtensorMap map)
{
    typedef Brick<S, VISC> B;
    typedef BrickLayout<S, VISC> LY;
    extern __shared__ __align__(128) unsigned char smem[];
    double *sU = reinterpret_cast<double *>(smem);
    Real *sP = reinterpret_cast<Real *>(smem + LY::p_off);
    Real *sF = reinterpret_cast<Real *>(smem + LY::f_off);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + LY::bar_off);

    const int tid = threadIdx.x + B::TX * (threadIdx.y + B::TY * threadIdx.z);
    // tile origin (first updated node) and brick origin
    const int i0 = g.lo[0] + blockIdx.x * B::SX;
    const int j0 = g.lo[1] + blockIdx.y * B::SY;
    const int k0 = g.lo[2] + blockIdx.z * B::SZ;
    const int xs = (i0 - B::HX) & ~1;
    const int ys = j0 - B::HY;
    const int zs = k0 - B::HZ;

    if (tid == 0) {
        tma::mbar_init(bar, 1);
    }
    __syncthreads();
    if (tid == 0) {
        tma::mbar_expect_tx(bar, LY::u_bytes);
        tma::load_5d(sU, &map, xs, ys, zs, 0, a.tn, bar);
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

    const bool ok = tma::mbar_wait_bounded(bar, 0, a.status, 4, kTmaWaitLimit);
    if (!__syncthreads_and(ok)) {
        // time-out: give the copy a second bounded chance to land, then leave
        if (tid == 0) {
            for (long long it = 0; it < kTmaWaitLimit && !tma::mbar_try_wait(bar, 0); ++it) {
            }
        }
        __syncthreads();
        return;
    }

    // brick index of node (x, y, z), variable v
    auto bidx = [&](int x, int y, int z) { return ((z - zs) * B::BY + (y - ys)) * B::BX + (x - xs); };

    // A. primitives of every brick node (viscous cases)
    if (VISC) {
        const Real cvinv = Real(1.0 / mp.cv);
        for (int n = tid; n < LY::nodes; n += kBrickThreads) {
            const Real r = Real(sU[n]);
            const Real ir = fast::rcp<Real>(r);
            const Real u = Real(sU[LY::nodes + n]) * ir;
            const Real v = Real(sU[2 * LY::nodes + n]) * ir;
            const Real w = Real(sU[3 * LY::nodes + n]) * ir;
            const Real e = Real(sU[4 * LY::nodes + n]) * ir;
            sP[n] = u;
            sP[LY::nodes + n] = v;
            sP[2 * LY::nodes + n] = w;
            sP[3 * LY::nodes + n] = (e - Real(0.5) * (u * u + v * v + w * w)) * cvinv;
        }
        __syncthreads();
    }

    // B. interface flux
    if (fl_left || fl_right) {
        const int c = bidx(i, j, k);                       // node i of the interface
        const int bs = (S == 0) ? 1 : (S == 1 ? B::BX : B::BX * B::BY);  // brick stride along s
        constexpr int NN = LY::nodes;
        constexpr int ctr = NP / 2 - 1;
        constexpr int first = -ctr;
        const Real gamma = Real(mp.gamma);
        // Roe / arithmetic state of the interface
        Real UL[5], UR[5], Uo[6];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            UL[v] = Real(sU[v * NN + c]);
            UR[v] = Real(sU[v * NN + c + bs]);
        }
        fast::interface_state<Real>(mp.jacobMean, gamma, UL, UR, Uo);
        const Real V[3] = {Uo[1], Uo[2], Uo[3]};
        const Real hT = Uo[4];
        const Real cs = Uo[5];
        const Real qk = Real(0.5) * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
        const Real d = fast::rcp<Real>(Real(2) * cs);
        const Real b = (gamma - Real(1)) * (Real(2) * d * d);
        const Real b2 = Real(2) * b;
        Real lp[5], ln[5];
        {
            Real lam[5];
            lam[0] = V[S] - cs;
            lam[1] = lam[2] = lam[3] = V[S];
            lam[4] = V[S] + cs;
            if (mp.fluxSplit == 0) {
                const Real ls = fabs(V[S]) + cs;
#pragma unroll
                for (int r = 0; r < 5; ++r) {
                    lp[r] = Real(0.5) * (lam[r] + ls);
                    ln[r] = Real(0.5) * (lam[r] - ls);
                }
            } else {
#pragma unroll
                for (int r = 0; r < 5; ++r) {
                    const Real sr = sqrt(lam[r] * lam[r] + Real(1.0e-6));
                    lp[r] = Real(0.5) * (lam[r] + sr);
                    ln[r] = Real(0.5) * (lam[r] - sr);
                }
            }
        }
        // the two scalars of every stencil point
        Real A[NP], Bv[NP];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            const int p = c + (first + m) * bs;
            const Real u0 = Real(sU[p]), u1 = Real(sU[NN + p]), u2 = Real(sU[2 * NN + p]);
            const Real u3 = Real(sU[3 * NN + p]), u4 = Real(sU[4 * NN + p]);
            A[m] = qk * u0 - V[0] * u1 - V[1] * u2 - V[2] * u3 + u4;
            const Real us = (S == 0) ? u1 : (S == 1 ? u2 : u3);
            Bv[m] = V[S] * u0 - us;
        }
        // field by field: W, WENO on both split fluxes
        Real G[5];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            Real W[NP];
#pragma unroll
            for (int m = 0; m < NP; ++m) {
                const int p = c + (first + m) * bs;
                if (r == 0) {
                    W[m] = b * A[m] + d * Bv[m];
                } else if (r == 4) {
                    W[m] = b * A[m] - d * Bv[m];
                } else if (r == S + 1) {
                    W[m] = Real(sU[p]) - b2 * A[m];
                } else {
                    W[m] = Real(sU[r * NN + p]) - b2 * V[r - 1] * A[m];
                }
            }
            Real hp, hn;
            if (NP == 6) {
                hp = fast::weno5<Real>(lp[r] * W[0], lp[r] * W[1], lp[r] * W[2], lp[r] * W[3], lp[r] * W[4]);
                hn = fast::weno5<Real>(ln[r] * W[5], ln[r] * W[4], ln[r] * W[3], ln[r] * W[2], ln[r] * W[1]);
            } else {
                hp = fast::weno3<Real>(lp[r] * W[0], lp[r] * W[1], lp[r] * W[2]);
                hn = fast::weno3<Real>(ln[r] * W[3], ln[r] * W[2], ln[r] * W[1]);
            }
            G[r] = hp + hn;
        }
        Real F[5];
        F[0] = G[0] + G[S + 1] + G[4];
        Real e4 = hT * (G[0] + G[4]) + V[S] * cs * (G[4] - G[0]) + (V[S] * V[S] - qk) * G[S + 1];
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            if (t == S) {
                F[t + 1] = V[S] * (G[0] + G[S + 1] + G[4]) + cs * (G[4] - G[0]);
            } else {
                F[t + 1] = V[t] * (G[0] + G[4]) + G[t + 1];
                e4 += V[t] * G[t + 1];
            }
        }
        F[4] = e4;
        if (VISC) {
            // central viscous flux from the brick primitives
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
                tau[v] = (v == S) ? mu * (Real(2) * grad[S][S] - Real(2.0 / 3.0) * divV)
                                  : mu * (grad[S][v] + grad[v][S]);
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
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            sF[v * kBrickThreads + tid] = F[v];
        }
    }
    __syncthreads();

    // C. node update (the first interface of each line only feeds its right neighbour)
    if (fl_left && sl >= 1) {
        const int lt = tid - ((S == 0) ? 1 : (S == 1 ? B::TX : B::TX * B::TY));
        const int c = bidx(i, j, k);
        const double r = (a.dt_scale * a.dt[0]) * g.dd[S];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            const double phi = double(sF[v * kBrickThreads + lt]) - double(sF[v * kBrickThreads + tid]);
            const long long qv = v * g.nn + node;
            const double un = sU[v * LY::nodes + c];
            if (a.accumulate) {
                a.Um[qv] = a.Um[qv] + a.coeB * r * phi;
            } else {
                const double uo = (a.to == a.tn) ? un : a.Uo[qv];
                a.Um[qv] = a.coeA * uo + a.coeB * (un + r * phi);
            }
        }
    }
}

template <int S, int NP, bool VISC>
static int launch_brick_one(const Grid &g, const ModelParams &m, const StageArgs &a, cudaStream_t st)
{
    typedef Brick<S, VISC> B;
    typedef BrickLayout<S, VISC> LY;
    static bool configured[64] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && !configured[dev]) {
        cudaError_t e = cudaFuncSetAttribute(stage_brick<S, NP, VISC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             LY::total);
        if (e != cudaSuccess) return cuda_status(e, "cudaFuncSetAttribute(stage_brick)");
        configured[dev] = true;
    }
    const int L0 = g.hi[0] - g.lo[0], L1 = g.hi[1] - g.lo[1], L2 = g.hi[2] - g.lo[2];
    dim3 grid((L0 + B::SX - 1) / B::SX, (L1 + B::SY - 1) / B::SY, (L2 + B::SZ - 1) / B::SZ);
    dim3 block(B::TX, B::TY, B::TZ);
    stage_brick<S, NP, VISC><<<grid, block, LY::total, st>>>(g, m, a, a.maps[S]);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "stage_brick launch");
}

template <int NP, bool VISC>
static int launch_brick_np(const Grid &g, const ModelParams &m, const StageArgs &a, int s, cudaStream_t st)
{
    if (s == 0) return launch_brick_one<0, NP, VISC>(g, m, a, st);
    if (s == 1) return launch_brick_one<1, NP, VISC>(g, m, a, st);
    return launch_brick_one<2, NP, VISC>(g, m, a, st);
}

static int launch_brick_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s, bool viscous,
                             cudaStream_t st)
{
    if (g.hi[0] <= g.lo[0] || g.hi[1] <= g.lo[1] || g.hi[2] <= g.lo[2]) {
        return ACFD_OK;
    }
    if (m.sScheme == 1) {
        return viscous ? launch_brick_np<6, true>(g, m, a, s, st) : launch_brick_np<6, false>(g, m, a, s, st);
    }
    return viscous ? launch_brick_np<4, true>(g, m, a, s, st) : launch_brick_np<4, false>(g, m, a, s, st);
}

}  // namespace ACFD_NS
}  // namespace acfd

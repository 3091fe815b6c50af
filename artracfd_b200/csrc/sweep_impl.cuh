// One LLLU stage (fluid_dynamics.c:157-274) as fused sm_100a kernels:
// interface fluxes (convective + viscous) are computed once per interface,
// exchanged through shared memory, and each fluid PIN node is updated with
//   U[tm] = coeA*U[to] + coeB*(U[tn] + r*(Fl - Fr + Fvr - Fvl))
// (or U[tm] += coeB*r*Phi for the operator-by-operator Y/Z sweeps).
//
// Included by sweep_exact.cu, sweep_fast.cu and sweep_fp32.cu, which define
//   ACFD_FORM   0 exact FP64 (reference order), 1 fast FP64, 2 FP32 stencil
//   ACFD_NS     the namespace of the translation unit
// before including this file.
//
// Thread layouts (both coalesced along x):
//  * X sweeps: a flat index over (line, interface) with x fastest; tiles of
//    kTileX interfaces overlap by one so that every node finds both of its
//    interfaces in one tile.
//  * Y/Z sweeps: kColX columns (consecutive x, then the other transverse
//    index) x kTileS interfaces along s; a block marches along its segment of
//    the line, carrying the last interface flux to the next pass.
#pragma once

#include "acfd_internal.cuh"
#include "flux_math.cuh"

namespace acfd {
namespace ACFD_NS {

#if ACFD_FORM == 2
typedef float Real;
#else
typedef double Real;
#endif

constexpr bool kExact = (ACFD_FORM == 0);
// values kept per interface in shared memory: exact keeps Fhat and Fvhat
// apart to reproduce the reference's summation order
constexpr int kKeep = kExact ? 10 : 5;
constexpr int kTileX = 128;
constexpr int kColX = 32;
constexpr int kTileS = 8;

__device__ __forceinline__ long long node_of(const Grid &g, int i, int j, int k)
{
    return ((long long)k * g.n[1] + j) * g.pitch + i;
}

template <int S>
__device__ __forceinline__ long long stride_of(const Grid &g)
{
    return S == 0 ? 1LL : (S == 1 ? (long long)g.pitch : (long long)g.pitch * g.n[1]);
}

// ---------------------------------------------------------------------------
// viscous numerical flux at the interface between node c and c + e_S
// (diffusive_flux.c:58-312); velocities by division (exact) or by the
// reciprocal density (fast)
// ---------------------------------------------------------------------------
template <int S>
__device__ __forceinline__ void velocity(const double *__restrict__ U, long long nn, long long id,
                                         Real V[3])
{
    const double r0 = U[id];
    if (kExact) {
        V[0] = U[nn + id] / r0;
        V[1] = U[2 * nn + id] / r0;
        V[2] = U[3 * nn + id] / r0;
    } else {
        const Real ir = Real(1) / Real(r0);
        V[0] = Real(U[nn + id]) * ir;
        V[1] = Real(U[2 * nn + id]) * ir;
        V[2] = Real(U[3 * nn + id]) * ir;
    }
}

template <int S>
__device__ __forceinline__ void viscous_flux(const Grid &g, const ModelParams &mp,
                                             const double *__restrict__ U, long long c,
                                             Real Fv[5])
{
    const long long nn = g.nn;
    const long long p = c + stride_of<S>(g);
    Real Vc[3], Vp[3];
    velocity<S>(U, nn, c, Vc);
    velocity<S>(U, nn, p, Vp);
    Real Tc, Tp;
    {
        double Uc[5], Up[5];
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            Uc[v] = U[v * nn + c];
            Up[v] = U[v * nn + p];
        }
        if (kExact) {
            Tc = exact::temperature_cv(mp.cv, Uc);
            Tp = exact::temperature_cv(mp.cv, Up);
        } else {
            const Real icv = Real(1) / Real(mp.cv);
            const Real ic = Real(1) / Real(Uc[0]);
            const Real ip = Real(1) / Real(Up[0]);
            Tc = (Real(Uc[4]) - Real(0.5) * (Real(Uc[1]) * Real(Uc[1]) + Real(Uc[2]) * Real(Uc[2]) +
                                             Real(Uc[3]) * Real(Uc[3])) * ic) * ic * icv;
            Tp = (Real(Up[4]) - Real(0.5) * (Real(Up[1]) * Real(Up[1]) + Real(Up[2]) * Real(Up[2]) +
                                             Real(Up[3]) * Real(Up[3])) * ip) * ip * icv;
        }
    }
    Real grad[3][3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        grad[a][S] = (Vp[a] - Vc[a]) * Real(g.dd[S]);
    }
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t == S) {
            continue;
        }
        const long long st = (t == 0) ? 1LL : (t == 1 ? (long long)g.pitch : (long long)g.pitch * g.n[1]);
        Real Vcm[3], Vcp[3], Vpm[3], Vpp[3];
        velocity<S>(U, nn, c - st, Vcm);
        velocity<S>(U, nn, c + st, Vcp);
        velocity<S>(U, nn, p - st, Vpm);
        velocity<S>(U, nn, p + st, Vpp);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            grad[a][t] = Real(0.25) * (Vcp[a] + Vpp[a] - Vcm[a] - Vpm[a]) * Real(g.dd[t]);
        }
    }
    const Real dT = (Tp - Tc) * Real(g.dd[S]);
    Real Vh[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        Vh[a] = Real(0.5) * (Vc[a] + Vp[a]);
    }
    const Real Th = Real(0.5) * (Tc + Tp);
    Real mu, heatK;
    if (kExact) {
        mu = mp.refMu * exact::sutherland(Th * mp.refT);
        heatK = mp.gamma * mp.cv * mu / 0.71;
    } else {
        // Sutherland's law with T^1.5 = T*sqrt(T)
        const Real Ts = Th * Real(mp.refT);
        mu = Real(mp.refMu) * (Real(1.458e-6) * Ts * sqrt(Ts) / (Ts + Real(110.4)));
        heatK = Real(mp.gamma * mp.cv / 0.71) * mu;
    }
    const Real divV = grad[0][0] + grad[1][1] + grad[2][2];
    Real tau[3];
    tau[S] = mu * (grad[S][S] + grad[S][S] - Real(2.0 / 3.0) * divV);
    if (S == 0) {
        tau[1] = mu * (grad[0][1] + grad[1][0]);
        tau[2] = mu * (grad[0][2] + grad[2][0]);
    } else if (S == 1) {
        tau[0] = mu * (grad[1][0] + grad[0][1]);
        tau[2] = mu * (grad[1][2] + grad[2][1]);
    } else {
        tau[0] = mu * (grad[2][0] + grad[0][2]);
        tau[1] = mu * (grad[2][1] + grad[1][2]);
    }
    Fv[0] = Real(0);
    Fv[1] = tau[0];
    Fv[2] = tau[1];
    Fv[3] = tau[2];
    Fv[4] = heatK * dT + tau[0] * Vh[0] + tau[1] * Vh[1] + tau[2] * Vh[2];
}

// ---------------------------------------------------------------------------
// full interface flux at (c, c+e_S); out[0..4] = Fhat, out[5..9] = Fvhat
// (exact) or out[0..4] = Fhat - Fvhat (fast forms)
// ---------------------------------------------------------------------------
template <int S, int NP, bool VISC>
__device__ __forceinline__ void interface_flux(const Grid &g, const ModelParams &mp,
                                               const double *__restrict__ U, long long c,
                                               Real out[kKeep])
{
    const long long st = stride_of<S>(g);
    const long long nn = g.nn;
    constexpr int first = -(NP / 2 - 1);  // -2 (WENO5) or -1 (WENO3)
    Real Fh[5];
    if (kExact) {
        double Ust[6][5];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            const long long id = c + (long long)(first + m) * st;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                Ust[m][v] = U[v * nn + id];
            }
        }
#pragma unroll
        for (int m = NP; m < 6; ++m) {
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                Ust[m][v] = 0.0;
            }
        }
        double F[5];
        exact::fhat<S, NP>(mp, Ust, F);
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            Fh[v] = F[v];
        }
    } else {
        Real Ust[6][5];
#pragma unroll
        for (int m = 0; m < NP; ++m) {
            const long long id = c + (long long)(first + m) * st;
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                Ust[m][v] = Real(U[v * nn + id]);
            }
        }
#pragma unroll
        for (int m = NP; m < 6; ++m) {
#pragma unroll
            for (int v = 0; v < 5; ++v) {
                Ust[m][v] = Real(0);
            }
        }
        fast::fhat<Real, S, NP>(mp.jacobMean, mp.fluxSplit, Real(mp.gamma), Ust, Fh);
    }
    Real Fv[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)};
    if (VISC) {
        viscous_flux<S>(g, mp, U, c, Fv);
    }
    if (kExact) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            out[v] = Fh[v];
            out[5 + v] = Fv[v];
        }
    } else {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            out[v] = Fh[v] - Fv[v];
        }
    }
}

// node update from the left and right interface values
__device__ __forceinline__ void update_node(const StageArgs &a, long long nn, long long id, double r,
                                            const Real *L, const Real *R)
{
#pragma unroll
    for (int v = 0; v < 5; ++v) {
        double phi;
        if (kExact) {
            phi = L[v] - R[v] + R[5 + v] - L[5 + v];
        } else {
            phi = double(L[v]) - double(R[v]);
        }
        const long long q = v * nn + id;
        if (a.accumulate) {
            a.Um[q] = a.Um[q] + a.coeB * r * phi;
        } else {
            a.Um[q] = a.coeA * a.Uo[q] + a.coeB * (a.Un[q] + r * phi);
        }
    }
}

// ---------------------------------------------------------------------------
// X sweep
// ---------------------------------------------------------------------------
template <int NP, bool VISC>
__global__ void __launch_bounds__(kTileX) stage_x(Grid g, ModelParams mp, StageArgs a)
{
    pdl_wait();
    __shared__ Real sF[kKeep][kTileX];
    const int L = g.hi[0] - g.lo[0];
    const int IF = L + 1;
    const int Ly = g.hi[1] - g.lo[1];
    const long long nlines = (long long)Ly * (g.hi[2] - g.lo[2]);
    const long long f = (long long)blockIdx.x * (kTileX - 1) + threadIdx.x;
    const bool valid = f < nlines * IF;
    int iota = 0;
    long long c = 0;
    bool fl_left = false, fl_right = false;
    if (valid) {
        const long long line = f / IF;
        iota = (int)(f - line * IF) - 1;
        const int j = g.lo[1] + (int)(line % Ly);
        const int k = g.lo[2] + (int)(line / Ly);
        const int i = g.lo[0] + iota;
        c = node_of(g, i, j, k);
        fl_left = (iota >= 0) && (a.did[c] == 0);
        fl_right = (iota + 1 < L) && (a.did[c + 1] == 0);
    }
    if (fl_left || fl_right) {
        Real out[kKeep];
        interface_flux<0, NP, VISC>(g, mp, a.Un, c, out);
#pragma unroll
        for (int v = 0; v < kKeep; ++v) {
            sF[v][threadIdx.x] = out[v];
        }
    }
    __syncthreads();
    if (fl_left && threadIdx.x >= 1) {
        const double r = (a.dt_scale * a.dt[0]) * g.dd[0];
        Real Lf[kKeep], Rf[kKeep];
#pragma unroll
        for (int v = 0; v < kKeep; ++v) {
            Lf[v] = sF[v][threadIdx.x - 1];
            Rf[v] = sF[v][threadIdx.x];
        }
        update_node(a, g.nn, c, r, Lf, Rf);
    }
}

// ---------------------------------------------------------------------------
// Y and Z sweeps
// ---------------------------------------------------------------------------
template <int S, int NP, bool VISC>
__global__ void __launch_bounds__(kColX *kTileS) stage_yz(Grid g, ModelParams mp, StageArgs a, int seg)
{
    pdl_wait();
    __shared__ Real sF[kTileS + 1][kKeep][kColX];
    constexpr int T2 = (S == 1) ? 2 : 1;  // the other transverse direction
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int Lx = g.hi[0] - g.lo[0];
    const int Lt = g.hi[T2] - g.lo[T2];
    const int Ls = g.hi[S] - g.lo[S];
    const long long col = (long long)blockIdx.x * kColX + tx;
    const bool valid = col < (long long)Lx * Lt;
    const int i = g.lo[0] + (int)(valid ? col % Lx : 0);
    const int t2 = g.lo[T2] + (int)(valid ? col / Lx : 0);
    const int q0 = blockIdx.y * seg;
    const int q1 = min(Ls, q0 + seg);
    const long long st = stride_of<S>(g);
    // node at q (PIN coordinate along s) of this column
    long long c0;
    if (S == 1) {
        c0 = node_of(g, i, g.lo[1], t2);
    } else {
        c0 = node_of(g, i, t2, g.lo[2]);
    }
    const double r = (a.dt_scale * a.dt[0]) * g.dd[S];
    for (int base = q0 - 1; base < q1; base += kTileS) {
        const int iota = base + ty;  // interface between q = iota and iota+1
        const long long c = c0 + (long long)iota * st;
        bool fl_left = false, fl_right = false;
        if (valid && iota <= q1 - 1) {
            fl_left = (iota >= 0) && (a.did[c] == 0);
            fl_right = (iota + 1 < Ls) && (a.did[c + st] == 0);
        }
        if (fl_left || fl_right) {
            Real out[kKeep];
            interface_flux<S, NP, VISC>(g, mp, a.Un, c, out);
#pragma unroll
            for (int v = 0; v < kKeep; ++v) {
                sF[ty + 1][v][tx] = out[v];
            }
        }
        __syncthreads();
        if (fl_left && iota >= q0) {
            Real Lf[kKeep], Rf[kKeep];
#pragma unroll
            for (int v = 0; v < kKeep; ++v) {
                Lf[v] = sF[ty][v][tx];
                Rf[v] = sF[ty + 1][v][tx];
            }
            update_node(a, g.nn, c, r, Lf, Rf);
        }
        __syncthreads();
        if (ty == 0) {
#pragma unroll
            for (int v = 0; v < kKeep; ++v) {
                sF[0][v][tx] = sF[kTileS][v][tx];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// launcher
// ---------------------------------------------------------------------------
template <int NP, bool VISC>
static int launch_np(const Grid &g, const ModelParams &m, const StageArgs &a, int s, cudaStream_t st)
{
    const long long L0 = g.hi[0] - g.lo[0], L1 = g.hi[1] - g.lo[1], L2 = g.hi[2] - g.lo[2];
    if (L0 <= 0 || L1 <= 0 || L2 <= 0) {
        return ACFD_OK;
    }
    if (s == 0) {
        const long long slots = L1 * L2 * (L0 + 1);
        const long long blocks = (slots + (kTileX - 1) - 1) / (kTileX - 1);
        if (blocks > 0x7fffffffLL) {
            set_error("X sweep grid too large");
            return ACFD_ERR_ARG;
        }
        ACFD_CUDA(launch_k(stage_x<NP, VISC>, dim3((unsigned)blocks), dim3(kTileX), 0, st, g, m, a));
    } else {
        const long long Lx = L0;
        const long long Lt = (s == 1) ? L2 : L1;
        const long long Ls = (s == 1) ? L1 : L2;
        const long long cols = (Lx * Lt + kColX - 1) / kColX;
        // split lines into segments when there are too few columns to fill
        // the GPU (about four blocks per SM on 148 SMs)
        long long nseg = (4 * 148 + cols - 1) / cols;
        long long seg = (Ls + nseg - 1) / nseg;
        if (seg < 2 * kTileS) {
            seg = 2 * kTileS;
        }
        nseg = (Ls + seg - 1) / seg;
        dim3 grid((unsigned)cols, (unsigned)nseg);
        dim3 block(kColX, kTileS);
        if (s == 1) {
            ACFD_CUDA(launch_k(stage_yz<1, NP, VISC>, grid, block, 0, st, g, m, a, (int)seg));
        } else {
            ACFD_CUDA(launch_k(stage_yz<2, NP, VISC>, grid, block, 0, st, g, m, a, (int)seg));
        }
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        return cuda_status(e, "stage kernel launch");
    }
    return ACFD_OK;
}

static int launch_stage_impl(const Grid &g, const ModelParams &m, const StageArgs &a, int s,
                             bool viscous, cudaStream_t st)
{
    if (m.sScheme == 1) {
        return viscous ? launch_np<6, true>(g, m, a, s, st) : launch_np<6, false>(g, m, a, s, st);
    }
    return viscous ? launch_np<4, true>(g, m, a, s, st) : launch_np<4, false>(g, m, a, s, st);
}


// ---------------------------------------------------------------------------
// per-point twins for unit tests: WENO on count stencils, ComputeFhat on
// count 6-point stencils
// ---------------------------------------------------------------------------
__global__ void weno_batch_kernel(int scheme, const double *__restrict__ F, double *__restrict__ out, int count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) {
        return;
    }
    const double *f = F + (long long)t * 25;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        double h;
        if (kExact) {
            h = (scheme == 1) ? exact::weno5(f[r], f[5 + r], f[10 + r], f[15 + r], f[20 + r])
                              : exact::weno3(f[r], f[5 + r], f[10 + r]);
        } else {
            h = (scheme == 1) ? double(fast::weno5<Real>(Real(f[r]), Real(f[5 + r]), Real(f[10 + r]),
                                                         Real(f[15 + r]), Real(f[20 + r])))
                              : double(fast::weno3<Real>(Real(f[r]), Real(f[5 + r]), Real(f[10 + r])));
        }
        out[(long long)t * 5 + r] = h;
    }
}

template <int S, int NP>
__global__ void fhat_batch_kernel(ModelParams mp, const double *__restrict__ U, double *__restrict__ out, int count)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) {
        return;
    }
    const double *u = U + (long long)t * 30;
    Real F[5];
    if (kExact) {
        double Ust[6][5];
#pragma unroll
        for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int v = 0; v < 5; ++v) Ust[m][v] = u[m * 5 + v];
        double Fd[5];
        exact::fhat<S, NP>(mp, Ust, Fd);
#pragma unroll
        for (int v = 0; v < 5; ++v) F[v] = Fd[v];
    } else {
        Real Ust[6][5];
#pragma unroll
        for (int m = 0; m < 6; ++m)
#pragma unroll
            for (int v = 0; v < 5; ++v) Ust[m][v] = Real(u[m * 5 + v]);
        fast::fhat<Real, S, NP>(mp.jacobMean, mp.fluxSplit, Real(mp.gamma), Ust, F);
    }
#pragma unroll
    for (int v = 0; v < 5; ++v) out[(long long)t * 5 + v] = double(F[v]);
}

static int launch_weno_batch_impl(int scheme, const double *F, double *out, int count, cudaStream_t st)
{
    if (count <= 0) return ACFD_OK;
    weno_batch_kernel<<<(count + 127) / 128, 128, 0, st>>>(scheme, F, out, count);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "weno_batch launch");
}

static int launch_fhat_batch_impl(const ModelParams &m, int s, const double *U, double *out, int count,
                                  cudaStream_t st)
{
    if (count <= 0) return ACFD_OK;
    const unsigned b = (count + 127) / 128;
    if (m.sScheme == 1) {
        if (s == 0) fhat_batch_kernel<0, 6><<<b, 128, 0, st>>>(m, U, out, count);
        else if (s == 1) fhat_batch_kernel<1, 6><<<b, 128, 0, st>>>(m, U, out, count);
        else fhat_batch_kernel<2, 6><<<b, 128, 0, st>>>(m, U, out, count);
    } else {
        if (s == 0) fhat_batch_kernel<0, 4><<<b, 128, 0, st>>>(m, U, out, count);
        else if (s == 1) fhat_batch_kernel<1, 4><<<b, 128, 0, st>>>(m, U, out, count);
        else fhat_batch_kernel<2, 4><<<b, 128, 0, st>>>(m, U, out, count);
    }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "fhat_batch launch");
}

}  // namespace ACFD_NS
}  // namespace acfd

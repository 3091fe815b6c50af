// Learned smoothness sensor (no counterpart in the reference).
//
// A small MLP, 10 -> 32 -> 32 -> 1 (ReLU, ReLU, sigmoid), looks at the
// density and pressure on the 5-point stencil i-2..i+2 along a sweep axis and
// predicts whether the WENO5 nonlinear weights (weno5.c:41-55) at the node's
// two interfaces depart from the linear weights C = (0.1, 0.6, 0.3) enough to
// change the reconstruction.  Nodes the network does not flag use the
// linear-weight limit of the same characteristic scheme in the hybrid sweep.
//
// Features: 10 * (q_m - mean(q)) / mean(q) for q = rho then p, m = i-2..i+2.
// Label (training): max over the node's two interfaces, both split fluxes and
// the five characteristic fields of |sum_k (omega_k - C_k) q_k|, the change of
// the reconstruction caused by the departure of the weights, divided by the
// interface's flux scale (|u_s| + c) * max|W|; computed from the method's own
// characteristic fluxes (Roe average, LLF splitting).  A node is non-smooth
// where it exceeds the training threshold.
//
// Kernels: feature/label extraction, MLP forward, MLP loss gradient (one
// thread per sample, warp-reduced into shared then global accumulators),
// Adam update, and flag inference for the three sweep axes: a pass that
// stores (rho, p) of every node as float2, then a warp-per-32-nodes pass that
// runs layers 1 and 2 as f16 tensor-core MMAs with f32 accumulation.
#include <algorithm>
#include <cstdint>

#include <cuda_fp16.h>

#include "acfd_internal.cuh"
#include "fast_div.h"
#include "flux_math.cuh"

namespace acfd {
namespace sensor {

constexpr int kIn = 10, kH = 32;
constexpr int oW1 = 0, oB1 = kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
constexpr int kParams = oB3 + 1;  // 1441

__device__ __forceinline__ long long node_of(const Grid &g, int i, int j, int k)
{
    return ((long long)k * g.n[1] + j) * g.pitch + i;
}

__device__ __forceinline__ long long stride(const Grid &g, int s)
{
    return s == 0 ? 1LL : (s == 1 ? (long long)g.pitch : (long long)g.pitch * g.n[1]);
}

__device__ __forceinline__ void features(const double *U, long long nn, long long id, long long st, double gm1,
                                         float f[kIn])
{
    double rho[5], p[5], mr = 0.0, mp = 0.0;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        const long long q = id + (m - 2) * st;
        const double r = U[q];
        const double mx = U[nn + q], my = U[2 * nn + q], mz = U[3 * nn + q], e = U[4 * nn + q];
        rho[m] = r;
        p[m] = (e - 0.5 * (mx * mx + my * my + mz * mz) / r) * gm1;
        mr += r;
        mp += p[m];
    }
    const double ir = 5.0 / mr, ip = 5.0 / mp;
#pragma unroll
    for (int m = 0; m < 5; ++m) {
        f[m] = (float)(10.0 * (rho[m] * ir - 1.0));
        f[5 + m] = (float)(10.0 * (p[m] * ip - 1.0));
    }
}

// WENO5 weights of one stencil (weno5.c:41-55) and how far their departure
// from C moves the reconstruction: |sum_k (omega_k - C_k) q_k| (divided by
// the interface's flux scale by the caller).  At smooth extrema the weights of
// WENO-JS depart from C although the three candidates q_k agree, which this
// measure ignores.
__device__ __forceinline__ double weight_departure(double f0, double f1, double f2, double f3, double f4)
{
    const double eps = 1.0e-6;
    const double t0 = f0 - 2.0 * f1 + f2, u0 = f0 - 4.0 * f1 + 3.0 * f2;
    const double t1 = f1 - 2.0 * f2 + f3, u1 = f1 - f3;
    const double t2 = f2 - 2.0 * f3 + f4, u2 = 3.0 * f2 - 4.0 * f3 + f4;
    const double is0 = (13.0 / 12.0) * t0 * t0 + 0.25 * u0 * u0;
    const double is1 = (13.0 / 12.0) * t1 * t1 + 0.25 * u1 * u1;
    const double is2 = (13.0 / 12.0) * t2 * t2 + 0.25 * u2 * u2;
    const double a0 = 0.1 / ((eps + is0) * (eps + is0));
    const double a1 = 0.6 / ((eps + is1) * (eps + is1));
    const double a2 = 0.3 / ((eps + is2) * (eps + is2));
    const double s = a0 + a1 + a2;
    const double q0 = (2.0 * f0 - 7.0 * f1 + 11.0 * f2) / 6.0;
    const double q1 = (-f1 + 5.0 * f2 + 2.0 * f3) / 6.0;
    const double q2 = (2.0 * f2 + 5.0 * f3 - f4) / 6.0;
    return fabs((a0 / s - 0.1) * q0 + (a1 / s - 0.6) * q1 + (a2 / s - 0.3) * q2);
}

// departure at the interface between node c and c + st (6-point stencil c-2..c+3)
__device__ double interface_departure(const double *U, long long nn, long long c, long long st, int s,
                                      const ModelParams &mp)
{
    double Ust[6][5];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
#pragma unroll
        for (int v = 0; v < 5; ++v) {
            Ust[m][v] = U[v * nn + c + (m - 2) * st];
        }
    }
    double Uo[6];
    fast::interface_state<double>(mp.jacobMean, mp.gamma, Ust[2], Ust[3], Uo);
    const double V[3] = {Uo[1], Uo[2], Uo[3]};
    const double cs = Uo[5];
    const double q = 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    const double d = 1.0 / (2.0 * cs);
    const double b = (mp.gamma - 1.0) * (2.0 * d * d);
    double lam[5] = {V[s] - cs, V[s], V[s], V[s], V[s] + cs};
    const double ls = fabs(V[s]) + cs;
    double W[6][5];
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const double *u = Ust[m];
        const double A = q * u[0] - V[0] * u[1] - V[1] * u[2] - V[2] * u[3] + u[4];
        const double B = V[s] * u[0] - u[s + 1];
        W[m][0] = b * A + d * B;
        W[m][4] = b * A - d * B;
        for (int t = 0; t < 3; ++t) {
            W[m][t + 1] = (t == s) ? u[0] - 2.0 * b * A : u[t + 1] - 2.0 * b * V[t] * A;
        }
    }
    // flux scale of the interface: (|u_s| + c) times the largest
    // characteristic variable of the stencil
    double wmax = 0.0;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
#pragma unroll
        for (int r = 0; r < 5; ++r) wmax = fmax(wmax, fabs(W[m][r]));
    }
    double dep = 0.0;
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        const double lp = 0.5 * (lam[r] + ls), ln = 0.5 * (lam[r] - ls);
        dep = fmax(dep, weight_departure(lp * W[0][r], lp * W[1][r], lp * W[2][r], lp * W[3][r], lp * W[4][r]));
        dep = fmax(dep, weight_departure(ln * W[5][r], ln * W[4][r], ln * W[3][r], ln * W[2][r], ln * W[1][r]));
    }
    return dep / (ls * wmax + 1.0e-300);
}

__global__ void features_kernel(Grid g, ModelParams mp, const double *U, const int *did, int s, float *feat,
                                float *dep)
{
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)Lx * Ly * Lz) return;
    const int i = g.lo[0] + (int)(t % Lx);
    const long long rest = t / Lx;
    const int j = g.lo[1] + (int)(rest % Ly);
    const int k = g.lo[2] + (int)(rest / Ly);
    const long long id = node_of(g, i, j, k);
    const long long st = stride(g, s);
    float f[kIn];
    features(U, g.nn, id, st, mp.gamma - 1.0, f);
#pragma unroll
    for (int q = 0; q < kIn; ++q) feat[t * kIn + q] = f[q];
    if (did[id] != 0) {
        dep[t] = -1.0f;  // not a fluid node: no label
        return;
    }
    const double d0 = interface_departure(U, g.nn, id - st, st, s, mp);
    const double d1 = interface_departure(U, g.nn, id, st, s, mp);
    dep[t] = (float)fmax(d0, d1);
}

// ---------------------------------------------------------------------------
// the MLP
// ---------------------------------------------------------------------------
__device__ __forceinline__ float mlp_logit(const float *P, const float x[kIn], float h1[kH], float h2[kH])
{
#pragma unroll 4
    for (int a = 0; a < kH; ++a) {
        float z = P[oB1 + a];
#pragma unroll
        for (int q = 0; q < kIn; ++q) z = fmaf(P[oW1 + a * kIn + q], x[q], z);
        h1[a] = fmaxf(z, 0.0f);
    }
#pragma unroll 4
    for (int a = 0; a < kH; ++a) {
        float z = P[oB2 + a];
#pragma unroll
        for (int q = 0; q < kH; ++q) z = fmaf(P[oW2 + a * kH + q], h1[q], z);
        h2[a] = fmaxf(z, 0.0f);
    }
    float z = P[oB3];
#pragma unroll
    for (int q = 0; q < kH; ++q) z = fmaf(P[oW3 + q], h2[q], z);
    return z;
}

__global__ void mlp_forward_kernel(const float *params, const float *X, int n, float *prob)
{
    __shared__ float P[kParams];
    for (int q = threadIdx.x; q < kParams; q += blockDim.x) P[q] = params[q];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float x[kIn], h1[kH], h2[kH];
#pragma unroll
    for (int q = 0; q < kIn; ++q) x[q] = X[(long long)t * kIn + q];
    const float z = mlp_logit(P, x, h1, h2);
    prob[t] = 1.0f / (1.0f + expf(-z));
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the samples of the weighted binary cross-entropy and of its
// gradient: loss = w*(softplus(z) - y*z), dL/dz = w*(sigmoid(z) - y), with
// w = pos_weight for y = 1.  grad and loss are accumulated (the caller
// zeroes them).
__global__ void __launch_bounds__(256) mlp_grad_kernel(const float *params, const float *X, const float *Y, int n,
                                                       float pos_weight, float *grad, float *loss)
{
    __shared__ float P[kParams];
    __shared__ float G[kParams];
    for (int q = threadIdx.x; q < kParams; q += blockDim.x) {
        P[q] = params[q];
        G[q] = 0.0f;
    }
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = t < n;
    float x[kIn], h1[kH], h2[kH];
#pragma unroll
    for (int q = 0; q < kIn; ++q) x[q] = valid ? X[(long long)t * kIn + q] : 0.0f;
    const float z = mlp_logit(P, x, h1, h2);
    const float y = valid ? Y[t] : 0.0f;
    const float w = valid ? (y > 0.5f ? pos_weight : 1.0f) : 0.0f;
    const float sp = (z > 0.0f) ? z + log1pf(expf(-z)) : log1pf(expf(z));
    const float l = w * (sp - y * z);
    const float dz = w * (1.0f / (1.0f + expf(-z)) - y);
    const int lane = threadIdx.x & 31;
    // layer 3
    float s = warp_sum(dz);
    if (lane == 0) atomicAdd(&G[oB3], s);
    float d2[kH];
#pragma unroll
    for (int q = 0; q < kH; ++q) {
        s = warp_sum(dz * h2[q]);
        if (lane == 0) atomicAdd(&G[oW3 + q], s);
        d2[q] = (h2[q] > 0.0f) ? dz * P[oW3 + q] : 0.0f;
    }
    // layer 2
    float d1[kH];
#pragma unroll
    for (int q = 0; q < kH; ++q) d1[q] = 0.0f;
    for (int a = 0; a < kH; ++a) {
        s = warp_sum(d2[a]);
        if (lane == 0) atomicAdd(&G[oB2 + a], s);
#pragma unroll
        for (int q = 0; q < kH; ++q) {
            s = warp_sum(d2[a] * h1[q]);
            if (lane == 0) atomicAdd(&G[oW2 + a * kH + q], s);
            d1[q] = fmaf(d2[a], P[oW2 + a * kH + q], d1[q]);
        }
    }
    // layer 1
    for (int a = 0; a < kH; ++a) {
        const float da = (h1[a] > 0.0f) ? d1[a] : 0.0f;
        s = warp_sum(da);
        if (lane == 0) atomicAdd(&G[oB1 + a], s);
#pragma unroll
        for (int q = 0; q < kIn; ++q) {
            s = warp_sum(da * x[q]);
            if (lane == 0) atomicAdd(&G[oW1 + a * kIn + q], s);
        }
    }
    s = warp_sum(l);
    if (lane == 0) atomicAdd(loss, s);
    __syncthreads();
    for (int q = threadIdx.x; q < kParams; q += blockDim.x) atomicAdd(&grad[q], G[q]);
}

// Adam (Kingma & Ba 2015) on the summed gradient times `scale`
__global__ void mlp_adam_kernel(float *params, const float *grad, float *m, float *v, int step, float lr, float scale,
                                float b1, float b2, float eps)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kParams) return;
    const float gq = grad[q] * scale;
    const float mq = b1 * m[q] + (1.0f - b1) * gq;
    const float vq = b2 * v[q] + (1.0f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / (1.0f - powf(b1, (float)step));
    const float vh = vq / (1.0f - powf(b2, (float)step));
    params[q] -= lr * mh / (sqrtf(vh) + eps);
}

// ---------------------------------------------------------------------------
// tensor-core inference
// ---------------------------------------------------------------------------
// pass 1: density and pressure of every node, as float2
__global__ void rho_p_kernel(long long nn, double gm1, const double *U, float2 *rp)
{
    pdl_wait();
    const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (id >= nn) return;
    const double r = U[id];
    const double mx = U[nn + id], my = U[2 * nn + id], mz = U[3 * nn + id], e = U[4 * nn + id];
    const double p = (e - 0.5 * (mx * mx + my * my + mz * mz) / r) * gm1;
    rp[id] = make_float2((float)r, (float)p);
}

__device__ __forceinline__ uint32_t pack_half2(float lo, float hi)
{
    const __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&h);
}

// D = A (16x16, f16, row) * B (16x8, f16, col) + C (f32)
__device__ __forceinline__ void mma_16816(float d[4], const uint32_t a[4], const uint32_t b[2], const float c[4])
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%10,%11,%12,%13};"
        : "=f"(d[0]), "=f"(d[1]), "=f"(d[2]), "=f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]), "f"(c[0]), "f"(c[1]), "f"(c[2]),
          "f"(c[3]));
}

constexpr int kFlagWarps = 8;

// pass 2: each warp takes 32 consecutive PIN nodes of one sweep axis at a
// time; lane l builds the features of node l into shared memory, then the
// warp runs layer 1 (16x16 . 16x32) and layer 2 (16x32 . 32x32) on tensor
// cores for two 16-row tiles; the output layer is a dot product finished by
// quad shuffles.  Layer-1 accumulators are reused as layer-2 A fragments.
// Flags: flags[s][node] = 1 where the network's logit exceeds the threshold
// or the node is not a fluid node, 0 elsewhere; nodes outside PIN keep the 1
// written when the sensor was loaded.  count (optional) accumulates the flags set.
// div_x, div_y: division by the PIN extents along x and y.
__global__ void __launch_bounds__(kFlagWarps * 32) flags_mma_kernel(Grid g, const float2 *rp, const int *did,
                                                                    const float *params, float logit_threshold,
                                                                    uint8_t *flags, unsigned long long *count,
                                                                    FastDiv div_x, FastDiv div_y)
{
    pdl_wait();
    // one 32 x 16 f16 feature tile per warp, rows padded to 12 words so that
    // the fragment loads (8 rows x 4 words) hit 32 distinct banks
    constexpr int kRow = 12;
    __shared__ uint32_t Xs[kFlagWarps][32 * kRow];
    __shared__ float Zs[kFlagWarps][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gq = lane >> 2, t = lane & 3;
    // weights as B fragments (k >= 10 of layer 1 are zero padding)
    uint32_t B1[4][2], B2[2][4][2];
    float bias1[4][2], bias2[4][2], w3[4][2];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int n = 8 * j + gq;
        const float *W1 = params + oW1 + n * kIn;
        B1[j][0] = pack_half2(W1[2 * t], W1[2 * t + 1]);
        B1[j][1] = (2 * t + 8 < kIn) ? pack_half2(W1[2 * t + 8], W1[2 * t + 9]) : 0u;
#pragma unroll
        for (int kk = 0; kk < 2; ++kk) {
            const float *W2 = params + oW2 + n * kH + 16 * kk;
            B2[kk][j][0] = pack_half2(W2[2 * t], W2[2 * t + 1]);
            B2[kk][j][1] = pack_half2(W2[2 * t + 8], W2[2 * t + 9]);
        }
#pragma unroll
        for (int c = 0; c < 2; ++c) {
            bias1[j][c] = params[oB1 + 8 * j + 2 * t + c];
            bias2[j][c] = params[oB2 + 8 * j + 2 * t + c];
            w3[j][c] = params[oW3 + 8 * j + 2 * t + c];
        }
    }
    const float b3 = params[oB3];
    // 32-bit work indices (the launcher checks that 3 * PIN and the node
    // count fit): 64-bit divisions would cost more than the network
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const int pin = Lx * Ly * Lz;
    const int ngroups = ((pin + 31) / 32) * 3;
    const int nwarps = (int)gridDim.x * kFlagWarps;
    const int sy = g.pitch, sz = g.pitch * g.n[1];
    unsigned nflag = 0;
    for (int grp = (int)blockIdx.x * kFlagWarps + w; grp < ngroups; grp += nwarps) {
        const int gq3 = grp / 3;
        const int s = grp - 3 * gq3;
        const int q = gq3 * 32 + lane;
        const bool valid = q < pin;
        long long id = 0;
        float f[kIn];
#pragma unroll
        for (int m = 0; m < kIn; ++m) f[m] = 0.0f;
        if (valid) {
            const int rest = (int)fast_div((uint32_t)q, div_x);
            const int i = g.lo[0] + (q - rest * Lx);
            const int kk = (int)fast_div((uint32_t)rest, div_y);
            const int j = g.lo[1] + (rest - kk * Ly);
            const int k = g.lo[2] + kk;
            id = (long long)(k * sz + j * sy + i);
            const long long st = (s == 0) ? 1 : (s == 1 ? sy : sz);
            float2 v[5];
            float mr = 0.0f, mp = 0.0f;
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                v[m] = rp[id + (m - 2) * st];
                mr += v[m].x;
                mp += v[m].y;
            }
            // 5 / mean, with the approximate division (2 ulp): the features
            // go to f16 next
            const float ir = __fdividef(5.0f, mr), ip = __fdividef(5.0f, mp);
#pragma unroll
            for (int m = 0; m < 5; ++m) {
                f[m] = 10.0f * (v[m].x * ir - 1.0f);
                f[5 + m] = 10.0f * (v[m].y * ip - 1.0f);
            }
        }
        uint32_t *row = &Xs[w][lane * kRow];
#pragma unroll
        for (int m = 0; m < kIn / 2; ++m) row[m] = pack_half2(f[2 * m], f[2 * m + 1]);
#pragma unroll
        for (int m = kIn / 2; m < 8; ++m) row[m] = 0u;
        __syncwarp();
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
            const int r0 = 16 * mt + gq, r1 = r0 + 8;
            uint32_t A[4];
            A[0] = Xs[w][r0 * kRow + t];
            A[1] = Xs[w][r1 * kRow + t];
            A[2] = Xs[w][r0 * kRow + t + 4];
            A[3] = Xs[w][r1 * kRow + t + 4];
            float H1[4][4];
            const float zero[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                mma_16816(H1[j], A, B1[j], zero);
                H1[j][0] = fmaxf(H1[j][0] + bias1[j][0], 0.0f);
                H1[j][1] = fmaxf(H1[j][1] + bias1[j][1], 0.0f);
                H1[j][2] = fmaxf(H1[j][2] + bias1[j][0], 0.0f);
                H1[j][3] = fmaxf(H1[j][3] + bias1[j][1], 0.0f);
            }
            uint32_t A2[2][4];
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                A2[kk][0] = pack_half2(H1[2 * kk][0], H1[2 * kk][1]);
                A2[kk][1] = pack_half2(H1[2 * kk][2], H1[2 * kk][3]);
                A2[kk][2] = pack_half2(H1[2 * kk + 1][0], H1[2 * kk + 1][1]);
                A2[kk][3] = pack_half2(H1[2 * kk + 1][2], H1[2 * kk + 1][3]);
            }
            float z0 = 0.0f, z1 = 0.0f;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                float H2[4];
                mma_16816(H2, A2[0], B2[0][j], zero);
                mma_16816(H2, A2[1], B2[1][j], H2);
                z0 += fmaxf(H2[0] + bias2[j][0], 0.0f) * w3[j][0] + fmaxf(H2[1] + bias2[j][1], 0.0f) * w3[j][1];
                z1 += fmaxf(H2[2] + bias2[j][0], 0.0f) * w3[j][0] + fmaxf(H2[3] + bias2[j][1], 0.0f) * w3[j][1];
            }
            z0 += __shfl_xor_sync(0xffffffffu, z0, 1);
            z0 += __shfl_xor_sync(0xffffffffu, z0, 2);
            z1 += __shfl_xor_sync(0xffffffffu, z1, 1);
            z1 += __shfl_xor_sync(0xffffffffu, z1, 2);
            if (t == 0) {
                Zs[w][r0] = z0 + b3;
                Zs[w][r1] = z1 + b3;
            }
        }
        __syncwarp();
        if (valid) {
            // a logit that is not a number (a non-physical state) flags the node
            const uint8_t fl = (did[id] != 0 || !(Zs[w][lane] <= logit_threshold)) ? 1 : 0;
            flags[s * g.nn + id] = fl;
            nflag += fl;
        }
        __syncwarp();
    }
    if (count) {
        const unsigned c = __reduce_add_sync(0xffffffffu, nflag);
        if (lane == 0 && c) atomicAdd(count, (unsigned long long)c);
    }
}

}  // namespace sensor

int sensor_param_count()
{
    return sensor::kParams;
}

int launch_sensor_flags(const Grid &g, const ModelParams &m, const double *U, const int *did, const float *params,
                        float logit_threshold, float2 *rho_p, uint8_t *flags, unsigned long long *count,
                        cudaStream_t st)
{
    const long long pin = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    if (pin <= 0) return ACFD_OK;
    if (3 * pin + 96 > (long long)INT32_MAX || g.nn > (long long)INT32_MAX) {
        set_error("sensor flags: case of %lld computed nodes exceeds the 32-bit work indices", pin);
        return ACFD_ERR_ARG;
    }
    ACFD_CUDA(launch_k(sensor::rho_p_kernel, dim3((unsigned)((g.nn + 255) / 256)), dim3(256), 0, st, g.nn,
                       m.gamma - 1.0, U, rho_p));
    const long long groups = ((pin + 31) / 32) * 3;
    const long long blocks = std::min<long long>((groups + sensor::kFlagWarps - 1) / sensor::kFlagWarps, 148LL * 8);
    const FastDiv div_x = make_fast_div((uint32_t)(g.hi[0] - g.lo[0]));
    const FastDiv div_y = make_fast_div((uint32_t)(g.hi[1] - g.lo[1]));
    ACFD_CUDA(launch_k(sensor::flags_mma_kernel, dim3((unsigned)blocks), dim3(sensor::kFlagWarps * 32), 0, st, g,
                       (const float2 *)rho_p, did, params, logit_threshold, flags, count, div_x, div_y));
    return ACFD_OK;
}

int launch_sensor_features(const Grid &g, const ModelParams &m, const double *U, const int *did, int s, float *feat,
                           float *dep, cudaStream_t st)
{
    const long long pin = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    if (pin <= 0) return ACFD_OK;
    sensor::features_kernel<<<(unsigned)((pin + 127) / 128), 128, 0, st>>>(g, m, U, did, s, feat, dep);
    ACFD_CUDA(cudaGetLastError());
    return ACFD_OK;
}

}  // namespace acfd

extern "C" {

int acfd_mlp_param_count(void)
{
    return acfd::sensor::kParams;
}

int acfd_mlp_forward(const float *params, const float *X, int n, float *prob, void *stream)
{
    if (!params || !X || !prob || n < 0) {
        acfd::set_error("acfd_mlp_forward: bad arguments");
        return ACFD_ERR_ARG;
    }
    if (n == 0) return ACFD_OK;
    acfd::sensor::mlp_forward_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, X, n, prob);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : acfd::cuda_status(e, "mlp_forward launch");
}

int acfd_mlp_grad(const float *params, const float *X, const float *Y, int n, float pos_weight, float *grad,
                  float *loss, void *stream)
{
    if (!params || !X || !Y || !grad || !loss || n < 0) {
        acfd::set_error("acfd_mlp_grad: bad arguments");
        return ACFD_ERR_ARG;
    }
    if (n == 0) return ACFD_OK;
    acfd::sensor::mlp_grad_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(params, X, Y, n, pos_weight,
                                                                                     grad, loss);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : acfd::cuda_status(e, "mlp_grad launch");
}

int acfd_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float scale,
                  void *stream)
{
    if (!params || !grad || !m || !v || step < 1) {
        acfd::set_error("acfd_mlp_adam: bad arguments");
        return ACFD_ERR_ARG;
    }
    const int n = acfd::sensor::kParams;
    acfd::sensor::mlp_adam_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        params, grad, m, v, step, lr, scale, 0.9f, 0.999f, 1.0e-8f);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : acfd::cuda_status(e, "mlp_adam launch");
}

}  // extern "C"

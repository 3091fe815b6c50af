// Per-interface arithmetic of the fluid step on the device.
//
// Two forms of the same mathematics:
//
//  * namespace exact  -- the reference's operation order, operation for
//    operation (SymmetricAverage, EigenvectorL/R, CharacteristicVariable,
//    WENO5/WENO3, InverseProjection: cfd_commons.c:79-246,
//    convective_flux.c:48-124, weno5.c:35-62, weno3.c:35-55,
//    diffusive_flux.c:58-312).  Compiled with --fmad=false, its FP64 results
//    equal the reference's bit for bit (IEEE +,-,*,/,sqrt), except pow().
//
//  * namespace fast   -- the same operator written for throughput: the
//    closed-form eigenvector products reduced to two scalars per stencil point
//    (W = L*U needs A = q*U0 - V.U[1..3] + U4 and B = V_s*U0 - U_{s+1}),
//    right-eigenvector products by columns, and the WENO weights with one
//    division per field (omega_k = C_k*prod_{j!=k} D_j / sum), FMA-contracted.
//    Templated on the arithmetic type (double or float).
//
// The sweep direction S is a template parameter so that all indexing into
// the small register arrays is static.
#pragma once

#include <cuda_runtime.h>

namespace acfd {

// ===========================================================================
// exact FP64 form
// ===========================================================================
namespace exact {

__device__ __forceinline__ double sq(double x) { return x * x; }

// cfd_commons.c:79-112
__device__ __forceinline__ void symmetric_average(int averager, double gamma, const double *UL,
                                                  const double *UR, double Uo[6])
{
    const double uL = UL[1] / UL[0];
    const double vL = UL[2] / UL[0];
    const double wL = UL[3] / UL[0];
    const double hTL = (UL[4] / UL[0]) * gamma - 0.5 * (uL * uL + vL * vL + wL * wL) * (gamma - 1.0);
    const double uR = UR[1] / UR[0];
    const double vR = UR[2] / UR[0];
    const double wR = UR[3] / UR[0];
    const double hTR = (UR[4] / UR[0]) * gamma - 0.5 * (uR * uR + vR * vR + wR * wR) * (gamma - 1.0);
    if (averager == 0) {
        Uo[1] = 0.5 * (uL + uR);
        Uo[2] = 0.5 * (vL + vR);
        Uo[3] = 0.5 * (wL + wR);
        Uo[4] = 0.5 * (hTL + hTR);
    } else {
        const double D = sqrt(UR[0] / UL[0]);
        Uo[1] = (uL + D * uR) / (1.0 + D);
        Uo[2] = (vL + D * vR) / (1.0 + D);
        Uo[3] = (wL + D * wR) / (1.0 + D);
        Uo[4] = (hTL + D * hTR) / (1.0 + D);
    }
    Uo[5] = sqrt((gamma - 1.0) * (Uo[4] - 0.5 * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3])));
}

// eigenvalue splitting, cfd_commons.c:113-148
template <int S>
__device__ __forceinline__ void split(int splitter, const double Uo[6], double lp[5], double ln[5])
{
    double lam[5];
    lam[0] = Uo[S + 1] - Uo[5];
    lam[1] = Uo[S + 1];
    lam[2] = Uo[S + 1];
    lam[3] = Uo[S + 1];
    lam[4] = Uo[S + 1] + Uo[5];
    if (splitter == 0) {
        const double ls = fabs(lam[2]) + lam[4] - lam[2];
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            lp[r] = 0.5 * (lam[r] + ls);
            ln[r] = 0.5 * (lam[r] - ls);
        }
    } else {
        const double eps = 1.0e-3;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            lp[r] = 0.5 * (lam[r] + sqrt(lam[r] * lam[r] + eps * eps));
            ln[r] = 0.5 * (lam[r] - sqrt(lam[r] * lam[r] + eps * eps));
        }
    }
}

// left eigenvectors, cfd_commons.c:149-205 (mixed velocity products are
// (2b*V[hi])*V[lo] in every direction of the reference)
template <int S>
__device__ __forceinline__ void left_eig(double gamma, const double Uo[6], double L[5][5])
{
    const double V[3] = {Uo[1], Uo[2], Uo[3]};
    const double c = Uo[5];
    const double q = 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    const double b = (gamma - 1.0) / (2.0 * c * c);
    const double d = 1.0 / (2.0 * c);
    L[0][0] = b * q + d * V[S];
    L[4][0] = b * q - d * V[S];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t == S) {
            L[0][t + 1] = -b * V[t] - d;
            L[4][t + 1] = -b * V[t] + d;
        } else {
            L[0][t + 1] = -b * V[t];
            L[4][t + 1] = -b * V[t];
        }
    }
    L[0][4] = b;
    L[4][4] = b;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a == S) {
            L[a + 1][0] = -2.0 * b * q + 1.0;
            L[a + 1][1] = 2.0 * b * V[0];
            L[a + 1][2] = 2.0 * b * V[1];
            L[a + 1][3] = 2.0 * b * V[2];
            L[a + 1][4] = -2.0 * b;
        } else {
            L[a + 1][0] = -2.0 * b * q * V[a];
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int hi = (a > t) ? a : t;
                const int lo = (a > t) ? t : a;
                double e = 2.0 * b * V[hi] * V[lo];
                if (t == a) {
                    e = e + 1.0;
                }
                L[a + 1][t + 1] = e;
            }
            L[a + 1][4] = -2.0 * b * V[a];
        }
    }
}

// right eigenvectors, cfd_commons.c:206-246
template <int S>
__device__ __forceinline__ void right_eig(const double Uo[6], double R[5][5])
{
    const double V[3] = {Uo[1], Uo[2], Uo[3]};
    const double hT = Uo[4];
    const double c = Uo[5];
    const double q = 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
#pragma unroll
        for (int cc = 0; cc < 5; ++cc) {
            R[r][cc] = 0.0;
        }
    }
    R[0][0] = 1.0;
    R[0][4] = 1.0;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        R[t + 1][0] = V[t];
        R[t + 1][4] = V[t];
    }
    R[S + 1][0] = V[S] - c;
    R[S + 1][4] = V[S] + c;
    R[4][0] = hT - V[S] * c;
    R[4][4] = hT + V[S] * c;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (a == S) {
            R[0][a + 1] = 1.0;
            R[S + 1][a + 1] = V[S];
            R[4][a + 1] = V[S] * V[S] - q;
        } else {
            R[a + 1][a + 1] = 1.0;
            R[4][a + 1] = V[a];
        }
    }
}

// weno5.c:35-62 for one characteristic field
__device__ __forceinline__ double weno5(double f0, double f1, double f2, double f3, double f4)
{
    const double C0 = 1.0 / 10.0, C1 = 6.0 / 10.0, C2 = 3.0 / 10.0;
    const double eps = 1.0e-6;
    const double is0 = (13.0 / 12.0) * sq(f0 - 2.0 * f1 + f2) + (1.0 / 4.0) * sq(f0 - 4.0 * f1 + 3.0 * f2);
    const double is1 = (13.0 / 12.0) * sq(f1 - 2.0 * f2 + f3) + (1.0 / 4.0) * sq(f1 - f3);
    const double is2 = (13.0 / 12.0) * sq(f2 - 2.0 * f3 + f4) + (1.0 / 4.0) * sq(3.0 * f2 - 4.0 * f3 + f4);
    const double a0 = C0 / sq(eps + is0);
    const double a1 = C1 / sq(eps + is1);
    const double a2 = C2 / sq(eps + is2);
    const double w0 = a0 / (a0 + a1 + a2);
    const double w1 = a1 / (a0 + a1 + a2);
    const double w2 = a2 / (a0 + a1 + a2);
    const double q0 = (1.0 / 6.0) * (2.0 * f0 - 7.0 * f1 + 11.0 * f2);
    const double q1 = (1.0 / 6.0) * (-f1 + 5.0 * f2 + 2.0 * f3);
    const double q2 = (1.0 / 6.0) * (2.0 * f2 + 5.0 * f3 - f4);
    return w0 * q0 + w1 * q1 + w2 * q2;
}

// weno3.c:35-55 for one characteristic field
__device__ __forceinline__ double weno3(double f0, double f1, double f2)
{
    const double C0 = 1.0 / 3.0, C1 = 2.0 / 3.0;
    const double eps = 1.0e-6;
    const double is0 = sq(f1 - f0);
    const double is1 = sq(f2 - f1);
    const double a0 = C0 / sq(eps + is0);
    const double a1 = C1 / sq(eps + is1);
    const double w0 = a0 / (a0 + a1);
    const double w1 = a1 / (a0 + a1);
    const double q0 = (1.0 / 2.0) * (-f0 + 3.0 * f1);
    const double q1 = (1.0 / 2.0) * (f1 + f2);
    return w0 * q0 + w1 * q1;
}

// ComputeFhat (convective_flux.c:48-124) on a register stencil.  NP = 6
// (WENO5, points i-2..i+3) or 4 (WENO3, points i-1..i+2); the interface lies
// between Ust[NP/2-1] and Ust[NP/2].
template <int S, int NP>
__device__ __forceinline__ void fhat(const ModelParams &mp, const double (&Ust)[6][5], double Fhat[5])
{
    constexpr int ctr = NP / 2 - 1;
    double Uo[6];
    symmetric_average(mp.jacobMean, mp.gamma, Ust[ctr], Ust[ctr + 1], Uo);
    double lp[5], ln[5];
    split<S>(mp.fluxSplit, Uo, lp, ln);
    double W[NP][5];
    {
        double L[5][5];
        left_eig<S>(mp.gamma, Uo, L);
#pragma unroll
        for (int m = 0; m < NP; ++m) {
#pragma unroll
            for (int r = 0; r < 5; ++r) {
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < 5; ++c) {
                    acc = acc + L[r][c] * Ust[m][c];
                }
                W[m][r] = acc;
            }
        }
    }
    double G[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        double hp, hn;
        if (NP == 6) {
            hp = weno5(lp[r] * W[0][r], lp[r] * W[1][r], lp[r] * W[2][r], lp[r] * W[3][r], lp[r] * W[4][r]);
            hn = weno5(ln[r] * W[5][r], ln[r] * W[4][r], ln[r] * W[3][r], ln[r] * W[2][r], ln[r] * W[1][r]);
        } else {
            hp = weno3(lp[r] * W[0][r], lp[r] * W[1][r], lp[r] * W[2][r]);
            hn = weno3(ln[r] * W[3][r], ln[r] * W[2][r], ln[r] * W[1][r]);
        }
        G[r] = hp + hn;
    }
    double R[5][5];
    right_eig<S>(Uo, R);
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            acc = acc + R[r][c] * G[c];
        }
        Fhat[r] = acc;
    }
}

__device__ __forceinline__ double temperature_cv(double cv, const double U[5])
{
    return (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]) / (U[0] * cv);
}

__device__ __forceinline__ double sutherland(double T)
{
    return 1.458e-6 * pow(T, 1.5) / (T + 110.4);
}

}  // namespace exact

// ===========================================================================
// fast form (double or float)
// ===========================================================================
namespace fast {

// Reciprocal for the fast forms.  FP64: the hardware approximation
// (rcp.approx.ftz.f64) refined by two Newton-Raphson steps
// y <- y + y*(1 - x*y), each of which doubles the number of correct bits, so
// the result is within about one ulp of 1/x (not always correctly rounded).
// FP32: the fast approximate reciprocal.  Inputs here are positive normal
// numbers (densities, sound speeds, WENO denominators >= 1e-12).
template <typename T>
__device__ __forceinline__ T rcp(T x);

template <>
__device__ __forceinline__ double rcp<double>(double x)
{
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    return y;
}

template <>
__device__ __forceinline__ float rcp<float>(float x)
{
    return __fdividef(1.0f, x);
}

// a*b - c*d with one fused operation in a fixed form.  Left to the compiler,
// the contraction of such an expression into a fused multiply-add may differ
// between two inlined copies of the same code; where two copies compute the
// same value for neighbouring blocks (the node left of a plane-march segment
// and the same node carried inside the segment before it) they must round
// alike, or the flux of the interface between the blocks differs by an ulp.
template <typename T>
__device__ __forceinline__ T diff_prod(T a, T b, T c, T d)
{
    return fma(a, b, -(c * d));
}

// Roe/arithmetic interface state: Uo[1..3] velocity, Uo[4] total enthalpy,
// Uo[5] sound speed.
template <typename T>
__device__ __forceinline__ void interface_state(int averager, T gamma, const T *UL, const T *UR, T Uo[6])
{
    const T gm1 = gamma - T(1);
    const T irL = rcp(UL[0]);
    const T irR = rcp(UR[0]);
    const T uL = UL[1] * irL, vL = UL[2] * irL, wL = UL[3] * irL;
    const T uR = UR[1] * irR, vR = UR[2] * irR, wR = UR[3] * irR;
    const T hL = UL[4] * irL * gamma - T(0.5) * gm1 * (uL * uL + vL * vL + wL * wL);
    const T hR = UR[4] * irR * gamma - T(0.5) * gm1 * (uR * uR + vR * vR + wR * wR);
    if (averager == 0) {
        Uo[1] = T(0.5) * (uL + uR);
        Uo[2] = T(0.5) * (vL + vR);
        Uo[3] = T(0.5) * (wL + wR);
        Uo[4] = T(0.5) * (hL + hR);
    } else {
        const T D = sqrt(UR[0] * irL);
        const T iw = rcp(T(1) + D);
        Uo[1] = (uL + D * uR) * iw;
        Uo[2] = (vL + D * vR) * iw;
        Uo[3] = (wL + D * wR) * iw;
        Uo[4] = (hL + D * hR) * iw;
    }
    const T q = T(0.5) * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3]);
    Uo[5] = sqrt(gm1 * (Uo[4] - q));
}

// WENO5 with one division: omega_k = C_k prod_{j!=k} D_j / sum, D_j = (eps+IS_j)^2
template <typename T>
__device__ __forceinline__ T weno5(T f0, T f1, T f2, T f3, T f4)
{
    const T eps = T(1.0e-6);
    const T c1312 = T(13.0 / 12.0);
    const T t0 = f0 - T(2) * f1 + f2, u0 = f0 - T(4) * f1 + T(3) * f2;
    const T t1 = f1 - T(2) * f2 + f3, u1 = f1 - f3;
    const T t2 = f2 - T(2) * f3 + f4, u2 = T(3) * f2 - T(4) * f3 + f4;
    T d0 = eps + (c1312 * t0 * t0 + T(0.25) * u0 * u0);
    T d1 = eps + (c1312 * t1 * t1 + T(0.25) * u1 * u1);
    T d2 = eps + (c1312 * t2 * t2 + T(0.25) * u2 * u2);
    d0 = d0 * d0;
    d1 = d1 * d1;
    d2 = d2 * d2;
    const T a0 = T(0.1) * (d1 * d2);
    const T a1 = T(0.6) * (d0 * d2);
    const T a2 = T(0.3) * (d0 * d1);
    const T q0 = T(2) * f0 - T(7) * f1 + T(11) * f2;
    const T q1 = -f1 + T(5) * f2 + T(2) * f3;
    const T q2 = T(2) * f2 + T(5) * f3 - f4;
    return (a0 * q0 + a1 * q1 + a2 * q2) * rcp<T>(T(6) * (a0 + a1 + a2));
}

// hp + hn of one characteristic field, H+ from l+ * W[0..4] and H- from
// l- * W[5..1], with the split eigenvalues factored out: every smoothness
// indicator is quadratic in its stencil, so WENO5(l f) = l * sum_k w_k q_k(f)
// / 6 with the weights taken from eps + l^2 IS_k(f).  The second differences
// shared by the two sides are formed once and the two normalisations share
// one reciprocal: G = (l+ N+ S- + l- N- S+) / (6 S+ S-), N the weighted sum
// of the candidates and S the sum of the weights of a side.  For the FP64
// form (the product of the two weight sums stays far inside the double
// range); the same values as two weno5 calls up to rounding.
template <typename T>
__device__ __forceinline__ T weno5_pair(const T (&W)[6], T lp, T ln)
{
    // smoothness indicators as squares of scaled differences, so that each is
    // one multiply and one fused multiply-add: IS = (s D)^2 + (u / 2)^2 with
    // s = sqrt(13/12), D the second difference and u the first-difference
    // term of the reference's indicator
    const T eps = T(1.0e-6);
    const T s = T(1.0408329997330663);  // sqrt(13/12)
    const T D0 = s * (W[0] - T(2) * W[1] + W[2]);
    const T D1 = s * (W[1] - T(2) * W[2] + W[3]);
    const T D2 = s * (W[2] - T(2) * W[3] + W[4]);
    const T D3 = s * (W[3] - T(2) * W[4] + W[5]);
    const T lp2 = lp * lp, ln2 = ln * ln;
    // + side: stencil W0..W4
    const T up0 = T(0.5) * W[0] - T(2) * W[1] + T(1.5) * W[2];
    const T up1 = T(0.5) * (W[1] - W[3]);
    const T up2 = T(1.5) * W[2] - T(2) * W[3] + T(0.5) * W[4];
    T p0 = eps + lp2 * (D0 * D0 + up0 * up0);
    T p1 = eps + lp2 * (D1 * D1 + up1 * up1);
    T p2 = eps + lp2 * (D2 * D2 + up2 * up2);
    p0 = p0 * p0;
    p1 = p1 * p1;
    p2 = p2 * p2;
    // weights C_k prod_{j != k} p_j; the C_k folded into the candidates
    const T P12 = p1 * p2, P02 = p0 * p2, P01 = p0 * p1;
    const T Np = P12 * (T(0.2) * W[0] - T(0.7) * W[1] + T(1.1) * W[2]) +
                 P02 * (T(-0.6) * W[1] + T(3.0) * W[2] + T(1.2) * W[3]) +
                 P01 * (T(0.6) * W[2] + T(1.5) * W[3] - T(0.3) * W[4]);
    const T Sp = T(0.1) * P12 + T(0.6) * P02 + T(0.3) * P01;
    // - side: stencil W5..W1 (second differences are symmetric)
    const T un0 = T(0.5) * W[5] - T(2) * W[4] + T(1.5) * W[3];
    const T un1 = T(0.5) * (W[4] - W[2]);
    const T un2 = T(1.5) * W[3] - T(2) * W[2] + T(0.5) * W[1];
    T m0 = eps + ln2 * (D3 * D3 + un0 * un0);
    T m1 = eps + ln2 * (D2 * D2 + un1 * un1);
    T m2 = eps + ln2 * (D1 * D1 + un2 * un2);
    m0 = m0 * m0;
    m1 = m1 * m1;
    m2 = m2 * m2;
    const T M12 = m1 * m2, M02 = m0 * m2, M01 = m0 * m1;
    const T Nn = M12 * (T(0.2) * W[5] - T(0.7) * W[4] + T(1.1) * W[3]) +
                 M02 * (T(-0.6) * W[4] + T(3.0) * W[3] + T(1.2) * W[2]) +
                 M01 * (T(0.6) * W[3] + T(1.5) * W[2] - T(0.3) * W[1]);
    const T Sn = T(0.1) * M12 + T(0.6) * M02 + T(0.3) * M01;
    return (lp * Np * Sn + ln * Nn * Sp) * rcp<T>(T(6) * (Sp * Sn));
}

template <typename T>
__device__ __forceinline__ T weno3(T f0, T f1, T f2)
{
    const T eps = T(1.0e-6);
    T d0 = eps + (f1 - f0) * (f1 - f0);
    T d1 = eps + (f2 - f1) * (f2 - f1);
    d0 = d0 * d0;
    d1 = d1 * d1;
    const T a0 = d1;            // (1/3)/d0 scaled by 3*d0*d1
    const T a1 = T(2) * d0;     // (2/3)/d1 scaled by 3*d0*d1
    const T q0 = -f0 + T(3) * f1;
    const T q1 = f1 + f2;
    return (a0 * q0 + a1 * q1) * rcp<T>(T(2) * (a0 + a1));
}

// linear fifth-order upwind reconstruction (the WENO5 limit omega = C)
template <typename T>
__device__ __forceinline__ T upwind5(T f0, T f1, T f2, T f3, T f4)
{
    return (T(2) * f0 - T(13) * f1 + T(47) * f2 + T(27) * f3 - T(3) * f4) * T(1.0 / 60.0);
}

// ComputeFhat on a register stencil (see exact::fhat for the layout).
template <typename T, int S, int NP>
__device__ __forceinline__ void fhat(int jacobMean, int fluxSplit, T gamma, const T (&Ust)[6][5], T Fhat[5])
{
    constexpr int ctr = NP / 2 - 1;
    T Uo[6];
    interface_state<T>(jacobMean, gamma, Ust[ctr], Ust[ctr + 1], Uo);
    const T V[3] = {Uo[1], Uo[2], Uo[3]};
    const T hT = Uo[4];
    const T c = Uo[5];
    const T q = T(0.5) * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    const T d = rcp(T(2) * c);
    const T b = (gamma - T(1)) * (T(2) * d * d);  // (gamma-1)/(2c^2)
    const T b2 = T(2) * b;
    // eigenvalues and splitting
    T lam[5];
    lam[0] = V[S] - c;
    lam[1] = V[S];
    lam[2] = V[S];
    lam[3] = V[S];
    lam[4] = V[S] + c;
    T lp[5], ln[5];
    if (fluxSplit == 0) {
        const T ls = fabs(V[S]) + c;
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            lp[r] = T(0.5) * (lam[r] + ls);
            ln[r] = T(0.5) * (lam[r] - ls);
        }
    } else {
        const T e2 = T(1.0e-6);
#pragma unroll
        for (int r = 0; r < 5; ++r) {
            const T sr = sqrt(lam[r] * lam[r] + e2);
            lp[r] = T(0.5) * (lam[r] + sr);
            ln[r] = T(0.5) * (lam[r] - sr);
        }
    }
    // characteristic variables: W0 = bA + dB, W4 = bA - dB, W_{s+1} = U0 - 2bA,
    // W_{t+1} = U_{t+1} - 2b V_t A for the transverse components
    T W[NP][5];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
        const T *U = Ust[m];
        const T A = q * U[0] - V[0] * U[1] - V[1] * U[2] - V[2] * U[3] + U[4];
        const T B = V[S] * U[0] - U[S + 1];
        const T bA = b * A;
        W[m][0] = bA + d * B;
        W[m][4] = bA - d * B;
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            if (t == S) {
                W[m][t + 1] = U[0] - b2 * A;
            } else {
                W[m][t + 1] = U[t + 1] - b2 * V[t] * A;
            }
        }
    }
    T G[5];
#pragma unroll
    for (int r = 0; r < 5; ++r) {
        T hp, hn;
        if (NP == 6) {
            hp = weno5<T>(lp[r] * W[0][r], lp[r] * W[1][r], lp[r] * W[2][r], lp[r] * W[3][r], lp[r] * W[4][r]);
            hn = weno5<T>(ln[r] * W[5][r], ln[r] * W[4][r], ln[r] * W[3][r], ln[r] * W[2][r], ln[r] * W[1][r]);
        } else {
            hp = weno3<T>(lp[r] * W[0][r], lp[r] * W[1][r], lp[r] * W[2][r]);
            hn = weno3<T>(ln[r] * W[3][r], ln[r] * W[2][r], ln[r] * W[1][r]);
        }
        G[r] = hp + hn;
    }
    // back projection by the columns of R
    Fhat[0] = G[0] + G[S + 1] + G[4];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t == S) {
            Fhat[t + 1] = V[S] * (G[0] + G[S + 1] + G[4]) + c * (G[4] - G[0]);
        } else {
            Fhat[t + 1] = V[t] * (G[0] + G[4]) + G[t + 1];
        }
    }
    T e4 = hT * (G[0] + G[4]) + V[S] * c * (G[4] - G[0]) + (V[S] * V[S] - q) * G[S + 1];
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t != S) {
            e4 += V[t] * G[t + 1];
        }
    }
    Fhat[4] = e4;
}

}  // namespace fast
}  // namespace acfd

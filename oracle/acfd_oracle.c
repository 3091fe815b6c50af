/*
 * acfd_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * A CPU restatement of the ArtraCFD fluid time step.  Each function cites the
 * reference lines it follows.  Arithmetic is written in the reference's
 * evaluation order and must be compiled with -ffp-contract=off (as the
 * reference's -std=c99 x86-64 build is) so that FP64 results are bitwise equal
 * to the reference on identical inputs.  The data are the ABI types of
 * include/acfd.h (node records with the reference Node layout).
 */
#include "acfd_oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

enum { NX_ = 0, NY_ = 1, NZ_ = 2 };
enum { PIN_ = 0, PWB_ = 1, PEB_ = 2, PSB_ = 3, PNB_ = 4, PFB_ = 5, PBB_ = 6,
       PWG_ = 7, PEG_ = 8, PSG_ = 9, PNG_ = 10, PFG_ = 11, PBG_ = 12, PHY_ = 13, PAL_ = 14 };
enum { BC_INFLOW = 0, BC_OUTFLOW = 1, BC_SLIPWALL = 2, BC_NOSLIPWALL = 3, BC_PERIODIC = 4 };

static inline int nidx(const acfd_partition_t *part, int k, int j, int i)
{
    /* cfd_commons.c:323-326 */
    return (k * part->n[NY_] + j) * part->n[NX_] + i;
}

static inline double sq(double x) { return x * x; }

static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* ------------------------------------------------------------------------
 * state maps: cfd_commons.c:296-322
 * ------------------------------------------------------------------------ */
static void to_primitive(double gamma, double gasR, const double U[5], double Uo[6])
{
    Uo[0] = U[0];
    Uo[1] = U[1] / U[0];
    Uo[2] = U[2] / U[0];
    Uo[3] = U[3] / U[0];
    Uo[4] = (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]) * (gamma - 1.0);
    Uo[5] = Uo[4] / (Uo[0] * gasR);
}

static void to_conservative(double gamma, const double Uo[6], double U[5])
{
    U[0] = Uo[0];
    U[1] = Uo[0] * Uo[1];
    U[2] = Uo[0] * Uo[2];
    U[3] = Uo[0] * Uo[3];
    U[4] = 0.5 * Uo[0] * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3]) + Uo[4] / (gamma - 1.0);
}

static double temperature_cv(double cv, const double U[5])
{
    /* cfd_commons.c:310-313 */
    return (U[4] - 0.5 * (U[1] * U[1] + U[2] * U[2] + U[3] * U[3]) / U[0]) / (U[0] * cv);
}

static double sutherland(double T)
{
    /* cfd_commons.c:288-291 */
    return 1.458e-6 * pow(T, 1.5) / (T + 110.4);
}

/* ------------------------------------------------------------------------
 * interface average and eigen-system: cfd_commons.c:79-246
 * ------------------------------------------------------------------------ */
void orc_symmetric_average(int averager, double gamma, const double UL[5],
        const double UR[5], double Uo[6])
{
    /* left/right velocity and total enthalpy h_T = gamma*e_T - (gamma-1)|V|^2/2,
     * cfd_commons.c:82-91 */
    double vl[3], vr[3];
    for (int s = 0; s < 3; ++s) {
        vl[s] = UL[s + 1] / UL[0];
    }
    const double hl = (UL[4] / UL[0]) * gamma - 0.5 * (vl[0] * vl[0] + vl[1] * vl[1] + vl[2] * vl[2]) * (gamma - 1.0);
    for (int s = 0; s < 3; ++s) {
        vr[s] = UR[s + 1] / UR[0];
    }
    const double hr = (UR[4] / UR[0]) * gamma - 0.5 * (vr[0] * vr[0] + vr[1] * vr[1] + vr[2] * vr[2]) * (gamma - 1.0);
    if (0 == averager) {
        /* arithmetic mean, :94-99 */
        for (int s = 0; s < 3; ++s) {
            Uo[s + 1] = 0.5 * (vl[s] + vr[s]);
        }
        Uo[4] = 0.5 * (hl + hr);
    } else if (1 == averager) {
        /* Roe mean with D = sqrt(rhoR/rhoL), :100-106 */
        const double D = sqrt(UR[0] / UL[0]);
        for (int s = 0; s < 3; ++s) {
            Uo[s + 1] = (vl[s] + D * vr[s]) / (1.0 + D);
        }
        Uo[4] = (hl + D * hr) / (1.0 + D);
    }
    /* speed of sound, :110 */
    Uo[5] = sqrt((gamma - 1.0) * (Uo[4] - 0.5 * (Uo[1] * Uo[1] + Uo[2] * Uo[2] + Uo[3] * Uo[3])));
}

static void eigen_split(int splitter, int s, const double Uo[6], double lp[5], double ln[5])
{
    /* eigenvalues u_s-c, u_s, u_s, u_s, u_s+c (cfd_commons.c:113-121) */
    double lam[5];
    lam[0] = Uo[s + 1] - Uo[5];
    lam[1] = Uo[s + 1];
    lam[2] = Uo[s + 1];
    lam[3] = Uo[s + 1];
    lam[4] = Uo[s + 1] + Uo[5];
    if (0 == splitter) {
        /* local Lax-Friedrichs with lambda* = |u_s| + c written as
         * (|lam2| + lam4) - lam2, cfd_commons.c:128-138 */
        const double ls = fabs(lam[2]) + lam[4] - lam[2];
        for (int r = 0; r < 5; ++r) {
            lp[r] = 0.5 * (lam[r] + ls);
            ln[r] = 0.5 * (lam[r] - ls);
        }
    } else {
        /* Steger-Warming with epsilon = 1e-3, cfd_commons.c:139-148 */
        const double eps = 1.0e-3;
        for (int r = 0; r < 5; ++r) {
            lp[r] = 0.5 * (lam[r] + sqrt(lam[r] * lam[r] + eps * eps));
            ln[r] = 0.5 * (lam[r] - sqrt(lam[r] * lam[r] + eps * eps));
        }
    }
}

/*
 * Left eigenvectors (cfd_commons.c:149-205).  The three directions share one
 * pattern: two acoustic rows (0, 4), one row for the sweep direction's
 * velocity (entropy row) and two rows for the transverse velocity components.
 * Mixed velocity products are formed as (2b*V[hi])*V[lo] for hi > lo, exactly
 * as written in the reference for every direction.
 */
static void left_eigenvectors(int s, double gamma, const double Uo[6], double L[5][5])
{
    const double V[3] = {Uo[1], Uo[2], Uo[3]};
    const double c = Uo[5];
    const double q = 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    const double b = (gamma - 1.0) / (2.0 * c * c);
    const double d = 1.0 / (2.0 * c);
    /* acoustic rows */
    L[0][0] = b * q + d * V[s];
    L[4][0] = b * q - d * V[s];
    for (int t = 0; t < 3; ++t) {
        if (t == s) {
            L[0][t + 1] = -b * V[t] - d;
            L[4][t + 1] = -b * V[t] + d;
        } else {
            L[0][t + 1] = -b * V[t];
            L[4][t + 1] = -b * V[t];
        }
    }
    L[0][4] = b;
    L[4][4] = b;
    /* velocity rows: row index = component index + 1 */
    for (int a = 0; a < 3; ++a) {
        double *row = L[a + 1];
        if (a == s) {
            row[0] = -2.0 * b * q + 1.0;
            row[1] = 2.0 * b * V[0];
            row[2] = 2.0 * b * V[1];
            row[3] = 2.0 * b * V[2];
            row[4] = -2.0 * b;
            continue;
        }
        row[0] = -2.0 * b * q * V[a];
        for (int t = 0; t < 3; ++t) {
            const int hi = (a > t) ? a : t;
            const int lo = (a > t) ? t : a;
            row[t + 1] = 2.0 * b * V[hi] * V[lo];
            if (t == a) {
                row[t + 1] = row[t + 1] + 1.0;
            }
        }
        row[4] = -2.0 * b * V[a];
    }
}

static void right_eigenvectors(int s, const double Uo[6], double R[5][5])
{
    /* cfd_commons.c:206-246 */
    const double V[3] = {Uo[1], Uo[2], Uo[3]};
    const double hT = Uo[4];
    const double c = Uo[5];
    const double q = 0.5 * (V[0] * V[0] + V[1] * V[1] + V[2] * V[2]);
    memset(R, 0, 25 * sizeof(double));
    R[0][0] = 1.0;
    R[0][4] = 1.0;
    for (int t = 0; t < 3; ++t) {
        R[t + 1][0] = V[t];
        R[t + 1][4] = V[t];
    }
    R[s + 1][0] = V[s] - c;
    R[s + 1][4] = V[s] + c;
    R[4][0] = hT - V[s] * c;
    R[4][4] = hT + V[s] * c;
    for (int a = 0; a < 3; ++a) {
        /* column a+1: entropy wave along s, shear waves otherwise */
        if (a == s) {
            R[0][a + 1] = 1.0;
            R[s + 1][a + 1] = V[s];
            R[4][a + 1] = V[s] * V[s] - q;
        } else {
            R[a + 1][a + 1] = 1.0;
            R[4][a + 1] = V[a];
        }
    }
}

/* ------------------------------------------------------------------------
 * WENO: weno5.c:35-62, weno3.c:35-55 (Jiang & Shu 1996)
 * ------------------------------------------------------------------------ */
void orc_weno5(const double F[5][5], double Fhat[5])
{
    const double C0 = 1.0 / 10.0, C1 = 6.0 / 10.0, C2 = 3.0 / 10.0;
    const double eps = 1.0e-6;
    for (int r = 0; r < 5; ++r) {
        const double f0 = F[0][r], f1 = F[1][r], f2 = F[2][r], f3 = F[3][r], f4 = F[4][r];
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
        Fhat[r] = w0 * q0 + w1 * q1 + w2 * q2;
    }
}

void orc_weno3(const double F[3][5], double Fhat[5])
{
    const double C0 = 1.0 / 3.0, C1 = 2.0 / 3.0;
    const double eps = 1.0e-6;
    for (int r = 0; r < 5; ++r) {
        const double f0 = F[0][r], f1 = F[1][r], f2 = F[2][r];
        const double is0 = sq(f1 - f0);
        const double is1 = sq(f2 - f1);
        const double a0 = C0 / sq(eps + is0);
        const double a1 = C1 / sq(eps + is1);
        const double w0 = a0 / (a0 + a1);
        const double w1 = a1 / (a0 + a1);
        const double q0 = (1.0 / 2.0) * (-f0 + 3.0 * f1);
        const double q1 = (1.0 / 2.0) * (f1 + f2);
        Fhat[r] = w0 * q0 + w1 * q1;
    }
}

/* the left and right eigenvectors of direction s at the averaged state Uo
 * (rows of L, columns of R; EigenvectorL / EigenvectorR, cfd_commons.c:149-246) */
void orc_eigenvectors(int s, double gamma, const double Uo[6], double L[5][5], double R[5][5])
{
    left_eigenvectors(s, gamma, Uo, L);
    right_eigenvectors(s, Uo, R);
}

/* ------------------------------------------------------------------------
 * convective numerical flux at i+1/2: convective_flux.c:48-124
 * Ust holds U at the stencil points sL..sR along s (6 points for WENO5,
 * 4 for WENO3); the interface lies between Ust[-sL] and Ust[-sL+1].
 * ------------------------------------------------------------------------ */
void orc_fhat_stencil(const acfd_model_t *model, int s, const double Ust[6][5], double Fhat[5])
{
    const int npt = model->sR - model->sL + 1;  /* 6 or 4 */
    const int ctr = -model->sL;                 /* index of node i in Ust */
    double Uo[6];
    orc_symmetric_average(model->jacobMean, model->gamma, Ust[ctr], Ust[ctr + 1], Uo);
    double L[5][5], R[5][5], lp[5], ln[5];
    eigen_split(model->fluxSplit, s, Uo, lp, ln);
    left_eigenvectors(s, model->gamma, Uo, L);
    right_eigenvectors(s, Uo, R);
    /* characteristic variables W = L*U at every stencil point (:85-103) */
    double W[6][5];
    for (int m = 0; m < npt; ++m) {
        for (int r = 0; r < 5; ++r) {
            double acc = 0.0;
            for (int c = 0; c < 5; ++c) {
                acc = acc + L[r][c] * Ust[m][c];
            }
            W[m][r] = acc;
        }
    }
    /* split characteristic fluxes; the negative one runs backwards (:104-113) */
    const int tot = npt - 1;
    double Hp[5][5], Hn[5][5], hp[5], hn[5];
    for (int m = 0; m < tot; ++m) {
        for (int r = 0; r < 5; ++r) {
            Hp[m][r] = lp[r] * W[m][r];
            Hn[m][r] = ln[r] * W[tot - m][r];
        }
    }
    if (1 == model->sScheme) {
        orc_weno5((const double (*)[5])Hp, hp);
        orc_weno5((const double (*)[5])Hn, hn);
    } else {
        orc_weno3((const double (*)[5])Hp, hp);
        orc_weno3((const double (*)[5])Hn, hn);
    }
    /* back to physical space (:114-124) */
    for (int r = 0; r < 5; ++r) {
        double acc = 0.0;
        for (int c = 0; c < 5; ++c) {
            acc = acc + R[r][c] * (hp[c] + hn[c]);
        }
        Fhat[r] = acc;
    }
}

void orc_compute_fhat(int tn, int s, int k, int j, int i, const acfd_partition_t *part,
        const acfd_node_t *node, const acfd_model_t *model, double Fhat[5])
{
    const int h[3] = {s == 0, s == 1, s == 2};
    double Ust[6][5];
    for (int n = model->sL, m = 0; n <= model->sR; ++n, ++m) {
        const int id = nidx(part, k + n * h[2], j + n * h[1], i + n * h[0]);
        memcpy(Ust[m], node[id].U[tn], sizeof(Ust[m]));
    }
    orc_fhat_stencil(model, s, (const double (*)[5])Ust, Fhat);
}

/* ------------------------------------------------------------------------
 * viscous numerical flux at i+1/2: diffusive_flux.c:46-312
 * Velocity gradients: normal ones by a two-point difference, transverse ones
 * by the average of the two centred differences at i and i+1.
 * ------------------------------------------------------------------------ */
static void velocity_at(const acfd_node_t *nd, int tn, double V[3])
{
    const double *U = nd->U[tn];
    V[0] = U[1] / U[0];
    V[1] = U[2] / U[0];
    V[2] = U[3] / U[0];
}

void orc_compute_fvhat(int tn, int s, int k, int j, int i, const acfd_partition_t *part,
        const acfd_node_t *node, const acfd_model_t *model, double Fvhat[5])
{
    if (0.0 >= model->refMu) {
        memset(Fvhat, 0, 5 * sizeof(double));
        return;
    }
    const double *dd = part->dd;
    int o[3] = {i, j, k};
    /* nodes: C (i), P (i+1 along s), and for each transverse t: C-t, C+t, P-t, P+t */
    int cs[3], ps[3];
    memcpy(cs, o, sizeof(cs));
    memcpy(ps, o, sizeof(ps));
    ps[s] += 1;
    double Vc[3], Vp[3];
    velocity_at(&node[nidx(part, cs[2], cs[1], cs[0])], tn, Vc);
    velocity_at(&node[nidx(part, ps[2], ps[1], ps[0])], tn, Vp);
    const double Tc = temperature_cv(model->cv, node[nidx(part, cs[2], cs[1], cs[0])].U[tn]);
    const double Tp = temperature_cv(model->cv, node[nidx(part, ps[2], ps[1], ps[0])].U[tn]);
    /* grad[a][b] = d V_a / d x_b at the interface */
    double grad[3][3];
    for (int a = 0; a < 3; ++a) {
        grad[a][s] = (Vp[a] - Vc[a]) * dd[s];
    }
    for (int t = 0; t < 3; ++t) {
        if (t == s) {
            continue;
        }
        int cm[3], cp[3], pm[3], pp[3];
        memcpy(cm, cs, sizeof(cm)); cm[t] -= 1;
        memcpy(cp, cs, sizeof(cp)); cp[t] += 1;
        memcpy(pm, ps, sizeof(pm)); pm[t] -= 1;
        memcpy(pp, ps, sizeof(pp)); pp[t] += 1;
        double Vcm[3], Vcp[3], Vpm[3], Vpp[3];
        velocity_at(&node[nidx(part, cm[2], cm[1], cm[0])], tn, Vcm);
        velocity_at(&node[nidx(part, cp[2], cp[1], cp[0])], tn, Vcp);
        velocity_at(&node[nidx(part, pm[2], pm[1], pm[0])], tn, Vpm);
        velocity_at(&node[nidx(part, pp[2], pp[1], pp[0])], tn, Vpp);
        for (int a = 0; a < 3; ++a) {
            /* 0.25 * (V(c+t) + V(p+t) - V(c-t) - V(p-t)) * dd[t] */
            grad[a][t] = 0.25 * (Vcp[a] + Vpp[a] - Vcm[a] - Vpm[a]) * dd[t];
        }
    }
    const double dT = (Tp - Tc) * dd[s];
    double Vh[3];
    for (int a = 0; a < 3; ++a) {
        Vh[a] = 0.5 * (Vc[a] + Vp[a]);
    }
    const double Th = 0.5 * (Tc + Tp);
    const double mu = model->refMu * sutherland(Th * model->refT);
    const double heatK = model->gamma * model->cv * mu / 0.71;
    const double divV = grad[0][0] + grad[1][1] + grad[2][2];
    /* stress row s; the order of the two shear terms follows each
     * ComputeFvhatX/Y/Z: tau_sa = mu*(dV_a/dx_s + dV_s/dx_a) written with the
     * lower-index component's derivative first for X, and as listed below */
    double tau[3];
    for (int a = 0; a < 3; ++a) {
        if (a == s) {
            tau[a] = mu * (grad[s][s] + grad[s][s] - (2.0 / 3.0) * divV);
        }
    }
    if (0 == s) {
        tau[1] = mu * (grad[0][1] + grad[1][0]);   /* du_dy + dv_dx, :138 */
        tau[2] = mu * (grad[0][2] + grad[2][0]);   /* du_dz + dw_dx, :139 */
    } else if (1 == s) {
        tau[0] = mu * (grad[1][0] + grad[0][1]);   /* dv_dx + du_dy, :222 */
        tau[2] = mu * (grad[1][2] + grad[2][1]);   /* dv_dz + dw_dy, :224 */
    } else {
        tau[0] = mu * (grad[2][0] + grad[0][2]);   /* dw_dx + du_dz, :307 */
        tau[1] = mu * (grad[2][1] + grad[1][2]);   /* dw_dy + dv_dz, :308 */
    }
    Fvhat[0] = 0.0;
    Fvhat[1] = tau[0];
    Fvhat[2] = tau[1];
    Fvhat[3] = tau[2];
    Fvhat[4] = heatK * dT + Fvhat[1] * Vh[0] + Fvhat[2] * Vh[1] + Fvhat[3] * Vh[2];
}

/* gravity source: source_term.c:21-39 */
static void source_phi(int tn, int k, int j, int i, const acfd_partition_t *part,
        const acfd_node_t *node, const acfd_model_t *model, double Phi[5])
{
    if (0 == model->sState) {
        memset(Phi, 0, 5 * sizeof(double));
        return;
    }
    const double *U = node[nidx(part, k, j, i)].U[tn];
    const double V[3] = {U[1] / U[0], U[2] / U[0], U[3] / U[0]};
    const double fb[3] = {U[0] * model->g[0], U[0] * model->g[1], U[0] * model->g[2]};
    Phi[0] = 0.0;
    Phi[1] = fb[0];
    Phi[2] = fb[1];
    Phi[3] = fb[2];
    Phi[4] = fb[0] * V[0] + fb[1] * V[1] + fb[2] * V[2];
}

/* ------------------------------------------------------------------------
 * one stage: fluid_dynamics.c:157-274
 * ------------------------------------------------------------------------ */
static void stage_update(int multidim, int s, double coeA, double coeB, const double *Uo,
        const double *Un, double *Um, double r, const double Phi[5])
{
    if ((1 == multidim) && (0 != s)) {
        for (int n = 0; n < 5; ++n) {
            Um[n] = Um[n] + coeB * r * Phi[n];
        }
        return;
    }
    for (int n = 0; n < 5; ++n) {
        Um[n] = coeA * Uo[n] + coeB * (Un[n] + r * Phi[n]);
    }
}

void orc_lllu(double dt, double coeA, double coeB, int to, int tn, int tm, int p,
        acfd_node_t *node, const acfd_partition_t *part, const acfd_model_t *model)
{
    const double r[3] = {dt * part->dd[0], dt * part->dd[1], dt * part->dd[2]};
    int s0, s1;
    if (ACFD_PHI == p) {
        s0 = 0; s1 = 1;
    } else if (ACFD_DIMS == p) {
        s0 = 0; s1 = 3;
    } else {
        s0 = p; s1 = p + 1;
    }
    for (int s = s0; s < s1; ++s) {
        const int h[3] = {s == 0, s == 1, s == 2};
        for (int c2 = part->np[s][2][0]; c2 < part->np[s][2][1]; ++c2) {
            for (int c1 = part->np[s][1][0]; c1 < part->np[s][1][1]; ++c1) {
                /* flux at the left interface of the previous node is carried
                 * over; recomputed at each line start and after a solid node */
                double fl[5], fr[5], vl[5], vr[5], Phi[5];
                int have_left = 0;
                for (int c0 = part->np[s][0][0]; c0 < part->np[s][0][1]; ++c0) {
                    int i, j, k;
                    if (0 == s) { i = c0; j = c1; k = c2; }
                    else if (1 == s) { i = c1; j = c0; k = c2; }
                    else { i = c1; j = c2; k = c0; }
                    const int id = nidx(part, k, j, i);
                    if (0 != node[id].did) {
                        have_left = 0;
                        continue;
                    }
                    if (ACFD_PHI == p) {
                        source_phi(tn, k, j, i, part, node, model, Phi);
                        stage_update(0, s, coeA, coeB, node[id].U[to], node[id].U[tn],
                                node[id].U[tm], dt, Phi);
                        continue;
                    }
                    if (have_left) {
                        memcpy(fl, fr, sizeof(fl));
                        memcpy(vl, vr, sizeof(vl));
                    } else {
                        orc_compute_fhat(tn, s, k - h[2], j - h[1], i - h[0], part, node, model, fl);
                        orc_compute_fvhat(tn, s, k - h[2], j - h[1], i - h[0], part, node, model, vl);
                        have_left = 1;
                    }
                    orc_compute_fhat(tn, s, k, j, i, part, node, model, fr);
                    orc_compute_fvhat(tn, s, k, j, i, part, node, model, vr);
                    for (int n = 0; n < 5; ++n) {
                        Phi[n] = fl[n] - fr[n] + vr[n] - vl[n];
                    }
                    stage_update(model->multidim, s, coeA, coeB, node[id].U[to], node[id].U[tn],
                            node[id].U[tm], r[s], Phi);
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * domain ghost fill: boundary_treatment.c:28-192
 * ------------------------------------------------------------------------ */
static void mirror_over(const double UoI[6], const double UoO[6], double UoG[6])
{
    /* method of images, immersed_boundary.c:341-356 */
    UoG[1] = UoO[1] + UoO[1] - UoI[1];
    UoG[2] = UoO[2] + UoO[2] - UoI[2];
    UoG[3] = UoO[3] + UoO[3] - UoI[3];
    UoG[4] = UoI[4];
    UoG[5] = UoI[5];
}

static void fill_face(int p, int r, const int box[3][2], int tn, acfd_node_t *node,
        const acfd_partition_t *part, const acfd_model_t *model)
{
    const int *N = part->N[p];
    const int type = part->typeBC[p];
    const double *given = part->varBC[p];
    const int LN[3] = {part->m[0] * N[0], part->m[1] * N[1], part->m[2] * N[2]};
    for (int k = box[2][0]; k < box[2][1]; ++k) {
        for (int j = box[1][0]; j < box[1][1]; ++j) {
            for (int i = box[0][0]; i < box[0][1]; ++i) {
                double *U = node[nidx(part, k, j, i)].U[tn];
                if (0 != r) {
                    /* ghost layer r */
                    if ((BC_SLIPWALL == type) || (BC_NOSLIPWALL == type)) {
                        double UoO[6], UoI[6], UoG[6];
                        to_primitive(model->gamma, model->gasR,
                                node[nidx(part, k - r * N[2], j - r * N[1], i - r * N[0])].U[tn], UoO);
                        to_primitive(model->gamma, model->gasR,
                                node[nidx(part, k - 2 * r * N[2], j - 2 * r * N[1], i - 2 * r * N[0])].U[tn], UoI);
                        mirror_over(UoI, UoO, UoG);
                        UoG[0] = UoG[4] / (UoG[5] * model->gasR);
                        to_conservative(model->gamma, UoG, U);
                    } else if (BC_PERIODIC == type) {
                        memcpy(U, node[nidx(part, k - LN[2], j - LN[1], i - LN[0])].U[tn], 5 * sizeof(double));
                    } else {
                        memcpy(U, node[nidx(part, k - N[2], j - N[1], i - N[0])].U[tn], 5 * sizeof(double));
                    }
                    continue;
                }
                /* physical boundary node */
                const double *Uh = node[nidx(part, k - N[2], j - N[1], i - N[0])].U[tn];
                double Uoh[6], UoO[6];
                switch (type) {
                    case BC_INFLOW:
                        to_conservative(model->gamma, given, U);
                        break;
                    case BC_OUTFLOW:
                        memcpy(U, Uh, 5 * sizeof(double));
                        break;
                    case BC_SLIPWALL:
                    case BC_NOSLIPWALL:
                        to_primitive(model->gamma, model->gasR, Uh, Uoh);
                        if (BC_SLIPWALL == type) {
                            /* zero normal velocity, zero-gradient tangential */
                            UoO[1] = (!N[0]) * Uoh[1];
                            UoO[2] = (!N[1]) * Uoh[2];
                            UoO[3] = (!N[2]) * Uoh[3];
                        } else {
                            UoO[1] = 0.0;
                            UoO[2] = 0.0;
                            UoO[3] = 0.0;
                        }
                        UoO[4] = Uoh[4];
                        UoO[5] = (0.0 > given[5]) ? Uoh[5] : given[5];
                        UoO[0] = UoO[4] / (UoO[5] * model->gasR);
                        to_conservative(model->gamma, UoO, U);
                        break;
                    default:
                        break;
                }
            }
        }
    }
}

void orc_treat_domain_boundary(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model)
{
    const int *ng = part->ng;
    const int R = imax(ng[0], imax(ng[1], ng[2]));
    for (int r = 0; r <= R; ++r) {
        for (int p = PWB_; p <= PBB_; ++p) {
            const int *N = part->N[p];
            int box[3][2];
            int empty = 0;
            for (int s = 0; s < 3; ++s) {
                /* layer r of face p grows tangentially by r (capped at ng),
                 * boundary_treatment.c:54-57 */
                const int w = imin(r, ng[s]);
                box[s][0] = part->ns[p][s][0] + w * (N[s] - !N[s]);
                box[s][1] = part->ns[p][s][1] + w * (N[s] + !N[s]) - (ng[s] < r) * (!!N[s]);
                if (box[s][0] >= box[s][1]) {
                    empty = 1;
                }
            }
            if (!empty) {
                fill_face(p, r, (const int (*)[2])box, tn, node, part, model);
            }
        }
    }
}

void orc_treat_boundary(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    /* immersed ghosts first, then the domain shells (boundary_treatment.c:28-65) */
    orc_treat_ib(tn, node, part, model, poly, totN);
    orc_treat_domain_boundary(tn, node, part, model);
}

/* ------------------------------------------------------------------------
 * RK stages and Strang schedule: fluid_dynamics.c:55-148
 * ------------------------------------------------------------------------ */
void orc_discretize_time(double dt, int s, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    if (0 == model->tScheme) {
        orc_lllu(dt, 0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN, s, node, part, model);
        orc_treat_boundary(ACFD_TN, node, part, model, poly, totN);
        orc_lllu(dt, 1.0 / 2.0, 1.0 / 2.0, ACFD_TO, ACFD_TN, ACFD_TO, s, node, part, model);
        orc_treat_boundary(ACFD_TO, node, part, model, poly, totN);
        return;
    }
    orc_lllu(dt, 0.0, 1.0, ACFD_TO, ACFD_TO, ACFD_TN, s, node, part, model);
    orc_treat_boundary(ACFD_TN, node, part, model, poly, totN);
    orc_lllu(dt, 3.0 / 4.0, 1.0 / 4.0, ACFD_TO, ACFD_TN, ACFD_TM, s, node, part, model);
    orc_treat_boundary(ACFD_TM, node, part, model, poly, totN);
    orc_lllu(dt, 1.0 / 3.0, 2.0 / 3.0, ACFD_TO, ACFD_TM, ACFD_TO, s, node, part, model);
    orc_treat_boundary(ACFD_TO, node, part, model, poly, totN);
}

void orc_evolve_fluid(double dt, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    /* sweep order per collapse tag, fluid_dynamics.c:60-103; other tags
     * (e.g. all three dimensions collapsed) take no directional sweep */
    int order[6];
    int count = 0;
    switch (part->collapse) {
        case 0: { const int o[6] = {2, 1, 0, 0, 1, 2}; memcpy(order, o, sizeof(o)); count = 6; } break;
        case 1: { const int o[4] = {2, 1, 1, 2}; memcpy(order, o, sizeof(o)); count = 4; } break;
        case 2: { const int o[4] = {2, 0, 0, 2}; memcpy(order, o, sizeof(o)); count = 4; } break;
        case 3: { const int o[4] = {1, 0, 0, 1}; memcpy(order, o, sizeof(o)); count = 4; } break;
        case 5: order[0] = 2; order[1] = 2; count = 2; break;
        case 7: order[0] = 1; order[1] = 1; count = 2; break;
        case 8: order[0] = 0; order[1] = 0; count = 2; break;
        default: count = 0; break;
    }
    const double hdt = 0.5 * dt;
    if (0 != model->sState) {
        orc_discretize_time(hdt, ACFD_PHI, node, part, model, poly, totN);
    }
    if (0 == model->multidim) {
        for (int n = 0; n < count; ++n) {
            orc_discretize_time(hdt, order[n], node, part, model, poly, totN);
        }
    } else if (1 == model->multidim) {
        orc_discretize_time(hdt, ACFD_DIMS, node, part, model, poly, totN);
        orc_discretize_time(hdt, ACFD_DIMS, node, part, model, poly, totN);
    }
    if (0 != model->sState) {
        orc_discretize_time(hdt, ACFD_PHI, node, part, model, poly, totN);
    }
}

/* ------------------------------------------------------------------------
 * CFL: solve.c:108-153
 * ------------------------------------------------------------------------ */
void orc_cfl(const acfd_node_t *node, const acfd_partition_t *part, const acfd_model_t *model,
        double vmax[3])
{
    for (int k = part->ns[PIN_][2][0]; k < part->ns[PIN_][2][1]; ++k) {
        for (int j = part->ns[PIN_][1][0]; j < part->ns[PIN_][1][1]; ++j) {
            for (int i = part->ns[PIN_][0][0]; i < part->ns[PIN_][0][1]; ++i) {
                const acfd_node_t *nd = &node[nidx(part, k, j, i)];
                if (0 != nd->did) {
                    continue;
                }
                double Uo[6];
                to_primitive(model->gamma, model->gasR, nd->U[ACFD_TO], Uo);
                const double c = sqrt(model->gamma * model->gasR * Uo[5]);
                for (int s = 0; s < 3; ++s) {
                    const double V = fabs(Uo[s + 1]) + c;
                    if (vmax[s] < V) {
                        vmax[s] = V;
                    }
                }
            }
        }
    }
}

static double dmin(double x, double y) { return (x < y) ? x : y; }
static double dmax(double x, double y) { return (x > y) ? x : y; }

double orc_time_step(double numCFL, const acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    double vmax[3] = {0.0, 0.0, 0.0};
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t *P = poly + n;
        double V[3];
        V[0] = fabs(P->V[0]) + dmax(fabs(P->W[1]), fabs(P->W[2])) * P->r;
        V[1] = fabs(P->V[1]) + dmax(fabs(P->W[2]), fabs(P->W[0])) * P->r;
        V[2] = fabs(P->V[2]) + dmax(fabs(P->W[0]), fabs(P->W[1])) * P->r;
        for (int s = 0; s < 3; ++s) {
            if (vmax[s] < V[s]) {
                vmax[s] = V[s];
            }
        }
    }
    orc_cfl(node, part, model, vmax);
    return numCFL * dmin(part->d[0] / vmax[0], dmin(part->d[1] / vmax[1], part->d[2] / vmax[2]));
}

/* ------------------------------------------------------------------------
 * host set-up: cfd_parameters.c:46-124, domain_partition.c:19-150
 * ------------------------------------------------------------------------ */
void orc_set_node_number(acfd_partition_t *part, acfd_model_t *model)
{
    part->collapse = 0;
    if (0 == part->m[2] - 1) {
        part->collapse = 3;
    }
    if (0 == part->m[1] - 1) {
        part->collapse = 2 * part->collapse + 2;
    }
    if (0 == part->m[0] - 1) {
        part->collapse = 2 * part->collapse + 1;
    }
    if (0 == model->sScheme) {
        model->sL = -1; model->sR = 2; part->gl = 2;
    } else {
        model->sL = -2; model->sR = 3; part->gl = 3;
    }
    for (int s = 0; s < 3; ++s) {
        part->ng[s] = part->gl - 1;
    }
    if (0 == model->multidim) {
        const int c = part->collapse;
        if (1 == c || 5 == c || 7 == c) part->ng[0] = 0;
        if (2 == c || 5 == c || 8 == c) part->ng[1] = 0;
        if (3 == c || 7 == c || 8 == c) part->ng[2] = 0;
    }
    for (int s = 0; s < 3; ++s) {
        if (BC_PERIODIC == part->typeBC[1 + 2 * s]) {
            part->ng[s] = part->gl;
        }
    }
    for (int s = 0; s < 3; ++s) {
        part->m[s] = imax(part->m[s], 2);
        part->n[s] = part->m[s] + 1 + 2 * part->ng[s];
    }
    for (int s = 0; s < 3; ++s) {
        part->d[s] = (part->domain[s][1] - part->domain[s][0]) / (double)(part->m[s]);
        part->dd[s] = 1.0 / part->d[s];
    }
    part->tinyL = 1.0e-6 * dmin(part->d[0], dmin(part->d[1], part->d[2]));
    part->tinyL = part->tinyL * part->tinyL;
}

void orc_partition_domain(acfd_partition_t *part)
{
    static const int normals[7][3] = {{0, 0, 0}, {-1, 0, 0}, {1, 0, 0},
        {0, -1, 0}, {0, 1, 0}, {0, 0, -1}, {0, 0, 1}};
    memcpy(part->N, normals, sizeof(normals));
    for (int s = 0; s < 3; ++s) {
        const int lo = part->ng[s], hi = part->n[s] - part->ng[s];
        if (BC_PERIODIC == part->typeBC[1 + 2 * s]) {
            part->ns[PIN_][s][0] = lo;
            part->ns[PIN_][s][1] = hi;
        } else {
            part->ns[PIN_][s][0] = lo + 1;
            part->ns[PIN_][s][1] = hi - 1;
        }
        for (int p = PWB_; p <= PBB_; ++p) {
            part->ns[p][s][0] = lo;
            part->ns[p][s][1] = hi;
        }
        for (int p = PWG_; p <= PBG_; ++p) {
            part->ns[p][s][0] = 0;
            part->ns[p][s][1] = part->n[s];
        }
        part->ns[PHY_][s][0] = lo;
        part->ns[PHY_][s][1] = hi;
        part->ns[PAL_][s][0] = 0;
        part->ns[PAL_][s][1] = part->n[s];
    }
    for (int s = 0; s < 3; ++s) {
        /* boundary planes and ghost slabs of the two faces normal to s */
        part->ns[PWB_ + 2 * s][s][1] = part->ns[PWB_ + 2 * s][s][0] + 1;
        part->ns[PEB_ + 2 * s][s][0] = part->ns[PEB_ + 2 * s][s][1] - 1;
        part->ns[PWG_ + 2 * s][s][1] = part->ng[s];
        part->ns[PEG_ + 2 * s][s][0] = part->n[s] - part->ng[s];
    }
    /* dimension priority: the sweep direction runs innermost */
    static const int pri[3][3] = {{0, 1, 2}, {1, 0, 2}, {2, 0, 1}};
    for (int n = 0; n < 3; ++n) {
        for (int s = 0; s < 3; ++s) {
            part->np[n][s][0] = part->ns[PIN_][pri[n][s]][0];
            part->np[n][s][1] = part->ns[PIN_][pri[n][s]][1];
        }
    }
    /* interfacial search path: 6 face neighbours, 12 edge neighbours,
     * 6 at distance 2, 6 at distance 3 (domain_partition.c:130-149) */
    int n = 0;
    for (int s = 0; s < 3; ++s) {
        for (int sg = -1; sg <= 1; sg += 2) {
            memset(part->path[n], 0, sizeof(part->path[n]));
            part->path[n][s] = sg;
            ++n;
        }
    }
    static const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int q = 0; q < 3; ++q) {
        for (int b = -1; b <= 1; b += 2) {
            for (int a = -1; a <= 1; a += 2) {
                memset(part->path[n], 0, sizeof(part->path[n]));
                part->path[n][pairs[q][0]] = a;
                part->path[n][pairs[q][1]] = b;
                ++n;
            }
        }
    }
    for (int dist = 2; dist <= 3; ++dist) {
        for (int s = 0; s < 3; ++s) {
            for (int sg = -1; sg <= 1; sg += 2) {
                memset(part->path[n], 0, sizeof(part->path[n]));
                part->path[n][s] = sg * dist;
                ++n;
            }
        }
    }
    part->pathSep[1] = 6;
    part->pathSep[2] = part->pathSep[1] + 18;
    part->pathSep[3] = part->pathSep[2] + 6;
    part->pathSep[0] = part->pathSep[part->gl];
}

/*
 * acfd_oracle_ib.c -- TEST INFRASTRUCTURE ONLY (the parity checker).
 *
 * CPU restatement of the immersed-boundary node mapping and ghost-node
 * reconstruction of ArtraCFD (immersed_boundary.c, computational_geometry.c),
 * and of the node scans and surface motion of the rigid-body step
 * (IntegrateSurfaceForce and the contact scan of ApplyCollision,
 * solid_dynamics.c; TransformPolyhedron, computational_geometry.c).
 * Same evaluation order as the reference; build with -ffp-contract=off.
 */
#include "acfd_oracle.h"

#include <float.h>
#include <math.h>
#include <string.h>

enum { PIN_ = 0 };
enum { IB_R = 2, TYPED_ = -1, TYPEF_ = -2 };

static inline int nidx(const acfd_partition_t *part, int k, int j, int i)
{
    return (k * part->n[1] + j) * part->n[0] + i;
}

static inline double dot3(const double a[3], const double b[3])
{
    /* cfd_commons.c:407-410 */
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

static inline double dist2(const double a[3], const double b[3])
{
    const double v[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
    return dot3(v, v);
}

static inline int in_pin(const acfd_partition_t *part, int k, int j, int i)
{
    /* cfd_commons.c:327-333 */
    return (part->ns[PIN_][2][0] <= k) && (part->ns[PIN_][2][1] > k) &&
        (part->ns[PIN_][1][0] <= j) && (part->ns[PIN_][1][1] > j) &&
        (part->ns[PIN_][0][0] <= i) && (part->ns[PIN_][0][1] > i);
}

static inline int map_node(double s, double smin, double dds, int ng)
{
    /* cfd_commons.c:340-343 */
    return (int)((s - smin) * dds + 0.5) + ng;
}

static inline int confine(int n, int lo, int hi)
{
    /* cfd_commons.c:344-347 */
    const int a = (lo > n) ? lo : n;
    return (hi - 1 < a) ? hi - 1 : a;
}

static inline double map_point(int n, double smin, double ds, int ng)
{
    /* cfd_commons.c:348-351 */
    return smin + (n - ng) * ds;
}

static void node_point(const acfd_partition_t *part, int k, int j, int i, double p[3])
{
    p[0] = map_point(i, part->domain[0][0], part->d[0], part->ng[0]);
    p[1] = map_point(j, part->domain[1][0], part->d[1], part->ng[1]);
    p[2] = map_point(k, part->domain[2][0], part->d[2], part->ng[2]);
}

static void body_box(const acfd_partition_t *part, const acfd_polyhedron_t *P, int box[3][2])
{
    /* node-space box of a body confined to PIN (immersed_boundary.c:151-154) */
    for (int s = 0; s < 3; ++s) {
        const int lo = part->ns[PIN_][s][0], hi = part->ns[PIN_][s][1];
        box[s][0] = confine(map_node(P->box[s][0], part->domain[s][0], part->dd[s], part->ng[s]), lo, hi);
        box[s][1] = confine(map_node(P->box[s][1], part->domain[s][0], part->dd[s], part->ng[s]), lo, hi) + 1;
    }
}

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

/* ------------------------------------------------------------------------
 * point to triangle: computational_geometry.c:449-761 (Eberly 1999)
 * ------------------------------------------------------------------------ */
static void triangle(const acfd_polyhedron_t *P, int f, double v0[3], double v1[3],
        double v2[3], double e01[3], double e02[3])
{
    for (int s = 0; s < 3; ++s) {
        v0[s] = P->v[3 * P->f[3 * f + 0] + s];
        v1[s] = P->v[3 * P->f[3 * f + 1] + s];
        v2[s] = P->v[3 * P->f[3 * f + 2] + s];
        e01[s] = v1[s] - v0[s];
        e02[s] = v2[s] - v0[s];
    }
}

static double point_triangle(const double p[3], const double v0[3], const double e01[3],
        const double e02[3], double para[3])
{
    const double D[3] = {v0[0] - p[0], v0[1] - p[1], v0[2] - p[2]};
    const double a = dot3(e01, e01), b = dot3(e01, e02), c = dot3(e02, e02);
    const double d = dot3(e01, D), e = dot3(e02, D), f = dot3(D, D);
    const double det = a * c - b * b;
    double s = b * e - c * d;
    double t = b * d - a * e;
    double q;
    /* the seven regions of the (s,t) plane */
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

static int find_edge(const acfd_polyhedron_t *P, int v0, int v1)
{
    /* binary search of the sorted edge list, computational_geometry.c:137-161 */
    const int hi = (v0 > v1) ? v0 : v1, lo = (v0 > v1) ? v1 : v0;
    int a = 0, b = P->edgeN - 1;
    while (a <= b) {
        const int m = (a + b) / 2;
        const int *e = P->e + 4 * m;
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

static void closest_on_facet(const double p[3], int fid, const acfd_polyhedron_t *P,
        double pi[3], double N[3])
{
    /* closest point and its pseudo-normal (vertex, edge or face),
     * computational_geometry.c:689-761 */
    double v0[3], v1[3], v2[3], e01[3], e02[3], para[3];
    const int *fv = P->f + 3 * fid;
    triangle(P, fid, v0, v1, v2, e01, e02);
    point_triangle(p, v0, e01, e02, para);
    const double *nrm;
    int kind; /* 0 v0, 1 v1, 2 v2, 3 edge 02, 4 edge 01, 5 edge 12, 6 face */
    if (0.0 == para[1]) {
        if (0.0 == para[2]) kind = 0;
        else if (1.0 == para[2]) kind = 2;
        else kind = 3;
    } else if (1.0 == para[1]) {
        kind = 1;
    } else if (0.0 == para[2]) {
        kind = 4;
    } else if (0.0 == para[0]) {
        kind = 5;
    } else {
        kind = 6;
    }
    switch (kind) {
        case 0: nrm = P->Nv + 3 * fv[0]; for (int s = 0; s < 3; ++s) pi[s] = v0[s]; break;
        case 1: nrm = P->Nv + 3 * fv[1]; for (int s = 0; s < 3; ++s) pi[s] = v1[s]; break;
        case 2: nrm = P->Nv + 3 * fv[2]; for (int s = 0; s < 3; ++s) pi[s] = v2[s]; break;
        case 3:
            nrm = P->Ne + 3 * find_edge(P, fv[0], fv[2]);
            for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[2] * e02[s];
            break;
        case 4:
            nrm = P->Ne + 3 * find_edge(P, fv[0], fv[1]);
            for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s];
            break;
        case 5:
            nrm = P->Ne + 3 * find_edge(P, fv[1], fv[2]);
            for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s] + para[2] * e02[s];
            break;
        default:
            nrm = P->Nf + 3 * fid;
            for (int s = 0; s < 3; ++s) pi[s] = v0[s] + para[1] * e01[s] + para[2] * e02[s];
            break;
    }
    for (int s = 0; s < 3; ++s) {
        N[s] = nrm[s];
    }
}

int orc_point_in_polyhedron(const double p[3], const acfd_polyhedron_t *P, int *fid)
{
    /* nearest facet by brute force (first minimum wins), then the sign of
     * (p - closest).N, computational_geometry.c:463-506 */
    double best = FLT_MAX;
    int cid = 0;
    for (int n = 0; n < P->faceN; ++n) {
        double v0[3], v1[3], v2[3], e01[3], e02[3], para[3];
        triangle(P, n, v0, v1, v2, e01, e02);
        const double q = point_triangle(p, v0, e01, e02, para);
        if (best > q) {
            best = q;
            cid = n;
        }
    }
    *fid = cid;
    double pi[3], N[3];
    closest_on_facet(p, cid, P, pi, N);
    pi[0] = p[0] - pi[0];
    pi[1] = p[1] - pi[1];
    pi[2] = p[2] - pi[2];
    return (0.0 < dot3(pi, N)) ? 0 : 1;
}

static void surface_data(const double p[3], int fid, const acfd_polyhedron_t *P,
        double pi[3], double pm[3], double N[3])
{
    /* boundary point, image point and normal, computational_geometry.c:762-783 */
    if (0 >= P->faceN) {
        N[0] = p[0] - P->O[0];
        N[1] = p[1] - P->O[1];
        N[2] = p[2] - P->O[2];
        double dist = sqrt(dot3(N, N));
        for (int s = 0; s < 3; ++s) {
            N[s] = N[s] / dist;
        }
        dist = P->r - dist;
        for (int s = 0; s < 3; ++s) {
            pi[s] = p[s] + dist * N[s];
        }
    } else {
        closest_on_facet(p, fid, P, pi, N);
    }
    for (int s = 0; s < 3; ++s) {
        pm[s] = pi[s] + pi[s] - p[s];
    }
}

/* ------------------------------------------------------------------------
 * inverse distance weighting: immersed_boundary.c:413-487
 * ------------------------------------------------------------------------ */
static void add_weighted(const double Uoh[6], double tiny, double w, double *wsum, double Uo[6])
{
    if (tiny > w) {
        w = tiny;
    }
    w = 1.0 / w;
    for (int n = 0; n < 6; ++n) {
        Uo[n] = Uo[n] + Uoh[n] * w;
    }
    *wsum = *wsum + w;
}

static double idw(int tn, const int c[3], const double p[3], int h, int type, int did,
        const acfd_partition_t *part, const acfd_node_t *node, const acfd_model_t *model,
        double Uo[6])
{
    double wsum = 0.0;
    memset(Uo, 0, 6 * sizeof(double));
    /* grow a symmetric box until at least one qualifying node is found */
    for (int r = h, tally = 0; 0 == tally; ++r) {
        for (int kh = -r; kh <= r; ++kh) {
            for (int jh = -r; jh <= r; ++jh) {
                for (int ih = -r; ih <= r; ++ih) {
                    const int i = c[0] + ih, j = c[1] + jh, k = c[2] + kh;
                    if (!in_pin(part, k, j, i)) {
                        continue;
                    }
                    const acfd_node_t *nd = &node[nidx(part, k, j, i)];
                    if (did != nd->did) {
                        continue;
                    }
                    if (TYPEF_ == type) {
                        if ((did != nd->gst) || (0 > nd->fid)) {
                            continue;
                        }
                    } else if (TYPED_ != type) {
                        if (type != nd->gst) {
                            continue;
                        }
                    }
                    ++tally;
                    double ph[3], Uoh[6];
                    node_point(part, k, j, i, ph);
                    to_primitive(model->gamma, model->gasR, nd->U[tn], Uoh);
                    add_weighted(Uoh, part->tinyL, dist2(p, ph), &wsum, Uo);
                }
            }
        }
        if (r > part->n[0] + part->n[1] + part->n[2]) {
            break; /* no qualifying node anywhere; the reference would loop forever */
        }
    }
    return wsum;
}

static void orthogonal_space(const double N[3], double Ta[3], double Tb[3])
{
    /* cfd_commons.c:431-458 */
    int mark = 2;
    if (fabs(N[mark]) > fabs(N[1])) {
        mark = 1;
    }
    if (fabs(N[mark]) > fabs(N[0])) {
        mark = 0;
    }
    if (0 == mark) {
        Ta[0] = 0.0; Ta[1] = -N[2]; Ta[2] = N[1];
    } else if (1 == mark) {
        Ta[0] = N[2]; Ta[1] = 0.0; Ta[2] = -N[0];
    } else {
        Ta[0] = -N[1]; Ta[1] = N[0]; Ta[2] = 0.0;
    }
    const double nrm = sqrt(dot3(Ta, Ta));
    for (int s = 0; s < 3; ++s) {
        Ta[s] = Ta[s] / nrm;
    }
    Tb[0] = Ta[1] * N[2] - Ta[2] * N[1];
    Tb[1] = Ta[2] * N[0] - Ta[0] * N[2];
    Tb[2] = Ta[0] * N[1] - Ta[1] * N[0];
}

static void reconstruct_flow(int tn, const int c[3], const double p[3], const acfd_polyhedron_t *P,
        const acfd_partition_t *part, const acfd_node_t *node, const acfd_model_t *model,
        const double pO[3], const double N[3], double UoO[6], double Uo[6])
{
    /* immersed_boundary.c:357-412 */
    double wsum = idw(tn, c, p, IB_R, TYPED_, 0, part, node, model, Uo);
    const double w = 1.0 / wsum;
    const double r[3] = {pO[0] - P->O[0], pO[1] - P->O[1], pO[2] - P->O[2]};
    double Vs[3];
    Vs[0] = P->W[1] * r[2] - P->W[2] * r[1];
    Vs[1] = P->W[2] * r[0] - P->W[0] * r[2];
    Vs[2] = P->W[0] * r[1] - P->W[1] * r[0];
    Vs[0] = P->V[0] + Vs[0];
    Vs[1] = P->V[1] + Vs[1];
    Vs[2] = P->V[2] + Vs[2];
    if (0.0 < P->cf) {
        UoO[1] = Vs[0];
        UoO[2] = Vs[1];
        UoO[3] = Vs[2];
    } else {
        const double V[3] = {Uo[1] * w, Uo[2] * w, Uo[3] * w};
        double Ta[3], Tb[3], rhs[3];
        orthogonal_space(N, Ta, Tb);
        rhs[0] = dot3(Vs, N);
        rhs[1] = dot3(V, Ta);
        rhs[2] = dot3(V, Tb);
        for (int s = 0; s < 3; ++s) {
            UoO[s + 1] = N[s] * rhs[0] + Ta[s] * rhs[1] + Tb[s] * rhs[2];
        }
    }
    UoO[4] = Uo[4] * w;
    UoO[5] = (0.0 > P->T) ? Uo[5] * w : P->T;
    add_weighted(UoO, part->tinyL, dist2(p, pO), &wsum, Uo);
    for (int n = 0; n < 6; ++n) {
        Uo[n] = Uo[n] / wsum;
    }
}

void orc_treat_ib(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    /* immersed_boundary.c:270-340: per body, ghost layers in order */
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t *P = poly + n;
        int box[3][2];
        body_box(part, P, box);
        for (int r = 1; r <= part->gl; ++r) {
            for (int k = box[2][0]; k < box[2][1]; ++k) {
                for (int j = box[1][0]; j < box[1][1]; ++j) {
                    for (int i = box[0][0]; i < box[0][1]; ++i) {
                        acfd_node_t *nd = &node[nidx(part, k, j, i)];
                        if ((r != nd->gst) || (n + 1 != nd->did)) {
                            continue;
                        }
                        double pG[3], UoG[6];
                        node_point(part, k, j, i, pG);
                        if (model->ibmLayer >= r) {
                            double pO[3], pI[3], N[3], UoO[6], UoI[6];
                            surface_data(pG, nd->fid, P, pO, pI, N);
                            int cI[3];
                            for (int s = 0; s < 3; ++s) {
                                cI[s] = map_node(pI[s], part->domain[s][0], part->dd[s], part->ng[s]);
                            }
                            reconstruct_flow(tn, cI, pI, P, part, node, model, pO, N, UoO, UoI);
                            UoG[1] = UoO[1] + UoO[1] - UoI[1];
                            UoG[2] = UoO[2] + UoO[2] - UoI[2];
                            UoG[3] = UoO[3] + UoO[3] - UoI[3];
                            UoG[4] = UoI[4];
                            UoG[5] = UoI[5];
                        } else {
                            const int cG[3] = {i, j, k};
                            const double ws = idw(tn, cG, pG, 1, r - 1, n + 1, part, node, model, UoG);
                            for (int q = 0; q < 6; ++q) {
                                UoG[q] = UoG[q] / ws;
                            }
                        }
                        UoG[0] = UoG[4] / (UoG[5] * model->gasR);
                        to_conservative(model->gamma, UoG, nd->U[tn]);
                    }
                }
            }
        }
    }
}

/* ------------------------------------------------------------------------
 * node mapping: immersed_boundary.c:65-264
 * ------------------------------------------------------------------------ */
static int layer_of(const acfd_partition_t *part, int n)
{
    for (int r = 1; r <= part->gl; ++r) {
        if (part->pathSep[r] > n) {
            return r;
        }
    }
    return 0;
}

void orc_compute_geometric_field(acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN)
{
    const int (*pin)[2] = part->ns[PIN_];
    /* 1. keep the old domain field in gst; release interfacial nodes of moving
     *    bodies (InitializeGeometricField :72-113) */
    for (int k = pin[2][0]; k < pin[2][1]; ++k) {
        for (int j = pin[1][0]; j < pin[1][1]; ++j) {
            for (int i = pin[0][0]; i < pin[0][1]; ++i) {
                acfd_node_t *nd = &node[nidx(part, k, j, i)];
                const int gid = nd->did;
                nd->gst = nd->did;
                if (0 == gid) {
                    nd->fid = 0;
                    continue;
                }
                if (1 == poly[gid - 1].state) {
                    continue;
                }
                if (0 < nd->lid) {
                    nd->did = 0;
                }
            }
        }
    }
    /* 2. map free nodes into bodies, first body wins (SetDomainField :128-182) */
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t *P = poly + n;
        if (1 == P->state) {
            continue;
        }
        int box[3][2];
        body_box(part, P, box);
        for (int k = box[2][0]; k < box[2][1]; ++k) {
            for (int j = box[1][0]; j < box[1][1]; ++j) {
                for (int i = box[0][0]; i < box[0][1]; ++i) {
                    acfd_node_t *nd = &node[nidx(part, k, j, i)];
                    if (0 != nd->did) {
                        continue;
                    }
                    double p[3];
                    node_point(part, k, j, i, p);
                    if (0 >= P->faceN) {
                        if (P->r * P->r >= dist2(P->O, p)) {
                            nd->did = n + 1;
                            nd->fid = 0;
                        }
                    } else {
                        int fid;
                        if (orc_point_in_polyhedron(p, P, &fid)) {
                            nd->did = n + 1;
                            nd->fid = fid;
                        }
                    }
                }
            }
        }
    }
    /* 3. interfacial and ghost layers; refill newly uncovered fluid nodes
     *    (SetInterfacialField :183-264) */
    for (int k = pin[2][0]; k < pin[2][1]; ++k) {
        for (int j = pin[1][0]; j < pin[1][1]; ++j) {
            for (int i = pin[0][0]; i < pin[0][1]; ++i) {
                acfd_node_t *nd = &node[nidx(part, k, j, i)];
                if ((nd->gst != nd->did) && (0 == nd->did)) {
                    const int c[3] = {i, j, k};
                    double p[3], Uo[6];
                    node_point(part, k, j, i, p);
                    const double ws = idw(ACFD_TO, c, p, IB_R, TYPEF_, nd->did, part, node, model, Uo);
                    for (int q = 0; q < 6; ++q) {
                        Uo[q] = Uo[q] / ws;
                    }
                    Uo[0] = Uo[4] / (Uo[5] * model->gasR);
                    to_conservative(model->gamma, Uo, nd->U[ACFD_TO]);
                    nd->fid = -1;
                }
                nd->lid = 0;
                nd->gst = 0;
                if (0 == nd->did) {
                    continue;
                }
                /* interfacial layer: first heterogeneous node on the path */
                for (int q = 0; q < part->pathSep[0]; ++q) {
                    const int kh = k + part->path[q][2], jh = j + part->path[q][1], ih = i + part->path[q][0];
                    if (!in_pin(part, kh, jh, ih)) {
                        continue;
                    }
                    if (nd->did != node[nidx(part, kh, jh, ih)].did) {
                        nd->lid = layer_of(part, q);
                        break;
                    }
                }
                if (0 < nd->lid) {
                    /* ghost layer: first fluid node on the path */
                    for (int q = 0; q < part->pathSep[0]; ++q) {
                        const int kh = k + part->path[q][2], jh = j + part->path[q][1], ih = i + part->path[q][0];
                        if (!in_pin(part, kh, jh, ih)) {
                            continue;
                        }
                        if (0 == node[nidx(part, kh, jh, ih)].did) {
                            nd->gst = layer_of(part, q);
                            break;
                        }
                    }
                }
            }
        }
    }
}

/* TransformPolyhedron (computational_geometry.c:162-208, with TransformVertex,
 * TransformNormal and TransformInertia :209-261): the surface of one body
 * moved about the reference point O (shift to O, scale, rotate about x, then
 * y, then z, offset, shift back), its normals rotated, its inertia tensor
 * restated on the rotated axes, its box rebuilt from FLT_MAX / FLT_MIN over
 * the vertices and then the centroid, vertex by vertex. */
static void orc_move_point(const double O[3], const double scale[3], const double R[3][3],
        const double offset[3], double p[3])
{
    double t[3];
    for (int s = 0; s < 3; ++s) {
        t[s] = p[s] - O[s];
    }
    for (int s = 0; s < 3; ++s) {
        t[s] = t[s] * scale[s];
    }
    for (int s = 0; s < 3; ++s) {
        p[s] = dot3(R[s], t);
    }
    for (int s = 0; s < 3; ++s) {
        p[s] = p[s] + offset[s] + O[s];
    }
}

static void orc_grow_box(double box[6], const double p[3])
{
    for (int s = 0; s < 3; ++s) {
        box[2 * s] = (box[2 * s] < p[s]) ? box[2 * s] : p[s];
        box[2 * s + 1] = (box[2 * s + 1] > p[s]) ? box[2 * s + 1] : p[s];
    }
}

void orc_transform_polyhedron(const double O[3], const double scale[3], const double angle[3],
        const double offset[3], int vertN, int faceN, int edgeN, double *v, double *Nf, double *Ne,
        double *Nv, double centroid[3], double inertia[9], double box[6])
{
    const double Sx = sin(angle[0]), Sy = sin(angle[1]), Sz = sin(angle[2]);
    const double Cx = cos(angle[0]), Cy = cos(angle[1]), Cz = cos(angle[2]);
    const double R[3][3] = {
        {Cy * Cz, -Cx * Sz + Sx * Sy * Cz, Sx * Sz + Cx * Sy * Cz},
        {Cy * Sz, Cx * Cz + Sx * Sy * Sz, -Sx * Cz + Cx * Sy * Sz},
        {-Sy, Sx * Cy, Cx * Cy}};
    const double Oref[3] = {O[0], O[1], O[2]};
    for (int s = 0; s < 3; ++s) {
        box[2 * s] = FLT_MAX;
        box[2 * s + 1] = FLT_MIN;
    }
    for (int n = 0; n < vertN; ++n) {
        orc_move_point(Oref, scale, R, offset, v + 3 * n);
        orc_grow_box(box, v + 3 * n);
    }
    double *normals[3] = {Nf, Ne, Nv};
    const int counts[3] = {faceN, edgeN, vertN};
    for (int a = 0; a < 3; ++a) {
        for (int n = 0; n < counts[a]; ++n) {
            double *N = normals[a] + 3 * n;
            const double t[3] = {N[0], N[1], N[2]};
            for (int s = 0; s < 3; ++s) {
                N[s] = dot3(R[s], t);
            }
        }
    }
    /* moments about the axes xx, yy, zz, xy, yz, zx of the rotated frame */
    const double h = 1.0 / sqrt(2.0);
    const double axes[6][3] = {{1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}, {0.0, 0.0, 1.0},
        {h, h, 0.0}, {0.0, h, h}, {h, 0.0, h}};
    double m[6];
    for (int q = 0; q < 6; ++q) {
        double a[3];
        for (int s = 0; s < 3; ++s) {
            const double col[3] = {R[0][s], R[1][s], R[2][s]};
            a[s] = dot3(col, axes[q]);
        }
        m[q] = inertia[0] * a[0] * a[0] + inertia[4] * a[1] * a[1] + inertia[8] * a[2] * a[2] +
            2.0 * inertia[1] * a[0] * a[1] + 2.0 * inertia[5] * a[1] * a[2] + 2.0 * inertia[6] * a[2] * a[0];
    }
    inertia[0] = m[0];
    inertia[1] = -m[3];
    inertia[2] = -m[5];
    inertia[3] = -m[3];
    inertia[4] = m[1];
    inertia[5] = -m[4];
    inertia[6] = -m[5];
    inertia[7] = -m[4];
    inertia[8] = m[2];
    orc_move_point(Oref, scale, R, offset, centroid);
    orc_grow_box(box, centroid);
}

/* IntegrateSurfaceForce (solid_dynamics.c:50-171): for every body with
 * state <= 0, the pressure force, shear force and torque summed over its
 * ghost nodes of layer 2 in node order (k, j, i), then scaled by -area over
 * its interfacial nodes of layer 2 (zero when the pressure samples are
 * uniform to FLT_EPSILON^2 of their mean).  force: totN x 9 (Fp, Fv, Tt);
 * rows of bodies with state > 0 are left as given.  The bodies' V and W are
 * their velocities at level TO. */
static void cross3(const double a[3], const double b[3], double c[3])
{
    /* cfd_commons.c:424-430 */
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

void orc_integrate_surface_force(const acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN, double *force)
{
    const double percent = (double)(FLT_EPSILON * FLT_EPSILON);
    for (int n = 0; n < totN; ++n) {
        const acfd_polyhedron_t *P = poly + n;
        if (0 < P->state) {
            continue;
        }
        double sumP[3] = {0.0, 0.0, 0.0}, sumV[3] = {0.0, 0.0, 0.0}, sumT[3] = {0.0, 0.0, 0.0};
        double first = 0.0, shift = 0.0, square = 0.0; /* pressure samples: first, sums of offsets */
        int lidN = 0, gstN = 0;
        int box[3][2];
        body_box(part, P, box);
        for (int k = box[2][0]; k < box[2][1]; ++k) {
            for (int j = box[1][0]; j < box[1][1]; ++j) {
                for (int i = box[0][0]; i < box[0][1]; ++i) {
                    const acfd_node_t *q = node + nidx(part, k, j, i);
                    if ((2 == q->lid) && (n + 1 == q->did)) {
                        ++lidN;
                    }
                    if ((2 != q->gst) || (n + 1 != q->did)) {
                        continue;
                    }
                    ++gstN;
                    double pG[3], pO[3], pI[3], N[3], Uo[6];
                    node_point(part, k, j, i, pG);
                    surface_data(pG, q->fid, P, pO, pI, N);
                    const double r[3] = {pO[0] - P->O[0], pO[1] - P->O[1], pO[2] - P->O[2]};
                    to_primitive(model->gamma, model->gasR, q->U[0], Uo);
                    const double Fp[3] = {Uo[4] * N[0], Uo[4] * N[1], Uo[4] * N[2]};
                    if (1 == gstN) {
                        first = Uo[4];
                    }
                    shift = shift + Uo[4] - first;
                    square = square + (Uo[4] - first) * (Uo[4] - first);
                    double Fv[3] = {0.0, 0.0, 0.0};
                    if ((0.0 < model->refMu) && (0.0 < P->cf)) {
                        const double T = Uo[5] * model->refT;
                        const double mu = model->refMu * (1.458e-6 * pow(T, 1.5) / (T + 110.4));
                        double V[3];
                        cross3(P->W, r, V);
                        for (int s = 0; s < 3; ++s) {
                            V[s] = Uo[1 + s] - (P->V[s] + V[s]);
                        }
                        const double Vn = dot3(V, N);
                        for (int s = 0; s < 3; ++s) {
                            Fv[s] = mu * (V[s] - Vn * N[s]) / sqrt(dist2(pG, pO));
                        }
                    }
                    const double Fs[3] = {Fp[0] + Fv[0], Fp[1] + Fv[1], Fp[2] + Fv[2]};
                    double Tt[3];
                    cross3(r, Fs, Tt);
                    for (int s = 0; s < 3; ++s) {
                        sumP[s] = sumP[s] + Fp[s];
                        sumV[s] = sumV[s] + Fv[s];
                        sumT[s] = sumT[s] + Tt[s];
                    }
                }
            }
        }
        double *out = force + 9 * (size_t)n;
        if ((0 == lidN) || (0 == gstN)) {
            /* the reference leaves the zeroed sums */
            for (int s = 0; s < 9; ++s) {
                out[s] = (s < 3) ? sumP[s] : ((s < 6) ? sumV[s - 3] : sumT[s - 6]);
            }
            continue;
        }
        double ds = P->area / lidN;
        const double variance = (square - shift * shift / gstN) / gstN;
        const double mean = shift / gstN + first;
        if (percent * mean * mean > variance) {
            ds = 0.0;
        }
        for (int s = 0; s < 3; ++s) {
            out[s] = -sumP[s] * ds;
            out[3 + s] = -sumV[s] * ds;
            out[6 + s] = -sumT[s] * ds;
        }
    }
}

/* The contact list ApplyCollision builds for body p (the node scan of
 * solid_dynamics.c:242-256 with DetectColState / AddColObject :327-379):
 * every interfacial node of layer 1 of body p, in node order, looks along
 * the first pathSep[1] steps of the search path; a node of another body met
 * on the way adds that body to the list (in the order first met) or adds the
 * step to its line of impact.  Returns the list length; gid[c] (body ids,
 * 1 = first body) and N[3c..3c+2] receive the entries.  A stationary body
 * (state 1) has no list. */
int orc_collision_scan(const acfd_node_t *node, const acfd_partition_t *part, const acfd_polyhedron_t *poly,
        int totN, int p, int *gid, int *N)
{
    if ((p < 0) || (p >= totN) || (1 == poly[p].state)) {
        return 0;
    }
    int count = 0;
    int box[3][2];
    body_box(part, poly + p, box);
    for (int k = box[2][0]; k < box[2][1]; ++k) {
        for (int j = box[1][0]; j < box[1][1]; ++j) {
            for (int i = box[0][0]; i < box[0][1]; ++i) {
                const acfd_node_t *q = node + nidx(part, k, j, i);
                if ((1 != q->lid) || (p + 1 != q->did)) {
                    continue;
                }
                for (int m = 0; m < part->pathSep[1]; ++m) {
                    const int *step = part->path[m];
                    const int kh = k + step[2], jh = j + step[1], ih = i + step[0];
                    if (!in_pin(part, kh, jh, ih)) {
                        continue;
                    }
                    const int did = node[nidx(part, kh, jh, ih)].did;
                    if ((0 == did) || (p + 1 == did)) {
                        continue;
                    }
                    int c = 0;
                    while ((c < count) && (gid[c] != did)) {
                        ++c;
                    }
                    if (c == count) {
                        gid[c] = did;
                        N[3 * c] = N[3 * c + 1] = N[3 * c + 2] = 0;
                        ++count;
                    }
                    for (int s = 0; s < 3; ++s) {
                        N[3 * c + s] = N[3 * c + s] + step[s];
                    }
                }
            }
        }
    }
    return count;
}

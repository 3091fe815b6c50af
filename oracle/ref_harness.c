/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY.
 *
 * Thin driver around the UNMODIFIED ArtraCFD sources, compiled from the
 * reference tree by oracle/Makefile into oracle/_ref/libacfd_ref.so.  It
 * exposes the reference's own functions (including the static ones of
 * solve.c and solid_dynamics.c, reached by including those files) with the plain types of
 * include/acfd.h so that tests can run the reference on exactly the inputs
 * given to the oracle restatement and to the GPU library.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include "solve.c" /* EvolveSolution / ComputeTimeStep are static there */
#include "solid_dynamics.c" /* DetectColState (the contact search) is static there */

#include "preprocess.h"
#include "postprocess.h"
#include "boundary_treatment.h"
#include "immersed_boundary.h"
#include "convective_flux.h"
#include "diffusive_flux.h"
#include "weno.h"
#include "computational_geometry.h"

#include "acfd.h"

static Time g_time;
static Space g_space;
static Model g_model;
static int g_loaded = 0;

/* Load a case directory (artracfd.case/.geo) exactly as the program does:
 * Preprocess then InitializeComputeDomain (writes initial output files into
 * the case directory). */
int ref_load(const char *case_dir)
{
    if (g_loaded) {
        Postprocess(&g_time, &g_space, &g_model);
        g_loaded = 0;
    }
    if (0 != chdir(case_dir)) {
        return 1;
    }
    memset(&g_time, 0, sizeof(g_time));
    memset(&g_space, 0, sizeof(g_space));
    memset(&g_model, 0, sizeof(g_model));
    g_space.part.proc[X] = 1;
    g_space.part.proc[Y] = 1;
    g_space.part.proc[Z] = 1;
    g_space.part.procN = 1;
    Preprocess(&g_time, &g_space, &g_model);
    InitializeComputeDomain(&g_time, &g_space, &g_model);
    g_loaded = 1;
    return 0;
}

void ref_get_partition(acfd_partition_t *out)
{
    const Partition *p = &g_space.part;
    memset(out, 0, sizeof(*out));
    for (int s = 0; s < 3; ++s) {
        out->m[s] = p->m[s];
        out->n[s] = p->n[s];
        out->ng[s] = p->ng[s];
        out->d[s] = p->d[s];
        out->dd[s] = p->dd[s];
        out->domain[s][0] = p->domain[s][0];
        out->domain[s][1] = p->domain[s][1];
    }
    out->gl = p->gl;
    out->collapse = p->collapse;
    out->tinyL = p->tinyL;
    memcpy(out->ns, p->ns, sizeof(out->ns));
    memcpy(out->np, p->np, sizeof(out->np));
    memcpy(out->path, p->path, sizeof(out->path));
    memcpy(out->pathSep, p->pathSep, sizeof(out->pathSep));
    for (int q = 0; q < NBC; ++q) {
        out->typeBC[q] = p->typeBC[q];
        for (int s = 0; s < 3; ++s) {
            out->N[q][s] = p->N[q][s];
        }
        for (int v = 0; v < VARBC; ++v) {
            out->varBC[q][v] = p->varBC[q][v];
        }
    }
}

void ref_get_model(acfd_model_t *out)
{
    const Model *m = &g_model;
    memset(out, 0, sizeof(*out));
    out->tScheme = m->tScheme;
    out->sScheme = m->sScheme;
    out->sL = m->sL;
    out->sR = m->sR;
    out->multidim = m->multidim;
    out->jacobMean = m->jacobMean;
    out->fluxSplit = m->fluxSplit;
    out->psi = m->psi;
    out->ibmLayer = m->ibmLayer;
    out->gState = m->gState;
    out->sState = m->sState;
    out->refMa = m->refMa;
    out->refMu = m->refMu;
    out->gamma = m->gamma;
    out->gasR = m->gasR;
    out->cv = m->cv;
    out->refL = m->refL;
    out->refRho = m->refRho;
    out->refV = m->refV;
    out->refT = m->refT;
    for (int s = 0; s < 3; ++s) {
        out->g[s] = m->g[s];
    }
}

void ref_get_time(double *end, double *now, double *numCFL, int *stepN, int *stepC)
{
    *end = g_time.end;
    *now = g_time.now;
    *numCFL = g_time.numCFL;
    *stepN = g_time.stepN;
    *stepC = g_time.stepC;
}

void ref_set_numerics(int tScheme, int sScheme, int jacobMean, int fluxSplit)
{
    /* switch schemes of an already loaded case with the same stencil width */
    g_model.tScheme = tScheme;
    g_model.sScheme = sScheme;
    g_model.jacobMean = jacobMean;
    g_model.fluxSplit = fluxSplit;
}

int ref_node_count(void)
{
    return g_space.part.n[X] * g_space.part.n[Y] * g_space.part.n[Z];
}

void ref_get_nodes(acfd_node_t *out)
{
    memcpy(out, g_space.node, (size_t)ref_node_count() * sizeof(Node));
}

void ref_set_nodes(const acfd_node_t *in)
{
    memcpy(g_space.node, in, (size_t)ref_node_count() * sizeof(Node));
}

int ref_geo_count(void)
{
    return g_space.geo.totN;
}

/* Describe body n with pointers into the reference's own arrays. */
void ref_get_poly(int n, acfd_polyhedron_t *out)
{
    const Polyhedron *P = g_space.geo.poly + n;
    memset(out, 0, sizeof(*out));
    out->faceN = P->faceN;
    out->edgeN = P->edgeN;
    out->vertN = P->vertN;
    out->state = P->state;
    out->r = P->r;
    out->T = P->T;
    out->cf = P->cf;
    for (int s = 0; s < 3; ++s) {
        out->O[s] = P->O[s];
        out->V[s] = P->V[TO][s];
        out->W[s] = P->W[TO][s];
        out->box[s][0] = P->box[s][0];
        out->box[s][1] = P->box[s][1];
    }
    out->f = (const int *)P->f;
    out->Nf = (const double *)P->Nf;
    out->e = (const int *)P->e;
    out->Ne = (const double *)P->Ne;
    out->v = (const double *)P->v;
    out->Nv = (const double *)P->Nv;
    out->area = P->area;
}

double ref_compute_time_step(void)
{
    return ComputeTimeStep(&g_time, &g_space, &g_model);
}

void ref_evolve_fluid(double dt)
{
    EvolveFluidDynamics(dt, &g_space, &g_model);
}

void ref_treat_boundary(int tn)
{
    TreatBoundary(tn, &g_space, &g_model);
}

void ref_compute_geometric_field(void)
{
    ComputeGeometricField(&g_space, &g_model);
}

void ref_treat_ib(int tn)
{
    TreatImmersedBoundary(tn, &g_space, &g_model);
}

void ref_evolve_solid(double now, double dt)
{
    EvolveSolidDynamics(now, dt, &g_space, &g_model);
}

/* IntegrateSurfaceForce (solid_dynamics.c:51-171) on the loaded state;
 * out: totN x 9 (Fp, Fv, Tt) as the bodies hold them afterwards. */
void ref_integrate_surface_force(double *out)
{
    IntegrateSurfaceForce(&g_space, &g_model);
    for (int n = 0; n < g_space.geo.totN; ++n) {
        const Polyhedron *P = g_space.geo.poly + n;
        for (int s = 0; s < 3; ++s) {
            out[9 * n + s] = P->Fp[s];
            out[9 * n + 3 + s] = P->Fv[s];
            out[9 * n + 6 + s] = P->Tt[s];
        }
    }
}

/* the reference's EigenvectorL / EigenvectorR (cfd_commons.c:149-246) */
void ref_eigenvectors(int s, double gamma, const double Uo[6], double L[25], double R[25])
{
    EigenvectorL(s, gamma, Uo, (Real (*)[DIMU])L);
    EigenvectorR(s, Uo, (Real (*)[DIMU])R);
}

/* TransformPolyhedron (computational_geometry.c:162-208) of body n, the
 * reference point O given apart from the body's centroid (ApplyMotion passes
 * the centroid itself). */
void ref_transform_polyhedron(int n, const double O[3], const double scale[3], const double angle[3],
        const double offset[3])
{
    const RealVec Oc = {O[0], O[1], O[2]};
    TransformPolyhedron(Oc, scale, angle, offset, g_space.geo.poly + n);
}

/* the inertia tensor of body n, row-major */
void ref_get_inertia(int n, double out[9])
{
    memcpy(out, g_space.geo.poly[n].I, 9 * sizeof(double));
}

/* The contact list that ApplyCollision builds for body p before its
 * velocity update (the node scan of solid_dynamics.c:242-256, calling the
 * reference's DetectColState); returns the list length, gid/N receive the
 * entries.  Stationary bodies have no list. */
int ref_collision_scan(int p, int *gid, int *N)
{
    Space *space = &g_space;
    const Partition *part = &space->part;
    Geometry *geo = &space->geo;
    const Polyhedron *P = geo->poly + p;
    if (1 == P->state) {
        return 0;
    }
    geo->colN = 0;
    int box[DIMS][LIMIT];
    for (int s = 0; s < DIMS; ++s) {
        box[s][MIN] = ConfineSpace(MapNode(P->box[s][MIN], part->domain[s][MIN], part->dd[s], part->ng[s]),
                part->ns[PIN][s][MIN], part->ns[PIN][s][MAX]);
        box[s][MAX] = ConfineSpace(MapNode(P->box[s][MAX], part->domain[s][MIN], part->dd[s], part->ng[s]),
                part->ns[PIN][s][MIN], part->ns[PIN][s][MAX]) + 1;
    }
    for (int k = box[Z][MIN]; k < box[Z][MAX]; ++k) {
        for (int j = box[Y][MIN]; j < box[Y][MAX]; ++j) {
            for (int i = box[X][MIN]; i < box[X][MAX]; ++i) {
                const int idx = IndexNode(k, j, i, part->n[Y], part->n[X]);
                if ((1 != space->node[idx].lid) || (p + 1 != space->node[idx].did)) {
                    continue;
                }
                DetectColState(k, j, i, p + 1, part->pathSep[1], part->path, space->node, part, geo);
            }
        }
    }
    for (int c = 0; c < geo->colN; ++c) {
        gid[c] = geo->col[c].gid;
        for (int s = 0; s < DIMS; ++s) {
            N[3 * c + s] = geo->col[c].N[s];
        }
    }
    const int count = geo->colN;
    geo->colN = 0;
    return count;
}

/* One pass of the loop body of EvolveSolution (solve.c:65-89) without output:
 * time step, dt rectification against the end time, solid/fluid/solid.
 * Returns the dt used, or a negative value when the run has ended. */
double ref_step(void)
{
    if (!((g_time.now < g_time.end) && (g_time.stepC < g_time.stepN))) {
        return -1.0;
    }
    ++(g_time.stepC);
    Real dt = ComputeTimeStep(&g_time, &g_space, &g_model);
    g_time.now = g_time.now + dt;
    if (g_time.now > g_time.end) {
        dt = g_time.end - (g_time.now - dt);
        g_time.now = g_time.end;
    }
    if (0 != g_model.psi) {
        EvolveSolidDynamics(g_time.now, 0.5 * dt, &g_space, &g_model);
    }
    EvolveFluidDynamics(dt, &g_space, &g_model);
    if (0 != g_model.psi) {
        EvolveSolidDynamics(g_time.now, 0.5 * dt, &g_space, &g_model);
    }
    return dt;
}

/* per-point functions on caller data */
void ref_weno5(const double F[5][5], double out[5])
{
    double tmp[5][5];
    memcpy(tmp, F, sizeof(tmp));
    WENO5(tmp, out);
}

void ref_weno3(const double F[3][5], double out[5])
{
    double tmp[5][5];
    memcpy(tmp, F, 3 * 5 * sizeof(double));
    WENO3(tmp, out);
}

void ref_compute_fhat(int tn, int s, int k, int j, int i, double out[5])
{
    ComputeFhat(tn, s, k, j, i, g_space.part.n, g_space.node, &g_model, out);
}

void ref_compute_fvhat(int tn, int s, int k, int j, int i, double out[5])
{
    ComputeFvhat(tn, s, k, j, i, g_space.part.n, g_space.part.dd, g_space.node, &g_model, out);
}

int ref_point_in_polyhedron(int n, const double p[3], int *fid)
{
    return PointInPolyhedron(p, g_space.geo.poly + n, fid);
}

void ref_close(void)
{
    if (g_loaded) {
        Postprocess(&g_time, &g_space, &g_model);
        g_loaded = 0;
    }
}

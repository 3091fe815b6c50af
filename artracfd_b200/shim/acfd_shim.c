/*
 * acfd_shim.c -- the reference-side drop-in for libacfd_gpu.
 *
 * Linked into the reference program together with the reference's own
 * sources, of which three functions are renamed at compile time (see the
 * Makefile): Solve -> RefSolve (solve.c:38), EvolveFluidDynamics ->
 * RefEvolveFluidDynamics (fluid_dynamics.c:55), TreatBoundary ->
 * RefTreatBoundary (boundary_treatment.c:28).  This file defines the three
 * names again with the reference signatures.  In GPU mode (`-m gpu`, see
 * main.c in this directory) they run on the B200 through the C ABI; in every
 * other mode they call the reference functions unchanged.
 *
 * GPU mode keeps the node array coherent at exactly the places where host
 * code reads or writes it: before output (solve.c:91-104), and around the
 * rigid-body step (solid_dynamics.c:38-49) only when that step runs on the
 * host (ACFD_SOLID=host); by default its node scans run on the device
 * (solid_gpu.c).
 *
 * Environment: ACFD_MODE = fp64 (default) | exact | fp32, ACFD_GRAPH = 1
 * (default, replay each step as a CUDA graph) | 0, ACFD_SOLID = device
 * (default) | host.
 */
#include "acfd_shim.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>

#include "commons.h"
#include "cfd_commons.h"
#include "boundary_treatment.h"
#include "fluid_dynamics.h"
#include "initialization.h"
#include "solid_dynamics.h"
#include "data_stream.h"
#include "solve.h"
#include "timer.h"

#include "acfd.h"

int g_acfd_gpu_mode = 0;

static acfd_case_t *g_case = NULL;
static int g_host_current = 1;   /* host node array holds the latest state */
static int g_dev_current = 0;    /* device holds the latest state */
static int g_use_graph = 1;
static int g_solid_host = 0;   /* ACFD_SOLID=host: rigid-body step on the host */

static void Check(int status, const char *what)
{
    if (ACFD_OK != status) {
        char msg[1024];
        acfd_last_error(msg, sizeof(msg));
        ShowError("%s failed (%d): %s", what, status, msg);
    }
}

static void ToPartition(const Partition *p, acfd_partition_t *o)
{
    memset(o, 0, sizeof(*o));
    for (int s = 0; s < DIMS; ++s) {
        o->m[s] = p->m[s];
        o->n[s] = p->n[s];
        o->ng[s] = p->ng[s];
        o->d[s] = p->d[s];
        o->dd[s] = p->dd[s];
        o->domain[s][0] = p->domain[s][MIN];
        o->domain[s][1] = p->domain[s][MAX];
    }
    o->gl = p->gl;
    o->collapse = p->collapse;
    o->tinyL = p->tinyL;
    memcpy(o->ns, p->ns, sizeof(o->ns));
    memcpy(o->np, p->np, sizeof(o->np));
    memcpy(o->path, p->path, sizeof(o->path));
    memcpy(o->pathSep, p->pathSep, sizeof(o->pathSep));
    for (int q = 0; q < NBC; ++q) {
        o->typeBC[q] = p->typeBC[q];
        for (int s = 0; s < DIMS; ++s) {
            o->N[q][s] = p->N[q][s];
        }
        for (int v = 0; v < VARBC; ++v) {
            o->varBC[q][v] = p->varBC[q][v];
        }
    }
}

static void ToModel(const Model *m, acfd_model_t *o)
{
    memset(o, 0, sizeof(*o));
    o->tScheme = m->tScheme;
    o->sScheme = m->sScheme;
    o->sL = m->sL;
    o->sR = m->sR;
    o->multidim = m->multidim;
    o->jacobMean = m->jacobMean;
    o->fluxSplit = m->fluxSplit;
    o->psi = m->psi;
    o->ibmLayer = m->ibmLayer;
    o->gState = m->gState;
    o->sState = m->sState;
    o->refMa = m->refMa;
    o->refMu = m->refMu;
    o->gamma = m->gamma;
    o->gasR = m->gasR;
    o->cv = m->cv;
    o->refL = m->refL;
    o->refRho = m->refRho;
    o->refV = m->refV;
    o->refT = m->refT;
    for (int s = 0; s < DIMS; ++s) {
        o->g[s] = m->g[s];
    }
}

/* bodies as they are now on the host (after ApplyMotion) */
void AcfdUploadGeometry(const Space *space)
{
    const Geometry *geo = &(space->geo);
    if (0 >= geo->totN) {
        return;
    }
    acfd_polyhedron_t *list = AssignStorage(geo->totN * sizeof(*list));
    for (int n = 0; n < geo->totN; ++n) {
        const Polyhedron *P = geo->poly + n;
        acfd_polyhedron_t *o = list + n;
        o->faceN = P->faceN;
        o->edgeN = P->edgeN;
        o->vertN = P->vertN;
        o->state = P->state;
        o->r = P->r;
        o->T = P->T;
        o->cf = P->cf;
        for (int s = 0; s < DIMS; ++s) {
            o->O[s] = P->O[s];
            o->V[s] = P->V[TO][s];
            o->W[s] = P->W[TO][s];
            o->box[s][0] = P->box[s][MIN];
            o->box[s][1] = P->box[s][MAX];
        }
        o->f = (const int *)P->f;
        o->Nf = (const double *)P->Nf;
        o->e = (const int *)P->e;
        o->Ne = (const double *)P->Ne;
        o->v = (const double *)P->v;
        o->Nv = (const double *)P->Nv;
        o->area = P->area;
    }
    Check(acfd_geo_upload(g_case, list, geo->totN), "acfd_geo_upload");
    RetrieveStorage(list);
}

static void EnsureCase(Space *space, const Model *model)
{
    if (NULL != g_case) {
        return;
    }
    acfd_partition_t part;
    acfd_model_t mod;
    ToPartition(&(space->part), &part);
    ToModel(model, &mod);
    Check(acfd_init(&part, &mod, &g_case), "acfd_init");
    int mode = ACFD_FP64;
    const char *env = getenv("ACFD_MODE");
    if (env && 0 == strcmp(env, "exact")) {
        mode = ACFD_FP64_EXACT;
    } else if (env && 0 == strcmp(env, "fp32")) {
        mode = ACFD_FP32_BULK;
    }
    Check(acfd_set_precision(g_case, mode), "acfd_set_precision");
    env = getenv("ACFD_GRAPH");
    g_use_graph = !(env && 0 == strcmp(env, "0"));
    env = getenv("ACFD_SOLID");
    g_solid_host = (env && 0 == strcmp(env, "host"));
    AcfdUploadGeometry(space);
    g_dev_current = 0;
    g_host_current = 1;
}

static void EnsureDevice(Space *space)
{
    if (!g_dev_current) {
        Check(acfd_sync_to_device(g_case, (const acfd_node_t *)space->node, ACFD_SYNC_ALL), "acfd_sync_to_device");
        g_dev_current = 1;
    }
}

static void EnsureHost(Space *space)
{
    if (!g_host_current) {
        Check(acfd_sync_to_host(g_case, (acfd_node_t *)space->node, ACFD_SYNC_ALL), "acfd_sync_to_host");
        g_host_current = 1;
    }
}

void AcfdShimFinalize(void)
{
    if (NULL != g_case) {
        acfd_finalize(g_case);
        g_case = NULL;
    }
}

/* TreatBoundary (boundary_treatment.c:28) */
void TreatBoundary(const int tn, Space *space, const Model *model)
{
    if (!g_acfd_gpu_mode) {
        RefTreatBoundary(tn, space, model);
        return;
    }
    EnsureCase(space, model);
    EnsureHost(space);        /* the caller may have changed host data */
    g_dev_current = 0;
    EnsureDevice(space);
    Check(acfd_treat_boundary(g_case, tn), "acfd_treat_boundary");
    g_host_current = 0;
    EnsureHost(space);
}

/* EvolveFluidDynamics (fluid_dynamics.c:55) */
void EvolveFluidDynamics(const Real dt, Space *space, const Model *model)
{
    if (!g_acfd_gpu_mode) {
        RefEvolveFluidDynamics(dt, space, model);
        return;
    }
    EnsureCase(space, model);
    EnsureDevice(space);
    if (g_use_graph) {
        Check(acfd_evolve_fluid_graph(g_case, dt), "acfd_evolve_fluid_graph");
    } else {
        Check(acfd_evolve_fluid(g_case, dt), "acfd_evolve_fluid");
    }
    g_host_current = 0;
}

/* ComputeTimeStep (solve.c:108-153): body speeds on the host, the fluid
 * maximum on the device */
static Real GpuTimeStep(const Time *time, const Space *space)
{
    const Partition *part = &(space->part);
    const Geometry *geo = &(space->geo);
    RealVec V = {0.0};
    RealVec Vmax = {0.0};
    for (int n = 0; n < geo->totN; ++n) {
        const Polyhedron *poly = geo->poly + n;
        V[X] = fabs(poly->V[TO][X]) + MaxReal(fabs(poly->W[TO][Y]), fabs(poly->W[TO][Z])) * poly->r;
        V[Y] = fabs(poly->V[TO][Y]) + MaxReal(fabs(poly->W[TO][Z]), fabs(poly->W[TO][X])) * poly->r;
        V[Z] = fabs(poly->V[TO][Z]) + MaxReal(fabs(poly->W[TO][X]), fabs(poly->W[TO][Y])) * poly->r;
        for (int s = 0; s < DIMS; ++s) {
            if (Vmax[s] < V[s]) {
                Vmax[s] = V[s];
            }
        }
    }
    double vf[3];
    Check(acfd_cfl(g_case, vf), "acfd_cfl");
    for (int s = 0; s < DIMS; ++s) {
        if (Vmax[s] < vf[s]) {
            Vmax[s] = vf[s];
        }
    }
    return time->numCFL * MinReal(part->d[X] / Vmax[X], MinReal(part->d[Y] / Vmax[Y], part->d[Z] / Vmax[Z]));
}

/* the rigid-body half step: by default with its node scans on the device
 * (solid_gpu.c), the node array staying there; ACFD_SOLID=host runs the
 * reference's EvolveSolidDynamics on the host instead, with the node array
 * brought to the host and the remapped nodes and moved bodies sent back */
static void GpuSolidStep(const Real now, const Real dt, Space *space, const Model *model)
{
    if (!g_solid_host) {
        EnsureDevice(space);
        AcfdDeviceSolidStep(g_case, now, dt, space, model);
        g_host_current = 0;
        return;
    }
    EnsureHost(space);
    EvolveSolidDynamics(now, dt, space, model);
    g_dev_current = 0;
    EnsureDevice(space);
    AcfdUploadGeometry(space);
}

/* EvolveSolution (solve.c:48-107) with the fluid step on the device */
static void GpuEvolveSolution(Time *time, Space *space, const Model *model)
{
    Real dt = time->end - time->now;
    const Real zero = 0.0;
    if (zero >= dt) {
        ShowWarning("  time.now >= time.end");
        return;
    }
    Timer tm;
    const Real dtData[NPROBE] = {time->end / (Real)(time->dataW[PROPT]),
        time->end / (Real)(time->dataW[PROLN]), time->end / (Real)(time->dataW[PROCV]),
        time->end / (Real)(time->dataW[PROFC]), time->end / (Real)(time->dataW[PROSD])};
    Real rcData[NPROBE] = {zero};
    const Real tmInt = (INT_MAX == time->dataW[PROSD]) ? time->end : dtData[PROSD];
    Real rcInt = zero;
    EnsureCase(space, model);
    EnsureDevice(space);
    while ((time->now < time->end) && (time->stepC < time->stepN)) {
        ++(time->stepC);
        dt = GpuTimeStep(time, space);
        if (rcInt + dt > tmInt) {
            dt = tmInt - rcInt;
            rcInt = zero;
        } else {
            rcInt = rcInt + dt;
        }
        time->now = time->now + dt;
        if (time->now > time->end) {
            dt = time->end - (time->now - dt);
            time->now = time->end;
        }
        ShowInfo("\nstep=%d; time=%.6g; remain=%.6g; dt=%.6g;\n",
                time->stepC, time->now, time->end - time->now, dt);
        TickTime(&tm);
        if (0 != model->psi) {
            GpuSolidStep(time->now, 0.5 * dt, space, model);
        }
        EvolveFluidDynamics(dt, space, model);
        if (0 != model->psi) {
            GpuSolidStep(time->now, 0.5 * dt, space, model);
        }
        Check(acfd_synchronize(g_case), "acfd_synchronize");
        ShowInfo("  elapsed: %.6gs\n", TockTime(&tm));
        for (int n = 0; n < NPROBE; ++n) {
            rcData[n] = rcData[n] + dt;
            if ((rcData[n] >= dtData[n]) || (time->now == time->end) || (time->stepC == time->stepN)) {
                EnsureHost(space);
                if (PROFC == n) {
                    IntegrateSurfaceForce(space, model);
                }
                if (PROSD == n) {
                    ShowInfo("  writing data...\n");
                    ++(time->dataC);
                }
                WriteData(n, time, space, model);
                rcData[n] = zero;
            }
        }
    }
    EnsureHost(space);
}

/* Solve (solve.c:38-47) */
int Solve(Time *time, Space *space, const Model *model)
{
    if (!g_acfd_gpu_mode) {
        return RefSolve(time, space, model);
    }
    ShowInfo("Solving (B200, libacfd_gpu)...\n");
    ShowInfo("  initializing...\n");
    InitializeComputeDomain(time, space, model);
    ShowInfo("  time marching...\n");
    GpuEvolveSolution(time, space, model);
    ShowInfo("Session");
    return 0;
}

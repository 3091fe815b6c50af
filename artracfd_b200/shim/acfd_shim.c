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
 * Environment: ACFD_MODE = fp64 (default) | exact | fp32 | hybrid (the
 * learned-sensor form; ACFD_SENSOR = weights file, default the shipped
 * sensor_weights.bin), ACFD_TILES = stage-kernel variants per axis (e.g.
 * 7,7,7), ACFD_AUTOTUNE = 1 (time the variants at the first step), ACFD_GRAPH = 1
 * (default, replay each step as a CUDA graph) | 0, ACFD_SOLID = device
 * (default) | host, ACFD_MOTION = device (default: the surfaces of moving
 * triangulated bodies are transformed on the device and come back to the
 * host only for output) | host (the reference's ApplyMotion on the host;
 * with ACFD_SOLID=device), ACFD_ASYNC_OUTPUT = 1 (default: the outputs of a step
 * come from a device snapshot and are written while the next step runs, when
 * no body moves) | 0, ACFD_CHECKPOINT = 0 (default) | 1 (an FP64 checkpoint
 * artracfd.ckpt.<n> with every space data output; a restart from output n
 * uses it when it exists).
 */
#define _POSIX_C_SOURCE 200809L /* readlink */
#include "acfd_shim.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <limits.h>
#include <unistd.h>

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
static int g_async_output = 1; /* ACFD_ASYNC_OUTPUT=0: output from a synchronous download */
static int g_checkpoint = 0;   /* ACFD_CHECKPOINT=1: FP64 checkpoint with every space data output */
static int g_autotune = 0;     /* ACFD_AUTOTUNE=1: time the stage-kernel variants at the first step */
static int g_motion_host = 0;  /* ACFD_MOTION=host: surfaces moved on the host */
static unsigned char *g_surface_on_device = NULL; /* per body: the host's surface is older */

/* outputs of one step written from a device snapshot while the next step runs */
typedef struct {
    int pending;
    int count;
    int which[NPROBE];
    Time time;
} PendingOutput;
static PendingOutput g_out;

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
        o->area = P->area;
        if (g_surface_on_device && g_surface_on_device[n]) {
            continue; /* NULL arrays: the device keeps the moved surface */
        }
        o->f = (const int *)P->f;
        o->Nf = (const double *)P->Nf;
        o->e = (const int *)P->e;
        o->Ne = (const double *)P->Ne;
        o->v = (const double *)P->v;
        o->Nv = (const double *)P->Nv;
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
    } else if (env && 0 == strcmp(env, "hybrid")) {
        mode = ACFD_FP32_HYBRID;
        /* the trained sensor: ACFD_SENSOR, else the weights shipped beside
         * the library (artracfd_b200/sensor_weights.bin) */
        char path[4096] = {0};
        const char *given = getenv("ACFD_SENSOR");
        if (given) {
            snprintf(path, sizeof(path), "%s", given);
        } else {
            char exe[4096] = {0};
            const ssize_t len = readlink("/proc/self/exe", exe, sizeof(exe) - 1);
            char *slash = (len > 0) ? strrchr(exe, '/') : NULL;
            if (NULL == slash) {
                ShowError("ACFD_MODE=hybrid: set ACFD_SENSOR to the sensor weights file");
            }
            *slash = '\0';
            snprintf(path, sizeof(path), "%s/../../sensor_weights.bin", exe);
        }
        Check(acfd_sensor_load_file(g_case, path), "acfd_sensor_load_file");
    }
    Check(acfd_set_precision(g_case, mode), "acfd_set_precision");
    env = getenv("ACFD_TILES");
    if (env) {
        int tiles[3];
        if (3 != sscanf(env, "%d,%d,%d", tiles, tiles + 1, tiles + 2)) {
            ShowError("ACFD_TILES: three variants, e.g. 7,7,7");
        }
        Check(acfd_set_tiles(g_case, tiles), "acfd_set_tiles");
    }
    env = getenv("ACFD_AUTOTUNE");
    g_autotune = (env && 0 == strcmp(env, "1"));
    env = getenv("ACFD_GRAPH");
    g_use_graph = !(env && 0 == strcmp(env, "0"));
    env = getenv("ACFD_SOLID");
    g_solid_host = (env && 0 == strcmp(env, "host"));
    env = getenv("ACFD_MOTION");
    g_motion_host = (env && 0 == strcmp(env, "host"));
    if (0 < space->geo.totN) {
        g_surface_on_device = calloc((size_t)space->geo.totN, 1);
        if (NULL == g_surface_on_device) {
            ShowError("out of memory");
        }
    }
    env = getenv("ACFD_ASYNC_OUTPUT");
    g_async_output = !(env && 0 == strcmp(env, "0"));
    env = getenv("ACFD_CHECKPOINT");
    g_checkpoint = (env && 0 == strcmp(env, "1"));
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

int AcfdMotionOnDevice(void)
{
    return !g_motion_host;
}

void AcfdMarkSurfaceOnDevice(int n)
{
    g_surface_on_device[n] = 1;
}

/* the surfaces moved on the device back into the host's polyhedra */
static void FetchSurfaces(Space *space)
{
    Geometry *geo = &(space->geo);
    for (int n = 0; g_surface_on_device && n < geo->totN; ++n) {
        if (!g_surface_on_device[n]) {
            continue;
        }
        Polyhedron *P = geo->poly + n;
        Check(acfd_geo_fetch(g_case, n, &P->v[0][0], &P->Nf[0][0], &P->Ne[0][0], &P->Nv[0][0]), "acfd_geo_fetch");
        g_surface_on_device[n] = 0;
    }
}

static void EnsureHost(Space *space)
{
    FetchSurfaces(space);
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
    free(g_surface_on_device);
    g_surface_on_device = NULL;
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
    if (g_autotune) {
        int tiles[3];
        Check(acfd_autotune(g_case, tiles), "acfd_autotune");
        ShowInfo("  stage kernels (autotuned): %d %d %d\n", tiles[0], tiles[1], tiles[2]);
        g_autotune = 0;
    }
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

/* ---- FP64 checkpoints ----------------------------------------------------
 * artracfd.ckpt.<dataC> beside the data files of the same output: the node
 * records of the device state (libacfd_gpu writes them) and, as the caller's
 * block, the time and every body's motion state and transformed surface, so
 * that a restart from output dataC continues bit for bit (the reference
 * restarts from its float32 / %.6g files, ReadData, data_stream.c:71-90). */
#define CKPT_BODY_REALS 64

static void CheckpointName(int dataC, char *name, size_t len)
{
    snprintf(name, len, "artracfd.ckpt.%05d", dataC);
}

static size_t CheckpointUserBytes(const Geometry *geo)
{
    size_t bytes = 3 * sizeof(double) + sizeof(int) * (1 + geo->totN);
    for (int n = 0; n < geo->totN; ++n) {
        const Polyhedron *P = geo->poly + n;
        bytes += CKPT_BODY_REALS * sizeof(double);
        if (0 < P->faceN) {
            bytes += 3 * sizeof(double) * (size_t)(2 * P->vertN + P->faceN + P->edgeN);
        }
    }
    return bytes;
}

/* the body members that change in a run, in one fixed order: pack (to the
 * block) or unpack (from it) */
static unsigned char *CheckpointBody(Polyhedron *P, unsigned char *q, int pack)
{
    double *r = (double *)q;
    /* the reference's restart re-reads r, rho, T, cf, area and volume from
     * the %.6g body file and recomputes the mass properties: kept here too */
    double *members[] = {P->O, &P->I[0][0], &P->V[0][0], &P->W[0][0], &P->at[0][0], &P->ar[0][0],
        P->Fp, P->Fv, P->Tt, &P->to, &P->box[0][0], &P->r, &P->rho, &P->T, &P->cf, &P->area, &P->volume};
    const int sizes[] = {3, 9, 3 * DIMTK, 3 * DIMTK, 3 * DIMTK, 3 * DIMTK, 3, 3, 3, 1, 2 * DIMS, 1, 1, 1, 1, 1, 1};
    int k = 0;
    for (int m = 0; m < (int)(sizeof(sizes) / sizeof(sizes[0])); ++m) {
        for (int c = 0; c < sizes[m]; ++c, ++k) {
            if (pack) {
                r[k] = members[m][c];
            } else {
                members[m][c] = r[k];
            }
        }
    }
    for (; k < CKPT_BODY_REALS; ++k) {
        if (pack) {
            r[k] = 0.0;
        }
    }
    q += CKPT_BODY_REALS * sizeof(double);
    if (0 < P->faceN) {
        Real *arrays[] = {&P->v[0][0], &P->Nv[0][0], &P->Nf[0][0], &P->Ne[0][0]};
        const size_t counts[] = {(size_t)P->vertN, (size_t)P->vertN, (size_t)P->faceN, (size_t)P->edgeN};
        for (int m = 0; m < 4; ++m) {
            const size_t bytes = 3 * sizeof(double) * counts[m];
            if (pack) {
                memcpy(q, arrays[m], bytes);
            } else {
                memcpy(arrays[m], q, bytes);
            }
            q += bytes;
        }
    }
    return q;
}

static unsigned char *CheckpointUser(const Time *time, const Space *space, size_t *bytes)
{
    const Geometry *geo = &(space->geo);
    *bytes = CheckpointUserBytes(geo);
    unsigned char *user = AssignStorage(*bytes);
    unsigned char *q = user;
    double t[3] = {time->now, (double)time->stepC, (double)time->dataC};
    memcpy(q, t, sizeof(t));
    q += sizeof(t);
    int *ids = (int *)q;
    ids[0] = geo->totN;
    for (int n = 0; n < geo->totN; ++n) {
        ids[1 + n] = geo->poly[n].state;
    }
    q += sizeof(int) * (1 + geo->totN);
    for (int n = 0; n < geo->totN; ++n) {
        q = CheckpointBody(geo->poly + n, q, 1);
    }
    return user;
}

/* restart from the checkpoint of output time->restart, when there is one */
static void RestoreCheckpoint(Time *time, Space *space)
{
    char name[64];
    CheckpointName(time->restart, name, sizeof(name));
    FILE *fp = fopen(name, "rb");
    if (NULL == fp) {
        ShowInfo("  no FP64 checkpoint %s: restarting from the data files\n", name);
        return;
    }
    fclose(fp);
    Geometry *geo = &(space->geo);
    size_t cap = CheckpointUserBytes(geo), got = 0;
    unsigned char *user = AssignStorage(cap);
    Check(acfd_checkpoint_load(g_case, name, user, cap, &got), "acfd_checkpoint_load");
    if (got != cap || ((int *)(user + 3 * sizeof(double)))[0] != geo->totN) {
        ShowError("checkpoint %s does not match the case's bodies", name);
    }
    const unsigned char *q = user;
    double t[3];
    memcpy(t, q, sizeof(t));
    q += sizeof(t) + sizeof(int) * (1 + geo->totN);
    time->now = t[0];
    time->stepC = (int)t[1];
    time->dataC = (int)t[2];
    const int *states = (const int *)(user + sizeof(t)) + 1;
    for (int n = 0; n < geo->totN; ++n) {
        geo->poly[n].state = states[n];
        q = CheckpointBody(geo->poly + n, (unsigned char *)q, 0);
    }
    RetrieveStorage(user);
    if (g_surface_on_device) {
        memset(g_surface_on_device, 0, (size_t)geo->totN);
    }
    AcfdUploadGeometry(space);
    g_dev_current = 1;
    g_host_current = 0;
    ShowInfo("  restarted from the FP64 checkpoint %s\n", name);
}

static void WriteCheckpoint(const Time *time, const Space *space, int from_snapshot)
{
    char name[64];
    CheckpointName(time->dataC, name, sizeof(name));
    size_t bytes = 0;
    unsigned char *user = CheckpointUser(time, space, &bytes);
    if (from_snapshot) {
        Check(acfd_snapshot_save(g_case, name, user, bytes), "acfd_snapshot_save");
    } else {
        Check(acfd_checkpoint_save(g_case, name, user, bytes), "acfd_checkpoint_save");
    }
    RetrieveStorage(user);
}

/* Does output n read the node array?  The probe writers (data_probe.c:23-197)
 * return at once when the case defines no probe of their kind, and a case
 * without a probe section leaves their frequencies at INT_MAX, which makes
 * them fire at every step of a long run; only the space data and defined
 * probes need the state on the host. */
static int OutputNeedsNodes(int n, const Time *time)
{
    return (PROSD == n) || (0 < time->dataN[n]);
}

/* the outputs of the snapshot step, written while the device runs on */
static void FlushOutput(Space *space, const Model *model)
{
    if (!g_out.pending) {
        return;
    }
    Check(acfd_snapshot_nodes(g_case, (acfd_node_t *)space->node), "acfd_snapshot_nodes");
    for (int q = 0; q < g_out.count; ++q) {
        const int n = g_out.which[q];
        if (PROFC == n) {
            IntegrateSurfaceForce(space, model);
        }
        if (PROSD == n) {
            ShowInfo("  writing data...\n");
        }
        WriteData(n, &(g_out.time), space, model);
        if (PROSD == n && g_checkpoint) {
            WriteCheckpoint(&(g_out.time), space, 1);
        }
    }
    g_out.pending = 0;
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
        /* the previous step's outputs, while the device computes this one */
        FlushOutput(space, model);
        if (0 != model->psi) {
            GpuSolidStep(time->now, 0.5 * dt, space, model);
        }
        Check(acfd_synchronize(g_case), "acfd_synchronize");
        ShowInfo("  elapsed: %.6gs\n", TockTime(&tm));
        /* outputs: from a snapshot written during the next step when the
         * bodies do not move (the data files also hold the bodies), else at once */
        const int deferred = g_async_output && (0 == model->psi);
        for (int n = 0; n < NPROBE; ++n) {
            rcData[n] = rcData[n] + dt;
            if ((rcData[n] >= dtData[n]) || (time->now == time->end) || (time->stepC == time->stepN)) {
                if (PROSD == n) {
                    ++(time->dataC);
                }
                rcData[n] = zero;
                if (!OutputNeedsNodes(n, time)) {
                    continue;  /* its writer has nothing to write */
                }
                if (deferred) {
                    if (!g_out.pending) {
                        Check(acfd_snapshot_begin(g_case), "acfd_snapshot_begin");
                        g_out.pending = 1;
                        g_out.count = 0;
                    }
                    g_out.which[g_out.count++] = n;
                    g_out.time = *time;
                    continue;
                }
                EnsureHost(space);
                if (PROFC == n) {
                    IntegrateSurfaceForce(space, model);
                }
                if (PROSD == n) {
                    ShowInfo("  writing data...\n");
                }
                WriteData(n, time, space, model);
                if (PROSD == n && g_checkpoint) {
                    WriteCheckpoint(time, space, 0);
                }
            }
        }
    }
    FlushOutput(space, model);
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
    if (0 != time->restart) {
        EnsureCase(space, model);
        RestoreCheckpoint(time, space);
    }
    ShowInfo("  time marching...\n");
    GpuEvolveSolution(time, space, model);
    ShowInfo("Session");
    return 0;
}

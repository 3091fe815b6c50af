/*
 * acfd.h -- C ABI of libacfd_gpu, the sm_100a implementation of the
 * ArtraCFD fluid time step (WENO3/WENO5 characteristic flux-split
 * convection, central viscous flux, RK2/RK3 stage updates inside Strang
 * operator splitting, CFL wave-speed reduction, domain and immersed-boundary
 * ghost-node fill).
 *
 * Every entry point is plain C: integers, doubles, plain structs and raw
 * pointers.  Each returns an int status (ACFD_OK == 0); on failure the message
 * is available from acfd_last_error().  Nothing here calls exit().
 *
 * Conventions shared with the reference code (ArtraCFD, C99):
 *   - node index (k * n[Y] + j) * n[X] + i            cfd_commons.c:323-326
 *   - time levels TO=0, TN=1, TM=2                     commons.h:45-48
 *   - conservative vector rho, rho*u, rho*v, rho*w, rho*eT   commons.h:50
 *   - boundary slots 0 interior, 1..6 west, east, south, north, front, back
 *     (commons.h:61-88), boundary kinds INFLOW=0 .. PERIODIC=4
 *   - partition ranges ns[15][3][2], np[3][3][2]       domain_partition.c:64-128
 */
#ifndef ACFD_H_
#define ACFD_H_

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ACFD_ABI_VERSION 1

/* status codes */
#define ACFD_OK 0
#define ACFD_ERR_ARG 1        /* invalid argument or size */
#define ACFD_ERR_CUDA 2       /* a CUDA runtime call failed */
#define ACFD_ERR_STATE 3      /* call out of order (e.g. no geometry uploaded) */
#define ACFD_ERR_DEVICE 4     /* a kernel reported an error through the device status word */
#define ACFD_ERR_NOMEM 5      /* device allocation failed */
#define ACFD_ERR_NOT_FOUND 6  /* e.g. edge search failed (computational_geometry.c:158-160) */
#define ACFD_ERR_IO 7         /* a checkpoint file could not be read or written */

/* time levels and operators (commons.h:27-48) */
#define ACFD_TO 0
#define ACFD_TN 1
#define ACFD_TM 2
#define ACFD_X 0
#define ACFD_Y 1
#define ACFD_Z 2
#define ACFD_DIMS 3
#define ACFD_PHI 4

/* arithmetic forms selectable with acfd_set_precision() */
#define ACFD_FP64_EXACT 0   /* reference operation order, no FMA contraction */
#define ACFD_FP64 1         /* FP64, reassociated and FMA-contracted (the plain GPU path) */
#define ACFD_FP32_BULK 2    /* stencil/flux/WENO in FP32, RK accumulation and reductions in FP64 */
#define ACFD_FP32_HYBRID 3  /* FP32 bulk + learned smoothness sensor selecting linear upwind-5 */

/* masks for host <-> device node transfers */
#define ACFD_SYNC_TO 0x1u     /* U[TO] */
#define ACFD_SYNC_TN 0x2u     /* U[TN] */
#define ACFD_SYNC_TM 0x4u     /* U[TM] */
#define ACFD_SYNC_U 0x7u      /* all three levels */
#define ACFD_SYNC_FLAGS 0x8u  /* did, fid, lid, gst */
#define ACFD_SYNC_ALL 0xFu

/*
 * Node record.  Same member order, types and size (136 bytes) as the
 * reference's Node (commons.h:128-134) so that a host Node array can be passed
 * as it is.
 */
typedef struct acfd_node {
    int did;          /* domain identifier: 0 fluid, n+1 inside body n, -1 outside PIN */
    int fid;          /* closest facet identifier */
    int lid;          /* interfacial layer identifier */
    int gst;          /* ghost layer identifier */
    double U[3][5];   /* conservative vector at time levels TO, TN, TM */
} acfd_node_t;

/*
 * Domain discretisation: the members of the reference Partition
 * (commons.h:136-159) that the fluid step reads, as plain arrays.
 */
typedef struct acfd_partition {
    int m[3];               /* mesh cells per dimension */
    int n[3];               /* nodes per dimension including ghosts */
    int ng[3];              /* ghost layers per dimension */
    int gl;                 /* ghost layers required by the scheme */
    int collapse;           /* collapse tag (commons.h:36-43) */
    double d[3];            /* mesh size */
    double dd[3];           /* reciprocal mesh size */
    double tinyL;           /* squared smallest length scale */
    int ns[15][3][2];       /* node range of each partition region */
    int np[3][3][2];        /* computational node range with dimension priority */
    int path[30][3];        /* interfacial neighbour search path */
    int pathSep[4];         /* separators in the search path */
    int typeBC[7];          /* boundary kind of each slot */
    int N[7][3];            /* outward normal of each slot */
    double varBC[7][6];     /* given primitive rho,u,v,w,p,T of each slot */
    double domain[3][2];    /* physical extent */
} acfd_partition_t;

/* Numerical and physical model: the reference Model (commons.h:244-268). */
typedef struct acfd_model {
    int tScheme;      /* 0 RK2, 1 RK3 */
    int sScheme;      /* 0 WENO3, 1 WENO5 */
    int sL, sR;       /* stencil offsets */
    int multidim;     /* 0 operator splitting, 1 operator-by-operator */
    int jacobMean;    /* 0 arithmetic, 1 Roe */
    int fluxSplit;    /* 0 local Lax-Friedrichs, 1 Steger-Warming */
    int psi;          /* phase interaction type */
    int ibmLayer;     /* interfacial layers using flow reconstruction */
    int gState;       /* gravity on/off */
    int sState;       /* source term on/off */
    double refMa, refMu, gamma, gasR, cv;
    double refL, refRho, refV, refT;
    double g[3];      /* normalised gravity */
} acfd_model_t;

/*
 * One immersed body: the members of the reference Polyhedron
 * (commons.h:173-204) read by the ghost-node fill and node mapping.
 * faceN <= 0 marks an analytical sphere (centre O, radius r).
 * Arrays are host pointers; acfd_geo_upload copies them.
 */
typedef struct acfd_polyhedron {
    int faceN, edgeN, vertN;
    int state;              /* 1 stationary, 2 no force, otherwise moving */
    double r;               /* radius (sphere) or bounding radius */
    double O[3];            /* centroid */
    double V[3];            /* translational velocity at TO */
    double W[3];            /* rotational velocity at TO */
    double T;               /* wall temperature, < 0 adiabatic */
    double cf;              /* roughness, > 0 no-slip */
    double box[3][2];       /* bounding box */
    const int *f;           /* faceN x 3 face-vertex list */
    const double *Nf;       /* faceN x 3 face normals */
    const int *e;           /* edgeN x 4 edge-vertex-face list, sorted */
    const double *Ne;       /* edgeN x 3 edge normals */
    const double *v;        /* vertN x 3 vertices */
    const double *Nv;       /* vertN x 3 vertex normals */
    double area;            /* surface area (read by acfd_integrate_surface_force) */
} acfd_polyhedron_t;

typedef struct acfd_case acfd_case_t;

/* ---- life cycle -------------------------------------------------------- */

/* Allocate device state for one case on the current CUDA device.
 * Replaces the device side of AllocateProgramMemory (preprocess.c:47-59). */
int acfd_init(const acfd_partition_t *part, const acfd_model_t *model, acfd_case_t **out);
/* Release all device memory of the case (postprocess.c:25-33 counterpart). */
int acfd_finalize(acfd_case_t *cs);
/* Copy the last error message of the calling thread into buf. */
int acfd_last_error(char *buf, size_t len);
/* Library ABI version (ACFD_ABI_VERSION). */
int acfd_abi_version(void);
/* Bind the case to a CUDA stream (cudaStream_t passed as void*; NULL = the
 * library's own stream). */
int acfd_set_stream(acfd_case_t *cs, void *stream);
/* Select the arithmetic form (ACFD_FP64_EXACT, ACFD_FP64, ACFD_FP32_BULK,
 * ACFD_FP32_HYBRID). */
int acfd_set_precision(acfd_case_t *cs, int mode);
/* Wait for all work queued on the case and report device-side errors (the
 * per-step wall clock of solve.c:81,89 needs a finished step). */
int acfd_synchronize(acfd_case_t *cs);
/* Stage-kernel variants of the fast forms (no reference counterpart):
 * 0 .. ACFD_BRICK_VARIANTS-1 are the shared-memory brick kernels with their
 * tile shapes; the next three the line-march kernels launched with 1, 2 or 4
 * waves of resident warps; ACFD_PLANE_VARIANT .. ACFD_STAGE_VARIANTS-1 the
 * plane-march kernels (a TMA ring of halo'd planes) with 1, 2 or 4 waves of
 * blocks, first with each tile's lines cut into equal segments, then with
 * equal shares of all tiles' planes per block.  The choice is kept per arithmetic form; the FP32 forms start on the
 * brick for X and the 4-wave plane march for Y and Z, the FP64 form on the
 * first brick; acfd_autotune replaces these with the measured fastest. */
#define ACFD_BRICK_VARIANTS 2
#define ACFD_PLANE_VARIANT 5
#define ACFD_STAGE_VARIANTS 11
/* Tile autotuner: times every stage-kernel variant of each sweep axis on this
 * case's current state (RK stage 2, reading U[TO] and U[TN] and writing
 * U[TM], after a stage 1 into U[TN]; both are overwritten by every step) for
 * the current arithmetic form and keeps the fastest; tiles[3] (optional)
 * receives the chosen variant per axis. */
int acfd_autotune(acfd_case_t *cs, int tiles[3]);
/* Select the stage-kernel variant of each sweep axis for the current
 * arithmetic form (tests and experiments; acfd_autotune picks by timing). */
int acfd_set_tiles(acfd_case_t *cs, const int tiles[3]);
/* Polls of the bounded device waits of the plane-march stage kernels (a TMA
 * plane in the ring, a free ring slot) before they give up: the kernel then
 * writes the case's status word and leaves, and the next call that reads the
 * status (acfd_sync_to_host, acfd_cfl, ...) returns ACFD_ERR_DEVICE and clears
 * it.  polls < 0 restores the default (4,194,304); 0 gives up at the first
 * wait, which is how failure detection is tested without a GPU fault.  No
 * counterpart in the reference (it has no device waits). */
int acfd_set_wait_limit(acfd_case_t *cs, long long polls);
/* Number of kernels this case has launched so far (graph replays count their
 * kernel nodes).  No reference counterpart: instrumentation (the reference
 * only times whole steps, timer.c:22-35). */
int acfd_stats(acfd_case_t *cs, long long *launches);

/* ---- host <-> device coherence ----------------------------------------- */

/* Upload a host Node array (n[X]*n[Y]*n[Z] records, reference layout).
 * mask selects U levels and/or flags. */
int acfd_sync_to_device(acfd_case_t *cs, const acfd_node_t *node, unsigned mask);
/* Download device state into a host Node array.  Host pages that are not
 * selected by mask are left untouched. */
int acfd_sync_to_host(acfd_case_t *cs, acfd_node_t *node, unsigned mask);
/* Device pointers of the structure-of-arrays state for callers that keep data
 * on the GPU: U[level][var][node] with node = (k*n[Y]+j)*pitch+i, and the four
 * int32 flag planes did, fid, lid, gst.  pitch >= n[X]. */
int acfd_device_state(acfd_case_t *cs, double **U, int **flags, int *pitch, size_t *plane);

/* ---- the fluid time step ----------------------------------------------- */

/* Fluid part of ComputeTimeStep (solve.c:132-151): per-direction maximum of
 * |u_s| + c over PIN nodes with did == 0 of U[TO].  The body-speed part and
 * dt = CFL * min(d/Vmax) stay with the caller.  A fluid node with a
 * non-finite wave speed (NaN or Inf in the state) is passed over by the
 * maxima, as in the reference, and reported: vmax is written and the call
 * returns ACFD_ERR_DEVICE. */
int acfd_cfl(acfd_case_t *cs, double vmax[3]);
/* The same maximum for callers that must not allocate device memory (hosts
 * whose device memory belongs to a pool allocator, or whose memory budget is
 * fixed at start-up so that cudaMalloc/cudaFree may fail or synchronize the
 * device in the time loop).  No counterpart in the reference.
 * U_to: device pointer to the five U[TO] planes (plane stride pitch*n[Y]*n[Z]),
 * did: device pointer to the did plane, vmax_dev: device pointer to 3 doubles
 * (written), stream: cudaStream_t or NULL.  Allocates nothing: its scratch is
 * a fixed 128 KiB device array in the library (4096 blocks' partial maxima and
 * non-finite flags), held on every GPU that loads the library until exit,
 * which limits a case to 33,554,432 computed nodes (larger cases, and PIN
 * ranges outside the node array: ACFD_ERR_ARG).  The call is asynchronous on
 * `stream`: when a fluid node has a non-finite wave speed (the condition for
 * which acfd_cfl returns ACFD_ERR_DEVICE) all three outputs are NaN.  The
 * first call on a device, and the first after its context changed (a device
 * reset), looks up that array's address, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race. */
int acfd_cfl_noalloc(const acfd_partition_t *part, const acfd_model_t *model, const double *U_to,
        const int *did, int pitch, double *vmax_dev, void *stream);
/* EvolveFluidDynamics (fluid_dynamics.c:55-116): one time step of size dt on
 * U[TO], including every TreatBoundary of the stages. */
int acfd_evolve_fluid(acfd_case_t *cs, double dt);
/* One directional solve DiscretizeTime(dt, s) (fluid_dynamics.c:121-148):
 * all RK stages of one sweep s in {X,Y,Z,ACFD_DIMS(=unsplit),ACFD_PHI}. */
int acfd_discretize_time(acfd_case_t *cs, double dt, int s);
/* One stage LLLU (fluid_dynamics.c:157-242):
 * U[tm] = coeA*U[to] + coeB*(U[tn] + dt/ds * L_s U[tn]) on fluid PIN nodes.
 * No boundary treatment. */
int acfd_lllu(acfd_case_t *cs, double dt, double coeA, double coeB,
        int to, int tn, int tm, int s);
/* TreatBoundary (boundary_treatment.c:28-65): immersed ghost nodes first,
 * then the domain ghost shells layer by layer, faces W,E,S,N,F,B. */
int acfd_treat_boundary(acfd_case_t *cs, int tn);
/* Capture one EvolveFluidDynamics into a CUDA graph keyed by dt and replay it
 * (same result as acfd_evolve_fluid). */
int acfd_evolve_fluid_graph(acfd_case_t *cs, double dt);
/* Pieces of a time step, as acfd_profile_step reports them. */
#define ACFD_PIECE_STAGE 0     /* an LLLU stage kernel along sweep axis[i] */
#define ACFD_PIECE_STAGE_XT 1  /* an LLLU stage along x, run as the Y sweep of the transposed state */
#define ACFD_PIECE_FILL 2      /* the ghost fill (TreatBoundary) after a stage */
#define ACFD_PIECE_TRANSPOSE 3 /* U[TO] or the x flags to or from the transposed state */
#define ACFD_PIECE_SENSOR 4    /* the learned sensor's flags of U[TO] */
/* acfd_evolve_fluid with CUDA events around each piece of the step on the
 * case's stream: piece i has kind[i] (ACFD_PIECE_*), axis[i] (the sweep axis,
 * -1 for none), stage[i] (RK stage 0..2 of a stage or fill, else 0) and its
 * device time ms[i].  *count receives the number of pieces, of which the
 * first cap are written.  The step is a real step (U[TO] advances); the call
 * synchronizes.  Instrumentation with no reference counterpart (the
 * reference times whole steps, timer.c:22-35). */
int acfd_profile_step(acfd_case_t *cs, double dt, int cap, int *kind, int *axis, int *stage, float *ms,
        int *count);

/* ---- immersed boundaries ---------------------------------------------- */

/* Upload (or replace after host-side motion) the body list.  On an update of
 * the same bodies, a triangulated body given with v, Nv, Nf and Ne all NULL
 * keeps the surface it has on the device (moved there by
 * acfd_transform_polyhedron); its f and e are then ignored. */
int acfd_geo_upload(acfd_case_t *cs, const acfd_polyhedron_t *poly, int totN);
/* TransformPolyhedron (computational_geometry.c:162-208) of triangulated
 * body n of the last acfd_geo_upload, with its surface on the device: the
 * vertices are shifted to the reference point O, scaled by scale, rotated by
 * angle (about x, then y, then z), offset by offset and shifted back; the
 * face, edge and vertex normals are rotated.  On the host: centroid[3] (in,
 * out) is moved like a vertex, inertia[9] (in, out; row-major I) is rotated,
 * and box[6] (out: min x, max x, min y, max y, min z, max z) receives the
 * reference's bounding box of the moved vertices and centroid.  Bitwise
 * equal to the reference.  The body list on the device keeps its old
 * centroid and box until the next acfd_geo_upload, which passes NULL surface
 * arrays to keep the moved surface.  ApplyMotion (solid_dynamics.c:380-410)
 * calls it with O = the centroid and scale = 1. */
int acfd_transform_polyhedron(acfd_case_t *cs, int n, const double O[3], const double scale[3],
                              const double angle[3], const double offset[3], double centroid[3],
                              double inertia[9], double box[6]);
/* The device surface of triangulated body n to host arrays: v[vertN*3],
 * Nf[faceN*3], Ne[edgeN*3], Nv[vertN*3]; a NULL output is skipped. */
int acfd_geo_fetch(acfd_case_t *cs, int n, double *v, double *Nf, double *Ne, double *Nv);
/* ComputeGeometricField (immersed_boundary.c:65-264): did, fid, lid, gst and
 * the reconstruction of newly uncovered fluid nodes on U[TO]. */
int acfd_compute_geometric_field(acfd_case_t *cs);
/* TreatImmersedBoundary (immersed_boundary.c:270-340) on level tn. */
int acfd_treat_ib(acfd_case_t *cs, int tn);
/* IntegrateSurfaceForce (solid_dynamics.c:51-171) on the device, from U[TO]
 * and the node flags: for every body with state <= 0 the pressure force Fp,
 * the shear force Fv and the torque Tt, summed over the body's ghost nodes of
 * layer 2 in the reference's node order and calibrated by its surface area
 * over its interfacial nodes of layer 2 (bitwise equal to the reference
 * except through pow() in the viscosity of no-slip viscous bodies).
 * force: totN x 9 doubles (Fp[3], Fv[3], Tt[3] per body) in host memory;
 * rows of bodies with state > 0 are left unchanged.  Uses the body list of
 * the last acfd_geo_upload (centroid, velocities, roughness, area). */
int acfd_integrate_surface_force(acfd_case_t *cs, double *force);
/* The contact scan of ApplyCollision (solid_dynamics.c:242-256, the search of
 * DetectColState and AddColObject :327-357) on the device: for every body p
 * with state != 1, the bodies met by the collision search path
 * (Partition.path[0 .. pathSep[1]-1]) from p's interfacial nodes of layer 1,
 * in the order of the reference's contact list, each with its line of impact
 * (the summed path offsets, before normalisation).  Host arrays, totN = the
 * body count: counts[totN], gid[totN * totN] (body ids, did numbering: 1 =
 * first body), N[totN * totN * 3]; contact c of body p is gid[p*totN + c],
 * N[(p*totN + c)*3 + 0..2]. */
int acfd_collision_scan(acfd_case_t *cs, int *counts, int *gid, int *N);

/* ---- output snapshots and FP64 checkpoints -----------------------------
 * The reference writes its fields as float32 (EnSight) or %.6g text
 * (ParaView) and restarts from those files (ReadData, data_stream.c:71-90),
 * losing precision.  A checkpoint holds the node records of every node
 * (ghosts included, all three levels and the flags, the reference's Node
 * layout) in FP64, after a 64-byte header {"ACFDCKP1", version 1, node
 * bytes, n[3], node count, size of the caller's block} and the caller's
 * block (e.g. time and body state), so a restart continues bit for bit.
 *
 * acfd_snapshot_begin queues, on the case's stream, a copy of the node
 * records into device memory and from there, on a stream of its own, into
 * pinned host memory, and returns at once: work queued afterwards overlaps
 * the copy.  acfd_snapshot_nodes / acfd_snapshot_save wait for that copy and
 * give the records (as acfd_sync_to_host with ACFD_SYNC_ALL would have at the
 * time of acfd_snapshot_begin) or write them as a checkpoint.  A new
 * snapshot replaces the previous one. */
int acfd_snapshot_begin(acfd_case_t *cs);
int acfd_snapshot_nodes(acfd_case_t *cs, acfd_node_t *node);
int acfd_snapshot_save(acfd_case_t *cs, const char *path, const void *user, size_t user_bytes);
/* Synchronous checkpoint of the current state (a snapshot written at once). */
int acfd_checkpoint_save(acfd_case_t *cs, const char *path, const void *user, size_t user_bytes);
/* Restore a checkpoint of a case with the same node counts: every node
 * record goes to the device; the caller's block (at most user_cap bytes) is
 * copied to user and its size to *user_bytes (also when it does not fit:
 * ACFD_ERR_ARG). */
int acfd_checkpoint_load(acfd_case_t *cs, const char *path, void *user, size_t user_cap, size_t *user_bytes);

/* ---- learned smoothness sensor (no counterpart in the reference) ------- */

/* Number of float parameters of the sensor MLP (10 -> 32 -> 32 -> 1):
 * W1[32][10], b1[32], W2[32][32], b2[32], w3[32], b3. */
int acfd_mlp_param_count(void);
/* Load trained parameters (host array) into the case and set the probability
 * threshold above which a node keeps the full WENO5 reconstruction; enables
 * acfd_set_precision(ACFD_FP32_HYBRID). */
int acfd_sensor_load(acfd_case_t *cs, const float *params, float threshold);
/* The same from a file: "ACFDSNS1", int32 parameter count, float32
 * threshold, float32 parameters (artracfd_b200/sensor_weights.bin holds the
 * trained sensor). */
int acfd_sensor_load_file(acfd_case_t *cs, const char *path);
/* Evaluate the sensor on U[TO] for the three sweep axes (the hybrid step does
 * this itself at its start); *flagged (optional) = number of flags set. */
int acfd_sensor_update(acfd_case_t *cs, unsigned long long *flagged);
/* Device pointer to the flags of the last evaluation: 3 planes (sweep axis
 * x, y, z) of uint8 in the node layout of acfd_device_state; 1 = full WENO5. */
int acfd_sensor_flags(acfd_case_t *cs, const unsigned char **flags);
/* Training data along axis s for every PIN node, in PIN order (x fastest):
 * features (device, count x 10) and the WENO5 weight departure of the
 * node's two interfaces (device, count; -1 for non-fluid nodes). */
int acfd_sensor_features(acfd_case_t *cs, int s, float *features, float *departure);
/* MLP on device arrays: probabilities of n samples. */
int acfd_mlp_forward(const float *params, const float *X, int n, float *prob, void *stream);
/* Sum over n samples of the weighted binary cross-entropy (weight pos_weight
 * for label 1) and of its gradient; *grad (param_count) and *loss are
 * accumulated, the caller zeroes them. */
int acfd_mlp_grad(const float *params, const float *X, const float *Y, int n, float pos_weight, float *grad,
        float *loss, void *stream);
/* One Adam step (beta1 0.9, beta2 0.999, eps 1e-8) on grad * scale. */
int acfd_mlp_adam(float *params, const float *grad, float *m, float *v, int step, float lr, float scale,
        void *stream);

/* ---- batch of independent cases (no reference counterpart) ------------ */

/* Many independent cases advanced together: each RK stage of every case is
 * one launch over the tiles of all cases (the plane-march or the persistent
 * brick stage kernel of the FP32 forms), each case keeps its own grid, model, boundary
 * conditions and time step (computed on the device from its CFL maximum, as
 * ComputeTimeStep does, solve.c:108-153), and one time step of the whole
 * batch is captured and replayed as a CUDA graph.  Cases must be 3D, WENO5,
 * dimension-split, without gravity, with one common RK scheme and no
 * immersed bodies. */
typedef struct acfd_batch acfd_batch_t;
/* Create a batch of ncase cases (parts[c], models[c]); each case gets its own
 * device state as acfd_init would allocate it. */
int acfd_batch_init(int ncase, const acfd_partition_t *parts, const acfd_model_t *models, acfd_batch_t **out);
int acfd_batch_finalize(acfd_batch_t *b);
/* The case handle of case c, for acfd_sync_to_device / acfd_sync_to_host /
 * acfd_treat_boundary / acfd_cfl on that case (not acfd_batch_finalize'd
 * separately). */
int acfd_batch_case(acfd_batch_t *b, int c, acfd_case_t **cs);
/* ACFD_FP32_BULK (default) or ACFD_FP32_HYBRID (after acfd_batch_sensor_load). */
int acfd_batch_set_precision(acfd_batch_t *b, int mode);
/* Load the learned sensor into every case (see acfd_sensor_load). */
int acfd_batch_sensor_load(acfd_batch_t *b, const float *params, float threshold);
/* Advance every case by `steps` time steps; cfl[c] is the CFL number of case
 * c; dts (optional, steps x ncase doubles) receives the dt of every case and
 * step.  Returns after the work has finished. */
int acfd_batch_advance(acfd_batch_t *b, const double *cfl, int steps, double *dts);
/* Stage kernel of the batch:
 *  ACFD_BATCH_PLANE       one plane-march launch per RK stage over all cases
 *                         (the default when all cases are viscous or all
 *                         inviscid);
 *  ACFD_BATCH_PERSISTENT  the RK stages of each directional half step of
 *                         every case in one persistent launch (six per time
 *                         step) of plane-march blocks and ghost fills,
 *                         linked by per-case counters (bounded waits); when
 *                         every case's ghost fill is a copy;
 *  ACFD_BATCH_BRICK       the persistent brick kernel that pulls (case, tile)
 *                         items from a counter, one launch per RK stage. */
#define ACFD_BATCH_BRICK 0
#define ACFD_BATCH_PLANE 1
#define ACFD_BATCH_PERSISTENT 2
int acfd_batch_set_kernel(acfd_batch_t *b, int kernel);
/* Run the batch's work on the caller's CUDA stream (cudaStream_t as void*);
 * the library's own stream is released. */
int acfd_batch_set_stream(acfd_batch_t *b, void *stream);
/* Kernels launched by the batch so far (graph replays count their kernel
 * nodes). */
int acfd_batch_stats(acfd_batch_t *b, long long *launches);

/* ---- per-point device twins (batched; host arrays in and out) --------- */

/* WENO3 (weno3.c:35-55) / WENO5 (weno5.c:35-62) on count stencils:
 * F is count x 5 x 5 (stencil point, component), Fhat count x 5. */
int acfd_weno_batch(int scheme, int mode, const double *F, double *Fhat, int count);
/* ComputeFhat (convective_flux.c:48-84) on count interfaces:
 * Ust is count x 6 x 5 (stencil points sL..sR of U along s; WENO3 uses the
 * first 4), Fhat count x 5. */
int acfd_fhat_batch(const acfd_model_t *model, int s, int mode, const double *Ust,
        double *Fhat, int count);

#ifdef __cplusplus
}
#endif

#endif /* ACFD_H_ */

/*
 * solid_gpu.c -- the rigid-body half step of GPU mode (EvolveSolidDynamics,
 * solid_dynamics.c:38-49) with every part that reads the node array on the
 * device, so that the node array never leaves the GPU in the time loop.
 *
 * The reference's solid_dynamics.c is compiled here as it is (it is included
 * below instead of being compiled on its own, see the Makefile) so that its
 * static ApplyKinematics and ApplyMotion run unchanged on the host.  The
 * parts that scan nodes run in libacfd_gpu:
 *   IntegrateSurfaceForce  -> acfd_integrate_surface_force
 *   the contact scan of ApplyCollision (DetectColState / AddColObject)
 *                          -> acfd_collision_scan
 *   TransformPolyhedron of ApplyMotion
 *                          -> acfd_transform_polyhedron (ACFD_MOTION=host
 *                             keeps the reference's ApplyMotion)
 *   ComputeGeometricField  -> acfd_compute_geometric_field
 *   TreatImmersedBoundary  -> acfd_treat_ib
 * and the velocity exchange of ApplyCollision (solid_dynamics.c:262-318)
 * runs here on the contact lists, in the reference's operation order.
 */
#include "solid_dynamics.c"

#include "acfd.h"
#include "acfd_shim.h"

static void SolidCheck(int status, const char *what)
{
    if (ACFD_OK != status) {
        char msg[1024];
        acfd_last_error(msg, sizeof(msg));
        ShowError("%s failed (%d): %s", what, status, msg);
    }
}

/* surface forces of the bodies from the device (rows of bodies with
 * state > 0 keep their values, as in the reference) */
static void DeviceSurfaceForce(acfd_case_t *cs, Space *space)
{
    Geometry *const geo = &(space->geo);
    double *force = AssignStorage(9 * geo->totN * sizeof(*force));
    for (int n = 0; n < geo->totN; ++n) {
        const Polyhedron *poly = geo->poly + n;
        for (int s = 0; s < DIMS; ++s) {
            force[9 * n + s] = poly->Fp[s];
            force[9 * n + 3 + s] = poly->Fv[s];
            force[9 * n + 6 + s] = poly->Tt[s];
        }
    }
    SolidCheck(acfd_integrate_surface_force(cs, force), "acfd_integrate_surface_force");
    for (int n = 0; n < geo->totN; ++n) {
        Polyhedron *poly = geo->poly + n;
        for (int s = 0; s < DIMS; ++s) {
            poly->Fp[s] = force[9 * n + s];
            poly->Fv[s] = force[9 * n + 3 + s];
            poly->Tt[s] = force[9 * n + 6 + s];
        }
    }
    RetrieveStorage(force);
}

/* ApplyCollision's velocity exchange on the device's contact lists: a body
 * with contacts starts from its averaged velocity (level TN); each contact
 * whose normalised line of impact closes the gap (positive relative normal
 * speed) removes the normal momentum share of the pair with the averaged
 * restitution coefficient and the tangential slip scaled by the averaged
 * roughness, and damps the relative spin; a body whose contacts all
 * separate keeps its original velocity.  Bodies that collided carry the
 * new velocity into level TN as well. */
static void DeviceCollision(acfd_case_t *cs, Space *space)
{
    Geometry *const geo = &(space->geo);
    const int totN = geo->totN;
    const int mark = INT_MAX / 2;
    const Real restitution[5] = {0.0, 0.25, 0.5, 0.75, 1.0};
    int *counts = AssignStorage(totN * sizeof(*counts));
    int *gid = AssignStorage(totN * totN * sizeof(*gid));
    int *lines = AssignStorage(3 * totN * totN * sizeof(*lines));
    SolidCheck(acfd_collision_scan(cs, counts, gid, lines), "acfd_collision_scan");
    for (int p = 0; p < totN; ++p) {
        Polyhedron *a = geo->poly + p;
        if ((1 == a->state) || (0 == counts[p])) {
            continue;
        }
        RealVec V0, W0;
        for (int s = 0; s < DIMS; ++s) {
            V0[s] = a->V[TO][s];
            W0[s] = a->W[TO][s];
            a->V[TO][s] = a->V[TN][s];
            a->W[TO][s] = a->W[TN][s];
        }
        const Real ma = a->rho * a->volume;
        for (int c = 0; c < counts[p]; ++c) {
            const int *line = lines + 3 * (p * totN + c);
            const int last = (counts[p] - 1 == c);
            RealVec L = {line[X], line[Y], line[Z]};
            if (0 == abs(line[X]) + abs(line[Y]) + abs(line[Z])) {
                if (last && (mark > a->state)) {
                    memcpy(a->V[TO], V0, sizeof(V0));
                    memcpy(a->W[TO], W0, sizeof(W0));
                }
                continue;
            }
            const Real len = sqrt(L[X] * L[X] + L[Y] * L[Y] + L[Z] * L[Z]);
            for (int s = 0; s < DIMS; ++s) {
                L[s] = L[s] / len;
            }
            const Polyhedron *b = geo->poly + gid[p * totN + c] - 1;
            RealVec dV, dW;
            for (int s = 0; s < DIMS; ++s) {
                dV[s] = a->V[TN][s] - b->V[TN][s];
                dW[s] = a->W[TN][s] - b->W[TN][s];
            }
            const Real vn = dV[X] * L[X] + dV[Y] * L[Y] + dV[Z] * L[Z];
            if (0.0 >= vn) {
                if (last && (mark > a->state)) {
                    memcpy(a->V[TO], V0, sizeof(V0));
                    memcpy(a->W[TO], W0, sizeof(W0));
                }
                continue;
            }
            if (mark > a->state) {
                a->state = a->state + mark;
            }
            const Real mb = b->rho * b->volume;
            const Real share = mb / (ma + mb);
            const Real e = 0.5 * (restitution[a->mid] + restitution[b->mid]);
            const Real mu = 0.5 * (a->cf + b->cf);
            for (int s = 0; s < DIMS; ++s) {
                a->V[TO][s] = a->V[TO][s] - share * (1.0 + e) * vn * L[s] - mu * (dV[s] - vn * L[s]);
                a->W[TO][s] = a->W[TO][s] - share * dW[s];
            }
        }
    }
    for (int p = 0; p < totN; ++p) {
        Polyhedron *a = geo->poly + p;
        if (mark > a->state) {
            continue;
        }
        a->state = a->state - mark;
        memcpy(a->V[TN], a->V[TO], sizeof(a->V[TO]));
        memcpy(a->W[TN], a->W[TO], sizeof(a->W[TO]));
    }
    RetrieveStorage(lines);
    RetrieveStorage(gid);
    RetrieveStorage(counts);
}

/* ApplyMotion (solid_dynamics.c:380-410) with the surfaces of triangulated
 * bodies transformed on the device (acfd_transform_polyhedron, the
 * reference's TransformPolyhedron): the host receives their centroid,
 * inertia tensor and box, and fetches the surface only for output */
static void DeviceMotion(acfd_case_t *cs, const Real dt, Space *space)
{
    Geometry *const geo = &(space->geo);
    const RealVec scale = {1.0, 1.0, 1.0};
    for (int n = 0; n < geo->totN; ++n) {
        Polyhedron *poly = geo->poly + n;
        if (1 == poly->state) {
            continue;
        }
        RealVec offset, angle;
        for (int s = 0; s < DIMS; ++s) {
            offset[s] = poly->V[TN][s] * dt;
            angle[s] = poly->W[TN][s] * dt;
        }
        if (0 >= poly->faceN) {
            for (int s = 0; s < DIMS; ++s) {
                poly->O[s] = poly->O[s] + offset[s];
            }
            for (int s = 0; s < DIMS; ++s) {
                poly->box[s][MIN] = poly->O[s] - poly->r;
                poly->box[s][MAX] = poly->O[s] + poly->r;
            }
            continue;
        }
        const RealVec O = {poly->O[X], poly->O[Y], poly->O[Z]};
        double box[6];
        SolidCheck(acfd_transform_polyhedron(cs, n, O, scale, angle, offset, poly->O, &poly->I[0][0], box),
                "acfd_transform_polyhedron");
        for (int s = 0; s < DIMS; ++s) {
            poly->box[s][MIN] = box[2 * s];
            poly->box[s][MAX] = box[2 * s + 1];
        }
        AcfdMarkSurfaceOnDevice(n);
    }
}

void AcfdDeviceSolidStep(acfd_case_t *cs, const Real now, const Real dt, Space *space, const Model *model)
{
    DeviceSurfaceForce(cs, space);
    ApplyKinematics(now, dt, space);
    if (1 != model->psi) {
        DeviceCollision(cs, space);
    }
    if (AcfdMotionOnDevice()) {
        DeviceMotion(cs, dt, space);
    } else {
        ApplyMotion(dt, space);
    }
    AcfdUploadGeometry(space);
    SolidCheck(acfd_compute_geometric_field(cs), "acfd_compute_geometric_field");
    SolidCheck(acfd_treat_ib(cs, TO), "acfd_treat_ib");
}

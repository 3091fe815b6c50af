/*
 * acfd_shim.h -- declarations of the reference-side drop-in (see acfd_shim.c).
 */
#ifndef ACFD_SHIM_H_
#define ACFD_SHIM_H_

#include "commons.h"
#include "acfd.h"

/* 1 when the program was started with -m gpu */
extern int g_acfd_gpu_mode;

/* the reference's own functions, renamed at compile time by the Makefile */
int RefSolve(Time *, Space *, const Model *);
void RefEvolveFluidDynamics(const Real, Space *, const Model *);
void RefTreatBoundary(const int, Space *, const Model *);

/* release the device case (called by main before Postprocess) */
void AcfdShimFinalize(void);

/* send the bodies as they are on the host to the device */
void AcfdUploadGeometry(const Space *);
/* 1 unless ACFD_MOTION=host: moving triangulated surfaces stay on the device */
int AcfdMotionOnDevice(void);
/* body n's surface was moved on the device (the host fetches it when needed) */
void AcfdMarkSurfaceOnDevice(int n);
/* the rigid-body half step with the node scans on the device (solid_gpu.c) */
void AcfdDeviceSolidStep(acfd_case_t *, const Real now, const Real dt, Space *, const Model *);

#endif

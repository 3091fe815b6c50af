/*
 * acfd_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the ArtraCFD fluid time step, used as the parity checker
 * for libacfd_gpu.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg load it; the product never links it.  Every function
 * follows the reference operation by operation (same evaluation order, no
 * FMA contraction: build with -ffp-contract=off) so that FP64 results are
 * bitwise identical to the reference on the same inputs, which the CPU tests
 * check against the reference itself (oracle/_ref) and against the committed
 * fixtures in tests/golden/.
 */
#ifndef ACFD_ORACLE_H_
#define ACFD_ORACLE_H_

#include "acfd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* per-point functions */
void orc_symmetric_average(int averager, double gamma, const double UL[5],
        const double UR[5], double Uo[6]);
void orc_eigenvectors(int s, double gamma, const double Uo[6], double L[5][5], double R[5][5]);
void orc_weno5(const double F[5][5], double Fhat[5]);
void orc_weno3(const double F[3][5], double Fhat[5]);
void orc_fhat_stencil(const acfd_model_t *model, int s, const double Ust[6][5], double Fhat[5]);
void orc_compute_fhat(int tn, int s, int k, int j, int i, const acfd_partition_t *part,
        const acfd_node_t *node, const acfd_model_t *model, double Fhat[5]);
void orc_compute_fvhat(int tn, int s, int k, int j, int i, const acfd_partition_t *part,
        const acfd_node_t *node, const acfd_model_t *model, double Fvhat[5]);

/* the time step */
void orc_lllu(double dt, double coeA, double coeB, int to, int tn, int tm, int p,
        acfd_node_t *node, const acfd_partition_t *part, const acfd_model_t *model);
void orc_treat_domain_boundary(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model);
void orc_treat_boundary(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);
void orc_discretize_time(double dt, int s, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);
void orc_evolve_fluid(double dt, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);
void orc_cfl(const acfd_node_t *node, const acfd_partition_t *part, const acfd_model_t *model,
        double vmax[3]);
double orc_time_step(double numCFL, const acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);

/* immersed boundary */
void orc_compute_geometric_field(acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);
void orc_treat_ib(int tn, acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN);
int orc_point_in_polyhedron(const double p[3], const acfd_polyhedron_t *poly, int *fid);
int orc_collision_scan(const acfd_node_t *node, const acfd_partition_t *part, const acfd_polyhedron_t *poly,
        int totN, int p, int *gid, int *N);
void orc_integrate_surface_force(const acfd_node_t *node, const acfd_partition_t *part,
        const acfd_model_t *model, const acfd_polyhedron_t *poly, int totN, double *force);
void orc_transform_polyhedron(const double O[3], const double scale[3], const double angle[3],
        const double offset[3], int vertN, int faceN, int edgeN, double *v, double *Nf, double *Ne,
        double *Nv, double centroid[3], double inertia[9], double box[6]);

/* host-side set-up restated from the reference (parameters and partition) */
void orc_set_node_number(acfd_partition_t *part, acfd_model_t *model);
void orc_partition_domain(acfd_partition_t *part);

#ifdef __cplusplus
}
#endif

#endif

/*
 * qz_dropin.h -- the QUANTIZER hot-path entry points exported by
 * libqz_dropin.so with the reference's own names and signatures, so that the
 * reference's main.c and its host bookkeeping (initialization, tree
 * construction / adaptation, I/O) link against this library in place of the
 * reference objects grid_density.o potential*.o grid_acceleration.o
 * particle_acceleration.o particle_updating.o ptcl_idx_to_box_idx.o reset.o
 * poisson_error.o and force_methods/*.o.
 *
 * Data passing is the reference's: globals (GL_ptcl_*, GL_ptr_tree, solver
 * parameters; headers/common.h:105-260), which the library looks up in the
 * host program by name at its first call (link the program with
 * -Wl,--export-dynamic, or build the bookkeeping as a shared object).  vtype
 * is double (_VTYPE_ 2).  Device state mirrors the host arrays; every entry
 * point writes the arrays it changes back to the host before returning, so
 * the reference's C code always reads current values.  Errors follow the
 * reference: a message on stdout and _FAILURE_ (1) from int functions.
 *
 * Each declaration cites the reference declaration it replaces.
 */
#ifndef QZ_DROPIN_H
#define QZ_DROPIN_H
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define QZ_DROPIN_API __attribute__((visibility("default")))
#else
#define QZ_DROPIN_API
#endif

struct node;

/* headers/grid_density.h:32 */
QZ_DROPIN_API void grid_density(void);
/* headers/potential.h:36 */
QZ_DROPIN_API int potential(void);
/* headers/potential_head_node.h:36 */
QZ_DROPIN_API int potential_head_node(void);
/* headers/potential_branches.h:35 */
QZ_DROPIN_API int potential_branches(void);
/* headers/grid_acceleration.h:32 */
QZ_DROPIN_API int grid_acceleration(void);
/* headers/particle_acceleration.h:32 */
QZ_DROPIN_API int particle_acceleration(void);
/* headers/particle_updating.h:33 */
QZ_DROPIN_API int particle_updating_A(double dt);
/* headers/particle_updating.h:34 */
QZ_DROPIN_API void particle_updating_B(double dt);
/* headers/ptcl_idx_to_box_idx.h:34 */
QZ_DROPIN_API int ptcl_idx_to_box_idx(struct node *ptr_node, int ptcl_idx);
/* headers/reset.h:33 */
QZ_DROPIN_API int reset(void);
/* headers/poisson_error.h:34 */
QZ_DROPIN_API bool poisson_error(struct node *ptr_node, double *error, double error_total_pow2,
                                 int type);
/* headers/multigrid.h:35 */
QZ_DROPIN_API void multigrid(double *phi, const double *rho, int gridsize, int type_multigrid);
/* headers/gauss_saidel.h:32 */
QZ_DROPIN_API void gauss_saidel(double *phi, const double *rho, int gridsize, int iter_max);
/* headers/jacobi.h:32 */
QZ_DROPIN_API void jacobi(double *phi, const double *rho, int gridsize, int iter_max);
/* headers/conjugate_gradient.h:33 */
QZ_DROPIN_API int conjugate_gradient(struct node *ptr_node);
/* headers/observables.h:32 */
QZ_DROPIN_API int observables(void);

/* headers/timestep.h: int timestep(vtype *ptr_dt) */
QZ_DROPIN_API int timestep(double *ptr_dt);

/* headers/conjugate_gradient_multigrid.h:32 */
QZ_DROPIN_API void conjugate_gradient_multigrid(double *phi, const double *rho, int gridsize,
                                                int conj_grad_iter);
/* headers/multigrid2.h (multigrid2 is not called by the reference: potential_head_node.c:77) */
QZ_DROPIN_API void multigrid2(double *phi, double *rho, int type_multigrid);

/* Library controls with no reference counterpart. */
/* Re-upload the particle state and head fields from the host globals (call
 * after host code other than these entry points modified them). */
QZ_DROPIN_API int qz_dropin_sync_from_host(void);
/* The library context behind the shim (a qz_sim *, see qz_b200.h), or NULL. */
QZ_DROPIN_API void *qz_dropin_context(void);

#ifdef __cplusplus
}
#endif
#endif

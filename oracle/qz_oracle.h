/*
 * qz_oracle.h -- CPU restatement of the QUANTIZER per-step particle-mesh
 * path, used ONLY as the checker of the CUDA library (tests/, smoke() and the
 * cpu_baseline leg of bench.py).  Never linked into the product.
 *
 * Every function restates one reference routine (cited per function in
 * qz_oracle.c) with the same floating-point expression order, so that with
 * -ffp-contract=off it reproduces the reference's FP64 results bit for bit on
 * the head-only path; tests pin it against fixtures dumped by the compiled
 * reference (tests/golden/).
 *
 * Head-node layout (source/initialization.c:47-270): level L, box of
 * B = 2^L + 2 cells per side (one ghost cell each side, box_ts = -1), grid
 * fields of D = B + 1 = 2^L + 3 points per side, linear index
 * i + j*D + k*D*D.  Solve grid = box points 1 .. 2^L+1 per axis.
 */
#ifndef QZ_ORACLE_H
#define QZ_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int L;               /* head level lmin */
    double G;            /* gravitational constant */
    double total_mass;   /* GL_total_mass_initial */
    int bdry;            /* 0 periodic, 1 reflexive, 2 outflow */
    int solver;          /* smoother: 0 Gauss-Seidel, 1 Jacobi, 2 CG */
    int cycle;           /* 0 V, 1 F, 2 W */
    int n_pre, n_post, n_coarse;
    double w_sor;        /* _w_SOR_HEAD_ */
    double tol, tol2;    /* residual and ratio thresholds */
    int check_every;     /* iter_between_check_potential_solution */
    int max_iter;        /* _MAX_NUMBER_OF_ITERATIONS_IN_POISSON_EQUATION_ */
    int check_method;    /* check_poisson_error_method 0/1/2 */
    int force_stencil;   /* 0 = 3-point, 1 = 5-point */
    int head_pot_method; /* 0 multigrid cycles, 1 node conjugate gradient */
} qzo_params;

void qzo_default_params(qzo_params *p, int L);
long qzo_grid_points(int L);

/* initial_potential_and_acceleration_head.c:297-334 (non-periodic). */
void qzo_initial_head(const qzo_params *p, double *pot, double *ax, double *ay, double *az);
/* reset.c:29-64 + grid_density.c:35-111 */
void qzo_deposit_head(const qzo_params *p, long n, const double *x, const double *y,
                      const double *z, const double *m, double *d);
/* force_methods/gauss_saidel.c:29-55 */
void qzo_gauss_saidel(double *phi, const double *rho, int gridsize, int iters, double w);
/* force_methods/jacobi.c:29-82 */
void qzo_jacobi(double *phi, const double *rho, int gridsize, int iters, double w);
/* timestep.c:35-157, 589-700 (head only) */
double qzo_timestep_head(int L, int method, double cfl, double max_dt, long n, const double *vx,
                         const double *vy, const double *vz, const double *ax, const double *ay,
                         const double *az);
/* conjugate_gradient_multigrid.c:29-176 */
void qzo_cg_smooth(double *phi, const double *rho, int gridsize, int iters);
/* force_methods/multigrid.c:106-229 */
void qzo_multigrid(const qzo_params *p, double *phi, const double *rho, int gridsize, int type);
/* poisson_error.c:36-133 for the head node; returns 1 when converged. */
int qzo_poisson_check_head(const qzo_params *p, double *pot, double *pot_old, const double *d,
                           double node_mass);
/* conjugate_gradient.c:322-463 on the head node with poisson_error.c:235-347
 * (type 1); returns iterations used (negative on failure). */
int qzo_cg_head(const qzo_params *p, double *pot, double *pot_old, const double *d,
                double node_mass);
/* potential_head_node.c:32-179; returns V-cycles (or conjugate gradient
 * iterations) used, negative on failure. */
int qzo_potential_head(const qzo_params *p, double *pot, double *pot_old, double *d,
                       double node_mass);
/* grid_acceleration.c:36-76 (3-point) */
void qzo_grid_accel_head(const qzo_params *p, const double *pot, double *ax, double *ay, double *az);
/* particle_acceleration.c:33-132 (adds into pax/pay/paz) */
void qzo_gather_head(const qzo_params *p, long n, const double *x, const double *y, const double *z,
                     const double *ax, const double *ay, const double *az,
                     double *pax, double *pay, double *paz);
/* particle_updating.c:39-207 (bdry 0/1; outflow not restated) */
int qzo_update_A_head(const qzo_params *p, long n, double dt, double *x, double *y, double *z,
                      double *vx, double *vy, double *vz, double *ax, double *ay, double *az);
/* particle_updating.c:123-196 (outflow, head only); returns the new count */
long qzo_update_A_outflow(long n, double dt, double *x, double *y, double *z, double *vx,
                          double *vy, double *vz, double *ax, double *ay, double *az,
                          const double *m, double *node_mass);
/* particle_updating.c:2677-2688 */
void qzo_update_B_head(long n, double dt, double *vx, double *vy, double *vz,
                       const double *ax, const double *ay, const double *az);
/* ptcl_idx_to_box_idx.c:30-139 for a non-periodic node geometry. */
int qzo_box_idx(int lv, int box_ts_x, int box_ts_y, int box_ts_z, int box_real_dim_x,
                int box_real_dim_y, double x, double y, double z);
void qzo_box_idx_batch(int lv, int box_ts_x, int box_ts_y, int box_ts_z, int box_real_dim_x,
                       int box_real_dim_y, long n, const double *x, const double *y,
                       const double *z, int *out);

/* Head-only state for a whole simulation (main.c:296-481 call order). */
typedef struct {
    qzo_params p;
    long n;
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
    double *pot, *pot_old, *d, *gax, *gay, *gaz;
    long vcycles_total;
    int last_vcycles;
    double head_mass; /* the head's node_mass (falls with outflow removals) */
} qzo_sim;

int qzo_sim_init(qzo_sim *s, const qzo_params *p, long n, const double *x, const double *y,
                 const double *z, const double *vx, const double *vy, const double *vz,
                 const double *m);
/* One step: update_A, reset, deposit, potential, grid accel, gather, update_B. */
int qzo_sim_step(qzo_sim *s, double dt);
void qzo_sim_free(qzo_sim *s);

#ifdef __cplusplus
}
#endif
#endif

/*
 * qz_b200.h -- C ABI of the B200 particle-mesh library (libqzb200.so).
 *
 * Plain pointers and sizes only.  All state lives in device memory owned by an
 * opaque qz_sim; host pointers passed to qz_set_* / qz_get_* are copied
 * through pinned staging buffers.  Every entry point returns QZ_SUCCESS (0)
 * or QZ_FAILURE (1), the reference's int convention (headers/common.h:81-82);
 * qz_last_error() gives the message.  There is no CPU fallback: without a
 * CUDA device every compute entry point fails.
 *
 * The per-stage functions mirror the reference's hot-path entry points one to
 * one (citations are QUANTIZER file:line of the routine each replaces):
 *   qz_grid_density          grid_density          source/grid_density.c:269-306
 *   qz_potential             potential             source/potential.c:29-51
 *                            potential_head_node   source/potential_head_node.c:99-179
 *   qz_grid_acceleration     grid_acceleration     source/grid_acceleration.c:694-738
 *   qz_particle_acceleration particle_acceleration source/particle_acceleration.c:522-573
 *   qz_particle_updating_A   particle_updating_A   source/particle_updating.c:2584-2675
 *   qz_particle_updating_B   particle_updating_B   source/particle_updating.c:2787-2837
 *   qz_reset                 reset                 source/reset.c:29-64
 * and the array-level kernels mirror the force_methods/ routines:
 *   qz_gauss_saidel          gauss_saidel          source/force_methods/gauss_saidel.c:29-55
 *   qz_jacobi                jacobi                source/force_methods/jacobi.c:29-82
 *   qz_multigrid             multigrid             source/force_methods/multigrid.c:106-229
 *   qz_ptcl_idx_to_box_idx   ptcl_idx_to_box_idx   source/ptcl_idx_to_box_idx.c:30-139
 */
#ifndef QZ_B200_H
#define QZ_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define QZ_API __attribute__((visibility("default")))
#else
#define QZ_API
#endif

#define QZ_SUCCESS 0
#define QZ_FAILURE 1

/* Smoother ordering of the Gauss-Seidel sweeps. */
#define QZ_GS_REDBLACK 0 /* two-colour sweeps: the fast path */
#define QZ_GS_LEX 1      /* lexicographic order as the reference, by wavefronts */

/* Arithmetic of the head Poisson solve. */
#define QZ_PREC_FP64 0  /* every stage in FP64 (the plain drop-in) */
#define QZ_PREC_MIXED 1 /* FP32 V-cycles inside FP64 defect correction */

/* Head grid fields for qz_get_head_field / qz_set_head_field. */
#define QZ_FIELD_POT 0
#define QZ_FIELD_POT_OLD 1
#define QZ_FIELD_DENSITY 2
#define QZ_FIELD_AX 3
#define QZ_FIELD_AY 4
#define QZ_FIELD_AZ 5

typedef struct qz_config {
    int lmin;           /* head level: 2^lmin cells per side (global_variables.c:252) */
    int lmax;           /* finest level; lmax == lmin is the head-only path */
    double G;           /* gravitational constant (_G_) */
    double total_mass;  /* GL_total_mass_initial: analytic boundary and mean density */
    int bdry;           /* 0 periodic, 1 reflexive (bdry_cond_type) */
    int smoother;       /* 0 Gauss-Seidel, 1 Jacobi, 2 conjugate gradient
                           (solverPreS/PostS/finddphic) */
    int gs_order;       /* QZ_GS_REDBLACK or QZ_GS_LEX */
    int cycle;          /* 0 V, 1 F, 2 W (multigrid_cycle) */
    int n_pre, n_post, n_coarse; /* _NiterPreS_, _NiterPostS_, _Niterfinddphic_ */
    double w_sor;       /* _w_SOR_HEAD_ */
    double tol, tol2;   /* residual and ratio thresholds of poisson_error */
    int check_every;    /* iter_between_check_potential_solution */
    int max_iter;       /* _MAX_NUMBER_OF_ITERATIONS_IN_POISSON_EQUATION_ */
    int check_method;   /* check_poisson_error_method 0/1/2 */
    int precision;      /* QZ_PREC_FP64 or QZ_PREC_MIXED */
    int inner_cycles;   /* mixed precision: FP32 V-cycles per FP64 correction */
    int force_stencil;  /* 0 = 3-point, 1 = 5-point where the cells exist
                           (force_stencil, grid_acceleration.c:694-738) */
    int ref_ptcl;       /* refine a cell holding >= ref_ptcl particles (ref_criterion_ptcl) */
    int box_extra;      /* cells added to a child box on top of its smallest box
                           (min_box_extra_size_per_side_real) */
    /* refinement levels: a node of more than branch_cg_cells cells is solved by
     * conjugate gradient, the others by red-black SOR of branch_sor_sweeps
     * sweeps per check iteration with weight w_sor_branch
     * (branches_maximal_node_number_to_activate_conjugate_gradient,
     * _Iter_branches_solver_, _w_SOR_; potential_branches.c:460-512) */
    int branch_cg_cells;
    int branch_sor_sweeps;
    double w_sor_branch;
    /* time step (timestep.c:589-700): _CFL_, _MAX_dt_, time_step_method
     * (0 velocity only, 1 velocity and acceleration) */
    double cfl;
    double max_dt;
    int time_step_method;
    /* head solve: 0 multigrid cycles, 1 conjugate gradient (head_pot_method,
     * potential_head_node.c:112-176) */
    int head_pot_method;
    /* adjoint Poisson solves (qz_force_vjp, qz_adjoint_final_loss): multigrid
     * cycles until |r| <= adjoint_tol |rhs| (2-norms over the head interior) */
    double adjoint_tol;
    /* refinement-node conjugate gradient: 0 the reference's two reductions per
     * iteration, 1 one reduction per iteration (Chronopoulos-Gear arrangement:
     * the same iterates in exact arithmetic, half the waits), 2 one reduction
     * per iteration in the pipelined arrangement (Ghysels-Vanroose: w = A r
     * by recurrence, one stencil and 12 loads a point) */
    int cg_variant;
    /* persistent multigrid cycles: finest-level points of one colour per thread,
     * which sets the launch's block count (at most two blocks per SM); results
     * do not depend on it (qz_ensemble_autotune picks it for ensembles) */
    int mg_points_per_thread;
    /* refinement tree frozen after its first construction (the differentiation
     * form's fixed tree): later steps keep the nodes and only reassign the
     * particles to them (each level's node of a particle from its parent's box
     * status, as the construction does) instead of rebuilding the tree */
    int freeze_tree;
    /* solver of the refinement nodes: QZ_NODE_CG the reference's node
     * conjugate gradient (FP64; conjugate_gradient.c:322-463), QZ_NODE_MG FP32
     * multigrid V-cycles preconditioning a flexible conjugate gradient in FP64
     * (one thread-block cluster per node); both stop at the reference's
     * convergence test */
    int node_solver;
    /* persistent multigrid cycles: the coarse levels above the single-block
     * sub-cycle in tiled phases (one grid phase for a level's pre-smoothing and
     * restriction, one for its prolongation and post-smoothing; halos
     * recomputed, the fields bit for bit those of the grid phases) where a
     * level's tiles take one round of the launch's blocks.  0: the first tile
     * core of QZ_MG_TILES that fits the shared memory, k >= 1: core k - 1 (if
     * it fits), -1: grid phases only; qz_ensemble_autotune picks it for
     * ensembles */
    int mg_tile;
    /* refinement-node solves start from the previous solve's solution where the
     * previous tree's node of the same index held the point as an interior
     * point (1), instead of the parent interpolation alone as the reference
     * does (0, default): fewer iterations, the same convergence test, results
     * that differ from the reference's by the solve tolerance */
    int node_warm;
    /* refinement steps whose head solve is one persistent launch: 1 (default)
     * runs that launch on a second stream of higher priority while the tree
     * construction and the level deposits, which read only the particles, run
     * on the simulation's stream; the level solves start when both are done.
     * 0 runs the stages one after another in main.c's order.  Results are the
     * same bit for bit either way. */
    int tree_overlap;
    /* refinement-node conjugate gradient: fewest interior points in a chunk
     * (one 512-thread block works a chunk; chunks never cross nodes).  0
     * (default): a level's points are cut into about 148 chunks, one a SM,
     * which suits one simulation on the GPU.  Many simulations side by side
     * (qz_ensemble_step) want larger chunks, e.g. 2048, so that a small
     * member's level takes a few SMs instead of all of them.  The chunks set
     * the order of the dot products' partial sums, so results depend on it at
     * rounding level (deterministically). */
    int cg_chunk_min;
} qz_config;

/* tile cores (x, y, z points) of the tiled multigrid phases, in mg_tile order */
#define QZ_MG_TILES {{8, 4, 4}, {16, 4, 4}, {8, 8, 4}, {16, 8, 4}, {8, 8, 8}, {16, 8, 8}, {4, 4, 4}}
#define QZ_MG_NTILES 7

#define QZ_NODE_CG 0
#define QZ_NODE_MG 1

typedef struct qz_stats {
    long long vcycles_total;   /* V-cycles (FP64 or FP32 inner) since creation */
    int last_vcycles;          /* V-cycles of the last potential solve */
    int last_converged;        /* 1 if the last solve met both thresholds */
    long long kernel_launches; /* kernels this library launched since creation */
    long long steps;           /* completed qz_step steps */
    int error_flags;           /* device-side bounds / sanity flags seen (bit set) */
    long long cg_iterations;   /* refinement-level conjugate-gradient iterations */
    int levels;                /* refinement levels in the current tree (1 = head only) */
    int nodes;                 /* nodes in the current tree, head included */
    double last_dt;            /* step size of the last qz_step step */
    double sim_time;           /* sum of the qz_step step sizes */
    long long adjoint_cycles;  /* multigrid cycles of the adjoint solves */
    long long node_mg_iterations; /* mixed form: defect-correction iterations of the
                                     refinement-level solves (slowest node of each) */
} qz_stats;

/* Result of qz_adjoint_final_loss. */
typedef struct qz_adjoint_stats {
    double loss;               /* (1/N) sum_p |x_T,p - x*_p|^2 */
    double forward_ms;         /* forward pass with checkpoints (device time) */
    double reverse_ms;         /* recomputation and reverse sweep (device time) */
    long long adjoint_cycles;  /* multigrid cycles of the adjoint Poisson solves */
    long long recomputed_steps;/* forward steps run again from checkpoints */
    int checkpoints;           /* stored checkpoints */
    double pool_peak_bytes;    /* high-water mark of the device memory pool during the call */
    double stored_bytes;       /* checkpoints + a segment's states + the final state */
} qz_adjoint_stats;

typedef struct qz_sim qz_sim;

/* Kernel categories of the per-launch profiler (qz_profile_*). */
#define QZ_PROF_SMOOTH 0     /* Gauss-Seidel / Jacobi sweeps */
#define QZ_PROF_RESTRICT 1   /* residual at injected points -> coarse rhs */
#define QZ_PROF_PROLONG 2    /* trilinear prolongation + correction */
#define QZ_PROF_CHECK 3      /* convergence test and pot_old update */
#define QZ_PROF_DEPOSIT 4    /* cell keys, segments, cell sums, point sums */
#define QZ_PROF_SORT 5       /* radix sort and scans of the deposit */
#define QZ_PROF_GRADIENT 6   /* finite-difference grid acceleration */
#define QZ_PROF_GATHER 7     /* CIC force gather */
#define QZ_PROF_LEAPFROG 8   /* kick-drift and kick */
#define QZ_PROF_OTHER 9      /* boundary fill, copies, mixed-precision residual */
#define QZ_PROF_TREE 10      /* refinement tree: counts, flags, zones, children, lists */
#define QZ_PROF_CG 11        /* refinement-node conjugate gradient */
#define QZ_PROF_NODE_MG 12   /* refinement-node FP32 multigrid in FP64 defect correction */
#define QZ_PROF_CATEGORIES 13

/* Configuration with the reference defaults (global_variables.c:300-341). */
QZ_API int qz_default_config(qz_config *cfg, int lmin);

/* Create a simulation for up to n_capacity particles on the current device. */
QZ_API int qz_create(const qz_config *cfg, long n_capacity, qz_sim **out);
QZ_API int qz_destroy(qz_sim *sim);

/* Host <-> device particle state (SoA, float64, length n). */
QZ_API int qz_set_particles(qz_sim *sim, long n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *m);
/* Any output pointer may be NULL; ax/ay/az are the particle accelerations. */
QZ_API int qz_get_particles(qz_sim *sim, double *x, double *y, double *z, double *vx, double *vy,
                     double *vz, double *ax, double *ay, double *az);
/* Sets the particle accelerations (the state the next kick starts from);
 * after it, qz_step does not recompute step-0 forces. */
QZ_API int qz_set_particle_accel(qz_sim *sim, const double *ax, const double *ay, const double *az);
QZ_API long qz_num_particles(const qz_sim *sim);

/* Head grid fields: (2^lmin + 3)^3 float64 values, index i + j*D + k*D*D. */
QZ_API long qz_head_grid_points(const qz_sim *sim);
QZ_API int qz_get_head_field(qz_sim *sim, int which, double *out);
QZ_API int qz_set_head_field(qz_sim *sim, int which, const double *in);

/* Per-stage entry points (device-resident state, stream-ordered). */
QZ_API int qz_initial_potential_head(qz_sim *sim); /* initial_potential_and_acceleration_head.c:30-375 */
QZ_API int qz_reset(qz_sim *sim);
QZ_API int qz_grid_density(qz_sim *sim);
QZ_API int qz_potential(qz_sim *sim);
/* potential.c:29-51 in its two halves: potential_head_node.c:99-179 and
 * potential_branches.c:401-532 (no-op without refinement) */
QZ_API int qz_potential_head_node(qz_sim *sim);
/* Outflow boundaries (bdry 2, particle_updating.c:123-196): the removals of
 * the last qz_particle_updating_A / step, in the reference's visiting order --
 * slots[r] lost its particle and received the one of sources[r] (when the slot
 * is below the new count).  slots / sources may be NULL to read the count. */
QZ_API int qz_outflow_removed(qz_sim *sim, long *count, int *slots, int *sources);
/* The head node's mass (node_mass): total_mass less outflow removals. */
QZ_API double qz_head_mass(const qz_sim *sim);
QZ_API int qz_potential_branches(qz_sim *sim);
QZ_API int qz_grid_acceleration(qz_sim *sim);
QZ_API int qz_particle_acceleration(qz_sim *sim);
QZ_API int qz_particle_updating_A(qz_sim *sim, double dt);
QZ_API int qz_particle_updating_B(qz_sim *sim, double dt);

/* poisson_error.c:290-347 for the head node (type 0): ratio test against
 * pot_old, then the residual test; pot_old <- pot when not converged.
 * *converged receives 1 or 0. */
QZ_API int qz_poisson_error(qz_sim *sim, int *converged);

/* tree_adaptation.c:8250-8590: rebuilds the refinement tree from the current
 * positions with the construction rules of tree_construction.c (no-op when
 * lmax == lmin). */
QZ_API int qz_tree_adaptation(qz_sim *sim);

/* Refinement-tree inspection (levels after the head exist when lmax > lmin).
 * info receives 22 ints: lv, parent, box_ts[3], box_real_dim[3], box_min[3],
 * box_max[3], cells, interior, boundary, sim-boundary grid points, particles,
 * first child, children, touches the simulation boundary. */
QZ_API int qz_amr_levels(qz_sim *sim);
QZ_API int qz_amr_num_nodes(qz_sim *sim, int level);
QZ_API int qz_amr_node_info(qz_sim *sim, int level, int node, int *info, double *mass);
QZ_API int qz_amr_node_cells(qz_sim *sim, int level, int node, int *xyz);
QZ_API int qz_amr_node_box(qz_sim *sim, int level, int node, int *out);
QZ_API int qz_amr_node_list(qz_sim *sim, int level, int node, int which, int *out);
QZ_API int qz_amr_node_field(qz_sim *sim, int level, int node, int which, double *out);

/* Step 0 force computation (main.c:296-338) and whole leapfrog steps
 * (main.c:375-481).  dt > 0: that fixed step; dt <= 0: each step takes the
 * CFL step of qz_timestep from the current state, as main.c:375 does. */
QZ_API int qz_init_forces(qz_sim *sim);
QZ_API int qz_step(qz_sim *sim, double dt, int nsteps);

/* One step (dt > 0) on host-resident state, as the reference's main loop keeps
 * it: x..vz, m and ax..az (length qz_num_particles) are copied in, the step is
 * qz_step's, and x..vz, ax..az are copied back before the call returns.  With
 * page-locked arrays the copies overlap the step (masses in during the
 * kick-drift and tree, positions out during the force computation); with
 * pageable ones they go through the staging buffer before and after it. */
QZ_API int qz_step_host(qz_sim *sim, double dt, double *x, double *y, double *z, double *vx,
                        double *vy, double *vz, const double *m, double *ax, double *ay,
                        double *az);

/* timestep (timestep.c:589-700, headers/timestep.h): the CFL time step of the
 * current velocities and accelerations, each particle with the cell size of its
 * finest node; reduced on the device (exact, order-independent min / max). */
QZ_API int qz_timestep(qz_sim *sim, double *dt);

/* Batching form: nsteps steps of each of nsims independent simulations,
 * member k with step dt[k] (qz_step's meaning; dt NULL: CFL steps for all),
 * stepped concurrently by nthreads host threads on the simulations' own
 * streams.  Each simulation's results equal those of qz_step on it alone.
 * Returns the first failure (with its index in qz_last_error). */
QZ_API int qz_ensemble_step(qz_sim **sims, int nsims, const double *dt, int nsteps,
                            int nthreads);

/* Autotuner of the batching form: times one ensemble step (host wall time to
 * completion) for every combination of host thread count (thread_opts),
 * multigrid points per thread (ppt_opts) and tile core of the tiled multigrid
 * phases (tile_opts: mg_tile values), restoring every simulation's state
 * (particles, accelerations, head potential, statistics) after each trial;
 * sets every simulation's mg_points_per_thread and mg_tile to the best
 * combination's and writes the best thread count, points per thread, tile and
 * step time (best_tile may be NULL).  The simulations are left as they were
 * (their results do not depend on the choice). */
QZ_API int qz_ensemble_autotune(qz_sim **sims, int nsims, const double *dt,
                                const int *thread_opts, int nthread_opts, const int *ppt_opts,
                                int nppt_opts, const int *tile_opts, int ntile_opts,
                                int *best_threads, int *best_ppt, int *best_tile,
                                double *best_ms);

/* Differentiation form (no reference counterpart: QUANTIZER has no adjoint).
 * FP64 runs with the 3-point stencil, reflexive walls and the multigrid head
 * solve, head-only or with refinement levels on a frozen tree (freeze_tree:
 * the node solves, parent averages, level deposits and finest-level gathers
 * are differentiated with the tree held fixed).  The force F(x, m) = gather(-grad Lap^-1 deposit(x, m))
 * of grid_density.c:35-111, potential_head_node.c:99-179,
 * grid_acceleration.c:36-76 and particle_acceleration.c:33-132 is
 * differentiated with the Poisson solve taken as exact (its adjoint is a
 * second solve with zero boundary, to adjoint_tol) and the shell boundary
 * linear in total_mass (which is taken as the sum of the masses).
 *
 * qz_force_vjp: for host a-bar (n each) at the current state (forces computed),
 * writes gx..gz = (dF/dx)^T abar and gm = (dF/dm)^T abar (host, n each).
 *
 * qz_adjoint_final_loss: from the current state (x0, v0, a0 = F(x0)), runs
 * nsteps fixed-dt steps (particle_updating.c:39-207, 2677-2688) with a
 * checkpoint every checkpoint_every steps (<= 0: one segment), then the
 * reverse sweep, recomputing each earlier segment from its checkpoint.
 * Writes the gradients of L = (1/N) sum_p |x_T,p - x*_p|^2 (targets tx..tz)
 * with respect to the initial positions, velocities and masses (host, n each)
 * and, when st is not NULL, the loss and timings.  The simulation is left at
 * the final state, as after qz_step(sim, dt, nsteps). */
QZ_API int qz_force_vjp(qz_sim *sim, const double *abx, const double *aby, const double *abz,
                        double *gx, double *gy, double *gz, double *gm);
QZ_API int qz_adjoint_final_loss(qz_sim *sim, int nsteps, double dt, int checkpoint_every,
                                 const double *tx, const double *ty, const double *tz,
                                 double *gx, double *gy, double *gz, double *gvx, double *gvy,
                                 double *gvz, double *gm, qz_adjoint_stats *st);

/* Snapshot file of output_snapshots.c:141-239 from the device-resident state:
 * m[N], x, y, z, vx, vy, vz in user units ((x - 0.5) / conversion_dist + cm_x
 * + cm_vx * real_time; vx / conversion_velocity + cm_vx), then, when
 * observables_type is 0 or 1, energies[3] and momentum[3] of qz_observables
 * with that potential type, then real_time = actual_time / conversion_time
 * (float64, native byte order).  units: {conversion_dist, conversion_velocity,
 * conversion_time, cm_x, cm_y, cm_z, cm_vx, cm_vy, cm_vz}, NULL for 1, 1, 1
 * and zeros; observables_type -1: none.  async != 0: the copy to the host and
 * the file write run behind the simulation's stream (the state may be stepped
 * at once); qz_snapshot_wait joins the write and reports its result (so does
 * the next qz_write_snapshot and qz_destroy). */
QZ_API int qz_write_snapshot(qz_sim *sim, const char *path, double actual_time,
                             const double *units, int observables_type, int async);
QZ_API int qz_snapshot_wait(qz_sim *sim);

/* observables (observables.c:661-696): out[0] kinetic, out[1] potential,
 * out[2] total energy, out[3..5] momentum.  potential_type 0: exact sum over
 * particle pairs (O(N^2), potential_energy_exact :77-112); 1: from the
 * potential grid at each particle's finest node (:590-618).  units: NULL for
 * code units, else {_conversion_velocity_, _conversion_time_,
 * _conversion_dist_, GL_cm_vx, GL_cm_vy, GL_cm_vz}.  FP64 sums in fixed
 * order (reproducible; equal to the reference's to rounding). */
QZ_API int qz_observables(qz_sim *sim, int potential_type, const double *units, double *out);

/* Solver schedule, for finite-difference checks of the adjoint.  A forward
 * Poisson solve normally stops at the reference's convergence test, so runs
 * from slightly different inputs can stop after different iteration counts and
 * the map from inputs to outputs jumps.  mode 1 starts recording the count of
 * every forward solve (the head: its cycles; a refinement level: one count per
 * node); mode 0 stops and copies up to cap counts to counts (*len = how many
 * were recorded); mode 2 replays counts[0..cap): every forward solve runs
 * exactly its recorded count with no convergence test, in the recorded order
 * (a run with more solves than recorded fails). */
QZ_API int qz_solve_schedule(qz_sim *sim, int mode, int *counts, long cap, long *len);

/* Synchronise the library stream and report statistics. */
QZ_API int qz_synchronize(qz_sim *sim);
QZ_API int qz_get_stats(qz_sim *sim, qz_stats *out);
/* The cudaStream_t the library launches on (for event timing by callers). */
QZ_API void *qz_stream(qz_sim *sim);
QZ_API const char *qz_last_error(void);

/* Per-launch profiler: when enabled, every kernel launch is bracketed by CUDA
 * events on the library stream and booked to its category with the
 * algorithmic bytes it must move.  qz_profile_read synchronises and returns
 * the category's launches, summed device time (ms) and algorithmic bytes. */
QZ_API int qz_profile_enable(qz_sim *sim, int on);
QZ_API int qz_profile_reset(qz_sim *sim);
QZ_API int qz_profile_read(qz_sim *sim, int category, long long *launches, double *total_ms,
                           double *bytes);

/* Array-level kernels on host arrays of gridsize^3 float64 values (copied to
 * the device and back), the reference's force_methods signatures plus the
 * parameters the reference reads from globals. */
QZ_API int qz_gauss_saidel(double *phi, const double *rho, int gridsize, int iter_max, double w,
                    int gs_order);
QZ_API int qz_jacobi(double *phi, const double *rho, int gridsize, int iter_max, double w);
/* conjugate_gradient_multigrid (force_methods/conjugate_gradient_multigrid.c:29-176):
 * iters conjugate-gradient iterations as a smoother, early exit below a
 * residual ratio of 1e-16; FP64 sums in block order (tolerance parity). */
QZ_API int qz_conjugate_gradient_multigrid(double *phi, const double *rho, int gridsize, int iters);
QZ_API int qz_multigrid(const qz_config *cfg, double *phi, const double *rho, int gridsize,
                 int type_multigrid);

/* Weighted Jacobi smoothing (the sweeps of jacobi above) on DEVICE arrays the
 * caller owns, that allocates no device memory: no cudaMalloc, no cudaFree, no
 * allocating library routine.  No counterpart in the reference, whose jacobi
 * mallocs its ping-pong copy on every call.  It is for callers that cannot
 * allocate: code that runs inside a host framework whose caching allocator or
 * memory pool already owns the device memory budget (a raw cudaMalloc there can
 * fail or fragment the pool), and loops that must not allocate once running,
 * because cudaMalloc and cudaFree synchronise the whole device and stall every
 * other stream.  The ping-pong copy lives in a fixed device array inside the
 * library, of QZ_NOALLOC_MAX_GRID^3 doubles (2.2 MB), which every GPU that
 * loads the library holds until the process exits; gridsize above
 * QZ_NOALLOC_MAX_GRID is rejected with an error.  phi (in/out) and rho are
 * gridsize^3 float64 device arrays; stream is a cudaStream_t (NULL for the
 * default stream); the call only enqueues work on it.  Every call looks up the
 * array's device address on the current device; the first call on a device
 * also loads the library's kernels there (make that first call before any
 * stream capture).  All calls share the array, which keeps the last call's
 * contents (each call starts by copying phi into it); calls that overlap on
 * the GPU race on it, so serialise them. */
#define QZ_NOALLOC_MAX_GRID 65
QZ_API int qz_jacobi_noalloc(double *phi, const double *rho, int gridsize, int iter_max,
                             double w, void *stream);

/* conjugate_gradient (force_methods/conjugate_gradient.c:322-463) on one node
 * given as HOST arrays, the fields of the reference's struct node: level lv,
 * box_real_dim, the interior list ptr_intr_box_grid_idx (grid_intr_size
 * entries), node_mass, cell_size, and the grid fields d, pot, pot_old of
 * (box_real_dim + 1)^3 points.  Solved by the device's node conjugate gradient
 * (same iterates, checks every check_every iterations with poisson_error's
 * tests, the reference's iteration cap); pot is overwritten with the solution
 * and pot_old as poisson_error leaves it.  QZ_FAILURE when the precision is
 * not reached, with the reference's message. */
QZ_API int qz_node_conjugate_gradient(qz_sim *sim, int lv, int box_real_dim_x, int box_real_dim_y,
                                      int box_real_dim_z, int grid_intr_size,
                                      const int *intr_box_grid_idx, double node_mass, int cell_size,
                                      const double *d, double *pot, double *pot_old);

/* Batched ptcl_idx_to_box_idx for one non-periodic node geometry. */
QZ_API int qz_ptcl_idx_to_box_idx(int lv, int box_ts_x, int box_ts_y, int box_ts_z,
                           int box_real_dim_x, int box_real_dim_y, long n, const double *x,
                           const double *y, const double *z, int *out);

/* Test hooks (no counterpart in the reference; used by the library's own tests).
 * qz_test_scan: the device's single-pass exclusive scan of n ints (host arrays
 * in / out; in_place scans one device buffer into itself; epoch != 0 first sets
 * the scan epoch counter, so that a test can run across its wrap).
 * qz_test_wait_gives_up: runs one bounded device wait that nothing satisfies
 * and returns what the library returns then (QZ_FAILURE and the message):
 * which 0 the scan's look-back on a tile that is never published, which 1 the
 * cooperative kernels' grid barrier (out2[0], out2[1]: 1 if the first / second
 * barrier of the probe returned true).  Each wait ends at its poll limit. */
QZ_API int qz_test_scan(qz_sim *sim, const int *in, int *out, long n, int in_place,
                        unsigned epoch);
QZ_API int qz_test_wait_gives_up(qz_sim *sim, int which, int *out2);

#ifdef __cplusplus
}
#endif
#endif

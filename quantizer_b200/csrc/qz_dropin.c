/*
 * qz_dropin.c -- libqz_dropin.so: the reference's hot-path symbols
 * (include/qz_dropin.h) implemented on libqzb200's device pipeline.
 *
 * At the first call the shim finds the reference's globals in the host
 * program (dlsym on the running image), creates a qz_sim from the parameters
 * the reference's global_variables() set, and uploads the particle arrays and
 * the head node's grid fields.  Afterwards the device copy is authoritative:
 * each entry point runs on the device and writes the arrays it changed back
 * to the host globals before returning (write-through), so host code that
 * reads them (timestep, observables, snapshots) always sees current values.
 *
 * Refinement runs (lmax > lmin): the tree bookkeeping stays in the reference's
 * C (tree_adaptation and the rest of its bookkeeping objects) and the host
 * particle arrays are authoritative for x and v: grid_density, timestep,
 * observables and particle_updating_A upload them first.  particle_updating_A
 * advances every particle on the device (kick, drift, reflection at the
 * walls) and the shim then applies the moves between the host tree's cell
 * lists that the reference makes in its cell loops (particle_updating.c:
 * 634-1381): same cell, another cell of the node, a child zone, the parent or
 * a sibling node, with the nodes' masses and particle counts.  The density,
 * potentials, grid and particle accelerations are computed on the device on
 * its own copy of the tree (built from the same rules, tree_construction.c;
 * its refined cells equal the reference's adapted tree); particle
 * accelerations and the head node's fields are written back, refinement
 * nodes' grid fields are not.
 *
 * Supported: reflexive boundaries, one smoother for all multigrid stages or
 * the head conjugate gradient, the particle refinement criterion with n_exp
 * = 1.  Other configurations are rejected with the reference's error
 * convention (message + _FAILURE_).
 *
 * Environment: QZ_GS_ORDER=lex selects the reference's lexicographic
 * Gauss-Seidel order for the head solve (default red-black);
 * QZ_PRECISION=mixed selects FP32 cycles inside FP64 defect correction.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/qz_b200.h"
#include "../../include/qz_dropin.h"
#include "qz_ref_abi.h"

#define REF_SUCCESS 0
#define REF_FAILURE 1

/* The reference's globals the hot path reads (headers/common.h:105-260). */
static struct {
    double **ptcl_mass, **ptcl_x, **ptcl_y, **ptcl_z, **ptcl_vx, **ptcl_vy, **ptcl_vz;
    double **ptcl_ax, **ptcl_ay, **ptcl_az;
    int *no_ptcl_final, *no_ptcl_initial, *lmin, *lmax, *bdry_cond_type;
    double *G, *total_mass_initial;
    struct node **ptr_tree;
    int *niter_pre, *niter_post, *niter_coarse, *solver_pre, *solver_post, *solver_coarse;
    int *cycle, *check_every, *max_iter, *check_method, *head_pot_method, *force_stencil;
    int *branch_cg_cells, *branch_sweeps;
    double *w_sor_branch, *cfl, *max_dt;
    double *conv_velocity, *conv_time, *conv_dist, *cm_vx, *cm_vy, *cm_vz;
    double **energies, **momentum;
    int *pe_type;
    int *time_step_method;
    double *w_sor_head, *tol, *tol2;
    int *ref_ptcl, *n_exp, *box_extra;
    double *ref_mass;
    int **ptcl_id;
    double *total_mass_final;
    /* the tree by levels and the particles' update flags (refinement runs) */
    struct node ****tentacles;
    int **tentacles_size;
    int *tentacles_level_max;
    bool **updating_flag;
    int (*space_check)(int *, int, float, const char *, ...);
    int resolved;
} R;

static qz_sim *g_sim = NULL;
static int g_failed = 0;
static int g_amr = 0; /* refinement run: host x, v authoritative */

static void *need(const char *name, int *ok)
{
    void *p = dlsym(RTLD_DEFAULT, name);
    if (!p)
    {
        printf("\nERROR (drop-in): the host program does not export the global '%s' "
               "(link it with -Wl,--export-dynamic)\n", name);
        *ok = 0;
    }
    return p;
}

static int resolve(void)
{
    if (R.resolved)
        return 1;
    int ok = 1;
    R.ptcl_mass = need("GL_ptcl_mass", &ok);
    R.ptcl_x = need("GL_ptcl_x", &ok);
    R.ptcl_y = need("GL_ptcl_y", &ok);
    R.ptcl_z = need("GL_ptcl_z", &ok);
    R.ptcl_vx = need("GL_ptcl_vx", &ok);
    R.ptcl_vy = need("GL_ptcl_vy", &ok);
    R.ptcl_vz = need("GL_ptcl_vz", &ok);
    R.ptcl_ax = need("GL_ptcl_ax", &ok);
    R.ptcl_ay = need("GL_ptcl_ay", &ok);
    R.ptcl_az = need("GL_ptcl_az", &ok);
    R.no_ptcl_final = need("GL_no_ptcl_final", &ok);
    R.no_ptcl_initial = need("GL_no_ptcl_initial", &ok);
    R.lmin = need("lmin", &ok);
    R.lmax = need("lmax", &ok);
    R.bdry_cond_type = need("bdry_cond_type", &ok);
    R.G = need("_G_", &ok);
    R.total_mass_initial = need("GL_total_mass_initial", &ok);
    R.ptr_tree = need("GL_ptr_tree", &ok);
    R.niter_pre = need("_NiterPreS_", &ok);
    R.niter_post = need("_NiterPostS_", &ok);
    R.niter_coarse = need("_Niterfinddphic_", &ok);
    R.solver_pre = need("solverPreS", &ok);
    R.solver_post = need("solverPostS", &ok);
    R.solver_coarse = need("solverfinddphic", &ok);
    R.cycle = need("multigrid_cycle", &ok);
    R.check_every = need("iter_between_check_potential_solution", &ok);
    R.max_iter = need("_MAX_NUMBER_OF_ITERATIONS_IN_POISSON_EQUATION_", &ok);
    R.check_method = need("check_poisson_error_method", &ok);
    R.head_pot_method = need("head_pot_method", &ok);
    R.force_stencil = need("force_stencil", &ok);
    R.branch_cg_cells = need("branches_maximal_node_number_to_activate_conjugate_gradient", &ok);
    R.branch_sweeps = need("_Iter_branches_solver_", &ok);
    R.w_sor_branch = need("_w_SOR_", &ok);
    R.cfl = need("_CFL_", &ok);
    R.max_dt = need("_MAX_dt_", &ok);
    R.time_step_method = need("time_step_method", &ok);
    R.conv_velocity = need("_conversion_velocity_", &ok);
    R.conv_time = need("_conversion_time_", &ok);
    R.conv_dist = need("_conversion_dist_", &ok);
    R.cm_vx = need("GL_cm_vx", &ok);
    R.cm_vy = need("GL_cm_vy", &ok);
    R.cm_vz = need("GL_cm_vz", &ok);
    R.energies = need("GL_energies", &ok);
    R.momentum = need("GL_momentum", &ok);
    R.pe_type = need("potential_energy_type", &ok);
    R.w_sor_head = need("_w_SOR_HEAD_", &ok);
    R.tol = need("_ERROR_THRESHOLD_IN_THE_POISSON_EQUATION_", &ok);
    R.tol2 = need("_ERROR_THRESHOLD_IN_THE_POISSON_EQUATION_2", &ok);
    R.ref_ptcl = need("ref_criterion_ptcl", &ok);
    R.ref_mass = need("ref_criterion_mass", &ok);
    R.n_exp = need("n_exp", &ok);
    R.box_extra = need("min_box_extra_size_per_side_real", &ok);
    R.ptcl_id = need("GL_ptcl_ID", &ok);
    R.total_mass_final = need("GL_total_mass_final", &ok);
    R.tentacles = need("GL_tentacles", &ok);
    R.tentacles_size = need("GL_tentacles_size", &ok);
    R.tentacles_level_max = need("GL_tentacles_level_max", &ok);
    R.updating_flag = need("GL_ptcl_updating_flag", &ok);
    *(void **)&R.space_check = need("space_check", &ok);
    R.resolved = ok;
    return ok;
}

static void fill_config(qz_config *c)
{
    qz_default_config(c, *R.lmin);
    c->lmax = *R.lmax;
    c->G = *R.G;
    c->total_mass = *R.total_mass_initial;
    c->bdry = *R.bdry_cond_type;
    c->smoother = *R.solver_pre;
    c->cycle = *R.cycle;
    c->n_pre = *R.niter_pre;
    c->n_post = *R.niter_post;
    c->n_coarse = *R.niter_coarse;
    c->w_sor = *R.w_sor_head;
    c->tol = *R.tol;
    c->tol2 = *R.tol2;
    c->check_every = *R.check_every;
    c->max_iter = *R.max_iter;
    c->check_method = *R.check_method;
    c->force_stencil = *R.force_stencil;
    c->branch_cg_cells = *R.branch_cg_cells;
    c->branch_sor_sweeps = *R.branch_sweeps;
    c->w_sor_branch = *R.w_sor_branch;
    c->cfl = *R.cfl;
    c->max_dt = *R.max_dt;
    c->time_step_method = *R.time_step_method;
    c->head_pot_method = *R.head_pot_method;
    c->ref_ptcl = *R.ref_ptcl;
    c->box_extra = *R.box_extra;
    const char *o = getenv("QZ_GS_ORDER");
    c->gs_order = (o && !strcmp(o, "lex")) ? QZ_GS_LEX : QZ_GS_REDBLACK;
    const char *p = getenv("QZ_PRECISION");
    c->precision = (p && !strcmp(p, "mixed")) ? QZ_PREC_MIXED : QZ_PREC_FP64;
}

static int fail(const char *what)
{
    printf("\nERROR (drop-in): %s: %s\n", what, qz_last_error());
    g_failed = 1;
    return REF_FAILURE;
}

static int upload_all(void)
{
    struct node *h = *R.ptr_tree;
    long n = *R.no_ptcl_final;
    if (qz_set_particles(g_sim, n, *R.ptcl_x, *R.ptcl_y, *R.ptcl_z, *R.ptcl_vx, *R.ptcl_vy,
                         *R.ptcl_vz, *R.ptcl_mass) ||
        qz_set_particle_accel(g_sim, *R.ptcl_ax, *R.ptcl_ay, *R.ptcl_az) ||
        qz_set_head_field(g_sim, QZ_FIELD_POT, h->ptr_pot) ||
        qz_set_head_field(g_sim, QZ_FIELD_POT_OLD, h->ptr_pot_old) ||
        qz_set_head_field(g_sim, QZ_FIELD_DENSITY, h->ptr_d) ||
        qz_set_head_field(g_sim, QZ_FIELD_AX, h->ptr_ax) ||
        qz_set_head_field(g_sim, QZ_FIELD_AY, h->ptr_ay) ||
        qz_set_head_field(g_sim, QZ_FIELD_AZ, h->ptr_az))
        return fail("upload of the host state");
    return REF_SUCCESS;
}

/* Creates the device context on first use. */
static int ensure(void)
{
    if (g_sim)
        return REF_SUCCESS;
    if (g_failed)
        return REF_FAILURE;
    if (!resolve())
    {
        g_failed = 1;
        return REF_FAILURE;
    }
    g_amr = *R.lmax > *R.lmin;
    if (g_amr && (*R.n_exp != 1 || *R.ref_mass < 1.0e99 || *R.bdry_cond_type != 1))
    {
        printf("\nERROR (drop-in): refinement runs need n_exp = 1, the particle criterion "
               "only (ref_criterion_mass off) and reflexive boundaries\n");
        g_failed = 1;
        return REF_FAILURE;
    }
    if (*R.head_pot_method < 0 || *R.head_pot_method > 1 || *R.solver_pre != *R.solver_post ||
        *R.solver_pre != *R.solver_coarse || *R.solver_pre > 2)
    {
        printf("\nERROR (drop-in): head solver configuration not supported "
               "(multigrid with one smoother for all stages, or conjugate gradient)\n");
        g_failed = 1;
        return REF_FAILURE;
    }
    qz_config c;
    fill_config(&c);
    if (qz_create(&c, *R.no_ptcl_initial, &g_sim))
    {
        g_sim = NULL;
        return fail("device context");
    }
    return upload_all();
}

/* Refinement runs: x, v (and m) from the host arrays, which the reference's
 * particle_updating moved; with_accel also the accelerations. */
static int sync_host_particles(int with_accel)
{
    if (!g_amr)
        return REF_SUCCESS;
    if (qz_set_particles(g_sim, *R.no_ptcl_final, *R.ptcl_x, *R.ptcl_y, *R.ptcl_z, *R.ptcl_vx,
                         *R.ptcl_vy, *R.ptcl_vz, *R.ptcl_mass) ||
        (with_accel && qz_set_particle_accel(g_sim, *R.ptcl_ax, *R.ptcl_ay, *R.ptcl_az)))
        return fail("upload of the host particles");
    return REF_SUCCESS;
}

static int head_field_back(int which, double *dst)
{
    if (qz_get_head_field(g_sim, which, dst))
        return fail("head field read-back");
    return REF_SUCCESS;
}

/* grid_density.c:269-306 */
void grid_density(void)
{
    if (ensure() || sync_host_particles(0))
        return;
    if ((g_amr && qz_tree_adaptation(g_sim)) || qz_grid_density(g_sim))
    {
        fail("grid_density");
        return;
    }
    head_field_back(QZ_FIELD_DENSITY, (*R.ptr_tree)->ptr_d);
}

/* potential_head_node.c:99-179 */
int potential_head_node(void)
{
    if (ensure())
        return REF_FAILURE;
    if (qz_potential_head_node(g_sim))
    {
        printf("\n\n Error running potential_head_node() function \n\n ");
        return fail("potential_head_node");
    }
    struct node *h = *R.ptr_tree;
    if (head_field_back(QZ_FIELD_POT, h->ptr_pot) || head_field_back(QZ_FIELD_POT_OLD, h->ptr_pot_old))
        return REF_FAILURE;
    return REF_SUCCESS;
}

/* potential_branches.c:401-532: the refinement levels' solves (none without
 * refinement). */
int potential_branches(void)
{
    if (ensure())
        return REF_FAILURE;
    if (qz_potential_branches(g_sim))
        return fail("potential_branches");
    return REF_SUCCESS;
}

/* potential.c:29-51 */
int potential(void)
{
    if (potential_head_node())
        return REF_FAILURE;
    if (*R.lmin < *R.lmax && potential_branches())
        return REF_FAILURE;
    return REF_SUCCESS;
}

/* grid_acceleration.c:694-738 */
int grid_acceleration(void)
{
    if (ensure())
        return REF_FAILURE;
    if (qz_grid_acceleration(g_sim))
        return fail("grid_acceleration");
    struct node *h = *R.ptr_tree;
    if (head_field_back(QZ_FIELD_AX, h->ptr_ax) || head_field_back(QZ_FIELD_AY, h->ptr_ay) ||
        head_field_back(QZ_FIELD_AZ, h->ptr_az))
        return REF_FAILURE;
    return REF_SUCCESS;
}

/* timestep.c:589-700: the CFL step of the current state, reduced on the device */
int timestep(double *ptr_dt)
{
    if (ensure() || sync_host_particles(1))
        return REF_FAILURE;
    if (qz_timestep(g_sim, ptr_dt))
        return fail("timestep");
    return REF_SUCCESS;
}

/* observables.c:661-696: energies into GL_energies, momentum into GL_momentum */
int observables(void)
{
    if (ensure() || sync_host_particles(1))
        return REF_FAILURE;
    const double units[6] = {*R.conv_velocity, *R.conv_time, *R.conv_dist,
                             *R.cm_vx, *R.cm_vy, *R.cm_vz};
    double out[6];
    if (*R.pe_type != 0 && *R.pe_type != 1)
    {
        printf("Error, the potential_energy_type value is different of 0 or 1\n");
        return REF_FAILURE;
    }
    if (qz_observables(g_sim, *R.pe_type, units, out))
        return fail("observables");
    for (int k = 0; k < 3; k++)
    {
        (*R.energies)[k] = out[k];
        (*R.momentum)[k] = out[3 + k];
    }
    return REF_SUCCESS;
}

/* particle_acceleration.c:522-573 */
int particle_acceleration(void)
{
    if (ensure())
        return REF_FAILURE;
    if (qz_particle_acceleration(g_sim) ||
        qz_get_particles(g_sim, NULL, NULL, NULL, NULL, NULL, NULL, *R.ptcl_ax, *R.ptcl_ay,
                         *R.ptcl_az))
        return fail("particle_acceleration");
    return REF_SUCCESS;
}

/* Appends particle p to cell b of node nd (the host tree's cell list), with
 * the cell's mass; capacity grows through the reference's space_check, as its
 * own appends do. */
static int cell_append(struct node *nd, int b, int p, double m)
{
    struct cell_struct *c = &nd->ptr_cell_struct[b];
    if (R.space_check(&c->ptcl_cap, c->ptcl_size + 1, 1.0f, "p1i1", &c->ptr_ptcl) == REF_FAILURE)
    {
        printf("Error, in space_check function\n");
        return REF_FAILURE;
    }
    c->ptr_ptcl[c->ptcl_size++] = p;
    c->cell_mass += m;
    return REF_SUCCESS;
}

/* The moves between the host tree's cell lists after the device advanced the
 * particles (reflexive boundaries; particle_updating.c:634-1381).  Nodes are
 * visited from the finest level to the head, cells in each node's cell order,
 * particles in list order; a visited particle takes the pass's update flag
 * and is not moved twice.  A particle whose box cell in its node changed goes
 *   into a refined cell (status >= 0):  the child zone's node, its cell there;
 *   outside the node (status -4):       the parent's cell there, or the
 *                                       sibling node whose zone holds it;
 *   anywhere else:                      its new cell of the node;
 * and leaves its old cell by taking the list's last entry into its place.
 * Node masses and particle counts follow the particle across nodes. */
static int apply_cell_moves(void)
{
    const double *mass = *R.ptcl_mass;
    bool *flag = *R.updating_flag;
    const bool status = !flag[0];
    struct node ***tent = *R.tentacles;
    const int *tsize = *R.tentacles_size;
    for (int lv = *R.tentacles_level_max; lv >= 0; lv--)
        for (int i = 0; i < tsize[lv]; i++)
        {
            struct node *nd = tent[lv][i];
            for (int c = 0; c < nd->cell_size; c++)
            {
                const int bo = nd->ptr_box_idx[c];
                if (nd->chn_size > 0 && nd->ptr_box[bo] >= 0)
                    continue; /* a refined cell: its particles belong to the child */
                struct cell_struct *cs = &nd->ptr_cell_struct[bo];
                int np = cs->ptcl_size;
                for (int j = 0; j < np; j++)
                {
                    const int p = cs->ptr_ptcl[j];
                    if (flag[p] == status)
                        continue;
                    flag[p] = status;
                    const int bn = ptcl_idx_to_box_idx(nd, p);
                    if (bn == bo)
                        continue;
                    const double m = mass[p];
                    const int st = nd->ptr_box[bn];
                    if (nd->chn_size > 0 && st >= 0)
                    {
                        struct node *ch = nd->pptr_chn[st];
                        if (cell_append(ch, ptcl_idx_to_box_idx(ch, p), p, m))
                            return REF_FAILURE;
                        ch->node_mass += m;
                        ch->no_ptcl_full_node++;
                    }
                    else if (st == -4)
                    {
                        struct node *pt = nd->ptr_pt;
                        const int bp = ptcl_idx_to_box_idx(pt, p);
                        if (pt->ptr_box[bp] >= 0)
                        {
                            struct node *sib = pt->pptr_chn[pt->ptr_box[bp]];
                            if (cell_append(sib, ptcl_idx_to_box_idx(sib, p), p, m))
                                return REF_FAILURE;
                            sib->node_mass += m;
                            sib->no_ptcl_full_node++;
                        }
                        else if (cell_append(pt, bp, p, m))
                            return REF_FAILURE;
                        nd->node_mass -= m;
                        nd->no_ptcl_full_node--;
                    }
                    else if (cell_append(nd, bn, p, m))
                        return REF_FAILURE;
                    cs->ptr_ptcl[j] = cs->ptr_ptcl[np - 1];
                    np--;
                    j--;
                    cs->cell_mass -= m;
                }
                cs->ptcl_size = np;
            }
        }
    return REF_SUCCESS;
}

/* Outflow removals of the last update, applied to the host's bookkeeping in
 * the reference's order (particle_updating.c:164-176): total and head masses,
 * counts, and the IDs, which move with the particles (the masses do not). */
static int apply_removals(void)
{
    long cnt = 0;
    if (qz_outflow_removed(g_sim, &cnt, NULL, NULL))
        return fail("outflow removals");
    if (cnt == 0)
        return REF_SUCCESS;
    int *slots = (int *)malloc(cnt * sizeof(int)), *srcs = (int *)malloc(cnt * sizeof(int));
    if (!slots || !srcs || qz_outflow_removed(g_sim, &cnt, slots, srcs))
    {
        free(slots);
        free(srcs);
        return fail("outflow removals");
    }
    struct node *h = *R.ptr_tree;
    for (long r = 0; r < cnt; r++)
    {
        const double m = (*R.ptcl_mass)[slots[r]];
        *R.total_mass_final -= m;
        (*R.no_ptcl_final)--;
        h->node_mass -= m;
        h->no_ptcl_full_node--;
        (*R.ptcl_id)[slots[r]] = (*R.ptcl_id)[srcs[r]];
    }
    free(slots);
    free(srcs);
    if (*R.no_ptcl_final == 0)
    {
        printf("Error, There are no particles in the simulation\n");
        return REF_FAILURE;
    }
    return REF_SUCCESS;
}

/* particle_updating.c:2584-2675 */
int particle_updating_A(double dt)
{
    if (ensure())
        return REF_FAILURE;
    if (g_amr)
    {
        /* the host arrays are authoritative: advance them on the device, bring
         * x, v and a (negated on reflection) back, then move the particles
         * between the host tree's cell lists */
        if (sync_host_particles(1) || qz_particle_updating_A(g_sim, dt) ||
            qz_get_particles(g_sim, *R.ptcl_x, *R.ptcl_y, *R.ptcl_z, *R.ptcl_vx, *R.ptcl_vy,
                             *R.ptcl_vz, *R.ptcl_ax, *R.ptcl_ay, *R.ptcl_az))
            return fail("particle_updating_A");
        return apply_cell_moves();
    }
    if (qz_particle_updating_A(g_sim, dt) || apply_removals() ||
        qz_get_particles(g_sim, *R.ptcl_x, *R.ptcl_y, *R.ptcl_z, *R.ptcl_vx, *R.ptcl_vy,
                         *R.ptcl_vz, *R.ptcl_ax, *R.ptcl_ay, *R.ptcl_az))
        return fail("particle_updating_A");
    return REF_SUCCESS;
}

/* particle_updating.c:2787-2837 */
void particle_updating_B(double dt)
{
    if (ensure())
        return;
    /* every particle's half kick (refinement runs: the reference kicks each
     * particle once, in the cell list of its finest node, particle_updating.c:
     * 2690-2785); the device's v and a are current (grid_density uploaded v,
     * particle_acceleration computed a) */
    if (qz_particle_updating_B(g_sim, dt) ||
        qz_get_particles(g_sim, NULL, NULL, NULL, *R.ptcl_vx, *R.ptcl_vy, *R.ptcl_vz, NULL, NULL,
                         NULL))
        fail("particle_updating_B");
}

/* reset.c:29-64: the host copies are zeroed with the device copies. */
int reset(void)
{
    if (ensure())
        return REF_FAILURE;
    if (qz_reset(g_sim))
        return fail("reset");
    long n = *R.no_ptcl_final;
    memset(*R.ptcl_ax, 0, n * sizeof(double));
    memset(*R.ptcl_ay, 0, n * sizeof(double));
    memset(*R.ptcl_az, 0, n * sizeof(double));
    struct node *h = *R.ptr_tree;
    memset(h->ptr_d, 0, (size_t)qz_head_grid_points(g_sim) * sizeof(double));
    return REF_SUCCESS;
}

/* ptcl_idx_to_box_idx.c:30-139.  The scalar form answers a host caller about
 * one host-resident particle (the reference's tree bookkeeping calls it per
 * particle), so it is evaluated in place with the reference's integer
 * arithmetic; batches go through qz_ptcl_idx_to_box_idx on the device. */
int ptcl_idx_to_box_idx(struct node *p, int i)
{
    if (!resolve())
        return 0;
    const int lv = p->lv;
    const double X = (*R.ptcl_x)[i], Y = (*R.ptcl_y)[i], Z = (*R.ptcl_z)[i];
    const double px = X * (1 << lv), py = Y * (1 << lv), pz = Z * (1 << lv);
    const int fx = px < 0 ? -1 : (int)px, fy = py < 0 ? -1 : (int)py, fz = pz < 0 ? -1 : (int)pz;
    int bx = fx - p->box_ts_x, by = fy - p->box_ts_y, bz = fz - p->box_ts_z;
    if (p->pbc_crosses_sim_box_bdry)
    {
        /* periodic nodes that straddle or span the box (ptcl_idx_to_box_idx.c:69-131) */
        const bool whole[3] = {p->pbc_crosses_whole_sim_box_x, p->pbc_crosses_whole_sim_box_y,
                               p->pbc_crosses_whole_sim_box_z};
        const bool cross[3] = {p->pbc_crosses_sim_box_bdry_x, p->pbc_crosses_sim_box_bdry_y,
                               p->pbc_crosses_sim_box_bdry_z};
        const int f[3] = {fx, fy, fz}, mx[3] = {p->box_max_x, p->box_max_y, p->box_max_z};
        const double q[3] = {X, Y, Z};
        int *b[3] = {&bx, &by, &bz};
        for (int c = 0; c < 3; c++)
        {
            if (!whole[c])
            {
                if (cross[c] && f[c] > mx[c] + 1)
                    *b[c] -= (1 << lv);
            }
            else if (q[c] < 0.)
                *b[c] += (1 << lv);
            else if (q[c] >= 1.)
                *b[c] -= (1 << lv);
        }
    }
    return bx + by * p->box_real_dim_x + bz * p->box_real_dim_x * p->box_real_dim_y;
}

/* poisson_error.c:290-347 for the head node (the only node of this build). */
bool poisson_error(struct node *p, double *error, double error_total_pow2, int type)
{
    (void)error;
    (void)error_total_pow2;
    if (ensure())
        return false;
    if (p != *R.ptr_tree || type != 0)
    {
        printf("\nERROR (drop-in): poisson_error supports the head node (type 0) only\n");
        return false;
    }
    int conv = 0;
    if (qz_set_head_field(g_sim, QZ_FIELD_POT, p->ptr_pot) ||
        qz_set_head_field(g_sim, QZ_FIELD_POT_OLD, p->ptr_pot_old) ||
        qz_set_head_field(g_sim, QZ_FIELD_DENSITY, p->ptr_d) || qz_poisson_error(g_sim, &conv) ||
        qz_get_head_field(g_sim, QZ_FIELD_POT_OLD, p->ptr_pot_old))
    {
        fail("poisson_error");
        return false;
    }
    return conv != 0;
}

static int dense_order(void)
{
    const char *o = getenv("QZ_GS_ORDER");
    return (o && !strcmp(o, "rb")) ? QZ_GS_REDBLACK : QZ_GS_LEX;
}

/* force_methods/multigrid.c:106-229 on caller arrays. */
void multigrid(double *phi, const double *rho, int gridsize, int type_multigrid)
{
    if (!resolve())
        return;
    qz_config c;
    fill_config(&c);
    c.gs_order = dense_order();
    c.precision = QZ_PREC_FP64;
    if (qz_multigrid(&c, phi, rho, gridsize, type_multigrid))
        fail("multigrid");
}

/* force_methods/gauss_saidel.c:29-55 */
void gauss_saidel(double *phi, const double *rho, int gridsize, int iter_max)
{
    if (!resolve())
        return;
    if (qz_gauss_saidel(phi, rho, gridsize, iter_max, *R.w_sor_head, dense_order()))
        fail("gauss_saidel");
}

/* force_methods/jacobi.c:29-82 */
void jacobi(double *phi, const double *rho, int gridsize, int iter_max)
{
    if (!resolve())
        return;
    if (qz_jacobi(phi, rho, gridsize, iter_max, *R.w_sor_head))
        fail("jacobi");
}

/* force_methods/conjugate_gradient.c:322-463: one node's solve on the device
 * (the node's grid fields are copied in and back; see qz_node_conjugate_gradient). */
int conjugate_gradient(struct node *p)
{
    if (!p || ensure())
        return REF_FAILURE;
    if (qz_node_conjugate_gradient(g_sim, p->lv, p->box_real_dim_x, p->box_real_dim_y,
                                   p->box_real_dim_z, p->grid_intr_size, p->ptr_intr_box_grid_idx,
                                   p->node_mass, p->cell_size, p->ptr_d, p->ptr_pot,
                                   p->ptr_pot_old))
    {
        fail("conjugate_gradient");
        return REF_FAILURE;
    }
    return REF_SUCCESS;
}

/* force_methods/conjugate_gradient_multigrid.c:29-176 */
void conjugate_gradient_multigrid(double *phi, const double *rho, int gridsize, int iters)
{
    if (qz_conjugate_gradient_multigrid(phi, rho, gridsize, iters))
        fail("conjugate_gradient_multigrid");
}

/* force_methods/multigrid2.c: never called by the reference; kept for linking. */
void multigrid2(double *phi, double *rho, int type_multigrid)
{
    (void)phi;
    (void)rho;
    (void)type_multigrid;
    printf("\nERROR (drop-in): multigrid2 is not supported by this build\n");
}

int qz_dropin_sync_from_host(void)
{
    if (ensure())
        return REF_FAILURE;
    return upload_all();
}

void *qz_dropin_context(void) { return g_sim; }

/*
 * ref_driver.c -- test harness that runs the QUANTIZER reference C (or the
 * drop-in library that replaces its hot path) on a synthetic initial
 * condition with a fixed time step, and dumps per-step fields.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is linked either
 *   (a) against every reference object except main.o  -> oracle/_ref/qz_ref_driver
 *       (the reference's own FP64 path: the oracle and the CPU baseline), or
 *   (b) against the reference's bookkeeping objects plus libqz_dropin.so
 *       -> oracle/_ref/qz_dropin_driver (the drop-in link test).
 * It restates the per-step call order of the reference's main loop
 * (source/main.c:296-338 for step 0, source/main.c:375-481 for each step),
 * replacing timestep() by a fixed dt and skipping observables/snapshots, which
 * are outside the timed step loop.
 *
 * Usage: qz_ref_driver IC.bin OUTDIR key=value ...
 *   keys: lmin, lmax, steps, dt, dump (comma list of steps, -1 = none),
 *         ref_ptcl, G, threads, solver (0 GS,1 Jacobi,2 CG), bdry, cg_head,
 *         stencil (force_stencil), branch_cg_cells (nodes of more cells use
 *         conjugate gradient, the others red-black SOR), tsm (time_step_method),
 *         cfl (_CFL_), max_dt (_MAX_dt_), obs (1: dump observables of both
 *         potential-energy forms as obs0 / obs1: energies[3], momentum[3]),
 *         check (check_poisson_error_method 0/1/2), snap (after the last step:
 *         1 output_snapshots(snap_time, 0) into OUTDIR/run/../output, 2 the same
 *         after observables() with compute_observables_FLAG set and
 *         potential_energy_type snap_pe), snap_time,
 *         cm (GL_cm_x,y,z,vx,vy,vz as a comma list)
 * IC.bin: int64 N, then x[N] y[N] z[N] vx[N] vy[N] vz[N] m[N] (float64).
 * Dumps: OUTDIR/s<step>_<field>.bin raw float64 (head grid and particles, and
 *        dtcfl: the reference's timestep() of that state),
 *        OUTDIR/s<step>_nodes.txt (AMR node summary when lmax > lmin).
 * The last stdout line is a JSON summary with the step-loop wall time.
 */
#include "main.h"
#include <stdint.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

static void die(const char *msg)
{
    fprintf(stderr, "ref_driver: %s\n", msg);
    exit(2);
}

static void write_f64(const char *dir, int step, const char *name,
                      const double *a, long n)
{
    char path[2048];
    snprintf(path, sizeof path, "%s/s%d_%s.bin", dir, step, name);
    FILE *f = fopen(path, "wb");
    if (!f)
        die("cannot open dump file");
    if (n > 0 && fwrite(a, sizeof(double), (size_t)n, f) != (size_t)n)
        die("short write");
    fclose(f);
}

static void write_i32(const char *dir, int step, const char *name,
                      const int *a, long n)
{
    char path[2048];
    snprintf(path, sizeof path, "%s/s%d_%s.bin", dir, step, name);
    FILE *f = fopen(path, "wb");
    if (!f)
        die("cannot open dump file");
    if (n > 0 && fwrite(a, sizeof(int), (size_t)n, f) != (size_t)n)
        die("short write");
    fclose(f);
}

/* Node summary: one line per node, then its interior/boundary/sim-boundary
 * grid-point lists and its box are dumped as int32 arrays. */
static void dump_nodes(const char *dir, int step)
{
    char path[2048];
    snprintf(path, sizeof path, "%s/s%d_nodes.txt", dir, step);
    FILE *f = fopen(path, "w");
    if (!f)
        die("cannot open node summary");
    fprintf(f, "# lv idx ID box_real_dim_xyz box_ts_xyz box_min_xyz box_max_xyz cell_size "
               "grid_intr grid_bdry grid_sim_bdry no_ptcl_full no_ptcl_outs chn_size node_mass parent_lv parent_idx\n");
    for (int lv = 0; lv <= GL_tentacles_level_max; lv++)
    {
        for (int i = 0; i < GL_tentacles_size[lv]; i++)
        {
            struct node *p = GL_tentacles[lv][i];
            int plv = -1, pidx = -1;
            if (p->ptr_pt)
            {
                plv = lv - 1;
                for (int q = 0; q < GL_tentacles_size[plv]; q++)
                    if (GL_tentacles[plv][q] == p->ptr_pt)
                        pidx = q;
            }
            fprintf(f, "%d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %d %.17g %d %d\n",
                    p->lv, i, p->ID, p->box_real_dim_x, p->box_real_dim_y, p->box_real_dim_z,
                    p->box_ts_x, p->box_ts_y, p->box_ts_z, p->box_min_x, p->box_min_y, p->box_min_z,
                    p->box_max_x, p->box_max_y, p->box_max_z, p->cell_size, p->grid_intr_size,
                    p->grid_bdry_size, p->grid_sim_bdry_size, p->no_ptcl_full_node,
                    p->no_ptcl_outs_ref_zones, p->chn_size, (double)p->node_mass, plv, pidx);
            char name[256];
            long gcap = (long)(p->box_real_dim_x + 1) * (p->box_real_dim_y + 1) * (p->box_real_dim_z + 1);
            long bcap = (long)p->box_real_dim_x * p->box_real_dim_y * p->box_real_dim_z;
            snprintf(name, sizeof name, "L%d_N%d_intr", lv, i);
            write_i32(dir, step, name, p->ptr_intr_box_grid_idx, p->grid_intr_size);
            snprintf(name, sizeof name, "L%d_N%d_bdry", lv, i);
            write_i32(dir, step, name, p->ptr_bdry_box_grid_idx, p->grid_bdry_size);
            snprintf(name, sizeof name, "L%d_N%d_simbdry", lv, i);
            write_i32(dir, step, name, p->ptr_sim_bdry_box_grid_idx, p->grid_sim_bdry_size);
            snprintf(name, sizeof name, "L%d_N%d_box", lv, i);
            write_i32(dir, step, name, p->ptr_box, bcap);
            snprintf(name, sizeof name, "L%d_N%d_cells", lv, i);
            write_i32(dir, step, name, p->ptr_box_idx, p->cell_size);
            snprintf(name, sizeof name, "L%d_N%d_cx", lv, i);
            write_i32(dir, step, name, p->ptr_cell_idx_x, p->cell_size);
            snprintf(name, sizeof name, "L%d_N%d_cy", lv, i);
            write_i32(dir, step, name, p->ptr_cell_idx_y, p->cell_size);
            snprintf(name, sizeof name, "L%d_N%d_cz", lv, i);
            write_i32(dir, step, name, p->ptr_cell_idx_z, p->cell_size);
            snprintf(name, sizeof name, "L%d_N%d_pot", lv, i);
            write_f64(dir, step, name, p->ptr_pot, gcap);
            snprintf(name, sizeof name, "L%d_N%d_d", lv, i);
            write_f64(dir, step, name, p->ptr_d, gcap);
            snprintf(name, sizeof name, "L%d_N%d_ax", lv, i);
            write_f64(dir, step, name, p->ptr_ax, gcap);
            snprintf(name, sizeof name, "L%d_N%d_ay", lv, i);
            write_f64(dir, step, name, p->ptr_ay, gcap);
            snprintf(name, sizeof name, "L%d_N%d_az", lv, i);
            write_f64(dir, step, name, p->ptr_az, gcap);
        }
    }
    fclose(f);
}

static int g_obs = 0; /* dump observables at each dumped step */

static void dump_step(const char *dir, int step, int amr)
{
    struct node *h = GL_ptr_tree;
    long cap = (long)(h->box_real_dim_x + 1) * (h->box_real_dim_y + 1) * (h->box_real_dim_z + 1);
    long n = GL_no_ptcl_final;
    write_f64(dir, step, "pot", h->ptr_pot, cap);
    write_f64(dir, step, "d", h->ptr_d, cap);
    write_f64(dir, step, "gax", h->ptr_ax, cap);
    write_f64(dir, step, "gay", h->ptr_ay, cap);
    write_f64(dir, step, "gaz", h->ptr_az, cap);
    write_f64(dir, step, "x", GL_ptcl_x, n);
    write_f64(dir, step, "y", GL_ptcl_y, n);
    write_f64(dir, step, "z", GL_ptcl_z, n);
    write_f64(dir, step, "vx", GL_ptcl_vx, n);
    write_f64(dir, step, "vy", GL_ptcl_vy, n);
    write_f64(dir, step, "vz", GL_ptcl_vz, n);
    write_f64(dir, step, "ax", GL_ptcl_ax, n);
    write_f64(dir, step, "ay", GL_ptcl_ay, n);
    write_f64(dir, step, "az", GL_ptcl_az, n);
    /* head-node box index of every particle (ptcl_idx_to_box_idx.c:30-139) */
    int *bidx = (int *)malloc((n > 0 ? n : 1) * sizeof(int));
    for (long i = 0; i < n; i++)
        bidx[i] = ptcl_idx_to_box_idx(h, (int)i);
    write_i32(dir, step, "bidx", bidx, n);
    free(bidx);
    if (amr)
        dump_nodes(dir, step);
    /* energies and momentum (observables.c:661-696), both potential-energy forms */
    if (g_obs)
    {
        int saved = potential_energy_type;
        for (int t = 0; t < 2; t++)
        {
            potential_energy_type = t;
            double o[6] = {0, 0, 0, 0, 0, 0};
            if (observables() == _FAILURE_)
                fprintf(stderr, "ref_driver: observables failed\n");
            for (int k = 0; k < 3; k++)
            {
                o[k] = GL_energies[k];
                o[3 + k] = GL_momentum[k];
            }
            write_f64(dir, step, t == 0 ? "obs0" : "obs1", o, 6);
        }
        potential_energy_type = saved;
    }
    /* the CFL step the main loop would take next (main.c:375, timestep.c:589-700) */
    double dtc = 0.0;
    if (timestep(&dtc) == _FAILURE_)
        fprintf(stderr, "ref_driver: timestep failed\n");
    write_f64(dir, step, "dtcfl", &dtc, 1);
}

static int in_list(const char *list, int step)
{
    if (!list)
        return 0;
    const char *p = list;
    while (*p)
    {
        char *end;
        long v = strtol(p, &end, 10);
        if (end == p)
            break;
        if (v == step)
            return 1;
        p = (*end == ',') ? end + 1 : end;
    }
    return 0;
}

static double now_s(void)
{
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

int main(int argc, char **argv)
{
    if (argc < 3)
        die("usage: qz_ref_driver IC.bin OUTDIR key=value...");
    const char *ic = argv[1];
    const char *out = argv[2];
    int L = 5, LMAX = -1, steps = 1, ref_ptcl = 9, threads = 1, solver = 0, bdry = 1;
    int cg_head = 0;
    int stencil = 0;        /* force_stencil */
    int tsm = -1;           /* time_step_method */
    double cfl = -1.0;      /* _CFL_ */
    double max_dt = -1.0;   /* _MAX_dt_ */
    int branch_cg_cells = -1; /* branches_maximal_node_number_to_activate_conjugate_gradient */
    int check = -1;           /* check_poisson_error_method */
    int snap = 0;             /* write a snapshot after the last step */
    double snap_time = 0.0;
    int snap_pe = -1;         /* potential_energy_type of the snapshot's observables */
    double cm[6] = {0, 0, 0, 0, 0, 0};
    double dt = 1e-4, G = 1.0;
    const char *dump = NULL;
    for (int a = 3; a < argc; a++)
    {
        char key[64];
        const char *eq = strchr(argv[a], '=');
        if (!eq || eq - argv[a] >= (long)sizeof key)
            die("bad key=value");
        memcpy(key, argv[a], eq - argv[a]);
        key[eq - argv[a]] = 0;
        const char *v = eq + 1;
        if (!strcmp(key, "lmin")) L = atoi(v);
        else if (!strcmp(key, "lmax")) LMAX = atoi(v);
        else if (!strcmp(key, "steps")) steps = atoi(v);
        else if (!strcmp(key, "dt")) dt = atof(v);
        else if (!strcmp(key, "G")) G = atof(v);
        else if (!strcmp(key, "dump")) dump = v;
        else if (!strcmp(key, "ref_ptcl")) ref_ptcl = atoi(v);
        else if (!strcmp(key, "threads")) threads = atoi(v);
        else if (!strcmp(key, "solver")) solver = atoi(v);
        else if (!strcmp(key, "bdry")) bdry = atoi(v);
        else if (!strcmp(key, "cg_head")) cg_head = atoi(v);
        else if (!strcmp(key, "stencil")) stencil = atoi(v);
        else if (!strcmp(key, "tsm")) tsm = atoi(v);
        else if (!strcmp(key, "cfl")) cfl = atof(v);
        else if (!strcmp(key, "max_dt")) max_dt = atof(v);
        else if (!strcmp(key, "obs")) g_obs = atoi(v);
        else if (!strcmp(key, "branch_cg_cells")) branch_cg_cells = atoi(v);
        else if (!strcmp(key, "check")) check = atoi(v);
        else if (!strcmp(key, "snap")) snap = atoi(v);
        else if (!strcmp(key, "snap_time")) snap_time = atof(v);
        else if (!strcmp(key, "snap_pe")) snap_pe = atoi(v);
        else if (!strcmp(key, "cm"))
        {
            const char *p = v;
            for (int q = 0; q < 6; q++)
            {
                char *end;
                cm[q] = strtod(p, &end);
                p = *end == ',' ? end + 1 : end;
            }
        }
        else die("unknown key");
    }
    if (LMAX < 0)
        LMAX = L;

    FILE *f = fopen(ic, "rb");
    if (!f)
        die("cannot open IC");
    int64_t n64;
    if (fread(&n64, sizeof n64, 1, f) != 1)
        die("bad IC header");
    int N = (int)n64;

    /* Reference defaults first (source/global_variables.c:467-516), then the
     * configuration of this run. */
    global_variables();
    _G_ = G;
    lmin = L;
    lmax = LMAX;
    no_lmin_cell = 1 << lmin;
    no_lmin_cell_pow2 = no_lmin_cell * no_lmin_cell;
    no_lmin_cell_pow3 = no_lmin_cell * no_lmin_cell * no_lmin_cell;
    no_grid = no_lmin_cell + 1;
    no_grid_pow2 = no_grid * no_grid;
    no_grid_pow3 = no_grid * no_grid * no_grid;
    ref_criterion_ptcl = ref_ptcl;
    compute_observables_FLAG = false;
    bdry_cond_type = bdry;
    solverPreS = solverPostS = solverfinddphic = solver;
    head_pot_method = cg_head;
    force_stencil = stencil;
    if (tsm >= 0)
        time_step_method = tsm;
    if (cfl > 0.0)
        _CFL_ = cfl;
    if (max_dt > 0.0)
        _MAX_dt_ = max_dt;
    if (branch_cg_cells >= 0)
        branches_maximal_node_number_to_activate_conjugate_gradient = branch_cg_cells;
    if (check >= 0)
        check_poisson_error_method = check;
    NUMBER_OF_THEADS = threads;
    omp_set_num_threads(threads);
    bder_os_sim = 1 > n_exp ? 1 : n_exp;
    box_side_lmin = no_lmin_cell + 2 * bder_os_sim;
    box_side_lmin_pow2 = box_side_lmin * box_side_lmin;
    box_side_lmin_pow3 = box_side_lmin * box_side_lmin * box_side_lmin;

    GL_no_ptcl_initial = GL_no_ptcl_final = N;
    double **arrs[10] = {&GL_ptcl_mass, &GL_ptcl_x, &GL_ptcl_y, &GL_ptcl_z, &GL_ptcl_vx,
                         &GL_ptcl_vy, &GL_ptcl_vz, &GL_ptcl_ax, &GL_ptcl_ay, &GL_ptcl_az};
    for (int q = 0; q < 10; q++)
    {
        free(*arrs[q]);
        *arrs[q] = (double *)calloc(N > 0 ? N : 1, sizeof(double));
        GL_ptcl[q] = *arrs[q];
    }
    double *order[7] = {GL_ptcl_x, GL_ptcl_y, GL_ptcl_z, GL_ptcl_vx, GL_ptcl_vy, GL_ptcl_vz, GL_ptcl_mass};
    for (int q = 0; q < 7; q++)
        if (fread(order[q], sizeof(double), N, f) != (size_t)N)
            die("short IC");
    fclose(f);
    GL_total_mass_initial = 0.0;
    for (int i = 0; i < N; i++)
        GL_total_mass_initial += GL_ptcl_mass[i];
    GL_cm_x = GL_cm_y = GL_cm_z = GL_cm_vx = GL_cm_vy = GL_cm_vz = 0.0;
    GL_cm_x = cm[0];
    GL_cm_y = cm[1];
    GL_cm_z = cm[2];
    GL_cm_vx = cm[3];
    GL_cm_vy = cm[4];
    GL_cm_vz = cm[5];

    if (initialization() == _FAILURE_)
        die("initialization failed");
    if (tree_construction() == _FAILURE_)
        die("tree_construction failed");

    int amr = lmin < lmax;
    double t0 = now_s();
    grid_density();
    if (potential() == _FAILURE_)
        die("potential failed");
    if (grid_acceleration() == _FAILURE_)
        die("grid_acceleration failed");
    if (particle_acceleration() == _FAILURE_)
        die("particle_acceleration failed");
    double t_init = now_s() - t0;
    if (in_list(dump, 0))
        dump_step(out, 0, amr);

    double t_loop = 0.0;
    for (int s = 1; s <= steps; s++)
    {
        double ts = now_s();
        if (particle_updating_A(dt) == _FAILURE_)
            die("particle_updating_A failed");
        if (reset() == _FAILURE_)
            die("reset failed");
        if (tree_adaptation() == _FAILURE_)
            die("tree_adaptation failed");
        grid_density();
        if (potential() == _FAILURE_)
            die("potential failed");
        if (grid_acceleration() == _FAILURE_)
            die("grid_acceleration failed");
        if (particle_acceleration() == _FAILURE_)
            die("particle_acceleration failed");
        particle_updating_B(dt);
        t_loop += now_s() - ts;
        if (in_list(dump, s))
            dump_step(out, s, amr);
    }
    if (snap)
    {
        /* output_snapshots writes under ../output relative to the working directory */
        char here[4096], run[4200];
        if (!getcwd(here, sizeof here))
            die("getcwd");
        snprintf(run, sizeof run, "%s/run", out);
        mkdir(run, 0777);
        if (chdir(run))
            die("chdir");
        if (snap == 2)
        {
            compute_observables_FLAG = true;
            if (snap_pe >= 0)
                potential_energy_type = snap_pe;
            if (observables() == _FAILURE_)
                die("observables failed");
        }
        if (output_snapshots(snap_time, 0) == _FAILURE_)
            die("output_snapshots failed");
        if (chdir(here))
            die("chdir back");
    }
    int nodes = 0;
    for (int lv = 0; lv <= GL_tentacles_level_max; lv++)
        nodes += GL_tentacles_size[lv];
    printf("\n{\"n\": %d, \"steps\": %d, \"init_s\": %.6f, \"loop_s\": %.6f, "
           "\"ptcl_steps_per_s\": %.6e, \"levels\": %d, \"nodes\": %d, \"threads\": %d, "
           "\"max_dt\": %.17e, \"cfl\": %.17e, \"time_step_method\": %d, "
           "\"conversion_velocity\": %.17e, \"conversion_time\": %.17e, "
           "\"conversion_dist\": %.17e}\n",
           N, steps, t_init, t_loop, steps > 0 ? (double)N * steps / t_loop : 0.0,
           GL_tentacles_level_max, nodes, threads, (double)_MAX_dt_, (double)_CFL_,
           time_step_method, (double)_conversion_velocity_, (double)_conversion_time_,
           (double)_conversion_dist_);
    return 0;
}

// qz_capi.cu -- the extern "C" surface of libqzb200 (include/qz_b200.h):
// context lifecycle, host <-> device copies through pinned staging buffers,
// per-stage entry points in the reference's main-loop order, and array-level
// wrappers of the force_methods routines.
#include <stdarg.h>
#include <stdlib.h>
#include <stdio.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "qz_internal.cuh"

namespace qz {

static thread_local char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

bool check_cuda(cudaError_t e, const char *what)
{
    if (e == cudaSuccess)
        return true;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return false;
}

cudaEvent_t prof_event(qz_sim *s)
{
    if (!s->ev_pool.empty())
    {
        cudaEvent_t e = s->ev_pool.back();
        s->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Books the elapsed time of every pending launch to its category and returns
// the events to the pool (the stream must be idle).
void prof_collect(qz_sim *s)
{
    for (auto &r : s->prof_pending)
    {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, r.b, r.e) == cudaSuccess)
        {
            s->prof_launches[r.cat]++;
            s->prof_ms[r.cat] += ms;
            s->prof_bytes[r.cat] += r.bytes;
        }
        s->ev_pool.push_back(r.b);
        s->ev_pool.push_back(r.e);
    }
    s->prof_pending.clear();
    cudaGetLastError();
}

long radix_tiles(long n);
void launch_box_idx(cudaStream_t st, long n, int lv, int tsx, int tsy, int tsz, int dimx,
                    int dimy, const double *x, const double *y, const double *z, int *out);

template <typename T>
static bool dmalloc(T **p, size_t count, const char *what)
{
    *p = nullptr;
    if (count == 0)
        count = 1;
    return check_cuda(cudaMalloc((void **)p, count * sizeof(T)), what);
}

static void dfree(void *p)
{
    if (p)
        cudaFree(p);
}

// Allocates the multigrid hierarchy below a fine level of n0 points per side:
// levels exist while the recursion of multigrid.c:175-191 reaches them
// (coarse size >= 4).
static bool build_levels(qz_sim *s, int n0)
{
    init_kernel_attributes();
    const bool mixed = s->cfg.precision == QZ_PREC_MIXED;
    const bool jac = s->cfg.smoother == 1;
    s->levels.clear();
    Level l0;
    l0.n = n0;
    s->levels.push_back(l0);
    int n = n0;
    while (true)
    {
        int nc = (n + 1) / 2;
        if (nc < 4)
            break;
        Level l;
        l.n = nc;
        size_t pts = (size_t)nc * nc * nc;
        if (!dmalloc(&l.phi, pts, "mg phi") || !dmalloc(&l.rho, pts, "mg rho"))
            return false;
        cudaMemset(l.rho, 0, pts * sizeof(double));
        if (mixed && (!dmalloc(&l.phif, pts, "mg phi32") || !dmalloc(&l.rhof, pts, "mg rho32")))
            return false;
        if (mixed)
            cudaMemset(l.rhof, 0, pts * sizeof(float));
        if (!dmalloc(&l.alt, pts, "mg alt"))
            return false;
        cudaMemset(l.alt, 0, pts * sizeof(double));
        if (mixed && !dmalloc(&l.altf, pts, "mg alt32"))
            return false;
        if (mixed)
            cudaMemset(l.altf, 0, pts * sizeof(float));
        s->levels.push_back(l);
        n = nc;
    }
    const bool cgs = s->cfg.smoother == 2;
    if (cgs && !s->cg_part && !dmalloc(&s->cg_part, 2 * QZ_CG_PART_MAX, "cg partials"))
        return false;
    // persistent cycles: per-block partials of the in-launch convergence test, its result
    if (!s->mg_part && !dmalloc(&s->mg_part, 2 * QZ_CG_PART_MAX + 8, "mg partials"))
        return false;
    for (auto &l : s->levels)
    {
        size_t pts = (size_t)l.n * l.n * l.n;
        if (jac && !dmalloc(&l.scr, pts, "jacobi scratch"))
            return false;
        if (jac && mixed && !dmalloc(&l.scrf, pts, "jacobi scratch32"))
            return false;
        if (cgs)
        {
            // r and p stay zero on the boundary (conjugate_gradient_multigrid.c:37-39)
            if (!dmalloc(&l.cgr, pts, "cg r") || !dmalloc(&l.cgp, pts, "cg p") ||
                !dmalloc(&l.cga, pts, "cg Ap"))
                return false;
            cudaMemset(l.cgr, 0, pts * sizeof(double));
            cudaMemset(l.cgp, 0, pts * sizeof(double));
            cudaMemset(l.cga, 0, pts * sizeof(double));
            if (mixed)
            {
                if (!dmalloc(&l.cgrf, pts, "cg r32") || !dmalloc(&l.cgpf, pts, "cg p32") ||
                    !dmalloc(&l.cgaf, pts, "cg Ap32"))
                    return false;
                cudaMemset(l.cgrf, 0, pts * sizeof(float));
                cudaMemset(l.cgpf, 0, pts * sizeof(float));
                cudaMemset(l.cgaf, 0, pts * sizeof(float));
            }
        }
    }
    if (mixed)
    {
        size_t pts = (size_t)n0 * n0 * n0;
        if (!dmalloc(&s->rf, pts, "rf") || !dmalloc(&s->ef, pts, "ef") ||
            !dmalloc(&s->ef_alt, pts, "ef alt"))
            return false;
        cudaMemset(s->rf, 0, pts * sizeof(float));
        cudaMemset(s->ef, 0, pts * sizeof(float));
        cudaMemset(s->ef_alt, 0, pts * sizeof(float));
    }
    return true;
}

static void free_levels(qz_sim *s)
{
    for (size_t i = 0; i < s->levels.size(); i++)
    {
        Level &l = s->levels[i];
        if (i > 0)
        {
            dfree(l.phi);
            dfree(l.rho);
            dfree(l.phif);
            dfree(l.rhof);
            dfree(l.alt);
            dfree(l.altf);
        }
        dfree(l.scr);
        dfree(l.scrf);
        void *cg[] = {l.cgr, l.cgp, l.cga, l.cgrf, l.cgpf, l.cgaf};
        for (void *q : cg)
            dfree(q);
    }
    s->levels.clear();
    dfree(s->cg_part);
    s->cg_part = nullptr;
    dfree(s->mg_part);
    s->mg_part = nullptr;
    dfree(s->rf);
    dfree(s->ef);
    dfree(s->ef_alt);
    dfree(s->fine_alt_buf);
    s->rf = s->ef = s->ef_alt = nullptr;
    s->fine_alt_buf = nullptr;
}

static bool ensure_stage(qz_sim *s, size_t bytes)
{
    if (s->h_stage_bytes >= bytes)
        return true;
    if (s->h_stage)
        cudaFreeHost(s->h_stage);
    s->h_stage = nullptr;
    s->h_stage_bytes = 0;
    if (!check_cuda(cudaMallocHost((void **)&s->h_stage, bytes), "pinned staging"))
        return false;
    s->h_stage_bytes = bytes;
    return true;
}

// Copies `count` doubles host -> device through the pinned stage (when the
// host pointer is pageable) on the library stream.
static bool h2d(qz_sim *s, double *dst, const double *src, long count)
{
    if (count <= 0)
        return true;
    size_t bytes = (size_t)count * sizeof(double);
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, src) == cudaSuccess && at.type == cudaMemoryTypeHost)
        return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s->stream),
                          "h2d");
    cudaGetLastError();
    if (!ensure_stage(s, bytes))
        return false;
    if (!check_cuda(cudaStreamSynchronize(s->stream), "h2d sync"))
        return false;
    memcpy(s->h_stage, src, bytes);
    return check_cuda(cudaMemcpyAsync(dst, s->h_stage, bytes, cudaMemcpyHostToDevice, s->stream),
                      "h2d");
}

static bool d2h(qz_sim *s, double *dst, const double *src, long count)
{
    if (count <= 0 || !dst)
        return true;
    size_t bytes = (size_t)count * sizeof(double);
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, dst) == cudaSuccess && at.type == cudaMemoryTypeHost)
        return check_cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s->stream),
                          "d2h") &&
               check_cuda(cudaStreamSynchronize(s->stream), "d2h sync");
    cudaGetLastError();
    if (!ensure_stage(s, bytes))
        return false;
    if (!check_cuda(cudaMemcpyAsync(s->h_stage, src, bytes, cudaMemcpyDeviceToHost, s->stream),
                    "d2h") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "d2h sync"))
        return false;
    memcpy(dst, s->h_stage, bytes);
    return true;
}

bool sched_take(qz_sim *s, int n, int *out)
{
    if (s->sched_pos + (size_t)n > s->sched.size())
    {
        set_error("solver schedule exhausted: the replayed run has more solves than the "
                  "recorded one");
        return false;
    }
    for (int q = 0; q < n; q++)
        out[q] = s->sched[s->sched_pos + q];
    s->sched_pos += n;
    return true;
}

void sched_put(qz_sim *s, const int *v, int n) { s->sched.insert(s->sched.end(), v, v + n); }

int check_flags(qz_sim *s)
{
    if (!check_cuda(cudaMemcpyAsync(s->h_flags, s->flags, F_COUNT * sizeof(int),
                                    cudaMemcpyDeviceToHost, s->stream),
                    "flags") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "flags sync"))
        return QZ_FAILURE;
    int e = s->h_flags[F_ERROR];
    s->stats.error_flags |= e;
    if (e)
    {
        cudaMemsetAsync(s->flags + F_ERROR, 0, sizeof(int), s->stream);
        if (e & E_BARRIER)
            set_error("a grid barrier wait in a cooperative kernel gave up (flags 0x%x)", e);
        else if (e & E_SCAN)
            set_error("a scan's wait for a preceding tile gave up (flags 0x%x)", e);
        else
            set_error("device bounds check failed (flags 0x%x): a particle left the unit box", e);
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

} // namespace qz

using namespace qz;

extern "C" {

const char *qz_last_error(void) { return g_err; }

int qz_default_config(qz_config *c, int lmin)
{
    if (!c)
        return QZ_FAILURE;
    memset(c, 0, sizeof *c);
    c->lmin = lmin;
    c->lmax = lmin;
    c->G = 1.0;
    c->total_mass = 1.0;
    c->bdry = 1;
    c->smoother = 0;
    c->gs_order = QZ_GS_REDBLACK;
    c->cycle = 0;
    c->n_pre = 2;
    c->n_post = 2;
    c->n_coarse = 2;
    c->w_sor = 1.0;
    c->tol = 1.0e-10;
    c->tol2 = 1.0e-10;
    c->check_every = 5;
    c->max_iter = 5000;
    c->check_method = 0;
    c->precision = QZ_PREC_FP64;
    c->inner_cycles = 1;
    c->force_stencil = 0;
    c->ref_ptcl = 4;   /* global_variables.c:289 */
    c->box_extra = 10; /* 2 * min_box_extra_size_per_side_user, global_variables.c:294-295 */
    c->branch_cg_cells = 0;    /* global_variables.c:334 */
    c->branch_sor_sweeps = 10; /* global_variables.c:328 */
    c->w_sor_branch = 1.0;     /* global_variables.c:329 */
    c->cfl = 0.5;              /* _CFL_, global_variables.c:291 */
    c->max_dt = 1.0e30;        /* _MAX_dt_ (0.005 Maxdt in the reference's units): no cap */
    c->time_step_method = 1;   /* global_variables.c:342 */
    c->head_pot_method = 0;    /* global_variables.c (multigrid) */
    c->adjoint_tol = 1e-10;
    c->cg_variant = 0;
    c->mg_points_per_thread = 4;
    c->freeze_tree = 0;
    c->node_solver = QZ_NODE_CG;
    c->mg_tile = 0;
    c->node_warm = 0;
    c->tree_overlap = 1;
    c->cg_chunk_min = 0;
    return QZ_SUCCESS;
}

// Stream-ordered pool of a device, shared by all simulations on it (created once,
// kept until the process exits): freed memory stays in the pool, so buffers that
// grow with the refinement tree never wait for the device.  One pool per
// simulation would not scale to ensembles of hundreds of simulations.
static bool make_pool(qz_sim *s)
{
    static std::mutex mu;
    static std::vector<cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    if ((int)pools.size() <= s->device)
        pools.resize(s->device + 1, nullptr);
    if (!pools[s->device])
    {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = s->device;
        cudaMemPool_t p = nullptr;
        if (!check_cuda(cudaMemPoolCreate(&p, &props), "memory pool"))
            return false;
        unsigned long long keep = ~0ULL;
        if (!check_cuda(cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep),
                        "memory pool threshold"))
            return false;
        pools[s->device] = p;
    }
    s->mem.pool = pools[s->device];
    s->mem.stream = s->stream;
    return true;
}

int qz_destroy(qz_sim *s)
{
    if (!s)
        return QZ_SUCCESS;
    if (s->stream)
        cudaStreamSynchronize(s->stream);
    prof_collect(s);
    snapshot_free(s);
    if (s->check_exec)
        cudaGraphExecDestroy(s->check_exec);
    for (cudaEvent_t e : s->ev_pool)
        cudaEventDestroy(e);
    s->ev_pool.clear();
    void *ptrs[] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->m,
                    s->pot, s->pot_old, s->d, s->gax, s->gay, s->gaz, s->sort.k0, s->sort.k1,
                    s->sort.v0, s->sort.v1, s->sort.hist, s->seg_head, s->seg_id, s->seg_start,
                    s->seg_cell, s->cell_seg, s->cell_sums, s->red, s->flags, s->d_ts,
                    s->gbar, s->long_seg};
    for (void *p : ptrs)
        dfree(p);
    free_levels(s);
    amr_free(s);
    node_mg_free(s);
    adjoint_free(s);
    s->ofl_state.release(s->mem);
    s->ofl_int.release(s->mem);
    if (s->mem.pool)
        pool_free(s->mem, s->scan_st);
    if (s->stream)
        cudaStreamSynchronize(s->stream); // the pool frees are stream-ordered
    if (s->mem.pool)
        cudaMemPoolTrimTo(s->mem.pool, 0); // unused memory back to the device
    if (s->h_flags)
        cudaFreeHost(s->h_flags);
    if (s->h_ofl)
        cudaFreeHost(s->h_ofl);
    if (s->h_ts)
        cudaFreeHost(s->h_ts);
    if (s->h_stage)
        cudaFreeHost(s->h_stage);
    if (s->xfer)
    {
        cudaStreamSynchronize(s->xfer);
        cudaStreamDestroy(s->xfer);
    }
    if (s->ev_mass)
        cudaEventDestroy(s->ev_mass);
    if (s->ev_drift)
        cudaEventDestroy(s->ev_drift);
    if (s->head_stream)
    {
        cudaStreamSynchronize(s->head_stream);
        cudaStreamDestroy(s->head_stream);
    }
    if (s->ev_fork)
        cudaEventDestroy(s->ev_fork);
    if (s->ev_head)
        cudaEventDestroy(s->ev_head);
    if (s->stream)
        cudaStreamDestroy(s->stream);
    delete s;
    return QZ_SUCCESS;
}

int qz_create(const qz_config *cfg, long n_capacity, qz_sim **out)
{
    if (!cfg || !out || n_capacity < 0)
    {
        set_error("qz_create: bad arguments");
        return QZ_FAILURE;
    }
    *out = nullptr;
    if (cfg->lmin < 2 || cfg->lmin > 9)
    {
        set_error("qz_create: lmin=%d outside the supported range 2..9", cfg->lmin);
        return QZ_FAILURE;
    }
    if (cfg->lmax < cfg->lmin || cfg->lmax - cfg->lmin > 12 || cfg->lmax > 20)
    {
        set_error("qz_create: lmax=%d outside lmin..min(lmin+12, 20)", cfg->lmax);
        return QZ_FAILURE;
    }
    if (cfg->lmax > cfg->lmin && (cfg->bdry != 1 || cfg->ref_ptcl < 1 || cfg->box_extra < 2 ||
                                  (cfg->box_extra & 1)))
    {
        set_error("qz_create: refinement needs reflexive boundaries, ref_ptcl >= 1 and an even "
                  "box_extra >= 2");
        return QZ_FAILURE;
    }
    if (cfg->bdry < 0 || cfg->bdry > 2 || (cfg->bdry != 1 && cfg->lmax > cfg->lmin))
    {
        // periodic and outflow boundaries are built for head-only runs; the
        // refinement tree follows the reflexive rules (no periodic ghost cells,
        // no removal inside refinement nodes)
        set_error("qz_create: bdry=%d not supported%s", cfg->bdry,
                  cfg->lmax > cfg->lmin ? " with refinement (reflexive only)" : "");
        return QZ_FAILURE;
    }
    if (cfg->force_stencil < 0 || cfg->force_stencil > 1 || cfg->smoother < 0 || cfg->smoother > 2 || cfg->cycle < 0 ||
        cfg->cycle > 2 || cfg->head_pot_method < 0 || cfg->head_pot_method > 1 ||
        cfg->cg_variant < 0 || cfg->cg_variant > 2 || cfg->mg_tile < -1 || cfg->mg_tile > QZ_MG_NTILES ||
        n_capacity > (1L << 30))
    {
        set_error("qz_create: unsupported configuration");
        return QZ_FAILURE;
    }
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    {
        cudaGetLastError();
        set_error("qz_create: no CUDA device is available (this library has no CPU path)");
        return QZ_FAILURE;
    }
    qz_sim *s = new qz_sim();
    s->cfg = *cfg;
    s->use_graphs = getenv("QZ_NO_GRAPHS") == nullptr;
    s->fused_rb = getenv("QZ_FUSED_RB") != nullptr;
    cudaGetDevice(&s->device);
    if (!check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream"))
    {
        delete s;
        return QZ_FAILURE;
    }
    if (!make_pool(s))
    {
        qz_destroy(s);
        return QZ_FAILURE;
    }
    s->cap = n_capacity;
    s->head_mass = cfg->total_mass; // initialization.c:190
    s->L = cfg->lmin;
    s->D = (1L << s->L) + 3;
    s->gpts = s->D * s->D * s->D;
    const long B = (1L << s->L) + 2;
    const long cap = n_capacity > 0 ? n_capacity : 1;
    bool ok = dmalloc(&s->x, cap, "x") && dmalloc(&s->y, cap, "y") && dmalloc(&s->z, cap, "z") &&
              dmalloc(&s->vx, cap, "vx") && dmalloc(&s->vy, cap, "vy") &&
              dmalloc(&s->vz, cap, "vz") && dmalloc(&s->ax, cap, "ax") &&
              dmalloc(&s->ay, cap, "ay") && dmalloc(&s->az, cap, "az") && dmalloc(&s->m, cap, "m");
    ok = ok && dmalloc(&s->pot, s->gpts, "pot") && dmalloc(&s->pot_old, s->gpts, "pot_old") &&
         dmalloc(&s->d, s->gpts, "d") && dmalloc(&s->gax, s->gpts, "gax") &&
         dmalloc(&s->gay, s->gpts, "gay") && dmalloc(&s->gaz, s->gpts, "gaz");
    long tiles = radix_tiles(cap);
    ok = ok && dmalloc(&s->sort.k0, cap, "keys") && dmalloc(&s->sort.k1, cap, "keys") &&
         dmalloc(&s->sort.v0, cap, "vals") && dmalloc(&s->sort.v1, cap, "vals") &&
         dmalloc(&s->sort.hist, 256 * std::max(tiles, 4L), "hist");
    ok = ok && dmalloc(&s->seg_head, cap, "seg") && dmalloc(&s->seg_id, cap, "seg") &&
         dmalloc(&s->seg_start, cap + 1, "seg") && dmalloc(&s->seg_cell, cap, "seg") &&
         dmalloc(&s->cell_seg, B * B * B, "cell_seg") && dmalloc(&s->cell_sums, 8 * cap, "cs") &&
         dmalloc(&s->long_seg, cap / SEG_LONG + 2, "long segments");
    s->red_blocks = 296;
    ok = ok && dmalloc(&s->red, s->red_blocks + 8, "red") && dmalloc(&s->flags, F_COUNT, "flags");
    ok = ok && check_cuda(cudaMallocHost((void **)&s->h_flags, F_COUNT * sizeof(int)), "pinned");
    ok = ok && dmalloc(&s->gbar, 4, "grid barrier");
    ok = ok && check_cuda(cudaMallocHost((void **)&s->h_ts, 34 * sizeof(unsigned long long)),
                          "pinned time step") &&
         dmalloc(&s->d_ts, 17, "time step");
    s->sort.cap = cap;
    s->sort.tiles_cap = tiles;
    if (ok)
    {
        cudaMemset(s->flags, 0, F_COUNT * sizeof(int));
        size_t gb = s->gpts * sizeof(double);
        cudaMemset(s->pot_old, 0, gb);
        cudaMemset(s->d, 0, gb);
        s->fine_phi = head_view(s, s->pot);
        s->fine_rho = head_view(s, s->d);
        ok = build_levels(s, (1 << s->L) + 1) && dmalloc(&s->fine_alt_buf, s->gpts, "pot alt");
        if (ok)
            s->fine_alt = head_view(s, s->fine_alt_buf);
    }
    if (ok)
        ok = head_initial(s) == QZ_SUCCESS;
    if (ok && cfg->lmax > cfg->lmin)
        ok = amr_init(s) == QZ_SUCCESS;
    if (ok)
        ok = check_cuda(cudaStreamSynchronize(s->stream), "create sync") &&
             check_cuda(cudaDeviceSynchronize(), "create device sync");
    if (!ok)
    {
        char keep[512];
        snprintf(keep, sizeof keep, "%s", g_err);
        qz_destroy(s);
        set_error("%s", keep);
        return QZ_FAILURE;
    }
    *out = s;
    return QZ_SUCCESS;
}

int qz_set_particles(qz_sim *s, long n, const double *x, const double *y, const double *z,
                     const double *vx, const double *vy, const double *vz, const double *m)
{
    if (!s || n < 0 || n > s->cap)
    {
        set_error("qz_set_particles: n=%ld exceeds capacity", n);
        return QZ_FAILURE;
    }
    s->n = n;
    s->head_mass = s->cfg.total_mass;
    s->ofl_removed = 0;
    bool ok = h2d(s, s->x, x, n) && h2d(s, s->y, y, n) && h2d(s, s->z, z, n) &&
              h2d(s, s->vx, vx, n) && h2d(s, s->vy, vy, n) && h2d(s, s->vz, vz, n) &&
              h2d(s, s->m, m, n);
    if (ok)
    {
        size_t b = (size_t)(n > 0 ? n : 1) * sizeof(double);
        ok = check_cuda(cudaMemsetAsync(s->ax, 0, b, s->stream), "memset") &&
             check_cuda(cudaMemsetAsync(s->ay, 0, b, s->stream), "memset") &&
             check_cuda(cudaMemsetAsync(s->az, 0, b, s->stream), "memset");
    }
    s->forces_ready = false;
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

int qz_set_particle_accel(qz_sim *s, const double *ax, const double *ay, const double *az)
{
    if (!s)
        return QZ_FAILURE;
    // accelerations supplied by the caller: the next step starts from them
    bool ok = h2d(s, s->ax, ax, s->n) && h2d(s, s->ay, ay, s->n) && h2d(s, s->az, az, s->n);
    s->forces_ready = ok;
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

int qz_get_particles(qz_sim *s, double *x, double *y, double *z, double *vx, double *vy,
                     double *vz, double *ax, double *ay, double *az)
{
    if (!s)
        return QZ_FAILURE;
    long n = s->n;
    bool ok = d2h(s, x, s->x, n) && d2h(s, y, s->y, n) && d2h(s, z, s->z, n) &&
              d2h(s, vx, s->vx, n) && d2h(s, vy, s->vy, n) && d2h(s, vz, s->vz, n) &&
              d2h(s, ax, s->ax, n) && d2h(s, ay, s->ay, n) && d2h(s, az, s->az, n);
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

long qz_num_particles(const qz_sim *s) { return s ? s->n : 0; }

long qz_head_grid_points(const qz_sim *s) { return s ? s->gpts : 0; }

static double *field_ptr(qz_sim *s, int which)
{
    switch (which)
    {
    case QZ_FIELD_POT: return s->pot;
    case QZ_FIELD_POT_OLD: return s->pot_old;
    case QZ_FIELD_DENSITY: return s->d;
    case QZ_FIELD_AX: return s->gax;
    case QZ_FIELD_AY: return s->gay;
    case QZ_FIELD_AZ: return s->gaz;
    default: return nullptr;
    }
}

int qz_get_head_field(qz_sim *s, int which, double *out)
{
    double *f = s ? field_ptr(s, which) : nullptr;
    if (!f || !out)
    {
        set_error("qz_get_head_field: bad field %d", which);
        return QZ_FAILURE;
    }
    return d2h(s, out, f, s->gpts) ? QZ_SUCCESS : QZ_FAILURE;
}

int qz_set_head_field(qz_sim *s, int which, const double *in)
{
    double *f = s ? field_ptr(s, which) : nullptr;
    if (!f || !in)
    {
        set_error("qz_set_head_field: bad field %d", which);
        return QZ_FAILURE;
    }
    return h2d(s, f, in, s->gpts) ? QZ_SUCCESS : QZ_FAILURE;
}

int qz_initial_potential_head(qz_sim *s) { return s ? head_initial(s) : QZ_FAILURE; }

// reset.c:29-64: particle accelerations and head density to zero.
int qz_reset(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    size_t b = (size_t)(s->n > 0 ? s->n : 1) * sizeof(double);
    bool ok = check_cuda(cudaMemsetAsync(s->ax, 0, b, s->stream), "reset") &&
              check_cuda(cudaMemsetAsync(s->ay, 0, b, s->stream), "reset") &&
              check_cuda(cudaMemsetAsync(s->az, 0, b, s->stream), "reset") &&
              check_cuda(cudaMemsetAsync(s->d, 0, s->gpts * sizeof(double), s->stream), "reset");
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

static bool amr_on(const qz_sim *s) { return s->cfg.lmax > s->cfg.lmin; }

int qz_tree_adaptation(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    if (!amr_on(s))
        return QZ_SUCCESS;
    if (s->cfg.freeze_tree && s->tree_built)
        return amr_reassign(s);
    if (amr_build(s))
        return QZ_FAILURE;
    s->tree_built = true;
    return QZ_SUCCESS;
}

int qz_grid_density(qz_sim *s)
{
    if (!s || deposit_head(s))
        return QZ_FAILURE;
    return amr_on(s) ? amr_deposit(s) : QZ_SUCCESS;
}

int qz_potential(qz_sim *s)
{
    if (!s || potential_head(s))
        return QZ_FAILURE;
    return amr_on(s) ? amr_potential(s) : QZ_SUCCESS;
}

int qz_outflow_removed(qz_sim *s, long *count, int *slots, int *sources)
{
    if (!s || !count)
        return QZ_FAILURE;
    *count = s->ofl_removed;
    if (s->ofl_removed == 0 || (!slots && !sources))
        return QZ_SUCCESS;
    const long n0 = s->ofl_layout_n;
    const int *base = s->ofl_int.p;
    bool ok = true;
    if (slots)
        ok = ok && check_cuda(cudaMemcpyAsync(slots, base + 2 * n0, s->ofl_removed * sizeof(int),
                                              cudaMemcpyDeviceToHost, s->stream), "removed");
    if (sources)
        ok = ok && check_cuda(cudaMemcpyAsync(sources, base + 3 * n0, s->ofl_removed * sizeof(int),
                                              cudaMemcpyDeviceToHost, s->stream), "removed");
    return ok && check_cuda(cudaStreamSynchronize(s->stream), "removed sync") ? QZ_SUCCESS
                                                                               : QZ_FAILURE;
}

double qz_head_mass(const qz_sim *s) { return s ? s->head_mass : 0.0; }

int qz_potential_head_node(qz_sim *s) { return s ? potential_head(s) : QZ_FAILURE; }

int qz_potential_branches(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    return amr_on(s) ? amr_potential(s) : QZ_SUCCESS;
}

int qz_poisson_error(qz_sim *s, int *converged)
{
    if (!s || !converged)
        return QZ_FAILURE;
    return poisson_error_head(s, converged);
}

int qz_grid_acceleration(qz_sim *s)
{
    if (!s || grid_accel_head(s))
        return QZ_FAILURE;
    return amr_on(s) ? amr_grid_accel(s) : QZ_SUCCESS;
}

int qz_particle_acceleration(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    return amr_on(s) ? amr_gather(s) : gather_head(s);
}

int qz_particle_updating_A(qz_sim *s, double dt) { return s ? kick_drift(s, dt) : QZ_FAILURE; }

int qz_particle_updating_B(qz_sim *s, double dt) { return s ? kick(s, dt) : QZ_FAILURE; }

int qz_init_forces(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    if (qz_reset(s) || qz_tree_adaptation(s) || qz_grid_density(s) || qz_potential(s) ||
        qz_grid_acceleration(s) || qz_particle_acceleration(s) || check_flags(s))
        return QZ_FAILURE;
    s->forces_ready = true;
    return QZ_SUCCESS;
}

} // extern "C"

namespace qz {
// Tree, densities and potentials of a step (main.c:417-447).  The tree and the
// level deposits read only the particles, and the head solve reads only the
// head density, so in refinement runs whose head solve is one persistent
// launch (tree_overlap) that launch runs on a stream of higher priority (its
// blocks are placed before the tree kernels' waiting blocks) while the tree is
// built and the levels deposited on the simulation's stream, with the host
// waits of the tree construction overlapping the solve; the level solves wait
// for both.  Every kernel computes what it computes in the sequential order.
// Measured on the 1M-particle sphere (128^3 head, three levels), ms a step:
// sequential 10.54-10.59; overlapped with 4 points a thread (two blocks on
// every SM: the tree kernels wait for the solve) 10.61, 8 points 9.66-9.80,
// 10 points 9.57, 12 points 9.53, 16 points 9.95.
constexpr int OVERLAP_PPT = 12;

// Outcomes a step reads at its end: the head launch (when it ran on the second
// stream) and the queued level solves.
struct StepPending {
    bool head = false;
    bool levels = false;
    std::vector<CgPending> pend;
};

// Reads the outcomes in the order the stages ran (head, then levels); the head
// stream is always waited for.
static int step_finish(qz_sim *s, StepPending &sp)
{
    int rc = QZ_SUCCESS;
    if (sp.head && potential_head_finish(s, s->head_stream))
        rc = QZ_FAILURE;
    if (rc == QZ_SUCCESS && sp.levels && amr_potential_collect(s, sp.pend))
        rc = QZ_FAILURE;
    sp = StepPending();
    return rc;
}

static int tree_density_potential(qz_sim *s, StepPending &sp)
{
    if (!amr_on(s) || !s->cfg.tree_overlap || s->no_overlap || !head_one_launch(s))
        return (qz_tree_adaptation(s) || qz_grid_density(s) || qz_potential(s)) ? QZ_FAILURE
                                                                                : QZ_SUCCESS;
    if (!s->head_stream)
    {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        if (!check_cuda(cudaStreamCreateWithPriority(&s->head_stream, cudaStreamNonBlocking,
                                                     greatest),
                        "head-solve stream") ||
            !check_cuda(cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming), "event") ||
            !check_cuda(cudaEventCreateWithFlags(&s->ev_head, cudaEventDisableTiming), "event"))
            return QZ_FAILURE;
    }
    bool issued = false;
    if (deposit_head(s) || !check_cuda(cudaEventRecord(s->ev_fork, s->stream), "fork") ||
        !check_cuda(cudaStreamWaitEvent(s->head_stream, s->ev_fork, 0), "fork"))
        return QZ_FAILURE;
    // the head launch takes at least OVERLAP_PPT points a thread: fewer blocks,
    // so that SMs keep room for the tree's kernels (128^3 head: 177 blocks of
    // 512 threads instead of two on every SM)
    s->mg_ppt_floor = OVERLAP_PPT;
    const int rc_issue = potential_head_issue(s, s->head_stream, &issued);
    s->mg_ppt_floor = 0;
    if (rc_issue || !check_cuda(cudaEventRecord(s->ev_head, s->head_stream), "join"))
    {
        cudaStreamSynchronize(s->head_stream);
        return QZ_FAILURE;
    }
    bool ok = !qz_tree_adaptation(s) && !amr_deposit(s) &&
              check_cuda(cudaStreamWaitEvent(s->stream, s->ev_head, 0), "join");
    // queued level solves: issued with no host wait, so the first level starts as
    // soon as the head solve ends and the gradient, gather and kick follow the
    // last level on the stream; the outcomes (head, then levels) are read at
    // the end of the step (step_finish)
    sp.head = true;
    if (ok && amr_potential_queues(s))
    {
        sp.levels = true;
        ok = !amr_potential_issue(s, sp.pend);
        return ok ? QZ_SUCCESS : QZ_FAILURE;
    }
    // the head launch is always waited for, whatever the other stages' outcome
    sp.head = false;
    const bool head_ok = !potential_head_finish(s, s->head_stream);
    if (!ok || !head_ok)
        return QZ_FAILURE;
    return amr_potential(s);
}

// main.c:375-481 with a given dt: kick-drift, reset, tree, deposit, potential,
// gradient, gather, kick.
int step_core(qz_sim *s, double h)
{
    StepPending sp;
    const bool ok = !kick_drift(s, h) && !qz_reset(s) && !tree_density_potential(s, sp) &&
                    !qz_grid_acceleration(s) && !qz_particle_acceleration(s) && !kick(s, h);
    if (step_finish(s, sp) || !ok)
        return QZ_FAILURE;
    s->stats.steps++;
    s->stats.last_dt = h;
    s->stats.sim_time += h;
    return QZ_SUCCESS;
}
bool state_save(qz_sim *s, SavedState &st)
{
    const long n = s->n;
    if (!st.buf.ensure(s->mem, 9 * n + s->gpts))
        return false;
    const double *src[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    for (int q = 0; q < 9; q++)
        if (!check_cuda(cudaMemcpyAsync(st.buf.p + q * n, src[q], n * sizeof(double),
                                        cudaMemcpyDeviceToDevice, s->stream), "state save"))
            return false;
    st.n = n;
    st.head_mass = s->head_mass;
    st.forces_ready = s->forces_ready;
    st.stats = s->stats;
    return check_cuda(cudaMemcpyAsync(st.buf.p + 9 * n, s->pot, s->gpts * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s->stream), "state save");
}

bool state_restore(qz_sim *s, const SavedState &st)
{
    const long n = st.n;
    double *dst[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    for (int q = 0; q < 9; q++)
        if (!check_cuda(cudaMemcpyAsync(dst[q], st.buf.p + q * n, n * sizeof(double),
                                        cudaMemcpyDeviceToDevice, s->stream), "state restore"))
            return false;
    s->n = n;
    s->head_mass = st.head_mass;
    s->forces_ready = st.forces_ready;
    s->stats = st.stats;
    return check_cuda(cudaMemcpyAsync(s->pot, st.buf.p + 9 * n, s->gpts * sizeof(double),
                                      cudaMemcpyDeviceToDevice, s->stream), "state restore");
}

void state_free(qz_sim *s, SavedState &st) { st.buf.release(s->mem); }

} // namespace qz

extern "C" {

int qz_step(qz_sim *s, double dt, int nsteps)
{
    if (!s)
        return QZ_FAILURE;
    if (!s->forces_ready && qz_init_forces(s))
        return QZ_FAILURE;
    for (int q = 0; q < nsteps; q++)
    {
        double h = dt;
        if (dt <= 0.0 && timestep_cfl(s, &h))
            return QZ_FAILURE;
        if (step_core(s, h))
            return QZ_FAILURE;
    }
    return check_flags(s);
}

// One step on host-resident state.  Page-locked arrays (every one of the ten):
// x..vz and ax..az go in on the simulation's stream, the masses on a second
// stream beside them and the kick-drift (the deposit is the first stage that
// reads them), and the drifted positions come back on the second stream
// while the forces are computed; velocities and accelerations come back after
// the kick.  Pageable arrays: the staged copies of qz_set_particles /
// qz_get_particles around qz_step.  The arithmetic is qz_step's either way.
int qz_step_host(qz_sim *s, double dt, double *x, double *y, double *z, double *vx, double *vy,
                 double *vz, const double *m, double *ax, double *ay, double *az)
{
    if (!s || !(dt > 0.0) || !x || !y || !z || !vx || !vy || !vz || !m || !ax || !ay || !az)
    {
        set_error("qz_step_host: bad arguments (dt must be > 0)");
        return QZ_FAILURE;
    }
    const long n = s->n;
    const void *arrays[10] = {x, y, z, vx, vy, vz, m, ax, ay, az};
    bool pinned = true;
    for (const void *p : arrays)
    {
        cudaPointerAttributes at;
        pinned = pinned && cudaPointerGetAttributes(&at, p) == cudaSuccess &&
                 at.type == cudaMemoryTypeHost;
        cudaGetLastError();
    }
    // outflow boundaries remove particles in the kick-drift: the plain sequence
    if (!pinned || s->cfg.bdry == 2 || n == 0)
        return (qz_set_particles(s, n, x, y, z, vx, vy, vz, m) ||
                qz_set_particle_accel(s, ax, ay, az) || qz_step(s, dt, 1) ||
                qz_get_particles(s, x, y, z, vx, vy, vz, ax, ay, az))
                   ? QZ_FAILURE
                   : QZ_SUCCESS;
    if (!s->xfer &&
        (!check_cuda(cudaStreamCreateWithFlags(&s->xfer, cudaStreamNonBlocking), "copy stream") ||
         !check_cuda(cudaEventCreateWithFlags(&s->ev_mass, cudaEventDisableTiming), "event") ||
         !check_cuda(cudaEventCreateWithFlags(&s->ev_drift, cudaEventDisableTiming), "event")))
        return QZ_FAILURE;
    const size_t b = (size_t)n * sizeof(double);
    double *dst[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    const double *src[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    for (int q = 0; q < 9; q++)
        if (!check_cuda(cudaMemcpyAsync(dst[q], src[q], b, cudaMemcpyHostToDevice, s->stream), "h2d"))
            return QZ_FAILURE;
    // the masses on the second stream: nothing before the deposit reads them
    if (!check_cuda(cudaMemcpyAsync(s->m, m, b, cudaMemcpyHostToDevice, s->xfer), "h2d mass") ||
        !check_cuda(cudaEventRecord(s->ev_mass, s->xfer), "event"))
        return QZ_FAILURE;
    s->head_mass = s->cfg.total_mass;
    s->ofl_removed = 0;
    s->forces_ready = true;
    if (kick_drift(s, dt) || !check_cuda(cudaEventRecord(s->ev_drift, s->stream), "event") ||
        !check_cuda(cudaStreamWaitEvent(s->xfer, s->ev_drift, 0), "wait"))
        return QZ_FAILURE;
    double *hx[3] = {x, y, z};
    const double *dx[3] = {s->x, s->y, s->z};
    for (int q = 0; q < 3; q++)
        if (!check_cuda(cudaMemcpyAsync(hx[q], dx[q], b, cudaMemcpyDeviceToHost, s->xfer), "d2h"))
            return QZ_FAILURE;
    StepPending sp;
    const bool ok = !qz_reset(s) &&
                    check_cuda(cudaStreamWaitEvent(s->stream, s->ev_mass, 0), "wait") &&
                    !tree_density_potential(s, sp) && !qz_grid_acceleration(s) &&
                    !qz_particle_acceleration(s) && !kick(s, dt);
    // the copies back are queued before the step's outcomes are read
    double *ho[6] = {vx, vy, vz, ax, ay, az};
    const double *dout[6] = {s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    bool copied = ok;
    for (int q = 0; q < 6 && copied; q++)
        copied = check_cuda(cudaMemcpyAsync(ho[q], dout[q], b, cudaMemcpyDeviceToHost, s->stream),
                            "d2h");
    if (step_finish(s, sp) || !copied)
    {
        cudaStreamSynchronize(s->xfer);
        cudaStreamSynchronize(s->stream);
        return QZ_FAILURE;
    }
    s->stats.steps++;
    s->stats.last_dt = dt;
    s->stats.sim_time += dt;
    if (!check_cuda(cudaStreamSynchronize(s->xfer), "copy stream sync") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "step sync"))
        return QZ_FAILURE;
    return check_flags(s);
}

int qz_solve_schedule(qz_sim *s, int mode, int *counts, long cap, long *len)
{
    if (!s || mode < 0 || mode > 2 || cap < 0 || (cap > 0 && !counts))
    {
        set_error("qz_solve_schedule: bad arguments");
        return QZ_FAILURE;
    }
    if (mode == 0)
    {
        if (len)
            *len = (long)s->sched.size();
        for (long q = 0; q < cap && q < (long)s->sched.size(); q++)
            counts[q] = s->sched[q];
        s->sched_mode = 0;
        return QZ_SUCCESS;
    }
    if (mode == 1)
    {
        s->sched.clear();
        s->sched_pos = 0;
        s->sched_mode = 1;
        return QZ_SUCCESS;
    }
    s->sched.assign(counts, counts + cap);
    s->sched_pos = 0;
    s->sched_mode = 2;
    return QZ_SUCCESS;
}

int qz_synchronize(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    return check_cuda(cudaStreamSynchronize(s->stream), "synchronize") ? QZ_SUCCESS : QZ_FAILURE;
}

int qz_get_stats(qz_sim *s, qz_stats *out)
{
    if (!s || !out)
        return QZ_FAILURE;
    *out = s->stats;
    out->levels = amr_on(s) ? s->amr_nlev : 1;
    out->nodes = 1;
    if (amr_on(s))
        for (int l = 1; l < s->amr_nlev; l++)
            out->nodes += s->amr[l].nnodes;
    return QZ_SUCCESS;
}

// ---- refinement tree inspection ---------------------------------------------------------
static const AmrNode *tree_node(qz_sim *s, int level, int node)
{
    if (!s || !amr_on(s) || level < 0 || level >= s->amr_nlev || node < 0 ||
        node >= s->amr[level].nnodes)
    {
        set_error("no node %d at level %d", node, level);
        return nullptr;
    }
    return &s->amr[level].h[node];
}

int qz_amr_levels(qz_sim *s) { return !s ? 0 : amr_on(s) ? s->amr_nlev : 1; }

int qz_amr_num_nodes(qz_sim *s, int level)
{
    if (!s || !amr_on(s) || level < 0 || level >= s->amr_nlev)
        return level == 0 && s ? 1 : 0;
    return s->amr[level].nnodes;
}

int qz_amr_node_info(qz_sim *s, int level, int node, int *info, double *mass)
{
    const AmrNode *N = tree_node(s, level, node);
    if (!N || !info)
        return QZ_FAILURE;
    int v[22] = {N->lv, N->parent, N->ts[0], N->ts[1], N->ts[2], N->rd[0], N->rd[1], N->rd[2],
                 N->bmin[0], N->bmin[1], N->bmin[2], N->bmax[0], N->bmax[1], N->bmax[2],
                 N->ncells, N->nintr, N->nbdry, N->nsimb, N->nptcl, N->zone_base, N->nzones,
                 N->contact};
    memcpy(info, v, sizeof v);
    if (mass)
        *mass = N->mass;
    return QZ_SUCCESS;
}

static bool d2h_int(qz_sim *s, int *dst, const int *src, long count)
{
    return count <= 0 ||
           (check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(int), cudaMemcpyDeviceToHost,
                                       s->stream), "tree d2h") &&
            check_cuda(cudaStreamSynchronize(s->stream), "tree d2h sync"));
}

int qz_amr_node_cells(qz_sim *s, int level, int node, int *xyz)
{
    const AmrNode *N = tree_node(s, level, node);
    if (!N || !xyz)
        return QZ_FAILURE;
    return d2h_int(s, xyz, s->amr[level].cell_xyz.p + 3L * N->cell_off, 3L * N->ncells)
               ? QZ_SUCCESS
               : QZ_FAILURE;
}

int qz_amr_node_box(qz_sim *s, int level, int node, int *out)
{
    const AmrNode *N = tree_node(s, level, node);
    if (!N || !out)
        return QZ_FAILURE;
    return d2h_int(s, out, s->amr[level].box.p + N->box_off, (long)N->rd[0] * N->rd[1] * N->rd[2])
               ? QZ_SUCCESS
               : QZ_FAILURE;
}

// which: 0 interior, 1 boundary, 2 simulation boundary; node-local grid indices.
int qz_amr_node_list(qz_sim *s, int level, int node, int which, int *out)
{
    const AmrNode *N = tree_node(s, level, node);
    if (!N || !out || level == 0 || which < 0 || which > 2)
        return QZ_FAILURE;
    AmrLevel &L = s->amr[level];
    const int *src = which == 0 ? L.intr.p + N->intr_off : which == 1 ? L.bdry.p + N->bdry_off
                                                                       : L.simb.p + N->simb_off;
    const int cnt = which == 0 ? N->nintr : which == 1 ? N->nbdry : N->nsimb;
    if (!d2h_int(s, out, src, cnt))
        return QZ_FAILURE;
    for (int i = 0; i < cnt; i++)
        out[i] -= (int)N->grid_off;
    return QZ_SUCCESS;
}

int qz_amr_node_field(qz_sim *s, int level, int node, int which, double *out)
{
    const AmrNode *N = tree_node(s, level, node);
    if (!N || !out)
        return QZ_FAILURE;
    AmrLevel &L = s->amr[level];
    const double *f = which == QZ_FIELD_POT ? L.pot : which == QZ_FIELD_POT_OLD ? L.pot_old
                    : which == QZ_FIELD_DENSITY ? L.d : which == QZ_FIELD_AX ? L.ax
                    : which == QZ_FIELD_AY ? L.ay : which == QZ_FIELD_AZ ? L.az : nullptr;
    if (!f)
    {
        set_error("field %d not available at level %d", which, level);
        return QZ_FAILURE;
    }
    const long cnt = (long)(N->rd[0] + 1) * (N->rd[1] + 1) * (N->rd[2] + 1);
    return check_cuda(cudaMemcpyAsync(out, f + N->grid_off, cnt * sizeof(double),
                                      cudaMemcpyDeviceToHost, s->stream), "field d2h") &&
                   check_cuda(cudaStreamSynchronize(s->stream), "field d2h sync")
               ? QZ_SUCCESS
               : QZ_FAILURE;
}

void *qz_stream(qz_sim *s) { return s ? (void *)s->stream : nullptr; }

int qz_profile_enable(qz_sim *s, int on)
{
    if (!s)
        return QZ_FAILURE;
    if (!check_cuda(cudaStreamSynchronize(s->stream), "profile sync"))
        return QZ_FAILURE;
    prof_collect(s);
    s->prof = on != 0;
    return QZ_SUCCESS;
}

int qz_profile_reset(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    if (!check_cuda(cudaStreamSynchronize(s->stream), "profile sync"))
        return QZ_FAILURE;
    prof_collect(s);
    for (int c = 0; c < QZ_PROF_CATEGORIES; c++)
    {
        s->prof_launches[c] = 0;
        s->prof_ms[c] = 0.0;
        s->prof_bytes[c] = 0.0;
    }
    return QZ_SUCCESS;
}

int qz_profile_read(qz_sim *s, int cat, long long *launches, double *total_ms, double *bytes)
{
    if (!s || cat < 0 || cat >= QZ_PROF_CATEGORIES)
        return QZ_FAILURE;
    if (!check_cuda(cudaStreamSynchronize(s->stream), "profile sync"))
        return QZ_FAILURE;
    prof_collect(s);
    if (launches)
        *launches = s->prof_launches[cat];
    if (total_ms)
        *total_ms = s->prof_ms[cat];
    if (bytes)
        *bytes = s->prof_bytes[cat];
    return QZ_SUCCESS;
}

// ---- array-level wrappers ------------------------------------------------------------
// A minimal context whose fine level is a dense gridsize^3 device copy of the
// caller's arrays.
static qz_sim *dense_context(const qz_config *cfg, int gridsize, double **dphi, double **drho)
{
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    {
        cudaGetLastError();
        set_error("no CUDA device is available (this library has no CPU path)");
        return nullptr;
    }
    qz_sim *s = new qz_sim();
    s->cfg = *cfg;
    s->fused_rb = getenv("QZ_FUSED_RB") != nullptr;
    cudaGetDevice(&s->device);
    size_t pts = (size_t)gridsize * gridsize * gridsize;
    if (!check_cuda(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream") ||
        !make_pool(s) || !dmalloc(&s->gbar, 4, "grid barrier") ||
        !dmalloc(&s->flags, F_COUNT, "flags") || !dmalloc(dphi, pts, "phi") || !dmalloc(drho, pts, "rho") ||
        !check_cuda(cudaMallocHost((void **)&s->h_flags, F_COUNT * sizeof(int)), "pinned"))
    {
        qz_destroy(s);
        return nullptr;
    }
    cudaMemset(s->flags, 0, F_COUNT * sizeof(int));
    s->fine_phi = dense_view(*dphi, gridsize);
    s->fine_rho = dense_view(*drho, gridsize);
    if (!build_levels(s, gridsize) || !dmalloc(&s->fine_alt_buf, pts, "phi alt"))
    {
        qz_destroy(s);
        return nullptr;
    }
    s->fine_alt = dense_view(s->fine_alt_buf, gridsize);
    return s;
}

static int run_dense(const qz_config *cfg, double *phi, const double *rho, int gridsize,
                     int (*body)(qz_sim *, void *), void *arg)
{
    if (!phi || !rho || gridsize < 3 || (long)gridsize * gridsize * gridsize >= (1L << 31))
    {
        set_error("bad grid arguments (3 <= gridsize, gridsize^3 < 2^31)");
        return QZ_FAILURE;
    }
    double *dphi = nullptr, *drho = nullptr;
    qz_sim *s = dense_context(cfg, gridsize, &dphi, &drho);
    if (!s)
        return QZ_FAILURE;
    long pts = (long)gridsize * gridsize * gridsize;
    int rc = (h2d(s, dphi, phi, pts) && h2d(s, drho, rho, pts)) ? body(s, arg) : QZ_FAILURE;
    if (rc == QZ_SUCCESS && !d2h(s, phi, dphi, pts))
        rc = QZ_FAILURE;
    if (rc == QZ_SUCCESS)
        rc = check_flags(s);
    dfree(dphi);
    dfree(drho);
    qz_destroy(s);
    return rc;
}

struct SmoothArg {
    int iters;
};
static int smooth_body(qz_sim *s, void *a)
{
    return smooth(s, s->fine_phi, s->fine_rho, ((SmoothArg *)a)->iters);
}
struct CycleArg {
    int type;
};
static int cycle_body(qz_sim *s, void *a)
{
    sync_fine_alt(s);
    return vcycle(s, 0, ((CycleArg *)a)->type);
}

int qz_gauss_saidel(double *phi, const double *rho, int gridsize, int iter_max, double w,
                    int gs_order)
{
    qz_config c;
    qz_default_config(&c, 2);
    c.smoother = 0;
    c.w_sor = w;
    c.gs_order = gs_order;
    SmoothArg a{iter_max};
    return run_dense(&c, phi, rho, gridsize, smooth_body, &a);
}

int qz_jacobi(double *phi, const double *rho, int gridsize, int iter_max, double w)
{
    qz_config c;
    qz_default_config(&c, 2);
    c.smoother = 1;
    c.w_sor = w;
    SmoothArg a{iter_max};
    return run_dense(&c, phi, rho, gridsize, smooth_body, &a);
}

int qz_conjugate_gradient_multigrid(double *phi, const double *rho, int gridsize, int iters)
{
    qz_config c;
    qz_default_config(&c, 2);
    c.smoother = 2;
    SmoothArg a{iters};
    return run_dense(&c, phi, rho, gridsize, smooth_body, &a);
}

int qz_multigrid(const qz_config *cfg, double *phi, const double *rho, int gridsize,
                 int type_multigrid)
{
    if (!cfg)
        return QZ_FAILURE;
    qz_config c = *cfg;
    c.precision = QZ_PREC_FP64;
    CycleArg a{type_multigrid};
    return run_dense(&c, phi, rho, gridsize, cycle_body, &a);
}

int qz_ptcl_idx_to_box_idx(int lv, int tsx, int tsy, int tsz, int dimx, int dimy, long n,
                           const double *x, const double *y, const double *z, int *out)
{
    if (n <= 0)
        return QZ_SUCCESS;
    if (!x || !y || !z || !out)
        return QZ_FAILURE;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0)
    {
        cudaGetLastError();
        set_error("no CUDA device is available (this library has no CPU path)");
        return QZ_FAILURE;
    }
    double *d[3] = {nullptr, nullptr, nullptr};
    int *dout = nullptr;
    const double *h[3] = {x, y, z};
    bool ok = true;
    for (int c = 0; c < 3 && ok; c++)
        ok = dmalloc(&d[c], n, "box idx") &&
             check_cuda(cudaMemcpy(d[c], h[c], n * sizeof(double), cudaMemcpyHostToDevice),
                        "box idx h2d");
    ok = ok && dmalloc(&dout, n, "box idx");
    if (ok)
    {
        launch_box_idx(0, n, lv, tsx, tsy, tsz, dimx, dimy, d[0], d[1], d[2], dout);
        ok = check_cuda(cudaGetLastError(), "box idx") &&
             check_cuda(cudaMemcpy(out, dout, n * sizeof(int), cudaMemcpyDeviceToHost),
                        "box idx d2h");
    }
    for (int c = 0; c < 3; c++)
        dfree(d[c]);
    dfree(dout);
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

} // extern "C"

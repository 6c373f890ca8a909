// qz_internal.cuh -- device state and kernel declarations of libqzb200.
//
// Memory layout in HBM (one qz_sim):
//   particles  SoA float64 x y z vx vy vz ax ay az m, length n (ID order)
//   head grid  six float64 fields of D^3 points, D = 2^L + 3, index
//              i + j*D + k*D*D (the reference's box grid, initialization.c:248-255);
//              the multigrid finest level is the embedded (2^L+1)^3 solve grid
//              at offset (1,1,1) -- no copy in/out per V-cycle.
//   MG levels  coarse phi / rho of n_l^3 points, n_{l+1} = (n_l + 1) / 2, in
//              float64 (and float32 for the mixed-precision form)
//   deposit    sort keys / permutation (ping-pong), segment tables, per-cell
//              CIC corner sums (8 float64 per occupied cell)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <vector>

#include "../../include/qz_b200.h"
#include <utility>

namespace qz {

// Strided view of an n^3 multigrid level: point (i,j,k) at p[off + i + j*sy + k*sz].
// Every grid has fewer than 2^31 points (head grids of at most (2^9 + 3)^3,
// array-level grids checked at entry), so offsets and strides are 32-bit and
// index arithmetic stays in 32 bits unless a kernel widens it.
template <typename T>
struct Grid {
    T *p;
    int off;
    int sy;
    int sz;
    int n;
};

struct Level {
    int n = 0;
    double *phi = nullptr, *rho = nullptr;  // FP64 correction / right-hand side
    float *phif = nullptr, *rhof = nullptr; // FP32 hierarchy (mixed precision)
    double *scr = nullptr;                  // Jacobi ping-pong buffers (smoother 1)
    float *scrf = nullptr;
    double *alt = nullptr;                  // red-black ping-pong partners (zero boundary)
    float *altf = nullptr;
    double *cgr = nullptr, *cgp = nullptr, *cga = nullptr; // CG smoothing r, p, Ap (smoother 2)
    float *cgrf = nullptr, *cgpf = nullptr, *cgaf = nullptr;
};

// Deposit segments (occupied cells) of more than SEG_LONG particles are reduced
// by a whole block each instead of one warp: the densest cells of a centrally
// concentrated system hold thousands of particles, and one warp walking them
// would set the length of the deposit.
constexpr int SEG_LONG = 256;
constexpr int SEG_LONG_THREADS = 1024;

#ifdef __CUDACC__
// Block-wide sums of acc[0..NV): xor-shuffle trees in each warp, then the warps'
// values added in warp order by thread c < NV, which receives sum c in acc[0]
// (a fixed order: the same inputs give the same bits).  shw holds
// (blockDim / 32) * NV doubles; the caller syncs before reusing it.
template <int NV> __device__ __forceinline__ void seg_block_sums(double (&acc)[NV], double *shw)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < NV; c++)
    {
        double v = acc[c];
        for (int o = 16; o > 0; o >>= 1)
            v += __shfl_xor_sync(0xffffffffu, v, o);
        acc[c] = v;
    }
    if (lane == 0)
    {
#pragma unroll
        for (int c = 0; c < NV; c++)
            shw[w * NV + c] = acc[c];
    }
    __syncthreads();
    if ((int)threadIdx.x < NV)
    {
        double t = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++)
            t += shw[k * NV + threadIdx.x];
        acc[0] = t;
    }
}
#endif

// Device-side flag words (int).
enum Flag {
    F_RATIO_FAIL = 0, // ratio test |phi/phi_old - 1| > tol2 somewhere
    F_CONVERGED = 1,  // result of the last convergence check
    F_ERROR = 2,      // bitmask of bounds errors seen by kernels
    F_NSEG = 3,       // number of occupied cells (deposit segments)
    F_RESID_FAIL = 4, // method-1 pointwise residual failure
    F_AMR_CONV = 5,   // refinement nodes converged in the current level solve
    F_NLONG = 6,      // deposit segments longer than SEG_LONG (listed in long_seg)
    F_COUNT = 8
};
enum ErrorBits { E_PTCL_OUTSIDE = 1, E_SORT_RANGE = 2, E_BARRIER = 8, E_SCAN = 16 };

// Grid-wide barrier of a cooperative launch with bounded waits.  word[0]
// counts arrivals, word[2] is the generation and word[3] is set once a wait of
// this launch gave up (words 2 and 3 are read together by one 64-bit acquire
// load); all four words are zero at launch.  A block arrives with one
// acquire-release atomic add (which also releases the block's writes, ordered
// before it by the block barrier); the last one resets the count and advances
// the generation with a release; the others poll the generation with acquire
// loads.  Two dependent L2 round trips on the critical path: the arrival and
// the poll that sees the new generation.  A wait that hits the poll limit sets
// word[3] and E_BARRIER in flags[F_ERROR]; from then on every barrier of the
// launch returns false at once, so the kernel finishes.
constexpr int GBAR_POLL_LIMIT = 1 << 21;

struct GridBar {
    unsigned *word;
    int *flags;
};

__device__ __forceinline__ unsigned gbar_ld_acquire(const unsigned *p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long gbar_ld_acquire64(const unsigned *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ bool gbar_sync(const GridBar &B, int *sh_ok)
{
    __syncthreads();
    if (threadIdx.x == 0)
    {
        unsigned long long gw = gbar_ld_acquire64(&B.word[2]); // generation | gave-up << 32
        const unsigned gen = (unsigned)gw;
        int ok = (gw >> 32) == 0;
        if (ok)
        {
            unsigned prev;
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;"
                         : "=r"(prev)
                         : "l"(&B.word[0])
                         : "memory");
            if (prev == gridDim.x - 1)
            {
                asm volatile("st.relaxed.gpu.global.u32 [%0], 0;" ::"l"(&B.word[0]) : "memory");
                asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&B.word[2])
                             : "memory");
            }
            else
            {
                int polls = 0;
                for (;;)
                {
                    gw = gbar_ld_acquire64(&B.word[2]);
                    if ((unsigned)gw != gen)
                        break;
                    if ((gw >> 32) != 0 || ++polls > GBAR_POLL_LIMIT)
                    {
                        ok = 0;
                        break;
                    }
                }
            }
        }
        if (!ok)
        {
            atomicExch(&B.word[3], 1u);
            atomicOr(&B.flags[F_ERROR], E_BARRIER);
        }
        *sh_ok = ok;
    }
    __syncthreads();
    return *sh_ok != 0;
}

struct Sort {
    // Stable LSD radix sort of (uint32 key, int32 value) pairs.
    unsigned *k0 = nullptr, *k1 = nullptr;
    int *v0 = nullptr, *v1 = nullptr;
    int *hist = nullptr; // 256 * tiles
    long cap = 0;
    long tiles_cap = 0;
};

// One node of the refinement tree (host and device copies are identical PODs).
// Box coordinates are cell indices at the node's level minus ts; the node's
// grid fields have (rd + 1)^3 points, linear index i + j*(rd_x+1) + k*(rd_x+1)*(rd_y+1)
// (initialize_node.h:63-216, tree_construction.c:1032-2349).
struct AmrNode {
    int lv;          // absolute level
    int parent;      // index in the parent level's node array (-1: head)
    int ts[3];       // box_ts
    int rd[3];       // box_real_dim
    int bmin[3];     // smallest box, level coordinates
    int bmax[3];
    long box_off;    // first cell of the node box in the level's box pool
    long grid_off;   // first point of the node grid in the level's grid pools
    int cell_off, ncells;                 // node cells in the level's cell pool
    int intr_off, nintr, bdry_off, nbdry, simb_off, nsimb; // grid-point lists
    long cls_off;    // first point of the node's classification range
    int zone_base;   // first child (index in the next level)
    int nzones;
    int nptcl;       // particles in the node (no_ptcl_full_node)
    int contact;     // touches the simulation boundary (sim_bdry_contact)
    double mass;     // node_mass
};

struct AmrChunk {
    int node, begin, end; // [begin, end) of the level's interior list, one node
};

// Stream-ordered allocation context of a simulation: the device's memory pool
// (shared by the simulations on the device; it keeps freed memory, release
// threshold at its maximum) and the stream the simulation's work runs on, so
// that growing a buffer never synchronises the device.
struct MemCtx {
    cudaMemPool_t pool = nullptr;
    cudaStream_t stream = nullptr;
};

template <typename T> bool pool_alloc(const MemCtx &m, T **p, long count)
{
    *p = nullptr;
    return cudaMallocFromPoolAsync((void **)p, (size_t)count * sizeof(T), m.pool, m.stream) ==
           cudaSuccess;
}

inline void pool_free(const MemCtx &m, void *p)
{
    if (p)
        cudaFreeAsync(p, m.stream);
}

// Grow-only device buffer (1.5x growth, stream-ordered).
template <typename T>
struct DBuf {
    T *p = nullptr;
    long cap = 0;
    bool ensure(const MemCtx &m, long need)
    {
        if (need < 1)
            need = 1;
        if (p && need <= cap)
            return true;
        long nc = need > cap * 3 / 2 + 1024 ? need : cap * 3 / 2 + 1024;
        pool_free(m, p);
        p = nullptr;
        cap = 0;
        if (!pool_alloc(m, &p, nc))
        {
            p = nullptr;
            return false;
        }
        cap = nc;
        return true;
    }
    void release(const MemCtx &m)
    {
        pool_free(m, p);
        p = nullptr;
        cap = 0;
    }
};

// Device pools of one refinement level.  Level 0 is the head: its grid pools
// alias the head fields and its box is the (2^L + 2)^3 head box.
struct AmrLevel {
    int nnodes = 0;
    std::vector<AmrNode> h;
    DBuf<AmrNode> nodes;
    long box_total = 0, grid_total = 0, cls_total = 0;
    int cell_total = 0, intr_total = 0, bdry_total = 0, simb_total = 0;
    DBuf<int> box;        // cell status (-5 outside sim, -4 not in node, -3 in node,
                          // -1 refine, >= 0 zone id)
    DBuf<int> cnt;        // particles per box cell
    DBuf<int> pos_of_box; // level cell position of a box cell, -1 if none
    DBuf<int> cell_seg;   // deposit segment of a box cell, -1 if none
    DBuf<int> cell_box;   // per cell: level box-pool index
    DBuf<int> cell_xyz;   // per cell: level coordinates (x, y, z)
    DBuf<int> cell_node;  // per cell: node index
    DBuf<int> intr, bdry, simb, intr_node, bdry_node, simb_node; // level grid-pool indices
    double *pot = nullptr, *pot_old = nullptr, *d = nullptr, *ax = nullptr, *ay = nullptr,
           *az = nullptr; // head aliases on level 0
    // conjugate gradient: residual r and the two p buffers (p and Ap, by iteration parity)
    DBuf<double> gpot, gpot_old, gd, gax, gay, gaz, r, p, Ap;
    DBuf<double> apv; // conjugate gradient: Ap at the interior points
    DBuf<double> cg1; // single-reduction conjugate gradient: s and p, two parities each
    DBuf<int> nint; // node chunk ranges, converged flags, ratio-test flags, status
    DBuf<AmrChunk> chunks;
    DBuf<double> chunk_part; // per chunk: two p.Ap and two r.r partials
    DBuf<double> mass_part;  // node mass slices (32 a node)
    DBuf<int> mass_range;    // per node: segment range
    DBuf<int> sor;           // red-black SOR nodes of the level and their iteration counts
    int nchunks = 0;
    int h_active = 0; // host copy of the unconverged-node count at the start of a solve
    std::vector<AmrChunk> hchunks;
    std::vector<int> hnode_chunk; // node chunk ranges and flags uploaded with the chunks
    // warm start (node_warm): the level's solution, nodes and interior mask of the
    // previous solve
    DBuf<double> wpot;
    DBuf<AmrNode> wnodes;
    DBuf<unsigned char> wmask;
    int wnn = 0;
};

} // namespace qz

#define QZ_CG_PART_MAX 1024

namespace qz {
struct Adjoint;  // qz_adjoint.cu
struct NodeMgState; // qz_node_mg.cu
struct Snapshot; // qz_snapshot.cu
}

struct qz_sim {
    qz_config cfg;
    int device = 0;
    cudaStream_t stream = nullptr;
    qz::MemCtx mem; // stream-ordered pool for buffers that grow during a run
    double *cg_part = nullptr; // conjugate-gradient smoothing: 2 x QZ_CG_PART_MAX partial sums
    double *mg_part = nullptr; // mixed head cycles: block partials of the convergence test + result
    int mg_ran = 0, mg_conv = 0; // mixed head cycles: iterations of the last launch, converged
    double mg_cycle_bytes = 0.0; // deferred head launch: profiler bytes of one cycle
    int mg_prof_idx = -1;        // deferred head launch: its profiler record, or -1
    // refinement steps: higher-priority stream of the head solve while the tree
    // and the level deposits run on `stream`, and the fork / join events
    cudaStream_t head_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_head = nullptr;
    bool no_overlap = false; // set by qz_ensemble_step: members stay on one stream
    int mg_ppt_floor = 0;    // fewest finest-level points a thread of the head launch takes
    unsigned *gbar = nullptr;  // grid barrier words of the cooperative launches (4)
    long n = 0, cap = 0;
    double *x = nullptr, *y = nullptr, *z = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;
    double *ax = nullptr, *ay = nullptr, *az = nullptr, *m = nullptr;

    int L = 0;
    long D = 0, gpts = 0;
    double *pot = nullptr, *pot_old = nullptr, *d = nullptr, *gax = nullptr, *gay = nullptr,
           *gaz = nullptr;
    // mixed precision: FP64 residual of the fine grid stored as FP32 rhs, FP32 correction
    float *rf = nullptr, *ef = nullptr;
    std::vector<qz::Level> levels; // levels[0].n = 2^L + 1 (embedded), levels[l>0] owned
    qz::Grid<double> fine_phi{}, fine_rho{}; // level-0 views (head solve grid)
    qz::Grid<double> fine_alt{};             // level-0 red-black ping-pong partner
    double *fine_alt_buf = nullptr;
    float *ef_alt = nullptr;

    // deposit scratch
    qz::Sort sort;
    int *seg_head = nullptr;  // n: 1 at first particle of a cell run
    int *seg_id = nullptr;    // n: exclusive scan of seg_head
    int *seg_start = nullptr; // n + 1
    int *seg_cell = nullptr;  // n
    int *long_seg = nullptr;  // capacity / SEG_LONG + 2: deposit segments left to k_seg_long
    int *cell_seg = nullptr;  // B^3 cells: segment of the cell or -1
    double *cell_sums = nullptr; // 8 * n
    // single-pass scan: per-tile status words (tagged with the call's epoch) and,
    // after them, the tile counter; the host keeps the counter's value at the
    // start of the next call (scan_base) and the epoch
    unsigned long long *scan_st = nullptr;
    long scan_st_cap = 0;
    unsigned long long scan_base = 0;
    unsigned scan_epoch = 0;

    double *red = nullptr; // reduction partials
    int red_blocks = 0;
    int *flags = nullptr;  // device flag words
    int *h_flags = nullptr; // pinned mirror
    unsigned long long *d_ts = nullptr; // time-step reduction words (17)
    unsigned long long *h_ts = nullptr; // pinned: 17 words out, 17 back
    double *h_red = nullptr; // pinned scalar readback
    double *h_stage = nullptr; // pinned staging for host copies
    size_t h_stage_bytes = 0;
    // qz_step_host: second stream for the copies that overlap the step, and its
    // events (masses in, drifted positions ready)
    cudaStream_t xfer = nullptr;
    cudaEvent_t ev_mass = nullptr, ev_drift = nullptr;

    qz_stats stats{};
    bool forces_ready = false;

    // refinement tree (lmax > lmin): levels[0] = head, rebuilt every step
    std::vector<qz::AmrLevel> amr;
    qz::AmrLevel head_cg; // the head as a one-node level (head_pot_method 1)
    qz::AmrLevel node_cg; // one host node solved by the node conjugate gradient (qz_node_conjugate_gradient)
    qz::Adjoint *adj = nullptr; // adjoint buffers (qz_force_vjp, qz_adjoint_final_loss)
    qz::NodeMgState *node_mg = nullptr; // mixed-form refinement-level multigrid buffers
    // Solver schedule (qz_solve_schedule): mode 1 records the iterations of every
    // forward Poisson solve (head: one count; a level: one count per node), mode 2
    // replays recorded counts -- each solve runs exactly its count, without
    // convergence tests, so that runs from perturbed inputs apply the same map.
    int sched_mode = 0;
    std::vector<int> sched;
    size_t sched_pos = 0;
    qz::Snapshot *snap = nullptr; // snapshot staging and writer thread (qz_write_snapshot)
    // the head node's mass (node_mass): the configured total mass, lowered by
    // outflow removals; the convergence tests of the head solve use it
    double head_mass = 0.0;
    // outflow boundaries: advanced state (9 n), flags / scan / removal lists, the
    // last step's removals (count on the host, lists on the device)
    qz::DBuf<double> ofl_state;
    qz::DBuf<int> ofl_int;
    double *h_ofl = nullptr; // pinned: bound, count, head mass
    long ofl_removed = 0;
    long ofl_layout_n = 0; // particle count the lists of the last step were laid out for
    int amr_nlev = 1;                  // levels in use this step
    bool tree_built = false;           // a tree exists (freeze_tree keeps it)
    std::vector<qz::DBuf<int>> node_of; // per level: node of each particle or -1
    qz::DBuf<int> amr_tmp, amr_tmp2;   // scratch (labels, scans, compaction)
    qz::DBuf<int> zone_box;            // per zone: min x,y,z, max x,y,z
    qz::DBuf<int> zone_cells;          // per zone: cells
    qz::DBuf<int> gather_idx;          // small gathers of scan values
    qz::DBuf<double> seg_mass;         // per deposit segment: mass
    int *h_small = nullptr;            // pinned read-back buffer
    long h_small_cap = 0;

    // CUDA graph of one convergence-check block of the head solve
    bool use_graphs = true;
    // one-launch tiled red-black sweep (k_gs_rb_tile) for levels of >= 64
    // interior points per side; off by default (slower than two k_gs_rb
    // launches on B200 at 257^3, see profiles/)
    bool fused_rb = false;
    cudaGraphExec_t check_exec = nullptr;
    long long check_graph_kernels = 0;

    // per-kernel-category timing (qz_profile_*): begin/end events per launch
    bool prof = false;
    struct ProfRec {
        int cat;
        double bytes;
        cudaEvent_t b, e;
    };
    std::vector<ProfRec> prof_pending;
    std::vector<cudaEvent_t> ev_pool;
    long long prof_launches[QZ_PROF_CATEGORIES] = {};
    double prof_ms[QZ_PROF_CATEGORIES] = {};
    double prof_bytes[QZ_PROF_CATEGORIES] = {};
};

namespace qz {

// ---- launch accounting and errors ------------------------------------------
void set_error(const char *fmt, ...);
int timestep_cfl(qz_sim *s, double *dt_out); // qz_observe.cu
int head_cg_solve(qz_sim *s);                 // qz_amr.cu
int solve_zero_bc(qz_sim *s, double *lam, double *f, double rtol, double *scratch,
                  double *host, int *cycles);  // qz_poisson.cu
int check_flags(qz_sim *s);                   // qz_capi.cu
int step_core(qz_sim *s, double dt);          // qz_capi.cu: one fixed-dt step, no flag check
void adjoint_free(qz_sim *s);                 // qz_adjoint.cu
int node_mg_level(qz_sim *s, AmrLevel &L, int level_index); // qz_node_mg.cu
// solver schedule (qz_capi.cu): counts of the next solve in replay mode (false and
// an error when the schedule is exhausted); append in record mode
bool sched_take(qz_sim *s, int n, int *out);
void sched_put(qz_sim *s, const int *v, int n);
void node_mg_free(qz_sim *s);                               // qz_node_mg.cu
void snapshot_free(qz_sim *s);                // qz_snapshot.cu
// A copy of the state a step reads (particles, accelerations, head potential)
// and of the statistics, to run trial steps and put the simulation back
// (qz_capi.cu).
struct SavedState {
    DBuf<double> buf;
    long n = 0;
    double head_mass = 0.0;
    bool forces_ready = false;
    qz_stats stats{};
};
bool state_save(qz_sim *s, SavedState &st);
bool state_restore(qz_sim *s, const SavedState &st);
void state_free(qz_sim *s, SavedState &st);
bool check_cuda(cudaError_t e, const char *what);
#define QZ_LAUNCHED(sim) ((sim)->stats.kernel_launches++)

cudaEvent_t prof_event(qz_sim *s);
void prof_collect(qz_sim *s);

// Launches kernel k on the library stream; counts it, and when profiling is
// on brackets it with events and books `bytes` algorithmic bytes to `cat`.
template <typename... KArgs, typename... Args>
inline void launch_shm(qz_sim *s, int cat, double bytes, size_t shm, void (*k)(KArgs...), dim3 g,
                       dim3 b, Args &&...args)
{
    cudaEvent_t eb = nullptr, ee = nullptr;
    if (s->prof)
    {
        eb = prof_event(s);
        ee = prof_event(s);
        cudaEventRecord(eb, s->stream);
    }
    k<<<g, b, shm, s->stream>>>(std::forward<Args>(args)...);
    s->stats.kernel_launches++;
    if (s->prof)
    {
        cudaEventRecord(ee, s->stream);
        s->prof_pending.push_back({cat, bytes, eb, ee});
    }
}

template <typename... KArgs, typename... Args>
inline void launch(qz_sim *s, int cat, double bytes, void (*k)(KArgs...), dim3 g, dim3 b,
                   Args &&...args)
{
    cudaEvent_t eb = nullptr, ee = nullptr;
    if (s->prof)
    {
        eb = prof_event(s);
        ee = prof_event(s);
        cudaEventRecord(eb, s->stream);
    }
    k<<<g, b, 0, s->stream>>>(std::forward<Args>(args)...);
    s->stats.kernel_launches++;
    if (s->prof)
    {
        cudaEventRecord(ee, s->stream);
        s->prof_pending.push_back({cat, bytes, eb, ee});
    }
}

// ---- kernels-side entry points (host wrappers) ------------------------------
int head_initial(qz_sim *s);
int deposit_head(qz_sim *s);
int grid_accel_head(qz_sim *s);
int grid_accel_head_from(qz_sim *s, const double *pot);
int head_segments(qz_sim *s, const double *x, const double *y, const double *z, int **perm_out);
int deposit_segments(qz_sim *s, long m, int bits, int *cell_seg, long ncells_box,
                     unsigned **ks_out, int **perm_out, unsigned morton_B);
int gather_head(qz_sim *s);
int kick_drift(qz_sim *s, double dt);
int kick(qz_sim *s, double dt);

int potential_head(qz_sim *s);
int amr_init(qz_sim *s);
void amr_free(qz_sim *s);
int amr_build(qz_sim *s);
int amr_reassign(qz_sim *s); // frozen tree: particles to the existing nodes
int cg_level_adjoint(qz_sim *s, int l, double *lam, double *rhs, double *scratch,
                     const double *thr_dev, const std::vector<char> &skip);
int amr_deposit(qz_sim *s);
int amr_potential(qz_sim *s);
// What the host needs after a level's conjugate-gradient launch: where its
// status words are and how its outcome is booked.
struct CgPending {
    bool launched = false; // a cooperative launch was queued (else nothing to read)
    bool record = false, replay = false, one = false, pipe = false;
    int nn = 0;
    const int *status = nullptr; // status (3) then iterations (nn)
    int prof_idx = -1;           // the launch's profiler record, or -1
};
bool amr_potential_queues(const qz_sim *s);
int amr_potential_issue(qz_sim *s, std::vector<CgPending> &pend);
int amr_potential_collect(qz_sim *s, const std::vector<CgPending> &pend);
int amr_grid_accel(qz_sim *s);
int amr_gather(qz_sim *s);
int poisson_error_head(qz_sim *s, int *converged);
bool head_one_launch(const qz_sim *s);
int potential_head_issue(qz_sim *s, cudaStream_t st, bool *issued);
int potential_head_finish(qz_sim *s, cudaStream_t st);
int smooth(qz_sim *s, Grid<double> phi, Grid<double> rho, int iters);
void sync_fine_alt(qz_sim *s);
void init_kernel_attributes();
int vcycle(qz_sim *s, int level, int type);

int radix_sort_pairs(qz_sim *s, long n, int bits, unsigned **keys_out, int **vals_out);
long radix_tiles(long n);
int scan_exclusive(qz_sim *s, const int *in, int *out, long n);
int scan_wait_probe(qz_sim *s);
bool ensure_sort(qz_sim *s, long need); // qz_amr.cu: radix-sort buffers for need pairs
void scan_set_epoch(qz_sim *s, unsigned epoch);

// grid views
inline Grid<double> head_view(qz_sim *s, double *field)
{
    Grid<double> g;
    g.p = field;
    g.off = 1 + s->D + s->D * s->D;
    g.sy = s->D;
    g.sz = s->D * s->D;
    g.n = (1 << s->L) + 1;
    return g;
}
template <typename T>
inline Grid<T> dense_view(T *p, int n)
{
    Grid<T> g;
    g.p = p;
    g.off = 0;
    g.sy = n;
    g.sz = (long)n * n;
    g.n = n;
    return g;
}

inline int blocks_for(long n, int threads)
{
    long b = (n + threads - 1) / threads;
    return (int)(b < 1 ? 1 : b);
}

} // namespace qz

// qz_node_mg.cu -- mixed-precision Poisson solves of the refinement nodes:
// FP32 multigrid V-cycles inside FP64 defect correction, one thread-block
// cluster per node.
//
// The reference solves every refinement node by unpreconditioned conjugate
// gradient in FP64 (potential_branches.c:401-532 -> conjugate_gradient.c:
// 322-463), checking the node every 5 iterations with the ratio test against
// the previous check and the residual test of conj_grad_error
// (poisson_error.c:36-81, 236-288).  The plain FP64 path of this library keeps
// that solver (k_cg_nodes, qz_amr.cu).  The mixed-precision form replaces it
// by defect correction:
//
//   repeat:  r = d - Lap_H(phi)                      (FP64, interior points)
//            convergence test on phi (ratio test against the previous iterate,
//            residual test on r: the reference's test, FP64)
//            z ~= Lap_H^-1 r by one FP32 V-cycle      (zero on non-interior points)
//            phi += alpha p, p = z + beta p_old       (FP64)
//
// with alpha and beta those of the flexible conjugate gradient (Notay 2000,
// Polak-Ribiere beta = r.(z - z_old) / (r_old.z_old), alpha = r.z / p.Lap p).
// Plain defect correction (phi += z) converges slowly on refinement nodes: a
// node's interior ends at odd fine-grid coordinates (zone surfaces are faces of
// parent cells), so every coarse level places its zero boundary up to one of
// its cells outside the true one and over-corrects the smoothest error (at
// 1M particles, 128^3 head, three levels: 40-300 iterations, one node not
// converging in 5000).  The conjugate-gradient step makes the cycle a
// preconditioner and removes that sensitivity.
//
// The V-cycle works on the node's grid box with a mask: level 0 is the node
// grid ((rd + 1)^3 points, unknowns at the node's interior points, in the
// node's colour-coded interior list), level k + 1 has ceil(c_k / 2) cells per
// axis and a point X is an unknown when the fine point 2^k X is an interior
// point (every other point holds zero: homogeneous Dirichlet values for the
// correction).  Smoothing is red-black Gauss-Seidel with the arithmetic of the
// head's sweeps (k_gs_rb: phi = (sum of neighbours - h^2 rho) / 6), restriction
// takes half the residual at the coincident fine point (the red-black head
// cycle's half injection), prolongation is trilinear and adds at unknowns
// only.  The coarsest level (at most 4 cells per axis) is solved by FP64
// red-black sweeps.
//
// Execution: one cluster of CS CTAs (16 where the device allows, else 8) per
// node, all nodes of a level in one launch.  Phases are separated by hardware
// cluster barriers (barrier.cluster arrive.release / wait.acquire), which make
// every store before a barrier visible to every load after it across the
// cluster (plain, L1-cached loads).
// The fine level and the first coarse levels are swept by the whole cluster;
// the levels small enough for shared memory run as a sub-cycle inside CTA 0
// while the others wait at the next cluster barrier.  The FP64 residual pass
// also forms the new iterate: phi_{k+1} = phi_k + e is written to the other of
// the node's two potential buffers (pot / pot_old), so the ratio test compares
// the two buffers without a copy; a node that stops with its iterate in
// pot_old copies its interior points back to pot.  Residual sums: warp
// shuffle trees, warps in order, CTAs in rank order read through distributed
// shared memory -- every CTA obtains the same sums and takes the same
// decisions, and runs are bit-reproducible.  A node that does not converge
// within max_iter iterations fails the solve, as the reference's solver does.
#include <cooperative_groups.h>
#include <mutex>
#include <stdlib.h>

#include "qz_amr_dev.cuh"

namespace cg = cooperative_groups;

namespace qz {

#define QZ_PI_NMG 3.14159265358979323846

constexpr int NMG_THREADS = 512;
constexpr int NMG_MAXLEV = 10;
constexpr size_t NMG_SMEM_MAX = 160 * 1024; // shared-memory sub-cycle (CTA 0)
constexpr int NMG_COARSE_SWEEPS = 8; // FP64 red-black sweeps on the coarsest level (default)
// Red-black sweeps before and after each coarse correction.  Measured on the
// 1M-particle sphere with three refinement levels (node solves per step): 2
// sweeps 69 iterations, 14.9 ms; 3 sweeps 36, 9.7 ms; 4 sweeps 27, 8.6 ms.
constexpr int NMG_SWEEPS = 4;

struct NmgLev {
    int nx, ny, nz; // points per axis
    long off;       // first point in the coarse pools (levels >= 1)
};

struct NmgNode {
    int q;          // node index in the level
    int nlev;       // multigrid levels (0: the node grid)
    int nsmall;     // first level of CTA 0's shared-memory sub-cycle (>= 1)
    int ib, ie;     // the node's range of the level's interior list
    long goff;      // node grid offset in the level's grid pools
    double oh2;     // 1 / H^2
    double thr;     // residual test: r.r threshold (check methods 0 and 2)
    double rmt;     // check method 1: tol * (4 pi G rho_mean)
    int cap;        // most iterations (a replayed schedule: exactly this many)
    int replay;     // no convergence test: run cap iterations
    int smem_need;  // bytes of the sub-cycle
    float h2[NMG_MAXLEV];
    NmgLev lv[NMG_MAXLEV];
    int soff[NMG_MAXLEV]; // sub-cycle levels: byte offset of e (float), f (float), mask (uchar)
    int coff;             // coarsest level FP64 arrays (e, f)
};

struct NmgArgs {
    const NmgNode *tab;
    const int *intr;       // level interior list (grid-pool indices)
    int *cl;               // the list by colour within each CTA's slice
    const double *d;
    double *pot, *pot_old; // the node's two potential buffers
    float *ef, *rf;        // level 0 correction and residual (grid-pool layout)
    unsigned char *msk;    // level 0 interior mask (grid-pool layout)
    float *ec, *fc;        // coarse levels
    unsigned char *mc;
    int *status;           // per entry: converged, iterations
    double *pv;            // flexible CG direction (grid-pool layout, zero off the interior)
    float *efo;            // the previous preconditioned residual (interior points)
    double tol2;
    int method;
    int n_pre, n_post;
    int n_coarse; // red-black sweeps of the coarsest level
};

// ---- small helpers ------------------------------------------------------------------------
// Loads of data that other CTAs of the cluster wrote earlier in the launch:
// plain (L1-cached) loads.  Every phase ends at a cluster barrier whose arrive
// has release and whose wait has acquire semantics at cluster scope, so by the
// PTX memory model a load after the barrier observes every store made before
// it by any thread of the cluster; neighbouring stencil points then share L1
// lines instead of each load going to L2.
__device__ __forceinline__ float ldg_f(const float *p) { return *p; }
__device__ __forceinline__ double ldg_d(const double *p) { return *p; }
__device__ __forceinline__ unsigned char ldg_u8(const unsigned char *p) { return *p; }
template <typename T> __device__ __forceinline__ void stg(T *p, T v) { *p = v; }

// Items of one colour of a dense level: rows (j, k) over the interior, i of the
// row's parity.  Item t -> (i, j, k) or false when beyond the row.
struct ColourWalk {
    int mx, my, mz, hmax;
    long items;
    __device__ ColourWalk(int nx, int ny, int nz)
    {
        mx = nx - 2;
        my = ny - 2;
        mz = nz - 2;
        hmax = (mx + 1) / 2;
        items = (mx > 0 && my > 0 && mz > 0) ? (long)hmax * my * mz : 0;
    }
    // item counts stay below 2^31 (a level has at most the node grid's points)
    __device__ bool at(long t, int col, int &i, int &j, int &k) const
    {
        const unsigned tt = (unsigned)t, hm = (unsigned)hmax;
        const unsigned row = tt / hm;
        const int u = (int)(tt - row * hm);
        const unsigned kk = row / (unsigned)my;
        j = 1 + (int)(row - kk * (unsigned)my);
        k = 1 + (int)kk;
        i = ((((1 + j + k) & 1) == col) ? 1 : 2) + 2 * u;
        return i <= mx;
    }
};

// One colour of a red-black sweep of a dense level.  G: arrays in global
// memory (L2 loads).  FIRST: the level's correction starts at zero (the other
// colour's values are not read).
template <bool G, typename T>
__device__ __forceinline__ void dense_sweep(T *e, const T *f, const unsigned char *m, int nx, int ny,
                                            int nz, T h2, int col, bool first, long t0, long nt)
{
    const ColourWalk W(nx, ny, nz);
    const long sy = nx, sz = (long)nx * ny;
    const T one_sixth = (T)(1.0 / 6.0);
    for (long t = t0; t < W.items; t += nt)
    {
        int i, j, k;
        if (!W.at(t, col, i, j, k))
            continue;
        const long x = i + j * sy + k * sz;
        const unsigned char a = G ? ldg_u8(m + x) : m[x];
        if (!a)
            continue;
        T fx, s;
        if constexpr (G)
        {
            fx = ldg_f(f + x);
            s = first ? (T)0
                      : ldg_f(e + x + 1) + ldg_f(e + x - 1) + ldg_f(e + x + sy) + ldg_f(e + x - sy) +
                            ldg_f(e + x + sz) + ldg_f(e + x - sz);
        }
        else
        {
            fx = f[x];
            s = first ? (T)0 : e[x + 1] + e[x - 1] + e[x + sy] + e[x - sy] + e[x + sz] + e[x - sz];
        }
        const T v = one_sixth * (-h2 * fx + s);
        if constexpr (G)
            stg(e + x, v);
        else
            e[x] = v;
    }
}

// Residual of the fine level (k-1) at 2X, halved, into the coarse rhs at the
// coarse unknowns X of a dense level k.  GF: the fine arrays are global; GC:
// the coarse ones are.
template <bool GF, bool GC>
__device__ __forceinline__ void dense_restrict(const float *ef, const float *ff, int fnx, int fny,
                                               float foh2, float *fcrs, const unsigned char *mcrs,
                                               int nx, int ny, int nz, long t0, long nt)
{
    const long fsy = fnx, fsz = (long)fnx * fny;
    const long sy = nx, sz = (long)nx * ny;
    const int mx = nx - 2, my = ny - 2, mz = nz - 2;
    if (mx < 1 || my < 1 || mz < 1)
        return;
    const long items = (long)mx * my * mz;
    for (long t = t0; t < items; t += nt)
    {
        const unsigned tt = (unsigned)t, r = tt / (unsigned)mx;
        const int i = 1 + (int)(tt - r * (unsigned)mx);
        const unsigned rk = r / (unsigned)my;
        const int j = 1 + (int)(r - rk * (unsigned)my), k = 1 + (int)rk;
        const long x = i + j * sy + k * sz;
        if (!(GC ? ldg_u8(mcrs + x) : mcrs[x]))
            continue;
        const long g = 2L * i + 2L * j * fsy + 2L * k * fsz;
        float c, s;
        if (GF)
        {
            c = ldg_f(ef + g);
            s = ldg_f(ef + g + 1) + ldg_f(ef + g - 1) + ldg_f(ef + g + fsy) + ldg_f(ef + g - fsy) +
                ldg_f(ef + g + fsz) + ldg_f(ef + g - fsz);
        }
        else
        {
            c = ef[g];
            s = ef[g + 1] + ef[g - 1] + ef[g + fsy] + ef[g - fsy] + ef[g + fsz] + ef[g - fsz];
        }
        const float rv = (GF ? ldg_f(ff + g) : ff[g]) + foh2 * (6.0f * c - s);
        const float v = 0.5f * rv;
        if (GC)
            stg(fcrs + x, v);
        else
            fcrs[x] = v;
    }
}

// Trilinear value of the coarse correction at fine point (i, j, k).
template <bool G>
__device__ __forceinline__ float prolong_at(const float *ec, int cnx, int cny, int i, int j, int k)
{
    const long csy = cnx, csz = (long)cnx * cny;
    const int x0 = i >> 1, x1 = (i + 1) >> 1, y0 = j >> 1, y1 = (j + 1) >> 1, z0 = k >> 1,
              z1 = (k + 1) >> 1;
    auto E = [&](int a, int b, int c) -> float {
        const long x = a + b * csy + c * csz;
        return G ? ldg_f(ec + x) : ec[x];
    };
    const float wx = (i & 1) ? 0.5f : 1.0f, wy = (j & 1) ? 0.5f : 1.0f, wz = (k & 1) ? 0.5f : 1.0f;
    float acc = E(x0, y0, z0);
    if (i & 1)
        acc += E(x1, y0, z0);
    if (j & 1)
    {
        acc += E(x0, y1, z0);
        if (i & 1)
            acc += E(x1, y1, z0);
    }
    if (k & 1)
    {
        acc += E(x0, y0, z1);
        if (i & 1)
            acc += E(x1, y0, z1);
        if (j & 1)
        {
            acc += E(x0, y1, z1);
            if (i & 1)
                acc += E(x1, y1, z1);
        }
    }
    return wx * wy * wz * acc;
}

// e_k += P e_{k+1} at the unknowns of a dense level k.
template <bool GF, bool GC>
__device__ __forceinline__ void dense_prolong(float *e, const unsigned char *m, int nx, int ny,
                                              int nz, const float *ec, int cnx, int cny, long t0,
                                              long nt)
{
    const long sy = nx, sz = (long)nx * ny;
    const int mx = nx - 2, my = ny - 2, mz = nz - 2;
    if (mx < 1 || my < 1 || mz < 1)
        return;
    const long items = (long)mx * my * mz;
    for (long t = t0; t < items; t += nt)
    {
        const unsigned tt = (unsigned)t, r = tt / (unsigned)mx;
        const int i = 1 + (int)(tt - r * (unsigned)mx);
        const unsigned rk = r / (unsigned)my;
        const int j = 1 + (int)(r - rk * (unsigned)my), k = 1 + (int)rk;
        const long x = i + j * sy + k * sz;
        if (!(GF ? ldg_u8(m + x) : m[x]))
            continue;
        const float add = prolong_at<GC>(ec, cnx, cny, i, j, k);
        if (GF)
            stg(e + x, ldg_f(e + x) + add);
        else
            e[x] += add;
    }
}

// ---- the kernel -------------------------------------------------------------------------
__global__ void __launch_bounds__(NMG_THREADS, 1) k_node_mg(const __grid_constant__ NmgArgs A)
{
    cg::cluster_group cluster = cg::this_cluster();
    const int CS = (int)cluster.num_blocks();
    const int rank = (int)cluster.block_rank();
    const int ent = (int)(blockIdx.x / CS);
    __shared__ NmgNode N;
    __shared__ double wsum[32], wsum2[32];
    __shared__ int wflag[32];
    // this CTA's partials of the three reductions of an iteration (read by the
    // others through distributed shared memory; one slot set per reduction, so a
    // slot is rewritten only an iteration later, many cluster barriers on)
    __shared__ double part_d[3][2];
    __shared__ int part_f[3];
    __shared__ double tot_d[2];
    __shared__ int tot_f;
    extern __shared__ __align__(16) unsigned char nmg_dyn[];
    const int tid = threadIdx.x, NT = blockDim.x;
    if (tid == 0)
        N = A.tab[ent];
    __syncthreads();
    const long ct = (long)rank * NT + tid, CT = (long)CS * NT;
    const int nl = N.ie - N.ib;
    const int sb = N.ib + (int)((long)nl * rank / CS), se = N.ib + (int)((long)nl * (rank + 1) / CS);
    const NmgLev L0 = N.lv[0];
    const long sy0 = L0.nx, sz0 = (long)L0.nx * L0.ny;
    float *ef = A.ef + N.goff;
    float *rf = A.rf + N.goff;
    unsigned char *mk0 = A.msk + N.goff;

    // set-up 1: the fine mask, and this CTA's slice of the interior list split by
    // colour into cl (even points from sb up, odd points from se down; the order
    // inside a colour does not matter to a sweep, and the sums below walk the
    // interior list itself, in its fixed order)
    __shared__ int s_nred, s_nblk;
    if (tid == 0)
        s_nred = s_nblk = 0;
    __syncthreads();
    for (int e = sb + tid; e < se; e += NT)
    {
        const int g = A.intr[e];
        long l = g - N.goff;
        const int z = (int)(l / sz0);
        l -= z * sz0;
        const int y = (int)(l / sy0);
        const int x = (int)(l - y * sy0);
        if ((x + y + z) & 1)
            A.cl[se - 1 - atomicAdd(&s_nblk, 1)] = g;
        else
            A.cl[sb + atomicAdd(&s_nred, 1)] = g;
        stg(A.msk + g, (unsigned char)1);
    }
    __syncthreads();
    const int nred = s_nred; // cl[sb, sb + nred): even points; [sb + nred, se): odd
    cluster.sync();
    // set-up 2: coarse masks, X is an unknown where the fine point 2^k X is one
    for (int k = 1; k < N.nlev; k++)
    {
        const NmgLev Lk = N.lv[k];
        const int mx = Lk.nx - 2, my = Lk.ny - 2, mz = Lk.nz - 2;
        if (mx < 1 || my < 1 || mz < 1)
            continue;
        const long items = (long)mx * my * mz;
        for (long t = ct; t < items; t += CT)
        {
            const unsigned tt = (unsigned)t, r = tt / (unsigned)mx;
            const int i = 1 + (int)(tt - r * (unsigned)mx);
            const unsigned rk = r / (unsigned)my;
            const int j = 1 + (int)(r - rk * (unsigned)my), kk = 1 + (int)rk;
            const long g = ((long)i << k) + ((long)j << k) * sy0 + ((long)kk << k) * sz0;
            A.mc[Lk.off + i + (long)j * Lk.nx + (long)kk * Lk.nx * Lk.ny] = ldg_u8(mk0 + g);
        }
    }
    cluster.sync();
    // CTA 0: zero the sub-cycle arrays once and copy their masks
    if (rank == 0)
    {
        for (int k = N.nsmall; k < N.nlev; k++)
        {
            const NmgLev Lk = N.lv[k];
            const long P = (long)Lk.nx * Lk.ny * Lk.nz;
            float *se_ = reinterpret_cast<float *>(nmg_dyn + N.soff[k]);
            float *sf_ = se_ + P;
            unsigned char *sm_ = reinterpret_cast<unsigned char *>(sf_ + P);
            for (long t = tid; t < P; t += NT)
            {
                se_[t] = 0.0f;
                sf_[t] = 0.0f;
                sm_[t] = ldg_u8(A.mc + Lk.off + t);
            }
        }
        __syncthreads();
    }

    auto sub_e = [&](int k) { return reinterpret_cast<float *>(nmg_dyn + N.soff[k]); };
    auto sub_f = [&](int k) {
        return reinterpret_cast<float *>(nmg_dyn + N.soff[k]) + (long)N.lv[k].nx * N.lv[k].ny * N.lv[k].nz;
    };
    auto sub_m = [&](int k) {
        const long P = (long)N.lv[k].nx * N.lv[k].ny * N.lv[k].nz;
        return reinterpret_cast<unsigned char *>(reinterpret_cast<float *>(nmg_dyn + N.soff[k]) + 2 * P);
    };
    auto ge = [&](int k) { return k == 0 ? ef : A.ec + N.lv[k].off; };
    auto gf = [&](int k) { return k == 0 ? rf : A.fc + N.lv[k].off; };

    // one colour of a sweep of the fine level over this CTA's slice of the list
    // one colour of a sweep of the fine level over this CTA's points of that
    // colour, NB points a thread at a time (their loads in flight together; points
    // of one colour are never neighbours)
    constexpr int NB = 4;
    auto fine_sweep = [&](int col, bool first) {
        const float h2 = N.h2[0];
        const float one_sixth = (float)(1.0 / 6.0);
        const int b0 = col == 0 ? sb : sb + nred, b1 = col == 0 ? sb + nred : se;
        for (int e0 = b0 + tid; e0 < b1; e0 += NB * NT)
        {
            long g[NB];
            float fx[NB], sm[NB];
#pragma unroll
            for (int u = 0; u < NB; u++)
            {
                const int e = e0 + u * NT;
                g[u] = e < b1 ? (long)A.cl[e] : -1L;
            }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                {
                    const long x = g[u];
                    fx[u] = ldg_f(A.rf + x);
                    sm[u] = first ? 0.0f
                                  : ldg_f(A.ef + x + 1) + ldg_f(A.ef + x - 1) + ldg_f(A.ef + x + sy0) +
                                        ldg_f(A.ef + x - sy0) + ldg_f(A.ef + x + sz0) +
                                        ldg_f(A.ef + x - sz0);
                }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                    stg(A.ef + g[u], one_sixth * (-h2 * fx[u] + sm[u]));
        }
    };

    // Cluster-wide sums of (a, b) and OR of f in slot set `slot`: warp trees,
    // warps in order, CTAs in rank order; every CTA gets the same values.
    auto reduce = [&](int slot, double a, double b, int f) {
        for (int o = 16; o > 0; o >>= 1)
        {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            b += __shfl_xor_sync(0xffffffffu, b, o);
        }
        f = (int)__reduce_or_sync(0xffffffffu, (unsigned)f);
        if ((tid & 31) == 0)
        {
            wsum[tid >> 5] = a;
            wsum2[tid >> 5] = b;
            wflag[tid >> 5] = f;
        }
        __syncthreads();
        if (tid == 0)
        {
            double t = 0.0, u = 0.0;
            int g = 0;
            for (int w = 0; w < (NT >> 5); w++)
            {
                t += wsum[w];
                u += wsum2[w];
                g |= wflag[w];
            }
            part_d[slot][0] = t;
            part_d[slot][1] = u;
            part_f[slot] = g;
        }
        cluster.sync();
        if (tid == 0)
        {
            double t = 0.0, u = 0.0;
            int g = 0;
            for (int r = 0; r < CS; r++)
            {
                const double *pr = cluster.map_shared_rank(&part_d[slot][0], r);
                t += pr[0];
                u += pr[1];
                g |= *cluster.map_shared_rank(&part_f[slot], r);
            }
            tot_d[0] = t;
            tot_d[1] = u;
            tot_f = g;
        }
        __syncthreads();
    };

    double *bufs[2] = {A.pot, A.pot_old};
    int it = 0;
    bool conv = false;
    double alpha = 0.0, rz_prev = 1.0;
    for (;;)
    {
        // FP64: new iterate phi + alpha p, its residual (FP32 copy for the cycle),
        // ratio test against the previous iterate
        const double *ph = bufs[it & 1];
        double *pn = bufs[(it + 1) & 1];
        double acc = 0.0;
        int fl = 0; // 1: ratio test failed, 2: point residual test failed (method 1)
        auto P = [&](long x) -> double {
            return it > 0 ? ldg_d(ph + x) + alpha * ldg_d(A.pv + x) : ldg_d(ph + x);
        };
        for (int e0 = sb + tid; e0 < se; e0 += 2 * NT)
        {
            long g[2];
            double c0[2], r[2], old[2];
#pragma unroll
            for (int u = 0; u < 2; u++)
            {
                const int e = e0 + u * NT;
                g[u] = e < se ? (long)A.intr[e] : -1L;
            }
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (g[u] >= 0)
                {
                    const long x = g[u];
                    old[u] = ldg_d(ph + x);
                    c0[u] = P(x);
                    r[u] = A.d[x] + N.oh2 * (6.0 * c0[u] - P(x + 1) - P(x - 1) - P(x + sy0) -
                                             P(x - sy0) - P(x + sz0) - P(x - sz0));
                }
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (g[u] >= 0)
                {
                    stg(pn + g[u], c0[u]);
                    stg(A.rf + g[u], (float)r[u]);
                    acc += r[u] * r[u];
                    const double aux = c0[u] / old[u];
                    if ((1.0 - A.tol2 > aux) || (1.0 + A.tol2 < aux))
                        fl |= 1;
                    if (A.method == 1 && fabs(r[u]) >= N.rmt)
                        fl |= 2;
                }
        }
        reduce(0, acc, 0.0, fl);
        conv = !N.replay && it > 0 && !(tot_f & 1) &&
               (A.method == 1 ? !(tot_f & 2) : tot_d[0] < N.thr);
        if (conv || it >= N.cap)
            break;

        // ---- one FP32 V-cycle on (ef, rf) -----------------------------------------
        for (int sw = 0; sw < A.n_pre; sw++)
            for (int col = 0; col < 2; col++)
            {
                fine_sweep(col, sw == 0 && col == 0);
                cluster.sync();
            }
        for (int k = 1; k < N.nsmall; k++)
        {
            const NmgLev F = N.lv[k - 1], C = N.lv[k];
            dense_restrict<true, true>(ge(k - 1), gf(k - 1), F.nx, F.ny, 1.0f / N.h2[k - 1],
                                       A.fc + C.off, A.mc + C.off, C.nx, C.ny, C.nz, ct, CT);
            cluster.sync();
            for (int sw = 0; sw < A.n_pre; sw++)
                for (int col = 0; col < 2; col++)
                {
                    dense_sweep<true, float>(A.ec + C.off, A.fc + C.off, A.mc + C.off, C.nx, C.ny,
                                             C.nz, N.h2[k], col, sw == 0 && col == 0, ct, CT);
                    cluster.sync();
                }
        }
        if (rank == 0)
        {
            // sub-cycle of the small levels in shared memory
            const int ks = N.nsmall;
            {
                const NmgLev F = N.lv[ks - 1], C = N.lv[ks];
                dense_restrict<true, false>(ge(ks - 1), gf(ks - 1), F.nx, F.ny, 1.0f / N.h2[ks - 1],
                                            sub_f(ks), sub_m(ks), C.nx, C.ny, C.nz, tid, NT);
                __syncthreads();
            }
            for (int k = ks; k < N.nlev - 1; k++)
            {
                const NmgLev C = N.lv[k], D = N.lv[k + 1];
                for (int sw = 0; sw < A.n_pre; sw++)
                    for (int col = 0; col < 2; col++)
                    {
                        dense_sweep<false, float>(sub_e(k), sub_f(k), sub_m(k), C.nx, C.ny, C.nz,
                                                  N.h2[k], col, sw == 0 && col == 0, tid, NT);
                        __syncthreads();
                    }
                dense_restrict<false, false>(sub_e(k), sub_f(k), C.nx, C.ny, 1.0f / N.h2[k],
                                             sub_f(k + 1), sub_m(k + 1), D.nx, D.ny, D.nz, tid, NT);
                __syncthreads();
            }
            {
                // coarsest level: FP64 red-black sweeps from zero
                const int k = N.nlev - 1;
                const NmgLev C = N.lv[k];
                const long P = (long)C.nx * C.ny * C.nz;
                double *e64 = reinterpret_cast<double *>(nmg_dyn + N.coff);
                double *f64 = e64 + P;
                const float *fk = sub_f(k);
                for (long t = tid; t < P; t += NT)
                {
                    e64[t] = 0.0;
                    f64[t] = (double)fk[t];
                }
                __syncthreads();
                const double h2 = (double)N.h2[k];
                for (int sw = 0; sw < A.n_coarse; sw++)
                    for (int col = 0; col < 2; col++)
                    {
                        dense_sweep<false, double>(e64, f64, sub_m(k), C.nx, C.ny, C.nz, h2, col,
                                                   false, tid, NT);
                        __syncthreads();
                    }
                float *ek = sub_e(k);
                const unsigned char *mk = sub_m(k);
                for (long t = tid; t < P; t += NT)
                    if (mk[t])
                        ek[t] = (float)e64[t];
                __syncthreads();
            }
            for (int k = N.nlev - 2; k >= ks; k--)
            {
                const NmgLev C = N.lv[k], D = N.lv[k + 1];
                dense_prolong<false, false>(sub_e(k), sub_m(k), C.nx, C.ny, C.nz, sub_e(k + 1), D.nx,
                                            D.ny, tid, NT);
                __syncthreads();
                for (int sw = 0; sw < A.n_post; sw++)
                    for (int col = 0; col < 2; col++)
                    {
                        dense_sweep<false, float>(sub_e(k), sub_f(k), sub_m(k), C.nx, C.ny, C.nz,
                                                  N.h2[k], col, false, tid, NT);
                        __syncthreads();
                    }
            }
            {
                const NmgLev C = N.lv[ks];
                const long P = (long)C.nx * C.ny * C.nz;
                const float *sek = sub_e(ks);
                const unsigned char *smk = sub_m(ks);
                float *gek = A.ec + C.off;
                for (long t = tid; t < P; t += NT)
                    if (smk[t])
                        stg(gek + t, sek[t]);
            }
        }
        cluster.sync();
        for (int k = N.nsmall - 1; k >= 1; k--)
        {
            const NmgLev C = N.lv[k], D = N.lv[k + 1];
            dense_prolong<true, true>(A.ec + C.off, A.mc + C.off, C.nx, C.ny, C.nz, A.ec + D.off,
                                      D.nx, D.ny, ct, CT);
            cluster.sync();
            for (int sw = 0; sw < A.n_post; sw++)
                for (int col = 0; col < 2; col++)
                {
                    dense_sweep<true, float>(A.ec + C.off, A.fc + C.off, A.mc + C.off, C.nx, C.ny,
                                             C.nz, N.h2[k], col, false, ct, CT);
                    cluster.sync();
                }
        }
        {
            // prolongation to the fine unknowns (this CTA's slice of the list)
            const NmgLev D = N.lv[1];
            const float *e1 = A.ec + D.off;
            for (int e0 = sb + tid; e0 < se; e0 += NB * NT)
            {
                long g[NB];
                float add[NB], old[NB];
#pragma unroll
                for (int u = 0; u < NB; u++)
                {
                    const int e = e0 + u * NT;
                    g[u] = e < se ? (long)A.cl[e] : -1L;
                }
#pragma unroll
                for (int u = 0; u < NB; u++)
                    if (g[u] >= 0)
                    {
                        const unsigned l = (unsigned)(g[u] - N.goff);
                        const unsigned z = l / (unsigned)sz0;
                        const unsigned rem = l - z * (unsigned)sz0;
                        const unsigned y = rem / (unsigned)sy0;
                        const unsigned x = rem - y * (unsigned)sy0;
                        old[u] = ldg_f(A.ef + g[u]);
                        add[u] = prolong_at<true>(e1, D.nx, D.ny, (int)x, (int)y, (int)z);
                    }
#pragma unroll
                for (int u = 0; u < NB; u++)
                    if (g[u] >= 0)
                        stg(A.ef + g[u], old[u] + add[u]);
            }
        }
        cluster.sync();
        for (int sw = 0; sw < A.n_post; sw++)
            for (int col = 0; col < 2; col++)
            {
                fine_sweep(col, false);
                cluster.sync();
            }

        // ---- flexible conjugate gradient with z = ef (Notay 2000; Polak-Ribiere
        // beta), FP64 arithmetic on the FP32 vectors r (rf) and z ------------------
        double rz = 0.0, rzo = 0.0;
        for (int e0 = sb + tid; e0 < se; e0 += NB * NT)
        {
            long g[NB];
            float rv[NB], zv[NB], zo[NB];
#pragma unroll
            for (int u = 0; u < NB; u++)
            {
                const int e = e0 + u * NT;
                g[u] = e < se ? (long)A.intr[e] : -1L;
            }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                {
                    rv[u] = ldg_f(A.rf + g[u]);
                    zv[u] = ldg_f(A.ef + g[u]);
                    zo[u] = it > 0 ? ldg_f(A.efo + g[u]) : 0.0f;
                }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                {
                    rz += (double)rv[u] * (double)zv[u];
                    rzo += (double)rv[u] * (double)zo[u];
                }
        }
        reduce(1, rz, rzo, 0);
        rz = tot_d[0];
        const double beta = it > 0 ? (rz - tot_d[1]) / rz_prev : 0.0;
        rz_prev = rz;
        for (int e0 = sb + tid; e0 < se; e0 += NB * NT)
        {
            long g[NB];
            float zv[NB];
            double po[NB];
#pragma unroll
            for (int u = 0; u < NB; u++)
            {
                const int e = e0 + u * NT;
                g[u] = e < se ? (long)A.intr[e] : -1L;
            }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                {
                    zv[u] = ldg_f(A.ef + g[u]);
                    po[u] = it > 0 ? ldg_d(A.pv + g[u]) : 0.0;
                }
#pragma unroll
            for (int u = 0; u < NB; u++)
                if (g[u] >= 0)
                {
                    stg(A.pv + g[u], (double)zv[u] + (it > 0 ? beta * po[u] : 0.0));
                    stg(A.efo + g[u], zv[u]);
                }
        }
        cluster.sync();
        double pq = 0.0;
        for (int e0 = sb + tid; e0 < se; e0 += 2 * NT)
        {
            long g[2];
            double pc[2], lap[2];
#pragma unroll
            for (int u = 0; u < 2; u++)
            {
                const int e = e0 + u * NT;
                g[u] = e < se ? (long)A.intr[e] : -1L;
            }
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (g[u] >= 0)
                {
                    const long x = g[u];
                    pc[u] = ldg_d(A.pv + x);
                    lap[u] = N.oh2 * (ldg_d(A.pv + x + 1) + ldg_d(A.pv + x - 1) +
                                      ldg_d(A.pv + x + sy0) + ldg_d(A.pv + x - sy0) +
                                      ldg_d(A.pv + x + sz0) + ldg_d(A.pv + x - sz0) - 6.0 * pc[u]);
                }
#pragma unroll
            for (int u = 0; u < 2; u++)
                if (g[u] >= 0)
                    pq += pc[u] * lap[u];
        }
        reduce(2, pq, 0.0, 0);
        alpha = tot_d[0] != 0.0 ? rz / tot_d[0] : 0.0;
        it++;
    }
    // the iterate that passed the test is in bufs[(it + 1) & 1]
    if ((it + 1) & 1)
        for (int e = sb + tid; e < se; e += NT)
        {
            const long g = A.intr[e];
            A.pot[g] = ldg_d(A.pot_old + g);
        }
    if (rank == 0 && tid == 0)
    {
        A.status[2 * ent] = conv ? 1 : 0;
        A.status[2 * ent + 1] = it;
    }
    // no CTA leaves while another may still read its partials
    cluster.sync();
}

// ---- host ---------------------------------------------------------------------------------
struct NodeMgBufs {
    DBuf<NmgNode> tab;
    DBuf<int> cl, status;
    DBuf<float> ef, rf, ec, fc, efo;
    DBuf<double> pv;
    DBuf<unsigned char> msk, mc;
};

struct NodeMgState {
    NodeMgBufs lv[AMR_MAX_LEVELS]; // one set per refinement level (each keeps its sizes)
};

static NodeMgBufs &bufs_of(qz_sim *s, int level)
{
    if (!s->node_mg)
        s->node_mg = new NodeMgState();
    return s->node_mg->lv[level];
}

// Cluster size and dynamic shared memory of the launch (set once).
static int cluster_size(size_t smem)
{
    static int cs = 0;
    static std::once_flag once;
    std::call_once(once, [&] {
        cudaFuncSetAttribute((const void *)k_node_mg, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)NMG_SMEM_MAX);
        cudaFuncSetAttribute((const void *)k_node_mg, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        for (int c : {16, 8, 4, 2, 1})
        {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(c);
            cfg.blockDim = dim3(NMG_THREADS);
            cfg.dynamicSmemBytes = NMG_SMEM_MAX;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = c;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            int n = 0;
            if (cudaOccupancyMaxActiveClusters(&n, (const void *)k_node_mg, &cfg) == cudaSuccess &&
                n > 0)
            {
                cs = c;
                break;
            }
        }
        cudaGetLastError();
    });
    (void)smem;
    return cs;
}

int node_mg_level(qz_sim *s, AmrLevel &L, int level_index)
{
    const qz_config &c = s->cfg;
    NodeMgBufs &B = bufs_of(s, level_index);
    std::vector<NmgNode> tab;
    // solver schedule: replay gives every node its recorded count
    std::vector<int> caps;
    if (s->sched_mode == 2)
    {
        caps.resize(L.nnodes);
        if (!sched_take(s, L.nnodes, caps.data()))
            return QZ_FAILURE;
    }
    long coarse = 0;
    size_t smem = 0;
    for (int q = 0; q < L.nnodes; q++)
    {
        const AmrNode &nd = L.h[q];
        if (nd.nintr <= 0)
            continue;
        NmgNode N;
        memset(&N, 0, sizeof N);
        N.q = q;
        N.ib = nd.intr_off;
        N.ie = nd.intr_off + nd.nintr;
        N.goff = nd.grid_off;
        const double H = 1.0 / (1 << nd.lv);
        N.oh2 = 1.0 / (H * H);
        const double rm = 4.0 * c.G * QZ_PI_NMG * nd.mass / (nd.ncells * H * H * H);
        const double tt = c.tol * rm;
        N.thr = nd.nintr * tt * tt;
        if (c.check_method == 2)
            N.thr = N.thr * (cbrt((double)nd.nintr) * cbrt((double)nd.nintr));
        N.rmt = c.tol * rm;
        N.cap = caps.empty() ? c.max_iter : caps[q];
        N.replay = caps.empty() ? 0 : 1;
        int cx = nd.rd[0], cy = nd.rd[1], cz = nd.rd[2];
        int k = 0;
        for (;;)
        {
            N.lv[k].nx = cx + 1;
            N.lv[k].ny = cy + 1;
            N.lv[k].nz = cz + 1;
            N.h2[k] = (float)((H * (1 << k)) * (H * (1 << k)));
            if (k > 0)
            {
                N.lv[k].off = coarse;
                coarse += (long)(cx + 1) * (cy + 1) * (cz + 1);
            }
            if (k >= 1 && (std::max(cx, std::max(cy, cz)) <= 4 || k == NMG_MAXLEV - 1))
                break;
            cx = (cx + 1) / 2;
            cy = (cy + 1) / 2;
            cz = (cz + 1) / 2;
            k++;
        }
        N.nlev = k + 1;
        // sub-cycle levels: the longest tail of levels (from level 1 on) that fits
        const long Plast = (long)N.lv[N.nlev - 1].nx * N.lv[N.nlev - 1].ny * N.lv[N.nlev - 1].nz;
        int ks = N.nlev - 1;
        size_t need = 16 * (size_t)Plast + 9 * (size_t)Plast + 64;
        while (ks > 1)
        {
            const long P = (long)N.lv[ks - 1].nx * N.lv[ks - 1].ny * N.lv[ks - 1].nz;
            if (need + 9 * (size_t)P + 64 > NMG_SMEM_MAX)
                break;
            need += 9 * (size_t)P + 64;
            ks--;
        }
        N.nsmall = ks;
        size_t off = 0;
        for (int j = ks; j < N.nlev; j++)
        {
            N.soff[j] = (int)off;
            const long P = (long)N.lv[j].nx * N.lv[j].ny * N.lv[j].nz;
            off += ((9 * (size_t)P + 15) / 16) * 16;
        }
        N.coff = (int)off;
        off += 16 * (size_t)Plast;
        N.smem_need = (int)off;
        if (off > NMG_SMEM_MAX)
        {
            set_error("node multigrid: the coarse levels of a node need %zu bytes of shared memory",
                      off);
            return QZ_FAILURE;
        }
        smem = std::max(smem, off);
        tab.push_back(N);
    }
    if (tab.empty())
    {
        if (s->sched_mode == 1)
        {
            std::vector<int> z(L.nnodes, 0);
            sched_put(s, z.data(), L.nnodes);
        }
        return QZ_SUCCESS;
    }
    const int nt = (int)tab.size();
    if (!B.tab.ensure(s->mem, nt) || !B.status.ensure(s->mem, 2L * nt) ||
        !B.cl.ensure(s->mem, L.intr_total) || !B.ef.ensure(s->mem, L.grid_total) ||
        !B.rf.ensure(s->mem, L.grid_total) || !B.msk.ensure(s->mem, L.grid_total) ||
        !B.ec.ensure(s->mem, coarse) || !B.fc.ensure(s->mem, coarse) || !B.mc.ensure(s->mem, coarse) ||
        !B.pv.ensure(s->mem, L.grid_total) || !B.efo.ensure(s->mem, L.grid_total))
    {
        set_error("node multigrid buffers");
        return QZ_FAILURE;
    }
    const int cs = cluster_size(smem);
    if (cs < 1)
    {
        set_error("node multigrid: no cluster of the kernel can be resident");
        return QZ_FAILURE;
    }
    if (!check_cuda(cudaMemcpyAsync(B.tab.p, tab.data(), nt * sizeof(NmgNode),
                                    cudaMemcpyHostToDevice, s->stream),
                    "node multigrid table"))
        return QZ_FAILURE;
    cudaMemsetAsync(B.msk.p, 0, L.grid_total, s->stream);
    cudaMemsetAsync(B.ef.p, 0, L.grid_total * sizeof(float), s->stream);
    cudaMemsetAsync(B.ec.p, 0, std::max(coarse, 1L) * sizeof(float), s->stream);
    cudaMemsetAsync(B.mc.p, 0, std::max(coarse, 1L), s->stream);
    cudaMemsetAsync(B.pv.p, 0, L.grid_total * sizeof(double), s->stream);
    NmgArgs A;
    A.tab = B.tab.p;
    A.intr = L.intr.p;
    A.cl = B.cl.p;
    A.d = L.d;
    A.pot = L.pot;
    A.pot_old = L.pot_old;
    A.ef = B.ef.p;
    A.rf = B.rf.p;
    A.msk = B.msk.p;
    A.ec = B.ec.p;
    A.fc = B.fc.p;
    A.mc = B.mc.p;
    A.status = B.status.p;
    A.pv = B.pv.p;
    A.efo = B.efo.p;
    A.tol2 = c.tol2;
    A.method = c.check_method;
    // smoothing of the node cycles: NMG_SWEEPS red-black sweeps before and after
    // the coarse correction unless QZ_NODE_MG_SWEEPS (pre = post) and
    // QZ_NODE_MG_COARSE (coarsest-level sweeps) set them
    static const char *env_sw = getenv("QZ_NODE_MG_SWEEPS");
    static const char *env_co = getenv("QZ_NODE_MG_COARSE");
    A.n_pre = std::max(1, env_sw ? atoi(env_sw) : NMG_SWEEPS);
    A.n_post = std::max(0, env_sw ? atoi(env_sw) : NMG_SWEEPS);
    A.n_coarse = std::max(1, env_co ? atoi(env_co) : NMG_COARSE_SWEEPS);

    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nt * cs);
    cfg.blockDim = dim3(NMG_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cs;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    cudaEvent_t eb = nullptr, ee = nullptr;
    if (s->prof)
    {
        eb = prof_event(s);
        ee = prof_event(s);
        cudaEventRecord(eb, s->stream);
    }
    if (!check_cuda(cudaLaunchKernelEx(&cfg, k_node_mg, A), "node multigrid"))
        return QZ_FAILURE;
    s->stats.kernel_launches++;
    if (s->prof)
    {
        cudaEventRecord(ee, s->stream);
        s->prof_pending.push_back({QZ_PROF_NODE_MG, 0.0, eb, ee});
    }
    std::vector<int> st(2 * nt);
    if (!check_cuda(cudaMemcpyAsync(st.data(), B.status.p, 2L * nt * sizeof(int),
                                    cudaMemcpyDeviceToHost, s->stream),
                    "node multigrid status") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "node multigrid sync"))
        return QZ_FAILURE;
    int worst = 0, unconv = 0;
    double pts_it = 0.0;
    for (int e = 0; e < nt; e++)
    {
        worst = std::max(worst, st[2 * e + 1]);
        unconv += st[2 * e] == 0;
        pts_it += (double)(tab[e].ie - tab[e].ib) * st[2 * e + 1];
    }
    s->stats.node_mg_iterations += worst;
    if (s->sched_mode == 1)
    {
        std::vector<int> per(L.nnodes, 0);
        for (int e = 0; e < nt; e++)
            per[tab[e].q] = st[2 * e + 1];
        sched_put(s, per.data(), L.nnodes);
    }
    if (s->sched_mode == 2)
        unconv = 0; // replayed counts: no convergence test
    if (s->prof)
    {
        // per fine unknown and iteration: the FP64 pass reads d, phi, p (the 7
        // stencil values come from cache lines shared with neighbours) and
        // writes the new phi and r (36 B); each red-black sweep reads e, r and
        // writes e (12 B); restriction and prolongation about 8 B, the coarse
        // levels about a seventh of that; the conjugate-gradient passes read r,
        // z, z_old (12 B), read z, p and write p, z_old (24 B), read p (8 B)
        const double sweeps = (double)(A.n_pre + A.n_post);
        s->prof_pending.back().bytes = pts_it * (36.0 + (12.0 * sweeps + 8.0) * 8.0 / 7.0 + 44.0);
    }
    if (unconv)
    {
        set_error("the precision was not reached in refinement level %d after %d multigrid "
                  "iterations (%d nodes)",
                  level_index, worst, unconv);
        return QZ_FAILURE;
    }
    return check_cuda(cudaGetLastError(), "node multigrid") ? QZ_SUCCESS : QZ_FAILURE;
}

void node_mg_free(qz_sim *s)
{
    if (!s->node_mg)
        return;
    for (auto &B : s->node_mg->lv)
    {
        B.tab.release(s->mem);
        B.cl.release(s->mem);
        B.status.release(s->mem);
        B.ef.release(s->mem);
        B.rf.release(s->mem);
        B.ec.release(s->mem);
        B.fc.release(s->mem);
        B.msk.release(s->mem);
        B.mc.release(s->mem);
        B.pv.release(s->mem);
        B.efo.release(s->mem);
    }
    delete s->node_mg;
    s->node_mg = nullptr;
}

} // namespace qz

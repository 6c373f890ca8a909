// qz_adjoint.cu -- reverse-mode derivative of the particle-mesh step (the head
// node, and the refinement levels of a frozen tree further below).
//
// The forward map of one step (particle_updating.c:39-207, 2677-2688 around
// grid_density.c:35-111, potential_head_node.c:99-179, grid_acceleration.c:36-76
// and particle_acceleration.c:33-132) is, per particle p and axis c,
//
//   v_h = v_n + (a_n dt) 0.5;  x_{n+1} = R (x_n + v_h dt) (+ wall);  v_h <- R v_h
//   a_{n+1} = F(x_{n+1}, m);   v_{n+1} = v_h + (a_{n+1} dt) 0.5
//
// with R = -1 where the drift left [0, 1) (reflexive walls), and the force
//
//   d_g = sum_p (4 pi G / H^3) m_p w_g(x_p)             CIC deposit
//   Lap_h phi = d on the interior, phi = shell(M) on the solve-grid boundary
//   A_g = (phi_{g-e} - phi_{g+e}) / 2H  (interior g),   A_g = shell accel(M) else
//   F_p = sum_g w_g(x_p) A_g                            CIC gather
//
// with M the configured total mass (the analytic shell of
// initial_potential_and_acceleration_head.c:297-334 is linear in M).  Its
// vector-Jacobian product for an accelerations' adjoint abar:
//
//   Abar_g   = sum_p w_g(x_p) abar_p                    gather^T = a deposit
//   phibar_h = sum_e (Abar_{h+e} [h+e interior] - Abar_{h-e} [h-e interior]) / 2H
//                                                       gradient^T = -divergence
//   Lap_h lam = phibar, lam = 0 on the boundary         the solve is self-adjoint
//   xbar_p  += sum_g grad w_g(x_p) (abar_p . A_g + (4 pi G / H^3) m_p lam_g)
//   mbar_p  += (4 pi G / H^3) sum_g w_g(x_p) lam_g  +  Mbar
//   Mbar     = (1/M) sum_{b boundary} [ phi_b (phibar_b - (1/H^2) sum_nbr lam)
//                                        + Abar_b . A_b ]
//
// The trajectory's adjoint runs the steps backwards from the loss
// L = (1/N) sum_p |x_T,p - x*_p|^2 with checkpoints of (x, v, a, phi) every K
// steps; a segment's states are recomputed from its checkpoint (bit-identical:
// the forward is deterministic) before its reverse sweep.  The adjoint
// deposit is a sort by head cell and a warp-segmented reduction like the
// forward deposit (no float atomics); every reduction has a fixed order.
#include "qz_amr_dev.cuh"

namespace qz {

#define QZ_PI_D 3.14159265358979323846

constexpr int ADJ_RED_BLOCKS = 296;

// Per-simulation adjoint buffers (grown on first use).
struct Adjoint {
    DBuf<double> xb, vb, mb, ac, ab; // 3N adjoints of x, v; N of m; 3N carried / pulled a-bar
    DBuf<double> Ab;                 // 3 gpts: deposit of a-bar
    DBuf<double> phib, lam;          // gpts: -div(Abar), adjoint potential
    DBuf<double> cs;                 // 24 per deposit segment
    DBuf<double> ck, seg, fin;       // checkpoints, a segment's states, the final state
    DBuf<double> tgt;                // 3N targets
    DBuf<double> red;                // reduction partials and results
    double *host = nullptr;          // 8 pinned doubles
    long seg_recs = 0, ck_recs = 0;
    // refinement levels (index = level): a-bar deposits (3 x grid), children's
    // phi-bar contributions, phi-bar, lam (kept: the next solve's start on a frozen
    // tree), scratch, interior masks, node thresholds
    std::vector<DBuf<double>> lA, lphic, lphib, llam, lscr, lthr;
    std::vector<DBuf<int>> lmask;
    DBuf<int> finest;   // per particle: its finest level
    DBuf<double> abh;   // a-bar of the particles whose finest node is the head (3n)
    DBuf<double> phic0; // children's phi-bar contributions on the head grid
    DBuf<double> nrm;   // per node sums
};

void adjoint_free(qz_sim *s)
{
    Adjoint *A = s->adj;
    if (!A)
        return;
    DBuf<double> *b[] = {&A->xb, &A->vb, &A->mb, &A->ac, &A->ab, &A->Ab, &A->phib, &A->lam,
                         &A->cs, &A->ck, &A->seg, &A->fin, &A->tgt, &A->red, &A->abh,
                         &A->phic0, &A->nrm};
    for (auto *q : b)
        q->release(s->mem);
    for (auto *v : {&A->lA, &A->lphic, &A->lphib, &A->llam, &A->lscr, &A->lthr})
        for (auto &q : *v)
            q.release(s->mem);
    for (auto &q : A->lmask)
        q.release(s->mem);
    A->finest.release(s->mem);
    if (A->host)
        cudaFreeHost(A->host);
    delete A;
    s->adj = nullptr;
}

__device__ __forceinline__ double adj_block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
        sh[warp] = v;
    __syncthreads();
    double r = 0.0;
    if (warp == 0)
    {
        r = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1)
            r += __shfl_xor_sync(0xffffffffu, r, o);
    }
    __syncthreads();
    return r;
}

// Sums partial[0..nb) in a fixed order; mode 0: out[0] = sum * scale, mode 1: out[0] += sum * scale.
__global__ void k_adj_final(int nb, const double *__restrict__ partial, double scale, int mode,
                            double *__restrict__ out)
{
    __shared__ double sh[32];
    double a = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x)
        a += partial[q];
    a = adj_block_sum(a, sh);
    if (threadIdx.x == 0)
        out[0] = mode == 0 ? a * scale : out[0] + a * scale;
}

// ---- deposit of a-bar (gather transpose) ------------------------------------------------
// Particle i's CIC corner weights times its a-bar, three components, added to
// acc (component * 8 + corner).
__device__ __forceinline__ void adj_cic_add(int i, double scale, const double *__restrict__ x,
                                            const double *__restrict__ y,
                                            const double *__restrict__ z,
                                            const double *__restrict__ abx,
                                            const double *__restrict__ aby,
                                            const double *__restrict__ abz, double acc[24])
{
    double px = x[i] * scale, py = y[i] * scale, pz = z[i] * scale;
    int fx = (int)px, fy = (int)py, fz = (int)pz;
    double wx1 = px - fx, wy1 = py - fy, wz1 = pz - fz;
    double wx2 = 1.0 - wx1, wy2 = 1.0 - wy1, wz2 = 1.0 - wz1;
    double w[8];
    w[0] = wx2 * wy2 * wz2;
    w[1] = wx1 * wy2 * wz2;
    w[2] = wx2 * wy1 * wz2;
    w[3] = wx1 * wy1 * wz2;
    w[4] = wx2 * wy2 * wz1;
    w[5] = wx1 * wy2 * wz1;
    w[6] = wx2 * wy1 * wz1;
    w[7] = wx1 * wy1 * wz1;
    const double a0 = abx[i], a1 = aby[i], a2 = abz[i];
#pragma unroll
    for (int c = 0; c < 8; c++)
    {
        acc[c] += a0 * w[c];
        acc[8 + c] += a1 * w[c];
        acc[16 + c] += a2 * w[c];
    }
}

// One warp per occupied cell of at most SEG_LONG particles (longer cells are
// listed for k_adj_seg_long): for each of the 8 corners the sums of w * abar
// over the cell's particles, three components.  cs: segment * 24 + component *
// 8 + corner.
__global__ void k_adj_seg_reduce(int L, const int *__restrict__ perm,
                                 const int *__restrict__ seg_start, int *__restrict__ flags,
                                 int *__restrict__ long_list, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ abx, const double *__restrict__ aby,
                                 const double *__restrict__ abz, double *__restrict__ cs)
{
    const int lane = threadIdx.x & 31;
    const long warp0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const int nseg = flags[F_NSEG];
    const double scale = (double)(1 << L);
    for (long sg = warp0; sg < nseg; sg += nwarps)
    {
        const int b = seg_start[sg], e = seg_start[sg + 1];
        if (e - b > SEG_LONG)
        {
            if (lane == 0)
                long_list[atomicAdd(&flags[F_NLONG], 1)] = (int)sg;
            continue;
        }
        double acc[24];
#pragma unroll
        for (int c = 0; c < 24; c++)
            acc[c] = 0.0;
        for (int q = b + lane; q < e; q += 32)
            adj_cic_add(perm[q], scale, x, y, z, abx, aby, abz, acc);
#pragma unroll
        for (int c = 0; c < 24; c++)
        {
            double v = acc[c];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[c] = v;
        }
        if (lane < 24)
        {
            double v = acc[0];
#pragma unroll
            for (int c = 1; c < 24; c++)
                if (lane == c)
                    v = acc[c];
            cs[sg * 24 + lane] = v;
        }
    }
}

// One block per listed cell of more than SEG_LONG particles: thread t adds
// particles t, t + blockDim, ... (two at a time), then block sums in a fixed
// order.  512 threads: the 24 sums a thread need more than 64 registers.
constexpr int ADJ_SEG_LONG_THREADS = 512;
__global__ void __launch_bounds__(ADJ_SEG_LONG_THREADS)
    k_adj_seg_long(int L, const int *__restrict__ perm, const int *__restrict__ seg_start,
                   const int *__restrict__ flags, const int *__restrict__ long_list,
                   const double *__restrict__ x, const double *__restrict__ y,
                   const double *__restrict__ z, const double *__restrict__ abx,
                   const double *__restrict__ aby, const double *__restrict__ abz,
                   double *__restrict__ cs)
{
    __shared__ double shw[(ADJ_SEG_LONG_THREADS / 32) * 24];
    const int nl = flags[F_NLONG];
    const double scale = (double)(1 << L);
    const int bs = (int)blockDim.x;
    for (int li = blockIdx.x; li < nl; li += gridDim.x)
    {
        const int sg = long_list[li];
        const int b = seg_start[sg], e = seg_start[sg + 1];
        double acc[24];
#pragma unroll
        for (int c = 0; c < 24; c++)
            acc[c] = 0.0;
        for (int q0 = b + (int)threadIdx.x; q0 < e; q0 += 2 * bs)
        {
            const int q1 = q0 + bs;
            const int i0 = perm[q0], i1 = q1 < e ? perm[q1] : -1;
            adj_cic_add(i0, scale, x, y, z, abx, aby, abz, acc);
            if (i1 >= 0)
                adj_cic_add(i1, scale, x, y, z, abx, aby, abz, acc);
        }
        seg_block_sums<24>(acc, shw);
        if (threadIdx.x < 24)
            cs[(long)sg * 24 + threadIdx.x] = acc[0];
        __syncthreads(); // shw is rewritten for the next cell
    }
}

// Each grid point sums the corner contributions of its (up to) 8 adjacent
// occupied cells in a fixed order, three components.
__global__ void k_adj_point_gather(long D, const int *__restrict__ cell_seg,
                                   const double *__restrict__ cs, double *__restrict__ Abx,
                                   double *__restrict__ Aby, double *__restrict__ Abz)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= D * D * D)
        return;
    const long B = D - 1;
    int gx = (int)(t % D), gy = (int)((t / D) % D), gz = (int)(t / (D * D));
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int c = 0; c < 2; c++)
    {
        int cz = gz - 1 + c;
        if (cz < 0 || cz >= B)
            continue;
        for (int b = 0; b < 2; b++)
        {
            int cy = gy - 1 + b;
            if (cy < 0 || cy >= B)
                continue;
            for (int a = 0; a < 2; a++)
            {
                int cx = gx - 1 + a;
                if (cx < 0 || cx >= B)
                    continue;
                int sg = cell_seg[cx + cy * B + (long)cz * B * B];
                if (sg >= 0)
                {
                    const int corner = (1 - a) + 2 * (1 - b) + 4 * (1 - c);
                    a0 += cs[(long)sg * 24 + corner];
                    a1 += cs[(long)sg * 24 + 8 + corner];
                    a2 += cs[(long)sg * 24 + 16 + corner];
                }
            }
        }
    }
    Abx[t] = a0;
    Aby[t] = a1;
    Abz[t] = a2;
}

// ---- gradient transpose -------------------------------------------------------------------
__device__ __forceinline__ bool adj_interior(long i, long j, long k, int hi)
{
    return i >= 2 && i <= hi && j >= 2 && j <= hi && k >= 2 && k <= hi;
}

// -div of Abar taken over the interior points where the gradient is evaluated.
__device__ __forceinline__ double adj_negdiv(long i, long j, long k, long D, int hi, double o2h,
                                             const double *__restrict__ Abx,
                                             const double *__restrict__ Aby,
                                             const double *__restrict__ Abz)
{
    const long D2 = D * D;
    const long g = i + j * D + k * D2;
    double v = 0.0;
    if (adj_interior(i + 1, j, k, hi))
        v += Abx[g + 1];
    if (adj_interior(i - 1, j, k, hi))
        v -= Abx[g - 1];
    if (adj_interior(i, j + 1, k, hi))
        v += Aby[g + D];
    if (adj_interior(i, j - 1, k, hi))
        v -= Aby[g - D];
    if (adj_interior(i, j, k + 1, hi))
        v += Abz[g + D2];
    if (adj_interior(i, j, k - 1, hi))
        v -= Abz[g - D2];
    return v * o2h;
}

__global__ void k_adj_negdiv(int L, long D, double o2h, const double *__restrict__ Abx,
                             const double *__restrict__ Aby, const double *__restrict__ Abz,
                             double *__restrict__ phib)
{
    const int m = (1 << L) - 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)m * m * m)
        return;
    const long i = 2 + t % m, j = 2 + (t / m) % m, k = 2 + t / ((long)m * m);
    phib[i + j * D + k * D * D] = adj_negdiv(i, j, k, D, 1 << L, o2h, Abx, Aby, Abz);
}

// ---- total-mass term ----------------------------------------------------------------------
// Per block: sum over the solve grid's boundary points b (coordinates in
// 1..2^L+1, one of them 1 or 2^L+1) of
// phi_b (phibar_b - (1/H^2) sum of lam at the 6 neighbours) + Abar_b . A_b.
__global__ void k_adj_shell(int L, long D, double o2h, double oh2, const double *__restrict__ pot,
                            const double *__restrict__ lam, const double *__restrict__ Abx,
                            const double *__restrict__ Aby, const double *__restrict__ Abz,
                            const double *__restrict__ gx, const double *__restrict__ gy,
                            const double *__restrict__ gz, const double *__restrict__ phic,
                            double *__restrict__ partial)
{
    __shared__ double sh[32];
    const int n = (1 << L) + 1, hi = 1 << L;
    const long total = (long)n * n * n;
    const long D2 = D * D;
    double acc = 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x)
    {
        const long i = 1 + t % n, j = 1 + (t / n) % n, k = 1 + t / ((long)n * n);
        if (adj_interior(i, j, k, hi))
            continue;
        const long g = i + j * D + k * D2;
        const double nb = lam[g + 1] + lam[g - 1] + lam[g + D] + lam[g - D] + lam[g + D2] +
                          lam[g - D2];
        const double pb = adj_negdiv(i, j, k, D, hi, o2h, Abx, Aby, Abz) - oh2 * nb +
                          (phic ? phic[g] : 0.0);
        acc += pot[g] * pb + (Abx[g] * gx[g] + Aby[g] * gy[g] + Abz[g] * gz[g]);
    }
    acc = adj_block_sum(acc, sh);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = acc;
}

// ---- gather of the adjoint (deposit and gather weight derivatives) ------------------------
__global__ void k_adj_gather(long n, int L, long D, double coeff, const double *__restrict__ x,
                             const double *__restrict__ y, const double *__restrict__ z,
                             const double *__restrict__ m, const double *__restrict__ abx,
                             const double *__restrict__ aby, const double *__restrict__ abz,
                             const double *__restrict__ gx, const double *__restrict__ gy,
                             const double *__restrict__ gz, const double *__restrict__ lam,
                             double *__restrict__ xb, double *__restrict__ yb,
                             double *__restrict__ zb, double *__restrict__ mb,
                             int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double scale = (double)(1 << L);
    double px = x[i] * scale, py = y[i] * scale, pz = z[i] * scale;
    if (!(px >= 0.0 && py >= 0.0 && pz >= 0.0) || px >= scale + 1.0 || py >= scale + 1.0 ||
        pz >= scale + 1.0)
    {
        atomicOr(&flags[F_ERROR], E_PTCL_OUTSIDE);
        return;
    }
    int fx = (int)px, fy = (int)py, fz = (int)pz;
    double wx[2], wy[2], wz[2];
    wx[1] = px - fx;
    wy[1] = py - fy;
    wz[1] = pz - fz;
    wx[0] = 1.0 - wx[1];
    wy[0] = 1.0 - wy[1];
    wz[0] = 1.0 - wz[1];
    const double sgn[2] = {-scale, scale};
    const double a0 = abx[i], a1 = aby[i], a2 = abz[i];
    const double cm = coeff * m[i];
    const long D2 = D * D;
    const long g0 = (fx + 1) + (long)(fy + 1) * D + (long)(fz + 1) * D2;
    double dx = 0.0, dy = 0.0, dz = 0.0, dm = 0.0;
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
            {
                const long q = g0 + ii + jj * D + kk * D2;
                const double lq = lam[q];
                const double sv = a0 * gx[q] + a1 * gy[q] + a2 * gz[q] + cm * lq;
                dx += sgn[ii] * wy[jj] * wz[kk] * sv;
                dy += wx[ii] * sgn[jj] * wz[kk] * sv;
                dz += wx[ii] * wy[jj] * sgn[kk] * sv;
                dm += wx[ii] * wy[jj] * wz[kk] * lq;
            }
    xb[i] += dx;
    yb[i] += dy;
    zb[i] += dz;
    mb[i] += coeff * dm;
}

// ---- leapfrog transposes ------------------------------------------------------------------
// kick (particle_updating.c:2677-2688) transposed: abar = carried + vbar dt 0.5
__global__ void k_adj_kick(long n3, double dt, const double *__restrict__ vb,
                           const double *__restrict__ ac, double *__restrict__ ab)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n3)
        ab[i] = ac[i] + vb[i] * dt * 0.5;
}

// kick-drift with reflection (particle_updating.c:39-207) transposed, with the
// walls found by re-evaluating the forward's expressions on the stored state.
__global__ void k_adj_kick_drift(long n, double dt, const double *__restrict__ st,
                                 double *__restrict__ xb, double *__restrict__ vb,
                                 double *__restrict__ ac)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
#pragma unroll
    for (int c = 0; c < 3; c++)
    {
        const double x = st[c * n + i], v = st[(3 + c) * n + i], a = st[(6 + c) * n + i];
        double q = v;
        q += a * dt * 0.5;
        double p = x;
        p += q * dt;
        const double R = (p < 0.0 || p >= 1.0) ? -1.0 : 1.0;
        const long k = c * n + i;
        const double xt = R * xb[k];
        const double vh = R * vb[k] + dt * xt;
        xb[k] = xt;
        vb[k] = vh;
        ac[k] = vh * dt * 0.5;
    }
}

// ---- loss ---------------------------------------------------------------------------------
__global__ void k_adj_loss(long n, const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, const double *__restrict__ t,
                           double *__restrict__ xb, double *__restrict__ partial)
{
    __shared__ double sh[32];
    const double s2 = 2.0 / (double)n;
    double acc = 0.0;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
    {
        const double dx = x[i] - t[i], dy = y[i] - t[n + i], dz = z[i] - t[2 * n + i];
        acc += dx * dx + dy * dy + dz * dz;
        xb[i] = s2 * dx;
        xb[n + i] = s2 * dy;
        xb[2 * n + i] = s2 * dz;
    }
    acc = adj_block_sum(acc, sh);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = acc;
}

__global__ void k_adj_add_scalar(long n, const double *__restrict__ v, double *__restrict__ out)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] += v[0];
}

// ---- refinement levels (frozen tree) ------------------------------------------------------
// The level forward (grid_density.c:113-267, potential_branches.c:93-331,
// grid_acceleration.c:199-394, particle_acceleration.c:134-355) is linear in the
// node densities and in the parents' fields:
//   d_l   = sum_p (4 pi G / H^6) m_p W_l(x_p)   particles of level l's nodes
//   phi_l = A_l^-1 (d_l - B phi_b / H^2),  phi_b = P(phi_{l-1}) at node boundary
//           points, shell(M) at simulation-boundary points
//   a_l   = -grad phi_l (interior), P(a_{l-1}) (boundary), shell accel(M) (sim boundary)
//   F_p   = sum_g w_g(x_p) a_{l*}[g]          l* the particle's finest level
// with P the 8-point parent average of from_parent.  The pull-back runs from the
// finest level down: the gather's transpose deposits a-bar on each particle's
// finest level; on each level the gradient's transpose (-div over the interior
// points), children's contributions, the node solves with zero boundary, and the
// transposes of P (to the parent's a-bar and phi-bar: contributions sorted by
// parent point and added in list order), the shell (to the total mass) and the
// deposit (to x and m).  Every sum has a fixed order: the gradient is
// bit-reproducible.

struct NodeOfPtrs {
    const int *p[AMR_MAX_LEVELS];
};

// finest level holding each particle (0: the head)
__global__ void k_adj_finest(long n, int nlev, NodeOfPtrs no, int *__restrict__ fin)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int l = nlev - 1;
    for (; l > 0; l--)
        if (no.p[l][i] >= 0)
            break;
    fin[i] = l;
}

__global__ void k_adj_mask_ab(long n, const int *__restrict__ fin, const double *__restrict__ ab,
                              double *__restrict__ abh)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const bool h = fin[i] == 0;
    abh[i] = h ? ab[i] : 0.0;
    abh[n + i] = h ? ab[n + i] : 0.0;
    abh[2 * n + i] = h ? ab[2 * n + i] : 0.0;
}

__global__ void k_adj_flag_level(long n, const int *__restrict__ fin, int l, int *__restrict__ flag)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        flag[i] = fin[i] == l ? 1 : 0;
}

// cell keys (level box pool) of the particles whose finest level is l
__global__ void k_adj_lvl_keys(long n, int l, const int *__restrict__ fin,
                               const int *__restrict__ node_of, const AmrNode *__restrict__ nodes,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const int *__restrict__ slot,
                               unsigned *__restrict__ keys, int *__restrict__ vals)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || fin[i] != l)
        return;
    const AmrNode N = nodes[node_of[i]];
    const double sc = (double)(1 << N.lv);
    const int cx = (int)(x[i] * sc), cy = (int)(y[i] * sc), cz = (int)(z[i] * sc);
    keys[slot[i]] = (unsigned)(N.box_off + box_index(N, cx, cy, cz));
    vals[slot[i]] = (int)i;
}

// grid points of level l: the 8 corner sums of their adjacent occupied cells, three
// components (cs: segment * 24 + component * 8 + corner)
__global__ void k_adj_lvl_point_gather3(long total, int nn, const AmrNode *__restrict__ nodes,
                                        const int *__restrict__ cell_seg,
                                        const double *__restrict__ cs, double *__restrict__ A0,
                                        double *__restrict__ A1, double *__restrict__ A2)
{
    long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total)
        return;
    const AmrNode N = nodes[find_node(nodes, nn, g, 0)];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    for (int c = 0; c < 2; c++)
    {
        const int cz = gz - 1 + c;
        if (cz < 0 || cz >= N.rd[2])
            continue;
        for (int b = 0; b < 2; b++)
        {
            const int cy = gy - 1 + b;
            if (cy < 0 || cy >= N.rd[1])
                continue;
            for (int a = 0; a < 2; a++)
            {
                const int cx = gx - 1 + a;
                if (cx < 0 || cx >= N.rd[0])
                    continue;
                const int sg =
                    cell_seg[N.box_off + cx + (long)cy * N.rd[0] + (long)cz * N.rd[0] * N.rd[1]];
                if (sg >= 0)
                {
                    const int corner = (1 - a) + 2 * (1 - b) + 4 * (1 - c);
                    a0 += cs[(long)sg * 24 + corner];
                    a1 += cs[(long)sg * 24 + 8 + corner];
                    a2 += cs[(long)sg * 24 + 16 + corner];
                }
            }
        }
    }
    A0[g] = a0;
    A1[g] = a1;
    A2[g] = a2;
}

// the gather's weight derivatives for particles whose finest level is a refinement
// level: xbar += sum_g grad w_g (abar . a_l[g])
__global__ void k_adj_gather_w(long n, LevelRefs R, const int *__restrict__ fin,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ ab,
                               double *__restrict__ xb)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int l = fin[i];
    if (l == 0)
        return;
    const AmrNode N = R.nodes[l][R.node_of[l][i]];
    const double sc = (double)(1 << N.lv);
    const double px = x[i] * sc, py = y[i] * sc, pz = z[i] * sc;
    const int fx = (int)px, fy = (int)py, fz = (int)pz;
    double wx[2], wy[2], wz[2];
    wx[1] = px - fx;
    wy[1] = py - fy;
    wz[1] = pz - fz;
    wx[0] = 1.0 - wx[1];
    wy[0] = 1.0 - wy[1];
    wz[0] = 1.0 - wz[1];
    const double sgn[2] = {-sc, sc};
    const double a0 = ab[i], a1 = ab[n + i], a2 = ab[2 * n + i];
    const long sx = N.rd[0] + 1, sxy = sx * (N.rd[1] + 1);
    const long g0 = grid_index(N, fx - N.ts[0], fy - N.ts[1], fz - N.ts[2]);
    const double *gx = R.ax[l], *gy = R.ay[l], *gz = R.az[l];
    double dx = 0.0, dy = 0.0, dz = 0.0;
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
            {
                const long q = g0 + ii + jj * sx + kk * sxy;
                const double sv = a0 * gx[q] + a1 * gy[q] + a2 * gz[q];
                dx += sgn[ii] * wy[jj] * wz[kk] * sv;
                dy += wx[ii] * sgn[jj] * wz[kk] * sv;
                dz += wx[ii] * wy[jj] * sgn[kk] * sv;
            }
    xb[i] += dx;
    xb[n + i] += dy;
    xb[2 * n + i] += dz;
}

__global__ void k_adj_set_mask(int nlist, const int *__restrict__ list, int *__restrict__ mask)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e < nlist)
        mask[list[e]] = 1;
}

// phi-bar at every grid point of level l: -div of a-bar over the interior points
// where the gradient is taken (neighbours inside the node grid), plus the
// children's contributions
__global__ void k_adj_lvl_negdiv(long total, int nn, const AmrNode *__restrict__ nodes,
                                 const int *__restrict__ mask, const double *__restrict__ A0,
                                 const double *__restrict__ A1, const double *__restrict__ A2,
                                 const double *__restrict__ phic, double *__restrict__ out)
{
    long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total)
        return;
    const AmrNode N = nodes[find_node(nodes, nn, g, 0)];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const double o2h = 1.0 / (2.0 * (1.0 / (1 << N.lv)));
    const long sy = N.rd[0] + 1, sz = sy * (N.rd[1] + 1);
    double v = 0.0;
    if (gx + 1 <= N.rd[0] && mask[g + 1])
        v += A0[g + 1];
    if (gx - 1 >= 0 && mask[g - 1])
        v -= A0[g - 1];
    if (gy + 1 <= N.rd[1] && mask[g + sy])
        v += A1[g + sy];
    if (gy - 1 >= 0 && mask[g - sy])
        v -= A1[g - sy];
    if (gz + 1 <= N.rd[2] && mask[g + sz])
        v += A2[g + sz];
    if (gz - 1 >= 0 && mask[g - sz])
        v -= A2[g - sz];
    out[g] = v * o2h + phic[g];
}

// per node: sum of rhs^2 over its interior list (one block a node, fixed order)
__global__ void k_adj_node_norm(const AmrNode *__restrict__ nodes, const int *__restrict__ intr,
                                const double *__restrict__ rhs, double *__restrict__ out)
{
    __shared__ double sh[32];
    const AmrNode N = nodes[blockIdx.x];
    double acc = 0.0;
    for (int e = threadIdx.x; e < N.nintr; e += blockDim.x)
    {
        const double v = rhs[intr[N.intr_off + e]];
        acc += v * v;
    }
    acc = adj_block_sum(acc, sh);
    if (threadIdx.x == 0)
        out[blockIdx.x] = acc;
}

// phi-bar of a boundary point after the solve: its own minus the solve's
// coupling (1/H^2) sum of lam at the six neighbours (lam is zero off the interior)
__device__ __forceinline__ double adj_phit(const AmrNode &N, long g, const double *phib,
                                           const double *lam)
{
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const double H = 1.0 / (1 << N.lv);
    const long sy = N.rd[0] + 1, sz = sy * (N.rd[1] + 1);
    double nb = 0.0;
    if (gx + 1 <= N.rd[0])
        nb += lam[g + 1];
    if (gx - 1 >= 0)
        nb += lam[g - 1];
    if (gy + 1 <= N.rd[1])
        nb += lam[g + sy];
    if (gy - 1 >= 0)
        nb += lam[g - sy];
    if (gz + 1 <= N.rd[2])
        nb += lam[g + sz];
    if (gz - 1 >= 0)
        nb += lam[g - sz];
    return phib[g] - nb / (H * H);
}

// Transposes of the parent averages at the node boundary points: 0.125 of the
// point's phi-bar (after the solve) and a-bar go to each of its 8 parent points
// (a point on an even coordinate names the same parent point twice).  The
// contributions are made deterministic by sorting them by target: pass 1 writes
// one (parent point, 8 e + corner) pair per contribution, a stable radix sort
// orders them by parent point and then by boundary-list position, and pass 2
// adds each parent point's run in that order.
__device__ __forceinline__ long adj_bdry_target(const AmrNode &N, const AmrNode &P, long g, int c)
{
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const int cx = gx + N.ts[0], cy = gy + N.ts[1], cz = gz + N.ts[2];
    const int ii = c & 1, jj = (c >> 1) & 1, kk = c >> 2;
    const int x = (ii ? ((cx + 1) >> 1) : (cx >> 1)) - P.ts[0];
    const int y = (jj ? ((cy + 1) >> 1) : (cy >> 1)) - P.ts[1];
    const int z = (kk ? ((cz + 1) >> 1) : (cz >> 1)) - P.ts[2];
    const long sx = P.rd[0] + 1, sxy = sx * (P.rd[1] + 1);
    return P.grid_off + x + y * sx + z * sxy;
}

__global__ void k_adj_bdry_keys(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                                const AmrNode *__restrict__ nodes, const AmrNode *__restrict__ pnodes,
                                unsigned *__restrict__ key, int *__restrict__ val)
{
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 8L * nlist)
        return;
    const int e = (int)(t >> 3), c = (int)(t & 7);
    const AmrNode N = nodes[lnode[e]];
    key[t] = (unsigned)adj_bdry_target(N, pnodes[N.parent], list[e], c);
    val[t] = (int)t;
}

__global__ void k_adj_bdry_sum(long m, const unsigned *__restrict__ key, const int *__restrict__ val,
                               const int *__restrict__ list, const int *__restrict__ lnode,
                               const AmrNode *__restrict__ nodes, const double *__restrict__ phib,
                               const double *__restrict__ lam, const double *__restrict__ A0,
                               const double *__restrict__ A1, const double *__restrict__ A2,
                               double *__restrict__ pA0, double *__restrict__ pA1,
                               double *__restrict__ pA2, double *__restrict__ pphic)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m || (i > 0 && key[i - 1] == key[i]))
        return;
    const unsigned q = key[i];
    double sf = 0.0, s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (long j = i; j < m && key[j] == q; j++)
    {
        const int e = val[j] >> 3;
        const long g = list[e];
        const AmrNode N = nodes[lnode[e]];
        sf += 0.125 * adj_phit(N, g, phib, lam);
        s0 += 0.125 * A0[g];
        s1 += 0.125 * A1[g];
        s2 += 0.125 * A2[g];
    }
    pphic[q] += sf;
    pA0[q] += s0;
    pA1[q] += s1;
    pA2[q] += s2;
}

// simulation-boundary points (analytic, linear in M): per block partial sums of
// phi-bar (after the solve) times phi plus a-bar . a
__global__ void k_adj_simb_T(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                             const AmrNode *__restrict__ nodes, const double *__restrict__ phib,
                             const double *__restrict__ lam, const double *__restrict__ pot,
                             const double *__restrict__ A0, const double *__restrict__ A1,
                             const double *__restrict__ A2, const double *__restrict__ a0,
                             const double *__restrict__ a1, const double *__restrict__ a2,
                             double *__restrict__ partial)
{
    __shared__ double sh[32];
    double acc = 0.0;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nlist; e += gridDim.x * blockDim.x)
    {
        const long g = list[e];
        const AmrNode N = nodes[lnode[e]];
        acc += adj_phit(N, g, phib, lam) * pot[g] + (A0[g] * a0[g] + A1[g] * a1[g] + A2[g] * a2[g]);
    }
    acc = adj_block_sum(acc, sh);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = acc;
}

// the level deposit's transpose for every particle of level l's nodes (branch
// weights w1 = x - H floor(x / H), w2 = H - w1, times 4 pi G m / H^6)
__global__ void k_adj_lvl_depT(long n, double coeff, const int *__restrict__ node_of,
                               const AmrNode *__restrict__ nodes, const double *__restrict__ x,
                               const double *__restrict__ y, const double *__restrict__ z,
                               const double *__restrict__ m, const double *__restrict__ lam,
                               double *__restrict__ xb, double *__restrict__ mb)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int nd = node_of[i];
    if (nd < 0)
        return;
    const AmrNode N = nodes[nd];
    const double H = 1.0 / (1 << N.lv), ooh = (double)(1 << N.lv);
    const int fx = (int)(x[i] * ooh), fy = (int)(y[i] * ooh), fz = (int)(z[i] * ooh);
    double wx[2], wy[2], wz[2];
    wx[1] = x[i] - H * fx;
    wy[1] = y[i] - H * fy;
    wz[1] = z[i] - H * fz;
    wx[0] = H - wx[1];
    wy[0] = H - wy[1];
    wz[0] = H - wz[1];
    const double sgn[2] = {-1.0, 1.0};
    const double cm = coeff * m[i];
    const long sx = N.rd[0] + 1, sxy = sx * (N.rd[1] + 1);
    const long g0 = grid_index(N, fx - N.ts[0], fy - N.ts[1], fz - N.ts[2]);
    double dx = 0.0, dy = 0.0, dz = 0.0, dm = 0.0;
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
            {
                const double lq = lam[g0 + ii + jj * sx + kk * sxy];
                dx += sgn[ii] * wy[jj] * wz[kk] * lq;
                dy += wx[ii] * sgn[jj] * wz[kk] * lq;
                dz += wx[ii] * wy[jj] * sgn[kk] * lq;
                dm += wx[ii] * wy[jj] * wz[kk] * lq;
            }
    xb[i] += cm * dx;
    xb[n + i] += cm * dy;
    xb[2 * n + i] += cm * dz;
    mb[i] += coeff * dm;
}

// the head's phi-bar at its interior points gains the children's contributions
__global__ void k_adj_add_interior(int L, long D, const double *__restrict__ phic,
                                   double *__restrict__ phib)
{
    const int m = (1 << L) - 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long)m * m * m)
        return;
    const long i = 2 + t % m, j = 2 + (t / m) % m, k = 2 + t / ((long)m * m);
    const long g = i + j * D + k * D * D;
    phib[g] += phic[g];
}

// ---- host side ----------------------------------------------------------------------------
static int adj_check(qz_sim *s)
{
    const qz_config &c = s->cfg;
    if ((c.lmax != c.lmin && !c.freeze_tree) || c.force_stencil != 0 || c.bdry != 1 ||
        c.precision != QZ_PREC_FP64 || c.head_pot_method != 0)
    {
        set_error("adjoint: FP64 runs with the 3-point stencil, reflexive walls and the "
                  "multigrid head solve, head-only or with a frozen refinement tree only");
        return QZ_FAILURE;
    }
    if (c.total_mass <= 0.0)
    {
        set_error("adjoint: total_mass must be positive");
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

static bool amr_adj(const qz_sim *s);

// record layout of a stored state: x y z vx vy vz ax ay az (n each), the head
// potential (gpts), then on a frozen refinement tree every level's potential
static long rec_len(const qz_sim *s)
{
    long r = 9 * s->n + s->gpts;
    if (amr_adj(s))
        for (int l = 1; l < s->amr_nlev; l++)
            r += s->amr[l].grid_total;
    return r;
}

static bool copy_d2d(qz_sim *s, double *dst, const double *src, long count)
{
    return check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToDevice,
                                      s->stream),
                      "adjoint state copy");
}

static bool save_state(qz_sim *s, double *rec)
{
    const long n = s->n;
    const double *src[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    for (int q = 0; q < 9; q++)
        if (!copy_d2d(s, rec + q * n, src[q], n))
            return false;
    if (!copy_d2d(s, rec + 9 * n, s->pot, s->gpts))
        return false;
    if (amr_adj(s))
    {
        long o = 9 * n + s->gpts;
        for (int l = 1; l < s->amr_nlev; l++)
        {
            if (!copy_d2d(s, rec + o, s->amr[l].pot, s->amr[l].grid_total))
                return false;
            o += s->amr[l].grid_total;
        }
    }
    return true;
}

static bool load_state(qz_sim *s, const double *rec)
{
    const long n = s->n;
    double *dst[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    for (int q = 0; q < 9; q++)
        if (!copy_d2d(s, dst[q], rec + q * n, n))
            return false;
    if (!copy_d2d(s, s->pot, rec + 9 * n, s->gpts))
        return false;
    if (amr_adj(s))
    {
        long o = 9 * n + s->gpts;
        for (int l = 1; l < s->amr_nlev; l++)
        {
            if (!copy_d2d(s, s->amr[l].pot, rec + o, s->amr[l].grid_total))
                return false;
            o += s->amr[l].grid_total;
        }
    }
    return true;
}

// A stored state made current for a pull-back: particles and potentials loaded,
// particles reassigned to the frozen tree, grid accelerations recomputed.
static int prepare_state(qz_sim *s, const double *rec)
{
    if (!load_state(s, rec))
        return QZ_FAILURE;
    if (!amr_adj(s))
        return QZ_SUCCESS;
    return (amr_reassign(s) || grid_accel_head(s) || amr_grid_accel(s)) ? QZ_FAILURE
                                                                         : QZ_SUCCESS;
}

static int adj_alloc(qz_sim *s, long ck_recs, long seg_recs)
{
    if (!s->adj)
        s->adj = new Adjoint();
    Adjoint &A = *s->adj;
    const long n = s->n > 0 ? s->n : 1, rl = rec_len(s);
    const bool fresh_lam = A.lam.p == nullptr || A.lam.cap < s->gpts;
    const bool fresh_phib = A.phib.p == nullptr || A.phib.cap < s->gpts;
    if (!A.xb.ensure(s->mem, 3 * n) || !A.vb.ensure(s->mem, 3 * n) || !A.mb.ensure(s->mem, n) ||
        !A.ac.ensure(s->mem, 3 * n) || !A.ab.ensure(s->mem, 3 * n) ||
        !A.Ab.ensure(s->mem, 3 * s->gpts) || !A.phib.ensure(s->mem, s->gpts) ||
        !A.lam.ensure(s->mem, s->gpts) || !A.cs.ensure(s->mem, 24 * n) ||
        !A.red.ensure(s->mem, 2L * ADJ_RED_BLOCKS + 16) ||
        (ck_recs > 0 && !A.ck.ensure(s->mem, ck_recs * rl)) ||
        (seg_recs > 0 && !A.seg.ensure(s->mem, seg_recs * rl)) ||
        (seg_recs > 0 && !A.fin.ensure(s->mem, rl)) || !A.tgt.ensure(s->mem, 3 * n))
    {
        set_error("adjoint buffers: out of device memory");
        return QZ_FAILURE;
    }
    // phibar is written on the interior only: its boundary stays zero
    if (fresh_phib)
        cudaMemsetAsync(A.phib.p, 0, A.phib.cap * sizeof(double), s->stream);
    if (fresh_lam)
        cudaMemsetAsync(A.lam.p, 0, A.lam.cap * sizeof(double), s->stream);
    if (!A.host && !check_cuda(cudaMallocHost((void **)&A.host, 8 * sizeof(double)),
                               "adjoint pinned"))
        return QZ_FAILURE;
    return QZ_SUCCESS;
}

// mbar += the total-mass term of this pull-back is accumulated in red[2*RB + 8].
static double *mbar_acc(qz_sim *s) { return s->adj->red.p + 2L * ADJ_RED_BLOCKS + 8; }

static bool amr_adj(const qz_sim *s) { return s->cfg.lmax > s->cfg.lmin && s->amr_nlev > 1; }

// Per-level adjoint buffers for the current tree.
static int adj_alloc_levels(qz_sim *s)
{
    Adjoint &A = *s->adj;
    const int nl = s->amr_nlev;
    auto grow = [&](auto &v) {
        if ((int)v.size() < nl)
            v.resize(nl);
    };
    grow(A.lA);
    grow(A.lphic);
    grow(A.lphib);
    grow(A.llam);
    grow(A.lscr);
    grow(A.lthr);
    grow(A.lmask);
    const long n = s->n > 0 ? s->n : 1;
    if (!A.finest.ensure(s->mem, n) || !A.abh.ensure(s->mem, 3 * n) ||
        !A.phic0.ensure(s->mem, s->gpts))
        return QZ_FAILURE;
    long nnmax = 1;
    for (int l = 1; l < nl; l++)
    {
        const AmrLevel &L = s->amr[l];
        const long gt = L.grid_total > 0 ? L.grid_total : 1;
        const bool fresh = A.llam[l].p == nullptr || A.llam[l].cap < gt;
        if (!A.lA[l].ensure(s->mem, 3 * gt) || !A.lphic[l].ensure(s->mem, gt) ||
            !A.lphib[l].ensure(s->mem, gt) || !A.llam[l].ensure(s->mem, gt) ||
            !A.lscr[l].ensure(s->mem, gt) || !A.lmask[l].ensure(s->mem, gt) ||
            !A.lthr[l].ensure(s->mem, L.nnodes > 0 ? L.nnodes : 1))
            return QZ_FAILURE;
        if (fresh)
            cudaMemsetAsync(A.llam[l].p, 0, A.llam[l].cap * sizeof(double), s->stream);
        nnmax = std::max(nnmax, (long)L.nnodes);
    }
    return A.nrm.ensure(s->mem, nnmax) ? QZ_SUCCESS : QZ_FAILURE;
}

// a-bar deposited on the grid of level l >= 1 from the particles whose finest
// level is l (sort by level cell, segmented sums, point sums: fixed order)
static int adj_level_deposit(qz_sim *s, int l, const double *x, const double *y, const double *z,
                             const double *ab)
{
    Adjoint &A = *s->adj;
    AmrLevel &L = s->amr[l];
    const long n = s->n;
    double *A0 = A.lA[l].p, *A1 = A0 + L.grid_total, *A2 = A1 + L.grid_total;
    if (!s->amr_tmp.ensure(s->mem, 2 * n + 2) || !L.cell_seg.ensure(s->mem, L.box_total))
        return QZ_FAILURE;
    int *flag = s->amr_tmp.p, *slot = flag + n;
    launch(s, QZ_PROF_DEPOSIT, 8.0 * n, k_adj_flag_level, dim3(blocks_for(n, 256)), dim3(256), n,
           A.finest.p, l, flag);
    if (scan_exclusive(s, flag, slot, n))
        return QZ_FAILURE;
    int t[2];
    if (!check_cuda(cudaMemcpyAsync(A.host, slot + n - 1, sizeof(int), cudaMemcpyDeviceToHost,
                                    s->stream), "adjoint level count") ||
        !check_cuda(cudaMemcpyAsync((char *)A.host + sizeof(int), flag + n - 1, sizeof(int),
                                    cudaMemcpyDeviceToHost, s->stream), "adjoint level count") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "adjoint level count"))
        return QZ_FAILURE;
    memcpy(t, A.host, sizeof t);
    const long m = (long)t[0] + t[1];
    if (m == 0)
    {
        cudaMemsetAsync(A0, 0, 3 * L.grid_total * sizeof(double), s->stream);
        return QZ_SUCCESS;
    }
    launch(s, QZ_PROF_DEPOSIT, 44.0 * n, k_adj_lvl_keys, dim3(blocks_for(n, 256)), dim3(256), n, l,
           A.finest.p, s->node_of[l].p, L.nodes.p, x, y, z, slot, s->sort.k0, s->sort.v0);
    int bits = 1;
    while ((1L << bits) < L.box_total)
        bits++;
    unsigned *ks;
    int *perm;
    if (deposit_segments(s, m, bits, L.cell_seg.p, L.box_total, &ks, &perm, 0u))
        return QZ_FAILURE;
    if (!A.cs.ensure(s->mem, 24 * m + 24))
        return QZ_FAILURE;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const long blocks = std::min((m * 32 + 255) / 256, (long)sms * 16);
    cudaMemsetAsync(s->flags + F_NLONG, 0, sizeof(int), s->stream);
    launch(s, QZ_PROF_DEPOSIT, 56.0 * m, k_adj_seg_reduce, dim3((int)blocks), dim3(256),
           L.h[0].lv, perm, s->seg_start, s->flags, s->long_seg, x, y, z, ab, ab + n, ab + 2 * n,
           A.cs.p);
    launch(s, QZ_PROF_DEPOSIT, 0.0, k_adj_seg_long, dim3(2 * sms), dim3(ADJ_SEG_LONG_THREADS), L.h[0].lv,
           perm, s->seg_start, s->flags, s->long_seg, x, y, z, ab, ab + n, ab + 2 * n, A.cs.p);
    launch(s, QZ_PROF_DEPOSIT, 24.0 * L.grid_total, k_adj_lvl_point_gather3,
           dim3(blocks_for(L.grid_total, 256)), dim3(256), L.grid_total, L.nnodes, L.nodes.p,
           L.cell_seg.p, A.cs.p, A0, A1, A2);
    return check_cuda(cudaGetLastError(), "adjoint level deposit") ? QZ_SUCCESS : QZ_FAILURE;
}

// Vector-Jacobian product of the force at the positions (x, y, z) with
// potential pot, for the accelerations' adjoint ab (3n): adds into xb (3n), mb
// (n) and the total-mass accumulator.  lam is the solve's initial guess.  With
// refinement levels (a frozen tree), the levels' potentials, accelerations and
// particle assignments must be those of this state.
static int force_vjp(qz_sim *s, const double *x, const double *y, const double *z,
                     const double *pot, const double *ab, int *cycles)
{
    Adjoint &A = *s->adj;
    const long n = s->n;
    const int L = s->L;
    const long D = s->D;
    const double H = 1.0 / (1 << L);
    const double o2h = 1.0 / (2.0 * H), oh2 = 1.0 / (H * H);
    const double coeff = 4.0 * s->cfg.G * QZ_PI_D / (H * H * H);
    *cycles = 0;
    if (n == 0)
        return QZ_SUCCESS;
    const bool amr = amr_adj(s);
    const int nl = amr ? s->amr_nlev : 1;
    const double *abh = ab;
    if (amr)
    {
        if (adj_alloc_levels(s))
        {
            set_error("adjoint level buffers: out of device memory");
            return QZ_FAILURE;
        }
        NodeOfPtrs no{};
        for (int l = 0; l < nl; l++)
            no.p[l] = s->node_of[l].p;
        launch(s, QZ_PROF_GATHER, 8.0 * n * nl, k_adj_finest, dim3(blocks_for(n, 256)), dim3(256),
               n, nl, no, A.finest.p);
        launch(s, QZ_PROF_GATHER, 56.0 * n, k_adj_mask_ab, dim3(blocks_for(n, 256)), dim3(256), n,
               A.finest.p, ab, A.abh.p);
        abh = A.abh.p;
    }
    // head grid accelerations of this state (interior; the shell values stay)
    if (grid_accel_head_from(s, pot))
        return QZ_FAILURE;
    int *perm;
    if (head_segments(s, x, y, z, &perm))
        return QZ_FAILURE;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const long blocks = std::min((n * 32 + 255) / 256, (long)sms * 16);
    if (!A.cs.ensure(s->mem, 24 * n + 24))
        return QZ_FAILURE;
    cudaMemsetAsync(s->flags + F_NLONG, 0, sizeof(int), s->stream);
    launch(s, QZ_PROF_DEPOSIT, 56.0 * n, k_adj_seg_reduce, dim3((int)blocks), dim3(256), L, perm,
           s->seg_start, s->flags, s->long_seg, x, y, z, abh, abh + n, abh + 2 * n, A.cs.p);
    launch(s, QZ_PROF_DEPOSIT, 0.0, k_adj_seg_long, dim3(2 * sms), dim3(ADJ_SEG_LONG_THREADS), L, perm,
           s->seg_start, s->flags, s->long_seg, x, y, z, abh, abh + n, abh + 2 * n, A.cs.p);
    double *Abx = A.Ab.p, *Aby = A.Ab.p + s->gpts, *Abz = A.Ab.p + 2 * s->gpts;
    launch(s, QZ_PROF_DEPOSIT, 24.0 * s->gpts, k_adj_point_gather, dim3(blocks_for(s->gpts, 256)),
           dim3(256), D, s->cell_seg, A.cs.p, Abx, Aby, Abz);
    if (amr)
    {
        // the finest-level gathers' transposes, then the levels from the finest down
        for (int l = 1; l < nl; l++)
            if (adj_level_deposit(s, l, x, y, z, ab))
                return QZ_FAILURE;
        LevelRefs R{};
        R.nlev = nl;
        for (int l = 0; l < nl; l++)
        {
            R.nodes[l] = s->amr[l].nodes.p;
            R.node_of[l] = s->node_of[l].p;
            R.ax[l] = l == 0 ? s->gax : s->amr[l].ax;
            R.ay[l] = l == 0 ? s->gay : s->amr[l].ay;
            R.az[l] = l == 0 ? s->gaz : s->amr[l].az;
        }
        launch(s, QZ_PROF_GATHER, 112.0 * n, k_adj_gather_w, dim3(blocks_for(n, 256)), dim3(256), n,
               R, A.finest.p, x, y, z, ab, A.xb.p);
        cudaMemsetAsync(A.phic0.p, 0, s->gpts * sizeof(double), s->stream);
        for (int l = 1; l < nl; l++)
            cudaMemsetAsync(A.lphic[l].p, 0, s->amr[l].grid_total * sizeof(double), s->stream);
        for (int l = nl - 1; l >= 1; l--)
        {
            AmrLevel &Lv = s->amr[l];
            AmrLevel &P = s->amr[l - 1];
            const long gt = Lv.grid_total;
            double *A0 = A.lA[l].p, *A1 = A0 + gt, *A2 = A1 + gt;
            double *pA0, *pA1, *pA2, *pphic;
            if (l == 1)
            {
                pA0 = Abx;
                pA1 = Aby;
                pA2 = Abz;
                pphic = A.phic0.p;
            }
            else
            {
                const long pg = P.grid_total;
                pA0 = A.lA[l - 1].p;
                pA1 = pA0 + pg;
                pA2 = pA1 + pg;
                pphic = A.lphic[l - 1].p;
            }
            cudaMemsetAsync(A.lmask[l].p, 0, gt * sizeof(int), s->stream);
            if (Lv.intr_total > 0)
                launch(s, QZ_PROF_OTHER, 8.0 * Lv.intr_total, k_adj_set_mask,
                       dim3(blocks_for(Lv.intr_total, 256)), dim3(256), Lv.intr_total, Lv.intr.p,
                       A.lmask[l].p);
            launch(s, QZ_PROF_GRADIENT, 60.0 * gt, k_adj_lvl_negdiv, dim3(blocks_for(gt, 256)),
                   dim3(256), gt, Lv.nnodes, Lv.nodes.p, A.lmask[l].p, A0, A1, A2, A.lphic[l].p,
                   A.lphib[l].p);
            // node thresholds from the rhs norms; nodes with a zero rhs keep lam = 0
            launch(s, QZ_PROF_OTHER, 8.0 * Lv.intr_total, k_adj_node_norm, dim3(Lv.nnodes),
                   dim3(256), Lv.nodes.p, Lv.intr.p, A.lphib[l].p, A.nrm.p);
            std::vector<double> nrm(Lv.nnodes);
            if (!check_cuda(cudaMemcpyAsync(nrm.data(), A.nrm.p, Lv.nnodes * sizeof(double),
                                            cudaMemcpyDeviceToHost, s->stream), "node norms") ||
                !check_cuda(cudaStreamSynchronize(s->stream), "node norms"))
                return QZ_FAILURE;
            std::vector<char> skip(Lv.nnodes, 0);
            std::vector<double> thr(Lv.nnodes, 0.0);
            const double rt = s->cfg.adjoint_tol;
            for (int q = 0; q < Lv.nnodes; q++)
            {
                skip[q] = nrm[q] == 0.0 || Lv.h[q].nintr == 0;
                thr[q] = rt * rt * nrm[q];
                if (skip[q])
                {
                    const AmrNode &N = Lv.h[q];
                    const long pts = (long)(N.rd[0] + 1) * (N.rd[1] + 1) * (N.rd[2] + 1);
                    cudaMemsetAsync(A.llam[l].p + N.grid_off, 0, pts * sizeof(double), s->stream);
                }
            }
            if (!check_cuda(cudaMemcpyAsync(A.lthr[l].p, thr.data(), Lv.nnodes * sizeof(double),
                                            cudaMemcpyHostToDevice, s->stream), "node thresholds"))
                return QZ_FAILURE;
            const long long it0 = s->stats.cg_iterations;
            if (cg_level_adjoint(s, l, A.llam[l].p, A.lphib[l].p, A.lscr[l].p, A.lthr[l].p, skip))
                return QZ_FAILURE;
            *cycles += (int)(s->stats.cg_iterations - it0);
            s->stats.cg_iterations = it0; // the forward's count stays the forward's
            if (Lv.bdry_total > 0)
            {
                const long m8 = 8L * Lv.bdry_total;
                if (!ensure_sort(s, m8))
                {
                    set_error("adjoint boundary transposes: sort buffers");
                    return QZ_FAILURE;
                }
                int bits = 1;
                while (bits < 32 && (1L << bits) < P.grid_total)
                    bits++;
                launch(s, QZ_PROF_OTHER, 8.0 * m8, k_adj_bdry_keys, dim3(blocks_for(m8, 256)),
                       dim3(256), Lv.bdry_total, Lv.bdry.p, Lv.bdry_node.p, Lv.nodes.p, P.nodes.p,
                       s->sort.k0, s->sort.v0);
                unsigned *bk;
                int *bv;
                if (radix_sort_pairs(s, m8, bits, &bk, &bv))
                    return QZ_FAILURE;
                launch(s, QZ_PROF_OTHER, 160.0 * Lv.bdry_total, k_adj_bdry_sum,
                       dim3(blocks_for(m8, 256)), dim3(256), m8, bk, bv, Lv.bdry.p,
                       Lv.bdry_node.p, Lv.nodes.p, A.lphib[l].p, A.llam[l].p, A0, A1, A2, pA0,
                       pA1, pA2, pphic);
            }
            if (Lv.simb_total > 0)
            {
                launch(s, QZ_PROF_OTHER, 96.0 * Lv.simb_total, k_adj_simb_T, dim3(ADJ_RED_BLOCKS),
                       dim3(256), Lv.simb_total, Lv.simb.p, Lv.simb_node.p, Lv.nodes.p,
                       A.lphib[l].p, A.llam[l].p, Lv.pot, A0, A1, A2, Lv.ax, Lv.ay, Lv.az,
                       A.red.p);
                launch(s, QZ_PROF_OTHER, 8.0 * ADJ_RED_BLOCKS, k_adj_final, dim3(1), dim3(256),
                       ADJ_RED_BLOCKS, A.red.p, 1.0 / s->cfg.total_mass, 1, mbar_acc(s));
            }
            const double Hl = 1.0 / (1 << Lv.h[0].lv);
            const double cl = 4.0 * s->cfg.G * QZ_PI_D / (Hl * Hl * Hl * Hl * Hl * Hl);
            launch(s, QZ_PROF_GATHER, 144.0 * n, k_adj_lvl_depT, dim3(blocks_for(n, 256)),
                   dim3(256), n, cl, s->node_of[l].p, Lv.nodes.p, x, y, z, s->m, A.llam[l].p,
                   A.xb.p, A.mb.p);
        }
    }
    const long m = (1L << L) - 1;
    launch(s, QZ_PROF_GRADIENT, 32.0 * m * m * m, k_adj_negdiv, dim3(blocks_for(m * m * m, 256)),
           dim3(256), L, D, o2h, Abx, Aby, Abz, A.phib.p);
    if (amr)
        launch(s, QZ_PROF_GRADIENT, 16.0 * m * m * m, k_adj_add_interior,
               dim3(blocks_for(m * m * m, 256)), dim3(256), L, D, A.phic0.p, A.phib.p);
    int hc = 0;
    if (solve_zero_bc(s, A.lam.p, A.phib.p, s->cfg.adjoint_tol, A.red.p, A.host, &hc))
        return QZ_FAILURE;
    *cycles += hc;
    const long nb = (1L << L) + 1;
    launch(s, QZ_PROF_OTHER, 80.0 * (nb * nb * nb - m * m * m), k_adj_shell,
           dim3(ADJ_RED_BLOCKS), dim3(256), L, D, o2h, oh2, pot, A.lam.p, Abx, Aby, Abz, s->gax,
           s->gay, s->gaz, amr ? (const double *)A.phic0.p : nullptr, A.red.p);
    launch(s, QZ_PROF_OTHER, 8.0 * ADJ_RED_BLOCKS, k_adj_final, dim3(1), dim3(256), ADJ_RED_BLOCKS,
           A.red.p, 1.0 / s->cfg.total_mass, 1, mbar_acc(s));
    launch(s, QZ_PROF_GATHER, 112.0 * n + 32.0 * 8 * n, k_adj_gather, dim3(blocks_for(n, 256)),
           dim3(256), n, L, D, coeff, x, y, z, s->m, abh, abh + n, abh + 2 * n, s->gax, s->gay,
           s->gaz, A.lam.p, A.xb.p, A.xb.p + n, A.xb.p + 2 * n, A.mb.p, s->flags);
    return check_cuda(cudaGetLastError(), "adjoint force") ? QZ_SUCCESS : QZ_FAILURE;
}

static bool d2h_pinned_or_staged(qz_sim *s, double *dst, const double *src, long count)
{
    if (count <= 0 || !dst)
        return true;
    return check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyDeviceToHost,
                                      s->stream),
                      "adjoint d2h");
}

static bool h2d_any(qz_sim *s, double *dst, const double *src, long count)
{
    return check_cuda(cudaMemcpyAsync(dst, src, count * sizeof(double), cudaMemcpyHostToDevice,
                                      s->stream),
                      "adjoint h2d") &&
           check_cuda(cudaStreamSynchronize(s->stream), "adjoint h2d sync");
}

// Restores the simulation to the stored state rec and makes its density and
// grid fields consistent with it.
static int restore_full(qz_sim *s, const double *rec)
{
    if (!load_state(s, rec))
        return QZ_FAILURE;
    if (amr_adj(s))
        return (amr_reassign(s) || deposit_head(s) || amr_deposit(s) || grid_accel_head(s) ||
                amr_grid_accel(s))
                   ? QZ_FAILURE
                   : QZ_SUCCESS;
    return (deposit_head(s) || grid_accel_head(s)) ? QZ_FAILURE : QZ_SUCCESS;
}

} // namespace qz

using namespace qz;

extern "C" {

int qz_force_vjp(qz_sim *s, const double *abx, const double *aby, const double *abz, double *gx,
                 double *gy, double *gz, double *gm)
{
    if (!s || !abx || !aby || !abz)
    {
        set_error("qz_force_vjp: null argument");
        return QZ_FAILURE;
    }
    if (adj_check(s))
        return QZ_FAILURE;
    if (!s->forces_ready && qz_init_forces(s))
        return QZ_FAILURE;
    if (adj_alloc(s, 0, 0))
        return QZ_FAILURE;
    Adjoint &A = *s->adj;
    const long n = s->n;
    cudaMemsetAsync(A.xb.p, 0, 3 * n * sizeof(double), s->stream);
    cudaMemsetAsync(A.mb.p, 0, n * sizeof(double), s->stream);
    cudaMemsetAsync(A.lam.p, 0, s->gpts * sizeof(double), s->stream);
    cudaMemsetAsync(mbar_acc(s), 0, sizeof(double), s->stream);
    if (amr_adj(s))
    {
        if (adj_alloc_levels(s))
        {
            set_error("adjoint level buffers: out of device memory");
            return QZ_FAILURE;
        }
        for (int l = 1; l < s->amr_nlev; l++)
            cudaMemsetAsync(A.llam[l].p, 0, A.llam[l].cap * sizeof(double), s->stream);
    }
    if (!h2d_any(s, A.ab.p, abx, n) || !h2d_any(s, A.ab.p + n, aby, n) ||
        !h2d_any(s, A.ab.p + 2 * n, abz, n))
        return QZ_FAILURE;
    int cyc = 0;
    if (force_vjp(s, s->x, s->y, s->z, s->pot, A.ab.p, &cyc))
        return QZ_FAILURE;
    launch(s, QZ_PROF_OTHER, 16.0 * n, k_adj_add_scalar, dim3(blocks_for(n, 256)), dim3(256), n,
           mbar_acc(s), A.mb.p);
    // the grid fields again hold this state's accelerations (force_vjp recomputed them)
    if (!d2h_pinned_or_staged(s, gx, A.xb.p, n) || !d2h_pinned_or_staged(s, gy, A.xb.p + n, n) ||
        !d2h_pinned_or_staged(s, gz, A.xb.p + 2 * n, n) || !d2h_pinned_or_staged(s, gm, A.mb.p, n))
        return QZ_FAILURE;
    s->stats.adjoint_cycles += cyc;
    return check_flags(s);
}

int qz_adjoint_final_loss(qz_sim *s, int nsteps, double dt, int checkpoint_every,
                          const double *tx, const double *ty, const double *tz, double *gx,
                          double *gy, double *gz, double *gvx, double *gvy, double *gvz,
                          double *gm, qz_adjoint_stats *st)
{
    if (!s || nsteps < 1 || !(dt > 0.0) || !tx || !ty || !tz)
    {
        set_error("qz_adjoint_final_loss: bad arguments (nsteps >= 1, dt > 0, targets)");
        return QZ_FAILURE;
    }
    if (adj_check(s))
        return QZ_FAILURE;
    if (!s->forces_ready && qz_init_forces(s))
        return QZ_FAILURE;
    const long n = s->n;
    const int K = (checkpoint_every <= 0 || checkpoint_every > nsteps) ? nsteps : checkpoint_every;
    const int nseg = (nsteps + K - 1) / K;
    const int n0_last = (nseg - 1) * K;
    cudaMemPool_t pool = s->mem.pool;
    unsigned long long zero = 0;
    if (pool)
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &zero);
    if (adj_alloc(s, nseg, K + 1))
        return QZ_FAILURE;
    Adjoint &A = *s->adj;
    const long rl = rec_len(s);
    if (!h2d_any(s, A.tgt.p, tx, n) || !h2d_any(s, A.tgt.p + n, ty, n) ||
        !h2d_any(s, A.tgt.p + 2 * n, tz, n))
        return QZ_FAILURE;
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    int rc = QZ_FAILURE;
    long long cycles = 0, recomputed = 0;
    do
    {
        cudaEventRecord(e0, s->stream);
        // ---- forward: checkpoints every K steps, the last segment's states kept
        if (!save_state(s, A.ck.p))
            break;
        if (n0_last == 0 && !save_state(s, A.seg.p))
            break;
        bool ok = true;
        for (int q = 0; q < nsteps && ok; q++)
        {
            if (step_core(s, dt))
            {
                ok = false;
                break;
            }
            const int k = q + 1;
            if (k % K == 0 && k < nsteps)
                ok = save_state(s, A.ck.p + (long)(k / K) * rl);
            if (ok && k >= n0_last)
                ok = save_state(s, A.seg.p + (long)(k - n0_last) * rl);
        }
        if (!ok || !save_state(s, A.fin.p) || check_flags(s))
            break;
        // ---- loss and the adjoint of the final state
        launch(s, QZ_PROF_OTHER, 56.0 * n, k_adj_loss, dim3(ADJ_RED_BLOCKS), dim3(256), n, s->x,
               s->y, s->z, A.tgt.p, A.xb.p, A.red.p);
        launch(s, QZ_PROF_OTHER, 8.0 * ADJ_RED_BLOCKS, k_adj_final, dim3(1), dim3(256),
               ADJ_RED_BLOCKS, A.red.p, 1.0 / (double)n, 0, A.red.p + 2L * ADJ_RED_BLOCKS + 4);
        cudaMemsetAsync(A.vb.p, 0, 3 * n * sizeof(double), s->stream);
        cudaMemsetAsync(A.ac.p, 0, 3 * n * sizeof(double), s->stream);
        cudaMemsetAsync(A.mb.p, 0, n * sizeof(double), s->stream);
        cudaMemsetAsync(A.lam.p, 0, s->gpts * sizeof(double), s->stream);
        cudaMemsetAsync(mbar_acc(s), 0, sizeof(double), s->stream);
        if (amr_adj(s))
        {
            if (adj_alloc_levels(s))
            {
                set_error("adjoint level buffers: out of device memory");
                break;
            }
            for (int l = 1; l < s->amr_nlev; l++)
                cudaMemsetAsync(A.llam[l].p, 0, A.llam[l].cap * sizeof(double), s->stream);
        }
        cudaEventRecord(e1, s->stream);
        // ---- reverse sweep, segment by segment
        for (int sg = nseg - 1; sg >= 0 && ok; sg--)
        {
            const int n0 = sg * K, n1 = std::min(n0 + K, nsteps);
            if (sg != nseg - 1)
            {
                if (!load_state(s, A.ck.p + (long)sg * rl) ||
                    !copy_d2d(s, A.seg.p, A.ck.p + (long)sg * rl, rl))
                {
                    ok = false;
                    break;
                }
                for (int j = 1; j <= n1 - n0 && ok; j++)
                {
                    if (step_core(s, dt))
                        ok = false;
                    else
                        ok = save_state(s, A.seg.p + (long)j * rl);
                    recomputed++;
                }
            }
            for (int q = n1 - 1; q >= n0 && ok; q--)
            {
                const double *Sn = A.seg.p + (long)(q - n0) * rl;
                const double *S1 = A.seg.p + (long)(q + 1 - n0) * rl;
                launch(s, QZ_PROF_LEAPFROG, 72.0 * n, k_adj_kick, dim3(blocks_for(3 * n, 256)),
                       dim3(256), 3 * n, dt, A.vb.p, A.ac.p, A.ab.p);
                int cyc = 0;
                if (amr_adj(s))
                {
                    // the levels' fields of the state are rebuilt in the simulation
                    if (prepare_state(s, S1) ||
                        force_vjp(s, s->x, s->y, s->z, s->pot, A.ab.p, &cyc))
                    {
                        ok = false;
                        break;
                    }
                }
                else if (force_vjp(s, S1, S1 + n, S1 + 2 * n, S1 + 9 * n, A.ab.p, &cyc))
                {
                    ok = false;
                    break;
                }
                cycles += cyc;
                launch(s, QZ_PROF_LEAPFROG, 144.0 * n, k_adj_kick_drift,
                       dim3(blocks_for(n, 256)), dim3(256), n, dt, Sn, A.xb.p, A.vb.p, A.ac.p);
            }
        }
        if (!ok)
            break;
        // a_0 = F(x_0) of the step-0 forces feeds the first kick
        {
            const double *S0 = A.seg.p;
            int cyc = 0;
            if (amr_adj(s))
            {
                if (prepare_state(s, S0) || force_vjp(s, s->x, s->y, s->z, s->pot, A.ac.p, &cyc))
                    break;
            }
            else if (force_vjp(s, S0, S0 + n, S0 + 2 * n, S0 + 9 * n, A.ac.p, &cyc))
                break;
            cycles += cyc;
        }
        launch(s, QZ_PROF_OTHER, 16.0 * n, k_adj_add_scalar, dim3(blocks_for(n, 256)), dim3(256),
               n, mbar_acc(s), A.mb.p);
        cudaEventRecord(e2, s->stream);
        if (restore_full(s, A.fin.p))
            break;
        if (!d2h_pinned_or_staged(s, gx, A.xb.p, n) ||
            !d2h_pinned_or_staged(s, gy, A.xb.p + n, n) ||
            !d2h_pinned_or_staged(s, gz, A.xb.p + 2 * n, n) ||
            !d2h_pinned_or_staged(s, gvx, A.vb.p, n) ||
            !d2h_pinned_or_staged(s, gvy, A.vb.p + n, n) ||
            !d2h_pinned_or_staged(s, gvz, A.vb.p + 2 * n, n) ||
            !d2h_pinned_or_staged(s, gm, A.mb.p, n) ||
            !check_cuda(cudaMemcpyAsync(A.host, A.red.p + 2L * ADJ_RED_BLOCKS + 4, sizeof(double),
                                        cudaMemcpyDeviceToHost, s->stream),
                        "loss"))
            break;
        if (check_flags(s))
            break;
        float f_ms = 0.f, r_ms = 0.f;
        cudaEventElapsedTime(&f_ms, e0, e1);
        cudaEventElapsedTime(&r_ms, e1, e2);
        s->stats.adjoint_cycles += cycles;
        if (st)
        {
            memset(st, 0, sizeof *st);
            st->loss = A.host[0];
            st->forward_ms = f_ms;
            st->reverse_ms = r_ms;
            st->adjoint_cycles = cycles;
            st->recomputed_steps = recomputed;
            st->checkpoints = nseg;
            unsigned long long hi = 0;
            if (pool)
                cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemHigh, &hi);
            st->pool_peak_bytes = (double)hi;
            st->stored_bytes = 8.0 * rl * (nseg + K + 2);
        }
        rc = QZ_SUCCESS;
    } while (0);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    return rc;
}

} // extern "C"

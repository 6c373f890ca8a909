// qz_poisson.cu -- head-node Poisson solve (potential_head_node.c:32-179) by
// multigrid cycles (force_methods/multigrid.c:106-229) on the embedded solve
// grid of the head fields, with the convergence test of poisson_error.c:36-133.
//
// Kernels (FP64, and FP32 instances for the mixed-precision form):
//   k_gs_rb          one colour of a red-black Gauss-Seidel sweep
//   k_gs_lex_cta     lexicographic Gauss-Seidel in the reference's order, by
//                    i+j+k wavefronts inside one CTA (parity mode)
//   k_jacobi         weighted Jacobi ping-pong sweep (jacobi.c:29-82)
//   k_resid_restrict residual at the even fine points only, injected into the
//                    coarse right-hand side (multigrid.c:140-150 + 29-49: the
//                    reference computes the residual everywhere but reads only
//                    the injected points)
//   k_prolong_add    trilinear prolongation written as a gather over the coarse
//                    points in the reference's scatter order, fused with
//                    phi += dphi (multigrid.c:51-104, 199-209)
//   k_check_*        ratio test + residual norm, fixed-tree deterministic sums
#include <cooperative_groups.h>
#include <cuda_pipeline.h>
#include <mutex>

#include "qz_internal.cuh"

namespace qz {

#define QZ_PI_D 3.14159265358979323846

template <typename T>
__device__ __forceinline__ T gs_point(const T *__restrict__ rho, T *__restrict__ phi, long g,
                                      long sy, long sz, T H2, T w)
{
    const T one_sixth = (T)(1.0 / 6.0);
    T a = one_sixth * (-H2 * rho[g] + phi[g + 1] + phi[g - 1] + phi[g + sy] + phi[g - sy] +
                       phi[g + sz] + phi[g - sz]);
    return w * a + ((T)1.0 - w) * phi[g];
}

template <typename T>
__global__ void k_gs_rb(Grid<T> phi, Grid<T> rho, int color, T H2, T w)
{
    const int m = phi.n - 2;
    const int half = (m + 1) / 2;
    int ti = blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y;
    int k = 1 + blockIdx.z;
    if (ti >= half)
        return;
    int i0 = (((1 + j + k) & 1) == color) ? 1 : 2;
    int i = i0 + 2 * ti;
    if (i > m)
        return;
    long gp = phi.off + i + j * phi.sy + k * phi.sz;
    long gr = rho.off + i + j * rho.sy + k * rho.sz;
    const T one_sixth = (T)(1.0 / 6.0);
    T *p = phi.p;
    T a = one_sixth * (-H2 * rho.p[gr] + p[gp + 1] + p[gp - 1] + p[gp + phi.sy] +
                       p[gp - phi.sy] + p[gp + phi.sz] + p[gp - phi.sz]);
    p[gp] = w * a + ((T)1.0 - w) * p[gp];
}

// One whole red-black sweep per launch (the result of a red k_gs_rb launch
// followed by a black one, bit for bit), reading phi from `pin` and writing
// `pout` (ping-pong: CTAs never race on halos), with every phi value loaded
// from memory once per CTA and written once.  A CTA owns a tile of ZM_TX x
// ZM_TY interior points in (x, y) and a chunk of ZM_TZ planes in z, and marches
// up the chunk with a ring of phi planes in shared memory, staged by
// asynchronous copies (cp.async) two planes ahead of the arithmetic:
//   step s: load plane s+2 (the tile plus 2 points a side);
//           red points of plane s-1 over the tile and a 1-point ring around it
//           (from the old black values of planes s-2, s-1, s);
//           black points of plane s-2 over the tile (from the new red values
//           of planes s-3, s-2, s-1), and both points of each x pair of plane
//           s-2 written to pout.
// rho is read from memory where a point is updated (coalesced along x), each
// thread's loads issued at the top of the step so that they overlap the wait
// for the plane.  A
// ring point is a neighbouring CTA's tile point: both compute it from the same
// old values, so they agree bit for bit.  Algorithmic traffic: 24 B a point
// (phi and rho read, phi written); the phi halo adds (68 x 20) / (64 x 16) - 1
// = 0.33 reads a point and the rho ring 0.16, mostly served by L2.
constexpr int ZM_TX = 64, ZM_TY = 16; // z-chunks are sized by the host (zm_chunk)
constexpr int ZM_WX = ZM_TX + 4, ZM_WY = ZM_TY + 4; // phi window
constexpr int ZM_RX = ZM_TX + 2, ZM_RY = ZM_TY + 2; // red ring
constexpr int ZM_PH = 6;                            // planes held (two in flight)
constexpr int ZM_THREADS = 512;

template <typename T> constexpr size_t zm_smem_bytes()
{
    return sizeof(T) * (size_t)ZM_PH * ZM_WX * ZM_WY;
}

__device__ __forceinline__ int zm_slot(int z) { return ((z % ZM_PH) + ZM_PH) % ZM_PH; }

template <typename T>
__global__ void __launch_bounds__(ZM_THREADS)
    k_gs_rb_zm(Grid<T> pin, Grid<T> pout, Grid<T> rho, T H2, T w, int tz)
{
    extern __shared__ __align__(16) unsigned char zm_raw[];
    T *PH = reinterpret_cast<T *>(zm_raw); // [ZM_PH][ZM_WY][ZM_WX]
    const int n = pin.n, m = n - 2, last = n - 1;
    const int tid = threadIdx.x;
    const int x0 = 1 + blockIdx.x * ZM_TX, y0 = 1 + blockIdx.y * ZM_TY;
    const int kb = 1 + blockIdx.z * tz, ke = min(m, kb + tz - 1);
    const T one_sixth = (T)(1.0 / 6.0);
    // asynchronous loads of the phi window of plane z (points in range)
    auto load = [&](int z) {
        if (z >= 0 && z <= last && z >= kb - 2 && z <= ke + 2)
        {
            T *dst = PH + (size_t)zm_slot(z) * ZM_WX * ZM_WY;
            for (int e = tid; e < ZM_WX * ZM_WY; e += ZM_THREADS)
            {
                const int wy = e / ZM_WX, wx = e - wy * ZM_WX;
                const int gx = x0 - 2 + wx, gy = y0 - 2 + wy;
                if (gx >= 0 && gx <= last && gy >= 0 && gy <= last)
                    __pipeline_memcpy_async(dst + e, pin.p + pin.off + gx + gy * pin.sy + (long)z * pin.sz,
                                            sizeof(T));
            }
        }
        __pipeline_commit();
    };
    auto P = [&](int z) { return PH + (size_t)zm_slot(z) * ZM_WX * ZM_WY; };
    // a thread's red pairs (at most two: 33 x 18 = 594 pairs for 512 threads) and
    // its black pair (exactly one: 32 x 16), fixed for the whole march
    constexpr int NRP = ((ZM_RX / 2) * ZM_RY + ZM_THREADS - 1) / ZM_THREADS;
    static_assert((ZM_TX / 2) * ZM_TY == ZM_THREADS, "one black pair a thread");
    int rpx[NRP], rpy[NRP];
    for (int q = 0; q < NRP; q++)
    {
        const int e = tid + q * ZM_THREADS;
        rpy[q] = e / (ZM_RX / 2);
        rpx[q] = 2 * (e - rpy[q] * (ZM_RX / 2));
        if (e >= (ZM_RX / 2) * ZM_RY)
            rpy[q] = -1;
    }
    const int bty = tid / (ZM_TX / 2), bpx = 2 * (tid - bty * (ZM_TX / 2));
    load(kb - 2);
    load(kb - 1);
    for (int sp = kb - 2; sp <= ke + 2; sp++)
    {
        load(sp + 2);
        const int zr = sp - 1, zb = sp - 2;
        const bool do_red = zr >= kb - 1 && zr <= ke + 1 && zr >= 1 && zr <= m;
        const bool do_black = zb >= kb && zb <= ke;
        // this step's rho values, loaded before the wait
        T rv[NRP], bv = (T)0;
        int rl[NRP];
        for (int q = 0; q < NRP; q++)
        {
            rl[q] = -1;
            rv[q] = (T)0;
            if (!do_red || rpy[q] < 0)
                continue;
            const int gy = y0 - 1 + rpy[q];
            int rx = rpx[q], gx = x0 - 1 + rx;
            if ((gx + gy + zr) & 1)
            {
                rx++;
                gx++;
            }
            if (gx < 1 || gx > m || gy < 1 || gy > m)
                continue;
            rl[q] = (rx + 1) + (rpy[q] + 1) * ZM_WX;
            rv[q] = rho.p[rho.off + gx + gy * rho.sy + (long)zr * rho.sz];
        }
        const int bgy = y0 + bty, bgxa = x0 + bpx;
        const bool bpair = do_black && bgy <= m && bgxa <= m;
        const int bb = ((bgxa + bgy + zb) & 1) ? 0 : 1; // offset of the black member
        const bool bupd = bpair && bgxa + bb <= m;
        if (bupd)
            bv = rho.p[rho.off + bgxa + bb + bgy * rho.sy + (long)zb * rho.sz];
        __pipeline_wait_prior(2); // plane sp has landed
        __syncthreads();
        // red points of plane zr over the tile and its ring
        if (do_red)
        {
            T *pc = P(zr), *pd = P(zr - 1), *pu = P(zr + 1);
            for (int q = 0; q < NRP; q++)
            {
                const int l = rl[q];
                if (l < 0)
                    continue;
                const T a = one_sixth * (-H2 * rv[q] + pc[l + 1] + pc[l - 1] + pc[l + ZM_WX] +
                                         pc[l - ZM_WX] + pu[l] + pd[l]);
                pc[l] = w * a + ((T)1.0 - w) * pc[l];
            }
        }
        __syncthreads();
        // black point of this thread's pair of plane zb; the pair (its red member
        // final since the last step) goes to pout
        if (bpair)
        {
            T *pc = P(zb), *pd = P(zb - 1), *pu = P(zb + 1);
            T *out = pout.p + pout.off + (long)zb * pout.sz;
            const int la = (bpx + 2) + (bty + 2) * ZM_WX;
            const int l = la + bb;
            if (bupd)
            {
                const T a = one_sixth * (-H2 * bv + pc[l + 1] + pc[l - 1] + pc[l + ZM_WX] +
                                         pc[l - ZM_WX] + pu[l] + pd[l]);
                pc[l] = w * a + ((T)1.0 - w) * pc[l];
            }
            out[bgxa + bgy * pout.sy] = pc[la];
            if (bgxa + 1 <= m)
                out[bgxa + 1 + bgy * pout.sy] = pc[la + 1];
        }
        __syncthreads(); // the next step's load reuses the slot of plane sp - 4
    }
}

// Opt the fused sweep in to more than 48 KB of dynamic shared memory.
void init_kernel_attributes()
{
    cudaFuncSetAttribute(k_gs_rb_zm<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)zm_smem_bytes<double>());
    cudaFuncSetAttribute(k_gs_rb_zm<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)zm_smem_bytes<float>());
}

template <typename T>
__global__ void k_copy_interior(Grid<T> dst, Grid<T> src)
{
    const int m = src.n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > m)
        return;
    dst.p[dst.off + i + j * dst.sy + (long)k * dst.sz] = src.p[src.off + i + j * src.sy + (long)k * src.sz];
}

// Lexicographic sweeps (k slowest, i fastest) reproduced exactly: the update
// of point (i,j,k) reads new values at i-1, j-1, k-1 and old values at i+1,
// j+1, k+1, so all points with the same i+j+k are independent.
template <typename T>
__global__ void k_gs_lex_cta(Grid<T> phi, Grid<T> rho, int iters, T H2, T w)
{
    const int m = phi.n - 2;
    const long pairs = (long)m * m;
    const T one_sixth = (T)(1.0 / 6.0);
    T *p = phi.p;
    for (int it = 0; it < iters; it++)
    {
        for (int sidx = 3; sidx <= 3 * m; sidx++)
        {
            for (long q = threadIdx.x; q < pairs; q += blockDim.x)
            {
                int j = 1 + (int)(q % m), k = 1 + (int)(q / m);
                int i = sidx - j - k;
                if (i < 1 || i > m)
                    continue;
                long gp = phi.off + i + j * phi.sy + k * phi.sz;
                long gr = rho.off + i + j * rho.sy + k * rho.sz;
                T a = one_sixth * (-H2 * rho.p[gr] + p[gp + 1] + p[gp - 1] + p[gp + phi.sy] +
                                   p[gp - phi.sy] + p[gp + phi.sz] + p[gp - phi.sz]);
                p[gp] = w * a + ((T)1.0 - w) * p[gp];
            }
            __syncthreads();
        }
    }
}

template <typename T>
__global__ void k_jacobi(Grid<T> oldp, Grid<T> newp, Grid<T> rho, T C, T w)
{
    const int m = oldp.n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y;
    int k = 1 + blockIdx.z;
    if (i > m)
        return;
    long go = oldp.off + i + j * oldp.sy + k * oldp.sz;
    long gn = newp.off + i + j * newp.sy + k * newp.sz;
    long gr = rho.off + i + j * rho.sy + k * rho.sz;
    const T one_sixth = (T)(1.0 / 6.0);
    const T *o = oldp.p;
    T a = one_sixth * (C * rho.p[gr] + o[go + 1] + o[go - 1] + o[go + oldp.sy] + o[go - oldp.sy] +
                       o[go + oldp.sz] + o[go - oldp.sz]);
    newp.p[gn] = w * a + ((T)1.0 - w) * newp.p[gn];
}

template <typename T>
__global__ void k_copy_grid(Grid<T> dst, Grid<T> src)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y, k = blockIdx.z;
    if (i >= src.n)
        return;
    dst.p[dst.off + i + j * dst.sy + k * dst.sz] = src.p[src.off + i + j * src.sy + k * src.sz];
}

// rho_c(l) = scale * (rho(2l) + ooh2 * (6 phi(2l) - sum of 6 neighbours)) at
// the coarse interior points; the coarse boundary stays zero.  scale is 1 in
// the reference's lexicographic mode (plain injection, multigrid.c:29-49) and
// 1/2 with red-black smoothing: after a red-black sweep the residual lives on
// the red points only, and plain injection of it makes the cycle diverge
// (measured growth x4 per cycle on a Plummer density), while half injection
// converges at about 0.1 per cycle.
template <typename T>
__global__ void k_resid_restrict(Grid<T> phi, Grid<T> rho, Grid<T> rc, T ooh2, T scale)
{
    const int mc = rc.n - 2;
    int lx = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int ly = 1 + blockIdx.y;
    int lz = 1 + blockIdx.z;
    if (lx > mc)
        return;
    long gp = phi.off + 2 * lx + 2 * ly * phi.sy + 2 * lz * phi.sz;
    long gr = rho.off + 2 * lx + 2 * ly * rho.sy + 2 * lz * rho.sz;
    const T *p = phi.p;
    T r = rho.p[gr] + ooh2 * ((T)6 * p[gp] - p[gp + 1] - p[gp - 1] - p[gp + phi.sy] -
                              p[gp - phi.sy] - p[gp + phi.sz] - p[gp - phi.sz]);
    rc.p[rc.off + lx + ly * rc.sy + lz * rc.sz] = scale * r;
}

// phi(fine interior) += sum over contributing interior coarse points, in the
// coarse lexicographic order of the reference's scatter loop, of w * dphic.
template <typename T>
__global__ void k_prolong_add(Grid<T> phi, Grid<T> c)
{
    const int m = phi.n - 2;
    const int mc = c.n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y;
    int k = 1 + blockIdx.z;
    if (i > m)
        return;
    int cx0, cx1, cy0, cy1, cz0, cz1;
    T wx, wy, wz;
    if (i & 1) { cx0 = (i - 1) >> 1; cx1 = cx0 + 1; wx = (T)0.5; } else { cx0 = cx1 = i >> 1; wx = (T)1; }
    if (j & 1) { cy0 = (j - 1) >> 1; cy1 = cy0 + 1; wy = (T)0.5; } else { cy0 = cy1 = j >> 1; wy = (T)1; }
    if (k & 1) { cz0 = (k - 1) >> 1; cz1 = cz0 + 1; wz = (T)0.5; } else { cz0 = cz1 = k >> 1; wz = (T)1; }
    T acc;
    if (!(i & 1) && !(j & 1) && !(k & 1))
        acc = c.p[c.off + cx0 + cy0 * c.sy + cz0 * c.sz];
    else
    {
        const T wgt = wx * wy * wz;
        acc = (T)0;
        for (int cz = cz0; cz <= cz1; cz++)
        {
            if (cz < 1 || cz > mc)
                continue;
            for (int cy = cy0; cy <= cy1; cy++)
            {
                if (cy < 1 || cy > mc)
                    continue;
                for (int cx = cx0; cx <= cx1; cx++)
                {
                    if (cx < 1 || cx > mc)
                        continue;
                    acc += wgt * c.p[c.off + cx + cy * c.sy + cz * c.sz];
                }
            }
        }
    }
    phi.p[phi.off + i + j * phi.sy + k * phi.sz] += acc;
}

// ---- conjugate gradient as the smoother (smoother 2) ----------------------------
// conjugate_gradient_multigrid.c:29-176 on one level: r = rho + (1/H^2)(6 phi - sum),
// p = r, then up to min(iters, interior points) iterations of plain CG, leaving
// early when rs_new / rs_old < 1e-16.  One cooperative launch per call; each
// block adds its points' contributions in a fixed order, and after a grid
// barrier every block adds the block partials in block order, so all blocks hold
// the same sums (FP64) and take the same early exit.

template <typename T> struct CgsArgs {
    Grid<T> phi, rho;
    T *r, *p, *ap; // dense n^3, zero on the boundary
    double *part;  // 2 * gridDim partial sums
    int iters;
    GridBar bar;
};

__device__ __forceinline__ double cgs_block_sum(double v, double *sh)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0)
        sh[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
        t += sh[w];
    __syncthreads();
    return t;
}

// Sum of the gridDim partials at part, in block order (every block, every thread).
__device__ __forceinline__ double cgs_grid_sum(const double *part, double *sh)
{
    double v = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x)
        v += __ldcg(&part[b]);
    return cgs_block_sum(v, sh);
}

template <typename T> __global__ void __launch_bounds__(256) k_cg_smooth(CgsArgs<T> A)
{
    __shared__ double sh[32];
    __shared__ int sh_ok;
    const int n = A.phi.n, m = n - 2;
    const unsigned um = (unsigned)m, total = um * um * um;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
    const long n2 = (long)n * n;
    const T H = (T)1.0 / (T)(n - 1);
    const T oh2 = (T)1.0 / (H * H);
    const Grid<T> &P = A.phi, &R = A.rho;
    double *part0 = A.part, *part1 = A.part + gridDim.x;
    double acc = 0.0;
    for (unsigned t = gtid; t < total; t += gn)
    {
        const int i = 1 + (int)(t % um), j = 1 + (int)((t / um) % um), k = 1 + (int)(t / (um * um));
        const long gp = P.off + i + j * P.sy + k * P.sz;
        const long l = i + j * (long)n + k * n2;
        const T *ph = P.p;
        const T rv = R.p[R.off + i + j * R.sy + k * R.sz] +
                     oh2 * ((T)6.0 * ph[gp] - ph[gp + 1] - ph[gp - 1] - ph[gp + P.sy] -
                            ph[gp - P.sy] - ph[gp + P.sz] - ph[gp - P.sz]);
        A.r[l] = rv;
        A.p[l] = rv;
        acc += (double)rv * (double)rv;
    }
    double b = cgs_block_sum(acc, sh);
    if (threadIdx.x == 0)
        part0[blockIdx.x] = b;
    gbar_sync(A.bar, &sh_ok);
    double rsold = cgs_grid_sum(part0, sh);
    const long cap = (long)m * m * m;
    const long cycle = A.iters < cap ? A.iters : cap;
    for (long it = 0; it < cycle; it++)
    {
        acc = 0.0;
        for (unsigned t = gtid; t < total; t += gn)
        {
            const int i = 1 + (int)(t % um), j = 1 + (int)((t / um) % um), k = 1 + (int)(t / (um * um));
            const long l = i + j * (long)n + k * n2;
            const T *pp = A.p;
            const T a = -oh2 * ((T)6.0 * pp[l] - pp[l + 1] - pp[l - 1] - pp[l + n] - pp[l - n] -
                                pp[l + n2] - pp[l - n2]);
            A.ap[l] = a;
            acc += (double)pp[l] * (double)a;
        }
        b = cgs_block_sum(acc, sh);
        if (threadIdx.x == 0)
            part1[blockIdx.x] = b;
        gbar_sync(A.bar, &sh_ok);
        const T alpha = (T)(rsold / cgs_grid_sum(part1, sh));
        acc = 0.0;
        for (unsigned t = gtid; t < total; t += gn)
        {
            const int i = 1 + (int)(t % um), j = 1 + (int)((t / um) % um), k = 1 + (int)(t / (um * um));
            const long l = i + j * (long)n + k * n2;
            P.p[P.off + i + j * P.sy + k * P.sz] += alpha * A.p[l];
            const T rv = A.r[l] - alpha * A.ap[l];
            A.r[l] = rv;
            acc += (double)rv * (double)rv;
        }
        b = cgs_block_sum(acc, sh);
        if (threadIdx.x == 0)
            part0[blockIdx.x] = b;
        gbar_sync(A.bar, &sh_ok);
        const double rsnew = cgs_grid_sum(part0, sh);
        if (rsnew / rsold < 1.0e-16)
            break;
        const T beta = (T)(rsnew / rsold);
        for (unsigned t = gtid; t < total; t += gn)
        {
            const int i = 1 + (int)(t % um), j = 1 + (int)((t / um) % um), k = 1 + (int)(t / (um * um));
            const long l = i + j * (long)n + k * n2;
            A.p[l] = A.r[l] + beta * A.p[l];
        }
        rsold = rsnew;
        gbar_sync(A.bar, &sh_ok);
    }
}

// ---- host-side multigrid -----------------------------------------------------
template <typename T> struct CgsScratch {
    T *r = nullptr, *p = nullptr, *ap = nullptr;
};

template <typename T>
static int smooth_t(qz_sim *s, Grid<T> phi, Grid<T> rho, int iters, Grid<T> scratch,
                    Grid<T> alt, CgsScratch<T> cgs_scratch = CgsScratch<T>())
{
    const qz_config &c = s->cfg;
    const int n = phi.n;
    const int m = n - 2;
    if (m <= 0 || iters <= 0)
        return QZ_SUCCESS;
    if (c.smoother == 0)
    {
        T H2 = (T)((1.0 / (n - 1)) * (1.0 / (n - 1)));
        T w = (T)c.w_sor;
        if (c.gs_order == QZ_GS_LEX)
        {
            launch(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 3.0 * m * m * m * iters, k_gs_lex_cta<T>, dim3(1), dim3(1024), phi, rho, iters, H2, w);
        }
        else if (alt.p && m >= 64 && s->fused_rb)
        {
            // fused sweeps, ping-pong phi <-> alt (alt has phi's boundary values)
            // z-chunks: as many as keep the whole launch resident at once (one wave;
            // a CTA's march is a chain of dependent plane steps)
            const size_t shm = zm_smem_bytes<T>();
            int per_sm = 1, sms = 148;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gs_rb_zm<T>, ZM_THREADS, shm);
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
            const int txy = ((m + ZM_TX - 1) / ZM_TX) * ((m + ZM_TY - 1) / ZM_TY);
            const int nch = std::max(1, std::min(m, (std::max(per_sm, 1) * sms) / txy));
            const int tz = (m + nch - 1) / nch;
            dim3 grid((m + ZM_TX - 1) / ZM_TX, (m + ZM_TY - 1) / ZM_TY, (m + tz - 1) / tz);
            Grid<T> a = phi, b = alt;
            for (int it = 0; it < iters; it++)
            {
                launch_shm(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 3.0 * m * m * m, shm,
                           k_gs_rb_zm<T>, grid, dim3(ZM_THREADS), a, b, rho, H2, w, tz);
                Grid<T> t = a;
                a = b;
                b = t;
            }
            if (iters & 1)
            {
                int tx = m < 128 ? ((m + 31) / 32) * 32 : 128;
                launch(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 2.0 * m * m * m, k_copy_interior<T>,
                       dim3((m + tx - 1) / tx, m, m), dim3(tx), phi, alt);
            }
        }
        else
        {
            int half = (m + 1) / 2;
            int tx = half < 128 ? ((half + 31) / 32) * 32 : 128;
            dim3 grid((half + tx - 1) / tx, m, m);
            for (int it = 0; it < iters; it++)
                for (int color = 0; color < 2; color++)
                {
                    launch(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 1.5 * m * m * m, k_gs_rb<T>, dim3(grid), dim3(tx), phi, rho, color, H2, w);
                }
        }
    }
    else if (c.smoother == 1)
    {
        // jacobi.c:62-82: ping-pong through a copy; odd counts run one more sweep
        T C = (T)(-(1.0 / (n - 1)) * (1.0 / (n - 1)));
        T w = (T)c.w_sor;
        int tx = m < 128 ? ((m + 31) / 32) * 32 : 128;
        dim3 grid((m + tx - 1) / tx, m, m);
        dim3 gfull((n + tx - 1) / tx, n, n);
        launch(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 2.0 * n * n * n, k_copy_grid<T>, dim3(gfull), dim3(tx), scratch, phi);
        int sweeps = iters % 2 == 0 ? iters : iters + 1;
        Grid<T> a = iters % 2 == 0 ? phi : scratch;
        Grid<T> b = iters % 2 == 0 ? scratch : phi;
        for (int it = 0; it < sweeps; it++)
        {
            launch(s, QZ_PROF_SMOOTH, (double)sizeof(T) * 3.0 * m * m * m, k_jacobi<T>, dim3(grid), dim3(tx), a, b, rho, C, w);
            Grid<T> t = a;
            a = b;
            b = t;
        }
    }
    else if (c.smoother == 2)
    {
        if (!cgs_scratch.r || !s->cg_part)
        {
            set_error("conjugate-gradient smoothing buffers missing");
            return QZ_FAILURE;
        }
        CgsArgs<T> A;
        A.phi = phi;
        A.rho = rho;
        A.r = cgs_scratch.r;
        A.p = cgs_scratch.p;
        A.ap = cgs_scratch.ap;
        A.part = s->cg_part;
        A.iters = iters;
        A.bar = GridBar{s->gbar, s->flags};
        cudaMemsetAsync(s->gbar, 0, 4 * sizeof(unsigned), s->stream);
        static int per_sm[2] = {0, 0};
        static std::once_flag once;
        std::call_once(once, [] {
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_cg_smooth<double>, 256, 0);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_cg_smooth<float>, 256, 0);
        });
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
        const int ps = per_sm[sizeof(T) == 4 ? 1 : 0];
        const long want = ((long)m * m * m + 255) / 256;
        const int blocks = (int)std::max(1L, std::min(want, (long)std::min(ps, 2) * sms));
        if (ps < 1 || blocks > QZ_CG_PART_MAX)
        {
            set_error("conjugate-gradient smoothing kernel cannot be resident");
            return QZ_FAILURE;
        }
        void *args[] = {&A};
        cudaEvent_t eb = nullptr, ee = nullptr;
        if (s->prof)
        {
            eb = prof_event(s);
            ee = prof_event(s);
            cudaEventRecord(eb, s->stream);
        }
        if (!check_cuda(cudaLaunchCooperativeKernel((const void *)k_cg_smooth<T>, dim3(blocks),
                                                    dim3(256), args, 0, s->stream),
                        "conjugate-gradient smoothing"))
            return QZ_FAILURE;
        s->stats.kernel_launches++;
        if (s->prof)
        {
            cudaEventRecord(ee, s->stream);
            // the residual pass (24 B a point) and 88 B a point per iteration, FP64 units
            s->prof_pending.push_back({QZ_PROF_SMOOTH,
                                       (double)sizeof(T) * (24.0 + 88.0 * iters) * m * m * m / 8.0,
                                       eb, ee});
        }
    }
    else
    {
        set_error("smoother %d is not supported", c.smoother);
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

template <typename T>
struct LevelViews {
    static Grid<T> phi(qz_sim *s, int l);
    static Grid<T> rho(qz_sim *s, int l);
    static Grid<T> scratch(qz_sim *s, int l);
    static Grid<T> alt(qz_sim *s, int l);
    static CgsScratch<T> cgs(qz_sim *s, int l);
};

template <> CgsScratch<double> LevelViews<double>::cgs(qz_sim *s, int l)
{
    const Level &v = s->levels[l];
    return CgsScratch<double>{v.cgr, v.cgp, v.cga};
}
template <> CgsScratch<float> LevelViews<float>::cgs(qz_sim *s, int l)
{
    const Level &v = s->levels[l];
    return CgsScratch<float>{v.cgrf, v.cgpf, v.cgaf};
}

// Level 0 of the FP64 hierarchy is the fine grid view of the context (the head
// solve grid embedded in the head fields, or a dense array for the array-level
// entry points); level 0 of the FP32 hierarchy is the fine correction /
// residual pair ef / rf (dense n0^3).
template <>
Grid<double> LevelViews<double>::phi(qz_sim *s, int l)
{
    return l == 0 ? s->fine_phi : dense_view(s->levels[l].phi, s->levels[l].n);
}
template <>
Grid<double> LevelViews<double>::rho(qz_sim *s, int l)
{
    return l == 0 ? s->fine_rho : dense_view(s->levels[l].rho, s->levels[l].n);
}
template <>
Grid<double> LevelViews<double>::scratch(qz_sim *s, int l)
{
    return dense_view(s->levels[l].scr, s->levels[l].n);
}
template <>
Grid<double> LevelViews<double>::alt(qz_sim *s, int l)
{
    return l == 0 ? s->fine_alt : dense_view(s->levels[l].alt, s->levels[l].n);
}
template <>
Grid<float> LevelViews<float>::alt(qz_sim *s, int l)
{
    return dense_view(l == 0 ? s->ef_alt : s->levels[l].altf, s->levels[l].n);
}
template <>
Grid<float> LevelViews<float>::phi(qz_sim *s, int l)
{
    return l == 0 ? dense_view(s->ef, s->levels[0].n) : dense_view(s->levels[l].phif, s->levels[l].n);
}
template <>
Grid<float> LevelViews<float>::rho(qz_sim *s, int l)
{
    return l == 0 ? dense_view(s->rf, s->levels[0].n) : dense_view(s->levels[l].rhof, s->levels[l].n);
}
template <>
Grid<float> LevelViews<float>::scratch(qz_sim *s, int l)
{
    return dense_view(s->levels[l].scrf, s->levels[l].n);
}

template <typename T>
static int vcycle_t(qz_sim *s, int l, int type)
{
    const qz_config &c = s->cfg;
    Grid<T> phi = LevelViews<T>::phi(s, l), rho = LevelViews<T>::rho(s, l);
    const int n = phi.n;
    const int nc = (n + 1) / 2;
    Grid<T> scr{}, alt{};
    if (c.smoother == 1)
        scr = LevelViews<T>::scratch(s, l);
    if (c.smoother == 0 && c.gs_order == QZ_GS_REDBLACK)
        alt = LevelViews<T>::alt(s, l);
    const CgsScratch<T> cgw = LevelViews<T>::cgs(s, l);
    if (smooth_t<T>(s, phi, rho, c.n_pre, scr, alt, cgw))
        return QZ_FAILURE;
    if (nc < 4)
    {
        // multigrid.c:158-173: the coarse correction stays zero; the fine grid
        // gets n_coarse more smoothing sweeps instead.
        if (smooth_t<T>(s, phi, rho, c.n_coarse, scr, alt, cgw))
            return QZ_FAILURE;
    }
    else
    {
        if (l + 1 >= (int)s->levels.size())
        {
            set_error("multigrid hierarchy too shallow");
            return QZ_FAILURE;
        }
        Grid<T> cphi = LevelViews<T>::phi(s, l + 1), crho = LevelViews<T>::rho(s, l + 1);
        size_t cbytes = (size_t)nc * nc * nc * sizeof(T);
        cudaMemsetAsync(cphi.p, 0, cbytes, s->stream);
        int mc = nc - 2;
        int tx = mc < 128 ? ((mc + 31) / 32) * 32 : 128;
        dim3 g((mc + tx - 1) / tx, mc, mc);
        T ooh2 = (T)(double)((n - 1) * (n - 1));
        const T scale = (c.smoother == 0 && c.gs_order == QZ_GS_REDBLACK) ? (T)0.5 : (T)1.0;
        launch(s, QZ_PROF_RESTRICT, (double)sizeof(T) * 9.0 * mc * mc * mc, k_resid_restrict<T>, dim3(g), dim3(tx), phi, rho, crho, ooh2, scale);
        if (type == 0)
        {
            if (vcycle_t<T>(s, l + 1, 0))
                return QZ_FAILURE;
        }
        else if (type == 1)
        {
            if (vcycle_t<T>(s, l + 1, 1) || vcycle_t<T>(s, l + 1, 0))
                return QZ_FAILURE;
        }
        else
        {
            if (vcycle_t<T>(s, l + 1, 2) || vcycle_t<T>(s, l + 1, 2))
                return QZ_FAILURE;
        }
        int m = n - 2;
        int tf = m < 128 ? ((m + 31) / 32) * 32 : 128;
        dim3 gf((m + tf - 1) / tf, m, m);
        launch(s, QZ_PROF_PROLONG, (double)sizeof(T) * 2.125 * m * m * m, k_prolong_add<T>, dim3(gf), dim3(tf), phi, cphi);
    }
    if (smooth_t<T>(s, phi, rho, c.n_post, scr, alt, cgw))
        return QZ_FAILURE;
    return check_cuda(cudaGetLastError(), "multigrid cycle") ? QZ_SUCCESS : QZ_FAILURE;
}

int vcycle(qz_sim *s, int level, int type) { return vcycle_t<double>(s, level, type); }

// ---- persistent V-cycles ----------------------------------------------------------
// The red-black V-cycle (multigrid.c:106-229 with the smoother, restriction and
// prolongation above) as one cooperative launch that runs several cycles.  A
// cycle is a fixed sequence of dependent phases on grids that fit in L2, so one
// launch per phase costs more than the work; here the levels larger than
// MG_SMALL_N points a side run their phases on the whole grid separated by grid
// barriers, and the smaller levels run inside block 0 with block barriers while
// the other blocks wait at the next grid barrier.  Every point update uses the
// arithmetic of the kernels above, and the order of updates within a phase does
// not matter (one colour of a red-black sweep, restriction and prolongation read
// only what earlier phases wrote), so the result equals the launch-per-phase
// path bit for bit.  In the mixed-precision form a launch also holds the FP64
// fine residual and the FP64 correction of each iteration.

constexpr int MG_MAXLEV = 12;
constexpr int MG_SMALL_N = 17;
constexpr int MG_THREADS = 512;
static_assert(MG_THREADS == 512, "the single-block sub-cycle maps its threads to an 8 x 8 x 8 cube");
constexpr size_t MG_SMEM_MAX = 100 * 1024; // two resident blocks a SM
constexpr int MG_CLUSTER_MAX = 16;          // largest (non-portable) thread-block cluster

template <typename T> struct MgArgs {
    Grid<T> phi[MG_MAXLEV], rho[MG_MAXLEV];
    int nlev;   // levels; the last one is smoothed instead of corrected
    int nsmall; // first level of at most MG_SMALL_N points a side
    int n_pre, n_post, n_coarse;
    T w, scale;
    T h2[MG_MAXLEV]; // (1 / (n - 1))^2 of each level, as k_gs_rb's caller computes it
    int iters; // cycles (mixed: defect-correction iterations) in this launch
    int mixed;
    Grid<double> fphi, frho; // FP64 fine grid (mixed form): phi[0] / rho[0] are ef / rf
    int smem;                // the small levels live in block 0's shared memory
    int soff[MG_MAXLEV];     // their offsets there (phi, then rho), in elements
    GridBar bar;
    // mixed form with the convergence test inside the launch (poisson_error.c:
    // 36-133 on the fine interior, evaluated before each iteration's cycle from
    // the second on; pot_old holds the previous iterate)
    int check;
    double *pold;           // FP64 pot_old, the layout of fphi's array
    double *part;           // per block: residual partial [b], flags [QZ_CG_PART_MAX + b]
    int *outst;             // [0] iterations run, [1] converged
    double tm, tp, rm, tol; // 1 -/+ tol2, 4 pi G rho_mean, tol
    int method;
    long nintr;
    int every; // FP64 form: the test after every `every` cycles (the reference's cadence)
    // coarse levels 1 .. nsmall-1 in tiled phases (mg_tile_down / mg_tile_up):
    // bit l of tiled set for a tiled level, tile cores of tc[0] x tc[1] x tc[2] points
    int tiled;
    int tc[3];
    Grid<T> mid[MG_MAXLEV]; // partner arrays of the tiled levels (zero boundary)
    // the launch is one thread-block cluster (at most MG_CLUSTER_MAX blocks):
    // its grid-wide barrier is the hardware cluster barrier
    int cluster;
};

// Work item t = a + n0 (b + n1 c) of a grid-stride loop (t = tid, tid + stride,
// ...): the coordinates are advanced by the stride's own decomposition with
// carries, so the loop divides only when it starts.  Requires stride > 0; the
// loop ends when c reaches the third extent.
struct Walk3 {
    unsigned a, b, c, da, db, dc, n0, n1;
    __device__ __forceinline__ Walk3(unsigned t, unsigned stride, unsigned n0_, unsigned n1_)
        : n0(n0_), n1(n1_)
    {
        a = t % n0;
        unsigned r = t / n0;
        b = r % n1;
        c = r / n1;
        da = stride % n0;
        r = stride / n0;
        db = r % n1;
        dc = r / n1;
    }
    __device__ __forceinline__ void next()
    {
        a += da;
        const unsigned ca = a >= n0 ? 1u : 0u;
        a -= ca ? n0 : 0u;
        b += db + ca;
        const unsigned cb = b >= n1 ? 1u : 0u;
        b -= cb ? n1 : 0u;
        c += dc + cb;
    }
};

// The red-black update of point (i, j, k) (k_gs_rb's arithmetic).  G: Grid<T>
// (64-bit strides) or DGrid<T> (a dense grid of the single-block sub-cycle in
// shared memory, 32-bit index arithmetic).
template <typename T, typename G>
__device__ __forceinline__ void mg_rb_point(const G &phi, const G &rho, int i, int j, int k, T H2,
                                            T w)
{
    const T one_sixth = (T)(1.0 / 6.0);
    const auto gp = phi.off + i + j * phi.sy + k * phi.sz;
    const auto gr = rho.off + i + j * rho.sy + k * rho.sz;
    T *p = phi.p;
    T a = one_sixth * (-H2 * rho.p[gr] + p[gp + 1] + p[gp - 1] + p[gp + phi.sy] +
                       p[gp - phi.sy] + p[gp + phi.sz] + p[gp - phi.sz]);
    p[gp] = w * a + ((T)1.0 - w) * p[gp];
}

// One colour of a red-black sweep over work items t = tid, tid + nthr, ...
template <typename T>
__device__ __forceinline__ void mg_rb_half(const Grid<T> &phi, const Grid<T> &rho, int color,
                                           T H2, T w, unsigned tid, unsigned nthr)
{
    const int m = phi.n - 2;
    const unsigned half = (unsigned)(m + 1) / 2;
#pragma unroll 4
    for (Walk3 x(tid, nthr, half, (unsigned)m); x.c < (unsigned)m; x.next())
    {
        const int j = 1 + (int)x.b, k = 1 + (int)x.c;
        const int i = ((((1 + j + k) & 1) == color) ? 1 : 2) + 2 * (int)x.a;
        if (i > m)
            continue;
        mg_rb_point(phi, rho, i, j, k, H2, w);
    }
}

// Block-level loops over the small grids of the single-block sub-cycle: the
// block's MG_THREADS = 512 threads form an 8 x 8 x 8 cube and step through a
// grid by 8 along each axis, with no index division.
struct MgCube {
    int x, y, z;
};
__device__ __forceinline__ MgCube mg_cube()
{
    const int t = (int)threadIdx.x;
    return MgCube{t & 7, (t >> 3) & 7, t >> 6};
}

template <typename T, typename G>
__device__ __forceinline__ void mg_rb_half_blk(const G &phi, const G &rho, int color, T H2, T w)
{
    const int m = phi.n - 2, half = (m + 1) / 2;
    const MgCube q = mg_cube();
    for (int k = 1 + q.z; k <= m; k += 8)
        for (int j = 1 + q.y; j <= m; j += 8)
        {
            const int i0 = (((1 + j + k) & 1) == color) ? 1 : 2;
            for (int ti = q.x; ti < half; ti += 8)
            {
                const int i = i0 + 2 * ti;
                if (i <= m)
                    mg_rb_point(phi, rho, i, j, k, H2, w);
            }
        }
}

// rho_c at coarse point (lx, ly, lz) = scale * the residual at the injected fine point.
template <typename T, typename G>
__device__ __forceinline__ void mg_restrict_point(const G &phi, const G &rho, const G &crho, T ooh2,
                                                  T scale, int lx, int ly, int lz)
{
    const auto gp = phi.off + 2 * lx + 2 * ly * phi.sy + 2 * lz * phi.sz;
    const auto gr = rho.off + 2 * lx + 2 * ly * rho.sy + 2 * lz * rho.sz;
    const T *p = phi.p;
    T rv = rho.p[gr] + ooh2 * ((T)6 * p[gp] - p[gp + 1] - p[gp - 1] - p[gp + phi.sy] -
                               p[gp - phi.sy] - p[gp + phi.sz] - p[gp - phi.sz]);
    crho.p[crho.off + lx + ly * crho.sy + lz * crho.sz] = scale * rv;
}

// rho_c = scale * residual at the injected points; phi_c = 0 everywhere.
template <typename T>
__device__ __forceinline__ void mg_restrict(const Grid<T> &phi, const Grid<T> &rho,
                                            const Grid<T> &cphi, const Grid<T> &crho, T ooh2,
                                            T scale, unsigned tid, unsigned nthr)
{
    const unsigned nc = (unsigned)cphi.n;
    for (Walk3 x(tid, nthr, nc, nc); x.c < nc; x.next())
        cphi.p[cphi.off + (long)x.a + (long)x.b * cphi.sy + (long)x.c * cphi.sz] = (T)0;
    const unsigned mc = nc - 2;
    for (Walk3 x(tid, nthr, mc, mc); x.c < mc; x.next())
        mg_restrict_point(phi, rho, crho, ooh2, scale, 1 + (int)x.a, 1 + (int)x.b, 1 + (int)x.c);
}

template <typename T, typename G>
__device__ __forceinline__ void mg_restrict_blk(const G &phi, const G &rho, const G &cphi,
                                                const G &crho, T ooh2, T scale)
{
    const int nc = cphi.n, mc = nc - 2;
    const MgCube q = mg_cube();
    for (int k = q.z; k < nc; k += 8)
        for (int j = q.y; j < nc; j += 8)
            for (int i = q.x; i < nc; i += 8)
                cphi.p[cphi.off + i + j * cphi.sy + k * cphi.sz] = (T)0;
    for (int k = 1 + q.z; k <= mc; k += 8)
        for (int j = 1 + q.y; j <= mc; j += 8)
            for (int i = 1 + q.x; i <= mc; i += 8)
                mg_restrict_point(phi, rho, crho, ooh2, scale, i, j, k);
}

// phi += the trilinear interpolation of the coarse correction c (k_prolong_add's
// arithmetic).  A work item is the pair of fine points i = 2a+1 (odd) and
// i + 1 (even) of one row: both draw on the coarse columns a and a + 1 only, so
// their up to eight coarse values are loaded once, together.  Each point adds
// its terms in k_prolong_add's z, y, x order, skipping coarse points outside
// 1..mc; a point even in all three coordinates takes its coarse value as is.
template <typename T, typename G>
__device__ __forceinline__ void mg_prolong_pair(const G &phi, const G &c, int mc, int a, int j,
                                                int k)
{
    const int i0 = 2 * a + 1;
    const bool second = a < mc; // i0 + 1 <= m
    // y and z: coarse planes and their presence (odd: (j-1)/2 and (j+1)/2, even: j/2)
    const bool jo = j & 1, ko = k & 1;
    const int oy0 = jo ? (j - 1) >> 1 : j >> 1, oz0 = ko ? (k - 1) >> 1 : k >> 1;
    bool vy[2], vz[2];
    vy[0] = jo ? oy0 >= 1 : true;
    vy[1] = jo && oy0 + 1 <= mc;
    vz[0] = ko ? oz0 >= 1 : true;
    vz[1] = ko && oz0 + 1 <= mc;
    const bool vx0 = a >= 1, vx1 = a + 1 <= mc;
    const T wy = jo ? (T)0.5 : (T)1, wz = ko ? (T)0.5 : (T)1;
    const auto cb = c.off + a + oy0 * c.sy + oz0 * c.sz;
    T v[8]; // [z][y][x] with x = column a, a + 1
#pragma unroll
    for (int q = 0; q < 8; q++)
    {
        const int az = q >> 2, ay = (q >> 1) & 1, ax = q & 1;
        const bool ok = vz[az] && vy[ay] && (ax ? vx1 : vx0);
        v[q] = ok ? c.p[cb + ax + ay * c.sy + az * c.sz] : (T)0;
    }
    const auto f0 = phi.off + i0 + j * phi.sy + k * phi.sz;
    const T p0 = phi.p[f0];
    const T p1 = second ? phi.p[f0 + 1] : (T)0;
    // odd point i0: x weight 1/2 on both columns
    const T w0 = (T)0.5 * wy * wz;
    T acc0 = (T)0;
#pragma unroll
    for (int q = 0; q < 8; q++)
    {
        const int az = q >> 2, ay = (q >> 1) & 1, ax = q & 1;
        if (vz[az] && vy[ay] && (ax ? vx1 : vx0))
            acc0 += w0 * v[q];
    }
    phi.p[f0] = p0 + acc0;
    if (second)
    {
        // even point i0 + 1: column a + 1 at x weight 1
        T acc1;
        if (!jo && !ko)
            acc1 = v[1];
        else
        {
            const T w1 = (T)1 * wy * wz;
            acc1 = (T)0;
#pragma unroll
            for (int q = 0; q < 4; q++)
            {
                const int az = q >> 1, ay = q & 1;
                if (vz[az] && vy[ay])
                    acc1 += w1 * v[2 * q + 1];
            }
        }
        phi.p[f0 + 1] = p1 + acc1;
    }
}

template <typename T>
__device__ __forceinline__ void mg_prolong(const Grid<T> &phi, const Grid<T> &c, unsigned tid,
                                           unsigned nthr)
{
    const int m = phi.n - 2, mc = c.n - 2;
    const unsigned um = (unsigned)m, pairs = (unsigned)mc + 1; // m = 2 mc + 1
    for (Walk3 x(tid, nthr, pairs, um); x.c < um; x.next())
        mg_prolong_pair<T>(phi, c, mc, (int)x.a, 1 + (int)x.b, 1 + (int)x.c);
}

template <typename T, typename G>
__device__ __forceinline__ void mg_prolong_blk(const G &phi, const G &c)
{
    const int m = phi.n - 2, mc = c.n - 2;
    const MgCube q = mg_cube();
    for (int k = 1 + q.z; k <= m; k += 8)
        for (int j = 1 + q.y; j <= m; j += 8)
            for (int a = q.x; a <= mc; a += 8)
                mg_prolong_pair<T>(phi, c, mc, a, j, k);
}

// Smoothing sweeps of level l over the whole grid of threads; sync() separates
// the colours.
template <typename T, typename Sync>
__device__ __forceinline__ void mg_smooth(const MgArgs<T> &A, int l, int sweeps, unsigned tid,
                                          unsigned nthr, Sync sync)
{
    for (int it = 0; it < sweeps; it++)
        for (int color = 0; color < 2; color++)
        {
            mg_rb_half(A.phi[l], A.rho[l], color, A.h2[l], A.w, tid, nthr);
            sync();
        }
}

// The same inside one block (grids of the single-block sub-cycle).
template <typename T, typename G>
__device__ __forceinline__ void mg_smooth_blk(const G &phi, const G &rho, T H2, T w, int sweeps)
{
    for (int it = 0; it < sweeps; it++)
        for (int color = 0; color < 2; color++)
        {
            mg_rb_half_blk(phi, rho, color, H2, w);
            __syncthreads();
        }
}

// A dense n^3 grid in shared memory (the single-block sub-cycle): 32-bit strides.
template <typename T> struct DGrid {
    T *p;
    static constexpr int off = 0;
    int sy, sz, n;
};

template <typename T> __device__ __forceinline__ DGrid<T> mg_dense(T *p, int n)
{
    DGrid<T> g;
    g.p = p;
    g.sy = n;
    g.sz = n * n;
    g.n = n;
    return g;
}

// Block-wide copies between a level's grid and its shared-memory copy.  A
// dense level (offset 0, strides n and n^2: every level below the finest) moves
// as a flat array, by asynchronous copies in, all in flight at once.
template <typename T> __device__ __forceinline__ bool mg_is_dense(const Grid<T> &a)
{
    return a.off == 0 && a.sy == a.n && a.sz == (long)a.n * a.n;
}

template <typename T>
__device__ __forceinline__ void mg_copy_in(const Grid<T> &a, const DGrid<T> &b, unsigned tid,
                                           unsigned nthr)
{
    const unsigned n = (unsigned)a.n, n3 = n * n * n;
    if (mg_is_dense(a))
    {
        for (unsigned t = tid; t < n3; t += nthr)
            __pipeline_memcpy_async(&b.p[t], &a.p[t], sizeof(T));
        __pipeline_commit();
        __pipeline_wait_prior(0);
        return;
    }
    for (Walk3 x(tid, nthr, n, n); x.c < n; x.next())
        b.p[x.a + x.b * b.sy + x.c * b.sz] =
            a.p[a.off + (long)x.a + (long)x.b * a.sy + (long)x.c * a.sz];
}

template <typename T>
__device__ __forceinline__ void mg_copy_out(const DGrid<T> &a, const Grid<T> &b, unsigned tid,
                                            unsigned nthr)
{
    const unsigned n = (unsigned)a.n;
    if (mg_is_dense(b))
    {
        const unsigned n3 = n * n * n;
#pragma unroll 4
        for (unsigned t = tid; t < n3; t += nthr)
            b.p[t] = a.p[t];
        return;
    }
    for (Walk3 x(tid, nthr, n, n); x.c < n; x.next())
        b.p[b.off + (long)x.a + (long)x.b * b.sy + (long)x.c * b.sz] =
            a.p[x.a + x.b * a.sy + x.c * a.sz];
}

// The levels of the single-block sub-cycle (P(l), R(l): a level's phi and rho,
// in shared or global memory).
template <typename T, typename PF, typename RF>
__device__ __forceinline__ void mg_subcycle_levels(const MgArgs<T> &A, PF P, RF R)
{
    for (int l = A.nsmall; l < A.nlev; l++)
    {
        mg_smooth_blk(P(l), R(l), A.h2[l], A.w, A.n_pre);
        if (l == A.nlev - 1)
            mg_smooth_blk(P(l), R(l), A.h2[l], A.w, A.n_coarse);
        else
        {
            const int n = A.phi[l].n;
            mg_restrict_blk(P(l), R(l), P(l + 1), R(l + 1), (T)(double)((n - 1) * (n - 1)), A.scale);
            __syncthreads();
        }
    }
    for (int l = A.nlev - 1; l >= A.nsmall; l--)
    {
        if (l < A.nlev - 1)
        {
            mg_prolong_blk<T>(P(l), P(l + 1));
            __syncthreads();
        }
        mg_smooth_blk(P(l), R(l), A.h2[l], A.w, A.n_post);
    }
}

// ---- coarse levels in tiled phases ------------------------------------------------------
// A coarse level's pre-smoothing and restriction (2 n_pre + 1 grid phases)
// become one phase, and its prolongation and post-smoothing (2 n_post + 1)
// another.  Every block takes tiles of the level's interior: it sets up a tile's
// core with a halo deep enough for all the colour phases in shared memory,
// runs the colour phases on regions that shrink by one point a phase, and
// writes back the core.  A halo point is computed by every tile that holds it,
// from the same values with the same arithmetic, so it equals the owner's; the
// pre-smoothing halo is 2 n_pre + 1 (the residual at a restriction point needs
// its smoothed neighbours), the post-smoothing halo 2 n_post.  A tile must not
// read what another tile of the same phase writes, so the down phase starts
// from zero (the restriction into a coarse level zeroes it) and writes its
// cores to the level's partner array (mid), and the up phase reads mid and
// writes the level's correction.  Point updates, restriction and prolongation
// keep the arithmetic of mg_rb_point, mg_restrict_point and mg_prolong_pair,
// so the fields equal those of the grid-phase path bit for bit.

// Region [x0, x1) x [y0, y1) x [z0, z1) of a level.
struct MgBox {
    int x0, x1, y0, y1, z0, z1;
};

// The core [c0, c1) of each axis widened by h, clipped to [lo, hi).
__device__ __forceinline__ MgBox mg_box(const int c0[3], const int c1[3], int h, int lo, int hi)
{
    MgBox b;
    b.x0 = max(c0[0] - h, lo);
    b.x1 = min(c1[0] + h, hi);
    b.y0 = max(c0[1] - h, lo);
    b.y1 = min(c1[1] + h, hi);
    b.z0 = max(c0[2] - h, lo);
    b.z1 = min(c1[2] + h, hi);
    return b;
}

// A shared-memory copy of a box of a level: point (i, j, k) at
// (i - o[0]) + (j - o[1]) sx + (k - o[2]) sxy.
template <typename T> struct MgTile {
    T *s;
    int o[3];
    int sx, sxy;
    __device__ __forceinline__ int at(int i, int j, int k) const
    {
        return (i - o[0]) + (j - o[1]) * sx + (k - o[2]) * sxy;
    }
};

// Starts asynchronous copies of box b of a level into the tile (cp.async, one
// element each: every load of a tile is in flight at once); mg_tile_wait ends them.
template <typename T>
__device__ __forceinline__ void mg_tile_load(const Grid<T> &g, const MgBox &b, const MgTile<T> &t)
{
    const int nx = b.x1 - b.x0, ny = b.y1 - b.y0, nz = b.z1 - b.z0;
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return;
    for (Walk3 w(threadIdx.x, blockDim.x, (unsigned)nx, (unsigned)ny); w.c < (unsigned)nz; w.next())
    {
        const int i = b.x0 + (int)w.a, j = b.y0 + (int)w.b, k = b.z0 + (int)w.c;
        __pipeline_memcpy_async(&t.s[t.at(i, j, k)], &g.p[g.off + i + (long)j * g.sy + (long)k * g.sz],
                                sizeof(T));
    }
}

__device__ __forceinline__ void mg_tile_wait()
{
    __pipeline_commit();
    __pipeline_wait_prior(0);
    __syncthreads();
}

// Zero over box b of the tile.
template <typename T> __device__ __forceinline__ void mg_tile_zero(const MgBox &b, const MgTile<T> &t)
{
    const int nx = b.x1 - b.x0, ny = b.y1 - b.y0, nz = b.z1 - b.z0;
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return;
    for (Walk3 w(threadIdx.x, blockDim.x, (unsigned)nx, (unsigned)ny); w.c < (unsigned)nz; w.next())
        t.s[t.at(b.x0 + (int)w.a, b.y0 + (int)w.b, b.z0 + (int)w.c)] = (T)0;
}

template <typename T>
__device__ __forceinline__ void mg_tile_store(const Grid<T> &g, const MgBox &b, const MgTile<T> &t)
{
    const int nx = b.x1 - b.x0, ny = b.y1 - b.y0, nz = b.z1 - b.z0;
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return;
    for (Walk3 w(threadIdx.x, blockDim.x, (unsigned)nx, (unsigned)ny); w.c < (unsigned)nz; w.next())
    {
        const int i = b.x0 + (int)w.a, j = b.y0 + (int)w.b, k = b.z0 + (int)w.c;
        g.p[g.off + i + (long)j * g.sy + (long)k * g.sz] = t.s[t.at(i, j, k)];
    }
}

// One colour of a red-black sweep over the points of box u (mg_rb_point's
// arithmetic; colour (i + j + k) & 1 as in mg_rb_half).
template <typename T>
__device__ __forceinline__ void mg_tile_rb(const MgTile<T> &P, const MgTile<T> &R, const MgBox &u,
                                           int color, T H2, T w)
{
    const int nx = u.x1 - u.x0, ny = u.y1 - u.y0, nz = u.z1 - u.z0;
    if (nx <= 0 || ny <= 0 || nz <= 0)
        return;
    const T one_sixth = (T)(1.0 / 6.0);
    const unsigned hw = (unsigned)(nx + 1) / 2;
    T *p = P.s;
    for (Walk3 x(threadIdx.x, blockDim.x, hw, (unsigned)ny); x.c < (unsigned)nz; x.next())
    {
        const int j = u.y0 + (int)x.b, k = u.z0 + (int)x.c;
        const int i = ((((u.x0 + j + k) & 1) == color) ? u.x0 : u.x0 + 1) + 2 * (int)x.a;
        if (i >= u.x1)
            continue;
        const int q = P.at(i, j, k);
        const T a = one_sixth * (-H2 * R.s[R.at(i, j, k)] + p[q + 1] + p[q - 1] + p[q + P.sx] +
                                 p[q - P.sx] + p[q + P.sxy] + p[q - P.sxy]);
        p[q] = w * a + ((T)1.0 - w) * p[q];
    }
}

// The correction k_prolong_add (mg_prolong_pair) adds at fine point (i, j, k),
// from coarse values at(a, b, c): the odd point of a pair adds its up to eight
// terms in z, y, x order, the even point takes its column's value as is (j, k
// even) or adds its up to four terms in z, y order.
template <typename T, typename CF>
__device__ __forceinline__ T mg_prolong_value(CF cv, int mc, int i, int j, int k)
{
    const bool jo = j & 1, ko = k & 1;
    const int oy0 = jo ? (j - 1) >> 1 : j >> 1, oz0 = ko ? (k - 1) >> 1 : k >> 1;
    bool vy[2], vz[2];
    vy[0] = jo ? oy0 >= 1 : true;
    vy[1] = jo && oy0 + 1 <= mc;
    vz[0] = ko ? oz0 >= 1 : true;
    vz[1] = ko && oz0 + 1 <= mc;
    const T wy = jo ? (T)0.5 : (T)1, wz = ko ? (T)0.5 : (T)1;
    if (i & 1)
    {
        const int a = (i - 1) >> 1;
        const bool vx0 = a >= 1, vx1 = a + 1 <= mc;
        const T w0 = (T)0.5 * wy * wz;
        T acc = (T)0;
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
            const int az = q >> 2, ay = (q >> 1) & 1, ax = q & 1;
            if (vz[az] && vy[ay] && (ax ? vx1 : vx0))
                acc += w0 * cv(a + ax, oy0 + ay, oz0 + az);
        }
        return acc;
    }
    const int b = i >> 1;
    if (!jo && !ko)
        return cv(b, oy0, oz0);
    const T w1 = (T)1 * wy * wz;
    T acc = (T)0;
#pragma unroll
    for (int q = 0; q < 4; q++)
    {
        const int az = q >> 1, ay = q & 1;
        if (vz[az] && vy[ay])
            acc += w1 * cv(b, oy0 + ay, oz0 + az);
    }
    return acc;
}

// Tiles of a level's interior [1, m]^3 with cores of tc points per axis.
struct MgTiling {
    int nt[3];
    __device__ __forceinline__ MgTiling(int m, const int tc[3])
    {
        for (int d = 0; d < 3; d++)
            nt[d] = (m + tc[d] - 1) / tc[d];
    }
    __device__ __forceinline__ int count() const { return nt[0] * nt[1] * nt[2]; }
    __device__ __forceinline__ void core(int t, int m, const int tc[3], int c0[3], int c1[3]) const
    {
        const int tt[3] = {t % nt[0], (t / nt[0]) % nt[1], t / (nt[0] * nt[1])};
        for (int d = 0; d < 3; d++)
        {
            c0[d] = 1 + tt[d] * tc[d];
            c1[d] = min(c0[d] + tc[d], m + 1);
        }
    }
};

// Shared-memory elements of the two tiled phases (the host sizes the launch with it).
__host__ __device__ inline long mg_tile_elems(const int tc[3], int n_pre, int n_post)
{
    auto vol = [&](int h) { return (long)(tc[0] + 2 * h) * (tc[1] + 2 * h) * (tc[2] + 2 * h); };
    const int hd = 2 * n_pre + 1, hu = 2 * n_post;
    const long down = vol(hd) + vol(hd - 1);
    long coarse = 1;
    for (int d = 0; d < 3; d++)
        coarse *= (tc[d] + 2 * hu + 1) / 2 + 2;
    const long up = vol(hu) + vol(hu > 0 ? hu - 1 : 0) + coarse;
    return down > up ? down : up;
}

// Level l (zero at the start): n_pre sweeps into mid_l, the restriction into level
// l + 1 (phi_{l+1} = 0).
template <typename T>
__device__ __noinline__ void mg_tile_down(const MgArgs<T> &A, int l, T *sm, unsigned gtid, unsigned gn)
{
    const Grid<T> &R = A.rho[l], &CP = A.phi[l + 1], &CR = A.rho[l + 1];
    const int n = A.phi[l].n, m = n - 2, nc = CP.n, mc = nc - 2;
    const unsigned unc = (unsigned)nc;
    for (Walk3 x(gtid, gn, unc, unc); x.c < unc; x.next())
        CP.p[CP.off + (long)x.a + (long)x.b * CP.sy + (long)x.c * CP.sz] = (T)0;
    const int hd = 2 * A.n_pre + 1, hr = hd - 1;
    MgTile<T> tp, tr;
    tp.s = sm;
    tp.sx = A.tc[0] + 2 * hd;
    tp.sxy = tp.sx * (A.tc[1] + 2 * hd);
    tr.s = sm + (long)tp.sxy * (A.tc[2] + 2 * hd);
    tr.sx = A.tc[0] + 2 * hr;
    tr.sxy = tr.sx * (A.tc[1] + 2 * hr);
    const T H2 = A.h2[l], w = A.w, ooh2 = (T)(double)((n - 1) * (n - 1)), scale = A.scale;
    const MgTiling tl(m, A.tc);
    for (int t = blockIdx.x; t < tl.count(); t += gridDim.x)
    {
        int c0[3], c1[3];
        tl.core(t, m, A.tc, c0, c1);
        for (int d = 0; d < 3; d++)
        {
            tp.o[d] = c0[d] - hd;
            tr.o[d] = c0[d] - hr;
        }
        mg_tile_zero(mg_box(c0, c1, hd, 0, n), tp); // the level starts at zero
        mg_tile_load(R, mg_box(c0, c1, hr, 1, m + 1), tr);
        mg_tile_wait();
        for (int c = 0; c < 2 * A.n_pre; c++)
        {
            mg_tile_rb(tp, tr, mg_box(c0, c1, hd - 1 - c, 1, m + 1), c & 1, H2, w);
            __syncthreads();
        }
        // coarse points whose injected fine point 2X lies in the core
        MgBox cb;
        cb.x0 = max((c0[0] + 1) >> 1, 1);
        cb.x1 = min((c1[0] + 1) >> 1, mc + 1);
        cb.y0 = max((c0[1] + 1) >> 1, 1);
        cb.y1 = min((c1[1] + 1) >> 1, mc + 1);
        cb.z0 = max((c0[2] + 1) >> 1, 1);
        cb.z1 = min((c1[2] + 1) >> 1, mc + 1);
        const int nx = cb.x1 - cb.x0, ny = cb.y1 - cb.y0, nz = cb.z1 - cb.z0;
        if (nx > 0 && ny > 0 && nz > 0)
        {
            const T *p = tp.s;
            for (Walk3 x(threadIdx.x, blockDim.x, (unsigned)nx, (unsigned)ny); x.c < (unsigned)nz;
                 x.next())
            {
                const int lx = cb.x0 + (int)x.a, ly = cb.y0 + (int)x.b, lz = cb.z0 + (int)x.c;
                const int q = tp.at(2 * lx, 2 * ly, 2 * lz);
                const T rv = tr.s[tr.at(2 * lx, 2 * ly, 2 * lz)] +
                             ooh2 * ((T)6 * p[q] - p[q + 1] - p[q - 1] - p[q + tp.sx] - p[q - tp.sx] -
                                     p[q + tp.sxy] - p[q - tp.sxy]);
                CR.p[CR.off + lx + (long)ly * CR.sy + (long)lz * CR.sz] = scale * rv;
            }
        }
        mg_tile_store(A.mid[l], mg_box(c0, c1, 0, 1, m + 1), tp);
        __syncthreads(); // the next tile reloads the arrays
    }
}

// Level l: phi_l = mid_l + the prolonged correction of level l + 1, then n_post
// sweeps.
template <typename T> __device__ __noinline__ void mg_tile_up(const MgArgs<T> &A, int l, T *sm)
{
    const Grid<T> &P = A.phi[l], &R = A.rho[l], &C = A.phi[l + 1];
    const int n = P.n, m = n - 2, nc = C.n, mc = nc - 2;
    const int hu = 2 * A.n_post, hr = hu > 0 ? hu - 1 : 0;
    MgTile<T> tp, tr, tc;
    tp.s = sm;
    tp.sx = A.tc[0] + 2 * hu;
    tp.sxy = tp.sx * (A.tc[1] + 2 * hu);
    tr.s = sm + (long)tp.sxy * (A.tc[2] + 2 * hu);
    tr.sx = A.tc[0] + 2 * hr;
    tr.sxy = tr.sx * (A.tc[1] + 2 * hr);
    tc.s = tr.s + (long)tr.sxy * (A.tc[2] + 2 * hr);
    tc.sx = (A.tc[0] + 2 * hu + 1) / 2 + 2;
    tc.sxy = tc.sx * ((A.tc[1] + 2 * hu + 1) / 2 + 2);
    const T H2 = A.h2[l], w = A.w;
    const MgTiling tl(m, A.tc);
    for (int t = blockIdx.x; t < tl.count(); t += gridDim.x)
    {
        int c0[3], c1[3];
        tl.core(t, m, A.tc, c0, c1);
        for (int d = 0; d < 3; d++)
        {
            tp.o[d] = c0[d] - hu;
            tr.o[d] = c0[d] - hr;
        }
        const MgBox pb = mg_box(c0, c1, hu, 0, n), ib = mg_box(c0, c1, hu, 1, m + 1);
        // coarse columns of the interior points of the box: [(f0 - 1) >> 1, (f1 + 1) >> 1]
        MgBox cb;
        cb.x0 = (ib.x0 - 1) >> 1;
        cb.x1 = min(((ib.x1 - 1 + 1) >> 1) + 1, nc);
        cb.y0 = (ib.y0 - 1) >> 1;
        cb.y1 = min(((ib.y1 - 1 + 1) >> 1) + 1, nc);
        cb.z0 = (ib.z0 - 1) >> 1;
        cb.z1 = min(((ib.z1 - 1 + 1) >> 1) + 1, nc);
        tc.o[0] = cb.x0;
        tc.o[1] = cb.y0;
        tc.o[2] = cb.z0;
        mg_tile_load(A.mid[l], pb, tp);
        if (hu > 0)
            mg_tile_load(R, mg_box(c0, c1, hr, 1, m + 1), tr);
        mg_tile_load(C, cb, tc);
        mg_tile_wait();
        {
            const int nx = ib.x1 - ib.x0, ny = ib.y1 - ib.y0, nz = ib.z1 - ib.z0;
            const T *cs = tc.s;
            auto cv = [&](int a, int b, int c) -> T { return cs[tc.at(a, b, c)]; };
            if (nx > 0 && ny > 0 && nz > 0)
                for (Walk3 x(threadIdx.x, blockDim.x, (unsigned)nx, (unsigned)ny); x.c < (unsigned)nz;
                     x.next())
                {
                    const int i = ib.x0 + (int)x.a, j = ib.y0 + (int)x.b, k = ib.z0 + (int)x.c;
                    const int q = tp.at(i, j, k);
                    tp.s[q] = tp.s[q] + mg_prolong_value<T>(cv, mc, i, j, k);
                }
        }
        __syncthreads();
        for (int c = 0; c < hu; c++)
        {
            mg_tile_rb(tp, tr, mg_box(c0, c1, hu - 1 - c, 1, m + 1), c & 1, H2, w);
            __syncthreads();
        }
        mg_tile_store(P, mg_box(c0, c1, 0, 1, m + 1), tp);
        __syncthreads();
    }
}

// The FP64 form's convergence test inside the launch after `it` cycles
// (k_check_partial / k_check_final / k_copy_if_unconverged on the fine
// interior): per-block residual partials and ratio-test flags, one grid
// barrier, the decision taken by every block from the partials in the same
// order; unconverged: pot_old = pot on the interior (its boundary equals pot's
// for the whole solve).  True when converged (block 0 records it in outst).
template <typename Sync>
__device__ bool mg_check64(const MgArgs<double> &A, int it, unsigned gtid, unsigned gn, Sync gsync)
{
    const Grid<double> &P = A.phi[0], &R = A.rho[0];
    const int n = P.n, m = n - 2;
    const double ooh2 = (double)((n - 1) * (n - 1));
    const unsigned um = (unsigned)m;
    double acc = 0.0;
    int fl = 0; // 1 ratio test failed, 2 point residual test failed (method 1)
    for (Walk3 x(gtid, gn, um, um); x.c < um; x.next())
    {
        const int i = 1 + (int)x.a, j = 1 + (int)x.b, k = 1 + (int)x.c;
        const int gp = P.off + i + j * P.sy + k * P.sz;
        const double *p = P.p;
        const double r = R.p[R.off + i + j * R.sy + k * R.sz] +
                         ooh2 * (6.0 * p[gp] - p[gp + 1] - p[gp - 1] - p[gp + P.sy] - p[gp - P.sy] -
                                 p[gp + P.sz] - p[gp - P.sz]);
        const double a = p[gp] / A.pold[gp];
        if ((A.tm > a) || (A.tp < a))
            fl |= 1;
        if (A.method == 1)
        {
            if (fabs(r) / A.rm >= A.tol)
                fl |= 2;
        }
        else
            acc += r * r;
    }
    for (int o = 16; o > 0; o >>= 1)
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
    fl = (int)__reduce_or_sync(0xffffffffu, (unsigned)fl);
    __shared__ double wacc[MG_THREADS / 32];
    __shared__ int wfl[MG_THREADS / 32];
    __shared__ int s_stop;
    if ((threadIdx.x & 31) == 0)
    {
        wacc[threadIdx.x >> 5] = acc;
        wfl[threadIdx.x >> 5] = fl;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0.0;
        int f = 0;
        for (int w = 0; w < MG_THREADS / 32; w++)
        {
            t += wacc[w];
            f |= wfl[w];
        }
        A.part[blockIdx.x] = t;
        A.part[QZ_CG_PART_MAX + blockIdx.x] = (double)f;
    }
    gsync();
    if (threadIdx.x < 32)
    {
        double t = 0.0;
        int f = 0;
        for (int b = threadIdx.x; b < (int)gridDim.x; b += 32)
        {
            t += __ldcg(A.part + b);
            f |= (int)__ldcg(A.part + QZ_CG_PART_MAX + b);
        }
        for (int o = 16; o > 0; o >>= 1)
            t += __shfl_xor_sync(0xffffffffu, t, o);
        f = (int)__reduce_or_sync(0xffffffffu, (unsigned)f);
        if (threadIdx.x == 0)
        {
            int ok;
            if (A.method == 1)
                ok = !(f & 2);
            else
            {
                double err = t / A.nintr;
                err = sqrt(err);
                err = err / A.rm;
                if (A.method == 2)
                    err = err / (cbrt((double)A.nintr) * cbrt((double)A.nintr));
                ok = err < A.tol;
            }
            s_stop = !(f & 1) && ok;
            if (s_stop && blockIdx.x == 0)
            {
                A.outst[0] = it;
                A.outst[1] = 1;
            }
        }
    }
    __syncthreads();
    if (s_stop)
        return true;
    for (Walk3 x(gtid, gn, um, um); x.c < um; x.next())
    {
        const int gp = P.off + 1 + (int)x.a + (1 + (int)x.b) * P.sy + (1 + (int)x.c) * P.sz;
        A.pold[gp] = P.p[gp];
    }
    // the partials are rewritten only after the next cycle's barriers
    return false;
}

template <typename T>
__global__ void __launch_bounds__(MG_THREADS, 2) k_mg_cycles(const __grid_constant__ MgArgs<T> A)
{
    extern __shared__ __align__(16) unsigned char mg_dyn[];
    __shared__ int sh_ok;
    const unsigned gtid = blockIdx.x * blockDim.x + threadIdx.x, gn = gridDim.x * blockDim.x;
    // every block reaches the same barriers in the same order (all decisions
    // come from values every block computes alike), so the cluster barrier,
    // which has no time limit, is met as surely as the bounded grid barrier
    auto gsync = [&]() {
        if (A.cluster)
            cooperative_groups::this_cluster().sync();
        else
            gbar_sync(A.bar, &sh_ok);
    };
    for (int it = 0; it < A.iters; it++)
    {
        if constexpr (std::is_same<T, double>::value)
            if (A.check && it > 0 && it % A.every == 0 && mg_check64(A, it, gtid, gn, gsync))
                return;
        if (A.mixed)
        {
            // rf = (float)(rho + ooh2 (6 phi - sum)) on the fine interior (FP64), ef = 0
            const Grid<double> &P = A.fphi, &R = A.frho;
            const int n = P.n, m = n - 2;
            const double ooh2 = (double)((n - 1) * (n - 1));
            const unsigned um = (unsigned)m, n3 = (unsigned)n * n * n;
            float *rf = (float *)A.rho[0].p, *ef = (float *)A.phi[0].p;
            for (unsigned t = gtid; t < n3; t += gn)
                ef[t] = 0.0f;
            double acc = 0.0;
            int fl = 0; // 1 ratio test failed, 2 point residual test failed (method 1)
            for (Walk3 x(gtid, gn, um, um); x.c < um; x.next())
            {
                const int i = 1 + (int)x.a, j = 1 + (int)x.b, k = 1 + (int)x.c;
                const long gp = P.off + i + j * P.sy + k * P.sz;
                const long gr = R.off + i + j * R.sy + k * R.sz;
                const double *p = P.p;
                const double r = R.p[gr] + ooh2 * (6.0 * p[gp] - p[gp + 1] - p[gp - 1] - p[gp + P.sy] -
                                                   p[gp - P.sy] - p[gp + P.sz] - p[gp - P.sz]);
                rf[i + (long)j * n + (long)k * n * n] = (float)r;
                if (A.check)
                {
                    // k_check_partial's tests on the same points, then pot_old = phi
                    const double pv = p[gp];
                    const double a = pv / A.pold[gp];
                    if ((A.tm > a) || (A.tp < a))
                        fl |= 1;
                    A.pold[gp] = pv;
                    if (A.method == 1)
                    {
                        if (fabs(r) / A.rm >= A.tol)
                            fl |= 2;
                    }
                    else
                        acc += r * r;
                }
            }
            if (A.check)
            {
                for (int o = 16; o > 0; o >>= 1)
                    acc += __shfl_xor_sync(0xffffffffu, acc, o);
                fl = (int)__reduce_or_sync(0xffffffffu, (unsigned)fl);
                __shared__ double wacc[MG_THREADS / 32];
                __shared__ int wfl[MG_THREADS / 32];
                if ((threadIdx.x & 31) == 0)
                {
                    wacc[threadIdx.x >> 5] = acc;
                    wfl[threadIdx.x >> 5] = fl;
                }
                __syncthreads();
                if (threadIdx.x == 0)
                {
                    double t = 0.0;
                    int f = 0;
                    for (int w = 0; w < MG_THREADS / 32; w++)
                    {
                        t += wacc[w];
                        f |= wfl[w];
                    }
                    A.part[blockIdx.x] = t;
                    A.part[QZ_CG_PART_MAX + blockIdx.x] = (double)f;
                }
            }
            gsync();
            if (A.check)
            {
                // every block adds the partials in the same order: the same decision
                __shared__ int s_stop;
                if (threadIdx.x < 32)
                {
                    double t = 0.0;
                    int f = 0;
                    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32)
                    {
                        t += __ldcg(A.part + b);
                        f |= (int)__ldcg(A.part + QZ_CG_PART_MAX + b);
                    }
                    for (int o = 16; o > 0; o >>= 1)
                        t += __shfl_xor_sync(0xffffffffu, t, o);
                    f = (int)__reduce_or_sync(0xffffffffu, (unsigned)f);
                    if (threadIdx.x == 0)
                    {
                        int ok;
                        if (A.method == 1)
                            ok = !(f & 2);
                        else
                        {
                            double err = t / A.nintr;
                            err = sqrt(err);
                            err = err / A.rm;
                            if (A.method == 2)
                                err = err / (cbrt((double)A.nintr) * cbrt((double)A.nintr));
                            ok = err < A.tol;
                        }
                        s_stop = it > 0 && !(f & 1) && ok;
                        if (s_stop && blockIdx.x == 0)
                        {
                            A.outst[0] = it;
                            A.outst[1] = 1;
                        }
                    }
                }
                __syncthreads();
                if (s_stop)
                    return;
                // the partials are rewritten only after the next iteration's barriers
            }
        }
        // levels above the small ones: grid-wide phases (coarse ones tiled)
        for (int l = 0; l < A.nsmall; l++)
        {
            if ((A.tiled >> l) & 1)
            {
                mg_tile_down(A, l, reinterpret_cast<T *>(mg_dyn), gtid, gn);
                gsync();
                continue;
            }
            mg_smooth(A, l, A.n_pre, gtid, gn, gsync);
            const int n = A.phi[l].n;
            mg_restrict(A.phi[l], A.rho[l], A.phi[l + 1], A.rho[l + 1], (T)(double)((n - 1) * (n - 1)),
                        A.scale, gtid, gn);
            gsync();
        }
        // the small levels: a whole sub-cycle inside block 0, in its shared memory
        // when they fit (the first small level is copied in and its correction out)
        if (blockIdx.x == 0)
        {
            const unsigned bt = threadIdx.x, bn = blockDim.x;
            if (A.smem)
            {
                T *sm = reinterpret_cast<T *>(mg_dyn);
                auto P = [&](int l) { return mg_dense(sm + A.soff[l], A.phi[l].n); };
                auto R = [&](int l) {
                    const int n = A.phi[l].n;
                    return mg_dense(sm + A.soff[l] + n * n * n, n);
                };
                // a coarse level's correction starts at zero (the restriction into
                // it zeroed it): only its rho is copied in
                const int ns = A.nsmall, n = A.phi[ns].n;
                if (ns > 0)
                {
                    const DGrid<T> p0 = P(ns);
                    for (int t = bt; t < n * n * n; t += bn)
                        p0.p[t] = (T)0;
                }
                else
                    mg_copy_in(A.phi[ns], P(ns), bt, bn);
                mg_copy_in(A.rho[ns], R(ns), bt, bn);
                __syncthreads();
                mg_subcycle_levels(A, P, R);
                mg_copy_out(P(ns), A.phi[ns], bt, bn);
            }
            else
                mg_subcycle_levels(A, [&](int l) { return A.phi[l]; },
                                   [&](int l) { return A.rho[l]; });
        }
        gsync();
        for (int l = A.nsmall - 1; l >= 0; l--)
        {
            if ((A.tiled >> l) & 1)
            {
                mg_tile_up(A, l, reinterpret_cast<T *>(mg_dyn));
                gsync();
                continue;
            }
            mg_prolong(A.phi[l], A.phi[l + 1], gtid, gn);
            gsync();
            mg_smooth(A, l, A.n_post, gtid, gn, gsync);
        }
        if (A.mixed)
        {
            const Grid<double> &P = A.fphi;
            const int n = P.n, m = n - 2;
            const unsigned um = (unsigned)m;
            const float *ef = (const float *)A.phi[0].p;
            for (Walk3 x(gtid, gn, um, um); x.c < um; x.next())
            {
                const int i = 1 + (int)x.a, j = 1 + (int)x.b, k = 1 + (int)x.c;
                P.p[P.off + i + j * P.sy + k * P.sz] += (double)ef[i + (long)j * n + (long)k * n * n];
            }
            gsync();
        }
    }
    if constexpr (std::is_same<T, double>::value)
        if (A.check && A.iters > 0 && A.iters % A.every == 0 && mg_check64(A, A.iters, gtid, gn, gsync))
            return;
    if (A.check && gtid == 0)
    {
        A.outst[0] = A.iters;
        A.outst[1] = 0;
    }
}

// True when the head solve runs as persistent launches (red-black Gauss-Seidel
// V-cycles, no tiled sweeps); QZ_MG_LAUNCHES=1 selects one launch per phase.
bool mg_persistent(const qz_sim *s)
{
    static const bool off = getenv("QZ_MG_LAUNCHES") != nullptr;
    const qz_config &c = s->cfg;
    return !off && c.smoother == 0 && c.gs_order == QZ_GS_REDBLACK && c.cycle == 0 &&
           !s->fused_rb && (int)s->levels.size() <= MG_MAXLEV;
}

// Whether one cluster of lc's shape (blocks, threads, shared memory) can be
// resident on the device: cudaOccupancyMaxActiveClusters once per shape (the
// first query also allows cluster sizes above the portable 8).
template <typename T> static bool mg_cluster_fits(const cudaLaunchConfig_t &lc)
{
    static std::mutex mu;
    static std::vector<std::pair<long, bool>> known; // (blocks << 32 | smem, fits)
    static bool attr_set = false;
    const long key = ((long)lc.gridDim.x << 32) | (long)lc.dynamicSmemBytes;
    std::lock_guard<std::mutex> lock(mu);
    for (const auto &k : known)
        if (k.first == key)
            return k.second;
    if (!attr_set)
    {
        cudaFuncSetAttribute((const void *)k_mg_cycles<T>,
                             cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        attr_set = true;
    }
    int nc = 0;
    const bool fits = cudaOccupancyMaxActiveClusters(&nc, (const void *)k_mg_cycles<T>, &lc) ==
                          cudaSuccess &&
                      nc > 0;
    cudaGetLastError();
    known.push_back({key, fits});
    return fits;
}

// check: the convergence test inside the launch; defer: no host wait for the
// launch's outcome (potential_head_finish reads it)
template <typename T>
static int mg_launch(qz_sim *s, int iters, bool check = false, bool defer = false)
{
    const qz_config &c = s->cfg;
    MgArgs<T> A;
    memset(&A, 0, sizeof A);
    A.nlev = (int)s->levels.size();
    A.nsmall = A.nlev - 1;
    for (int l = 0; l < A.nlev; l++)
    {
        A.phi[l] = LevelViews<T>::phi(s, l);
        A.rho[l] = LevelViews<T>::rho(s, l);
        if (A.phi[l].n <= MG_SMALL_N && l < A.nsmall)
            A.nsmall = l;
    }
    A.n_pre = c.n_pre;
    A.n_post = c.n_post;
    A.n_coarse = c.n_coarse;
    A.w = (T)c.w_sor;
    A.scale = (T)0.5; // red-black: half injection (see k_resid_restrict)
    for (int l = 0; l < A.nlev; l++)
    {
        const int n = A.phi[l].n;
        A.h2[l] = (T)((1.0 / (n - 1)) * (1.0 / (n - 1)));
    }
    A.iters = iters;
    A.mixed = std::is_same<T, float>::value ? 1 : 0;
    A.fphi = s->fine_phi;
    A.frho = s->fine_rho;
    A.bar = GridBar{s->gbar, s->flags};
    cudaMemsetAsync(s->gbar, 0, 4 * sizeof(unsigned), s->stream);
    A.check = check ? 1 : 0;
    A.every = A.mixed ? 1 : (c.check_every > 0 ? c.check_every : 1);
    if (A.check)
    {
        const int L = s->L;
        const int nc = 1 << L;
        const double H = 1.0 / nc;
        A.pold = s->pot_old;
        A.part = s->mg_part;
        A.outst = reinterpret_cast<int *>(s->mg_part + 2 * QZ_CG_PART_MAX);
        A.tm = 1.0 - c.tol2;
        A.tp = 1.0 + c.tol2;
        A.rm = 4.0 * c.G * QZ_PI_D * s->head_mass / ((double)nc * nc * nc * H * H * H);
        A.tol = c.tol;
        A.method = c.check_method;
        A.nintr = (long)(nc - 1) * (nc - 1) * (nc - 1);
        if (!s->mg_part)
        {
            set_error("mixed multigrid: partial-sum buffer missing");
            return QZ_FAILURE;
        }
    }
    // shared memory for the small levels (phi and rho of each)
    long elems = 0;
    for (int l = A.nsmall; l < A.nlev; l++)
    {
        A.soff[l] = (int)elems;
        const long n = A.phi[l].n;
        elems += 2 * n * n * n;
    }
    size_t smem = elems * sizeof(T);
    A.smem = smem <= MG_SMEM_MAX ? 1 : 0;
    if (!A.smem)
        smem = 0;
    static int per_sm[2] = {0, 0};
    static std::once_flag once;
    std::call_once(once, [] {
        cudaFuncSetAttribute((const void *)k_mg_cycles<double>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM_MAX);
        cudaFuncSetAttribute((const void *)k_mg_cycles<float>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, MG_SMEM_MAX);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[0], k_mg_cycles<double>, MG_THREADS,
                                                      MG_SMEM_MAX);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm[1], k_mg_cycles<float>, MG_THREADS,
                                                      MG_SMEM_MAX);
    });
    const int ps = per_sm[std::is_same<T, float>::value ? 1 : 0];
    if (ps < 1)
    {
        set_error("multigrid kernel cannot be resident");
        return QZ_FAILURE;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    // mg_points_per_thread points of one colour of the finest level per thread
    // (4 by default), at most two blocks per SM: small heads take few SMs, so
    // independent simulations can run their cycles side by side
    const long m0 = A.phi[0].n - 2;
    const long work = (m0 + 1) / 2 * m0 * m0;
    const long ppt = std::max((long)(c.mg_points_per_thread > 0 ? c.mg_points_per_thread : 4),
                              (long)s->mg_ppt_floor);
    const int blocks = (int)std::max(1L, std::min((long)std::min(ps, 2) * sms,
                                                  (work + ppt * MG_THREADS - 1) / (ppt * MG_THREADS)));
    // tiled coarse levels: the first core (or the configured one) whose two
    // phases fit the shared memory (shared with the sub-cycle's arrays); a level
    // is tiled when its tiles take one round of the launch's blocks
    A.tiled = 0;
    if (c.mg_tile >= 0 && A.nsmall > 1)
    {
        static const int cores[QZ_MG_NTILES][3] = QZ_MG_TILES;
        for (int k = c.mg_tile > 0 ? c.mg_tile - 1 : 0; k < (c.mg_tile > 0 ? c.mg_tile : QZ_MG_NTILES);
             k++)
        {
            const size_t need = (size_t)mg_tile_elems(cores[k], c.n_pre, c.n_post) * sizeof(T);
            if (need > MG_SMEM_MAX)
                continue;
            for (int d = 0; d < 3; d++)
                A.tc[d] = cores[k][d];
            for (int l = 1; l < A.nsmall; l++)
            {
                const long m = A.phi[l].n - 2;
                long nt = 1;
                for (int d = 0; d < 3; d++)
                    nt *= (m + cores[k][d] - 1) / cores[k][d];
                if (nt <= blocks)
                {
                    A.tiled |= 1 << l;
                    A.mid[l] = LevelViews<T>::alt(s, l);
                }
            }
            if (A.tiled)
                smem = std::max(smem, need);
            break;
        }
    }
    // algorithmic bytes of one cycle, as the launch-per-phase path counts them
    double bytes = 0.0;
    for (int l = 0; l < A.nlev; l++)
    {
        const double m = A.phi[l].n - 2;
        const int sweeps = c.n_pre + c.n_post + (l == A.nlev - 1 ? c.n_coarse : 0);
        bytes += sizeof(T) * 3.0 * m * m * m * sweeps;
        if (l < A.nlev - 1)
        {
            const double mc = A.phi[l + 1].n - 2;
            bytes += sizeof(T) * 9.0 * mc * mc * mc + sizeof(T) * 2.125 * m * m * m;
        }
    }
    if (A.mixed)
    {
        const double m = s->fine_phi.n - 2;
        bytes += (A.check ? 56.0 : 40.0) * m * m * m; // the test reads and writes pot_old
    }
    // launches of at most MG_CLUSTER_MAX blocks (small heads: 9 blocks on 33^3)
    // run as one thread-block cluster whose barrier is the hardware's, where
    // the device can place such a cluster with this shared memory
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute la[1];
    A.cluster = 0;
    if (blocks <= MG_CLUSTER_MAX)
    {
        lc.gridDim = dim3(blocks);
        lc.blockDim = dim3(MG_THREADS);
        lc.dynamicSmemBytes = smem;
        lc.stream = s->stream;
        la[0].id = cudaLaunchAttributeClusterDimension;
        la[0].val.clusterDim.x = blocks;
        la[0].val.clusterDim.y = 1;
        la[0].val.clusterDim.z = 1;
        lc.attrs = la;
        lc.numAttrs = 1;
        A.cluster = mg_cluster_fits<T>(lc) ? 1 : 0;
    }
    void *args[] = {&A};
    cudaEvent_t eb = nullptr, ee = nullptr;
    if (s->prof)
    {
        eb = prof_event(s);
        ee = prof_event(s);
        cudaEventRecord(eb, s->stream);
    }
    if (A.cluster)
    {
        if (!check_cuda(cudaLaunchKernelExC(&lc, (const void *)k_mg_cycles<T>, args),
                        "multigrid cycles (cluster)"))
            return QZ_FAILURE;
    }
    else if (!check_cuda(cudaLaunchCooperativeKernel((const void *)k_mg_cycles<T>, dim3(blocks),
                                                     dim3(MG_THREADS), args, smem, s->stream),
                         "multigrid cycles"))
        return QZ_FAILURE;
    s->stats.kernel_launches++;
    if (s->prof)
    {
        cudaEventRecord(ee, s->stream);
        s->prof_pending.push_back({QZ_PROF_SMOOTH, bytes * iters, eb, ee});
    }
    if (A.check && defer)
    {
        s->mg_cycle_bytes = bytes;
        s->mg_prof_idx = s->prof ? (int)s->prof_pending.size() - 1 : -1;
    }
    else if (A.check)
    {
        // iterations run and the test's outcome; the profiler's bytes follow the count
        int st[2] = {0, 0};
        if (!check_cuda(cudaMemcpyAsync(st, A.outst, sizeof st, cudaMemcpyDeviceToHost, s->stream),
                        "multigrid result") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "multigrid result"))
            return QZ_FAILURE;
        s->mg_ran = st[0];
        s->mg_conv = st[1];
        if (s->prof)
            s->prof_pending.back().bytes = bytes * st[0];
    }
    return QZ_SUCCESS;
}

int mg_cycles(qz_sim *s, int iters)
{
    return s->cfg.precision == QZ_PREC_MIXED ? mg_launch<float>(s, iters)
                                               : mg_launch<double>(s, iters);
}

int smooth(qz_sim *s, Grid<double> phi, Grid<double> rho, int iters)
{
    Grid<double> scr{}, alt{};
    if (s->cfg.smoother == 1)
        scr = LevelViews<double>::scratch(s, 0);
    if (s->cfg.smoother == 0 && s->cfg.gs_order == QZ_GS_REDBLACK)
    {
        sync_fine_alt(s);
        alt = LevelViews<double>::alt(s, 0);
    }
    return smooth_t<double>(s, phi, rho, iters, scr, alt, LevelViews<double>::cgs(s, 0));
}

// The fine level's ping-pong partner must carry the fine grid's boundary
// values (Dirichlet during a solve): refresh it from the fine grid.
void sync_fine_alt(qz_sim *s)
{
    if (!s->fine_alt.p)
        return;
    const int n = s->fine_phi.n;
    int tx = n < 128 ? ((n + 31) / 32) * 32 : 128;
    launch(s, QZ_PROF_OTHER, 16.0 * n * n * n, k_copy_grid<double>, dim3((n + tx - 1) / tx, n, n),
           dim3(tx), s->fine_alt, s->fine_phi);
}

// ---- mixed precision: FP64 defect, FP32 cycles ---------------------------------
// r32 = (float)(rho + ooh2 (6 phi - sum)) on the fine interior (FP64 arithmetic).
__global__ void k_fine_residual_f32(Grid<double> phi, Grid<double> rho, float *__restrict__ rf,
                                    double ooh2)
{
    const int n = phi.n, m = n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > m)
        return;
    long gp = phi.off + i + j * phi.sy + k * phi.sz;
    long gr = rho.off + i + j * rho.sy + k * rho.sz;
    const double *p = phi.p;
    double r = rho.p[gr] + ooh2 * (6.0 * p[gp] - p[gp + 1] - p[gp - 1] - p[gp + phi.sy] -
                                   p[gp - phi.sy] - p[gp + phi.sz] - p[gp - phi.sz]);
    rf[i + (long)j * n + (long)k * n * n] = (float)r;
}

__global__ void k_add_correction(Grid<double> phi, const float *__restrict__ ef)
{
    const int n = phi.n, m = n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > m)
        return;
    phi.p[phi.off + i + j * phi.sy + k * phi.sz] += (double)ef[i + (long)j * n + (long)k * n * n];
}

static int mixed_iteration(qz_sim *s)
{
    Grid<double> phi = s->fine_phi, rho = s->fine_rho;
    const int n = phi.n, m = n - 2;
    int tx = m < 128 ? ((m + 31) / 32) * 32 : 128;
    dim3 g((m + tx - 1) / tx, m, m);
    double ooh2 = (double)((n - 1) * (n - 1));
    launch(s, QZ_PROF_OTHER, 20.0 * m * m * m, k_fine_residual_f32, dim3(g), dim3(tx), phi, rho, s->rf, ooh2);
    cudaMemsetAsync(s->ef, 0, (size_t)n * n * n * sizeof(float), s->stream);
    int inner = s->cfg.inner_cycles > 0 ? s->cfg.inner_cycles : 1;
    for (int q = 0; q < inner; q++)
        if (vcycle_t<float>(s, 0, s->cfg.cycle))
            return QZ_FAILURE;
    launch(s, QZ_PROF_OTHER, 20.0 * m * m * m, k_add_correction, dim3(g), dim3(tx), phi, s->ef);
    return check_cuda(cudaGetLastError(), "mixed iteration") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- convergence test (poisson_error.c:36-133) ------------------------------------
constexpr int CK_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double *sh)
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

__global__ void k_check_partial(int L, long D, const double *__restrict__ pot,
                                const double *__restrict__ pot_old, const double *__restrict__ d,
                                double tm, double tp, double oh2, double rm, double tol,
                                int method, double *__restrict__ partial, int *__restrict__ flags)
{
    __shared__ double sh[32];
    const int m = (1 << L) - 1;
    const long total = (long)m * m * m;
    const long D2 = D * D;
    double acc = 0.0;
    int ratio_fail = 0, resid_fail = 0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x)
    {
        int i = 2 + (int)(t % m), j = 2 + (int)((t / m) % m), k = 2 + (int)(t / ((long)m * m));
        long g = i + j * D + k * D2;
        double a = pot[g] / pot_old[g];
        if ((tm > a) || (tp < a))
            ratio_fail = 1;
        double diff = d[g] + oh2 * (6.0 * pot[g] - pot[g + 1] - pot[g - 1] - pot[g + D] -
                                    pot[g - D] - pot[g + D2] - pot[g - D2]);
        if (method == 1)
        {
            if (fabs(diff) / rm >= tol)
                resid_fail = 1;
        }
        else
            acc += diff * diff;
    }
    if (__syncthreads_or(ratio_fail) && threadIdx.x == 0)
        flags[F_RATIO_FAIL] = 1;
    if (__syncthreads_or(resid_fail) && threadIdx.x == 0)
        flags[F_RESID_FAIL] = 1;
    double b = block_sum(acc, sh);
    if (threadIdx.x == 0)
        partial[blockIdx.x] = b;
}

__global__ void k_check_final(int nblocks, long nintr, double rm, double tol, int method,
                              const double *__restrict__ partial, int *__restrict__ flags,
                              double *__restrict__ err_out)
{
    __shared__ double sh[32];
    double acc = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
        acc += partial[b];
    double tot = block_sum(acc, sh);
    if (threadIdx.x == 0)
    {
        int ok;
        double err = 0.0;
        if (method == 1)
            ok = !flags[F_RESID_FAIL];
        else
        {
            err = tot / nintr;
            err = sqrt(err);
            err = err / rm;
            if (method == 2)
                err = err / (cbrt((double)nintr) * cbrt((double)nintr));
            ok = err < tol;
        }
        *err_out = err;
        flags[F_CONVERGED] = (!flags[F_RATIO_FAIL]) && ok;
    }
}

__global__ void k_copy_if_unconverged(long n, const double *__restrict__ src,
                                      double *__restrict__ dst, const int *__restrict__ flags)
{
    if (flags[F_CONVERGED])
        return;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

static int launch_check(qz_sim *s, double node_mass)
{
    const qz_config &c = s->cfg;
    const int L = s->L;
    const int nc = 1 << L;
    const double H = 1.0 / (1 << L);
    const double oh2 = 1.0 / (H * H);
    const int size = nc * nc * nc;
    const long nintr = (long)(nc - 1) * (nc - 1) * (nc - 1);
    const double rm = 4.0 * c.G * QZ_PI_D * node_mass / (size * H * H * H);
    cudaMemsetAsync(s->flags + F_RATIO_FAIL, 0, sizeof(int), s->stream);
    cudaMemsetAsync(s->flags + F_RESID_FAIL, 0, sizeof(int), s->stream);
    launch(s, QZ_PROF_CHECK, 24.0 * (double)nintr, k_check_partial, dim3(s->red_blocks), dim3(CK_THREADS), L, s->D, s->pot, s->pot_old, s->d, 1.0 - c.tol2, 1.0 + c.tol2, oh2, rm, c.tol, c.check_method, s->red, s->flags);
    launch(s, QZ_PROF_CHECK, 8.0 * s->red_blocks, k_check_final, dim3(1), dim3(256), s->red_blocks, nintr, rm, c.tol, c.check_method, s->red, s->flags, s->red + s->red_blocks);
    launch(s, QZ_PROF_CHECK, 16.0 * s->gpts, k_copy_if_unconverged, dim3(296), dim3(256), s->gpts, s->pot, s->pot_old, s->flags);
    cudaMemcpyAsync(s->h_flags, s->flags, F_COUNT * sizeof(int), cudaMemcpyDeviceToHost,
                    s->stream);
    return check_cuda(cudaGetLastError(), "convergence check") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- Poisson solve with zero Dirichlet boundary (adjoint of the head solve) ----------
// Partial sums, per block, of r^2 and f^2 over the head interior, r = f + (6 lam -
// sum of the 6 neighbours) / H^2 (the residual convention of the head solve).
__global__ void k_resid_norm_partial(int L, long D, const double *__restrict__ lam,
                                     const double *__restrict__ f, double oh2,
                                     double *__restrict__ partial)
{
    __shared__ double sh[32];
    const int m = (1 << L) - 1;
    const long total = (long)m * m * m;
    const long D2 = D * D;
    double rr = 0.0, ff = 0.0;
    for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long)gridDim.x * blockDim.x)
    {
        const long i = 2 + t % m, j = 2 + (t / m) % m, k = 2 + t / ((long)m * m);
        const long g = i + j * D + k * D2;
        const double r = f[g] + oh2 * (6.0 * lam[g] - lam[g + 1] - lam[g - 1] - lam[g + D] -
                                       lam[g - D] - lam[g + D2] - lam[g - D2]);
        rr += r * r;
        ff += f[g] * f[g];
    }
    const double a = block_sum(rr, sh);
    const double b = block_sum(ff, sh);
    if (threadIdx.x == 0)
    {
        partial[2 * blockIdx.x] = a;
        partial[2 * blockIdx.x + 1] = b;
    }
}

__global__ void k_resid_norm_final(int nb, const double *__restrict__ partial,
                                   double *__restrict__ out)
{
    __shared__ double sh[32];
    double a = 0.0, b = 0.0;
    for (int q = threadIdx.x; q < nb; q += blockDim.x)
    {
        a += partial[2 * q];
        b += partial[2 * q + 1];
    }
    a = block_sum(a, sh);
    b = block_sum(b, sh);
    if (threadIdx.x == 0)
    {
        out[0] = a;
        out[1] = b;
    }
}

// |r|^2 and |f|^2 of lam against f into host[0..1] (pinned), synchronising.
static int resid_norms(qz_sim *s, const double *lam, const double *f, double *scratch,
                       double *host)
{
    const double H = 1.0 / (1 << s->L);
    const long m = (1L << s->L) - 1;
    launch(s, QZ_PROF_CHECK, 16.0 * m * m * m, k_resid_norm_partial, dim3(s->red_blocks),
           dim3(CK_THREADS), s->L, s->D, lam, f, 1.0 / (H * H), scratch);
    launch(s, QZ_PROF_CHECK, 16.0 * s->red_blocks, k_resid_norm_final, dim3(1), dim3(256),
           s->red_blocks, scratch, scratch + 2 * s->red_blocks);
    if (!check_cuda(cudaMemcpyAsync(host, scratch + 2 * s->red_blocks, 2 * sizeof(double),
                                    cudaMemcpyDeviceToHost, s->stream),
                    "residual norm") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "residual norm sync"))
        return QZ_FAILURE;
    return QZ_SUCCESS;
}

// Solves Lap_h lam = f on the head interior with lam = 0 on the solve grid's
// boundary, by FP64 multigrid cycles of the configured kind (the operator of
// the head solve is symmetric, so this is also its adjoint), from the initial
// guess in lam, until |r| <= rtol |f| (checked every 2 cycles).  scratch holds
// 2 * red_blocks + 2 doubles; host 2 pinned doubles.  *cycles: cycles run.
int solve_zero_bc(qz_sim *s, double *lam, double *f, double rtol, double *scratch,
                  double *host, int *cycles)
{
    const qz_config &c = s->cfg;
    *cycles = 0;
    if (resid_norms(s, lam, f, scratch, host))
        return QZ_FAILURE;
    if (host[1] == 0.0)
    {
        cudaMemsetAsync(lam, 0, s->gpts * sizeof(double), s->stream);
        return QZ_SUCCESS;
    }
    const double goal = rtol * rtol * host[1];
    if (host[0] <= goal)
        return QZ_SUCCESS;
    const Grid<double> keep_phi = s->fine_phi, keep_rho = s->fine_rho;
    s->fine_phi = head_view(s, lam);
    s->fine_rho = head_view(s, f);
    sync_fine_alt(s);
    int rc = QZ_SUCCESS;
    bool done = false;
    while (!done && *cycles < c.max_iter)
    {
        const int k = std::min(2, c.max_iter - *cycles);
        if (mg_persistent(s))
            rc = mg_launch<double>(s, k);
        else
            for (int q = 0; q < k && !rc; q++)
                rc = vcycle(s, 0, c.cycle);
        if (rc)
            break;
        *cycles += k;
        if ((rc = resid_norms(s, lam, f, scratch, host)))
            break;
        if (!check_cuda(cudaMemcpyAsync(s->h_flags, s->flags, F_COUNT * sizeof(int),
                                        cudaMemcpyDeviceToHost, s->stream), "flags") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "flags sync"))
        {
            rc = QZ_FAILURE;
            break;
        }
        if (s->h_flags[F_ERROR] & E_BARRIER)
        {
            set_error("adjoint multigrid cycles: a grid barrier wait gave up");
            rc = QZ_FAILURE;
            break;
        }
        done = host[0] <= goal;
    }
    s->fine_phi = keep_phi;
    s->fine_rho = keep_rho;
    sync_fine_alt(s);
    if (!rc && !done)
    {
        set_error("adjoint Poisson solve: |r|/|f| = %.3e after %d cycles (goal %.3e)",
                  sqrt(host[0] / host[1]), *cycles, rtol);
        rc = QZ_FAILURE;
    }
    return rc;
}

// Captures `every` solver iterations followed by the convergence test into a
// CUDA graph (kernel parameters and buffers of a context never change).
static int capture_check_block(qz_sim *s, int every)
{
    const long long before = s->stats.kernel_launches;
    if (!check_cuda(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal),
                    "begin capture"))
        return QZ_FAILURE;
    int rc = QZ_SUCCESS;
    for (int q = 0; q < every && rc == QZ_SUCCESS; q++)
        rc = s->cfg.precision == QZ_PREC_MIXED ? mixed_iteration(s) : vcycle(s, 0, s->cfg.cycle);
    if (rc == QZ_SUCCESS)
        rc = launch_check(s, s->head_mass);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    s->check_graph_kernels = s->stats.kernel_launches - before;
    s->stats.kernel_launches = before;
    if (rc != QZ_SUCCESS || !check_cuda(e, "end capture"))
    {
        if (g)
            cudaGraphDestroy(g);
        return QZ_FAILURE;
    }
    e = cudaGraphInstantiate(&s->check_exec, g, 0);
    cudaGraphDestroy(g);
    return check_cuda(e, "graph instantiate") ? QZ_SUCCESS : QZ_FAILURE;
}

int poisson_error_head(qz_sim *s, int *converged)
{
    if (launch_check(s, s->head_mass))
        return QZ_FAILURE;
    if (!check_cuda(cudaStreamSynchronize(s->stream), "convergence readback"))
        return QZ_FAILURE;
    *converged = s->h_flags[F_CONVERGED] != 0;
    return QZ_SUCCESS;
}

// The head solve is one persistent launch with the convergence test inside it
// (multigrid cycles of the red-black V-cycle, FP64 or the mixed form, no
// replayed schedule).
bool head_one_launch(const qz_sim *s)
{
    return s->cfg.head_pot_method != 1 && s->sched_mode != 2 && mg_persistent(s);
}

// Iteration count, outcome and statistics of a head solve (potential_head_node.c:151-155:
// reaching the cap is a failure).
static int head_tail(qz_sim *s, int iter, bool check)
{
    const qz_config &c = s->cfg;
    s->stats.last_vcycles = iter;
    s->stats.vcycles_total += iter;
    s->stats.last_converged = check ? 1 : 0;
    if (s->sched_mode == 1)
        sched_put(s, &iter, 1);
    if (iter == c.max_iter)
    {
        set_error("the precision was not reached in the head node after %d multigrid cycles",
                  iter);
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

// First half of a one-launch head solve: pot_old, the fine-level views and the
// cooperative launch, all on stream st, with no host wait.  *issued is false
// (and nothing is queued) when the head solve is not one launch.
int potential_head_issue(qz_sim *s, cudaStream_t st, bool *issued)
{
    *issued = false;
    if (!head_one_launch(s))
        return QZ_SUCCESS;
    const qz_config &c = s->cfg;
    cudaStream_t keep = s->stream;
    s->stream = st;
    cudaMemcpyAsync(s->pot_old, s->pot, s->gpts * sizeof(double), cudaMemcpyDeviceToDevice,
                    s->stream);
    sync_fine_alt(s);
    // the mixed form tests after every defect-correction iteration (its FP64
    // residual is computed anyway); the FP64 form keeps the reference's cadence
    const int rc = c.precision == QZ_PREC_MIXED ? mg_launch<float>(s, c.max_iter, true, true)
                                                : mg_launch<double>(s, c.max_iter, true, true);
    s->stream = keep;
    *issued = rc == QZ_SUCCESS;
    return rc;
}

// Second half: waits for the launch on stream st and reads its iteration count,
// the test's outcome and the barrier status.
int potential_head_finish(qz_sim *s, cudaStream_t st)
{
    int out[2] = {0, 0};
    const int *outst = reinterpret_cast<const int *>(s->mg_part + 2 * QZ_CG_PART_MAX);
    if (!check_cuda(cudaMemcpyAsync(out, outst, sizeof out, cudaMemcpyDeviceToHost, st),
                    "multigrid result") ||
        !check_cuda(cudaMemcpyAsync(s->h_flags, s->flags, F_COUNT * sizeof(int),
                                    cudaMemcpyDeviceToHost, st),
                    "flags") ||
        !check_cuda(cudaStreamSynchronize(st), "multigrid result"))
        return QZ_FAILURE;
    s->mg_ran = out[0];
    s->mg_conv = out[1];
    if (s->mg_prof_idx >= 0 && s->mg_prof_idx < (int)s->prof_pending.size())
        s->prof_pending[s->mg_prof_idx].bytes = s->mg_cycle_bytes * out[0];
    s->mg_prof_idx = -1;
    if (s->h_flags[F_ERROR] & E_BARRIER)
    {
        set_error("multigrid cycles: a grid barrier wait gave up");
        return QZ_FAILURE;
    }
    return head_tail(s, s->mg_ran, s->mg_conv != 0);
}

int potential_head(qz_sim *s)
{
    const qz_config &c = s->cfg;
    if (head_one_launch(s))
    {
        bool issued = false;
        if (potential_head_issue(s, s->stream, &issued))
            return QZ_FAILURE;
        return potential_head_finish(s, s->stream);
    }
    cudaMemcpyAsync(s->pot_old, s->pot, s->gpts * sizeof(double), cudaMemcpyDeviceToDevice,
                    s->stream);
    if (c.head_pot_method == 1)
        return head_cg_solve(s);
    sync_fine_alt(s);
    int iter = 0;
    bool check = false;
    if (s->sched_mode == 2)
    {
        // replay: exactly the recorded number of cycles, no convergence test
        int n = 0;
        if (!sched_take(s, 1, &n))
            return QZ_FAILURE;
        if (mg_persistent(s))
        {
            if (n > 0 && mg_cycles(s, n))
                return QZ_FAILURE;
        }
        else
            for (int q = 0; q < n; q++)
                if (c.precision == QZ_PREC_MIXED ? mixed_iteration(s) : vcycle(s, 0, c.cycle))
                    return QZ_FAILURE;
        s->stats.last_vcycles = n;
        s->stats.vcycles_total += n;
        s->stats.last_converged = 1;
        return check_cuda(cudaGetLastError(), "replayed head solve") ? QZ_SUCCESS : QZ_FAILURE;
    }
    // the mixed form tests after every defect-correction iteration (its FP64
    // residual is computed anyway); the FP64 form keeps the reference's cadence
    const int every =
        c.precision == QZ_PREC_MIXED ? 1 : (c.check_every > 0 ? c.check_every : 1);
    const bool graphs = s->use_graphs && !s->prof;
    while (iter < c.max_iter && !check)
    {
        if (graphs && iter % every == 0 && c.max_iter - iter >= every)
        {
            // one graph launch = `every` cycles + the convergence test + flag read-back
            if (!s->check_exec && capture_check_block(s, every))
                return QZ_FAILURE;
            if (!check_cuda(cudaGraphLaunch(s->check_exec, s->stream), "check-block graph"))
                return QZ_FAILURE;
            s->stats.kernel_launches += s->check_graph_kernels;
            iter += every;
            if (!check_cuda(cudaStreamSynchronize(s->stream), "convergence readback"))
                return QZ_FAILURE;
            check = s->h_flags[F_CONVERGED] != 0;
            continue;
        }
        int k = every - (iter % every);
        if (k > c.max_iter - iter)
            k = c.max_iter - iter;
        for (int q = 0; q < k; q++)
        {
            int rc = c.precision == QZ_PREC_MIXED ? mixed_iteration(s) : vcycle(s, 0, c.cycle);
            if (rc)
                return QZ_FAILURE;
            iter++;
        }
        if (iter % every == 0)
        {
            if (launch_check(s, s->head_mass))
                return QZ_FAILURE;
            if (!check_cuda(cudaStreamSynchronize(s->stream), "convergence readback"))
                return QZ_FAILURE;
            check = s->h_flags[F_CONVERGED] != 0;
        }
    }
    return head_tail(s, iter, check);
}

} // namespace qz

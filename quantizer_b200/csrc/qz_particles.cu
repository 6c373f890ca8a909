// qz_particles.cu -- particle-side kernels of the head-node step:
//   CIC deposit      (grid_density.c:35-111)      sort + segmented reduce + gather
//   CIC gather       (particle_acceleration.c:33-132)
//   kick-drift       (particle_updating.c:39-207)
//   kick             (particle_updating.c:2677-2688)
//   box index        (ptcl_idx_to_box_idx.c:30-139)
//   head boundary    (initial_potential_and_acceleration_head.c:297-334)
//
// Floating-point expressions keep the reference's operand order; the library
// is built with -fmad=false, so products and sums round exactly as the
// reference's x86-64 FP64 code (no contraction).  The deposit differs from the
// reference only in the order in which particle contributions are summed at a
// grid point (cell by cell instead of particle index order), which is
// deterministic from run to run.
#include "qz_internal.cuh"

namespace qz {

#define QZ_PI_D 3.14159265358979323846

// ---- analytic head boundary ---------------------------------------------------
__global__ void k_initial_head(int L, long D, double G, double M, double *__restrict__ pot,
                               double *__restrict__ ax, double *__restrict__ ay,
                               double *__restrict__ az)
{
    const int B = (1 << L) + 2; // box cells per side; points 0..B-1 are filled
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    long total = (long)B * B * B;
    if (t >= total)
        return;
    int i = (int)(t % B), j = (int)((t / B) % B), k = (int)(t / ((long)B * B));
    const double H = 1.0 / (1 << L);
    double ai = (i - 1) * H - 0.5, aj = (j - 1) * H - 0.5, ak = (k - 1) * H - 0.5;
    double dist = ai * ai + aj * aj + ak * ak;
    dist = sqrt(dist);
    if (dist == 0.0)
        dist = 1.0 / (1 << L) * 1.0e-3;
    long g = i + (long)j * D + (long)k * D * D;
    double coeff = -G * M / (dist * dist * dist);
    pot[g] = -G * M / dist;
    ax[g] = coeff * ai;
    ay[g] = coeff * aj;
    az[g] = coeff * ak;
}

// Periodic boundaries (initial_potential_and_acceleration_head.c:78-296): only
// points with a box coordinate equal to 1 (coordinates 1 .. 2^L, k outer, i
// inner) are written, with -G M / d, d the smallest distance from the centre
// over the point and its images on the far faces (coordinate gl = 2^L + 1); the
// point's acceleration -G M (a_i, a_j, a_k) / d^3 is copied to its images.  The
// image indices are the reference's as written (:125-126, :178, :203, :225 use
// x coordinate 1 where the point's own i would be expected), so later points
// overwrite some far-face values and others stay zero.  Writes of a k-plane
// land in that plane (k = 1 also in plane gl), so one thread per plane keeps
// the reference's write order.
__device__ __forceinline__ long pgi(long i, long j, long k, long D) { return i + j * D + k * D * D; }

__global__ void k_initial_head_periodic(int L, long D, double G, double M,
                                        double *__restrict__ pot, double *__restrict__ ax,
                                        double *__restrict__ ay, double *__restrict__ az)
{
    const int nc = 1 << L, gl = nc + 1;
    const int k = 1 + (int)((long)blockIdx.x * blockDim.x + threadIdx.x);
    if (k >= gl)
        return;
    const double H = 1.0 / nc;
    const double a0 = (gl - 1) * H - 0.5;
    const double ak = (k - 1) * H - 0.5;
    for (int j = 1; j < gl; j++)
    {
        const double aj = (j - 1) * H - 0.5;
        for (int i = 1; i < gl; i++)
        {
            if (i != 1 && j != 1 && k != 1)
                continue;
            const double ai = (i - 1) * H - 0.5;
            long idx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            double dist = 0.0;
            int cnt = 0;
            if (i == 1)
            {
                idx[0] = pgi(i, j, k, D);
                idx[1] = pgi(gl, j, k, D);
                const double d0 = sqrt(ai * ai + aj * aj + ak * ak);
                const double d1 = sqrt(a0 * a0 + aj * aj + ak * ak);
                dist = d0 < d1 ? d0 : d1;
                cnt++;
            }
            if (j == 1)
            {
                if (cnt == 0)
                {
                    idx[0] = pgi(i, j, k, D);
                    idx[1] = pgi(1, gl, k, D);
                    const double d0 = sqrt(ai * ai + aj * aj + ak * ak);
                    const double d1 = sqrt(ai * ai + a0 * a0 + ak * ak);
                    dist = d0 < d1 ? d0 : d1;
                }
                else
                {
                    idx[2] = pgi(1, gl, k, D);
                    idx[3] = pgi(gl, gl, k, D);
                    const double d2 = sqrt(ai * ai + a0 * a0 + ak * ak);
                    const double d3 = sqrt(a0 * a0 + a0 * a0 + ak * ak);
                    dist = dist < d2 ? dist : d2;
                    dist = dist < d3 ? dist : d3;
                }
                cnt++;
            }
            if (k == 1)
            {
                if (cnt == 0)
                {
                    idx[0] = pgi(i, j, k, D);
                    idx[1] = pgi(1, j, gl, D);
                    const double d0 = sqrt(ai * ai + aj * aj + ak * ak);
                    const double d1 = sqrt(ai * ai + aj * aj + a0 * a0);
                    dist = d0 < d1 ? d0 : d1;
                }
                else if (cnt == 1)
                {
                    double d2, d3;
                    idx[2] = pgi(1, j, gl, D);
                    d2 = sqrt(ai * ai + aj * aj + a0 * a0);
                    if (i == 1)
                    {
                        idx[3] = pgi(gl, j, gl, D);
                        d3 = sqrt(a0 * a0 + aj * aj + a0 * a0);
                    }
                    else
                    {
                        idx[3] = pgi(i, gl, gl, D);
                        d3 = sqrt(ai * ai + a0 * a0 + a0 * a0);
                    }
                    dist = dist < d2 ? dist : d2;
                    dist = dist < d3 ? dist : d3;
                }
                else
                {
                    idx[4] = pgi(1, j, gl, D);
                    idx[5] = pgi(gl, j, gl, D);
                    idx[6] = pgi(1, gl, gl, D);
                    idx[7] = pgi(gl, gl, gl, D);
                    const double e4 = sqrt(ai * ai + aj * aj + a0 * a0);
                    const double e5 = sqrt(a0 * a0 + aj * aj + a0 * a0);
                    const double e6 = sqrt(ai * ai + a0 * a0 + a0 * a0);
                    const double e7 = sqrt(a0 * a0 + a0 * a0 + a0 * a0);
                    dist = dist < e4 ? dist : e4;
                    dist = dist < e5 ? dist : e5;
                    dist = dist < e6 ? dist : e6;
                    dist = dist < e7 ? dist : e7;
                }
                cnt++;
            }
            const double c = -G * M / dist;
            for (int l = 0; l < (1 << cnt); l++)
                pot[idx[l]] = c;
            const double c3 = -G * M / (dist * dist * dist);
            const double vx = c3 * ai, vy = c3 * aj, vz = c3 * ak;
            for (int l = 0; l < (1 << cnt); l++)
            {
                ax[idx[l]] = vx;
                ay[idx[l]] = vy;
                az[idx[l]] = vz;
            }
        }
    }
}

int head_initial(qz_sim *s)
{
    size_t bytes = (size_t)s->gpts * sizeof(double);
    cudaMemsetAsync(s->pot, 0, bytes, s->stream);
    cudaMemsetAsync(s->gax, 0, bytes, s->stream);
    cudaMemsetAsync(s->gay, 0, bytes, s->stream);
    cudaMemsetAsync(s->gaz, 0, bytes, s->stream);
    if (s->cfg.bdry == 0)
    {
        const int nc = 1 << s->L;
        launch(s, QZ_PROF_OTHER, 96.0 * 3 * nc * nc, k_initial_head_periodic,
               dim3(blocks_for(nc, 128)), dim3(128), s->L, s->D, s->cfg.G, s->cfg.total_mass,
               s->pot, s->gax, s->gay, s->gaz);
        return check_cuda(cudaGetLastError(), "initial head") ? QZ_SUCCESS : QZ_FAILURE;
    }
    long B = (1L << s->L) + 2;
    launch(s, QZ_PROF_OTHER, 32.0 * B * B * B, k_initial_head, dim3(blocks_for(B * B * B, 256)), dim3(256), s->L, s->D, s->cfg.G, s->cfg.total_mass, s->pot, s->gax, s->gay, s->gaz);
    return check_cuda(cudaGetLastError(), "initial head") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- deposit --------------------------------------------------------------------
// Cell key of a particle in the head box: box-cell coordinates floor(x 2^L) + 1
// (box_ts = -1), linear on B = 2^L + 2 cells per side.
__device__ __forceinline__ int cell_coord(double x, int L, int *err)
{
    int f = (int)(x * (1 << L));
    if (!(x >= 0.0) || f > (1 << L)) // outside [0, 1] or NaN: clamp and flag
    {
        *err |= E_PTCL_OUTSIDE;
        f = x > 0.5 ? (1 << L) : 0;
    }
    return f + 1;
}

// Morton (Z-order) keys of head cells: the bits of the three box coordinates
// interleaved (x lowest), 10 bits a coordinate at most.
__device__ __forceinline__ unsigned morton_spread(unsigned v)
{
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

__device__ __forceinline__ unsigned morton_compact(unsigned v)
{
    v &= 0x09249249u;
    v = (v ^ (v >> 2)) & 0x030c30c3u;
    v = (v ^ (v >> 4)) & 0x0300f00fu;
    v = (v ^ (v >> 8)) & 0x030000ffu;
    v = (v ^ (v >> 16)) & 0x3ffu;
    return v;
}

// Linear cell index of a key: keys are linear (morton_B == 0) or Morton codes
// of a box of morton_B cells a side.
__device__ __forceinline__ long key_cell(unsigned k, unsigned morton_B)
{
    if (!morton_B)
        return k;
    const long B = morton_B;
    return morton_compact(k) + morton_compact(k >> 1) * B + morton_compact(k >> 2) * B * B;
}

// Head cell key of every particle: the Morton code of its box cell when the
// codes fit (3 (L + 1) <= 30 bits), so that cells close in space are close in
// the sorted order; else the linear index bx + by B + bz B^2.
__global__ void k_head_keys(long n, int L, int morton, const double *__restrict__ x,
                            const double *__restrict__ y, const double *__restrict__ z,
                            unsigned *__restrict__ keys, int *__restrict__ vals,
                            int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const unsigned B = (1u << L) + 2u;
    int err = 0;
    unsigned bx = cell_coord(x[i], L, &err), by = cell_coord(y[i], L, &err),
             bz = cell_coord(z[i], L, &err);
    keys[i] = morton ? morton_spread(bx) | (morton_spread(by) << 1) | (morton_spread(bz) << 2)
                     : bx + by * B + bz * B * B;
    vals[i] = (int)i;
    if (err)
        atomicOr(&flags[F_ERROR], err);
}

__global__ void k_seg_heads(long n, const unsigned *__restrict__ k, int *__restrict__ head)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    head[i] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
}

__global__ void k_seg_fill(long n, unsigned morton_B, const unsigned *__restrict__ k,
                           const int *__restrict__ head, const int *__restrict__ sid,
                           int *__restrict__ seg_start, int *__restrict__ seg_cell,
                           int *__restrict__ cell_seg, int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    if (head[i])
    {
        int sgm = sid[i];
        seg_start[sgm] = (int)i;
        seg_cell[sgm] = (int)k[i];
        cell_seg[key_cell(k[i], morton_B)] = sgm;
    }
    if (i == n - 1)
    {
        int nseg = sid[i] + head[i];
        seg_start[nseg] = (int)n;
        flags[F_NSEG] = nseg;
    }
}

// One warp per occupied cell: the 8 CIC corner sums of coeff * m * w over the
// cell's particles (lane-strided partial sums, then a fixed xor-shuffle tree).
// Particle i's CIC corner weights times 4 pi G m / H^3, added to acc.
__device__ __forceinline__ void head_cic_add(int i, double scale, double coeff,
                                             const double *__restrict__ x,
                                             const double *__restrict__ y,
                                             const double *__restrict__ z,
                                             const double *__restrict__ m, double acc[8])
{
    double px = x[i] * scale, py = y[i] * scale, pz = z[i] * scale;
    int fx = (int)px, fy = (int)py, fz = (int)pz;
    double wx1 = px - fx, wy1 = py - fy, wz1 = pz - fz;
    double wx2 = 1.0 - wx1, wy2 = 1.0 - wy1, wz2 = 1.0 - wz1;
    double cm = coeff * m[i];
    acc[0] += cm * (wx2 * wy2 * wz2);
    acc[1] += cm * (wx1 * wy2 * wz2);
    acc[2] += cm * (wx2 * wy1 * wz2);
    acc[3] += cm * (wx1 * wy1 * wz2);
    acc[4] += cm * (wx2 * wy2 * wz1);
    acc[5] += cm * (wx1 * wy2 * wz1);
    acc[6] += cm * (wx2 * wy1 * wz1);
    acc[7] += cm * (wx1 * wy1 * wz1);
}

// One warp per occupied cell of at most SEG_LONG particles; longer cells are
// listed for k_seg_long.
__global__ void k_seg_reduce(int L, double coeff, const int *__restrict__ perm,
                             const int *__restrict__ seg_start, int *__restrict__ flags,
                             int *__restrict__ long_list, const double *__restrict__ x,
                             const double *__restrict__ y, const double *__restrict__ z,
                             const double *__restrict__ m, double *__restrict__ cs)
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
        double acc[8];
#pragma unroll
        for (int c = 0; c < 8; c++)
            acc[c] = 0.0;
        for (int q = b + lane; q < e; q += 32)
            head_cic_add(perm[q], scale, coeff, x, y, z, m, acc);
#pragma unroll
        for (int c = 0; c < 8; c++)
        {
            double v = acc[c];
            for (int o = 16; o > 0; o >>= 1)
                v += __shfl_xor_sync(0xffffffffu, v, o);
            acc[c] = v;
        }
        if (lane < 8)
        {
            double v = acc[0];
#pragma unroll
            for (int c = 1; c < 8; c++)
                if (lane == c)
                    v = acc[c];
            cs[sg * 8 + lane] = v;
        }
    }
}

// One block per occupied cell listed by k_seg_reduce (more than SEG_LONG
// particles): thread t adds particles t, t + blockDim, ... of the cell (four at
// a time, their loads together), then the block sums in a fixed order, so the
// result does not depend on scheduling.
__global__ void __launch_bounds__(SEG_LONG_THREADS)
    k_seg_long(int L, double coeff, const int *__restrict__ perm,
               const int *__restrict__ seg_start, const int *__restrict__ flags,
               const int *__restrict__ long_list, const double *__restrict__ x,
               const double *__restrict__ y, const double *__restrict__ z,
               const double *__restrict__ m, double *__restrict__ cs)
{
    __shared__ double shw[(SEG_LONG_THREADS / 32) * 8];
    const int nl = flags[F_NLONG];
    const double scale = (double)(1 << L);
    const int bs = (int)blockDim.x;
    for (int li = blockIdx.x; li < nl; li += gridDim.x)
    {
        const int sg = long_list[li];
        const int b = seg_start[sg], e = seg_start[sg + 1];
        double acc[8];
#pragma unroll
        for (int c = 0; c < 8; c++)
            acc[c] = 0.0;
        for (int q0 = b + (int)threadIdx.x; q0 < e; q0 += 4 * bs)
        {
            int iq[4];
#pragma unroll
            for (int u = 0; u < 4; u++)
            {
                const int q = q0 + u * bs;
                iq[u] = q < e ? perm[q] : -1;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (iq[u] >= 0)
                    head_cic_add(iq[u], scale, coeff, x, y, z, m, acc);
        }
        seg_block_sums<8>(acc, shw);
        if (threadIdx.x < 8)
            cs[(long)sg * 8 + threadIdx.x] = acc[0];
        __syncthreads(); // shw is rewritten for the next cell
    }
}

// Each grid point sums the corner contributions of its (up to) 8 adjacent
// occupied cells in a fixed order.
__global__ void k_point_gather(int L, long D, const int *__restrict__ cell_seg,
                               const double *__restrict__ cs, double *__restrict__ d)
{
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x, uD = (unsigned)D;
    if (t >= uD * uD * uD)
        return;
    const long B = D - 1;
    const unsigned q = t / uD, r = q / uD;
    const int gx = (int)(t - q * uD), gy = (int)(q - r * uD), gz = (int)r;
    double acc = 0.0;
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
                    acc += cs[(long)sg * 8 + (1 - a) + 2 * (1 - b) + 4 * (1 - c)];
            }
        }
    }
    d[t] = acc;
}

// Sorts the m (cell key, particle) pairs staged in s->sort.k0 / v0 and builds
// the cell segments: seg_start / seg_cell (the key) of every occupied cell,
// cell_seg (ncells_box entries by linear cell index, -1 for empty cells; keys
// are Morton codes of a box of morton_B cells a side when morton_B > 0) and
// flags[F_NSEG].
int deposit_segments(qz_sim *s, long m, int bits, int *cell_seg, long ncells_box,
                     unsigned **ks_out, int **perm_out, unsigned morton_B)
{
    unsigned *ks;
    int *perm;
    if (radix_sort_pairs(s, m, bits, &ks, &perm))
        return QZ_FAILURE;
    cudaMemsetAsync(cell_seg, 0xFF, (size_t)ncells_box * sizeof(int), s->stream);
    if (m > 0)
    {
        launch(s, QZ_PROF_DEPOSIT, 8.0 * m, k_seg_heads, dim3(blocks_for(m, 256)), dim3(256), m,
               ks, s->seg_head);
        if (scan_exclusive(s, s->seg_head, s->seg_id, m))
            return QZ_FAILURE;
        launch(s, QZ_PROF_DEPOSIT, 12.0 * m, k_seg_fill, dim3(blocks_for(m, 256)), dim3(256), m,
               morton_B, ks, s->seg_head, s->seg_id, s->seg_start, s->seg_cell, cell_seg,
               s->flags);
    }
    else
        cudaMemsetAsync(s->flags + F_NSEG, 0, sizeof(int), s->stream);
    *ks_out = ks;
    *perm_out = perm;
    return QZ_SUCCESS;
}

// Head cell keys of the particles at (x, y, z), sorted, and their cell
// segments (seg_start, cell_seg, flags[F_NSEG]); *perm_out: particle of each
// sorted position.
int head_segments(qz_sim *s, const double *x, const double *y, const double *z, int **perm_out)
{
    const long n = s->n;
    const int L = s->L;
    const long B = (1L << L) + 2;
    // Morton keys need L + 1 bits a coordinate (B <= 2^(L+1))
    const int morton = 3 * (L + 1) <= 30 ? 1 : 0;
    launch(s, QZ_PROF_DEPOSIT, 32.0 * n, k_head_keys, dim3(blocks_for(n, 256)), dim3(256), n, L,
           morton, x, y, z, s->sort.k0, s->sort.v0, s->flags);
    int bits = 1;
    if (morton)
        bits = 3 * (L + 1);
    else
        while ((1L << bits) < B * B * B)
            bits++;
    unsigned *ks;
    return deposit_segments(s, n, bits, s->cell_seg, B * B * B, &ks, perm_out,
                            morton ? (unsigned)B : 0u);
}

int deposit_head(qz_sim *s)
{
    const long n = s->n;
    const int L = s->L;
    if (n == 0)
        return cudaMemsetAsync(s->d, 0, s->gpts * sizeof(double), s->stream) == cudaSuccess
                   ? QZ_SUCCESS
                   : QZ_FAILURE;
    int *perm;
    if (head_segments(s, s->x, s->y, s->z, &perm))
        return QZ_FAILURE;
    const double H = 1.0 / (1 << L);
    const double coeff = 4.0 * s->cfg.G * QZ_PI_D / (H * H * H);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    long want_warps = n; // upper bound on segments
    long blocks = (want_warps * 32 + 255) / 256;
    long max_blocks = (long)sms * 16;
    if (blocks > max_blocks)
        blocks = max_blocks;
    cudaMemsetAsync(s->flags + F_NLONG, 0, sizeof(int), s->stream);
    launch(s, QZ_PROF_DEPOSIT, 36.0 * n, k_seg_reduce, dim3((int)blocks), dim3(256), L, coeff, perm,
           s->seg_start, s->flags, s->long_seg, s->x, s->y, s->z, s->m, s->cell_sums);
    launch(s, QZ_PROF_DEPOSIT, 0.0, k_seg_long, dim3(sms), dim3(SEG_LONG_THREADS), L, coeff, perm,
           s->seg_start, s->flags, s->long_seg, s->x, s->y, s->z, s->m, s->cell_sums);
    launch(s, QZ_PROF_DEPOSIT, 12.0 * s->gpts, k_point_gather, dim3(blocks_for(s->gpts, 256)), dim3(256), L, s->D, s->cell_seg, s->cell_sums, s->d);
    return check_cuda(cudaGetLastError(), "deposit") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- grid acceleration (3-point) ----------------------------------------------
// a = -grad phi on the head interior.  stencil 0: 3-point
// (grid_acceleration.c:36-76).  stencil 1 (grid_acceleration.c:78-197): the
// 5-point difference along an axis whose cells at -2 and +1 are inside the
// simulation (head box coordinates 3..2^L-1), else the 3-point one.
// Periodic boundaries with stencil 1 (grid_acceleration.c:139-145, 159-165,
// 179-185): where the 5-point condition fails (box coordinate 2 or 2^L) the
// 5-point difference still applies, the -2 neighbour taken 2^L further at
// coordinate 2 and the +2 neighbour 2^L back at coordinate 2^L.
__device__ __forceinline__ double grad5_periodic(const double *__restrict__ pot, long g, long st,
                                                 int c, int nc, double t3h, double o12h)
{
    long n7 = g + 2 * st, n8 = g - 2 * st;
    if (c == 2)
        n8 += (long)nc * st;
    else
        n7 -= (long)nc * st;
    return (pot[g - st] - pot[g + st]) * t3h - (pot[n8] - pot[n7]) * o12h;
}

__global__ void k_grid_accel_head(int L, long D, int stencil, int periodic,
                                  const double *__restrict__ pot, double *__restrict__ ax,
                                  double *__restrict__ ay, double *__restrict__ az)
{
    const int m = (1 << L) - 1; // interior points per axis: box coords 2..2^L
    // 32-bit index arithmetic (m^3 < 2^32 for every head grid this library builds)
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x, um = (unsigned)m;
    if (t >= um * um * um)
        return;
    const unsigned q = t / um, r = q / um;
    const int i = 2 + (int)(t - q * um), j = 2 + (int)(q - r * um), k = 2 + (int)r;
    const long D2 = D * D;
    long g = i + j * D + k * D2;
    const double H = 1.0 / (1 << L);
    const double o2h = 1.0 / (2.0 * H);
    if (stencil == 0)
    {
        ax[g] = o2h * (pot[g - 1] - pot[g + 1]);
        ay[g] = o2h * (pot[g - D] - pot[g + D]);
        az[g] = o2h * (pot[g - D2] - pot[g + D2]);
        return;
    }
    const double o12h = 1.0 / (12.0 * H);
    const double t3h = 2.0 / (3.0 * H);
    const int hi = (1 << L) - 1;
    const int nc = 1 << L;
    ax[g] = (i >= 3 && i <= hi)
                ? (pot[g - 1] - pot[g + 1]) * t3h - (pot[g - 2] - pot[g + 2]) * o12h
            : periodic ? grad5_periodic(pot, g, 1, i, nc, t3h, o12h)
                       : o2h * (pot[g - 1] - pot[g + 1]);
    ay[g] = (j >= 3 && j <= hi)
                ? (pot[g - D] - pot[g + D]) * t3h - (pot[g - 2 * D] - pot[g + 2 * D]) * o12h
            : periodic ? grad5_periodic(pot, g, D, j, nc, t3h, o12h)
                       : o2h * (pot[g - D] - pot[g + D]);
    az[g] = (k >= 3 && k <= hi)
                ? (pot[g - D2] - pot[g + D2]) * t3h - (pot[g - 2 * D2] - pot[g + 2 * D2]) * o12h
            : periodic ? grad5_periodic(pot, g, D2, k, nc, t3h, o12h)
                       : o2h * (pot[g - D2] - pot[g + D2]);
}

int grid_accel_head_from(qz_sim *s, const double *pot)
{
    long m = (1L << s->L) - 1;
    if (m <= 0)
        return QZ_SUCCESS;
    const double bytes = (s->cfg.force_stencil ? 56.0 : 32.0) * m * m * m;
    launch(s, QZ_PROF_GRADIENT, bytes, k_grid_accel_head, dim3(blocks_for(m * m * m, 256)), dim3(256),
           s->L, s->D, s->cfg.force_stencil, s->cfg.bdry == 0 ? 1 : 0, pot, s->gax, s->gay,
           s->gaz);
    return check_cuda(cudaGetLastError(), "grid accel") ? QZ_SUCCESS : QZ_FAILURE;
}

int grid_accel_head(qz_sim *s) { return grid_accel_head_from(s, s->pot); }

// ---- CIC gather ---------------------------------------------------------------
__global__ void k_gather_head(long n, int L, long D, const double *__restrict__ x,
                              const double *__restrict__ y, const double *__restrict__ z,
                              const double *__restrict__ gx, const double *__restrict__ gy,
                              const double *__restrict__ gz, double *__restrict__ pax,
                              double *__restrict__ pay, double *__restrict__ paz,
                              int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double scale = (double)(1 << L);
    double px = x[i] * scale, py = y[i] * scale, pz = z[i] * scale;
    int fx = (int)px, fy = (int)py, fz = (int)pz;
    if (!(px >= 0.0 && py >= 0.0 && pz >= 0.0) || fx > (1 << L) || fy > (1 << L) ||
        fz > (1 << L))
    {
        atomicOr(&flags[F_ERROR], E_PTCL_OUTSIDE);
        return;
    }
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
    const long D2 = D * D;
    long g = (fx + 1) + (long)(fy + 1) * D + (long)(fz + 1) * D2;
    double ax = pax[i], ay = pay[i], az = paz[i];
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
            {
                int a = ii + 2 * jj + 4 * kk;
                long q = g + ii + jj * D + kk * D2;
                ax += gx[q] * w[a];
                ay += gy[q] * w[a];
                az += gz[q] * w[a];
            }
    pax[i] = ax;
    pay[i] = ay;
    paz[i] = az;
}

int gather_head(qz_sim *s)
{
    if (s->n == 0)
        return QZ_SUCCESS;
    launch(s, QZ_PROF_GATHER, 72.0 * s->n + 24.0 * s->gpts, k_gather_head, dim3(blocks_for(s->n, 256)), dim3(256), s->n, s->L, s->D, s->x, s->y, s->z, s->gax, s->gay, s->gaz, s->ax, s->ay, s->az, s->flags);
    return check_cuda(cudaGetLastError(), "gather") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- leapfrog ---------------------------------------------------------------------
__device__ __forceinline__ void boundary(int bdry, double &x, double &v, double &a)
{
    if (x < 0.0 || x >= 1.0)
    {
        if (bdry == 0)
            x = x >= 1.0 ? x - 1.0 : 1.0 + x;
        else
        {
            x = x >= 1.0 ? 2.0 - x : -x;
            v *= -1.0;
            a *= -1.0;
        }
    }
}

__global__ void k_kick_drift(long n, double dt, int bdry, double *__restrict__ x,
                             double *__restrict__ y, double *__restrict__ z,
                             double *__restrict__ vx, double *__restrict__ vy,
                             double *__restrict__ vz, double *__restrict__ ax,
                             double *__restrict__ ay, double *__restrict__ az)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double px = x[i], py = y[i], pz = z[i];
    double qx = vx[i], qy = vy[i], qz = vz[i];
    double gx = ax[i], gy = ay[i], gz = az[i];
    qx += gx * dt * 0.5;
    qy += gy * dt * 0.5;
    qz += gz * dt * 0.5;
    px += qx * dt;
    py += qy * dt;
    pz += qz * dt;
    boundary(bdry, px, qx, gx);
    boundary(bdry, py, qy, gy);
    boundary(bdry, pz, qz, gz);
    x[i] = px;
    y[i] = py;
    z[i] = pz;
    vx[i] = qx;
    vy[i] = qy;
    vz[i] = qz;
    ax[i] = gx;
    ay[i] = gy;
    az[i] = gz;
}

// ---- outflow boundaries (particle_updating.c:123-196) ------------------------------
// The reference advances particles in index order; one that leaves [0, 1) on any
// axis is removed: the head's mass drops by the mass at its slot, the count by
// one, the last particle's x, v, a move into the slot (masses stay in their
// slots) and the loop continues with the next index, so the moved particle is
// not advanced in this step.  In parallel: every particle is advanced into a
// copy and flagged; with E(i) the flagged particles before i, index i is
// visited while i + E(i) < n, the first k indices; the E(k) visited flagged
// slots each receive the un-advanced state of index n - 1 - E(i); the count
// becomes n - E(k).
__global__ void k_outflow_advance(long n, double dt, const double *__restrict__ x,
                                  const double *__restrict__ y, const double *__restrict__ z,
                                  const double *__restrict__ vx, const double *__restrict__ vy,
                                  const double *__restrict__ vz, const double *__restrict__ ax,
                                  const double *__restrict__ ay, const double *__restrict__ az,
                                  double *__restrict__ st, int *__restrict__ flag)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double qx = vx[i], qy = vy[i], qz = vz[i];
    qx += ax[i] * dt * 0.5;
    qy += ay[i] * dt * 0.5;
    qz += az[i] * dt * 0.5;
    double px = x[i], py = y[i], pz = z[i];
    px += qx * dt;
    py += qy * dt;
    pz += qz * dt;
    st[i] = px;
    st[n + i] = py;
    st[2 * n + i] = pz;
    st[3 * n + i] = qx;
    st[4 * n + i] = qy;
    st[5 * n + i] = qz;
    flag[i] = (px < 0.0 || px >= 1.0 || py < 0.0 || py >= 1.0 || pz < 0.0 || pz >= 1.0) ? 1 : 0;
}

// bound[0] = k (first i with i + E(i) >= n), bound[1] = E(k); E(n) = total.
__global__ void k_outflow_bound(long n, const int *__restrict__ flag, const int *__restrict__ E,
                                int *__restrict__ bound)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i > n)
        return;
    auto e_at = [&](long q) { return q < n ? (long)E[q] : (long)E[n - 1] + flag[n - 1]; };
    const bool here = i + e_at(i) >= n;
    const bool before = i > 0 && (i - 1) + e_at(i - 1) >= n;
    if (here && !before)
    {
        bound[0] = (int)i;
        bound[1] = (int)e_at(i);
    }
}

__global__ void k_outflow_apply(long n, const double *__restrict__ st, const int *__restrict__ flag,
                                const int *__restrict__ E, const int *__restrict__ bound,
                                double *__restrict__ x, double *__restrict__ y,
                                double *__restrict__ z, double *__restrict__ vx,
                                double *__restrict__ vy, double *__restrict__ vz,
                                double *__restrict__ ax, double *__restrict__ ay,
                                double *__restrict__ az, int *__restrict__ slots,
                                int *__restrict__ srcs)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long k = bound[0], nf = n - bound[1];
    if (i >= k)
        return;
    double *F[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    if (!flag[i])
    {
        // visited and kept: its advanced state (i < k <= n - E(k) + ... is a kept slot)
        for (int q = 0; q < 6; q++)
            F[q][i] = st[q * n + i];
        return;
    }
    const long r = E[i], src = n - 1 - r;
    slots[r] = (int)i;
    srcs[r] = (int)src;
    if (i < nf) // a slot beyond the new count only drops its particle
        for (int q = 0; q < 9; q++)
            F[q][i] = F[q][src];
}

// the head's mass minus the removed slots' masses, in visiting order
__global__ void k_outflow_mass(int removed, const int *__restrict__ slots,
                               const double *__restrict__ m, const double *__restrict__ mass_in,
                               double *__restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0)
        return;
    double hm = mass_in[0];
    for (int r = 0; r < removed; r++)
        hm -= m[slots[r]];
    out[0] = hm;
}

static int outflow_step(qz_sim *s, double dt)
{
    const long n = s->n;
    if (!s->ofl_state.ensure(s->mem, 9 * n) || !s->ofl_int.ensure(s->mem, 4 * n + 8))
    {
        set_error("outflow buffers");
        return QZ_FAILURE;
    }
    if (!s->h_ofl && !check_cuda(cudaMallocHost((void **)&s->h_ofl, 4 * sizeof(double)),
                                 "outflow pinned"))
        return QZ_FAILURE;
    int *flag = s->ofl_int.p, *E = flag + n, *slots = flag + 2 * n, *srcs = flag + 3 * n,
        *bound = flag + 4 * n;
    double *dmass = s->red + s->red_blocks + 4; // two scratch words after the partials
    launch(s, QZ_PROF_LEAPFROG, 148.0 * n, k_outflow_advance, dim3(blocks_for(n, 256)), dim3(256),
           n, dt, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->ofl_state.p, flag);
    if (scan_exclusive(s, flag, E, n))
        return QZ_FAILURE;
    launch(s, QZ_PROF_LEAPFROG, 8.0 * n, k_outflow_bound, dim3(blocks_for(n + 1, 256)), dim3(256),
           n, flag, E, bound);
    launch(s, QZ_PROF_LEAPFROG, 104.0 * n, k_outflow_apply, dim3(blocks_for(n, 256)), dim3(256), n,
           s->ofl_state.p, flag, E, bound, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay,
           s->az, slots, srcs);
    if (!check_cuda(cudaMemcpyAsync(s->h_ofl, bound, 2 * sizeof(int), cudaMemcpyDeviceToHost,
                                    s->stream), "outflow bound") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "outflow sync"))
        return QZ_FAILURE;
    int hb[2];
    memcpy(hb, s->h_ofl, sizeof hb);
    const long removed = hb[1];
    s->ofl_removed = removed;
    s->ofl_layout_n = n;
    if (removed > 0)
    {
        s->h_ofl[2] = s->head_mass;
        if (!check_cuda(cudaMemcpyAsync(dmass, &s->h_ofl[2], sizeof(double),
                                        cudaMemcpyHostToDevice, s->stream), "outflow mass"))
            return QZ_FAILURE;
        launch(s, QZ_PROF_LEAPFROG, 8.0 * removed, k_outflow_mass, dim3(1), dim3(32), (int)removed,
               slots, s->m, dmass, dmass + 1);
        if (!check_cuda(cudaMemcpyAsync(&s->h_ofl[3], dmass + 1, sizeof(double),
                                        cudaMemcpyDeviceToHost, s->stream), "outflow mass") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "outflow sync"))
            return QZ_FAILURE;
        s->head_mass = s->h_ofl[3];
        s->n = n - removed;
        // the captured check block holds the old mass in its thresholds
        if (s->check_exec)
        {
            cudaGraphExecDestroy(s->check_exec);
            s->check_exec = nullptr;
        }
    }
    if (s->n == 0)
    {
        set_error("there are no particles in the simulation (all left through the outflow "
                  "boundaries)");
        return QZ_FAILURE;
    }
    return check_cuda(cudaGetLastError(), "outflow") ? QZ_SUCCESS : QZ_FAILURE;
}

int kick_drift(qz_sim *s, double dt)
{
    if (s->n == 0)
        return QZ_SUCCESS;
    if (s->cfg.bdry == 2)
        return outflow_step(s, dt);
    launch(s, QZ_PROF_LEAPFROG, 144.0 * s->n, k_kick_drift, dim3(blocks_for(s->n, 256)), dim3(256), s->n, dt, s->cfg.bdry, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az);
    return check_cuda(cudaGetLastError(), "kick drift") ? QZ_SUCCESS : QZ_FAILURE;
}

__global__ void k_kick(long n, double dt, double *__restrict__ vx, double *__restrict__ vy,
                       double *__restrict__ vz, const double *__restrict__ ax,
                       const double *__restrict__ ay, const double *__restrict__ az)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    vx[i] += ax[i] * dt * 0.5;
    vy[i] += ay[i] * dt * 0.5;
    vz[i] += az[i] * dt * 0.5;
}

int kick(qz_sim *s, double dt)
{
    if (s->n == 0)
        return QZ_SUCCESS;
    launch(s, QZ_PROF_LEAPFROG, 72.0 * s->n, k_kick, dim3(blocks_for(s->n, 256)), dim3(256), s->n, dt, s->vx, s->vy, s->vz, s->ax, s->ay, s->az);
    return check_cuda(cudaGetLastError(), "kick") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- particle -> box index ----------------------------------------------------------
__global__ void k_box_idx(long n, int lv, int tsx, int tsy, int tsz, int dimx, int dimy,
                          const double *__restrict__ x, const double *__restrict__ y,
                          const double *__restrict__ z, int *__restrict__ out)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double scale = (double)(1 << lv);
    double px = x[i] * scale, py = y[i] * scale, pz = z[i] * scale;
    int fx = px < 0 ? -1 : (int)px;
    int fy = py < 0 ? -1 : (int)py;
    int fz = pz < 0 ? -1 : (int)pz;
    out[i] = (fx - tsx) + (fy - tsy) * dimx + (fz - tsz) * dimx * dimy;
}

void launch_box_idx(cudaStream_t st, long n, int lv, int tsx, int tsy, int tsz, int dimx,
                    int dimy, const double *x, const double *y, const double *z, int *out)
{
    k_box_idx<<<blocks_for(n, 256), 256, 0, st>>>(n, lv, tsx, tsy, tsz, dimx, dimy, x, y, z, out);
}

} // namespace qz

// qz_amr.cu -- the refinement tree and the per-level physics of refinement nodes.
//
// The tree is rebuilt on the device every step from the particle positions,
// level by level from the head, with the reference's construction rules
// (tree_construction.c:508-598, 685-926, 1032-2349):
//   counts     particles per node cell
//   flags      a cell holding >= ref_ptcl particles, and its 26 neighbours that
//              belong to the same node, become "refine" (-1)
//   zones      6-connected components of refine cells, numbered inside each node
//              by the position of their first cell in the node's cell order
//              (union-find that hooks the larger root under the smaller: every
//              component ends rooted at its first cell, whatever the order in
//              which the edges are processed)
//   children   one node per zone: smallest box = twice the zone's bounding box,
//              box padded by box_extra cells, cells = the 8 children of each
//              zone cell in zone-cell order, box statuses -4 / -3 / -5
//   grid       points classified interior / boundary / simulation boundary from
//              the statuses of their 8 surrounding cells, listed in box order
// The reference adapts the previous tree instead (tree_adaptation.c); on the
// workloads checked the adapted tree equals the constructed one.  Zones smaller
// than ref_ptcl particles (tree_construction.c:2350-2390) cannot occur with the
// particle criterion: every zone holds a cell with >= ref_ptcl particles.
//
// Physics per refinement level (levels after the head, in order):
//   deposit    grid_density.c:113-267 (weights in H units, 4 pi G / H^6)
//   potential  potential_branches.c:93-332 (parent interpolation, analytic
//              simulation boundary) and conjugate_gradient.c:322-463, with all
//              nodes of a level in the same launches (per-node scalars, per-node
//              convergence, fixed-order reductions)
//   gradient   grid_acceleration.c:199-394 (analytic simulation boundary with the
//              reference's y coordinate, boundary points from the parent's
//              accelerations, 3-point interior)
//   gather     particle_acceleration.c:134-355: every particle from the finest
//              node whose cell holding it is not refined
#include <algorithm>
#include <climits>
#include <mutex>
#include <cooperative_groups.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "qz_amr_dev.cuh"

namespace cgrp = cooperative_groups;

namespace qz {

#define QZ_PI_D 3.14159265358979323846
// largest block of the conjugate gradient kernel (two blocks per SM at 64 registers)
constexpr int CG_MAX_THREADS = 512;


__device__ __forceinline__ double block_sum_d(double v, double *sh)
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

// ---- tree: counts, flags, zones ------------------------------------------------------
__global__ void k_fill_int(long n, int *a, int v)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = v;
}

__global__ void k_count(long n, const int *__restrict__ node_of, const AmrNode *__restrict__ nodes,
                        const double *__restrict__ x, const double *__restrict__ y,
                        const double *__restrict__ z, int *__restrict__ cnt, int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int nd = node_of[i];
    if (nd < 0)
        return;
    const AmrNode N = nodes[nd];
    const double sc = (double)(1 << N.lv);
    int cx = (int)(x[i] * sc), cy = (int)(y[i] * sc), cz = (int)(z[i] * sc);
    long b = box_index(N, cx, cy, cz);
    if (b < 0 || b >= (long)N.rd[0] * N.rd[1] * N.rd[2])
    {
        atomicOr(&flags[F_ERROR], E_PTCL_OUTSIDE);
        return;
    }
    atomicAdd(&cnt[N.box_off + b], 1);
}

__global__ void k_flag(int ncell, int ref_ptcl, const int *__restrict__ cell_box,
                       const int *__restrict__ cell_node, const AmrNode *__restrict__ nodes,
                       const int *__restrict__ cnt, int *__restrict__ box)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    long b = cell_box[c];
    if (cnt[b] < ref_ptcl)
        return;
    const AmrNode N = nodes[cell_node[c]];
    const long sy = N.rd[0], sz = (long)N.rd[0] * N.rd[1];
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++)
            {
                long nb = b + dx + dy * sy + dz * sz;
                if (box[nb] == -3)
                    box[nb] = -1; // every writer stores the same value
            }
}

// Union-find over the refine cells (status -1) of a level, joined through face
// neighbours inside a node's box.  Every parent pointer refers to a smaller cell
// position or to the cell itself, so the root of a component is its first cell
// and zones come out numbered in the order of their first cell, as the
// reference numbers them.  The start points every cell at its smallest refine
// face neighbour, which leaves short trees for the hooking pass.
__global__ void k_cc_init(int ncell, const int *__restrict__ cell_box,
                          const int *__restrict__ cell_node, const AmrNode *__restrict__ nodes,
                          const int *__restrict__ box, const int *__restrict__ pos_of_box,
                          int *__restrict__ parent)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    const long b = cell_box[c];
    if (box[b] != -1)
    {
        parent[c] = -1;
        return;
    }
    const AmrNode N = nodes[cell_node[c]];
    const long sy = N.rd[0], sz = (long)N.rd[0] * N.rd[1];
    const long off[6] = {1, -1, sy, -sy, sz, -sz};
    int m = c;
    for (int e = 0; e < 6; e++)
    {
        const long nb = b + off[e];
        if (box[nb] != -1)
            continue;
        const int q = pos_of_box[nb];
        if (q >= 0 && q < m)
            m = q;
    }
    parent[c] = m;
}

// Root of x, pointing every visited cell at its grandparent on the way (path
// splitting).  Loads bypass L1: parents change under concurrent hooking.  Only
// non-roots are rewritten, always to an ancestor, so the races are benign.
__device__ __forceinline__ int cc_find(int *parent, int x)
{
    int p = __ldcg(&parent[x]);
    for (int guard = 0; p != x && guard < (1 << 20); guard++)
    {
        const int gp = __ldcg(&parent[p]);
        if (gp != p)
            __stcg(&parent[x], gp);
        x = p;
        p = gp;
    }
    return x;
}

// Joins each refine cell with its +x, +y and +z refine neighbours (every face
// once): the larger root is hooked under the smaller one by compare-and-swap.
__global__ void k_cc_hook(int ncell, const int *__restrict__ cell_box,
                          const int *__restrict__ cell_node, const AmrNode *__restrict__ nodes,
                          const int *__restrict__ box, const int *__restrict__ pos_of_box,
                          int *parent, int *__restrict__ flags)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell || __ldcg(&parent[c]) < 0)
        return;
    const AmrNode N = nodes[cell_node[c]];
    const long b = cell_box[c];
    const long off[3] = {1, N.rd[0], (long)N.rd[0] * N.rd[1]};
    for (int e = 0; e < 3; e++)
    {
        const long nb = b + off[e];
        if (box[nb] != -1)
            continue;
        const int q = pos_of_box[nb];
        if (q < 0)
            continue;
        int ra = cc_find(parent, c), rb = cc_find(parent, q);
        int guard = 0;
        for (; guard < (1 << 10) && ra != rb; guard++)
        {
            if (ra < rb)
            {
                const int t = ra;
                ra = rb;
                rb = t;
            }
            const int old = atomicCAS(&parent[ra], ra, rb);
            if (old == ra)
                break;
            ra = cc_find(parent, old);
            rb = cc_find(parent, rb);
        }
        if (guard >= (1 << 10))
            atomicOr(&flags[F_ERROR], 4);
    }
}

// Every refine cell points at its root.
__global__ void k_cc_compress(int ncell, int *parent)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell || __ldcg(&parent[c]) < 0)
        return;
    const int r = cc_find(parent, c);
    __stcg(&parent[c], r);
}

__global__ void k_cc_roots(int ncell, const int *__restrict__ parent, int *__restrict__ is_root,
                           int *__restrict__ flagged)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    is_root[c] = parent[c] == c ? 1 : 0;
    flagged[c] = parent[c] >= 0 ? 1 : 0;
}

__global__ void k_gather_at(int m, const int *__restrict__ src, const int *__restrict__ idx,
                            int *__restrict__ out)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m)
        out[i] = src[idx[i]];
}

__global__ void k_zone_box_init(int nz, int *zone_box, int *zone_cells)
{
    int z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= nz)
        return;
    for (int q = 0; q < 3; q++)
    {
        zone_box[6 * z + q] = INT_MAX;
        zone_box[6 * z + 3 + q] = INT_MIN;
    }
    zone_cells[z] = 0;
}

// Zone ids: zrank (exclusive scan of roots over the level's cells) is the
// child index of each root in the next level; inside a node the zone id is
// the rank minus the node's first rank.  Statuses of refine cells become zone
// ids, and refine cells are written in cell order to (zone, cell) pairs.
__global__ void k_cc_label(int ncell, const int *__restrict__ cell_box,
                           const int *__restrict__ cell_node, const AmrNode *__restrict__ nodes,
                           const int *__restrict__ parent, const int *__restrict__ zrank,
                           const int *__restrict__ slot, int *__restrict__ box,
                           int *__restrict__ zone_box, int *__restrict__ zone_cells,
                           const int *__restrict__ cell_xyz, unsigned *__restrict__ key,
                           int *__restrict__ val)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    const int r = parent[c]; // the root (parents are compressed)
    const int zg = r >= 0 ? zrank[r] : -1;
    // lanes of one zone add their bounds and count once (a zone spans many cells)
    const unsigned grp = __match_any_sync(__activemask(), zg);
    if (r < 0)
        return;
    const int x = cell_xyz[3 * c + 0], y = cell_xyz[3 * c + 1], z = cell_xyz[3 * c + 2];
    const int x0 = __reduce_min_sync(grp, x), y0 = __reduce_min_sync(grp, y),
              z0 = __reduce_min_sync(grp, z);
    const int x1 = __reduce_max_sync(grp, x), y1 = __reduce_max_sync(grp, y),
              z1 = __reduce_max_sync(grp, z);
    if ((int)(threadIdx.x & 31) == __ffs(grp) - 1)
    {
        atomicMin(&zone_box[6 * zg + 0], x0);
        atomicMin(&zone_box[6 * zg + 1], y0);
        atomicMin(&zone_box[6 * zg + 2], z0);
        atomicMax(&zone_box[6 * zg + 3], x1);
        atomicMax(&zone_box[6 * zg + 4], y1);
        atomicMax(&zone_box[6 * zg + 5], z1);
        atomicAdd(&zone_cells[zg], __popc(grp));
    }
    const AmrNode N = nodes[cell_node[c]];
    box[cell_box[c]] = zg - N.zone_base;
    key[slot[c]] = (unsigned)zg;
    val[slot[c]] = c;
}

__global__ void k_set_zone_base(int nn, AmrNode *nodes, const int *__restrict__ zrank, int nz)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nn)
        return;
    int b = zrank[nodes[q].cell_off];
    int e = q + 1 < nn ? zrank[nodes[q + 1].cell_off] : nz;
    nodes[q].zone_base = b;
    nodes[q].nzones = e - b;
}

// Children: the j-th cell of zone z (cell order) spawns child cells
// 8 j + (ii + 2 jj + 4 kk) of child node z (tree_construction.c:1634-1671).
__global__ void k_child_cells(int nzc, const unsigned *__restrict__ zkey,
                              const int *__restrict__ zval, const int *__restrict__ zone_start,
                              const int *__restrict__ pcell_xyz, const AmrNode *__restrict__ cn,
                              int *__restrict__ cell_box, int *__restrict__ cell_xyz,
                              int *__restrict__ cell_node)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nzc)
        return;
    int z = (int)zkey[q];
    int pc = zval[q];
    int j = q - zone_start[z];
    const AmrNode N = cn[z];
    int px = 2 * pcell_xyz[3 * pc], py = 2 * pcell_xyz[3 * pc + 1], pz = 2 * pcell_xyz[3 * pc + 2];
    for (int sub = 0; sub < 8; sub++)
    {
        int ii = sub & 1, jj = (sub >> 1) & 1, kk = sub >> 2;
        int c = N.cell_off + 8 * j + sub;
        int cx = px + ii, cy = py + jj, cz = pz + kk;
        cell_xyz[3 * c] = cx;
        cell_xyz[3 * c + 1] = cy;
        cell_xyz[3 * c + 2] = cz;
        cell_box[c] = (int)(N.box_off + box_index(N, cx, cy, cz));
        cell_node[c] = z;
    }
}

__global__ void k_box_cells(int ncell, const int *__restrict__ cell_box, int *__restrict__ box,
                            int *__restrict__ pos_of_box)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncell)
        return;
    box[cell_box[c]] = -3;
    pos_of_box[cell_box[c]] = c;
}

// Cells beyond the simulation box of a node that touches it (tree_construction.c:1745-1841).
__global__ void k_box_simb(long total, int nn, const AmrNode *__restrict__ nodes,
                           int *__restrict__ box)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total)
        return;
    const AmrNode N = nodes[find_node(nodes, nn, t, 2)];
    if (!N.contact)
        return;
    long l = t - N.box_off;
    int i = (int)(l % N.rd[0]), j = (int)((l / N.rd[0]) % N.rd[1]),
        k = (int)(l / ((long)N.rd[0] * N.rd[1]));
    const int top = 1 << N.lv;
    const int g[3] = {i + N.ts[0], j + N.ts[1], k + N.ts[2]};
    bool outside = false;
    for (int a = 0; a < 3; a++)
    {
        if (N.bmin[a] == 0 && g[a] < 0)
            outside = true;
        if (N.bmax[a] == top - 1 && g[a] >= top)
            outside = true;
    }
    if (outside)
        box[t] = -5;
}

// Grid-point category from the 8 cells around the point (tree_construction.c:1935-2107):
// 0 none, 1 interior, 2 boundary, 3 simulation boundary.
__device__ __forceinline__ int classify_point(const int *box, long b, long sy, long sz, int gx,
                                              int gy, int gz, int top, int contact)
{
    auto in = [&](long off) { return box[b + off] > -4; };
    const bool c000 = in(0), c100 = in(-1), c010 = in(-sy), c110 = in(-1 - sy), c001 = in(-sz),
               c101 = in(-1 - sz), c011 = in(-sy - sz), c111 = in(-1 - sy - sz);
    bool bder = false;
    if (c000)
        bder = (!c100 && !c110 && !c101 && !c111) || (!c010 && !c110 && !c011 && !c111) ||
               (!c001 && !c101 && !c011 && !c111);
    else if (c100)
        bder = (!c010 && !c001 && !c011) || (!c010 && !c110 && !c011 && !c111) ||
               (!c001 && !c101 && !c011 && !c111);
    else if (c010)
        bder = (!c110 && !c101 && !c111) || (!c001 && !c101) || (!c001 && !c101 && !c011 && !c111);
    else if (c110)
        bder = (!c001 && !c011) || (!c001 && !c101) || (!c001 && !c101 && !c011 && !c111);
    else if (c001 || c101 || c011 || c111)
        bder = true;
    else
        return 0;
    if (contact && bder && (gx == 0 || gx == top || gy == 0 || gy == top || gz == 0 || gz == top))
        return 3;
    return bder ? 2 : 1;
}

// Per node, the box grid points [bmin - ts, bmax - ts + 1]^3 in box order; fl
// holds three flag arrays (interior | boundary | simulation boundary).
__global__ void k_classify(long total, int nn, const AmrNode *__restrict__ nodes,
                           const int *__restrict__ box, int *__restrict__ fl)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total)
        return;
    const AmrNode N = nodes[find_node(nodes, nn, t, 1)];
    const int ex = N.bmax[0] - N.bmin[0] + 2, ey = N.bmax[1] - N.bmin[1] + 2;
    long l = t - N.cls_off;
    int ii = N.bmin[0] - N.ts[0] + (int)(l % ex);
    int jj = N.bmin[1] - N.ts[1] + (int)((l / ex) % ey);
    int kk = N.bmin[2] - N.ts[2] + (int)(l / ((long)ex * ey));
    const long sy = N.rd[0], sz = (long)N.rd[0] * N.rd[1];
    long b = N.box_off + ii + jj * sy + kk * sz;
    int cat = classify_point(box, b, sy, sz, ii + N.ts[0], jj + N.ts[1], kk + N.ts[2], 1 << N.lv,
                             N.contact);
    fl[t] = cat == 1;
    fl[total + t] = cat == 2;
    fl[2 * total + t] = cat == 3;
}

__global__ void k_lists(long total, int nn, const AmrNode *__restrict__ nodes,
                        const int *__restrict__ fl, const int *__restrict__ pos, int base1,
                        int base2, int *__restrict__ intr, int *__restrict__ bdry,
                        int *__restrict__ simb, int *__restrict__ intr_node,
                        int *__restrict__ bdry_node, int *__restrict__ simb_node)
{
    long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= total)
        return;
    int cat = fl[t] ? 0 : fl[total + t] ? 1 : fl[2 * total + t] ? 2 : -1;
    if (cat < 0)
        return;
    int nd = find_node(nodes, nn, t, 1);
    const AmrNode N = nodes[nd];
    const int ex = N.bmax[0] - N.bmin[0] + 2, ey = N.bmax[1] - N.bmin[1] + 2;
    long l = t - N.cls_off;
    int ii = N.bmin[0] - N.ts[0] + (int)(l % ex);
    int jj = N.bmin[1] - N.ts[1] + (int)((l / ex) % ey);
    int kk = N.bmin[2] - N.ts[2] + (int)(l / ((long)ex * ey));
    int g = (int)grid_index(N, ii, jj, kk);
    int p = pos[cat * total + t];
    if (cat == 0)
    {
        intr[p] = g;
        intr_node[p] = nd;
    }
    else if (cat == 1)
    {
        bdry[p - base1] = g;
        bdry_node[p - base1] = nd;
    }
    else
    {
        simb[p - base2] = g;
        simb_node[p - base2] = nd;
    }
}

// Node of every particle one level down: the zone of its cell, if refined.
__global__ void k_next_node(long n, const int *__restrict__ node_of, const AmrNode *__restrict__ nodes,
                            const int *__restrict__ box, const double *__restrict__ x,
                            const double *__restrict__ y, const double *__restrict__ z,
                            int *__restrict__ next)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int nd = node_of[i];
    int out = -1;
    if (nd >= 0)
    {
        const AmrNode N = nodes[nd];
        const double sc = (double)(1 << N.lv);
        int cx = (int)(x[i] * sc), cy = (int)(y[i] * sc), cz = (int)(z[i] * sc);
        int st = box[N.box_off + box_index(N, cx, cy, cz)];
        if (st >= 0)
            out = N.zone_base + st;
    }
    next[i] = out;
}

// ---- host helpers ---------------------------------------------------------------------
static bool ensure_small(qz_sim *s, long need)
{
    if (need <= s->h_small_cap)
        return true;
    if (s->h_small)
        cudaFreeHost(s->h_small);
    s->h_small = nullptr;
    s->h_small_cap = 0;
    // freeing pinned memory waits for the device: grow rarely
    long nc = std::max(2 * need, 1L << 20);
    if (!check_cuda(cudaMallocHost((void **)&s->h_small, nc * sizeof(int)), "pinned small"))
        return false;
    s->h_small_cap = nc;
    return true;
}

// Stream-ordered read-back of `count` ints (synchronises).
static bool read_ints(qz_sim *s, const int *dsrc, long count, int *out)
{
    if (count <= 0)
        return true;
    if (!ensure_small(s, count))
        return false;
    if (!check_cuda(cudaMemcpyAsync(s->h_small, dsrc, count * sizeof(int), cudaMemcpyDeviceToHost,
                                    s->stream),
                    "read back") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "read back sync"))
        return false;
    memcpy(out, s->h_small, count * sizeof(int));
    return true;
}

// Reads src[idx[q]] for the host index list idx (one launch, one read-back).
static bool read_at(qz_sim *s, const int *dsrc, const std::vector<int> &idx, int *out)
{
    const int m = (int)idx.size();
    if (m == 0)
        return true;
    if (!s->gather_idx.ensure(s->mem, 2L * m) || !ensure_small(s, m))
    {
        set_error("gather buffer");
        return false;
    }
    memcpy(s->h_small, idx.data(), m * sizeof(int));
    if (!check_cuda(cudaMemcpyAsync(s->gather_idx.p, s->h_small, m * sizeof(int),
                                    cudaMemcpyHostToDevice, s->stream),
                    "gather h2d"))
        return false;
    launch(s, QZ_PROF_TREE, 12.0 * m, k_gather_at, dim3(blocks_for(m, 256)), dim3(256), m, dsrc,
           s->gather_idx.p, s->gather_idx.p + m);
    return read_ints(s, s->gather_idx.p + m, m, out);
}

static bool upload_nodes(qz_sim *s, AmrLevel &L)
{
    if (!L.nodes.ensure(s->mem, std::max(L.nnodes, 1)))
    {
        set_error("amr nodes");
        return false;
    }
    return L.nnodes == 0 ||
           check_cuda(cudaMemcpyAsync(L.nodes.p, L.h.data(), L.nnodes * sizeof(AmrNode),
                                      cudaMemcpyHostToDevice, s->stream),
                      "amr nodes h2d");
}

static void free_level(const MemCtx &m, AmrLevel &L)
{
    DBuf<int> *ib[] = {&L.box, &L.cnt, &L.pos_of_box, &L.cell_seg, &L.cell_box, &L.cell_xyz,
                       &L.cell_node, &L.intr, &L.bdry, &L.simb, &L.intr_node, &L.bdry_node,
                       &L.simb_node, &L.nint, &L.mass_range, &L.sor};
    for (auto *b : ib)
        b->release(m);
    DBuf<double> *db[] = {&L.gpot, &L.gpot_old, &L.gd, &L.gax, &L.gay, &L.gaz, &L.r, &L.p, &L.Ap,
                          &L.apv, &L.cg1, &L.chunk_part, &L.mass_part};
    for (auto *b : db)
        b->release(m);
    L.nodes.release(m);
    L.chunks.release(m);
    L.wpot.release(m);
    L.wnodes.release(m);
    L.wmask.release(m);
    L = AmrLevel();
}

void amr_free(qz_sim *s)
{
    for (auto &L : s->amr)
        free_level(s->mem, L);
    free_level(s->mem, s->head_cg);
    free_level(s->mem, s->node_cg);
    s->amr.clear();
    for (auto &b : s->node_of)
        b.release(s->mem);
    s->node_of.clear();
    s->amr_tmp.release(s->mem);
    s->amr_tmp2.release(s->mem);
    s->zone_box.release(s->mem);
    s->zone_cells.release(s->mem);
    s->gather_idx.release(s->mem);
    s->seg_mass.release(s->mem);
    if (s->h_small)
        cudaFreeHost(s->h_small);
    s->h_small = nullptr;
    s->h_small_cap = 0;
}

// Level 0: the head node over the head fields and the (2^L+2)^3 head box.
int amr_init(qz_sim *s)
{
    const int levels = s->cfg.lmax - s->cfg.lmin + 1;
    if (levels > AMR_MAX_LEVELS)
    {
        set_error("at most %d refinement levels", AMR_MAX_LEVELS - 1);
        return QZ_FAILURE;
    }
    s->amr.assign(levels, AmrLevel());
    s->node_of.assign(levels, DBuf<int>());
    for (int l = 0; l < levels; l++)
        if (!s->node_of[l].ensure(s->mem, s->cap))
        {
            set_error("node_of");
            return QZ_FAILURE;
        }
    AmrLevel &H = s->amr[0];
    const int L = s->L, nc = 1 << L, B = nc + 2;
    AmrNode h{};
    h.lv = L;
    h.parent = -1;
    for (int a = 0; a < 3; a++)
    {
        h.ts[a] = -1;
        h.rd[a] = B;
        h.bmin[a] = 0;
        h.bmax[a] = nc - 1;
    }
    h.ncells = nc * nc * nc;
    h.contact = 1;
    h.mass = s->cfg.total_mass;
    H.nnodes = 1;
    H.h.assign(1, h);
    H.box_total = (long)B * B * B;
    H.grid_total = s->gpts;
    H.cell_total = h.ncells;
    H.pot = s->pot;
    H.pot_old = s->pot_old;
    H.d = s->d;
    H.ax = s->gax;
    H.ay = s->gay;
    H.az = s->gaz;
    if (!upload_nodes(s, H) || !H.box.ensure(s->mem, H.box_total) || !H.cnt.ensure(s->mem, H.box_total) ||
        !H.pos_of_box.ensure(s->mem, H.box_total) || !H.cell_box.ensure(s->mem, H.cell_total) ||
        !H.cell_xyz.ensure(s->mem, 3L * H.cell_total) || !H.cell_node.ensure(s->mem, H.cell_total))
    {
        set_error("head tree buffers");
        return QZ_FAILURE;
    }
    // head cells in the reference's order (initialization.c:126-142): i fastest
    std::vector<int> cb(H.cell_total), cx(3L * H.cell_total), pb(H.box_total, -1);
    for (int k = 0; k < nc; k++)
        for (int j = 0; j < nc; j++)
            for (int i = 0; i < nc; i++)
            {
                int c = i + j * nc + k * nc * nc;
                int b = (i + 1) + (j + 1) * B + (k + 1) * B * B;
                cb[c] = b;
                cx[3 * c] = i;
                cx[3 * c + 1] = j;
                cx[3 * c + 2] = k;
                pb[b] = c;
            }
    bool ok = check_cuda(cudaMemcpy(H.cell_box.p, cb.data(), cb.size() * sizeof(int),
                                    cudaMemcpyHostToDevice), "head cells") &&
              check_cuda(cudaMemcpy(H.cell_xyz.p, cx.data(), cx.size() * sizeof(int),
                                    cudaMemcpyHostToDevice), "head cells") &&
              check_cuda(cudaMemcpy(H.pos_of_box.p, pb.data(), pb.size() * sizeof(int),
                                    cudaMemcpyHostToDevice), "head pos") &&
              check_cuda(cudaMemset(H.cell_node.p, 0, H.cell_total * sizeof(int)), "head cells") &&
              check_cuda(cudaDeviceSynchronize(), "head tree init");
    return ok ? QZ_SUCCESS : QZ_FAILURE;
}

bool ensure_sort(qz_sim *s, long need)
{
    Sort &S = s->sort;
    if (need <= S.cap)
        return true;
    long tiles = radix_tiles(need);
    void *ps[] = {S.k0, S.k1, S.v0, S.v1, S.hist};
    for (void *p : ps)
        if (p)
            cudaFree(p);
    S.k0 = S.k1 = nullptr;
    S.v0 = S.v1 = S.hist = nullptr;
    bool ok = check_cuda(cudaMalloc(&S.k0, need * sizeof(unsigned)), "sort") &&
              check_cuda(cudaMalloc(&S.k1, need * sizeof(unsigned)), "sort") &&
              check_cuda(cudaMalloc(&S.v0, need * sizeof(int)), "sort") &&
              check_cuda(cudaMalloc(&S.v1, need * sizeof(int)), "sort") &&
              check_cuda(cudaMalloc(&S.hist, 256L * std::max(tiles, 4L) * sizeof(int)), "sort");
    S.cap = ok ? need : 0;
    S.tiles_cap = ok ? tiles : 0;
    return ok;
}

// Rebuilds the tree below the head from the current positions.
// Frozen tree: the nodes stay; every particle's node on each level is found
// again from its position, level by level from the head, by the rule the
// construction uses (k_next_node).
int amr_reassign(qz_sim *s)
{
    const long n = s->n;
    cudaMemsetAsync(s->node_of[0].p, 0, (n > 0 ? n : 1) * sizeof(int), s->stream);
    for (int l = 0; l + 1 < s->amr_nlev; l++)
    {
        AmrLevel &P = s->amr[l];
        if (n > 0)
            launch(s, QZ_PROF_TREE, 36.0 * n, k_next_node, dim3(blocks_for(n, 256)), dim3(256), n,
                   s->node_of[l].p, P.nodes.p, P.box.p, s->x, s->y, s->z, s->node_of[l + 1].p);
    }
    return check_cuda(cudaGetLastError(), "amr reassign") ? QZ_SUCCESS : QZ_FAILURE;
}

int amr_build(qz_sim *s)
{
    const long n = s->n;
    const int levels = (int)s->amr.size();
    AmrLevel &H = s->amr[0];
    // head statuses (initialization.c:95-110): -5 on the ghost ring, -3 inside
    launch(s, QZ_PROF_TREE, 4.0 * H.box_total, k_fill_int, dim3(blocks_for(H.box_total, 256)),
           dim3(256), H.box_total, H.box.p, -5);
    launch(s, QZ_PROF_TREE, 8.0 * H.cell_total, k_box_cells, dim3(blocks_for(H.cell_total, 256)),
           dim3(256), H.cell_total, H.cell_box.p, H.box.p, H.pos_of_box.p);
    cudaMemsetAsync(s->node_of[0].p, 0, (n > 0 ? n : 1) * sizeof(int), s->stream);
    s->amr_nlev = 1;
    for (int l = 1; l < levels; l++)
        s->amr[l].nnodes = 0;
    for (int l = 0; l + 1 < levels; l++)
    {
        AmrLevel &P = s->amr[l];
        if (P.nnodes == 0)
            break;
        cudaMemsetAsync(P.cnt.p, 0, P.box_total * sizeof(int), s->stream);
        if (n > 0)
            launch(s, QZ_PROF_TREE, 28.0 * n, k_count, dim3(blocks_for(n, 256)), dim3(256), n,
                   s->node_of[l].p, P.nodes.p, s->x, s->y, s->z, P.cnt.p, s->flags);
        const int nc = P.cell_total;
        launch(s, QZ_PROF_TREE, 12.0 * nc, k_flag, dim3(blocks_for(nc, 256)), dim3(256), nc,
               s->cfg.ref_ptcl, P.cell_box.p, P.cell_node.p, P.nodes.p, P.cnt.p, P.box.p);
        // union-find over the refine cells: parent | is_root | zone rank | flagged | slot
        if (!s->amr_tmp.ensure(s->mem, 5L * nc + 8))
        {
            set_error("amr scratch");
            return QZ_FAILURE;
        }
        int *parent = s->amr_tmp.p, *isroot = parent + nc, *zrank = isroot + nc,
            *flagged = zrank + nc, *slot = flagged + nc;
        launch(s, QZ_PROF_TREE, 36.0 * nc, k_cc_init, dim3(blocks_for(nc, 256)), dim3(256), nc,
               P.cell_box.p, P.cell_node.p, P.nodes.p, P.box.p, P.pos_of_box.p, parent);
        launch(s, QZ_PROF_TREE, 32.0 * nc, k_cc_hook, dim3(blocks_for(nc, 256)), dim3(256), nc,
               P.cell_box.p, P.cell_node.p, P.nodes.p, P.box.p, P.pos_of_box.p, parent,
               s->flags);
        launch(s, QZ_PROF_TREE, 8.0 * nc, k_cc_compress, dim3(blocks_for(nc, 256)), dim3(256), nc,
               parent);
        launch(s, QZ_PROF_TREE, 12.0 * nc, k_cc_roots, dim3(blocks_for(nc, 256)), dim3(256), nc,
               parent, isroot, flagged);
        if (scan_exclusive(s, isroot, zrank, nc) || scan_exclusive(s, flagged, slot, nc))
            return QZ_FAILURE;
        // zones = last rank + last root flag; refine cells = last slot + last flag
        int t[4];
        if (!read_at(s, parent, {2 * nc + nc - 1, nc + nc - 1, 4 * nc + nc - 1, 3 * nc + nc - 1}, t))
            return QZ_FAILURE;
        const int nz = t[0] + t[1], nzc = t[2] + t[3];
        if (nz == 0)
        {
            for (auto &nd : P.h)
                nd.zone_base = nd.nzones = 0;
            upload_nodes(s, P);
            break;
        }
        if (!s->zone_box.ensure(s->mem, 6L * nz) || !s->zone_cells.ensure(s->mem, nz) || !ensure_sort(s, nzc))
        {
            set_error("zone buffers");
            return QZ_FAILURE;
        }
        launch(s, QZ_PROF_TREE, 4.0 * P.nnodes, k_set_zone_base, dim3(blocks_for(P.nnodes, 128)),
               dim3(128), P.nnodes, P.nodes.p, zrank, nz);
        launch(s, QZ_PROF_TREE, 28.0 * nz, k_zone_box_init, dim3(blocks_for(nz, 256)), dim3(256),
               nz, s->zone_box.p, s->zone_cells.p);
        launch(s, QZ_PROF_TREE, 48.0 * nc, k_cc_label, dim3(blocks_for(nc, 256)), dim3(256), nc,
               P.cell_box.p, P.cell_node.p, P.nodes.p, parent, zrank, slot, P.box.p,
               s->zone_box.p, s->zone_cells.p, P.cell_xyz.p, s->sort.k0, s->sort.v0);
        // zone cells in (zone, cell position) order: a stable sort on the zone id
        int zbits = 1;
        while ((1L << zbits) < nz)
            zbits++;
        unsigned *zk;
        int *zv;
        if (radix_sort_pairs(s, nzc, zbits, &zk, &zv))
            return QZ_FAILURE;
        std::vector<int> zbox(6L * nz), zcells(nz);
        std::vector<AmrNode> pnodes(P.nnodes);
        if (!read_ints(s, s->zone_box.p, 6L * nz, zbox.data()) ||
            !read_ints(s, s->zone_cells.p, nz, zcells.data()) ||
            !check_cuda(cudaMemcpyAsync(pnodes.data(), P.nodes.p, P.nnodes * sizeof(AmrNode),
                                        cudaMemcpyDeviceToHost, s->stream), "nodes d2h") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "nodes d2h sync"))
            return QZ_FAILURE;
        for (int q = 0; q < P.nnodes; q++)
        {
            P.h[q].zone_base = pnodes[q].zone_base;
            P.h[q].nzones = pnodes[q].nzones;
        }
        // ---- child level geometry (host) ---------------------------------------------
        AmrLevel &C = s->amr[l + 1];
        C.nnodes = nz;
        C.h.assign(nz, AmrNode());
        long box_total = 0, grid_total = 0, cls_total = 0;
        int cell_total = 0;
        const int clv = P.h[0].lv + 1;
        const int top = 1 << clv;
        std::vector<int> zstart(nz);
        for (int q = 0; q < P.nnodes; q++)
            for (int zz = 0; zz < P.h[q].nzones; zz++)
            {
                const int z = P.h[q].zone_base + zz;
                AmrNode &N = C.h[z];
                N.lv = clv;
                N.parent = q;
                for (int a = 0; a < 3; a++)
                {
                    N.bmin[a] = 2 * zbox[6 * z + a];
                    N.bmax[a] = 2 * zbox[6 * z + 3 + a] + 1;
                    const int dim = N.bmax[a] - N.bmin[a] + 1;
                    N.rd[a] = dim + s->cfg.box_extra;
                    N.ts[a] = N.bmin[a] - (N.rd[a] - dim) / 2;
                    if (N.bmin[a] == 0 || N.bmax[a] == top - 1)
                        N.contact = 1;
                }
                N.box_off = box_total;
                box_total += (long)N.rd[0] * N.rd[1] * N.rd[2];
                N.grid_off = grid_total;
                grid_total += (long)(N.rd[0] + 1) * (N.rd[1] + 1) * (N.rd[2] + 1);
                zstart[z] = cell_total / 8;
                N.cell_off = cell_total;
                N.ncells = 8 * zcells[z];
                cell_total += N.ncells;
                N.cls_off = cls_total;
                cls_total += (long)(N.bmax[0] - N.bmin[0] + 2) * (N.bmax[1] - N.bmin[1] + 2) *
                             (N.bmax[2] - N.bmin[2] + 2);
            }
        C.box_total = box_total;
        C.grid_total = grid_total;
        C.cell_total = cell_total;
        C.cls_total = cls_total;
        if (!C.box.ensure(s->mem, box_total) || !C.cnt.ensure(s->mem, box_total) ||
            !C.pos_of_box.ensure(s->mem, box_total) || !C.cell_box.ensure(s->mem, cell_total) ||
            !C.cell_xyz.ensure(s->mem, 3L * cell_total) || !C.cell_node.ensure(s->mem, cell_total) ||
            !s->amr_tmp2.ensure(s->mem, std::max((long)nz, 6L * cls_total + 8)))
        {
            set_error("child level buffers");
            return QZ_FAILURE;
        }
        if (!upload_nodes(s, C))
            return QZ_FAILURE;
        int *dzstart = s->amr_tmp2.p;
        if (!ensure_small(s, nz))
            return QZ_FAILURE;
        memcpy(s->h_small, zstart.data(), nz * sizeof(int));
        if (!check_cuda(cudaMemcpyAsync(dzstart, s->h_small, nz * sizeof(int),
                                        cudaMemcpyHostToDevice, s->stream),
                        "zone start") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "zone start sync"))
            return QZ_FAILURE;
        launch(s, QZ_PROF_TREE, 40.0 * nzc, k_child_cells, dim3(blocks_for(nzc, 256)), dim3(256),
               nzc, zk, zv, dzstart, P.cell_xyz.p, C.nodes.p, C.cell_box.p, C.cell_xyz.p,
               C.cell_node.p);
        launch(s, QZ_PROF_TREE, 4.0 * box_total, k_fill_int, dim3(blocks_for(box_total, 256)),
               dim3(256), box_total, C.box.p, -4);
        launch(s, QZ_PROF_TREE, 4.0 * box_total, k_fill_int, dim3(blocks_for(box_total, 256)),
               dim3(256), box_total, C.pos_of_box.p, -1);
        launch(s, QZ_PROF_TREE, 8.0 * cell_total, k_box_cells, dim3(blocks_for(cell_total, 256)),
               dim3(256), cell_total, C.cell_box.p, C.box.p, C.pos_of_box.p);
        launch(s, QZ_PROF_TREE, 4.0 * box_total, k_box_simb, dim3(blocks_for(box_total, 256)),
               dim3(256), box_total, C.nnodes, C.nodes.p, C.box.p);
        // grid-point lists
        int *fl = s->amr_tmp2.p, *pos = fl + 3 * cls_total;
        launch(s, QZ_PROF_TREE, 32.0 * cls_total, k_classify, dim3(blocks_for(cls_total, 256)),
               dim3(256), cls_total, C.nnodes, C.nodes.p, C.box.p, fl);
        if (scan_exclusive(s, fl, pos, 3 * cls_total))
            return QZ_FAILURE;
        // scan values at every node's range start in each category, and the totals
        std::vector<int> idx;
        for (int cat = 0; cat < 3; cat++)
            for (int q = 0; q < nz; q++)
                idx.push_back((int)(cat * cls_total + C.h[q].cls_off));
        idx.push_back((int)(3 * cls_total - 1));
        std::vector<int> sv(idx.size()), lastf(1);
        if (!read_at(s, pos, idx, sv.data()) || !read_at(s, fl, {(int)(3 * cls_total - 1)}, lastf.data()))
            return QZ_FAILURE;
        const int total_all = sv.back() + lastf[0];
        auto start = [&](int cat, int q) {
            if (q < nz)
                return sv[cat * nz + q];
            return cat < 2 ? sv[(cat + 1) * nz] : total_all;
        };
        C.intr_total = start(0, nz) - start(0, 0);
        C.bdry_total = start(1, nz) - start(1, 0);
        C.simb_total = start(2, nz) - start(2, 0);
        for (int q = 0; q < nz; q++)
        {
            AmrNode &N = C.h[q];
            N.intr_off = start(0, q) - start(0, 0);
            N.nintr = start(0, q + 1) - start(0, q);
            N.bdry_off = start(1, q) - start(1, 0);
            N.nbdry = start(1, q + 1) - start(1, q);
            N.simb_off = start(2, q) - start(2, 0);
            N.nsimb = start(2, q + 1) - start(2, q);
            N.zone_base = N.nzones = 0;
        }
        if (!C.intr.ensure(s->mem, C.intr_total) || !C.intr_node.ensure(s->mem, C.intr_total) ||
            !C.bdry.ensure(s->mem, C.bdry_total) || !C.bdry_node.ensure(s->mem, C.bdry_total) ||
            !C.simb.ensure(s->mem, C.simb_total) || !C.simb_node.ensure(s->mem, C.simb_total))
        {
            set_error("grid lists");
            return QZ_FAILURE;
        }
        launch(s, QZ_PROF_TREE, 24.0 * cls_total, k_lists, dim3(blocks_for(cls_total, 256)),
               dim3(256), cls_total, C.nnodes, C.nodes.p, fl, pos, start(1, 0), start(2, 0),
               C.intr.p, C.bdry.p, C.simb.p, C.intr_node.p, C.bdry_node.p, C.simb_node.p);
        if (!upload_nodes(s, C))
            return QZ_FAILURE;
        if (n > 0)
            launch(s, QZ_PROF_TREE, 36.0 * n, k_next_node, dim3(blocks_for(n, 256)), dim3(256), n,
                   s->node_of[l].p, P.nodes.p, P.box.p, s->x, s->y, s->z, s->node_of[l + 1].p);
        s->amr_nlev = l + 2;
        if (!check_cuda(cudaGetLastError(), "amr build"))
            return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}


// ---- deposit on refinement levels ------------------------------------------------------
__global__ void k_lvl_keys(long n, const int *__restrict__ node_of, const AmrNode *__restrict__ nodes,
                           const double *__restrict__ x, const double *__restrict__ y,
                           const double *__restrict__ z, const int *__restrict__ slot,
                           unsigned *__restrict__ keys, int *__restrict__ vals)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int nd = node_of[i];
    if (nd < 0)
        return;
    const AmrNode N = nodes[nd];
    const double sc = (double)(1 << N.lv);
    int cx = (int)(x[i] * sc), cy = (int)(y[i] * sc), cz = (int)(z[i] * sc);
    keys[slot[i]] = (unsigned)(N.box_off + box_index(N, cx, cy, cz));
    vals[slot[i]] = (int)i;
}

__global__ void k_in_level(long n, const int *__restrict__ node_of, int *__restrict__ flag)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        flag[i] = node_of[i] >= 0 ? 1 : 0;
}

// CIC corner sums with the branch weights (grid_density.c:166-245):
// w1 = x - H floor(x / H), w2 = H - w1, times 4 pi G m / H^6; plus the mass.
__device__ __forceinline__ void lvl_cic_add(int i, double H, double ooh, double coeff,
                                            const double *__restrict__ x,
                                            const double *__restrict__ y,
                                            const double *__restrict__ z,
                                            const double *__restrict__ m, double acc[9])
{
    int fx = (int)(x[i] * ooh), fy = (int)(y[i] * ooh), fz = (int)(z[i] * ooh);
    double wx1 = x[i] - H * fx, wy1 = y[i] - H * fy, wz1 = z[i] - H * fz;
    double wx2 = H - wx1, wy2 = H - wy1, wz2 = H - wz1;
    double cm = coeff * m[i];
    acc[0] += cm * (wx2 * wy2 * wz2);
    acc[1] += cm * (wx1 * wy2 * wz2);
    acc[2] += cm * (wx2 * wy1 * wz2);
    acc[3] += cm * (wx1 * wy1 * wz2);
    acc[4] += cm * (wx2 * wy2 * wz1);
    acc[5] += cm * (wx1 * wy2 * wz1);
    acc[6] += cm * (wx2 * wy1 * wz1);
    acc[7] += cm * (wx1 * wy1 * wz1);
    acc[8] += m[i];
}

// One warp per occupied cell of at most SEG_LONG particles (longer cells are
// listed for k_lvl_seg_long): the corner sums and the cell's mass.
__global__ void k_lvl_seg_reduce(int lv, double coeff, const int *__restrict__ perm,
                                 const int *__restrict__ seg_start, int *__restrict__ flags,
                                 int *__restrict__ long_list, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ m, double *__restrict__ cs,
                                 double *__restrict__ smass)
{
    const int lane = threadIdx.x & 31;
    const long warp0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long nwarps = ((long)gridDim.x * blockDim.x) >> 5;
    const int nseg = flags[F_NSEG];
    const double H = 1.0 / (1 << lv);
    const double ooh = (double)(1 << lv);
    // A warp takes four consecutive cells.  When each holds at most 8 particles,
    // lanes 8g..8g+7 sum cell g (one particle a lane): the xor tree over those 8
    // lanes is the tree the whole warp would apply to them (the other lanes hold
    // zeros, which add exactly), so the sums are bit for bit those of one warp a
    // cell.
    for (long s4 = warp0 * 4; s4 < nseg; s4 += nwarps * 4)
    {
        const int g = lane >> 3, gl = lane & 7;
        const long sgg = s4 + g;
        int bg = 0, eg = 0;
        if (sgg < nseg)
        {
            bg = seg_start[sgg];
            eg = seg_start[sgg + 1];
        }
        if (__all_sync(0xffffffffu, eg - bg <= 8))
        {
            double acc[9];
#pragma unroll
            for (int c = 0; c < 9; c++)
                acc[c] = 0.0;
            if (gl < eg - bg)
                lvl_cic_add(perm[bg + gl], H, ooh, coeff, x, y, z, m, acc);
#pragma unroll
            for (int c = 0; c < 9; c++)
            {
                double v = acc[c];
                for (int o = 4; o > 0; o >>= 1)
                    v += __shfl_xor_sync(0xffffffffu, v, o);
                acc[c] = v;
            }
            if (sgg < nseg)
            {
                double v = acc[0];
#pragma unroll
                for (int c = 1; c < 8; c++)
                    if (gl == c)
                        v = acc[c];
                cs[sgg * 8 + gl] = v;
                if (gl == 0)
                    smass[sgg] = acc[8];
            }
            continue;
        }
        // else pairs of cells of at most 16 particles, 16 lanes a cell (again the
        // warp's tree), and one warp a cell for the others
        for (int h = 0; h < 2; h++)
        {
            const long p0 = s4 + 2 * h;
            const int gh = lane >> 4, hl = lane & 15;
            const long sgp = p0 + gh;
            int bp = 0, ep = 0;
            if (sgp < nseg)
            {
                bp = seg_start[sgp];
                ep = seg_start[sgp + 1];
            }
            if (__all_sync(0xffffffffu, ep - bp <= 16))
            {
                double acc[9];
#pragma unroll
                for (int c = 0; c < 9; c++)
                    acc[c] = 0.0;
                if (hl < ep - bp)
                    lvl_cic_add(perm[bp + hl], H, ooh, coeff, x, y, z, m, acc);
#pragma unroll
                for (int c = 0; c < 9; c++)
                {
                    double v = acc[c];
                    for (int o = 8; o > 0; o >>= 1)
                        v += __shfl_xor_sync(0xffffffffu, v, o);
                    acc[c] = v;
                }
                if (sgp < nseg && hl < 8)
                {
                    double v = acc[0];
#pragma unroll
                    for (int c = 1; c < 8; c++)
                        if (hl == c)
                            v = acc[c];
                    cs[sgp * 8 + hl] = v;
                    if (hl == 0)
                        smass[sgp] = acc[8];
                }
                continue;
            }
            for (long sg = p0; sg < p0 + 2 && sg < nseg; sg++)
            {
                const int b = seg_start[sg], e = seg_start[sg + 1];
                if (e - b > SEG_LONG)
                {
                    if (lane == 0)
                        long_list[atomicAdd(&flags[F_NLONG], 1)] = (int)sg;
                    continue;
                }
                double acc[9];
#pragma unroll
                for (int c = 0; c < 9; c++)
                    acc[c] = 0.0;
                for (int q = b + lane; q < e; q += 32)
                    lvl_cic_add(perm[q], H, ooh, coeff, x, y, z, m, acc);
#pragma unroll
                for (int c = 0; c < 9; c++)
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
                if (lane == 0)
                    smass[sg] = acc[8];
            }
        }
    }
}

// One block per listed cell of more than SEG_LONG particles (as k_seg_long).
__global__ void __launch_bounds__(SEG_LONG_THREADS)
    k_lvl_seg_long(int lv, double coeff, const int *__restrict__ perm,
                   const int *__restrict__ seg_start, const int *__restrict__ flags,
                   const int *__restrict__ long_list, const double *__restrict__ x,
                   const double *__restrict__ y, const double *__restrict__ z,
                   const double *__restrict__ m, double *__restrict__ cs,
                   double *__restrict__ smass)
{
    __shared__ double shw[(SEG_LONG_THREADS / 32) * 9];
    const int nl = flags[F_NLONG];
    const double H = 1.0 / (1 << lv);
    const double ooh = (double)(1 << lv);
    const int bs = (int)blockDim.x;
    for (int li = blockIdx.x; li < nl; li += gridDim.x)
    {
        const int sg = long_list[li];
        const int b = seg_start[sg], e = seg_start[sg + 1];
        double acc[9];
#pragma unroll
        for (int c = 0; c < 9; c++)
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
                    lvl_cic_add(iq[u], H, ooh, coeff, x, y, z, m, acc);
        }
        seg_block_sums<9>(acc, shw);
        if (threadIdx.x < 8)
            cs[(long)sg * 8 + threadIdx.x] = acc[0];
        else if (threadIdx.x == 8)
            smass[sg] = acc[0];
        __syncthreads(); // shw is rewritten for the next cell
    }
}

__global__ void k_lvl_point_gather(long total, int nn, const AmrNode *__restrict__ nodes,
                                   const int *__restrict__ cell_seg, const double *__restrict__ cs,
                                   double *__restrict__ d)
{
    long g = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= total)
        return;
    const AmrNode N = nodes[find_node(nodes, nn, g, 0)];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    double acc = 0.0;
    for (int c = 0; c < 2; c++)
    {
        int cz = gz - 1 + c;
        if (cz < 0 || cz >= N.rd[2])
            continue;
        for (int b = 0; b < 2; b++)
        {
            int cy = gy - 1 + b;
            if (cy < 0 || cy >= N.rd[1])
                continue;
            for (int a = 0; a < 2; a++)
            {
                int cx = gx - 1 + a;
                if (cx < 0 || cx >= N.rd[0])
                    continue;
                int sg = cell_seg[N.box_off + cx + (long)cy * N.rd[0] + (long)cz * N.rd[0] * N.rd[1]];
                if (sg >= 0)
                    acc += cs[(long)sg * 8 + (1 - a) + 2 * (1 - b) + 4 * (1 - c)];
            }
        }
    }
    d[g] = acc;
}

// Node masses and particle counts from the cell segments (segments of a node
// are contiguous in key order).  Pass 1: block (node, j) adds the j-th of
// NM_PARTS equal slices of the node's segments; pass 2 adds the slices in order,
// so the sum does not depend on scheduling.
constexpr int NM_PARTS = 32;

__device__ __forceinline__ int seg_lower_bound(const int *seg_cell, int nseg, long key)
{
    int lo = 0, hi = nseg; // first segment with cell >= key
    while (lo < hi)
    {
        const int mid = (lo + hi) >> 1;
        if ((long)seg_cell[mid] < key)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

__global__ void k_node_mass_parts(int nn, const AmrNode *__restrict__ nodes,
                                  const int *__restrict__ seg_cell,
                                  const double *__restrict__ smass, const int *__restrict__ flags,
                                  double *__restrict__ part, int *__restrict__ range)
{
    __shared__ double sh[32];
    __shared__ int lo_hi[2];
    const int nd = blockIdx.x, j = blockIdx.y;
    const int nseg = flags[F_NSEG];
    if (threadIdx.x < 2)
    {
        const AmrNode N = nodes[nd];
        const long key = N.box_off + (threadIdx.x == 0 ? 0L : (long)N.rd[0] * N.rd[1] * N.rd[2]);
        lo_hi[threadIdx.x] = seg_lower_bound(seg_cell, nseg, key);
    }
    __syncthreads();
    const int lo = lo_hi[0], hi = lo_hi[1];
    const int len = (hi - lo + NM_PARTS - 1) / NM_PARTS;
    const int b = lo + j * len, e = min(hi, b + len);
    double acc = 0.0;
    for (int q = b + threadIdx.x; q < e; q += blockDim.x)
        acc += smass[q];
    const double tot = block_sum_d(acc, sh);
    if (threadIdx.x == 0)
    {
        part[nd * NM_PARTS + j] = tot;
        if (j == 0)
        {
            range[2 * nd] = lo;
            range[2 * nd + 1] = hi;
        }
    }
}

__global__ void k_node_mass(int nn, AmrNode *nodes, const int *__restrict__ seg_start,
                            const double *__restrict__ part, const int *__restrict__ range)
{
    const int nd = blockIdx.x * blockDim.x + threadIdx.x;
    if (nd >= nn)
        return;
    double tot = 0.0;
    for (int j = 0; j < NM_PARTS; j++)
        tot += part[nd * NM_PARTS + j];
    const int lo = range[2 * nd], hi = range[2 * nd + 1];
    nodes[nd].mass = tot;
    nodes[nd].nptcl = hi > lo ? seg_start[hi] - seg_start[lo] : 0;
}

int deposit_segments(qz_sim *s, long m, int bits, int *cell_seg, long ncells_box,
                     unsigned **ks_out, int **perm_out, unsigned morton_B); // qz_particles.cu

int amr_deposit(qz_sim *s)
{
    const long n = s->n;
    for (int l = 1; l < s->amr_nlev; l++)
    {
        AmrLevel &L = s->amr[l];
        if (L.nnodes == 0)
            break;
        if (!L.gd.ensure(s->mem, L.grid_total) || !L.cell_seg.ensure(s->mem, L.box_total) ||
            !s->amr_tmp.ensure(s->mem, 2 * n + 2) || !ensure_sort(s, n))
        {
            set_error("level deposit buffers");
            return QZ_FAILURE;
        }
        L.d = L.gd.p;
        int *flag = s->amr_tmp.p, *slot = flag + n;
        launch(s, QZ_PROF_DEPOSIT, 8.0 * n, k_in_level, dim3(blocks_for(n, 256)), dim3(256), n,
               s->node_of[l].p, flag);
        if (scan_exclusive(s, flag, slot, n))
            return QZ_FAILURE;
        int t[2];
        if (!read_at(s, s->amr_tmp.p, {(int)(2 * n - 1), (int)(n - 1)}, t))
            return QZ_FAILURE;
        const long m = t[0] + t[1];
        launch(s, QZ_PROF_DEPOSIT, 44.0 * n, k_lvl_keys, dim3(blocks_for(n, 256)), dim3(256), n,
               s->node_of[l].p, L.nodes.p, s->x, s->y, s->z, slot, s->sort.k0, s->sort.v0);
        int bits = 1;
        while ((1L << bits) < L.box_total)
            bits++;
        unsigned *ks;
        int *perm;
        if (deposit_segments(s, m, bits, L.cell_seg.p, L.box_total, &ks, &perm, 0u))
            return QZ_FAILURE;
        if (!s->seg_mass.ensure(s->mem, m + 1))
        {
            set_error("segment mass");
            return QZ_FAILURE;
        }
        const double H = 1.0 / (1 << L.h[0].lv);
        const double coeff = 4.0 * s->cfg.G * QZ_PI_D / (H * H * H * H * H * H);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
        long blocks = std::min((m * 32 + 255) / 256 + 1, (long)sms * 16);
        cudaMemsetAsync(s->flags + F_NLONG, 0, sizeof(int), s->stream);
        launch(s, QZ_PROF_DEPOSIT, 40.0 * m, k_lvl_seg_reduce, dim3((int)blocks), dim3(256),
               L.h[0].lv, coeff, perm, s->seg_start, s->flags, s->long_seg, s->x, s->y, s->z,
               s->m, s->cell_sums, s->seg_mass.p);
        launch(s, QZ_PROF_DEPOSIT, 0.0, k_lvl_seg_long, dim3(sms), dim3(SEG_LONG_THREADS),
               L.h[0].lv, coeff, perm, s->seg_start, s->flags, s->long_seg, s->x, s->y, s->z,
               s->m, s->cell_sums, s->seg_mass.p);
        launch(s, QZ_PROF_DEPOSIT, 12.0 * L.grid_total, k_lvl_point_gather,
               dim3(blocks_for(L.grid_total, 256)), dim3(256), L.grid_total, L.nnodes, L.nodes.p,
               L.cell_seg.p, s->cell_sums, L.d);
        if (!L.mass_part.ensure(s->mem, (long)NM_PARTS * L.nnodes) ||
            !L.mass_range.ensure(s->mem, 2L * L.nnodes))
        {
            set_error("node mass buffers");
            return QZ_FAILURE;
        }
        launch(s, QZ_PROF_DEPOSIT, 12.0 * m, k_node_mass_parts, dim3(L.nnodes, NM_PARTS), dim3(256),
               L.nnodes, L.nodes.p, s->seg_cell, s->seg_mass.p, s->flags, L.mass_part.p,
               L.mass_range.p);
        launch(s, QZ_PROF_DEPOSIT, 8.0 * NM_PARTS * L.nnodes, k_node_mass,
               dim3(blocks_for(L.nnodes, 128)), dim3(128), L.nnodes, L.nodes.p, s->seg_start,
               L.mass_part.p, L.mass_range.p);
        std::vector<AmrNode> tmp(L.nnodes);
        if (!check_cuda(cudaMemcpyAsync(tmp.data(), L.nodes.p, L.nnodes * sizeof(AmrNode),
                                        cudaMemcpyDeviceToHost, s->stream), "nodes d2h") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "nodes d2h sync"))
            return QZ_FAILURE;
        for (int q = 0; q < L.nnodes; q++)
        {
            L.h[q].mass = tmp[q].mass;
            L.h[q].nptcl = tmp[q].nptcl;
        }
        if (!check_cuda(cudaGetLastError(), "level deposit"))
            return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

// ---- potential on refinement levels -----------------------------------------------------
__global__ void k_pot_init(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                           const AmrNode *__restrict__ nodes, const AmrNode *__restrict__ pnodes,
                           const double *__restrict__ ppot, double *__restrict__ pot)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlist)
        return;
    const long g = list[e];
    const AmrNode N = nodes[lnode[e]];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    pot[g] = from_parent(pnodes[N.parent], ppot, gx + N.ts[0], gy + N.ts[1], gz + N.ts[2]);
}

// potential_branches.c:93-151: -G M / |r - 0.5|, with a coordinate on the box's
// faces (0 or 2^lv) taken as 0.
__global__ void k_pot_simb(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                           const AmrNode *__restrict__ nodes, double coeff, double *__restrict__ pot)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlist)
        return;
    const long g = list[e];
    const AmrNode N = nodes[lnode[e]];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const int top = 1 << N.lv;
    const double H = 1.0 / (1 << N.lv);
    const int cx = gx + N.ts[0], cy = gy + N.ts[1], cz = gz + N.ts[2];
    double ai = (cx == 0 || cx == top) ? 0.0 : cx * H;
    double aj = (cy == 0 || cy == top) ? 0.0 : cy * H;
    double ak = (cz == 0 || cz == top) ? 0.0 : cz * H;
    double dist = (ai - 0.5) * (ai - 0.5) + (aj - 0.5) * (aj - 0.5) + (ak - 0.5) * (ak - 0.5);
    dist = sqrt(dist);
    pot[g] = coeff / dist;
}

__global__ void k_copy_d(long n, const double *__restrict__ a, double *__restrict__ b)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        b[i] = a[i];
}

// The conjugate-gradient solves of all nodes of one level in one launch
// (conjugate_gradient.c:322-463 for every node at once).  Iteration k of a node
// has two phases:
//   P  (decision for the check at k-1, then) p_{k-1} = r_{k-1} + beta p_{k-2}
//      with beta = rs_{k-1} / rs_{k-2}, computed by every stencil on the fly for
//      its seven points (the owner stores it), Ap = -(1/H^2) L p_{k-1} and the
//      chunk's partial of p.Ap
//   U  alpha = rs_{k-1} / (p.Ap); pot += alpha p, r -= alpha Ap with Ap
//      recomputed from the stored p (the same expression, so the same value);
//      the chunk's partial of r.r; on check iterations the ratio test
//      (poisson_error.c:36-81) on the updated pot
// The residual test of a check iteration (poisson_error.c:236-254) is taken at
// the start of the next P phase: converged nodes stop there (the reference
// returns before updating p); the others copy pot to pot_old on their interior
// points, the only points the ratio test reads.  A node stops without
// converging after min(node grid points, max_iter) iterations, as there.
//
// Nodes are independent problems and there is no grid-wide barrier.  A chunk's
// partial is published with a release store into a slot that holds an all-ones
// word (a NaN payload that arithmetic never produces) until then; a block that
// needs the node's sum polls the node's slots with acquire loads until none
// holds the marker, which also makes the node's data of the previous phase
// visible.  Every block adds the same partials in the same fixed order, so all
// blocks of a node obtain the same sums and take the same decisions.  A slot is
// reset to the marker by its owner once the owner has seen every block of the
// node publish a later partial (so all of them have read it), before the owner
// publishes its own next partial.  p and the partials are double-buffered by
// iteration parity; r and both p buffers are zero off the interior points.
// Block b owns chunks b, b + gridDim, ... (its slots); their node constants and
// (up to ncache slots) grid indices sit in shared memory for the whole solve.
// All blocks are resident (cooperative launch); every wait gives up after a
// bounded number of polls and reports it in status[1].
struct CgArgs {
    const AmrChunk *chunks;
    int nchunks;
    int chunk;  // interior points per chunk
    int ncache; // slots per block whose grid indices are kept in shared memory
    const int *intr;
    const AmrNode *nodes;
    const int *node_chunk; // per node: first chunk, end chunk
    const double *d;
    double *pot, *pot_old, *r;
    double *pbuf[2]; // p_j in pbuf[j & 1]
    double *apv;     // Ap of the current iteration at the interior points
    double *pap[2];  // per chunk: partial p.Ap of iteration k in pap[k & 1]
    double *rr[2];   // per chunk: partial r_j.r_j in rr[j & 1]
    int *rfail[2];   // per node: ratio (or, check_method 1, residual) test failed at check j, in rfail[j & 1]
    int *status;     // [0] most iterations of a node, [1] a wait gave up, [2] unconverged nodes
    int *iters;      // per node: iterations run
    double tol, tol2, G;
    int every;
    int max_iter;
    int method; // check_method 0/1/2 of conj_grad_error (poisson_error.c:235-282)
    const double *thr_node; // per node r.r threshold in place of the mass-based one (or null)
    const int *cap_node;    // per node iteration count in place of the cap, with no
                            // convergence (a replayed schedule), or null
};

constexpr long long CG_EMPTY = -1LL; // all-ones word: partial not yet published
constexpr int CG_FILL = 148;         // chunks a level's CG points are cut into (B200's SMs)
// Interior points a thread in a chunk's update phase (chunks of up to CG_UPT x
// 512 points), with one block a SM and the registers of one (128 a thread).
// Measured on the 1M-particle sphere in one run (CG time a step): 2 points a
// thread and two blocks a SM 6.64 ms, 4 points and one block 6.33 ms.
constexpr int CG_UPT = 4;
// Partial-sum slots are 128 bytes apart (one L2 line each): every block of a
// node polls every slot of the node, so slots sharing lines would serialise the
// polls and the publications of many chunks on a few lines.
constexpr int CG_PS = 16;
constexpr int CG_POLL_LIMIT = 1 << 21;

__device__ __forceinline__ double cg_ld_acquire(const double *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double((long long)v);
}

__device__ __forceinline__ double cg_ld_relaxed(const double *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return __longlong_as_double((long long)v);
}

__device__ __forceinline__ void cg_st_relaxed(double *p, double v)
{
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p),
                 "l"((unsigned long long)__double_as_longlong(v))
                 : "memory");
}

__device__ __forceinline__ void cg_st_release(double *p, double v)
{
    asm volatile("st.release.gpu.global.b64 [%0], %1;" ::"l"(p),
                 "l"((unsigned long long)__double_as_longlong(v))
                 : "memory");
}

// Seven stencil operands of point g in the order of the Laplacian:
// g, g+1, g-1, g+sy, g-sy, g+sz, g-sz.
__device__ __forceinline__ void cg_load7(const double *v, int g, int sy, int sz, double o[7])
{
    o[0] = v[g];
    o[1] = v[g + 1];
    o[2] = v[g - 1];
    o[3] = v[g + sy];
    o[4] = v[g - sy];
    o[5] = v[g + sz];
    o[6] = v[g - sz];
}

// A block's view of one of its chunks (shared memory).
struct CgSlot {
    double oh2;     // 1 / H^2
    double thr;     // residual threshold of r.r: nintr (tol rm)^2, times cbrt(nintr)^2 for
                    // check_method 2 (poisson_error.c:236-282)
    double rm;      // 4 pi G rhomean of the node
    double rs_prev; // rs_{k-2} of the node
    double rs_cur;  // rs_{k-1} of the node
    int c, q, cb, ce; // chunk, node, node's chunk range
    int begin, n;     // interior list range of the chunk
    int sy, sz;       // grid strides of the node
    int cap;          // iteration cap of the node
    int done;         // node finished
};

// Block-wide sums of (a, b) and bitwise OR of f, returned to every thread.  Warp
// order and shuffle order are fixed, so every block of the launch (all of the
// same size) obtains the same values from the same inputs.
__device__ __forceinline__ double2 cg_reduce(double a, double b, int &f, double2 *sh2, int *shf)
{
    for (int o = 16; o > 0; o >>= 1)
    {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    f = (int)__reduce_or_sync(0xffffffffu, (unsigned)f);
    if ((threadIdx.x & 31) == 0)
    {
        sh2[threadIdx.x >> 5] = make_double2(a, b);
        shf[threadIdx.x >> 5] = f;
    }
    __syncthreads();
    double2 t = make_double2(0.0, 0.0);
    int any = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++)
    {
        t.x += sh2[w].x;
        t.y += sh2[w].y;
        any |= shf[w];
    }
    __syncthreads(); // the slots are rewritten by the next call
    f = any;
    return t;
}

// Sum of the published partials of chunks [cb, ce), waiting for each; thread t
// takes chunks cb + t, cb + t + blockDim, ...  ACQ: acquire loads (the partials
// also publish data), else relaxed.  *gave_up is set in every thread if a wait
// hit the poll limit.
template <bool ACQ>
__device__ __forceinline__ double cg_node_sum(const double *part, int cb, int ce, int *gave_up,
                                              double2 *sh2, int *shf)
{
    double s = 0.0;
    int bad = 0;
    for (int c = cb + (int)threadIdx.x; c < ce; c += (int)blockDim.x)
    {
        double v = ACQ ? cg_ld_acquire(&part[(long)c * CG_PS])
                       : cg_ld_relaxed(&part[(long)c * CG_PS]);
        int polls = 0;
        while (__double_as_longlong(v) == CG_EMPTY)
        {
            if (++polls > CG_POLL_LIMIT)
            {
                bad = 1;
                v = 0.0;
                break;
            }
            v = ACQ ? cg_ld_acquire(&part[(long)c * CG_PS])
                    : cg_ld_relaxed(&part[(long)c * CG_PS]);
        }
        s += v;
    }
    int f = bad;
    const double2 t = cg_reduce(s, 0.0, f, sh2, shf);
    *gave_up = f;
    return t.x;
}

__global__ void __launch_bounds__(CG_MAX_THREADS, 1) k_cg_nodes(CgArgs A)
{
    __shared__ double sh[32];
    __shared__ double2 sh2[CG_MAX_THREADS / 32];
    __shared__ int shf[CG_MAX_THREADS / 32];
    const int NT = blockDim.x;
    extern __shared__ __align__(16) unsigned char cg_dyn[];
    const double empty = __longlong_as_double(CG_EMPTY);
    // the host launches at most nchunks blocks: every block has at least one slot
    const int nslot = (A.nchunks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    CgSlot *slot = reinterpret_cast<CgSlot *>(cg_dyn);
    int *gidx = reinterpret_cast<int *>(slot + nslot);
    for (int s = threadIdx.x; s < nslot; s += NT)
    {
        const int c = blockIdx.x + s * gridDim.x;
        const AmrChunk C = A.chunks[c];
        const AmrNode N = A.nodes[C.node];
        CgSlot x;
        x.c = c;
        x.q = C.node;
        x.cb = A.node_chunk[2 * C.node];
        x.ce = A.node_chunk[2 * C.node + 1];
        x.begin = C.begin;
        x.n = C.end - C.begin;
        x.sy = N.rd[0] + 1;
        x.sz = x.sy * (N.rd[1] + 1);
        const double H = 1.0 / (1 << N.lv);
        x.oh2 = 1.0 / (H * H);
        const double rm = 4.0 * A.G * QZ_PI_D * N.mass / (N.ncells * H * H * H);
        const double tt = A.tol * rm;
        x.rm = rm;
        x.thr = N.nintr * tt * tt;
        if (A.method == 2)
            x.thr = x.thr * (cbrt((double)N.nintr) * cbrt((double)N.nintr));
        if (A.thr_node)
            x.thr = A.thr_node[C.node];
        const long size = (long)(N.rd[0] + 1) * (N.rd[1] + 1) * (N.rd[2] + 1);
        x.cap = (int)(size < A.max_iter ? size : A.max_iter);
        if (A.cap_node)
        {
            x.cap = A.cap_node[C.node];
            x.thr = -1.0; // r.r < -1 never holds: the node runs exactly cap iterations
        }
        x.rs_prev = x.rs_cur = 0.0;
        x.done = 0;
        slot[s] = x;
    }
    const int ncache = min(nslot, A.ncache);
    for (int s = 0; s < ncache; s++)
    {
        const AmrChunk C = A.chunks[blockIdx.x + s * gridDim.x];
        for (int e = threadIdx.x; e < C.end - C.begin; e += NT)
            gidx[s * A.chunk + e] = A.intr[C.begin + e];
    }
    __syncthreads();
    // grid index of entry e of slot s
    auto gi = [&](int s, int e) -> int {
        return s < ncache ? gidx[s * A.chunk + e] : A.intr[slot[s].begin + e];
    };
    // r_0 = d - (-(1/H^2) L pot), partial rs_0
    for (int s = 0; s < nslot; s++)
    {
        const CgSlot &x = slot[s];
        double acc = 0.0;
        for (int e = threadIdx.x; e < x.n; e += NT)
        {
            const int g = gi(s, e);
            const double *pt = A.pot;
            const double rv = A.d[g] + x.oh2 * (6.0 * pt[g] - pt[g + 1] - pt[g - 1] - pt[g + x.sy] -
                                                pt[g - x.sy] - pt[g + x.sz] - pt[g - x.sz]);
            A.r[g] = rv;
            acc += rv * rv;
        }
        const double t = block_sum_d(acc, sh);
        if (threadIdx.x == 0)
            cg_st_release(&A.rr[0][x.c * CG_PS], t);
    }
    int gave_up = 0;
    for (long k = 1;; k++)
    {
        // ---- P phase ----
        const bool decide = k > 1 && (k - 1) % A.every == 0;
        const double *pold = A.pbuf[k & 1];
        double *pnew = A.pbuf[(k - 1) & 1];
        int live = 0, cq = -1;
        double rs1 = 0.0;
        for (int s = 0; s < nslot && !gave_up; s++)
        {
            CgSlot &x = slot[s];
            if (x.done)
                continue;
            if (x.q != cq)
            {
                // rs_{k-1}; also makes the node's r of iteration k-1 visible
                rs1 = cg_node_sum<true>(A.rr[(k - 1) & 1], x.cb, x.ce, &gave_up, sh2, shf);
                cq = x.q;
                if (gave_up)
                    break;
            }
            // every block of the node has read the p.Ap partials of iteration k-1
            if (threadIdx.x == 0 && k > 1)
                A.pap[(k - 1) & 1][x.c * CG_PS] = empty;
            if (decide)
            {
                const int rf = __syncthreads_or(
                    threadIdx.x == 0 && __ldcg(&A.rfail[((k - 1) / A.every) & 1][x.q]));
                if (!rf && (A.method == 1 || rs1 < x.thr))
                {
                    if (threadIdx.x == 0)
                    {
                        x.done = 1;
                        if (x.c == x.cb) // once per node
                        {
                            A.iters[x.q] = (int)(k - 1);
                            atomicMax(&A.status[0], (int)(k - 1));
                            atomicSub(&A.status[2], 1);
                        }
                    }
                    continue;
                }
                for (int e = threadIdx.x; e < x.n; e += NT)
                {
                    const int g = gi(s, e);
                    A.pot_old[g] = A.pot[g];
                }
                // the ratio-test flags of the next check start clear
                if (threadIdx.x == 0 && x.c == x.cb)
                    A.rfail[((k - 1) / A.every + 1) & 1][x.q] = 0;
            }
            if (k > x.cap)
            {
                // the node used its iterations without converging
                if (threadIdx.x == 0)
                {
                    x.done = 1;
                    if (x.c == x.cb)
                    {
                        A.iters[x.q] = (int)(k - 1);
                        atomicMax(&A.status[0], (int)(k - 1));
                    }
                }
                continue;
            }
            live = 1;
            const double beta = k == 1 ? 0.0 : rs1 / x.rs_prev;
            const double oh2 = x.oh2;
            const int sy = x.sy, sz = x.sz;
            double acc = 0.0;
            // a thread's two points of a chunk together, so their loads overlap
            for (int e0 = threadIdx.x; e0 < x.n; e0 += 2 * NT)
            {
                const int e1 = e0 + NT;
                const bool has1 = e1 < x.n;
                const int ga = gi(s, e0), gb = has1 ? gi(s, e1) : ga;
                const double *r = A.r;
                double ra[7], pa[7], rb[7], pb[7];
                cg_load7(r, ga, sy, sz, ra);
                cg_load7(pold, ga, sy, sz, pa);
                cg_load7(r, gb, sy, sz, rb);
                cg_load7(pold, gb, sy, sz, pb);
                const double p0a = ra[0] + beta * pa[0];
                const double aa = -oh2 * (6.0 * p0a - (ra[1] + beta * pa[1]) - (ra[2] + beta * pa[2]) -
                                          (ra[3] + beta * pa[3]) - (ra[4] + beta * pa[4]) -
                                          (ra[5] + beta * pa[5]) - (ra[6] + beta * pa[6]));
                pnew[ga] = p0a;
                A.apv[ga] = aa;
                acc += p0a * aa;
                if (has1)
                {
                    const double p0b = rb[0] + beta * pb[0];
                    const double ab =
                        -oh2 * (6.0 * p0b - (rb[1] + beta * pb[1]) - (rb[2] + beta * pb[2]) -
                                (rb[3] + beta * pb[3]) - (rb[4] + beta * pb[4]) -
                                (rb[5] + beta * pb[5]) - (rb[6] + beta * pb[6]));
                    pnew[gb] = p0b;
                    A.apv[gb] = ab;
                    acc += p0b * ab;
                }
            }
            const double t = block_sum_d(acc, sh);
            if (threadIdx.x == 0)
            {
                x.rs_prev = rs1;
                x.rs_cur = rs1;
                // the U phase reads no other block's data of this phase: no fence
                cg_st_relaxed(&A.pap[k & 1][x.c * CG_PS], t);
            }
        }
        __syncthreads(); // slot flags written by thread 0 above
        if (gave_up || !live)
            break;
        // ---- U phase ----
        // Only this thread's own points are read (p_{k-1} and Ap stored by the P
        // phase, pot, r): their loads are issued before the wait for p.Ap.
        const bool check = k % A.every == 0;
        const bool res1 = A.method == 1; // per-point residual test joins the ratio test
        const double *pn = pnew;
        const double tm = 1.0 - A.tol2, tp = 1.0 + A.tol2;
        cq = -1;
        double pap = 0.0;
        for (int s = 0; s < nslot; s++)
        {
            CgSlot &x = slot[s];
            if (x.done)
                continue;
            // up to CG_UPT points a thread (chunks of up to CG_UPT x 512 points)
            int g[CG_UPT];
            bool h[CG_UPT];
            double apv[CG_UPT], pvv[CG_UPT], potv[CG_UPT], rvv[CG_UPT], oldv[CG_UPT];
#pragma unroll
            for (int u = 0; u < CG_UPT; u++)
            {
                const int e = threadIdx.x + u * NT;
                h[u] = e < x.n;
                g[u] = h[u] ? gi(s, e) : 0;
                apv[u] = pvv[u] = potv[u] = rvv[u] = 0.0;
                oldv[u] = 1.0;
                if (h[u])
                {
                    apv[u] = A.apv[g[u]];
                    pvv[u] = pn[g[u]];
                    potv[u] = A.pot[g[u]];
                    rvv[u] = A.r[g[u]];
                    if (check)
                        oldv[u] = A.pot_old[g[u]];
                }
            }
            if (x.q != cq)
            {
                pap = cg_node_sum<false>(A.pap[k & 1], x.cb, x.ce, &gave_up, sh2, shf);
                cq = x.q;
                if (gave_up)
                    break;
            }
            // every block of the node has read the r.r partials of iteration k-1
            if (threadIdx.x == 0)
                A.rr[(k - 1) & 1][x.c * CG_PS] = empty;
            const double alpha = x.rs_cur / pap;
            double acc = 0.0;
            int fail = 0;
#pragma unroll
            for (int u = 0; u < CG_UPT; u++)
                if (h[u])
                {
                    const double pv = potv[u] + alpha * pvv[u];
                    A.pot[g[u]] = pv;
                    const double rv = rvv[u] - alpha * apv[u];
                    A.r[g[u]] = rv;
                    acc += rv * rv;
                    if (check)
                    {
                        const double ratio = pv / oldv[u];
                        if ((tm > ratio) || (tp < ratio) || (res1 && fabs(rv) / x.rm >= A.tol))
                            fail = 1;
                    }
                }
            const double t = block_sum_d(acc, sh);
            fail = __syncthreads_or(fail);
            if (threadIdx.x == 0)
            {
                if (check && fail)
                    atomicOr(&A.rfail[(k / A.every) & 1][x.q], 1);
                // publishes this block's r and p of the iteration with the partial
                cg_st_release(&A.rr[k & 1][x.c * CG_PS], t);
            }
        }
        __syncthreads();
        if (gave_up)
            break;
    }
    if (gave_up && threadIdx.x == 0)
        atomicOr(&A.status[1], 1);
}

// ---- single-reduction conjugate gradient (cg_variant 1) ------------------------------
// The same iterates as the reference's conjugate_gradient (conjugate_gradient.c:
// 322-463) in exact arithmetic, in Chronopoulos and Gear's arrangement (1989):
// with w = A r and s = A p carried along, both dot products of an iteration,
// gamma = r.r and delta = w.r, come from one reduction:
//
//   beta_j  = gamma_j / gamma_{j-1}                      (beta_0 = 0)
//   alpha_j = gamma_j / (delta_j - beta_j gamma_j / alpha_{j-1})  (alpha_0 = gamma_0 / delta_0)
//   p_j = r_j + beta_j p_{j-1};  s_j = w_j + beta_j s_{j-1}
//   pot += alpha_j p_j;  r_{j+1} = r_j - alpha_j s_j;  w_{j+1} = A r_{j+1}
//
// so an iteration waits once for its node's partial sums instead of twice.
// w_{j+1} at a point needs r_{j+1} at its six neighbours; each thread recomputes
// those from the neighbours' r_j, w_j, s_{j-1} (the same expression, so the same
// bits as the neighbour's own thread), so no neighbour waits are needed.  r, w,
// s and p are double-buffered by iteration parity (a block overwrites a buffer
// only after every block of the node has published the iteration that read
// it); all four are zero off the interior points.  The partial sums are
// triple-buffered (iteration j in slot j mod 3): with one publication per
// iteration, the owner clears the slot of iteration j + 1 at the start of
// iteration j, after every block has read it (it held iteration j - 2), and a
// block reaches the wait on that slot only after seeing the owner's iteration j
// publication, which follows the clearing.  The convergence test of the reference after update j-1
// (gamma_j, and the ratio test of the new pot) is taken at the start of
// iteration j, before p_j, where the reference returns.  Rounding differs from
// the two-reduction order, so the iterates agree with the reference's to
// rounding, not bit for bit.
struct Cg1Args {
    const AmrChunk *chunks;
    int nchunks;
    int chunk;
    int ncache;
    const int *intr;
    const AmrNode *nodes;
    const int *node_chunk;
    const double *d;
    double *pot, *pot_old;
    double *rb[2], *wb[2], *sb[2], *pb[2]; // r_j in rb[j & 1], ...
    double *zv;                            // pipelined form: z = A s (rb[0], sb[0], pb[0] in place)
    double *pg[3], *pd[3];                 // per chunk: partial gamma, delta of j in [j % 3]
    int *rfail[2];
    int *status;
    int *iters;
    double tol, tol2, G;
    int every;
    int max_iter;
    int method;
};

struct Cg1Slot {
    double oh2, thr, rm;
    double g_prev, a_prev; // gamma_{j-1}, alpha_{j-1} of the node
    int c, q, cb, ce;
    int begin, n;
    int sy, sz;
    int cap;
    int done;
};

// r_{j+1} at point g from its r_j, w_j, s_{j-1} (zero off the interior)
__device__ __forceinline__ double cg1_rnext(const double *__restrict__ r,
                                            const double *__restrict__ w,
                                            const double *__restrict__ s, int g, double alpha,
                                            double beta)
{
    const double sv = w[g] + beta * s[g];
    return r[g] - alpha * sv;
}

// One point of an iteration, computed without stores: p_j, s_j, the new pot,
// r_{j+1} and w_{j+1} = A r_{j+1}.
struct Cg1Point {
    double p, s, x, r, w;
};

__device__ __forceinline__ Cg1Point cg1_point(const double *r, const double *w, const double *so,
                                              const double *po, const double *pot, int g, int sy,
                                              int sz, double alpha, double beta, double oh2)
{
    Cg1Point o;
    const double rg = r[g], wg = w[g];
    o.p = rg + beta * po[g];
    o.s = wg + beta * so[g];
    o.x = pot[g] + alpha * o.p;
    o.r = rg - alpha * o.s;
    const double r1 = cg1_rnext(r, w, so, g + 1, alpha, beta);
    const double r2 = cg1_rnext(r, w, so, g - 1, alpha, beta);
    const double r3 = cg1_rnext(r, w, so, g + sy, alpha, beta);
    const double r4 = cg1_rnext(r, w, so, g - sy, alpha, beta);
    const double r5 = cg1_rnext(r, w, so, g + sz, alpha, beta);
    const double r6 = cg1_rnext(r, w, so, g - sz, alpha, beta);
    o.w = -oh2 * (6.0 * o.r - r1 - r2 - r3 - r4 - r5 - r6);
    return o;
}

// Node sums of two published partials.  Both slots of a chunk are polled with
// relaxed loads in the same round trip; once both hold values, a gpu-scope
// fence makes the pair an acquire (the publisher's release of the gamma slot
// orders its data and its delta slot before it).
__device__ __forceinline__ double2 cg1_node_sum(const double *ga, const double *da, int cb, int ce,
                                                int *gave_up, double2 *sh2, int *shf)
{
    double sg = 0.0, sd = 0.0;
    int bad = 0, any = 0;
    for (int c = cb + (int)threadIdx.x; c < ce; c += (int)blockDim.x)
    {
        const long o = (long)c * CG_PS;
        double v = cg_ld_relaxed(&ga[o]), u = cg_ld_relaxed(&da[o]);
        int polls = 0;
        while (__double_as_longlong(v) == CG_EMPTY || __double_as_longlong(u) == CG_EMPTY)
        {
            if (++polls > CG_POLL_LIMIT)
            {
                bad = 1;
                v = u = 0.0;
                break;
            }
            v = cg_ld_relaxed(&ga[o]);
            u = cg_ld_relaxed(&da[o]);
        }
        sg += v;
        sd += u;
        any = 1;
    }
    if (any)
        asm volatile("fence.acq_rel.gpu;" ::: "memory");
    int f = bad;
    const double2 t = cg_reduce(sg, sd, f, sh2, shf);
    *gave_up = f;
    return t;
}

// ---- pipelined conjugate gradient (cg_variant 2) ----------------------------------------
// Ghysels and Vanroose's arrangement (2014) of the same iterates: besides
// w = A r and s = A p it carries z = A s, so that w_{j+1} = w_j - alpha_j z_j
// comes from a recurrence and the one stencil of an iteration is q_j = A w_j:
//
//   z_j = q_j + beta_j z_{j-1};  s_j = w_j + beta_j s_{j-1};  p_j = r_j + beta_j p_{j-1}
//   pot += alpha_j p_j;  r_{j+1} = r_j - alpha_j s_j;  w_{j+1} = w_j - alpha_j z_j
//
// with alpha and beta from gamma = r.r and delta = w.r as in the single-reduction
// form.  Only w is read at neighbouring points (double-buffered by parity); r,
// s, p and z are updated in place at the block's own points, so an iteration
// loads w at seven points and five vectors at one (12 loads, 6 stores a point)
// where the single-reduction form recomputes its neighbours' next residuals (23
// loads).  One wait a iteration, as there.  The recurrence for w lets the
// recursive residual drift from d - A pot by rounding; the convergence test
// reads the recursive gamma as the reference's reads its recursive rsnew.
// Points of one chunk a thread handles at once in the pipelined form (its chunks
// hold CG2_PPT x 512 points).  Measured on the 1M-particle sphere, 128^3 head,
// three levels (conjugate-gradient time a step): 2 points 7.09 ms, 4 points
// 7.01 ms, 8 points 12.0 ms; the two-phase form 7.02 ms.
constexpr int CG2_PPT = 4;
template <bool PIPE> __device__ __forceinline__ void cg1_solve(const Cg1Args &A);

__global__ void __launch_bounds__(CG_MAX_THREADS, 2) k_cg1_nodes(Cg1Args A)
{
    cg1_solve<false>(A);
}

// one block a SM: 128 registers for CG2_PPT points in flight without spills
__global__ void __launch_bounds__(CG_MAX_THREADS, 1) k_cg2_nodes(Cg1Args A)
{
    cg1_solve<true>(A);
}

template <bool PIPE> __device__ __forceinline__ void cg1_solve(const Cg1Args &A)
{
    __shared__ double2 sh2[CG_MAX_THREADS / 32];
    __shared__ int shf[CG_MAX_THREADS / 32];
    const int NT = blockDim.x;
    extern __shared__ __align__(16) unsigned char cg_dyn[];
    const double empty = __longlong_as_double(CG_EMPTY);
    const int nslot = (A.nchunks - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
    Cg1Slot *slot = reinterpret_cast<Cg1Slot *>(cg_dyn);
    int *gidx = reinterpret_cast<int *>(cg_dyn + nslot * sizeof(Cg1Slot));
    for (int s = threadIdx.x; s < nslot; s += NT)
    {
        const int c = blockIdx.x + s * gridDim.x;
        const AmrChunk C = A.chunks[c];
        const AmrNode N = A.nodes[C.node];
        Cg1Slot x;
        x.c = c;
        x.q = C.node;
        x.cb = A.node_chunk[2 * C.node];
        x.ce = A.node_chunk[2 * C.node + 1];
        x.begin = C.begin;
        x.n = C.end - C.begin;
        x.sy = N.rd[0] + 1;
        x.sz = x.sy * (N.rd[1] + 1);
        const double H = 1.0 / (1 << N.lv);
        x.oh2 = 1.0 / (H * H);
        const double rm = 4.0 * A.G * QZ_PI_D * N.mass / (N.ncells * H * H * H);
        const double tt = A.tol * rm;
        x.rm = rm;
        x.thr = N.nintr * tt * tt;
        if (A.method == 2)
            x.thr = x.thr * (cbrt((double)N.nintr) * cbrt((double)N.nintr));
        const long size = (long)(N.rd[0] + 1) * (N.rd[1] + 1) * (N.rd[2] + 1);
        x.cap = (int)(size < A.max_iter ? size : A.max_iter);
        x.g_prev = x.a_prev = 0.0;
        x.done = 0;
        slot[s] = x;
    }
    const int ncache = min(nslot, A.ncache);
    for (int s = 0; s < ncache; s++)
    {
        const AmrChunk C = A.chunks[blockIdx.x + s * gridDim.x];
        for (int e = threadIdx.x; e < C.end - C.begin; e += NT)
            gidx[s * A.chunk + e] = A.intr[C.begin + e];
    }
    __syncthreads();
    auto gi = [&](int s, int e) -> int {
        return s < ncache ? gidx[s * A.chunk + e] : A.intr[slot[s].begin + e];
    };
    int gave_up = 0;
    // ---- r_0 = d - A pot; partial gamma_0 into slot 2 (iteration -1) ----
    for (int s = 0; s < nslot; s++)
    {
        const Cg1Slot &x = slot[s];
        double acc = 0.0;
        for (int e = threadIdx.x; e < x.n; e += NT)
        {
            const int g = gi(s, e);
            const double *pt = A.pot;
            const double rv = A.d[g] + x.oh2 * (6.0 * pt[g] - pt[g + 1] - pt[g - 1] - pt[g + x.sy] -
                                                pt[g - x.sy] - pt[g + x.sz] - pt[g - x.sz]);
            A.rb[0][g] = rv;
            acc += rv * rv;
        }
        int f = 0;
        const double t = cg_reduce(acc, 0.0, f, sh2, shf).x;
        if (threadIdx.x == 0)
            cg_st_release(&A.pg[2][x.c * CG_PS], t);
    }
    // ---- w_0 = A r_0 once the node's r_0 is visible; partial delta_0 into slot 2 ----
    {
        int cq = -1;
        for (int s = 0; s < nslot && !gave_up; s++)
        {
            const Cg1Slot &x = slot[s];
            if (x.q != cq)
            {
                cg_node_sum<true>(A.pg[2], x.cb, x.ce, &gave_up, sh2, shf);
                cq = x.q;
                if (gave_up)
                    break;
            }
            const double *r = A.rb[0];
            double acc = 0.0;
            for (int e = threadIdx.x; e < x.n; e += NT)
            {
                const int g = gi(s, e);
                const double wv = -x.oh2 * (6.0 * r[g] - r[g + 1] - r[g - 1] - r[g + x.sy] -
                                            r[g - x.sy] - r[g + x.sz] - r[g - x.sz]);
                A.wb[0][g] = wv;
                acc += wv * r[g];
            }
            int f = 0;
            const double t = cg_reduce(acc, 0.0, f, sh2, shf).x;
            if (threadIdx.x == 0)
                cg_st_release(&A.pd[2][x.c * CG_PS], t); // also publishes w_0
        }
        __syncthreads();
    }
    for (long j = 0; !gave_up; j++)
    {
        // data buffers by parity; partial slots: this iteration's, the previous one's
        // (gamma_j, delta_j) and the next one's (cleared here)
        const int cur = (int)(j & 1), prv = cur ^ 1;
        const int scur = (int)(j % 3), sprv = (int)((j + 2) % 3), snxt = (int)((j + 1) % 3);
        const bool decide = j > 0 && j % A.every == 0;
        int live = 0, cq = -1;
        double2 gd = make_double2(0.0, 0.0);
        const bool check_next = (j + 1) % A.every == 0;
        const double tm = 1.0 - A.tol2, tp = 1.0 + A.tol2;
        for (int s = 0; s < nslot && !gave_up; s++)
        {
            Cg1Slot &x = slot[s];
            if (x.done)
                continue;
            if (x.q != cq)
            {
                gd = cg1_node_sum(A.pg[sprv], A.pd[sprv], x.cb, x.ce, &gave_up, sh2, shf);
                cq = x.q;
                if (gave_up)
                    break;
            }
            // every block of the node has read the partials of iteration j - 2: the
            // owner clears that slot, which iteration j + 1 publishes into
            if (threadIdx.x == 0)
            {
                cg_st_relaxed(&A.pd[snxt][x.c * CG_PS], empty);
                cg_st_relaxed(&A.pg[snxt][x.c * CG_PS], empty);
            }
            const double gamma = gd.x, delta = gd.y;
            if (decide)
            {
                const int rf = __syncthreads_or(
                    threadIdx.x == 0 && __ldcg(&A.rfail[(j / A.every) & 1][x.q]));
                if (!rf && (A.method == 1 || gamma < x.thr))
                {
                    if (threadIdx.x == 0)
                    {
                        x.done = 1;
                        if (x.c == x.cb)
                        {
                            A.iters[x.q] = (int)j;
                            atomicMax(&A.status[0], (int)j);
                            atomicSub(&A.status[2], 1);
                        }
                    }
                    continue;
                }
                for (int e = threadIdx.x; e < x.n; e += NT)
                {
                    const int g = gi(s, e);
                    A.pot_old[g] = A.pot[g];
                }
                if (threadIdx.x == 0 && x.c == x.cb)
                    A.rfail[(j / A.every + 1) & 1][x.q] = 0;
            }
            if (j >= x.cap)
            {
                if (threadIdx.x == 0)
                {
                    x.done = 1;
                    if (x.c == x.cb)
                    {
                        A.iters[x.q] = (int)j;
                        atomicMax(&A.status[0], (int)j);
                    }
                }
                continue;
            }
            live = 1;
            const double beta = j == 0 ? 0.0 : gamma / x.g_prev;
            const double alpha = j == 0 ? gamma / delta : gamma / (delta - beta * gamma / x.a_prev);
            const double oh2 = x.oh2;
            const int sy = x.sy, sz = x.sz;
            double ag = 0.0, ad = 0.0;
            int fail = 0;
            if constexpr (PIPE)
            {
                const double *w = A.wb[cur];
                double *wn = A.wb[prv], *r = A.rb[0], *sv = A.sb[0], *pv = A.pb[0], *zv = A.zv;
                // CG2_PPT points of a thread together: their loads are in flight at once
                for (int e0 = threadIdx.x; e0 < x.n; e0 += CG2_PPT * NT)
                {
                    int g[CG2_PPT];
                    double wc[CG2_PPT], q[CG2_PPT], rg[CG2_PPT], zo[CG2_PPT], so[CG2_PPT],
                        po[CG2_PPT], pt[CG2_PPT];
#pragma unroll
                    for (int u = 0; u < CG2_PPT; u++)
                    {
                        const int e = e0 + u * NT;
                        g[u] = e < x.n ? gi(s, e) : gi(s, e0);
                    }
#pragma unroll
                    for (int u = 0; u < CG2_PPT; u++)
                    {
                        const int gg = g[u];
                        wc[u] = w[gg];
                        q[u] = -oh2 * (6.0 * wc[u] - w[gg + 1] - w[gg - 1] - w[gg + sy] -
                                       w[gg - sy] - w[gg + sz] - w[gg - sz]);
                        rg[u] = r[gg];
                        zo[u] = j > 0 ? zv[gg] : 0.0;
                        so[u] = j > 0 ? sv[gg] : 0.0;
                        po[u] = j > 0 ? pv[gg] : 0.0;
                        pt[u] = A.pot[gg];
                    }
#pragma unroll
                    for (int u = 0; u < CG2_PPT; u++)
                    {
                        if (e0 + u * NT >= x.n)
                            break;
                        const int gg = g[u];
                        const double z = q[u] + beta * zo[u];
                        const double sn = wc[u] + beta * so[u];
                        const double p = rg[u] + beta * po[u];
                        const double xv = pt[u] + alpha * p;
                        const double rn = rg[u] - alpha * sn;
                        const double wv = wc[u] - alpha * z;
                        zv[gg] = z;
                        sv[gg] = sn;
                        pv[gg] = p;
                        A.pot[gg] = xv;
                        r[gg] = rn;
                        wn[gg] = wv;
                        ag += rn * rn;
                        ad += wv * rn;
                        if (check_next)
                        {
                            const double ratio = xv / A.pot_old[gg];
                            if ((tm > ratio) || (tp < ratio) ||
                                (A.method == 1 && fabs(rn) / x.rm >= A.tol))
                                fail = 1;
                        }
                    }
                }
            }
            const double *r = A.rb[cur], *w = A.wb[cur], *so = A.sb[prv], *po = A.pb[prv];
            double *rn = A.rb[prv], *wn = A.wb[prv], *sn = A.sb[cur], *pn = A.pb[cur];
            for (int e = threadIdx.x; !PIPE && e < x.n; e += NT)
            {
                const int g = gi(s, e);
                const Cg1Point a = cg1_point(r, w, so, po, A.pot, g, sy, sz, alpha, beta, oh2);
                pn[g] = a.p;
                sn[g] = a.s;
                A.pot[g] = a.x;
                rn[g] = a.r;
                wn[g] = a.w;
                ag += a.r * a.r;
                ad += a.w * a.r;
                if (check_next)
                {
                    const double ratio = a.x / A.pot_old[g];
                    if ((tm > ratio) || (tp < ratio) || (A.method == 1 && fabs(a.r) / x.rm >= A.tol))
                        fail = 1;
                }
            }
            const double2 t = cg_reduce(ag, ad, fail, sh2, shf);
            if (threadIdx.x == 0)
            {
                x.g_prev = gamma;
                x.a_prev = alpha;
                if (check_next && fail)
                    atomicOr(&A.rfail[((j + 1) / A.every) & 1][x.q], 1);
                cg_st_relaxed(&A.pd[scur][x.c * CG_PS], t.y);
                // publishes this block's r, w, s, p, pot of the iteration with gamma
                cg_st_release(&A.pg[scur][x.c * CG_PS], t.x);
            }
        }
        __syncthreads();
        if (gave_up || !live)
            break;
    }
    if (gave_up && threadIdx.x == 0)
        atomicOr(&A.status[1], 1);
}

// Red-black SOR on the nodes of a level with at most branch_cg_cells cells
// (potential_branches.c:35-91, 334-399, 471-512), one block per node: an
// iteration is `sweeps` red-black sweeps over the node's interior list (red:
// even sum of the level coordinates), every `every` iterations the test of
// poisson_error.c:290-347 (the ratio test, then the residual by
// check_method 0/1/2); a failed test copies pot to pot_old over the node grid.
// Reaching max_iter is a failure, as there.  The reference evaluates 1/6 in
// long double (1.0L / 6.0L) before rounding the update to double; here 1/6 is a
// double, so updates agree to rounding.
struct SorArgs {
    const int *sor_nodes; // node index of each block
    const AmrNode *nodes;
    const int *intr;
    const double *d;
    double *pot, *pot_old;
    int sweeps, every, max_iter, method;
    double w, tol, tol2, G;
    int *iters; // per block: iterations run; negative if not converged
};

__device__ __forceinline__ bool sor_red(const AmrNode &N, long g)
{
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    return (((gx + N.ts[0]) + (gy + N.ts[1]) + (gz + N.ts[2])) & 1) == 0;
}

__global__ void __launch_bounds__(256) k_sor_nodes(SorArgs A)
{
    __shared__ double sh[32];
    const int q = A.sor_nodes[blockIdx.x];
    const AmrNode N = A.nodes[q];
    const double H = 1.0 / (1 << N.lv);
    const double H2 = H * H, oh2 = 1.0 / (H * H);
    const long sy = N.rd[0] + 1, sz = sy * (N.rd[1] + 1);
    const long ngrid = sz * (N.rd[2] + 1);
    const double rm = 4.0 * A.G * QZ_PI_D * N.mass / (N.ncells * H * H * H);
    const double tm = 1.0 - A.tol2, tp = 1.0 + A.tol2;
    const double one_sixth = 1.0 / 6.0;
    const int *list = A.intr + N.intr_off;
    double *pot = A.pot;
    int iter = 0;
    bool check = false;
    while (iter < A.max_iter && !check)
    {
        iter++;
        for (int sw = 0; sw < A.sweeps; sw++)
            for (int color = 0; color < 2; color++)
            {
                for (int e = threadIdx.x; e < N.nintr; e += blockDim.x)
                {
                    const long g = list[e];
                    if (sor_red(N, g) != (color == 0))
                        continue;
                    double aux = one_sixth * (-H2 * A.d[g] + pot[g + 1] + pot[g - 1] + pot[g + sy] +
                                              pot[g - sy] + pot[g + sz] + pot[g - sz]);
                    pot[g] = A.w * aux + (1.0 - A.w) * pot[g];
                }
                __syncthreads();
            }
        if (iter % A.every == 0)
        {
            int ratio_fail = 0, resid_fail = 0;
            double acc = 0.0;
            for (int e = threadIdx.x; e < N.nintr; e += blockDim.x)
            {
                const long g = list[e];
                const double a = pot[g] / A.pot_old[g];
                if ((tm > a) || (tp < a))
                    ratio_fail = 1;
                const double diff = A.d[g] + oh2 * (6.0 * pot[g] - pot[g + 1] - pot[g - 1] -
                                                    pot[g + sy] - pot[g - sy] - pot[g + sz] -
                                                    pot[g - sz]);
                if (A.method == 1)
                {
                    if (fabs(diff) / rm >= A.tol)
                        resid_fail = 1;
                }
                else
                    acc += diff * diff;
            }
            ratio_fail = __syncthreads_or(ratio_fail);
            resid_fail = __syncthreads_or(resid_fail);
            const double tot = block_sum_d(acc, sh);
            int ok = 0;
            if (threadIdx.x == 0)
            {
                if (A.method == 1)
                    ok = !resid_fail;
                else
                {
                    double err = sqrt(tot / N.nintr) / rm;
                    if (A.method == 2)
                        err = err / (cbrt((double)N.nintr) * cbrt((double)N.nintr));
                    ok = err < A.tol;
                }
                ok = ok && !ratio_fail;
            }
            check = __syncthreads_or(ok) != 0;
            if (!check)
            {
                for (long t = threadIdx.x; t < ngrid; t += blockDim.x)
                    A.pot_old[N.grid_off + t] = pot[N.grid_off + t];
                __syncthreads();
            }
        }
    }
    if (threadIdx.x == 0)
        A.iters[blockIdx.x] = (check && iter < A.max_iter) ? iter : -iter;
}

static int sor_level(qz_sim *s, AmrLevel &L, int level_index, const std::vector<int> &sor_nodes)
{
    const qz_config &c = s->cfg;
    const int ns = (int)sor_nodes.size();
    if (!L.sor.ensure(s->mem, 2L * ns))
    {
        set_error("sor buffers");
        return QZ_FAILURE;
    }
    if (!check_cuda(cudaMemcpyAsync(L.sor.p, sor_nodes.data(), ns * sizeof(int),
                                    cudaMemcpyHostToDevice, s->stream), "sor nodes"))
        return QZ_FAILURE;
    SorArgs A;
    A.sor_nodes = L.sor.p;
    A.nodes = L.nodes.p;
    A.intr = L.intr.p;
    A.d = L.d;
    A.pot = L.pot;
    A.pot_old = L.pot_old;
    A.sweeps = c.branch_sor_sweeps > 0 ? c.branch_sor_sweeps : 1;
    A.every = c.check_every > 0 ? c.check_every : 1;
    A.max_iter = c.max_iter;
    A.method = c.check_method;
    A.w = c.w_sor_branch;
    A.tol = c.tol;
    A.tol2 = c.tol2;
    A.G = c.G;
    A.iters = L.sor.p + ns;
    double pts = 0.0;
    for (int q : sor_nodes)
        pts += L.h[q].nintr;
    launch(s, QZ_PROF_CG, 24.0 * pts * A.sweeps, k_sor_nodes, dim3(ns), dim3(256), A);
    std::vector<int> it(ns);
    if (!read_ints(s, A.iters, ns, it.data()))
        return QZ_FAILURE;
    for (int k = 0; k < ns; k++)
        if (it[k] < 0)
        {
            set_error("the precision was not reached in a refinement-level node (level %d) after "
                      "%d SOR iterations", level_index, -it[k]);
            return QZ_FAILURE;
        }
    return check_cuda(cudaGetLastError(), "sor") ? QZ_SUCCESS : QZ_FAILURE;
}

// Overrides of a solve that is not the reference's (the adjoint's): per-node
// r.r thresholds (device array), the ratio-test bound, nodes to leave out.
struct CgOverride {
    const double *thr;
    double tol2;
    std::vector<char> skip;
};

static int cg_level_collect(qz_sim *s, AmrLevel &L, int level_index, const CgPending &pd);

// Queues the set-up and the cooperative launch of a level's node solves on the
// simulation's stream with no host wait (red-black SOR nodes, if any, are
// solved first, with their own waits); cg_level_collect reads the outcome.
static int cg_level_issue(qz_sim *s, AmrLevel &L, int level_index, CgPending &pd,
                          bool allow_sor = true, const CgOverride *ov = nullptr)
{
    const qz_config &c = s->cfg;
    const int nn = L.nnodes;
    // Chunks of at most CG_UPT x 512 interior points (never across nodes), up to
    // CG_UPT points a thread of a 512-thread block (the pipelined form: 2048,
    // four points a thread).  Levels of up to one chunk per resident block-slot
    // give every block one chunk; larger levels give blocks several.
    constexpr int kCgSmem = 40 * 1024; // slot records and cached grid indices
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    static int occ[3] = {0, 0, 0};
    static std::once_flag occ_once;
    std::call_once(occ_once, [] {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[0], (const void *)k_cg_nodes,
                                                      CG_MAX_THREADS, kCgSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[1], (const void *)k_cg1_nodes,
                                                      CG_MAX_THREADS, kCgSmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ[2], (const void *)k_cg2_nodes,
                                                      CG_MAX_THREADS, kCgSmem);
    });
    // the overrides and replayed schedules are the two-phase kernel's
    const int variant = (!ov && s->sched_mode != 2) ? c.cg_variant : 0;
    const int per_sm = occ[variant];
    const bool one = variant >= 1, pipe = variant == 2;
    if (per_sm < 1)
    {
        set_error("conjugate gradient kernel cannot be resident");
        return QZ_FAILURE;
    }
    const long max_blocks = (long)per_sm * sms;
    const int nt = CG_MAX_THREADS;
    // The level's CG points are cut into about CG_FILL chunks (one block a SM),
    // or 2 CG_FILL when a chunk would exceed the CG_UPT points a thread the
    // update phase holds: the slowest SM sets every phase's length, so chunks fill
    // the SMs evenly.  Measured on the 1M-particle sphere with two points a
    // thread (CG time a step): fixed 1024-point chunks 6.98 ms, CG_FILL 148
    // 6.86 ms, 74 6.89, 222 7.88, 296 7.60.  CG_FILL is fixed, not the device's
    // SM count, so the partial sums and the results do not depend on the device.
    int chunk = (pipe ? CG2_PPT : 2) * nt;
    if (!pipe)
    {
        long tot = 0;
        for (int q = 0; q < nn; q++)
            if (!(ov && ov->skip[q]) && (!allow_sor || L.h[q].ncells > c.branch_cg_cells))
                tot += L.h[q].nintr;
        long target = CG_FILL;
        long cs = (tot + CG_FILL - 1) / CG_FILL;
        if (cs > (long)CG_UPT * nt)
        {
            target = 2L * CG_FILL;
            cs = (tot + 2L * CG_FILL - 1) / (2L * CG_FILL);
        }
        cs = (cs + 31) / 32 * 32;
        // chunks never cross nodes: on a level of several nodes the rounding
        // per node can push the count past the target, and the blocks given one
        // chunk more than the others would set every phase's length; grow the
        // chunk (by 32 points) until the count is within the target
        const long cap = (long)CG_UPT * nt;
        auto count = [&](long size) {
            long k = 0;
            for (int q = 0; q < nn; q++)
                if (!(ov && ov->skip[q]) && (!allow_sor || L.h[q].ncells > c.branch_cg_cells))
                    k += (L.h[q].nintr + size - 1) / size;
            return k;
        };
        while (cs < cap && count(cs) > target)
            cs += 32;
        cs = std::max(cs, (long)c.cg_chunk_min);
        chunk = (int)std::max(64L, std::min(cs, cap));
    }
    L.hchunks.clear();
    std::vector<int> &node_chunk = L.hnode_chunk;
    node_chunk.assign(2L * nn, 0);
    std::vector<int> sor_nodes; // nodes of at most branch_cg_cells cells: red-black SOR
    for (int q = 0; q < nn; q++)
    {
        node_chunk[2 * q] = (int)L.hchunks.size();
        const AmrNode &N = L.h[q];
        if (ov && ov->skip[q])
            ; // no work for this node
        else if (!allow_sor || N.ncells > c.branch_cg_cells)
            for (int b = N.intr_off; b < N.intr_off + N.nintr; b += chunk)
                L.hchunks.push_back({q, b, std::min(b + chunk, N.intr_off + N.nintr)});
        else if (N.nintr > 0)
            sor_nodes.push_back(q);
        node_chunk[2 * q + 1] = (int)L.hchunks.size();
    }
    L.nchunks = (int)L.hchunks.size();
    // solver schedule (forward solves only): replay gives every node its recorded count
    const bool replay = !ov && s->sched_mode == 2;
    const bool record = !ov && s->sched_mode == 1;
    std::vector<int> caps;
    if (replay)
    {
        if (!sor_nodes.empty())
        {
            set_error("a solver schedule cannot replay red-black SOR nodes");
            return QZ_FAILURE;
        }
        caps.resize(nn);
        if (!sched_take(s, nn, caps.data()))
            return QZ_FAILURE;
    }
    if (!sor_nodes.empty() && sor_level(s, L, level_index, sor_nodes))
        return QZ_FAILURE;
    pd = CgPending();
    pd.record = record;
    pd.replay = replay;
    pd.one = one;
    pd.pipe = pipe;
    pd.nn = nn;
    if (L.nchunks == 0)
        return QZ_SUCCESS;
    // nint: node_chunk (2 nn) | rfail[0] (nn) | rfail[1] (nn) | status (3) | iterations (nn)
    const long nparts = (one ? 3L : 4L) * L.nchunks * CG_PS;
    if (!L.chunks.ensure(s->mem, L.nchunks) || !L.chunk_part.ensure(s->mem, nparts) ||
        !L.nint.ensure(s->mem, 6L * nn + 3) || !L.r.ensure(s->mem, L.grid_total) ||
        !L.p.ensure(s->mem, L.grid_total) || !L.Ap.ensure(s->mem, L.grid_total) ||
        !L.apv.ensure(s->mem, L.grid_total) ||
        (one && !L.cg1.ensure(s->mem, 4 * L.grid_total)))
    {
        set_error("cg buffers");
        return QZ_FAILURE;
    }
    // status[2]: nodes with interior points, all unconverged at the start
    int active = 0;
    for (int q = 0; q < nn; q++)
        active += node_chunk[2 * q + 1] > node_chunk[2 * q];
    node_chunk.resize(6L * nn + 3, 0);
    node_chunk[4L * nn + 2] = active;
    for (int q = 0; q < (int)caps.size(); q++)
        node_chunk[5L * nn + 3 + q] = caps[q];
    if (!check_cuda(cudaMemcpyAsync(L.chunks.p, L.hchunks.data(), L.nchunks * sizeof(AmrChunk),
                                    cudaMemcpyHostToDevice, s->stream), "chunks") ||
        !check_cuda(cudaMemcpyAsync(L.nint.p, node_chunk.data(), (6L * nn + 3) * sizeof(int),
                                    cudaMemcpyHostToDevice, s->stream), "cg ints"))
        return QZ_FAILURE;
    // r and both p buffers are zero off the interior points; partials start unpublished
    cudaMemsetAsync(L.r.p, 0, L.grid_total * sizeof(double), s->stream);
    cudaMemsetAsync(L.p.p, 0, L.grid_total * sizeof(double), s->stream);
    cudaMemsetAsync(L.Ap.p, 0, L.grid_total * sizeof(double), s->stream);
    if (one)
    {
        cudaMemsetAsync(L.apv.p, 0, L.grid_total * sizeof(double), s->stream);
        cudaMemsetAsync(L.cg1.p, 0, 4 * L.grid_total * sizeof(double), s->stream);
    }
    cudaMemsetAsync(L.chunk_part.p, 0xff, nparts * sizeof(double), s->stream);
    CgArgs A;
    A.chunks = L.chunks.p;
    A.nchunks = L.nchunks;
    A.intr = L.intr.p;
    A.nodes = L.nodes.p;
    A.node_chunk = L.nint.p;
    A.d = L.d;
    A.pot = L.pot;
    A.pot_old = L.pot_old;
    A.r = L.r.p;
    A.pbuf[0] = L.p.p;
    A.pbuf[1] = L.Ap.p;
    A.apv = L.apv.p;
    A.pap[0] = L.chunk_part.p;
    A.pap[1] = L.chunk_part.p + (long)L.nchunks * CG_PS;
    A.rr[0] = L.chunk_part.p + 2L * L.nchunks * CG_PS;
    A.rr[1] = L.chunk_part.p + 3L * L.nchunks * CG_PS;
    A.rfail[0] = L.nint.p + 2 * nn;
    A.rfail[1] = L.nint.p + 3 * nn;
    A.status = L.nint.p + 4 * nn;
    A.iters = L.nint.p + 4 * nn + 3;
    A.tol = c.tol;
    A.tol2 = c.tol2;
    A.G = c.G;
    A.every = c.check_every > 0 ? c.check_every : 1;
    A.max_iter = c.max_iter;
    A.method = c.check_method;
    A.thr_node = nullptr;
    A.cap_node = replay ? L.nint.p + 5 * nn + 3 : nullptr;
    if (replay)
        A.method = 0; // decisions by the (never met) r.r threshold only
    if (ov)
    {
        A.tol2 = ov->tol2;
        A.method = 0;
        A.thr_node = ov->thr;
    }
    const int blocks = (int)std::min(max_blocks, (long)L.nchunks);
    const int nslot = (L.nchunks + blocks - 1) / blocks;
    A.chunk = chunk;
    const long slot_bytes = one ? (long)sizeof(Cg1Slot) : (long)sizeof(CgSlot);
    A.ncache = std::max(0, (int)((kCgSmem - nslot * slot_bytes) / (chunk * 4L)));
    const size_t smem = nslot * slot_bytes + (size_t)std::min(nslot, A.ncache) * chunk * 4;
    if (smem > (size_t)kCgSmem)
    {
        set_error("conjugate gradient: %d chunks per block exceed the shared memory budget", nslot);
        return QZ_FAILURE;
    }
    Cg1Args B;
    B.chunks = A.chunks;
    B.nchunks = A.nchunks;
    B.chunk = A.chunk;
    B.ncache = A.ncache;
    B.intr = A.intr;
    B.nodes = A.nodes;
    B.node_chunk = A.node_chunk;
    B.d = A.d;
    B.pot = A.pot;
    B.pot_old = A.pot_old;
    B.rb[0] = L.r.p;
    B.rb[1] = L.p.p;
    B.wb[0] = L.Ap.p;
    B.wb[1] = L.apv.p;
    B.sb[0] = one ? L.cg1.p : nullptr;
    B.sb[1] = one ? L.cg1.p + L.grid_total : nullptr;
    B.pb[0] = one ? L.cg1.p + 2 * L.grid_total : nullptr;
    B.pb[1] = one ? L.cg1.p + 3 * L.grid_total : nullptr;
    B.zv = pipe ? L.cg1.p + 3 * L.grid_total : nullptr; // the pipelined form uses no pb[1]
    for (int q = 0; q < 3; q++)
    {
        // gamma and delta of a chunk share its slot's line
        B.pg[q] = L.chunk_part.p + (long)q * L.nchunks * CG_PS;
        B.pd[q] = B.pg[q] + 1;
    }
    B.rfail[0] = A.rfail[0];
    B.rfail[1] = A.rfail[1];
    B.status = A.status;
    B.iters = A.iters;
    B.tol = A.tol;
    B.tol2 = A.tol2;
    B.G = A.G;
    B.every = A.every;
    B.max_iter = A.max_iter;
    B.method = A.method;
    void *args[] = {one ? (void *)&B : (void *)&A};
    cudaEvent_t eb = nullptr, ee = nullptr;
    if (s->prof)
    {
        eb = prof_event(s);
        ee = prof_event(s);
        cudaEventRecord(eb, s->stream);
    }
    if (!check_cuda(cudaLaunchCooperativeKernel(pipe  ? (const void *)k_cg2_nodes
                                                : one ? (const void *)k_cg1_nodes
                                                      : (const void *)k_cg_nodes,
                                                dim3(blocks), dim3(nt), args, smem, s->stream),
                    "cooperative cg"))
        return QZ_FAILURE;
    s->stats.kernel_launches++;
    if (s->prof)
    {
        cudaEventRecord(ee, s->stream);
        s->prof_pending.push_back({QZ_PROF_CG, 0.0, eb, ee});
        pd.prof_idx = (int)s->prof_pending.size() - 1;
    }
    pd.launched = true;
    pd.status = A.status;
    return QZ_SUCCESS;
}

// Reads a level's solve outcome (waits for the stream up to its launch): iteration
// counts, the schedule record, the profiler's bytes and the failure messages.
static int cg_level_collect(qz_sim *s, AmrLevel &L, int level_index, const CgPending &pd)
{
    const int nn = pd.nn;
    const bool record = pd.record, replay = pd.replay, one = pd.one, pipe = pd.pipe;
    if (!pd.launched)
    {
        if (record)
        {
            std::vector<int> z(nn, 0);
            sched_put(s, z.data(), nn);
        }
        return QZ_SUCCESS;
    }
    std::vector<int> st(3 + nn);
    if (!read_ints(s, pd.status, 3 + nn, st.data()))
        return QZ_FAILURE;
    s->stats.cg_iterations += st[0];
    if (pd.prof_idx >= 0 && pd.prof_idx < (int)s->prof_pending.size())
    {
        // bytes per iteration and interior point: the P phase reads r and p_{k-2} and
        // writes p_{k-1} (24 B), the U phase reads p, pot, r and writes pot, r (40 B);
        // the single-reduction form reads r, w, s, p, pot and writes the five (80 B),
        // the pipelined form reads w, z, s, p, r, pot and writes the six (96 B)
        double pts_it = 0.0;
        for (int q = 0; q < nn; q++)
            pts_it += (double)L.h[q].nintr * st[3 + q];
        s->prof_pending[pd.prof_idx].bytes = (pipe ? 96.0 : one ? 80.0 : 64.0) * pts_it;
    }
    if (st[1])
    {
        set_error("conjugate gradient in refinement level %d: a wait for partial sums gave up",
                  level_index);
        return QZ_FAILURE;
    }
    if (record)
        sched_put(s, st.data() + 3, nn);
    if (st[2] != 0 && !replay)
    {
        set_error("the precision was not reached in refinement level %d after %d conjugate "
                  "gradient iterations", level_index, st[0]);
        return QZ_FAILURE;
    }
    return check_cuda(cudaGetLastError(), "cg") ? QZ_SUCCESS : QZ_FAILURE;
}

static int cg_level(qz_sim *s, AmrLevel &L, int level_index, bool allow_sor = true,
                    const CgOverride *ov = nullptr)
{
    CgPending pd;
    if (cg_level_issue(s, L, level_index, pd, allow_sor, ov))
        return QZ_FAILURE;
    return cg_level_collect(s, L, level_index, pd);
}

// The adjoint's node solves on level l: Lap_h lam = rhs on every node's interior
// with lam = 0 on the node boundaries (the level's L.pot, L.d, L.pot_old are
// pointed at lam, rhs and scratch for the call), until r.r <= thr[node]; nodes
// with skip[node] are left out (their lam stays).
int cg_level_adjoint(qz_sim *s, int l, double *lam, double *rhs, double *scratch,
                     const double *thr_dev, const std::vector<char> &skip)
{
    AmrLevel &L = s->amr[l];
    double *kp = L.pot, *kd = L.d, *ko = L.pot_old;
    L.pot = lam;
    L.d = rhs;
    L.pot_old = scratch;
    CgOverride ov{thr_dev, INFINITY, skip};
    const int rc = cg_level(s, L, l, false, &ov);
    L.pot = kp;
    L.d = kd;
    L.pot_old = ko;
    return rc;
}

// Warm start: interior point g of node q takes the previous solve's value at the
// same level coordinates when node q of the previous tree holds that point as an
// interior point (the parent interpolation stays elsewhere).
__global__ void k_pot_warm(int n, const int *__restrict__ intr, const int *__restrict__ intr_node,
                           const AmrNode *__restrict__ nodes, const AmrNode *__restrict__ wnodes,
                           int wnn, const unsigned char *__restrict__ wmask,
                           const double *__restrict__ wpot, double *__restrict__ pot)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const int q = intr_node[t];
    if (q >= wnn)
        return;
    const AmrNode N = nodes[q], W = wnodes[q];
    const long g = intr[t];
    const long sy = N.rd[0] + 1, sz = sy * (N.rd[1] + 1);
    long l = g - N.grid_off;
    const long k = l / sz;
    l -= k * sz;
    const long j = l / sy, i = l - j * sy;
    const long pi = i + N.ts[0] - W.ts[0], pj = j + N.ts[1] - W.ts[1], pk = k + N.ts[2] - W.ts[2];
    if (pi < 0 || pj < 0 || pk < 0 || pi > W.rd[0] || pj > W.rd[1] || pk > W.rd[2])
        return;
    const long wsy = W.rd[0] + 1, wsz = wsy * (W.rd[1] + 1);
    const long pg = W.grid_off + pi + pj * wsy + pk * wsz;
    if (wmask[pg])
        pot[g] = wpot[pg];
}

__global__ void k_mark(int n, const int *__restrict__ idx, unsigned char *__restrict__ mask)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n)
        mask[idx[t]] = 1;
}

// Node CG without a recorded or replayed schedule: every level's set-up and
// solve are queued before any outcome is read back, so the GPU goes from one
// level's solve to the next without waiting for the host (a level's start
// values read its parent's solution in stream order).
bool amr_potential_queues(const qz_sim *s)
{
    return s->cfg.node_solver != QZ_NODE_MG && s->sched_mode == 0;
}

int amr_potential(qz_sim *s)
{
    std::vector<CgPending> pend;
    if (amr_potential_issue(s, pend))
        return QZ_FAILURE;
    return amr_potential_collect(s, pend);
}

int amr_potential_collect(qz_sim *s, const std::vector<CgPending> &pend)
{
    if (amr_potential_queues(s))
        for (int l = 1; l < s->amr_nlev && l < (int)pend.size() && s->amr[l].nnodes > 0; l++)
            if (cg_level_collect(s, s->amr[l], l, pend[l]))
                return QZ_FAILURE;
    return QZ_SUCCESS;
}

// The levels' potentials in order: start values, then the node solves (queued,
// or solved with their waits when amr_potential_queues is false).
int amr_potential_issue(qz_sim *s, std::vector<CgPending> &pend)
{
    const double coeff = -s->cfg.G * s->cfg.total_mass;
    const bool queue = amr_potential_queues(s);
    pend.assign(s->amr_nlev, CgPending());
    for (int l = 1; l < s->amr_nlev; l++)
    {
        AmrLevel &L = s->amr[l];
        AmrLevel &P = s->amr[l - 1];
        if (L.nnodes == 0)
            break;
        if (!L.gpot.ensure(s->mem, L.grid_total) || !L.gpot_old.ensure(s->mem, L.grid_total))
        {
            set_error("level potential buffers");
            return QZ_FAILURE;
        }
        L.pot = L.gpot.p;
        L.pot_old = L.gpot_old.p;
        cudaMemsetAsync(L.pot, 0, L.grid_total * sizeof(double), s->stream);
        if (L.simb_total > 0)
            launch(s, QZ_PROF_OTHER, 16.0 * L.simb_total, k_pot_simb,
                   dim3(blocks_for(L.simb_total, 256)), dim3(256), L.simb_total, L.simb.p,
                   L.simb_node.p, L.nodes.p, coeff, L.pot);
        if (L.bdry_total > 0)
            launch(s, QZ_PROF_OTHER, 80.0 * L.bdry_total, k_pot_init,
                   dim3(blocks_for(L.bdry_total, 256)), dim3(256), L.bdry_total, L.bdry.p,
                   L.bdry_node.p, L.nodes.p, P.nodes.p, P.pot, L.pot);
        if (L.intr_total > 0)
            launch(s, QZ_PROF_OTHER, 80.0 * L.intr_total, k_pot_init,
                   dim3(blocks_for(L.intr_total, 256)), dim3(256), L.intr_total, L.intr.p,
                   L.intr_node.p, L.nodes.p, P.nodes.p, P.pot, L.pot);
        const bool warm = s->cfg.node_warm && s->sched_mode == 0;
        if (warm && L.wnn > 0 && L.intr_total > 0)
            launch(s, QZ_PROF_OTHER, 40.0 * L.intr_total, k_pot_warm,
                   dim3(blocks_for(L.intr_total, 256)), dim3(256), L.intr_total, L.intr.p,
                   L.intr_node.p, L.nodes.p, L.wnodes.p, L.wnn, L.wmask.p, L.wpot.p, L.pot);
        launch(s, QZ_PROF_OTHER, 16.0 * L.grid_total, k_copy_d, dim3(blocks_for(L.grid_total, 256)),
               dim3(256), L.grid_total, L.pot, L.pot_old);
        // the reference's node conjugate gradient, or FP32 multigrid cycles
        // preconditioning a flexible conjugate gradient (qz_node_mg.cu)
        if (queue ? cg_level_issue(s, L, l, pend[l])
                  : s->cfg.node_solver == QZ_NODE_MG ? node_mg_level(s, L, l) : cg_level(s, L, l))
            return QZ_FAILURE;
        if (warm)
        {
            // keep this solve for the next one
            if (!L.wpot.ensure(s->mem, L.grid_total) || !L.wmask.ensure(s->mem, L.grid_total) ||
                !L.wnodes.ensure(s->mem, L.nnodes))
            {
                set_error("warm-start buffers");
                return QZ_FAILURE;
            }
            cudaMemcpyAsync(L.wpot.p, L.pot, L.grid_total * sizeof(double), cudaMemcpyDeviceToDevice,
                            s->stream);
            cudaMemcpyAsync(L.wnodes.p, L.nodes.p, L.nnodes * sizeof(AmrNode),
                            cudaMemcpyDeviceToDevice, s->stream);
            cudaMemsetAsync(L.wmask.p, 0, L.grid_total, s->stream);
            if (L.intr_total > 0)
                launch(s, QZ_PROF_OTHER, 5.0 * L.intr_total, k_mark,
                       dim3(blocks_for(L.intr_total, 256)), dim3(256), L.intr_total, L.intr.p,
                       L.wmask.p);
            L.wnn = L.nnodes;
        }
    }
    return QZ_SUCCESS;
}

// ---- head solved by conjugate gradient (head_pot_method 1) ----------------------------------
// potential_head_node.c:157-171: the head node's potential by the node conjugate
// gradient (conjugate_gradient.c:322-463) instead of multigrid cycles.  The head
// becomes a one-node level: grid (2^L+3)^3 with box_ts -1, interior list all
// points of box coordinates 2..2^L in lexicographic order, mass the total mass,
// 2^(3L) cells.
__global__ void k_head_intr(int L, long D, int *__restrict__ out)
{
    const long m = (1L << L) - 1;
    const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= m * m * m)
        return;
    const long i = 2 + t % m, j = 2 + (t / m) % m, k = 2 + t / (m * m);
    out[t] = (int)(i + j * D + k * D * D);
}

int head_cg_solve(qz_sim *s)
{
    AmrLevel &L = s->head_cg;
    const int Lv = s->cfg.lmin;
    const long m = (1L << Lv) - 1;
    if (L.nnodes == 0)
    {
        AmrNode N{};
        N.lv = Lv;
        N.parent = -1;
        for (int q = 0; q < 3; q++)
        {
            N.ts[q] = -1;
            N.rd[q] = (1 << Lv) + 2;
            N.bmin[q] = 0;
            N.bmax[q] = (1 << Lv) - 1;
        }
        N.ncells = 1 << (3 * Lv);
        N.intr_off = 0;
        N.nintr = (int)(m * m * m);
        N.contact = 1;
        L.nnodes = 1;
        L.h.assign(1, N);
        L.intr_total = N.nintr;
        L.grid_total = s->gpts;
        if (!L.intr.ensure(s->mem, L.intr_total))
        {
            set_error("head conjugate gradient buffers");
            return QZ_FAILURE;
        }
        launch(s, QZ_PROF_OTHER, 4.0 * L.intr_total, k_head_intr,
               dim3(blocks_for(L.intr_total, 256)), dim3(256), Lv, s->D, L.intr.p);
    }
    L.h[0].mass = s->head_mass;
    L.h[0].nptcl = (int)s->n;
    if (!upload_nodes(s, L))
        return QZ_FAILURE;
    L.d = s->d;
    L.pot = s->pot;
    L.pot_old = s->pot_old;
    return cg_level(s, L, 0, false);
}

// ---- one node given as host arrays (the drop-in's conjugate_gradient(struct node *)) -----
// conjugate_gradient.c:322-463 on one node: the node becomes a one-node level whose
// grid fields are device copies of the host arrays, solved by k_cg_nodes, and
// pot and pot_old are copied back.  poisson_error (poisson_error.c:339-342) copies
// the whole pot grid to pot_old at every failed check; the device kernel copies
// the interior points only (the only ones the ratio test reads), so the other
// points of pot_old take pot's values here when a check failed.
static int node_cg_host(qz_sim *s, int lv, const int rd[3], int nintr, const int *intr,
                        double mass, int ncells, const double *d, double *pot, double *pot_old)
{
    AmrLevel &L = s->node_cg;
    AmrNode N{};
    N.lv = lv;
    N.parent = -1;
    for (int q = 0; q < 3; q++)
        N.rd[q] = rd[q];
    N.ncells = ncells;
    N.intr_off = 0;
    N.nintr = nintr;
    N.grid_off = 0;
    N.mass = mass;
    const long gt = (long)(rd[0] + 1) * (rd[1] + 1) * (rd[2] + 1);
    L.nnodes = 1;
    L.h.assign(1, N);
    L.intr_total = nintr;
    L.grid_total = gt;
    if (!L.intr.ensure(s->mem, nintr) || !L.gpot.ensure(s->mem, gt) ||
        !L.gpot_old.ensure(s->mem, gt) || !L.gd.ensure(s->mem, gt) || !upload_nodes(s, L))
    {
        set_error("node conjugate gradient buffers");
        return QZ_FAILURE;
    }
    L.pot = L.gpot.p;
    L.pot_old = L.gpot_old.p;
    L.d = L.gd.p;
    if (!check_cuda(cudaMemcpyAsync(L.intr.p, intr, nintr * sizeof(int), cudaMemcpyHostToDevice,
                                    s->stream), "node list") ||
        !check_cuda(cudaMemcpyAsync(L.pot, pot, gt * sizeof(double), cudaMemcpyHostToDevice,
                                    s->stream), "node pot") ||
        !check_cuda(cudaMemcpyAsync(L.pot_old, pot_old, gt * sizeof(double),
                                    cudaMemcpyHostToDevice, s->stream), "node pot_old") ||
        !check_cuda(cudaMemcpyAsync(L.d, d, gt * sizeof(double), cudaMemcpyHostToDevice,
                                    s->stream), "node density"))
        return QZ_FAILURE;
    const long long it0 = s->stats.cg_iterations;
    const int rc = cg_level(s, L, 0, false);
    const long long iters = s->stats.cg_iterations - it0;
    if (!check_cuda(cudaMemcpyAsync(pot, L.pot, gt * sizeof(double), cudaMemcpyDeviceToHost,
                                    s->stream), "node pot back") ||
        !check_cuda(cudaMemcpyAsync(pot_old, L.pot_old, gt * sizeof(double),
                                    cudaMemcpyDeviceToHost, s->stream), "node pot_old back") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "node sync"))
        return QZ_FAILURE;
    const int every = s->cfg.check_every > 0 ? s->cfg.check_every : 1;
    if (iters > every || rc != QZ_SUCCESS)
    {
        std::vector<char> in(gt, 0);
        for (int e = 0; e < nintr; e++)
            in[intr[e]] = 1;
        for (long g = 0; g < gt; g++)
            if (!in[g])
                pot_old[g] = pot[g];
    }
    return rc;
}

// ---- gradient on refinement levels -------------------------------------------------------
// grid_acceleration.c:199-268, with the y coordinate not scaled by H (as there).
__global__ void k_acc_simb(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                           const AmrNode *__restrict__ nodes, double coeff1,
                           double *__restrict__ ax, double *__restrict__ ay,
                           double *__restrict__ az)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlist)
        return;
    const long g = list[e];
    const AmrNode N = nodes[lnode[e]];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const int top = 1 << N.lv;
    const double H = 1.0 / (1 << N.lv);
    const int cx = gx + N.ts[0], cy = gy + N.ts[1], cz = gz + N.ts[2];
    double ai = (cx == 0 || cx == top) ? 0.0 : cx * H;
    double aj = (cy == 0 || cy == top) ? 0.0 : (double)cy;
    double ak = (cz == 0 || cz == top) ? 0.0 : cz * H;
    double dist = (ai - 0.5) * (ai - 0.5) + (aj - 0.5) * (aj - 0.5) + (ak - 0.5) * (ak - 0.5);
    dist = sqrt(dist);
    double c2 = coeff1 / (dist * dist * dist);
    ax[g] = c2 * (ai - 0.5);
    ay[g] = c2 * (aj - 0.5);
    az[g] = c2 * (ak - 0.5);
}

__global__ void k_acc_bdry(int nlist, const int *__restrict__ list, const int *__restrict__ lnode,
                           const AmrNode *__restrict__ nodes, const AmrNode *__restrict__ pnodes,
                           const double *__restrict__ pax, const double *__restrict__ pay,
                           const double *__restrict__ paz, double *__restrict__ ax,
                           double *__restrict__ ay, double *__restrict__ az)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlist)
        return;
    const long g = list[e];
    const AmrNode N = nodes[lnode[e]];
    int gx, gy, gz;
    grid_coords(N, g, &gx, &gy, &gz);
    const AmrNode P = pnodes[N.parent];
    const int cx = gx + N.ts[0], cy = gy + N.ts[1], cz = gz + N.ts[2];
    ax[g] = from_parent(P, pax, cx, cy, cz);
    ay[g] = from_parent(P, pay, cx, cy, cz);
    az[g] = from_parent(P, paz, cx, cy, cz);
}

// Interior points.  stencil 0: 3-point (grid_acceleration.c:384-393).  stencil
// 1 (grid_acceleration.c:533-692): along x the 5-point difference where the node
// cells at -2 and +1 exist (status > -4); along y and z the reference keeps the
// 3-point difference without periodic boundaries (its 5-point test there never
// sets the flag that selects the 5-point formula, :606-613, :636-643).
__global__ void k_acc_intr(int nlist, int stencil, const int *__restrict__ list,
                           const int *__restrict__ lnode, const AmrNode *__restrict__ nodes,
                           const int *__restrict__ box, const double *__restrict__ pot,
                           double *__restrict__ ax, double *__restrict__ ay,
                           double *__restrict__ az)
{
    int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= nlist)
        return;
    const long g = list[e];
    const AmrNode N = nodes[lnode[e]];
    const double H = 1.0 / (1 << N.lv);
    const double o2h = 1.0 / (2.0 * H);
    const long sy = N.rd[0] + 1, sz = sy * (N.rd[1] + 1);
    bool five = false;
    if (stencil == 1)
    {
        int gx, gy, gz;
        grid_coords(N, g, &gx, &gy, &gz);
        const long b = N.box_off + gx + (long)gy * N.rd[0] + (long)gz * N.rd[0] * N.rd[1];
        five = box[b - 2] > -4 && box[b + 1] > -4;
    }
    if (five)
    {
        const double o12h = 1.0 / (12.0 * H);
        const double t3h = 2.0 / (3.0 * H);
        ax[g] = (pot[g - 1] - pot[g + 1]) * t3h - (pot[g - 2] - pot[g + 2]) * o12h;
    }
    else
        ax[g] = o2h * (pot[g - 1] - pot[g + 1]);
    ay[g] = o2h * (pot[g - sy] - pot[g + sy]);
    az[g] = o2h * (pot[g - sz] - pot[g + sz]);
}

int amr_grid_accel(qz_sim *s)
{
    const double coeff1 = -s->cfg.G * s->cfg.total_mass;
    for (int l = 1; l < s->amr_nlev; l++)
    {
        AmrLevel &L = s->amr[l];
        AmrLevel &P = s->amr[l - 1];
        if (L.nnodes == 0)
            break;
        if (!L.gax.ensure(s->mem, L.grid_total) || !L.gay.ensure(s->mem, L.grid_total) ||
            !L.gaz.ensure(s->mem, L.grid_total))
        {
            set_error("level acceleration buffers");
            return QZ_FAILURE;
        }
        L.ax = L.gax.p;
        L.ay = L.gay.p;
        L.az = L.gaz.p;
        for (double *f : {L.ax, L.ay, L.az})
            cudaMemsetAsync(f, 0, L.grid_total * sizeof(double), s->stream);
        if (L.simb_total > 0)
            launch(s, QZ_PROF_GRADIENT, 32.0 * L.simb_total, k_acc_simb,
                   dim3(blocks_for(L.simb_total, 256)), dim3(256), L.simb_total, L.simb.p,
                   L.simb_node.p, L.nodes.p, coeff1, L.ax, L.ay, L.az);
        if (L.bdry_total > 0)
            launch(s, QZ_PROF_GRADIENT, 224.0 * L.bdry_total, k_acc_bdry,
                   dim3(blocks_for(L.bdry_total, 256)), dim3(256), L.bdry_total, L.bdry.p,
                   L.bdry_node.p, L.nodes.p, P.nodes.p, P.ax, P.ay, P.az, L.ax, L.ay, L.az);
        if (L.intr_total > 0)
            launch(s, QZ_PROF_GRADIENT, (s->cfg.force_stencil ? 48.0 : 32.0) * L.intr_total,
                   k_acc_intr, dim3(blocks_for(L.intr_total, 256)), dim3(256), L.intr_total,
                   s->cfg.force_stencil, L.intr.p, L.intr_node.p, L.nodes.p, L.box.p, L.pot,
                   L.ax, L.ay, L.az);
    }
    return check_cuda(cudaGetLastError(), "level gradient") ? QZ_SUCCESS : QZ_FAILURE;
}

// ---- gather from the finest node -----------------------------------------------------------

__global__ void k_amr_gather(long n, LevelRefs R, const double *__restrict__ x,
                             const double *__restrict__ y, const double *__restrict__ z,
                             double *__restrict__ pax, double *__restrict__ pay,
                             double *__restrict__ paz, int *__restrict__ flags)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    int l = R.nlev - 1;
    int nd = -1;
    for (; l > 0; l--)
    {
        nd = R.node_of[l][i];
        if (nd >= 0)
            break;
    }
    if (l == 0)
        nd = 0;
    const AmrNode N = R.nodes[l][nd];
    const double sc = (double)(1 << N.lv);
    double px = x[i] * sc, py = y[i] * sc, pz = z[i] * sc;
    int fx = (int)px, fy = (int)py, fz = (int)pz;
    long b = box_index(N, fx, fy, fz);
    if (!(px >= 0.0 && py >= 0.0 && pz >= 0.0) || b < 0 || b >= (long)N.rd[0] * N.rd[1] * N.rd[2])
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
    const long sx = N.rd[0] + 1, sxy = sx * (N.rd[1] + 1);
    const long g = grid_index(N, fx - N.ts[0], fy - N.ts[1], fz - N.ts[2]);
    const double *gx = R.ax[l], *gy = R.ay[l], *gz = R.az[l];
    double ax = pax[i], ay = pay[i], az = paz[i];
#pragma unroll
    for (int kk = 0; kk < 2; kk++)
#pragma unroll
        for (int jj = 0; jj < 2; jj++)
#pragma unroll
            for (int ii = 0; ii < 2; ii++)
            {
                int a = ii + 2 * jj + 4 * kk;
                long q = g + ii + jj * sx + kk * sxy;
                ax += gx[q] * w[a];
                ay += gy[q] * w[a];
                az += gz[q] * w[a];
            }
    pax[i] = ax;
    pay[i] = ay;
    paz[i] = az;
}

// observables.c:205-424: m times the potential interpolated (CIC) at the
// particle from its finest node; per-block partial sums (fixed order).
__global__ void k_amr_pot_energy(long n, LevelRefs R, const double *__restrict__ x,
                                 const double *__restrict__ y, const double *__restrict__ z,
                                 const double *__restrict__ m, double *__restrict__ part)
{
    __shared__ double sh[32];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < n)
    {
        int l = R.nlev - 1;
        int nd = -1;
        for (; l > 0; l--)
        {
            nd = R.node_of[l][i];
            if (nd >= 0)
                break;
        }
        if (l == 0)
            nd = 0;
        const AmrNode N = R.nodes[l][nd];
        const double sc = (double)(1 << N.lv);
        const double px = x[i] * sc, py = y[i] * sc, pz = z[i] * sc;
        const int fx = (int)px, fy = (int)py, fz = (int)pz;
        const double wx1 = px - fx, wy1 = py - fy, wz1 = pz - fz;
        const double wx2 = 1.0 - wx1, wy2 = 1.0 - wy1, wz2 = 1.0 - wz1;
        double w[8];
        w[0] = wx2 * wy2 * wz2;
        w[1] = wx1 * wy2 * wz2;
        w[2] = wx2 * wy1 * wz2;
        w[3] = wx1 * wy1 * wz2;
        w[4] = wx2 * wy2 * wz1;
        w[5] = wx1 * wy2 * wz1;
        w[6] = wx2 * wy1 * wz1;
        w[7] = wx1 * wy1 * wz1;
        const long sx = N.rd[0] + 1, sxy = sx * (N.rd[1] + 1);
        const long g = grid_index(N, fx - N.ts[0], fy - N.ts[1], fz - N.ts[2]);
        const double *pot = R.ax[l];
        double a = 0.0;
        for (int kk = 0; kk < 2; kk++)
            for (int jj = 0; jj < 2; jj++)
                for (int ii = 0; ii < 2; ii++)
                    a += pot[g + ii + jj * sx + kk * sxy] * w[ii + 2 * jj + 4 * kk];
        e = m[i] * a;
    }
    const double t = block_sum_d(e, sh);
    if (threadIdx.x == 0)
        part[blockIdx.x] = t;
}

int amr_pot_energy_partials(qz_sim *s, double *part)
{
    LevelRefs R{};
    R.nlev = s->amr_nlev;
    for (int l = 0; l < s->amr_nlev; l++)
    {
        R.nodes[l] = s->amr[l].nodes.p;
        R.node_of[l] = s->node_of[l].p;
        R.ax[l] = s->amr[l].pot;
    }
    launch(s, QZ_PROF_OTHER, 96.0 * s->n, k_amr_pot_energy, dim3(blocks_for(s->n, 256)),
           dim3(256), s->n, R, s->x, s->y, s->z, s->m, part);
    return check_cuda(cudaGetLastError(), "potential energy") ? QZ_SUCCESS : QZ_FAILURE;
}

int amr_gather(qz_sim *s)
{
    if (s->n == 0)
        return QZ_SUCCESS;
    LevelRefs R{};
    R.nlev = s->amr_nlev;
    for (int l = 0; l < s->amr_nlev; l++)
    {
        R.nodes[l] = s->amr[l].nodes.p;
        R.node_of[l] = s->node_of[l].p;
        R.ax[l] = s->amr[l].ax;
        R.ay[l] = s->amr[l].ay;
        R.az[l] = s->amr[l].az;
    }
    launch(s, QZ_PROF_GATHER, 72.0 * s->n + 8.0 * s->n * s->amr_nlev, k_amr_gather,
           dim3(blocks_for(s->n, 256)), dim3(256), s->n, R, s->x, s->y, s->z, s->ax, s->ay, s->az,
           s->flags);
    return check_cuda(cudaGetLastError(), "amr gather") ? QZ_SUCCESS : QZ_FAILURE;
}
} // namespace qz

using namespace qz;

extern "C" int qz_node_conjugate_gradient(qz_sim *s, int lv, int box_real_dim_x,
                                          int box_real_dim_y, int box_real_dim_z,
                                          int grid_intr_size, const int *intr_box_grid_idx,
                                          double node_mass, int cell_size, const double *d,
                                          double *pot, double *pot_old)
{
    if (!s || lv < 0 || lv > 30 || box_real_dim_x < 2 || box_real_dim_y < 2 || box_real_dim_z < 2 ||
        grid_intr_size < 0 || (grid_intr_size > 0 && !intr_box_grid_idx) || !d || !pot ||
        !pot_old || cell_size <= 0)
    {
        set_error("qz_node_conjugate_gradient: bad arguments");
        return QZ_FAILURE;
    }
    if (grid_intr_size == 0)
        return QZ_SUCCESS;
    const long gt = (long)(box_real_dim_x + 1) * (box_real_dim_y + 1) * (box_real_dim_z + 1);
    const long sy = box_real_dim_x + 1, sz = sy * (box_real_dim_y + 1);
    for (int e = 0; e < grid_intr_size; e++)
    {
        const long g = intr_box_grid_idx[e];
        if (g - sz < 0 || g + sz >= gt)
        {
            set_error("qz_node_conjugate_gradient: interior point %ld has a neighbour outside "
                      "the node grid", g);
            return QZ_FAILURE;
        }
    }
    const int rd[3] = {box_real_dim_x, box_real_dim_y, box_real_dim_z};
    return node_cg_host(s, lv, rd, grid_intr_size, intr_box_grid_idx, node_mass, cell_size, d, pot,
                        pot_old);
}


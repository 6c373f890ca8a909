// qz_amr_dev.cuh -- device helpers of the refinement levels shared by the level
// kernels (qz_amr.cu) and their adjoints (qz_adjoint_amr.cu).
#pragma once
#include "qz_internal.cuh"

namespace qz {

constexpr int AMR_MAX_LEVELS = 16;

// ---- small device helpers --------------------------------------------------------------
// Index of the last node whose offset (0: grid_off, 1: cls_off, 2: box_off) is <= v.
__device__ __forceinline__ int find_node(const AmrNode *nodes, int nn, long v, int field)
{
    int lo = 0, hi = nn - 1;
    while (lo < hi)
    {
        int mid = (lo + hi + 1) >> 1;
        long off = field == 0 ? nodes[mid].grid_off : field == 1 ? nodes[mid].cls_off : nodes[mid].box_off;
        if (off <= v)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ long box_index(const AmrNode &N, int cx, int cy, int cz)
{
    return (long)(cx - N.ts[0]) + (long)(cy - N.ts[1]) * N.rd[0] +
           (long)(cz - N.ts[2]) * N.rd[0] * N.rd[1];
}

__device__ __forceinline__ long grid_index(const AmrNode &N, int gx, int gy, int gz)
{
    // box grid coordinates (not level coordinates)
    return N.grid_off + gx + (long)gy * (N.rd[0] + 1) + (long)gz * (N.rd[0] + 1) * (N.rd[1] + 1);
}

__device__ __forceinline__ void grid_coords(const AmrNode &N, long g, int *gx, int *gy, int *gz)
{
    long l = g - N.grid_off;
    const long sx = N.rd[0] + 1, sxy = sx * (N.rd[1] + 1);
    *gz = (int)(l / sxy);
    l -= (long)(*gz) * sxy;
    *gy = (int)(l / sx);
    *gx = (int)(l - (long)(*gy) * sx);
}

// Parent-interpolated start (potential_branches.c:204-331): 0.125 times the sum
// of the 8 parent values at (c >> 1, (c + 1) >> 1) per axis, in the reference's
// order; `field` selects potential or acceleration arrays of the parent.
__device__ __forceinline__ double from_parent(const AmrNode &P, const double *__restrict__ pf,
                                              int cx, int cy, int cz)
{
    const int x1 = (cx >> 1) - P.ts[0], x2 = ((cx + 1) >> 1) - P.ts[0];
    const int y1 = (cy >> 1) - P.ts[1], y2 = ((cy + 1) >> 1) - P.ts[1];
    const int z1 = (cz >> 1) - P.ts[2], z2 = ((cz + 1) >> 1) - P.ts[2];
    const long sx = P.rd[0] + 1, sxy = sx * (P.rd[1] + 1);
    const long o = P.grid_off;
    return 0.125 * (pf[o + x1 + y1 * sx + z1 * sxy] + pf[o + x2 + y1 * sx + z1 * sxy] +
                    pf[o + x1 + y2 * sx + z1 * sxy] + pf[o + x2 + y2 * sx + z1 * sxy] +
                    pf[o + x1 + y1 * sx + z2 * sxy] + pf[o + x2 + y1 * sx + z2 * sxy] +
                    pf[o + x1 + y2 * sx + z2 * sxy] + pf[o + x2 + y2 * sx + z2 * sxy]);
}


// The levels' node tables, particle assignments and grid accelerations, for the
// gathers from each particle's finest node.
struct LevelRefs {
    const AmrNode *nodes[AMR_MAX_LEVELS];
    const int *node_of[AMR_MAX_LEVELS];
    const double *ax[AMR_MAX_LEVELS], *ay[AMR_MAX_LEVELS], *az[AMR_MAX_LEVELS];
    int nlev;
};

} // namespace qz

// qz_sort.cu -- stable LSD radix sort of (uint32 key, int32 value) pairs and an
// exclusive int scan, both deterministic (no order-dependent atomics on the
// data path: per-tile digit counts use shared-memory integer atomics, whose
// totals do not depend on order; ranks come from warp match masks in the
// original element order).
//
// Tile = 8 warps x 8 iterations x 32 lanes = 2048 keys.  Warp w of tile t
// owns keys [t*2048 + w*256, +256); iteration r covers 32 consecutive keys in
// lane order, so (warp, iteration, lane) order is the input order and the
// scatter is stable.  Histograms are stored digit-major (digit * tiles + tile)
// so that one exclusive scan yields every (digit, tile) output base.
#include "qz_internal.cuh"

namespace qz {

constexpr int RS_WARPS = 8;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_WARPS * RS_ITEMS * 32; // 2048
constexpr int RS_RADIX = 256;

__global__ void k_rs_upsweep(const unsigned *__restrict__ keys, long n, int shift, int tiles,
                             int *__restrict__ hist)
{
    __shared__ int cnt[RS_RADIX];
    for (int i = threadIdx.x; i < RS_RADIX; i += blockDim.x)
        cnt[i] = 0;
    __syncthreads();
    long base = (long)blockIdx.x * RS_TILE;
    for (int it = threadIdx.x; it < RS_TILE; it += blockDim.x)
    {
        long i = base + it;
        if (i < n)
            atomicAdd(&cnt[(keys[i] >> shift) & 0xFF], 1);
    }
    __syncthreads();
    for (int dgt = threadIdx.x; dgt < RS_RADIX; dgt += blockDim.x)
        hist[(long)dgt * tiles + blockIdx.x] = cnt[dgt];
}

__global__ void k_rs_downsweep(const unsigned *__restrict__ kin, const int *__restrict__ vin,
                               unsigned *__restrict__ kout, int *__restrict__ vout, long n,
                               int shift, int tiles, const int *__restrict__ hist)
{
    __shared__ int woff[RS_WARPS][RS_RADIX];
    __shared__ int bbase[RS_RADIX];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < RS_WARPS * RS_RADIX; i += blockDim.x)
        (&woff[0][0])[i] = 0;
    for (int dgt = threadIdx.x; dgt < RS_RADIX; dgt += blockDim.x)
        bbase[dgt] = hist[(long)dgt * tiles + blockIdx.x];
    __syncthreads();
    const long wbase = (long)blockIdx.x * RS_TILE + (long)warp * RS_ITEMS * 32;
    // per-warp digit counts
    for (int r = 0; r < RS_ITEMS; r++)
    {
        long i = wbase + r * 32 + lane;
        if (i < n)
            atomicAdd(&woff[warp][(kin[i] >> shift) & 0xFF], 1);
    }
    __syncthreads();
    // exclusive prefix over warps, per digit
    for (int dgt = threadIdx.x; dgt < RS_RADIX; dgt += blockDim.x)
    {
        int run = 0;
        for (int w = 0; w < RS_WARPS; w++)
        {
            int c = woff[w][dgt];
            woff[w][dgt] = run;
            run += c;
        }
    }
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < RS_ITEMS; r++)
    {
        long i = wbase + r * 32 + lane;
        bool valid = i < n;
        unsigned active = __ballot_sync(0xffffffffu, valid);
        if (valid)
        {
            unsigned k = kin[i];
            int v = vin[i];
            int dgt = (k >> shift) & 0xFF;
            unsigned peers = __match_any_sync(active, dgt);
            int rank = __popc(peers & lt);
            int pos = bbase[dgt] + woff[warp][dgt] + rank;
            kout[pos] = k;
            vout[pos] = v;
            __syncwarp(active);
            if (rank == 0)
                woff[warp][dgt] += __popc(peers);
        }
        __syncwarp();
    }
}

// ---- exclusive scan (three phases, fixed tiling) -----------------------------
constexpr int SC_THREADS = 1024;
constexpr int SC_ITEMS = 4;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

__device__ __forceinline__ int block_excl_scan(int v, int *sh, int *total)
{
    // warp inclusive scan
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        sh[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        int nw = blockDim.x >> 5;
        int w = lane < nw ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1)
        {
            int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o)
                w += y;
        }
        if (lane < nw)
            sh[lane] = w;
    }
    __syncthreads();
    int wprefix = warp > 0 ? sh[warp - 1] : 0;
    int t = sh[(blockDim.x >> 5) - 1];
    __syncthreads();
    if (total)
        *total = t;
    return wprefix + x - v;
}

__global__ void k_scan_tiles(const int *__restrict__ in, long n, int *__restrict__ tile_sums)
{
    __shared__ int sh[32];
    long base = (long)blockIdx.x * SC_TILE + (long)threadIdx.x * SC_ITEMS;
    int s = 0;
    for (int q = 0; q < SC_ITEMS; q++)
        if (base + q < n)
            s += in[base + q];
    int total;
    block_excl_scan(s, sh, &total);
    if (threadIdx.x == 0)
        tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of m values in place (m may exceed the block).
__global__ void k_scan_single(int *__restrict__ a, long m)
{
    __shared__ int sh[32];
    int carry = 0;
    for (long base = 0; base < m; base += (long)SC_THREADS * SC_ITEMS)
    {
        long i0 = base + (long)threadIdx.x * SC_ITEMS;
        int v[SC_ITEMS];
        int s = 0;
        for (int q = 0; q < SC_ITEMS; q++)
        {
            v[q] = (i0 + q < m) ? a[i0 + q] : 0;
            s += v[q];
        }
        int total;
        int ex = block_excl_scan(s, sh, &total);
        int run = carry + ex;
        for (int q = 0; q < SC_ITEMS; q++)
        {
            if (i0 + q < m)
                a[i0 + q] = run;
            run += v[q];
        }
        carry += total;
        __syncthreads();
    }
}

// in and out may be the same array (each block reads its tile before writing it)
__global__ void k_scan_apply(const int *in, int *out, long n, const int *__restrict__ tile_offsets)
{
    __shared__ int sh[32];
    long base = (long)blockIdx.x * SC_TILE + (long)threadIdx.x * SC_ITEMS;
    int v[SC_ITEMS];
    int s = 0;
    for (int q = 0; q < SC_ITEMS; q++)
    {
        v[q] = (base + q < n) ? in[base + q] : 0;
        s += v[q];
    }
    int ex = block_excl_scan(s, sh, nullptr);
    int run = tile_offsets[blockIdx.x] + ex;
    for (int q = 0; q < SC_ITEMS; q++)
    {
        if (base + q < n)
            out[base + q] = run;
        run += v[q];
    }
}

int scan_exclusive(qz_sim *s, const int *in, int *out, long n)
{
    if (n <= 0)
        return QZ_SUCCESS;
    long tiles = (n + SC_TILE - 1) / SC_TILE;
    if (s->scan_tmp_cap < tiles)
    {
        pool_free(s->mem, s->scan_tmp);
        s->scan_tmp = nullptr;
        s->scan_tmp_cap = 0;
        const long cap = tiles + tiles / 2 + 64;
        if (!pool_alloc(s->mem, &s->scan_tmp, cap))
        {
            set_error("scan scratch: out of device memory");
            return QZ_FAILURE;
        }
        s->scan_tmp_cap = cap;
    }
    launch(s, QZ_PROF_SORT, 4.0 * n, k_scan_tiles, dim3((int)tiles), dim3(SC_THREADS), in, n, s->scan_tmp);
    launch(s, QZ_PROF_SORT, 8.0 * 256 * tiles, k_scan_single, dim3(1), dim3(SC_THREADS), s->scan_tmp, tiles);
    launch(s, QZ_PROF_SORT, 8.0 * n, k_scan_apply, dim3((int)tiles), dim3(SC_THREADS), in, out, n, s->scan_tmp);
    return check_cuda(cudaGetLastError(), "scan") ? QZ_SUCCESS : QZ_FAILURE;
}

// Sorts s->sort.k0/v0 (n pairs) on the low `bits` bits; the sorted result is
// returned through keys_out / vals_out (one of the two ping-pong buffers).
int radix_sort_pairs(qz_sim *s, long n, int bits, unsigned **keys_out, int **vals_out)
{
    Sort &S = s->sort;
    unsigned *ki = S.k0, *ko = S.k1;
    int *vi = S.v0, *vo = S.v1;
    if (n <= 0)
    {
        *keys_out = ki;
        *vals_out = vi;
        return QZ_SUCCESS;
    }
    int tiles = (int)((n + RS_TILE - 1) / RS_TILE);
    for (int shift = 0; shift < bits; shift += 8)
    {
        launch(s, QZ_PROF_SORT, 4.0 * n, k_rs_upsweep, dim3(tiles), dim3(RS_WARPS * 32), ki, n, shift, tiles, S.hist);
        // digit-major counts of all tiles: exclusive scan in place (one block when small)
        const long hm = (long)RS_RADIX * tiles;
        if (hm <= 4L * SC_TILE)
            launch(s, QZ_PROF_SORT, 8.0 * hm, k_scan_single, dim3(1), dim3(SC_THREADS), S.hist, hm);
        else if (scan_exclusive(s, S.hist, S.hist, hm))
            return QZ_FAILURE;
        launch(s, QZ_PROF_SORT, 16.0 * n, k_rs_downsweep, dim3(tiles), dim3(RS_WARPS * 32), ki, vi, ko, vo, n, shift, tiles, S.hist);
        unsigned *tk = ki;
        ki = ko;
        ko = tk;
        int *tv = vi;
        vi = vo;
        vo = tv;
    }
    *keys_out = ki;
    *vals_out = vi;
    return check_cuda(cudaGetLastError(), "radix sort") ? QZ_SUCCESS : QZ_FAILURE;
}

long radix_tiles(long n) { return (n + RS_TILE - 1) / RS_TILE; }

} // namespace qz

// qz_sort.cu -- stable LSD radix sort of (uint32 key, int32 value) pairs and an
// exclusive int scan, both deterministic (no order-dependent atomics on the
// data path: per-tile digit counts use shared-memory integer atomics, whose
// totals do not depend on order; ranks come from warp match masks in the
// original element order; the scan's tile numbers follow the blocks' arrival,
// but its results are integer sums and do not depend on it).
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
static_assert(SC_ITEMS == 4, "k_scan_lookback moves a thread's items as one int4");
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

// Single-pass exclusive scan (decoupled look-back, Merrill and Garland 2016).
// A block takes the next tile number from a counter (arrival order: every
// tile before it belongs to a block that is already running, so a wait always
// ends), scans its tile, publishes the tile's sum in its status word, then adds
// the published values of the tiles before it, walking back until one holds an
// inclusive prefix, and publishes its own inclusive prefix.  The walk is one
// warp's: lane l reads the status of the l-th tile back, so a window of 32
// predecessors costs one round trip; a window is used once every tile in it up
// to the nearest inclusive prefix has published.  A status word is flag (2
// bits: 1 = tile sum, 2 = inclusive prefix) | epoch (30 bits) | value (32
// bits): one word, so a reader sees a flag and its value together; words of an
// earlier call carry an older epoch and read as not yet published.  Integer
// sums: the result does not depend on the order of arrival.  A wait gives up
// after SCAN_POLL_LIMIT polls and sets E_SCAN in flags[F_ERROR].
constexpr long SCAN_POLL_LIMIT = 1L << 22;

__device__ __forceinline__ unsigned long long scan_ld(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void scan_st(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Sum of the published values of the tiles before `tile` (warp 0 of the block).
__device__ __forceinline__ int scan_lookback_warp(const unsigned long long *st, long tile,
                                                  unsigned epoch, int *flags)
{
    const int lane = threadIdx.x & 31;
    int prefix = 0;
    long polls = 0;
    for (long j = tile - 1; j >= 0;)
    {
        const long idx = j - lane;
        unsigned fl = 2, val = 0; // before tile 0: an inclusive zero (never reached past it)
        if (idx >= 0)
        {
            const unsigned long long w = scan_ld(&st[idx]);
            fl = (unsigned)(w >> 62);
            if ((unsigned)((w >> 32) & 0x3fffffffu) != epoch)
                fl = 0;
            val = (unsigned)w;
        }
        const unsigned m2 = __ballot_sync(0xffffffffu, fl == 2);
        const unsigned m0 = __ballot_sync(0xffffffffu, fl == 0);
        const int first2 = m2 ? __ffs(m2) - 1 : 32;
        // lanes up to the nearest inclusive prefix must all have published
        const unsigned need = first2 == 32 ? 0xffffffffu : ((2u << first2) - 1u);
        if (m0 & need)
        {
            if (++polls > SCAN_POLL_LIMIT)
            {
                if (lane == 0)
                    atomicOr(&flags[F_ERROR], E_SCAN);
                break;
            }
            continue;
        }
        int add = (lane <= first2) ? (int)val : 0;
        for (int o = 16; o > 0; o >>= 1)
            add += __shfl_xor_sync(0xffffffffu, add, o);
        prefix += add;
        if (first2 < 32)
            break;
        j -= 32;
    }
    return prefix;
}

__global__ void __launch_bounds__(SC_THREADS)
    k_scan_lookback(const int *in, int *out, long n, unsigned long long *__restrict__ st,
                    unsigned long long *__restrict__ ctr, unsigned long long base,
                    unsigned epoch, int *__restrict__ flags)
{
    __shared__ int sh[32];
    __shared__ long s_tile;
    __shared__ int s_prefix;
    if (threadIdx.x == 0)
        s_tile = (long)(atomicAdd(ctr, 1ull) - base);
    __syncthreads();
    const long tile = s_tile;
    const long i0 = tile * SC_TILE + (long)threadIdx.x * SC_ITEMS;
    int v[SC_ITEMS];
    int sum = 0;
    if (i0 + SC_ITEMS <= n && ((reinterpret_cast<unsigned long long>(in + i0) & 15) == 0))
    {
        const int4 q4 = *reinterpret_cast<const int4 *>(in + i0);
        v[0] = q4.x;
        v[1] = q4.y;
        v[2] = q4.z;
        v[3] = q4.w;
    }
    else
        for (int q = 0; q < SC_ITEMS; q++)
            v[q] = (i0 + q < n) ? in[i0 + q] : 0;
    for (int q = 0; q < SC_ITEMS; q++)
        sum += v[q];
    int total;
    const int ex = block_excl_scan(sum, sh, &total);
    if (threadIdx.x < 32)
    {
        const unsigned long long tag = (unsigned long long)epoch << 32;
        int prefix = 0;
        if (tile > 0)
        {
            if (threadIdx.x == 0)
                scan_st(&st[tile], (1ull << 62) | tag | (unsigned)total);
            prefix = scan_lookback_warp(st, tile, epoch, flags);
        }
        if (threadIdx.x == 0)
        {
            scan_st(&st[tile], (2ull << 62) | tag | (unsigned)(prefix + total));
            s_prefix = prefix;
        }
    }
    __syncthreads();
    int run = s_prefix + ex;
    int o[SC_ITEMS];
    for (int q = 0; q < SC_ITEMS; q++)
    {
        o[q] = run;
        run += v[q];
    }
    if (i0 + SC_ITEMS <= n && ((reinterpret_cast<unsigned long long>(out + i0) & 15) == 0))
        *reinterpret_cast<int4 *>(out + i0) = make_int4(o[0], o[1], o[2], o[3]);
    else
        for (int q = 0; q < SC_ITEMS; q++)
            if (i0 + q < n)
                out[i0 + q] = o[q];
}

// Status words for `tiles` tiles and a fresh epoch for the next scan.
static int scan_prepare(qz_sim *s, long tiles)
{
    if (s->scan_st_cap < tiles)
    {
        // status words and the counter start at zero (epoch 0 is never used)
        pool_free(s->mem, s->scan_st);
        s->scan_st = nullptr;
        s->scan_st_cap = 0;
        const long cap = tiles + tiles / 2 + 64;
        if (!pool_alloc(s->mem, &s->scan_st, cap + 1))
        {
            set_error("scan status words: out of device memory");
            return QZ_FAILURE;
        }
        cudaMemsetAsync(s->scan_st, 0, (cap + 1) * sizeof(unsigned long long), s->stream);
        s->scan_st_cap = cap;
        s->scan_base = 0;
    }
    if (++s->scan_epoch >= (1u << 30))
    {
        // the epoch field wraps: clear the old words once
        cudaMemsetAsync(s->scan_st, 0, s->scan_st_cap * sizeof(unsigned long long), s->stream);
        s->scan_epoch = 1;
    }
    return QZ_SUCCESS;
}

// in and out may be the same array (each block reads its tile before writing it)
int scan_exclusive(qz_sim *s, const int *in, int *out, long n)
{
    if (n <= 0)
        return QZ_SUCCESS;
    const long tiles = (n + SC_TILE - 1) / SC_TILE;
    if (scan_prepare(s, tiles))
        return QZ_FAILURE;
    launch(s, QZ_PROF_SORT, 8.0 * n, k_scan_lookback, dim3((int)tiles), dim3(SC_THREADS), in, out,
           n, s->scan_st, s->scan_st + s->scan_st_cap, s->scan_base, s->scan_epoch, s->flags);
    s->scan_base += (unsigned long long)tiles;
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

// Test hook for the look-back's bounded wait: one block of a fresh epoch that
// draws tile 1 (base one below the tile counter, which equals scan_base between
// scans), whose tile 0 is never published, so its wait must run to
// SCAN_POLL_LIMIT, set E_SCAN and return.  n = 0: the block reads and writes
// no element.
int scan_wait_probe(qz_sim *s)
{
    if (scan_prepare(s, 2))
        return QZ_FAILURE;
    launch(s, QZ_PROF_SORT, 0.0, k_scan_lookback, dim3(1), dim3(SC_THREADS), (const int *)nullptr,
           (int *)nullptr, 0L, s->scan_st, s->scan_st + s->scan_st_cap, s->scan_base - 1ull,
           s->scan_epoch, s->flags);
    s->scan_base += 1ull; // the counter advanced by one tile
    return check_cuda(cudaGetLastError(), "scan probe") ? QZ_SUCCESS : QZ_FAILURE;
}

// Test hook: sets the epoch the next scan increments (to reach the wrap).
void scan_set_epoch(qz_sim *s, unsigned epoch) { s->scan_epoch = epoch; }

} // namespace qz

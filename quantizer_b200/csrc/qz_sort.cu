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
// scatter is stable.  One pass per 8-bit digit, each a single launch
// (Adinets and Merrill's one-sweep arrangement, 2022): the digit counts of all
// passes come from one histogram launch, and a pass's tile finds the keys of
// its digits in earlier tiles by a decoupled look-back (one thread a digit)
// instead of an upsweep and a scan of per-tile counts.
#include <algorithm>

#include "qz_internal.cuh"

namespace qz {

constexpr int RS_WARPS = 8;
constexpr int RS_ITEMS = 8;
constexpr int RS_TILE = RS_WARPS * RS_ITEMS * 32; // 2048
constexpr int RS_RADIX = 256;

// ---- exclusive scan -------------------------------------------------------------------
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

// ---- radix sort ----------------------------------------------------------------------
// Digit counts of every pass (passes x 256, zeroed by the caller): block-local
// counts in shared memory, then one integer add per digit and block.
__global__ void k_rs_hist(const unsigned *__restrict__ keys, long n, int passes,
                          int *__restrict__ ghist)
{
    __shared__ int cnt[4][RS_RADIX];
    for (int i = threadIdx.x; i < 4 * RS_RADIX; i += blockDim.x)
        (&cnt[0][0])[i] = 0;
    __syncthreads();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
    {
        const unsigned k = keys[i];
        for (int p = 0; p < passes; p++)
            atomicAdd(&cnt[p][(k >> (8 * p)) & 0xFF], 1);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * RS_RADIX; i += blockDim.x)
    {
        const int c = (&cnt[0][0])[i];
        if (c)
            atomicAdd(&ghist[i], c);
    }
}

// One pass on the digit at `shift`.  A block takes the next tile number from
// the counter (arrival order, as the scan), counts its keys per warp and digit,
// publishes its per-digit counts in the status words of its tile (flag | epoch
// | value, as the scan's), and thread d adds the counts of digit d in the tiles
// before it, walking back to the first inclusive prefix; the digit's output
// base is the exclusive scan of the pass's global counts plus that prefix.  The
// scatter is the stable warp-ordered one.
__global__ void __launch_bounds__(RS_WARPS * 32)
    k_rs_onesweep(const unsigned *__restrict__ kin, const int *__restrict__ vin,
                  unsigned *__restrict__ kout, int *__restrict__ vout, long n, int shift,
                  const int *__restrict__ ghist, unsigned long long *__restrict__ st,
                  unsigned long long *__restrict__ ctr, unsigned long long base, unsigned epoch,
                  int *__restrict__ flags)
{
    static_assert(RS_WARPS * 32 == RS_RADIX, "one thread a digit");
    __shared__ int woff[RS_WARPS][RS_RADIX];
    __shared__ int bbase[RS_RADIX];
    __shared__ int sh[32];
    __shared__ long s_tile;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0)
        s_tile = (long)(atomicAdd(ctr, 1ull) - base);
    for (int i = tid; i < RS_WARPS * RS_RADIX; i += blockDim.x)
        (&woff[0][0])[i] = 0;
    // exclusive scan of the pass's global digit counts
    int total;
    const int gex = block_excl_scan(ghist[tid], sh, &total);
    __syncthreads();
    const long tile = s_tile;
    const long wbase = tile * RS_TILE + (long)warp * RS_ITEMS * 32;
    for (int r = 0; r < RS_ITEMS; r++)
    {
        const long i = wbase + r * 32 + lane;
        if (i < n)
            atomicAdd(&woff[warp][(kin[i] >> shift) & 0xFF], 1);
    }
    __syncthreads();
    // thread d: exclusive prefix over warps of digit d, the tile's count of d
    const int d = tid;
    int cnt = 0;
    for (int w = 0; w < RS_WARPS; w++)
    {
        const int c = woff[w][d];
        woff[w][d] = cnt;
        cnt += c;
    }
    const unsigned long long tag = (unsigned long long)epoch << 32;
    int prefix = 0;
    if (tile > 0)
    {
        scan_st(&st[tile * RS_RADIX + d], (1ull << 62) | tag | (unsigned)cnt);
        long polls = 0;
        for (long j = tile - 1; j >= 0;)
        {
            const unsigned long long w = scan_ld(&st[j * RS_RADIX + d]);
            const unsigned fl = (unsigned)(w >> 62);
            if (fl == 0 || (unsigned)((w >> 32) & 0x3fffffffu) != epoch)
            {
                if (++polls > SCAN_POLL_LIMIT)
                {
                    atomicOr(&flags[F_ERROR], E_SCAN);
                    break;
                }
                continue;
            }
            prefix += (int)(unsigned)w;
            if (fl == 2)
                break;
            j--;
        }
    }
    scan_st(&st[tile * RS_RADIX + d], (2ull << 62) | tag | (unsigned)(prefix + cnt));
    bbase[d] = gex + prefix;
    __syncthreads();
    const unsigned lt = (1u << lane) - 1u;
    for (int r = 0; r < RS_ITEMS; r++)
    {
        const long i = wbase + r * 32 + lane;
        const bool valid = i < n;
        const unsigned active = __ballot_sync(0xffffffffu, valid);
        if (valid)
        {
            const unsigned k = kin[i];
            const int v = vin[i];
            const int dg = (k >> shift) & 0xFF;
            const unsigned peers = __match_any_sync(active, dg);
            const int rank = __popc(peers & lt);
            const int pos = bbase[dg] + woff[warp][dg] + rank;
            kout[pos] = k;
            vout[pos] = v;
            __syncwarp(active);
            if (rank == 0)
                woff[warp][dg] += __popc(peers);
        }
        __syncwarp();
    }
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
    const long tiles = (n + RS_TILE - 1) / RS_TILE;
    const int passes = (bits + 7) / 8;
    if (passes > 4)
    {
        set_error("radix sort: %d key bits (at most 32)", bits);
        return QZ_FAILURE;
    }
    // global digit counts of every pass (S.hist holds at least 4 x 256 ints)
    cudaMemsetAsync(S.hist, 0, (size_t)passes * RS_RADIX * sizeof(int), s->stream);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const int hb = (int)std::min<long>(2L * sms, (n + 1023) / 1024);
    launch(s, QZ_PROF_SORT, 4.0 * n, k_rs_hist, dim3(hb), dim3(256), ki, n, passes, S.hist);
    for (int p = 0; p < passes; p++)
    {
        if (scan_prepare(s, tiles * RS_RADIX))
            return QZ_FAILURE;
        launch(s, QZ_PROF_SORT, 16.0 * n, k_rs_onesweep, dim3((int)tiles), dim3(RS_WARPS * 32), ki,
               vi, ko, vo, n, 8 * p, S.hist + p * RS_RADIX, s->scan_st, s->scan_st + s->scan_st_cap,
               s->scan_base, s->scan_epoch, s->flags);
        s->scan_base += (unsigned long long)tiles;
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

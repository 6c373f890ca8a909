// qz_observe.cu -- quantities the reference's main loop computes on the host
// from the particle state every step, here reduced on the device:
//   qz_timestep   the CFL time step (timestep.c:589-700 with the per-node helpers
//                 :35-587); min / max of non-negative doubles are taken on their
//                 bit patterns with integer atomics, so the result is exact and
//                 does not depend on the order of the reduction.
//   qz_observables energies and momentum (observables.c:661-696): kinetic
//                 energy, potential energy exact (pairs) or from the potential
//                 grid, momentum.
#include <stdio.h>
#include <string.h>

#include <vector>

#include "qz_internal.cuh"

namespace qz {

constexpr int TS_MAX_LEVELS = 16;

struct TsArgs {
    long n;
    const double *vx, *vy, *vz, *ax, *ay, *az;
    const int *node_of[TS_MAX_LEVELS]; // levels >= 1: node of each particle or -1
    int nlev, lmin, method;
    double cfl, max_dt;
    unsigned long long *out; // [0] min dt (method 1); [1 + l] max |v| of level l (method 0)
};

// timestep.c:92-157 for one axis: the step after which the particle has moved
// CFL * H, with the Taylor form where the square root would cancel.
__device__ __forceinline__ double ts_axis(double v, double a, double H, double cfl, double dt)
{
    if (fabs(a) < 1.0e-16)
    {
        if (fabs(v) > 1.0e-16)
        {
            const double aux = cfl * H / fabs(v);
            dt = dt < aux ? dt : aux;
        }
    }
    else
    {
        const double c = v * v + 2.0 * fabs(a) * H * cfl;
        double aux;
        if (1 - v * v / c > 1.0e-8)
            aux = (-fabs(v) + sqrt(c)) / fabs(a);
        else
        {
            const double eps = fabs(a * H * cfl / (v * v));
            aux = fabs(v / a) * (eps - eps * eps * 0.5);
        }
        dt = dt < aux ? dt : aux;
    }
    return dt;
}

__device__ __forceinline__ double warp_min_d(double v)
{
    for (int o = 16; o > 0; o >>= 1)
    {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

__device__ __forceinline__ double warp_max_d(double v)
{
    for (int o = 16; o > 0; o >>= 1)
    {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w > v ? w : v;
    }
    return v;
}

// Each particle belongs to its finest node: a node's helper visits only the
// particles of its cells that are not refined (timestep.c:220-290, 396-560).
__global__ void k_timestep(TsArgs A)
{
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < A.n;
    int l = 0;
    double dt = A.max_dt, vmax = 0.0;
    if (live)
    {
        for (l = A.nlev - 1; l > 0; l--)
            if (A.node_of[l][i] >= 0)
                break;
        const double H = 1.0 / (1 << (A.lmin + l));
        const double vx = A.vx[i], vy = A.vy[i], vz = A.vz[i];
        if (A.method == 1)
        {
            dt = ts_axis(vx, A.ax[i], H, A.cfl, dt);
            dt = ts_axis(vy, A.ay[i], H, A.cfl, dt);
            dt = ts_axis(vz, A.az[i], H, A.cfl, dt);
        }
        else
        {
            vmax = fabs(vx);
            vmax = vmax < fabs(vy) ? fabs(vy) : vmax;
            vmax = vmax < fabs(vz) ? fabs(vz) : vmax;
        }
    }
    const int lane = threadIdx.x & 31;
    if (A.method == 1)
    {
        dt = warp_min_d(dt);
        if (lane == 0)
            atomicMin(&A.out[0], (unsigned long long)__double_as_longlong(dt));
    }
    else
        for (int lev = 0; lev < A.nlev; lev++)
        {
            const double m = warp_max_d(live && l == lev ? vmax : 0.0);
            if (lane == 0 && m > 0.0)
                atomicMax(&A.out[1 + lev], (unsigned long long)__double_as_longlong(m));
        }
}

int timestep_cfl(qz_sim *s, double *dt_out)
{
    const qz_config &c = s->cfg;
    const int nlev = c.lmax > c.lmin ? s->amr_nlev : 1;
    if (nlev > TS_MAX_LEVELS || !s->d_ts || !s->h_ts)
    {
        set_error("timestep: unsupported level count or missing buffers");
        return QZ_FAILURE;
    }
    TsArgs A{};
    A.n = s->n;
    A.vx = s->vx;
    A.vy = s->vy;
    A.vz = s->vz;
    A.ax = s->ax;
    A.ay = s->ay;
    A.az = s->az;
    for (int l = 1; l < nlev; l++)
        A.node_of[l] = s->node_of[l].p;
    A.nlev = nlev;
    A.lmin = c.lmin;
    A.method = c.time_step_method;
    A.cfl = c.cfl;
    A.max_dt = c.max_dt;
    A.out = s->d_ts;
    // out[0] starts at +inf's bits above any dt; the maxima start at 0
    unsigned long long init[1 + TS_MAX_LEVELS];
    memcpy(&init[0], &c.max_dt, sizeof c.max_dt);
    for (int l = 0; l < TS_MAX_LEVELS; l++)
        init[1 + l] = 0ULL;
    memcpy(s->h_ts, init, sizeof init);
    if (!check_cuda(cudaMemcpyAsync(s->d_ts, s->h_ts, sizeof init, cudaMemcpyHostToDevice,
                                    s->stream), "timestep init"))
        return QZ_FAILURE;
    if (s->n > 0)
        launch(s, QZ_PROF_OTHER, 48.0 * s->n, k_timestep, dim3(blocks_for(s->n, 256)), dim3(256), A);
    if (!check_cuda(cudaMemcpyAsync(s->h_ts + 1 + TS_MAX_LEVELS, s->d_ts, sizeof init,
                                    cudaMemcpyDeviceToHost, s->stream), "timestep read") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "timestep sync"))
        return QZ_FAILURE;
    const unsigned long long *r = s->h_ts + 1 + TS_MAX_LEVELS;
    double dt;
    if (c.time_step_method == 1)
        memcpy(&dt, &r[0], sizeof dt);
    else
    {
        // timestep.c:35-72 per node; the per-node step does not grow with the node's
        // largest speed, so the level maximum gives the minimum over the level's nodes
        dt = c.max_dt;
        for (int l = 0; l < nlev; l++)
        {
            double vmax;
            memcpy(&vmax, &r[1 + l], sizeof vmax);
            const double H = 1.0 / (1 << (c.lmin + l));
            const double d = vmax < (c.cfl * H / c.max_dt) ? c.max_dt : (c.cfl * H / vmax);
            dt = dt > d ? d : dt;
        }
    }
    *dt_out = dt;
    return QZ_SUCCESS;
}

} // namespace qz

using namespace qz;

extern "C" QZ_API int qz_timestep(qz_sim *s, double *dt)
{
    if (!s || !dt)
    {
        set_error("qz_timestep: bad arguments");
        return QZ_FAILURE;
    }
    return timestep_cfl(s, dt);
}

// ---- observables (observables.c:661-696) ----------------------------------------------
// Energies and momentum of the particle state.  Every sum is a fixed-order
// reduction: per-block partials in block order (added on the host), so the
// results are bit-reproducible; the reference adds in its own loop order, so
// parity is to rounding.
namespace qz {

constexpr int OBS_THREADS = 256;

__device__ __forceinline__ double obs_block_sum(double v, double *sh)
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

// observables.c:38-75 and :620-659: per block, sum m |v_c|^2 and m v_c with
// v_c = v / conversion_velocity + cm_v.
__global__ void k_kin_mom(long n, const double *__restrict__ vx, const double *__restrict__ vy,
                          const double *__restrict__ vz, const double *__restrict__ m, double cv,
                          double cmx, double cmy, double cmz, double *__restrict__ part)
{
    __shared__ double sh[32];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double k = 0.0, px = 0.0, py = 0.0, pz = 0.0;
    if (i < n)
    {
        const double cx = vx[i] / cv + cmx, cy = vy[i] / cv + cmy, cz = vz[i] / cv + cmz;
        const double v2 = cx * cx + cy * cy + cz * cz;
        k = m[i] * v2;
        px = m[i] * cx;
        py = m[i] * cy;
        pz = m[i] * cz;
    }
    const double a = obs_block_sum(k, sh), b = obs_block_sum(px, sh), c = obs_block_sum(py, sh),
                 d = obs_block_sum(pz, sh);
    if (threadIdx.x == 0)
    {
        part[4 * blockIdx.x + 0] = a;
        part[4 * blockIdx.x + 1] = b;
        part[4 * blockIdx.x + 2] = c;
        part[4 * blockIdx.x + 3] = d;
    }
}

// observables.c:77-112: sum over pairs j < i of m_i m_j / |x_i - x_j|.  Thread i
// adds its partners in increasing j (tiles of j staged in shared memory).
__global__ void __launch_bounds__(OBS_THREADS)
    k_pot_exact(long n, const double *__restrict__ x, const double *__restrict__ y,
                const double *__restrict__ z, const double *__restrict__ m,
                double *__restrict__ part)
{
    __shared__ double tx[OBS_THREADS], ty[OBS_THREADS], tz[OBS_THREADS], tm[OBS_THREADS];
    __shared__ double sh[32];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const double xi = live ? x[i] : 0.0, yi = live ? y[i] : 0.0, zi = live ? z[i] : 0.0,
                 mi = live ? m[i] : 0.0;
    const long iend = min(n, (long)(blockIdx.x + 1) * blockDim.x); // last i of the block + 1
    double sum = 0.0;
    for (long j0 = 0; j0 < iend; j0 += OBS_THREADS)
    {
        const long j = j0 + threadIdx.x;
        if (j < n)
        {
            tx[threadIdx.x] = x[j];
            ty[threadIdx.x] = y[j];
            tz[threadIdx.x] = z[j];
            tm[threadIdx.x] = m[j];
        }
        __syncthreads();
        const long jmax = live ? min((long)OBS_THREADS, i - j0) : 0;
        for (long q = 0; q < jmax; q++)
        {
            const double dx = xi - tx[q], dy = yi - ty[q], dz = zi - tz[q];
            double dist = dx * dx + dy * dy + dz * dz;
            dist = sqrt(dist);
            sum += mi * tm[q] / dist;
        }
        __syncthreads();
    }
    const double t = obs_block_sum(sum, sh);
    if (threadIdx.x == 0)
        part[blockIdx.x] = t;
}

// observables.c:115-203 (head only): sum of m * CIC-interpolated potential.
__global__ void k_pot_cic_head(long n, int L, long D, const double *__restrict__ pot,
                               const double *__restrict__ x, const double *__restrict__ y,
                               const double *__restrict__ z, const double *__restrict__ m,
                               double *__restrict__ part)
{
    __shared__ double sh[32];
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    double e = 0.0;
    if (i < n)
    {
        const double sc = (double)(1 << L);
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
        // box_ts = -1: grid index of level point f is f + 1
        const long g = (fx + 1) + (fy + 1) * D + (fz + 1) * D * D;
        double a = 0.0;
        for (int kk = 0; kk < 2; kk++)
            for (int jj = 0; jj < 2; jj++)
                for (int ii = 0; ii < 2; ii++)
                    a += pot[g + ii + jj * D + kk * D * D] * w[ii + 2 * jj + 4 * kk];
        e = m[i] * a;
    }
    const double t = obs_block_sum(e, sh);
    if (threadIdx.x == 0)
        part[blockIdx.x] = t;
}

int amr_pot_energy_partials(qz_sim *s, double *part); // qz_amr.cu

static bool obs_read_sum(qz_sim *s, const double *dpart, long count, int stride, double *sums)
{
    std::vector<double> h(count * stride);
    if (!check_cuda(cudaMemcpyAsync(h.data(), dpart, h.size() * sizeof(double),
                                    cudaMemcpyDeviceToHost, s->stream), "observables read") ||
        !check_cuda(cudaStreamSynchronize(s->stream), "observables sync"))
        return false;
    for (int c = 0; c < stride; c++)
        sums[c] = 0.0;
    for (long b = 0; b < count; b++)
        for (int c = 0; c < stride; c++)
            sums[c] += h[b * stride + c];
    return true;
}

int observables(qz_sim *s, int potential_type, const double *units, double *out)
{
    const double cv = units ? units[0] : 1.0, ct = units ? units[1] : 1.0,
                 cd = units ? units[2] : 1.0;
    const double cmx = units ? units[3] : 0.0, cmy = units ? units[4] : 0.0,
                 cmz = units ? units[5] : 0.0;
    const long n = s->n;
    const int nb = blocks_for(n > 0 ? n : 1, OBS_THREADS);
    double *part = nullptr;
    if (!pool_alloc(s->mem, &part, 4L * nb))
    {
        set_error("observables: out of device memory");
        return QZ_FAILURE;
    }
    double km[4] = {0, 0, 0, 0}, w = 0.0;
    bool ok = true;
    if (n > 0)
    {
        launch(s, QZ_PROF_OTHER, 32.0 * n, k_kin_mom, dim3(nb), dim3(OBS_THREADS), n, s->vx, s->vy,
               s->vz, s->m, cv, cmx, cmy, cmz, part);
        ok = obs_read_sum(s, part, nb, 4, km);
        if (ok && potential_type == 0)
        {
            launch(s, QZ_PROF_OTHER, 32.0 * n, k_pot_exact, dim3(nb), dim3(OBS_THREADS), n, s->x,
                   s->y, s->z, s->m, part);
            ok = obs_read_sum(s, part, nb, 1, &w);
        }
        else if (ok)
        {
            if (s->cfg.lmax > s->cfg.lmin)
                ok = amr_pot_energy_partials(s, part) == QZ_SUCCESS;
            else
                launch(s, QZ_PROF_OTHER, 96.0 * n, k_pot_cic_head, dim3(nb), dim3(OBS_THREADS), n,
                       s->L, s->D, s->pot, s->x, s->y, s->z, s->m, part);
            ok = ok && obs_read_sum(s, part, nb, 1, &w);
        }
    }
    pool_free(s->mem, part);
    if (!ok || !check_cuda(cudaGetLastError(), "observables"))
        return QZ_FAILURE;
    const double G = s->cfg.G;
    out[0] = km[0] * 0.5;
    // observables.c:108-111 (exact) and :614-617 (grid approximation)
    out[1] = potential_type == 0 ? -w * G * (ct * ct) / (cd * cd) : w * 0.5 * G * (ct * ct) / (cd * cd);
    out[2] = out[0] + out[1];
    out[3] = km[1];
    out[4] = km[2];
    out[5] = km[3];
    return QZ_SUCCESS;
}

} // namespace qz

extern "C" QZ_API int qz_observables(qz_sim *s, int potential_type, const double *units,
                                     double *out)
{
    if (!s || !out || (potential_type != 0 && potential_type != 1))
    {
        set_error("qz_observables: bad arguments");
        return QZ_FAILURE;
    }
    return observables(s, potential_type, units, out);
}

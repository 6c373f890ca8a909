// qz_observe.cu -- quantities the reference's main loop computes on the host
// from the particle state every step, here reduced on the device:
//   qz_timestep   the CFL time step (timestep.c:589-700 with the per-node helpers
//                 :35-587); min / max of non-negative doubles are taken on their
//                 bit patterns with integer atomics, so the result is exact and
//                 does not depend on the order of the reduction.
#include <stdio.h>
#include <string.h>

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

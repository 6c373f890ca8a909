// qz_snapshot.cu -- snapshot files of output_snapshots.c:141-239 written from the
// device-resident state.
//
// File layout (native-endian float64): m[N], then x, y, z, vx, vy, vz in user
// units, then energies[3] and momentum[3] when observables are requested, then
// the time real_time = actual_time / conversion_time.  Conversion, per
// particle, in the reference's expression order:
//   x_user = (x - 0.5) / conversion_dist + cm_x + cm_vx * real_time
//   v_user = vx / conversion_velocity + cm_vx
// One kernel converts the state into a device staging buffer; a second stream
// copies it into pinned host memory and a host thread writes the file, so the
// step loop on the simulation's stream is not held up by the copy or the disk.
#include "qz_internal.cuh"

#include <string>
#include <thread>

namespace qz {

struct Snapshot {
    double *stage = nullptr; // device: 7 n
    long stage_cap = 0;
    double *host = nullptr;  // pinned: 7 n + 7
    long host_cap = 0;
    cudaStream_t copy = nullptr;
    cudaEvent_t converted = nullptr, copied = nullptr;
    std::thread writer;
    bool busy = false;
    int status = QZ_SUCCESS;
    std::string error;
};

__global__ void k_snapshot_convert(long n, const double *__restrict__ x,
                                   const double *__restrict__ y, const double *__restrict__ z,
                                   const double *__restrict__ vx, const double *__restrict__ vy,
                                   const double *__restrict__ vz, const double *__restrict__ m,
                                   double cd, double cv, double cmx, double cmy, double cmz,
                                   double cmvx, double cmvy, double cmvz, double rt,
                                   double *__restrict__ out)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    out[i] = m[i];
    out[n + i] = (x[i] - 0.5) / cd + cmx + cmvx * rt;
    out[2 * n + i] = (y[i] - 0.5) / cd + cmy + cmvy * rt;
    out[3 * n + i] = (z[i] - 0.5) / cd + cmz + cmvz * rt;
    out[4 * n + i] = vx[i] / cv + cmvx;
    out[5 * n + i] = vy[i] / cv + cmvy;
    out[6 * n + i] = vz[i] / cv + cmvz;
}

// Joins a pending write; returns its status.
static int snapshot_join(Snapshot &S)
{
    if (S.writer.joinable())
        S.writer.join();
    S.busy = false;
    if (S.status != QZ_SUCCESS)
    {
        set_error("%s", S.error.c_str());
        S.status = QZ_SUCCESS;
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

void snapshot_free(qz_sim *s)
{
    Snapshot *S = s->snap;
    if (!S)
        return;
    snapshot_join(*S);
    if (S->stage)
        cudaFree(S->stage);
    if (S->host)
        cudaFreeHost(S->host);
    if (S->converted)
        cudaEventDestroy(S->converted);
    if (S->copied)
        cudaEventDestroy(S->copied);
    if (S->copy)
        cudaStreamDestroy(S->copy);
    delete S;
    s->snap = nullptr;
}

static void write_file(Snapshot *S, std::string path, long n, int nobs)
{
    if (cudaEventSynchronize(S->copied) != cudaSuccess)
    {
        S->status = QZ_FAILURE;
        S->error = "snapshot: device to host copy failed";
        return;
    }
    FILE *f = fopen(path.c_str(), "wb");
    if (!f)
    {
        S->status = QZ_FAILURE;
        S->error = "snapshot: cannot open " + path;
        return;
    }
    const size_t count = (size_t)(7 * n + nobs + 1);
    const bool ok = fwrite(S->host, sizeof(double), count, f) == count;
    if (fclose(f) != 0 || !ok)
    {
        S->status = QZ_FAILURE;
        S->error = "snapshot: short write to " + path;
    }
}

} // namespace qz

using namespace qz;

extern "C" {

int qz_write_snapshot(qz_sim *s, const char *path, double actual_time, const double *units,
                      int observables_type, int async)
{
    if (!s || !path || observables_type < -1 || observables_type > 1)
    {
        set_error("qz_write_snapshot: bad arguments");
        return QZ_FAILURE;
    }
    if (!s->snap)
        s->snap = new Snapshot();
    Snapshot &S = *s->snap;
    if (snapshot_join(S))
        return QZ_FAILURE; // the previous file failed: report it once
    const long n = s->n;
    // units: conversion_dist, conversion_velocity, conversion_time, cm x y z, cm vx vy vz
    double u[9] = {1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    if (units)
        memcpy(u, units, sizeof u);
    const double real_time = actual_time / u[2];
    double obs[6] = {0, 0, 0, 0, 0, 0};
    const int nobs = observables_type >= 0 ? 6 : 0;
    if (nobs)
    {
        // observables.c:661-696 in user units: {conversion_velocity, conversion_time,
        // conversion_dist, cm_vx, cm_vy, cm_vz}
        const double ou[6] = {u[1], u[2], u[0], u[6], u[7], u[8]};
        if (qz_observables(s, observables_type, ou, obs))
            return QZ_FAILURE;
    }
    const long need = 7 * (n > 0 ? n : 1);
    if (S.stage_cap < need)
    {
        if (S.stage)
            cudaFree(S.stage);
        S.stage = nullptr;
        S.stage_cap = 0;
        if (!check_cuda(cudaMalloc((void **)&S.stage, need * sizeof(double)), "snapshot stage"))
            return QZ_FAILURE;
        S.stage_cap = need;
    }
    if (S.host_cap < need + 7)
    {
        if (S.host)
            cudaFreeHost(S.host);
        S.host = nullptr;
        S.host_cap = 0;
        if (!check_cuda(cudaMallocHost((void **)&S.host, (need + 7) * sizeof(double)),
                        "snapshot pinned"))
            return QZ_FAILURE;
        S.host_cap = need + 7;
    }
    if (!S.copy &&
        (!check_cuda(cudaStreamCreateWithFlags(&S.copy, cudaStreamNonBlocking), "snapshot stream") ||
         !check_cuda(cudaEventCreateWithFlags(&S.converted, cudaEventDisableTiming), "event") ||
         !check_cuda(cudaEventCreateWithFlags(&S.copied, cudaEventDisableTiming), "event")))
        return QZ_FAILURE;
    if (n > 0)
        launch(s, QZ_PROF_OTHER, 104.0 * n, k_snapshot_convert, dim3(blocks_for(n, 256)),
               dim3(256), n, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->m, u[0], u[1], u[3], u[4],
               u[5], u[6], u[7], u[8], real_time, S.stage);
    if (!check_cuda(cudaEventRecord(S.converted, s->stream), "snapshot event") ||
        !check_cuda(cudaStreamWaitEvent(S.copy, S.converted, 0), "snapshot wait") ||
        !check_cuda(cudaMemcpyAsync(S.host, S.stage, 7 * n * sizeof(double),
                                    cudaMemcpyDeviceToHost, S.copy),
                    "snapshot copy") ||
        !check_cuda(cudaEventRecord(S.copied, S.copy), "snapshot event"))
        return QZ_FAILURE;
    for (int q = 0; q < nobs; q++)
        S.host[7 * n + q] = obs[q];
    S.host[7 * n + nobs] = real_time;
    S.busy = true;
    S.writer = std::thread(write_file, &S, std::string(path), n, nobs);
    return async ? QZ_SUCCESS : snapshot_join(S);
}

int qz_snapshot_wait(qz_sim *s)
{
    if (!s)
        return QZ_FAILURE;
    return s->snap ? snapshot_join(*s->snap) : QZ_SUCCESS;
}

} // extern "C"

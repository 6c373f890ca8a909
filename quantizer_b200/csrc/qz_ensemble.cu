// qz_ensemble.cu -- the batching form: many independent simulations (for
// example an ensemble of initial conditions) stepped together on one GPU.
//
// One simulation's step is a chain of short kernels and a few host
// synchronisations (tree sizes, convergence checks); on its own it leaves most
// of the GPU idle.  Every qz_sim owns its stream (device memory comes from the
// device's shared stream-ordered pool), so the simulations of an ensemble are
// stepped concurrently by a pool of host threads: each thread takes the next simulation (atomic counter) and runs its
// steps, and the chains of different simulations overlap on the GPU.  Every
// simulation computes exactly what it computes alone (its kernels and their
// order are unchanged), so results do not depend on the number of threads.
#include <atomic>
#include <chrono>
#include <mutex>
#include <stdio.h>
#include <string.h>
#include <string>
#include <thread>
#include <vector>

#include "qz_internal.cuh"

using namespace qz;

extern "C" QZ_API int qz_ensemble_step(qz_sim **sims, int nsims, const double *dt, int nsteps,
                                       int nthreads)
{
    if (!sims || nsims < 0 || nsteps < 0)
    {
        set_error("qz_ensemble_step: bad arguments");
        return QZ_FAILURE;
    }
    for (int k = 0; k < nsims; k++)
        if (!sims[k])
        {
            set_error("qz_ensemble_step: simulation %d is null", k);
            return QZ_FAILURE;
        }
    if (nthreads < 1)
        nthreads = 1;
    if (nthreads > nsims)
        nthreads = nsims > 0 ? nsims : 1;
    // members run side by side already: each keeps its stages on its own stream
    for (int k = 0; k < nsims; k++)
        sims[k]->no_overlap = true;
    std::atomic<int> next{0};
    std::atomic<int> failed{-1};
    std::mutex mu;
    std::string first_error;
    auto worker = [&]() {
        for (;;)
        {
            const int k = next.fetch_add(1);
            if (k >= nsims || failed.load() >= 0)
                return;
            qz_sim *s = sims[k];
            int rc = cudaSetDevice(s->device) == cudaSuccess ? QZ_SUCCESS : QZ_FAILURE;
            if (rc == QZ_SUCCESS)
                rc = qz_step(s, dt ? dt[k] : 0.0, nsteps);
            if (rc == QZ_SUCCESS)
                rc = qz_synchronize(s);
            if (rc != QZ_SUCCESS)
            {
                int none = -1;
                if (failed.compare_exchange_strong(none, k))
                {
                    std::lock_guard<std::mutex> lock(mu);
                    first_error = qz_last_error();
                }
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nthreads; t++)
        pool.emplace_back(worker);
    worker();
    for (auto &th : pool)
        th.join();
    for (int k = 0; k < nsims; k++)
        sims[k]->no_overlap = false;
    if (failed.load() >= 0)
    {
        set_error("qz_ensemble_step: simulation %d: %s", failed.load(), first_error.c_str());
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

extern "C" QZ_API int qz_ensemble_autotune(qz_sim **sims, int nsims, const double *dt,
                                           const int *thread_opts, int nthread_opts,
                                           const int *ppt_opts, int nppt_opts,
                                           const int *tile_opts, int ntile_opts, int *best_threads,
                                           int *best_ppt, int *best_tile, double *best_ms)
{
    if (!sims || nsims < 1 || !thread_opts || nthread_opts < 1 || !ppt_opts || nppt_opts < 1 ||
        !tile_opts || ntile_opts < 1)
    {
        set_error("qz_ensemble_autotune: bad arguments");
        return QZ_FAILURE;
    }
    for (int a = 0; a < ntile_opts; a++)
        if (tile_opts[a] < -1 || tile_opts[a] > QZ_MG_NTILES)
        {
            set_error("qz_ensemble_autotune: tile option %d out of range", tile_opts[a]);
            return QZ_FAILURE;
        }
    std::vector<SavedState> saved(nsims);
    auto restore_all = [&]() {
        for (int k = 0; k < nsims; k++)
            if (!state_restore(sims[k], saved[k]) || qz_synchronize(sims[k]))
                return false;
        return true;
    };
    int rc = QZ_SUCCESS;
    for (int k = 0; k < nsims && rc == QZ_SUCCESS; k++)
    {
        if (!sims[k] || (!sims[k]->forces_ready && qz_init_forces(sims[k])) ||
            !state_save(sims[k], saved[k]) || qz_synchronize(sims[k]))
            rc = QZ_FAILURE;
    }
    int bt = thread_opts[0], bp = ppt_opts[0], bl = tile_opts[0];
    double bms = 1e300;
    for (int g = 0; g < ntile_opts && rc == QZ_SUCCESS; g++)
        for (int a = 0; a < nppt_opts && rc == QZ_SUCCESS; a++)
        {
            for (int k = 0; k < nsims; k++)
            {
                sims[k]->cfg.mg_points_per_thread = ppt_opts[a];
                sims[k]->cfg.mg_tile = tile_opts[g];
            }
            for (int b = 0; b < nthread_opts && rc == QZ_SUCCESS; b++)
            {
                const auto t0 = std::chrono::steady_clock::now();
                rc = qz_ensemble_step(sims, nsims, dt, 1, thread_opts[b]);
                const double ms =
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                        .count();
                if (rc == QZ_SUCCESS && ms < bms)
                {
                    bms = ms;
                    bt = thread_opts[b];
                    bp = ppt_opts[a];
                    bl = tile_opts[g];
                }
                if (rc == QZ_SUCCESS && !restore_all())
                    rc = QZ_FAILURE;
            }
        }
    for (int k = 0; k < nsims; k++)
    {
        sims[k]->cfg.mg_points_per_thread = bp;
        sims[k]->cfg.mg_tile = bl;
        state_free(sims[k], saved[k]);
    }
    if (rc != QZ_SUCCESS)
        return QZ_FAILURE;
    if (best_threads)
        *best_threads = bt;
    if (best_ppt)
        *best_ppt = bp;
    if (best_tile)
        *best_tile = bl;
    if (best_ms)
        *best_ms = bms;
    return QZ_SUCCESS;
}

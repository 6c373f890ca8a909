// qz_testhooks.cu -- entry points that exist for the library's own tests
// (declared at the end of include/qz_b200.h; no counterpart in the reference).
//
//   qz_test_scan         the single-pass exclusive scan on host arrays, in place
//                        or not, optionally from a chosen epoch (to cross the
//                        epoch wrap)
//   qz_test_wait_gives_up  runs one bounded wait that cannot be satisfied --
//                        the scan's look-back on a tile that is never
//                        published, or the cooperative kernels' grid barrier
//                        with an arrival count that no block completes -- so
//                        that the give-up path (error bit, kernel returns,
//                        QZ_FAILURE with the message) is exercised without a
//                        hang: each wait ends after its poll limit (a few
//                        seconds at most)
#include <vector>

#include "qz_internal.cuh"

namespace qz {

// Two grid barriers in one block: the first waits for arrivals that never come
// (word[0] starts at 1, so the block is never the last of gridDim.x = 1) and
// gives up; the second must return at once because the launch has given up.
__global__ void k_gbar_probe(GridBar B, int *out)
{
    __shared__ int ok;
    const bool first = gbar_sync(B, &ok);
    const bool second = gbar_sync(B, &ok);
    if (threadIdx.x == 0)
    {
        out[0] = first ? 1 : 0;
        out[1] = second ? 1 : 0;
    }
}

} // namespace qz

using namespace qz;

extern "C" {

int qz_test_scan(qz_sim *s, const int *in, int *out, long n, int in_place, unsigned epoch)
{
    if (!s || n < 0 || (n > 0 && (!in || !out)))
    {
        set_error("qz_test_scan: bad arguments");
        return QZ_FAILURE;
    }
    if (n == 0)
        return QZ_SUCCESS;
    DBuf<int> a, b;
    if (!a.ensure(s->mem, n) || (!in_place && !b.ensure(s->mem, n)))
    {
        a.release(s->mem);
        set_error("qz_test_scan: out of device memory");
        return QZ_FAILURE;
    }
    int *dout = in_place ? a.p : b.p;
    int rc = QZ_SUCCESS;
    if (!check_cuda(cudaMemcpyAsync(a.p, in, n * sizeof(int), cudaMemcpyHostToDevice, s->stream),
                    "scan input"))
        rc = QZ_FAILURE;
    if (rc == QZ_SUCCESS && epoch != 0)
        scan_set_epoch(s, epoch);
    if (rc == QZ_SUCCESS)
        rc = scan_exclusive(s, a.p, dout, n);
    if (rc == QZ_SUCCESS &&
        (!check_cuda(cudaMemcpyAsync(out, dout, n * sizeof(int), cudaMemcpyDeviceToHost, s->stream),
                     "scan output") ||
         !check_cuda(cudaStreamSynchronize(s->stream), "scan sync")))
        rc = QZ_FAILURE;
    if (rc == QZ_SUCCESS)
        rc = check_flags(s);
    a.release(s->mem);
    b.release(s->mem);
    return rc;
}

int qz_test_wait_gives_up(qz_sim *s, int which, int *out2)
{
    if (!s || (which != 0 && which != 1))
    {
        set_error("qz_test_wait_gives_up: bad arguments");
        return QZ_FAILURE;
    }
    if (which == 0)
    {
        if (scan_wait_probe(s))
            return QZ_FAILURE;
        if (!check_cuda(cudaStreamSynchronize(s->stream), "scan probe sync"))
            return QZ_FAILURE;
        if (out2)
            out2[0] = out2[1] = 0;
        return check_flags(s);
    }
    // barrier words: count, unused, generation, gave-up; then the probe's two results
    unsigned *w = nullptr;
    if (!pool_alloc(s->mem, &w, 8))
    {
        set_error("qz_test_wait_gives_up: out of device memory");
        return QZ_FAILURE;
    }
    const unsigned init[8] = {1u, 0u, 0u, 0u, 7u, 7u, 0u, 0u};
    int res[2] = {-1, -1};
    int rc = QZ_SUCCESS;
    if (!check_cuda(cudaMemcpyAsync(w, init, sizeof init, cudaMemcpyHostToDevice, s->stream),
                    "barrier probe words"))
        rc = QZ_FAILURE;
    if (rc == QZ_SUCCESS)
    {
        launch(s, QZ_PROF_OTHER, 0.0, k_gbar_probe, dim3(1), dim3(128), GridBar{w, s->flags},
               (int *)(w + 4));
        if (!check_cuda(cudaMemcpyAsync(res, w + 4, sizeof res, cudaMemcpyDeviceToHost, s->stream),
                        "barrier probe result") ||
            !check_cuda(cudaStreamSynchronize(s->stream), "barrier probe sync"))
            rc = QZ_FAILURE;
    }
    pool_free(s->mem, w);
    if (out2)
    {
        out2[0] = res[0];
        out2[1] = res[1];
    }
    if (rc != QZ_SUCCESS)
        return rc;
    return check_flags(s);
}

} // extern "C"

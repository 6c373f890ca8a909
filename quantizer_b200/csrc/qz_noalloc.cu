// qz_noalloc.cu -- weighted Jacobi smoothing on caller-owned device arrays with
// no device allocation at all (qz_jacobi_noalloc, include/qz_b200.h).
//
// The reference's jacobi() (force_methods/jacobi.c:62-82) copies phi into a
// malloc'ed buffer and ping-pongs between the two.  Here that buffer is a
// file-scope device array of fixed size: it is loaded with the module and
// held by every device that loads the library until the process exits, so a
// call allocates nothing.  Host code cannot use the array's name as a device
// address (in host code it names a host-side stand-in), so every call looks up
// the array's device address with cudaGetSymbolAddress, with the caller's
// device current, and passes it to the kernels.  The lookup allocates nothing
// and is not cached: an address kept from an earlier context (after
// cudaDeviceReset, the module is loaded again elsewhere) would be stale.  On
// the first call on a device the lookup also loads the module there, so make
// that first call before any stream capture.
//
// Every call shares the array and it keeps the last call's contents: each call
// first copies phi into it, so no state carries over between calls.  Calls
// that overlap on the GPU (two streams, or two host threads, at the same time
// on one device) race on the array and must be serialised by the caller.
#include <stdio.h>

#include "qz_internal.cuh"

#define QZ_NOALLOC_MAX_POINTS ((long)QZ_NOALLOC_MAX_GRID * QZ_NOALLOC_MAX_GRID * QZ_NOALLOC_MAX_GRID)

static __device__ __align__(256) double qz_noalloc_scratch[QZ_NOALLOC_MAX_POINTS];

namespace {

// Device address of the scratch array in the current device's context.
double *scratch_address()
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, qz_noalloc_scratch);
    if (e != cudaSuccess)
    {
        qz::set_error("qz_jacobi_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return nullptr;
    }
    return static_cast<double *>(p);
}

__global__ void k_na_copy(const double *__restrict__ src, double *__restrict__ dst, long n)
{
    long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        dst[i] = src[i];
}

// One Jacobi sweep over the interior of an n^3 grid, in the arithmetic of
// jacobi.c:44-51 (the library is built without fused multiply-add).
__global__ void k_na_jacobi(const double *__restrict__ oldp, double *__restrict__ newp,
                            const double *__restrict__ rho, int n, double C, double w)
{
    const int m = n - 2;
    int i = 1 + blockIdx.x * blockDim.x + threadIdx.x;
    int j = 1 + blockIdx.y, k = 1 + blockIdx.z;
    if (i > m)
        return;
    const long sy = n, sz = (long)n * n;
    const long g = i + j * sy + k * sz;
    const double one_sixth = 1.0 / 6.0;
    double a = one_sixth * (C * rho[g] + oldp[g + 1] + oldp[g - 1] + oldp[g + sy] + oldp[g - sy] +
                            oldp[g + sz] + oldp[g - sz]);
    newp[g] = w * a + (1.0 - w) * newp[g];
}

} // namespace

extern "C" int qz_jacobi_noalloc(double *phi, const double *rho, int gridsize, int iter_max,
                                 double w, void *stream)
{
    if (!phi || !rho || iter_max < 0)
    {
        qz::set_error("qz_jacobi_noalloc: bad arguments");
        return QZ_FAILURE;
    }
    if (gridsize < 3 || gridsize > QZ_NOALLOC_MAX_GRID)
    {
        qz::set_error("qz_jacobi_noalloc: gridsize %d outside 3..%d (the size of the library's "
                      "static scratch array)", gridsize, QZ_NOALLOC_MAX_GRID);
        return QZ_FAILURE;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
    {
        qz::set_error("qz_jacobi_noalloc: no usable CUDA device (%s)", cudaGetErrorString(e));
        return QZ_FAILURE;
    }
    double *scr = scratch_address();
    if (!scr)
        return QZ_FAILURE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = gridsize, m = n - 2;
    const long n3 = (long)n * n * n;
    // jacobi.c:62-82: the copy, then an even number of sweeps ending in phi
    k_na_copy<<<(unsigned)((n3 + 255) / 256), 256, 0, st>>>(phi, scr, n3);
    if (iter_max > 0)
    {
        const double C = -(1.0 / (n - 1)) * (1.0 / (n - 1));
        const int tx = m < 128 ? ((m + 31) / 32) * 32 : 128;
        const dim3 grid((m + tx - 1) / tx, m, m);
        const bool even = iter_max % 2 == 0;
        const int sweeps = even ? iter_max : iter_max + 1;
        double *a = even ? phi : scr;
        double *b = even ? scr : phi;
        for (int it = 0; it < sweeps; it++)
        {
            k_na_jacobi<<<grid, tx, 0, st>>>(a, b, rho, n, C, w);
            double *t = a;
            a = b;
            b = t;
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess)
    {
        qz::set_error("qz_jacobi_noalloc: launch failed: %s", cudaGetErrorString(e));
        return QZ_FAILURE;
    }
    return QZ_SUCCESS;
}

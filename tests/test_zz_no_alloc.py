"""qz_jacobi_noalloc: Jacobi smoothing on caller-owned device arrays that
allocates no device memory.

Some callers cannot allocate device memory -- code embedded in a framework
whose caching allocator already holds the device memory budget, or loops that
must not call cudaMalloc / cudaFree (which synchronise the whole device) once
running.  This entry point keeps its ping-pong copy in a fixed device array
inside the library instead.  The test calls it through the C ABI on device
arrays owned by the test, twice in a row (the shared array keeps the previous
call's contents, which must not leak into the next result), and compares each
result with the allocating entry point qz_jacobi on the same inputs, bit for bit
(the tolerance of the other Jacobi tests), at weights 1 and 0.7 (below 1 the
(1 - w) term reads the ping-pong copy's previous contents).  It lives in a file of its own that
pytest collects last.
"""
import ctypes as C

import numpy as np
import pytest

from quantizer_b200 import core

pytestmark = pytest.mark.gpu


def _lib():
    lib = core.load()
    lib.qz_jacobi_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_double,
                                      C.c_void_p]
    lib.qz_jacobi_noalloc.restype = C.c_int
    return lib


@pytest.mark.parametrize("n,iters,w", [(17, 3, 1.0), (33, 2, 1.0), (65, 5, 1.0), (33, 3, 0.7),
                                      (65, 4, 0.7)])
def test_noalloc_jacobi_matches_allocating_entry_point(n, iters, w):
    import torch
    lib = _lib()
    rng = np.random.default_rng(n)
    cases = [(rng.standard_normal(n ** 3), rng.standard_normal(n ** 3) * 10.0) for _ in range(2)]
    stream = torch.cuda.current_stream()
    for phi0, rho in cases:  # two calls in a row
        expected = core.jacobi(phi0, rho, iters, w)
        dphi = torch.tensor(phi0, dtype=torch.float64, device="cuda")
        drho = torch.tensor(rho, dtype=torch.float64, device="cuda")
        rc = lib.qz_jacobi_noalloc(dphi.data_ptr(), drho.data_ptr(), n, iters, w,
                                   stream.cuda_stream)
        assert rc == 0, lib.qz_last_error().decode()
        stream.synchronize()
        np.testing.assert_array_equal(dphi.cpu().numpy(), expected)


def test_noalloc_jacobi_rejects_grids_beyond_its_array():
    import torch
    lib = _lib()
    n = 67
    d = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    rc = lib.qz_jacobi_noalloc(d.data_ptr(), d.data_ptr(), n, 2, 1.0, None)
    assert rc == 1
    assert "gridsize" in lib.qz_last_error().decode()

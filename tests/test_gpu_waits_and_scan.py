"""The device scan and the bounded waits, through the test hooks of the C ABI.

* qz_test_scan: the single-pass exclusive scan (decoupled look-back with
  arrival-ordered tiles, status words tagged by a per-call epoch) against
  numpy for one tile, the tile edges and many tiles, in place and not, many
  calls on one context with a growing n (so the status-word buffer is
  reallocated and the tile counter restarts), and across the epoch wrap.
* qz_test_wait_gives_up: a look-back wait on a tile that is never published,
  and a grid barrier whose arrivals never complete, each end at their poll
  limit: the error bit is set, the kernel returns, the call returns
  QZ_FAILURE with the wait's message, and the simulation keeps working.
"""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

TILE = 4096  # elements per scan tile (SC_TILE in qz_sort.cu)


@pytest.fixture(scope="module")
def sim():
    ic = ics.plummer(1000, a=0.05, seed=3)
    s = core.Simulation(ic, 4)
    yield s
    s.close()


def _scan(sim, a, in_place=False, epoch=0):
    a = np.ascontiguousarray(a, dtype=np.int32)
    out = np.empty_like(a)
    rc = sim.lib.qz_test_scan(sim.h, core._p(a), core._p(out), a.size, int(in_place), epoch)
    assert rc == 0, sim.lib.qz_last_error().decode()
    return out


def _expected(a):
    e = np.zeros_like(a, dtype=np.int64)
    e[1:] = np.cumsum(a[:-1].astype(np.int64))
    return e.astype(np.int32)


@pytest.mark.parametrize("n", [1, TILE - 1, TILE, TILE + 1, 3 * TILE + 17, 3_000_000])
@pytest.mark.parametrize("in_place", [False, True])
def test_scan_matches_numpy(sim, n, in_place):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 50, n).astype(np.int32)
    np.testing.assert_array_equal(_scan(sim, a, in_place), _expected(a))


def test_scan_many_calls_with_growing_sizes(sim):
    rng = np.random.default_rng(5)
    n = 10
    for _ in range(40):
        a = rng.integers(0, 9, n).astype(np.int32)
        np.testing.assert_array_equal(_scan(sim, a), _expected(a))
        n = int(n * 1.4) + 3


def test_scan_across_the_epoch_wrap(sim):
    rng = np.random.default_rng(9)
    a = rng.integers(0, 100, 5 * TILE + 3).astype(np.int32)
    # the next call takes epoch 2^30 - 1, the one after wraps to 1 (old words cleared)
    np.testing.assert_array_equal(_scan(sim, a, epoch=(1 << 30) - 2), _expected(a))
    for _ in range(3):
        b = rng.integers(0, 100, 5 * TILE + 3).astype(np.int32)
        np.testing.assert_array_equal(_scan(sim, b), _expected(b))


def test_scan_lookback_wait_gives_up(sim):
    res = (core.C.c_int * 2)()
    rc = sim.lib.qz_test_wait_gives_up(sim.h, 0, res)
    assert rc == 1
    assert "scan's wait" in sim.lib.qz_last_error().decode()
    # the context is still usable: a scan afterwards is right
    a = np.arange(2 * TILE + 5, dtype=np.int32) % 7
    np.testing.assert_array_equal(_scan(sim, a), _expected(a))


def test_grid_barrier_wait_gives_up(sim):
    res = (core.C.c_int * 2)()
    rc = sim.lib.qz_test_wait_gives_up(sim.h, 1, res)
    assert rc == 1
    assert "grid barrier" in sim.lib.qz_last_error().decode()
    # the first barrier gave up; the second returned at once, also false
    assert list(res) == [0, 0]
    # the simulation still steps afterwards
    sim.init_forces()
    sim.step(1e-5, 1)
    assert sim.stats().steps >= 1

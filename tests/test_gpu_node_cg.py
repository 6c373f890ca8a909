"""qz_node_conjugate_gradient -- the node conjugate gradient on one node given
as host arrays, the call behind the drop-in's conjugate_gradient(struct node *)
-- against the reference's own conjugate_gradient (force_methods/
conjugate_gradient.c:322-463) on a synthetic node (tests/golden/node_cg.npz,
made by tests/golden/make_golden.py through the compiled reference).

Bars: the solution within 1e-9 of max |pot| (the device sums in chunk order,
the reference sequentially; both stop at the same checks), pot_old within the
same bar, and the call's success code equal to the reference's.
"""
import ctypes as C

import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def test_node_conjugate_gradient_matches_reference(request):
    from conftest import golden
    z = golden("node_cg.npz")
    lib = core.load()
    ic = ics.plummer(100, a=0.05, seed=1)
    with core.Simulation(ic, 4) as sim:
        pot = z["pot_in"].copy()
        pot_old = z["pot_in"].copy()
        d = z["d"].copy()
        intr = z["intr"].astype(np.int32)
        rd = [int(v) for v in z["rd"]]
        P = C.POINTER(C.c_double)
        rc = lib.qz_node_conjugate_gradient(
            sim.h, int(z["lv"][0]), rd[0], rd[1], rd[2], intr.size,
            intr.ctypes.data_as(C.POINTER(C.c_int)), float(z["mass"][0]), int(z["cells"][0]),
            d.ctypes.data_as(P), pot.ctypes.data_as(P), pot_old.ctypes.data_as(P))
        assert rc == int(z["rc"][0]), lib.qz_last_error().decode()
        assert sim.stats().cg_iterations > 0
    scale = np.abs(z["pot_out"]).max()
    assert np.abs(pot - z["pot_out"]).max() < 1e-9 * scale
    assert np.abs(pot_old - z["pot_old_out"]).max() < 1e-9 * scale


def test_node_conjugate_gradient_rejects_a_list_outside_the_grid():
    lib = core.load()
    ic = ics.plummer(100, a=0.05, seed=1)
    with core.Simulation(ic, 4) as sim:
        n = 9 ** 3
        a = np.zeros(n)
        intr = np.array([0], dtype=np.int32)  # the first point has no -x neighbour
        P = C.POINTER(C.c_double)
        rc = lib.qz_node_conjugate_gradient(sim.h, 5, 8, 8, 8, 1,
                                            intr.ctypes.data_as(C.POINTER(C.c_int)), 1.0, 64,
                                            a.ctypes.data_as(P), a.ctypes.data_as(P),
                                            a.ctypes.data_as(P))
        assert rc == 1
        assert "outside" in lib.qz_last_error().decode()

"""The head solve beside the tree construction (tree_overlap).

In refinement runs whose head solve is one persistent launch, qz_step runs
that launch on a second stream while the tree is built and the levels are
deposited on the simulation's stream.  No kernel's inputs change with the
schedule, so a run with tree_overlap = 1 must equal the sequential run
(tree_overlap = 0, main.c's stage order) bit for bit: positions, velocities,
accelerations, the head potential, the tree, and the solver statistics, in the
FP64 and the mixed form, through qz_step and through qz_step_host.
"""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _run(ic, dt, overlap, precision, host_steps):
    with core.Simulation(ic, 6, precision=precision, lmax=9, ref_ptcl=9,
                         tree_overlap=overlap) as sim:
        sim.init_forces()
        sim.step(dt, 3)
        if host_steps:
            p = sim.particles()
            state = {k: np.ascontiguousarray(p[k]) for k in KEYS}
            state["m"] = np.ascontiguousarray(ic["m"], dtype=np.float64)
            for _ in range(host_steps):
                sim.step_host(state, dt)
        out = sim.particles()
        pot = sim.field("pot")
        st = sim.stats()
        nodes = [sim.num_nodes(l) for l in range(sim.levels())]
    return out, pot, st, nodes


@pytest.mark.parametrize("precision", [0, 1])
def test_overlapped_head_solve_equals_sequential_stages(precision):
    ic = ics.plummer(120000, a=0.03, seed=11)
    dt = 1e-3 * ics.crossing_time(0.03)
    seq = _run(ic, dt, 0, precision, 2)
    ovl = _run(ic, dt, 1, precision, 2)
    for k in KEYS:
        np.testing.assert_array_equal(ovl[0][k], seq[0][k], err_msg=k)
    np.testing.assert_array_equal(ovl[1], seq[1])
    assert ovl[3] == seq[3] and len(seq[3]) > 1
    for f in ("vcycles_total", "cg_iterations", "steps", "nodes", "levels"):
        assert getattr(ovl[2], f) == getattr(seq[2], f), f

"""node_warm: refinement-node solves started from the previous step's solution.

The convergence test is the reference's, so the warm-started run stays within
the solve tolerance of the cold-started one (the reference's start from the
parent interpolation): accelerations within 1e-8 of the largest and positions
within 1e-12 box units after 5 steps, with no more conjugate-gradient
iterations than the cold run."""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("prec", [0, 1])
def test_warm_start_stays_within_tolerance(prec):
    ic = ics.plummer(60000, a=0.03, seed=21)
    dt = 1e-3 * ics.crossing_time(0.03)
    out, iters = {}, {}
    for warm in (0, 1):
        with core.Simulation(ic, 6, lmax=8, ref_ptcl=9, precision=prec, node_warm=warm) as sim:
            sim.init_forces()
            st0 = sim.stats()
            sim.step(dt, 5)
            iters[warm] = sim.stats().cg_iterations - st0.cg_iterations
            out[warm] = sim.particles()
    for k in ("ax", "ay", "az"):
        assert _rel(out[1][k], out[0][k]) < 1e-8, k
    for k in ("x", "y", "z"):
        assert np.abs(out[1][k] - out[0][k]).max() < 1e-12, k
    assert iters[1] <= iters[0], iters

"""GPU: the CFL time step (timestep.c:589-700) reduced on the device.

* head only, against the reference's timestep() on the head_L4 states
  (fixture): the lexicographic mode reproduces the reference's accelerations to
  ~1e-11, and the step is a min / max over the same per-particle formulas, so
  it agrees to 1e-10 relative;
* refinement run against the reference driver (each particle with the cell size
  of its finest node): 1e-6 relative, the tolerance of the accelerations;
* qz_step with dt <= 0 takes the CFL step each step: the trajectory equals,
  bit for bit, fixed steps of the dt that qz_timestep returns before each step.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _ic(g):
    return {k: g["ic_" + k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}


@pytest.mark.parametrize("method", [0, 1])
def test_timestep_head(head_golden, timestep_golden, method):
    g, t = head_golden, timestep_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    cfg = dict(gs_order=core.QZ_GS_LEX, cfl=float(t["cfl"][0]), max_dt=float(t["max_dt"][0]),
               time_step_method=method)
    with core.Simulation(_ic(g), 4, **cfg) as sim:
        sim.init_forces()
        d0 = sim.timestep()
        sim.step(dt, steps)
        d3 = sim.timestep()
    for d, s in ((d0, 0), (d3, steps)):
        ref = float(t[f"m{method}_s{s}_dt"][0])
        assert abs(d - ref) <= 1e-10 * ref, (method, s, d, ref)


def test_timestep_refinement(tmp_path):
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    summ = O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}",
                           lmin=lmin, lmax=lmax, ref_ptcl=rp, max_dt=1.0)
    cfg = dict(lmax=lmax, ref_ptcl=rp, cfl=summ["cfl"], max_dt=1.0, time_step_method=1)
    with core.Simulation(ic, lmin, **cfg) as sim:
        sim.init_forces()
        d0 = sim.timestep()
        sim.step(dt, steps)
        d3 = sim.timestep()
    for d, s in ((d0, 0), (d3, steps)):
        ref = float(O.read_dump(str(tmp_path), s, "dtcfl")[0])
        assert abs(d - ref) <= 1e-6 * ref, (s, d, ref)
    # the finest cells set the step: a head-only run would allow a larger one
    with core.Simulation(ic, lmin, cfl=summ["cfl"], max_dt=1.0) as head:
        head.init_forces()
        assert head.timestep() > d0


def test_adaptive_steps_match_fixed_steps():
    ic = ics.plummer(20000, a=0.05, seed=5)
    cfg = dict(lmax=7, ref_ptcl=9, cfl=0.5, max_dt=1.0)
    with core.Simulation(ic, 5, **cfg) as a, core.Simulation(ic, 5, **cfg) as b:
        a.init_forces()
        b.init_forces()
        total = 0.0
        for _ in range(4):
            h = b.timestep()
            b.step(h, 1)
            total += h
        a.step(0.0, 4)
        pa, pb = a.particles(), b.particles()
        st = a.stats()
    for k in pa:
        np.testing.assert_array_equal(pa[k], pb[k], err_msg=k)
    assert st.sim_time == total

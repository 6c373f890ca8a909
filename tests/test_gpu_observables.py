"""GPU: energies and momentum (observables.c:661-696) against the reference's
observables() on the same states (reference driver, both potential-energy
forms), in the reference's units (conversion factors from the reference driver).

Tolerances: kinetic energy 1e-12 relative and momentum 1e-12 of sum m|v| on
identical velocities (step 0; after steps, those of the velocities); exact
potential energy 1e-12 relative (same positions, sums in another order); the
grid form carries the potential's tolerance (lexicographic head 1e-11,
refinement 1e-8).
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def _check(sim, td, step, units, tol_k, tol_w_exact, tol_w_grid, m):
    p = sim.particles()
    for t, tol_w in ((0, tol_w_exact), (1, tol_w_grid)):
        ref = O.read_dump(td, step, f"obs{t}")
        mine = sim.observables(t, units)
        assert _rel(mine["kinetic"], ref[0]) < tol_k, (step, t)
        assert _rel(mine["potential"], ref[1]) < tol_w, (step, t, mine["potential"], ref[1])
        assert _rel(mine["total"], ref[2]) < max(tol_k, tol_w) * 10, (step, t)
        scale = sum(np.sum(m * np.abs(p[k])) for k in ("vx", "vy", "vz")) / units[0]
        assert np.abs(mine["momentum"] - ref[3:6]).max() <= tol_k * scale, (step, t)


def _run(tmp_path, ic, dt, steps, **kw):
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    summ = O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", obs=1, **kw)
    units = np.array([summ["conversion_velocity"], summ["conversion_time"],
                      summ["conversion_dist"], 0.0, 0.0, 0.0])
    return units


def test_observables_head(tmp_path):
    ic = ics.plummer(2000, a=0.05, seed=11)
    dt = 1e-3 * ics.crossing_time(0.05)
    units = _run(tmp_path, ic, dt, 2, lmin=4)
    with core.Simulation(ic, 4, gs_order=core.QZ_GS_LEX) as sim:
        sim.init_forces()
        _check(sim, str(tmp_path), 0, units, 1e-12, 1e-12, 1e-11, ic["m"])
        sim.step(dt, 2)
        _check(sim, str(tmp_path), 2, units, 1e-11, 1e-12, 1e-11, ic["m"])


def test_observables_refinement(tmp_path):
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    units = _run(tmp_path, ic, dt, 3, lmin=lmin, lmax=lmax, ref_ptcl=rp)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
        sim.init_forces()
        _check(sim, str(tmp_path), 0, units, 1e-12, 1e-12, 1e-8, ic["m"])
        sim.step(dt, 3)
        _check(sim, str(tmp_path), 3, units, 1e-9, 1e-10, 1e-8, ic["m"])

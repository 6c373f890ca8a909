"""The one-reduction conjugate gradients (cg_variant 1: Chronopoulos-Gear,
cg_variant 2: pipelined) against the reference.

Each produces the reference's iterates in exact arithmetic with another rounding,
so the bars are those of the refinement tests: node potentials 1e-8, node and
particle accelerations 1e-6 of the largest, positions after 3 steps 1e-10 box
units; the head solved by it (head_pot_method 1) against the fixture with the
bars of the two-reduction form; the iteration count within one check interval
(5) a level of the two-reduction form's.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("case", [(20000, 0.05, 5, 8, 9, 3), (60000, 0.03, 6, 8, 9, 4)])
def test_single_reduction_cg_refinement(tmp_path, case):
    n, a, lmin, lmax, rp, seed = case
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    p = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(p, ic)
    O.run_reference(p, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", lmin=lmin,
                    lmax=lmax, ref_ptcl=rp)
    ref = O.read_nodes(str(tmp_path), 0)
    iters = {}
    for variant in (0, 1, 2):
        with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp, cg_variant=variant) as sim:
            sim.init_forces()
            iters[variant] = sim.stats().cg_iterations
            p0 = sim.particles()
            if variant > 0:
                for nd in ref:
                    L, i = nd["level"], nd["idx"]
                    if L == 0:
                        continue
                    pts = sim.node_list(L, i, "intr")
                    for f, tol in (("pot", 1e-8), ("ax", 1e-6), ("ay", 1e-6), ("az", 1e-6)):
                        mine = sim.node_field(L, i, f)[pts]
                        theirs = O.node_dump(str(tmp_path), 0, L, i, f)[pts]
                        assert _rel(mine, theirs) < tol, (L, i, f, _rel(mine, theirs))
            sim.step(dt, steps)
            pend = sim.particles()
        if variant > 0:
            for k in ("ax", "ay", "az"):
                assert _rel(p0[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6
                assert _rel(pend[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
            for k in ("x", "y", "z"):
                assert np.abs(pend[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10
    levels = lmax - lmin
    assert abs(iters[1] - iters[0]) <= 5 * levels, iters
    assert abs(iters[2] - iters[0]) <= 5 * levels, iters


@pytest.mark.parametrize("variant", [1, 2])
def test_single_reduction_cg_head(cghead_golden, variant):
    g = cghead_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    ic = {k: g["ic_" + k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    with core.Simulation(ic, 4, head_pot_method=1, cg_variant=variant) as sim:
        sim.init_forces()
        pot0 = sim.field("pot")
        sim.step(dt, steps)
        p = sim.particles()
        pot = sim.field("pot")
    assert _rel(pot0, g["s0_pot"]) < 1e-9
    assert _rel(pot, g[f"s{steps}_pot"]) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-8, k
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-10

"""GPU parity of the reference's optional solver and stencil settings against
the compiled reference (oracle/_ref/qz_ref_driver) and its fixtures.

* force_stencil 1 (grid_acceleration.c:78-197, 396-692): head-only run in the
  lexicographic Gauss-Seidel mode (the reference's arithmetic order) against
  the fixture, tolerances of the 3-point pipeline test; a refinement run
  against the reference driver at step 0 and after 3 steps, tolerances of the
  refinement tests (node accelerations 1e-6 of the node's max, particle
  accelerations 1e-6, positions 1e-10 box units).
* conjugate gradient as the multigrid smoother (solver 2,
  conjugate_gradient_multigrid.c:29-176): the reference adds its dot products
  point by point, the GPU in fixed block order, so the iterates agree to
  rounding: arrays 1e-10 of the max, head pipeline potential 1e-9,
  accelerations 1e-8, positions 1e-10 box units.
* the head solved by the node conjugate gradient (head_pot_method 1,
  potential_head_node.c:157-171, conjugate_gradient.c:322-463): head run
  against the fixture with the cg-smoothing tolerances (the dot products are
  added in a different order); a refinement run against the reference driver with the
  same setting, tolerances of the refinement tests.
* red-black SOR for refinement nodes of at most branch_cg_cells cells
  (potential_branches.c:460-512; here 6000 cells, so the level-1 node takes SOR
  and the larger ones CG): refinement run against the reference driver with the same
  setting, node potentials 1e-8, particle accelerations 1e-6, positions 1e-10
  box units after 3 steps.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _ic(g):
    return {k: g["ic_" + k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}


def test_five_point_stencil_head(stencil5_golden):
    g = stencil5_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    with core.Simulation(_ic(g), 4, gs_order=core.QZ_GS_LEX, force_stencil=1) as sim:
        sim.init_forces()
        p0 = sim.particles()
        g0 = {k: sim.field(k) for k in ("ax", "ay", "az")}
        sim.step(dt, steps)
        p = sim.particles()
    for k in ("ax", "ay", "az"):
        assert _rel(g0[k], g[f"s0_g{k}"]) < 1e-11, k
        assert _rel(p0[k], g[f"s0_{k}"]) < 1e-11, k
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-11, k
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-13


def test_five_point_stencil_refinement(tmp_path):
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", lmin=lmin,
                    lmax=lmax, ref_ptcl=rp, stencil=1)
    ref = O.read_nodes(str(tmp_path), 0)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp, force_stencil=1) as sim:
        sim.init_forces()
        p0 = sim.particles()
        for nd in ref:
            L, i = nd["level"], nd["idx"]
            if L == 0:
                continue
            pts = sim.node_list(L, i, "intr")
            for f in ("ax", "ay", "az"):
                mine = sim.node_field(L, i, f)[pts]
                theirs = O.node_dump(str(tmp_path), 0, L, i, f)[pts]
                assert _rel(mine, theirs) < 1e-6, (L, i, f)
        sim.step(dt, steps)
        p = sim.particles()
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6
        assert _rel(p[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10


def test_cg_smoother_arrays(arrays_golden):
    g = arrays_golden
    for n in (9, 17):
        out = core.conjugate_gradient_multigrid(g[f"cgs_n{n}_in_phi"], g[f"cgs_n{n}_in_rho"],
                                                int(g[f"cgs_n{n}_iters"][0]))
        assert _rel(out, g[f"cgs_n{n}_out"]) < 1e-10, n


def test_cg_smoothing_head_pipeline(cgsmooth_golden):
    g = cgsmooth_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    with core.Simulation(_ic(g), 4, smoother=2) as sim:
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


def test_cg_head_pipeline(cghead_golden):
    g = cghead_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    with core.Simulation(_ic(g), 4, head_pot_method=1) as sim:
        sim.init_forces()
        pot0 = sim.field("pot")
        p0 = sim.particles()
        sim.step(dt, steps)
        p = sim.particles()
        pot = sim.field("pot")
    assert _rel(pot0, g["s0_pot"]) < 1e-9
    assert _rel(pot, g[f"s{steps}_pot"]) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], g[f"s0_{k}"]) < 1e-8, k
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-8, k
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-10


def test_cg_head_refinement(tmp_path):
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", lmin=lmin,
                    lmax=lmax, ref_ptcl=rp, cg_head=1)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp, head_pot_method=1) as sim:
        sim.init_forces()
        pot0 = sim.field("pot")
        p0 = sim.particles()
        sim.step(dt, steps)
        p = sim.particles()
    assert _rel(pot0, O.read_dump(str(tmp_path), 0, "pot")) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6
        assert _rel(p[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10


@pytest.mark.parametrize("check", [1, 2])
def test_cg_check_methods_refinement(tmp_path, check):
    """conj_grad_error (poisson_error.c:235-282) with check_method 1 (every
    interior residual below tol * 4 pi G rhomean) and 2 (the r.r threshold
    times cbrt(nintr)^2), head and refinement nodes by conjugate gradient."""
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 2
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", lmin=lmin,
                    lmax=lmax, ref_ptcl=rp, cg_head=1, check=check)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp, head_pot_method=1,
                         check_method=check) as sim:
        sim.init_forces()
        pot0 = sim.field("pot")
        sim.step(dt, steps)
        p = sim.particles()
    assert _rel(pot0, O.read_dump(str(tmp_path), 0, "pot")) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10


def test_sor_for_small_refinement_nodes(tmp_path):
    n, a, lmin, lmax, rp, seed = 20000, 0.05, 5, 8, 9, 3
    cells = 6000
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    O.run_reference(icp, str(tmp_path), steps=steps, dt=dt, dump=f"0,{steps}", lmin=lmin,
                    lmax=lmax, ref_ptcl=rp, branch_cg_cells=cells)
    ref = O.read_nodes(str(tmp_path), 0)
    n_sor = sum(1 for nd in ref if nd["level"] > 0 and nd["ncells"] <= cells)
    n_cg = sum(1 for nd in ref if nd["level"] > 0 and nd["ncells"] > cells)
    assert n_sor > 0 and n_cg > 0, (n_sor, n_cg)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp, branch_cg_cells=cells) as sim:
        sim.init_forces()
        p0 = sim.particles()
        for nd in ref:
            L, i = nd["level"], nd["idx"]
            if L == 0:
                continue
            pts = sim.node_list(L, i, "intr")
            mine = sim.node_field(L, i, "pot")[pts]
            theirs = O.node_dump(str(tmp_path), 0, L, i, "pot")[pts]
            assert _rel(mine, theirs) < 1e-8, (L, i, nd["ncells"])
        sim.step(dt, steps)
        p = sim.particles()
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6
        assert _rel(p[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10

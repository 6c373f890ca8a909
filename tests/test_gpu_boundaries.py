"""Periodic (bdry_cond_type 0) and outflow (2) boundaries of the head-only path,
against fixtures of the compiled reference (tests/golden: the 1000-particle
sphere plus 48 particles leaving through the six faces in the first step).

* periodic, 3- and 5-point stencils (initial_potential_and_acceleration_head.c
  :78-296, grid_acceleration.c:139-185, particle_updating.c:44-80) in the
  lexicographic Gauss-Seidel mode: the bars of the lexicographic pipeline
  test (potential 1e-12, positions 1e-13 box units, accelerations 1e-11) and
  the initial shell equal bit for bit;
* outflow (particle_updating.c:123-196): the particle count after each step
  and the arrays in the reference's order (removed slots refilled from the
  tail, the moved particle not advanced in that step), same bars; the removal
  lists of the first step as the reference's loop produces them;
* the drop-in link with both settings against the reference's own run.
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


def _check(g, sim, steps, dt):
    f0 = {k: sim.field(k) for k in ("pot", "ax", "ay", "az")}
    sim.step(dt, steps)
    p = sim.particles()
    pot = sim.field("pot")
    assert p["x"].size == g[f"s{steps}_x"].size
    assert _rel(pot, g[f"s{steps}_pot"]) < 1e-12
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-13, k
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-11, k
    return f0


@pytest.mark.parametrize("stencil", [0, 1])
def test_periodic_head_pipeline(periodic_golden, periodic5_golden, stencil):
    g = periodic_golden if stencil == 0 else periodic5_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    with core.Simulation(_ic(g), 4, bdry=0, force_stencil=stencil, gs_order=core.QZ_GS_LEX) as sim:
        sim.init_forces()
        p0 = sim.particles()
        f0 = _check(g, sim, steps, dt)
    # the initial shell is written before any solve: the boundary points of the
    # step-0 potential (coordinates 1 and 2^L + 1) come from it unchanged
    D = 2 ** 4 + 3
    c = np.arange(D)
    I, J, K = np.meshgrid(c, c, c, indexing="ij")
    shell = ((I == 1) | (I == 17) | (J == 1) | (J == 17) | (K == 1) | (K == 17)).transpose(2, 1, 0).ravel()
    assert np.array_equal(f0["pot"][shell], g["s0_pot"][shell])
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], g[f"s0_{k}"]) < 1e-11


def test_outflow_head_pipeline(outflow_golden):
    g = outflow_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    ic = _ic(g)
    n = ic["x"].size
    with core.Simulation(ic, 4, bdry=2, gs_order=core.QZ_GS_LEX) as sim:
        sim.init_forces()
        sim.step(dt, 1)
        cnt, slots, srcs = sim.outflow_removed()
        # the 48 leaving particles sit at the tail (1000 .. 1047): the front of the
        # loop meets the tail after 24 of them, each refilled from the far end
        assert cnt == 24 and sim.n == n - 24
        assert list(slots) == list(range(1000, 1024))
        assert list(srcs) == list(range(n - 1, n - 25, -1))
        hm = core.sequential_mass(ic["m"])
        for q in slots:
            hm -= ic["m"][q]
        assert sim.head_mass() == hm
    with core.Simulation(ic, 4, bdry=2, gs_order=core.QZ_GS_LEX) as sim:
        sim.init_forces()
        _check(g, sim, steps, dt)


@pytest.mark.parametrize("bdry", [0, 2])
def test_dropin_boundaries_match_reference(tmp_path, periodic_golden, bdry):
    g = periodic_golden
    for drv in (O.REF_DRIVER, O.DROPIN_DRIVER):
        assert os.path.exists(drv), f"{drv} missing: run `make -C oracle ref dropin`"
    p = str(tmp_path / "ic.bin")
    ics.write_ic(p, _ic(g))
    steps = 3
    kw = dict(lmin=4, steps=steps, dt=float(g["meta"][2]), dump=f"0,{steps}", bdry=bdry)
    os.makedirs(tmp_path / "ref")
    os.makedirs(tmp_path / "gpu")
    O.run_reference(p, str(tmp_path / "ref"), **kw)
    old = dict(os.environ)
    try:
        os.environ["QZ_GS_ORDER"] = "lex"
        O.run_reference(p, str(tmp_path / "gpu"), driver=O.DROPIN_DRIVER, **kw)
    finally:
        os.environ.clear()
        os.environ.update(old)
    for s in (0, steps):
        r = lambda f: O.read_dump(str(tmp_path / "ref"), s, f)
        q = lambda f: O.read_dump(str(tmp_path / "gpu"), s, f)
        assert q("x").size == r("x").size
        assert _rel(q("pot"), r("pot")) < 1e-12
        for f in ("x", "y", "z", "vx", "vy", "vz"):
            assert np.abs(q(f) - r(f)).max() < 1e-13, (s, f)

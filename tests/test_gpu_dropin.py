"""The drop-in link: the reference's own bookkeeping objects (initialization,
tree construction/adaptation, globals) linked with libqz_dropin.so in place of
its hot-path objects (oracle/_ref/qz_dropin_driver), run against the
unmodified reference (oracle/_ref/qz_ref_driver) on the same inputs.

Refinement runs (oracle/_ref/qz_dropin_amr_driver, the same link: the
reference's particle_updating.o is not in it -- the drop-in advances the
particles on the device and applies the moves between the host tree's cell
lists itself): positions after 4 steps within 1e-10 box units, particle
accelerations within 1e-6 of the largest, head potential within 1e-9, box
indices equal, and the reference's own adapted tree (node count and particles
per node, in node order) as in the plain run."""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.fixture(scope="module")
def ic_file(tmp_path_factory):
    d = tmp_path_factory.mktemp("dropin")
    p = str(d / "ic.bin")
    ics.write_ic(p, ics.plummer(4000, a=0.05, seed=21))
    return p


def _run(driver, ic_path, out, env=None, **kw):
    os.makedirs(out, exist_ok=True)
    old = dict(os.environ)
    try:
        if env:
            os.environ.update(env)
        return O.run_reference(ic_path, out, driver=driver, **kw)
    finally:
        os.environ.clear()
        os.environ.update(old)


# (Gauss-Seidel order, extra driver settings, potential / position tolerances); the
# conjugate-gradient smoother (solver 2) and the 5-point stencil are the
# reference's own settings, read by the drop-in from its globals
CASES = [
    ("lex", {}, 1e-12, 1e-13),
    ("rb", {}, 1e-9, 1e-9),
    ("rb", {"solver": 2}, 1e-9, 1e-9),
    ("lex", {"stencil": 1}, 1e-12, 1e-13),
    ("rb", {"cg_head": 1}, 1e-9, 1e-9),
]


@pytest.mark.parametrize("order,extra,tol_pot,tol_pos", CASES)
def test_dropin_driver_matches_reference(ic_file, tmp_path, order, extra, tol_pot, tol_pos):
    for drv in (O.REF_DRIVER, O.DROPIN_DRIVER):
        assert os.path.exists(drv), f"{drv} missing: run `make -C oracle ref dropin` where the reference is present"
    kw = dict(lmin=5, steps=6, dt=7e-5, dump="0,6", **extra)
    _run(O.REF_DRIVER, ic_file, str(tmp_path / "ref"), **kw)
    _run(O.DROPIN_DRIVER, ic_file, str(tmp_path / "gpu"), env={"QZ_GS_ORDER": order}, **kw)
    for s in (0, 6):
        r = lambda f: O.read_dump(str(tmp_path / "ref"), s, f)
        g = lambda f: O.read_dump(str(tmp_path / "gpu"), s, f)
        assert _rel(g("d"), r("d")) < 1e-12
        assert _rel(g("pot"), r("pot")) < tol_pot
        for f in ("gax", "gay", "gaz"):
            assert _rel(g(f), r(f)) < 100 * tol_pot
        for f in ("x", "y", "z"):
            assert np.abs(g(f) - r(f)).max() < tol_pos
        for f in ("ax", "ay", "az"):
            assert _rel(g(f), r(f)) < 100 * tol_pot
        np.testing.assert_array_equal(O.read_dump(str(tmp_path / "gpu"), s, "bidx", np.int32),
                                      O.read_dump(str(tmp_path / "ref"), s, "bidx", np.int32))


def test_dropin_refinement_run_matches_reference(tmp_path):
    drv = O.DROPIN_AMR_DRIVER
    assert os.path.exists(drv), f"{drv} missing: run `make -C oracle ref dropin`"
    p = str(tmp_path / "ic.bin")
    ics.write_ic(p, ics.plummer(20000, a=0.05, seed=3))
    steps = 4
    kw = dict(lmin=5, lmax=8, ref_ptcl=9, steps=steps,
              dt=1e-3 * ics.crossing_time(0.05), dump=f"0,{steps}")
    rr = _run(O.REF_DRIVER, p, str(tmp_path / "ref"), **kw)
    rg = _run(drv, p, str(tmp_path / "gpu"), **kw)
    assert rr["levels"] == rg["levels"] == 3 and rr["nodes"] == rg["nodes"]
    for s in (0, steps):
        r = lambda f: O.read_dump(str(tmp_path / "ref"), s, f)
        g = lambda f: O.read_dump(str(tmp_path / "gpu"), s, f)
        assert _rel(g("pot"), r("pot")) < 1e-9
        for f in ("x", "y", "z"):
            assert np.abs(g(f) - r(f)).max() < 1e-10, (s, f)
        for f in ("ax", "ay", "az"):
            assert _rel(g(f), r(f)) < 1e-6, (s, f)
        np.testing.assert_array_equal(O.read_dump(str(tmp_path / "gpu"), s, "bidx", np.int32),
                                      O.read_dump(str(tmp_path / "ref"), s, "bidx", np.int32))
        nr = O.read_nodes(str(tmp_path / "ref"), s)
        ng = O.read_nodes(str(tmp_path / "gpu"), s)
        assert [(n["lv"], n["nptcl"]) for n in nr] == [(n["lv"], n["nptcl"]) for n in ng]


def test_dropin_refinement_throughput_at_the_bench_size(tmp_path, capsys):
    """The bench workload (Plummer N = 1,048,576, a = 0.02, head 128^3, three
    refinement levels) through the drop-in in the reference's main-loop order,
    the host bookkeeping (tree_adaptation, cell lists) on all host threads:
    the run must complete and match the reference's positions after the steps;
    the step-loop rate of both is printed (particle-steps/s) for the record."""
    n, steps = 1048576, 3
    p = str(tmp_path / "ic.bin")
    ics.write_ic(p, ics.plummer(n, a=0.02, seed=1))
    kw = dict(lmin=7, lmax=10, ref_ptcl=9, steps=steps, dt=1e-3 * ics.crossing_time(0.02),
              dump=f"{steps}", threads=os.cpu_count() or 1)
    rr = _run(O.REF_DRIVER, p, str(tmp_path / "ref"), **kw)
    rg = _run(O.DROPIN_AMR_DRIVER, p, str(tmp_path / "gpu"), **kw)
    for f in ("x", "y", "z"):
        g = O.read_dump(str(tmp_path / "gpu"), steps, f)
        r = O.read_dump(str(tmp_path / "ref"), steps, f)
        assert np.abs(g - r).max() < 1e-10, f
    with capsys.disabled():
        print(f"\ndrop-in refinement run, {n} particles x {steps} steps: "
              f"drop-in {n * steps / rg['loop_s']:.4g} particle-steps/s, "
              f"reference {n * steps / rr['loop_s']:.4g} particle-steps/s "
              f"({os.cpu_count()} host threads)")

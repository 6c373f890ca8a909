"""The mixed-precision form with the node multigrid solver (node_solver =
QZ_NODE_MG): FP32 V-cycles on every refinement node preconditioning a flexible
conjugate gradient in FP64 (qz_node_mg.cu), with FP32 head cycles, against the
FP64 pipeline whose node solves are the reference's conjugate gradient (pinned
to the compiled reference in test_gpu_amr.py).

Bars (relative to the field's largest magnitude, per level and node):
  node potentials          1e-8   (both solves stop at the reference's test:
                                   ratio test 1e-10, residual 1e-10 rho-mean)
  particle accelerations   1e-5   largest relative force error per particle
                                  (the north-star bound for the mixed form)
  positions after 3 steps  1e-10  box units
Also: the node multigrid runs no node conjugate-gradient iteration and is
bit-reproducible (two runs equal), and the residual-test variants
(check_poisson_error_method 1 and 2) converge with it.
"""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _run(ic, lmin, lmax, dt, steps, **kw):
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=9, **kw) as sim:
        sim.init_forces()
        sim.step(dt, steps)
        p = sim.particles()
        pots = {}
        for l in range(1, sim.levels()):
            for q in range(sim.num_nodes(l)):
                info = sim.node_info(l, q)
                if info["nintr"] > 0:
                    g = sim.node_list(l, q, "intr")
                    pots[(l, q)] = sim.node_field(l, q, "pot")[g]
        return p, pots, sim.stats()


def _force_err(p, r):
    amag = np.sqrt(r["ax"] ** 2 + r["ay"] ** 2 + r["az"] ** 2)
    diff = np.sqrt((p["ax"] - r["ax"]) ** 2 + (p["ay"] - r["ay"]) ** 2 + (p["az"] - r["az"]) ** 2)
    return diff / np.maximum(amag, 1e-300)


@pytest.mark.parametrize("n,a,lmin,lmax,seed", [(60000, 0.03, 6, 8, 4), (200000, 0.02, 6, 9, 5)])
def test_node_multigrid_matches_fp64_conjugate_gradient(n, a, lmin, lmax, seed):
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    p64, pot64, st64 = _run(ic, lmin, lmax, dt, 3)
    pmx, potmx, stmx = _run(ic, lmin, lmax, dt, 3, precision=core.QZ_PREC_MIXED, node_solver=core.QZ_NODE_MG)
    assert stmx.levels == st64.levels and stmx.nodes == st64.nodes
    assert stmx.levels >= 3
    assert stmx.cg_iterations == 0 and stmx.node_mg_iterations > 0
    assert st64.cg_iterations > 0 and st64.node_mg_iterations == 0
    assert pot64.keys() == potmx.keys()
    for key in pot64:
        ref = pot64[key]
        err = np.abs(potmx[key] - ref).max() / np.abs(ref).max()
        assert err < 1e-8, f"node {key}: potential differs by {err:.2e}"
    assert _force_err(pmx, p64).max() < 1e-5
    for k in ("x", "y", "z"):
        assert np.abs(pmx[k] - p64[k]).max() < 1e-10


def test_node_multigrid_is_bit_reproducible():
    ic = ics.plummer(60000, a=0.03, seed=6)
    dt = 1e-3 * ics.crossing_time(0.03)
    a, pa, sa = _run(ic, 6, 8, dt, 2, precision=core.QZ_PREC_MIXED, node_solver=core.QZ_NODE_MG)
    b, pb, sb = _run(ic, 6, 8, dt, 2, precision=core.QZ_PREC_MIXED, node_solver=core.QZ_NODE_MG)
    assert sa.node_mg_iterations == sb.node_mg_iterations
    for k in ("x", "y", "z", "ax", "ay", "az"):
        np.testing.assert_array_equal(a[k], b[k])
    for key in pa:
        np.testing.assert_array_equal(pa[key], pb[key])


@pytest.mark.parametrize("method", [1, 2])
def test_node_multigrid_check_methods(method):
    ic = ics.plummer(60000, a=0.03, seed=7)
    dt = 1e-3 * ics.crossing_time(0.03)
    p64, _, _ = _run(ic, 6, 8, dt, 2, check_method=method)
    pmx, _, st = _run(ic, 6, 8, dt, 2, check_method=method, precision=core.QZ_PREC_MIXED, node_solver=core.QZ_NODE_MG)
    assert st.node_mg_iterations > 0
    assert _force_err(pmx, p64).max() < 1e-5

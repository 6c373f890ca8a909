"""The adjoint with refinement levels on a frozen tree (freeze_tree = 1: nodes
built once, particles reassigned to them every step) against central finite
differences of the frozen-tree forward.

* qz_force_vjp: J(x, m) = sum_p abar_p . F_p(x, m) on a 32^3 head with two
  refinement levels; every evaluation builds the tree at the base positions,
  then moves the particle and recomputes the forces on that tree, with the
  solves started from the same state, so the +eps and -eps runs take the same
  iterations (mass runs build on their own masses: the total mass, and with it
  the analytic shell, follows them).  Bar: 1e-6 of the gradient's largest entry (positions, eps 1e-6;
  masses, eps 1e-3 m_p).
"""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

L, LEV = 5, 2
TOL = dict(tol=1e-11, tol2=1e-11, adjoint_tol=1e-12, freeze_tree=1, lmax=L + LEV, ref_ptcl=9)


def _ic(n=6000, seed=5, a=0.03):
    return ics.plummer(n, a=a, seed=seed)


def _forces_on_tree(base, moved):
    """Forces at `moved` on the tree built at `base` (frozen)."""
    with core.Simulation(base, L, **TOL) as sim:
        sim.init_forces()
        sim.set_particles(moved)
        sim.init_forces()  # frozen: reassigns the particles, keeps the nodes
        assert sim.levels() == LEV + 1
        p = sim.particles()
    return np.stack([p["ax"], p["ay"], p["az"]])


def test_frozen_tree_recomputation_matches_the_build():
    ic = _ic()
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        p0 = sim.particles()
    f1 = _forces_on_tree(ic, ic)
    for q, k in enumerate(("ax", "ay", "az")):
        assert np.abs(f1[q] - p0[k]).max() <= 1e-9 * np.abs(p0[k]).max()


def test_force_vjp_with_refinement_against_finite_differences():
    ic = _ic()
    n = ic["x"].size
    rng = np.random.default_rng(1)
    ab = rng.standard_normal((3, n))
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        assert sim.levels() == LEV + 1
        g = sim.force_vjp(ab[0], ab[1], ab[2])
    J = lambda c: float(np.sum(ab * _forces_on_tree(ic, c)))
    Jm = lambda c: float(np.sum(ab * _forces_on_tree(c, c)))
    # particles in the refined centre (finest level 2 and 1) and one outside it
    r = np.sqrt((ic["x"] - 0.5) ** 2 + (ic["y"] - 0.5) ** 2 + (ic["z"] - 0.5) ** 2)
    order = np.argsort(r)
    picks = [order[0], order[1], order[n // 20], order[n // 8], order[n // 4], order[-1]]
    eps = 1e-6
    scale = max(np.abs(g[k]).max() for k in ("gx", "gy", "gz"))
    for p in picks:
        for ax, key in (("x", "gx"), ("y", "gy"), ("z", "gz")):
            cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
            cp[ax][p] += eps
            cm[ax][p] -= eps
            fd = (J(cp) - J(cm)) / (2 * eps)
            assert abs(fd - g[key][p]) <= 1e-6 * scale, (p, ax, fd, g[key][p])
    mscale = np.abs(g["gm"]).max()
    for p in picks[:3]:
        em = 1e-3 * ic["m"][p]
        cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
        cp["m"][p] += em
        cm["m"][p] -= em
        # the masses move the total mass (the shell): build each run on its own masses
        fd = (Jm(cp) - Jm(cm)) / (2 * em)
        assert abs(fd - g["gm"][p]) <= 1e-6 * mscale, (p, fd, g["gm"][p])


def _run_frozen(base, start, steps, dt):
    """Final particles of `steps` steps from `start` on the tree built at `base`."""
    with core.Simulation(base, L, **TOL) as sim:
        sim.init_forces()
        sim.set_particles(start)
        sim.init_forces()
        sim.step(dt, steps)
        return sim.particles()


def test_adjoint_trajectory_with_refinement_against_finite_differences():
    """L = mean_p |x_T,p - x*_p|^2 after 10 steps on the frozen tree, checkpoints
    every 4 steps (the first two segments recomputed), against central differences of the
    frozen-tree forward (eps 1e-6; masses 1e-3 m_p).  Bar: 1e-5 of the
    gradient's largest entry."""
    ic = _ic()
    n = ic["x"].size
    steps, dt = 10, 1e-3 * ics.crossing_time(0.03)
    rng = np.random.default_rng(7)
    pert = {k: v.copy() for k, v in ic.items()}
    for k in ("x", "y", "z"):
        pert[k] = pert[k] + rng.normal(0.0, 1e-3, n)
    pt = _run_frozen(ic, pert, steps, dt)
    tgt = {k: pt[k] for k in ("x", "y", "z")}
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        g = sim.adjoint_final_loss(steps, dt, tgt, checkpoint_every=4)
        pend = sim.particles()
    assert g["stats"]["recomputed_steps"] == 8  # segments [0, 4) and [4, 8)
    with core.Simulation(ic, L, **TOL) as sim:  # the same forward without the adjoint
        sim.init_forces()
        sim.step(dt, steps)
        ref = sim.particles()
    for k in ("x", "y", "z"):
        assert np.array_equal(pend[k], ref[k]), k

    def loss(base, start):
        p = _run_frozen(base, start, steps, dt)
        d = sum((p[k] - tgt[k]) ** 2 for k in ("x", "y", "z"))
        return float(d.sum() / n)

    d = sum((ref[k] - tgt[k]) ** 2 for k in ("x", "y", "z"))
    assert g["loss"] == pytest.approx(float(d.sum() / n), rel=1e-13)
    r = np.sqrt((ic["x"] - 0.5) ** 2 + (ic["y"] - 0.5) ** 2 + (ic["z"] - 0.5) ** 2)
    order = np.argsort(r)
    picks = [order[0], order[n // 20], order[n // 4], order[-1]]
    eps = 1e-6
    for field, key in (("x", "gx"), ("z", "gz"), ("vy", "gvy")):
        scale = np.abs(g[key]).max()
        for p in picks:
            cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
            cp[field][p] += eps
            cm[field][p] -= eps
            fd = (loss(ic, cp) - loss(ic, cm)) / (2 * eps)
            assert abs(fd - g[key][p]) <= 1e-5 * scale, (field, p, fd, g[key][p])
    mscale = np.abs(g["gm"]).max()
    for p in picks[:2]:
        em = 1e-3 * ic["m"][p]
        cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
        cp["m"][p] += em
        cm["m"][p] -= em
        fd = (loss(cp, cp) - loss(cm, cm)) / (2 * em)
        assert abs(fd - g["gm"][p]) <= 1e-5 * mscale, (p, fd, g["gm"][p])


def test_force_vjp_with_refinement_is_bit_reproducible():
    # every sum of the pull-back has a fixed order (the parent-average transposes
    # add their contributions sorted by parent point): two calls agree bit for bit
    ic = _ic(seed=9)
    n = ic["x"].size
    ab = np.random.default_rng(2).standard_normal((3, n))
    out = []
    for _ in range(2):
        with core.Simulation(ic, L, **TOL) as sim:
            sim.init_forces()
            out.append(sim.force_vjp(ab[0], ab[1], ab[2]))
    for k in ("gx", "gy", "gz", "gm"):
        np.testing.assert_array_equal(out[0][k], out[1][k], err_msg=k)

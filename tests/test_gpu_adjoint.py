"""Differentiation form: the adjoint of the head-node step against central
finite differences of the forward (which is itself pinned to the reference's
FP64 path by the pipeline tests).

* qz_force_vjp: J(x, m) = sum_p abar_p . F_p(x, m) for random abar; its
  gradient with respect to positions (gather weights, deposit weights and the
  field through the Poisson solve) and masses (deposit and the total-mass
  shell), central differences with eps = 1e-6 box units (positions) and
  1e-3 m_p (masses; J is linear in m).  Every evaluation starts from the
  analytic shell (a fresh simulation), so the solves of the +eps and -eps
  runs take the same cycles and the differences see the solve's derivative.
  Bar: 1e-6 relative to the gradient's largest entry.
* qz_adjoint_final_loss: L = mean_p |x_T,p - x*_p|^2 after 20 steps, targets
  from a forward run of ICs perturbed by N(0, 1e-3^2); gradients with respect
  to x0, v0, m against central differences (eps 1e-6; masses 1e-3 m_p) on
  random coordinates.  Bar: 1e-5 relative to the gradient's largest entry
  (the forward's warm-started solves are converged to the residual tolerance,
  not to rounding).  Checkpointing every 5 steps gives the same bits as one
  segment (the recomputation is exact); the loss equals the one of a plain
  forward run, and the simulation ends at the plain run's final state.
"""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

L = 5
TOL = dict(tol=1e-12, adjoint_tol=1e-12)


def _ic(n=2000, seed=5, a=0.05):
    return ics.plummer(n, a=a, seed=seed)


def _forces(ic):
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        p = sim.particles()
    return np.stack([p["ax"], p["ay"], p["az"]])


def test_force_vjp_against_finite_differences():
    ic = _ic()
    n = ic["x"].size
    rng = np.random.default_rng(1)
    ab = rng.standard_normal((3, n))
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        g = sim.force_vjp(ab[0], ab[1], ab[2])
    J = lambda c: float(np.sum(ab * _forces(c)))
    picks = rng.choice(n, 6, replace=False)
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
        fd = (J(cp) - J(cm)) / (2 * em)
        assert abs(fd - g["gm"][p]) <= 1e-6 * mscale, (p, fd, g["gm"][p])


def _targets(ic, steps, dt):
    rng = np.random.default_rng(7)
    pert = {k: v.copy() for k, v in ic.items()}
    for k in ("x", "y", "z"):
        pert[k] = pert[k] + rng.normal(0.0, 1e-3, pert[k].size)
    with core.Simulation(pert, L, **TOL) as sim:
        sim.init_forces()
        sim.step(dt, steps)
        p = sim.particles()
    return {k: p[k] for k in ("x", "y", "z")}


def _loss(ic, steps, dt, tgt):
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        sim.step(dt, steps)
        p = sim.particles()
    d = sum((p[k] - tgt[k]) ** 2 for k in ("x", "y", "z"))
    return float(d.sum() / d.size), p


def test_adjoint_trajectory_against_finite_differences():
    ic = _ic(n=4096, seed=9)
    n = ic["x"].size
    steps, dt = 20, 1e-3 * ics.crossing_time(0.05)
    tgt = _targets(ic, steps, dt)
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        g = sim.adjoint_final_loss(steps, dt, tgt, checkpoint_every=5)
        pend = sim.particles()
    with core.Simulation(ic, L, **TOL) as sim:
        sim.init_forces()
        g1 = sim.adjoint_final_loss(steps, dt, tgt, checkpoint_every=0)
    for k in ("gx", "gy", "gz", "gvx", "gvy", "gvz", "gm"):
        assert np.array_equal(g[k], g1[k]), k
    assert g["stats"]["recomputed_steps"] == 15 and g["stats"]["checkpoints"] == 4
    loss, pref = _loss(ic, steps, dt, tgt)
    assert abs(g["loss"] - loss) <= 1e-13 * loss
    for k in ("x", "y", "z", "vx", "vy", "vz"):
        assert np.array_equal(pend[k], pref[k]), k
    rng = np.random.default_rng(3)
    picks = rng.choice(n, 4, replace=False)
    eps = 1e-6
    for field, key in (("x", "gx"), ("y", "gy"), ("vx", "gvx"), ("vz", "gvz")):
        scale = np.abs(g[key]).max()
        for p in picks:
            cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
            cp[field][p] += eps
            cm[field][p] -= eps
            fd = (_loss(cp, steps, dt, tgt)[0] - _loss(cm, steps, dt, tgt)[0]) / (2 * eps)
            assert abs(fd - g[key][p]) <= 1e-5 * scale, (field, p, fd, g[key][p])
    mscale = np.abs(g["gm"]).max()
    for p in picks[:2]:
        em = 1e-3 * ic["m"][p]
        cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
        cp["m"][p] += em
        cm["m"][p] -= em
        fd = (_loss(cp, steps, dt, tgt)[0] - _loss(cm, steps, dt, tgt)[0]) / (2 * em)
        assert abs(fd - g["gm"][p]) <= 1e-5 * mscale, (p, fd, g["gm"][p])


def test_adjoint_rejects_unsupported_configurations():
    ic = _ic(n=500)
    with core.Simulation(ic, L, lmax=L + 2) as sim:
        sim.init_forces()
        with pytest.raises(core.QZError, match="head-only"):
            sim.force_vjp(np.zeros(500), np.zeros(500), np.zeros(500))


def test_replayed_schedule_reproduces_the_recorded_run():
    # replaying a run's own solver schedule from the same inputs gives the same bits
    ic = _ic(n=3000, seed=4)
    dt = 1e-3 * ics.crossing_time(0.05)
    out, sched = [], None
    for replay in (False, True):
        with core.Simulation(ic, L, **TOL) as sim:
            if replay:
                sim.replay_schedule(sched)
            else:
                sim.record_schedule()
            sim.init_forces()
            sim.step(dt, 5)
            out.append(sim.particles())
            if not replay:
                sched = sim.take_schedule()
    assert sched.size == 6 and np.all(sched > 0)  # step-0 solve and one per step
    for k in out[0]:
        assert np.array_equal(out[0][k], out[1][k]), k
    # a run with more solves than recorded fails instead of running unchecked
    with core.Simulation(ic, L, **TOL) as sim:
        sim.replay_schedule(sched[:2])
        sim.init_forces()
        sim.step(dt, 1)
        with pytest.raises(core.QZError, match="schedule exhausted"):
            sim.step(dt, 1)

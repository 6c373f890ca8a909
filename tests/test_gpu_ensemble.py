"""GPU: the batching form (qz_ensemble_step) steps independent simulations
concurrently; each one's state after the steps equals, bit for bit, that of
the same simulation stepped alone, and the thread count changes nothing.
Mixed sizes and heads (32^3 and 64^3, two refinement levels), a fixed step
per member and CFL steps."""
import numpy as np
import pytest

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

MEMBERS = [  # n, a, lmin, seed
    (2048, 0.05, 5, 1), (5000, 0.03, 5, 2), (9000, 0.08, 5, 3), (16384, 0.04, 6, 4),
    (3000, 0.06, 5, 5), (12000, 0.02, 5, 6), (20000, 0.05, 6, 7), (7000, 0.04, 5, 8),
]


def _make():
    sims = []
    for n, a, lmin, seed in MEMBERS:
        s = core.Simulation(ics.plummer(n, a=a, seed=seed), lmin, lmax=lmin + 2, ref_ptcl=9,
                            cfl=0.5, max_dt=1.0)
        s.init_forces()
        sims.append(s)
    return sims


@pytest.mark.parametrize("dt", [1e-4, None])
def test_ensemble_equals_members_alone(dt):
    alone = _make()
    dts = [1e-4 * (1 + 0.1 * k) for k in range(len(MEMBERS))] if dt else None
    for k, s in enumerate(alone):
        s.step(dts[k] if dts else 0.0, 3)
    want = [s.particles() for s in alone]
    for s in alone:
        s.close()
    for threads in (1, 4):
        ens = _make()
        core.ensemble_step(ens, dts, 3, threads=threads)
        for k, s in enumerate(ens):
            got = s.particles()
            for f in got:
                np.testing.assert_array_equal(got[f], want[k][f], err_msg=f"member {k} {f}")
            s.close()


def test_autotune_leaves_members_unchanged():
    """The autotuner's trial steps are put back: stepping after it gives the
    states of members stepped without it, for any multigrid points per thread
    and tile core (neither the multigrid launch's block count nor its tiled
    phases change its arithmetic)."""
    dts = [1e-4 * (1 + 0.1 * k) for k in range(len(MEMBERS))]
    ref = _make()
    core.ensemble_step(ref, dts, 2, threads=4)
    want = [s.particles() for s in ref]
    for s in ref:
        s.close()
    ens = _make()
    threads, ppt, tile, ms = core.ensemble_autotune(ens, dts, thread_opts=(1, 4),
                                                    ppt_opts=(1, 16), tile_opts=(-1, 6))
    assert threads in (1, 4) and ppt in (1, 16) and tile in (-1, 6) and ms > 0
    for s in ens:
        st = s.stats()
        assert st.steps == 0
    core.ensemble_step(ens, dts, 2, threads=threads)
    for k, s in enumerate(ens):
        got = s.particles()
        for f in got:
            np.testing.assert_array_equal(got[f], want[k][f], err_msg=f"member {k} {f}")
        s.close()

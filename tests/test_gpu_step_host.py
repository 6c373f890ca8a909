"""qz_step_host (one step on host-resident state, copies overlapped with the
step for page-locked arrays) gives the state of qz_set_particles +
qz_set_particle_accel + qz_step + qz_get_particles bit for bit, with refinement
and head-only, for page-locked and pageable host arrays, over several calls."""
import numpy as np
import pytest
import torch

from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

KEYS = ("x", "y", "z", "vx", "vy", "vz", "m", "ax", "ay", "az")


def _host(p, m, pinned):
    out = {}
    for k in KEYS:
        src = m if k == "m" else p[k]
        buf = torch.empty(src.size, dtype=torch.float64, pin_memory=pinned).numpy()
        buf[:] = src
        out[k] = buf
    return out


@pytest.mark.parametrize("levels", [0, 2])
@pytest.mark.parametrize("pinned", [True, False])
def test_step_host_equals_separate_calls(levels, pinned):
    ic = ics.plummer(30000, a=0.04, seed=11)
    lmin, dt = 5, 1e-3 * ics.crossing_time(0.04)
    with core.Simulation(ic, lmin, lmax=lmin + levels, ref_ptcl=9) as a, \
            core.Simulation(ic, lmin, lmax=lmin + levels, ref_ptcl=9) as b:
        a.init_forces()
        b.init_forces()
        state = _host(a.particles(), ic["m"], pinned)
        ref = {k: v.copy() for k, v in state.items()}
        for _ in range(3):
            a.step_host(state, dt)
            b.set_particles(ref)
            b.set_accelerations(ref["ax"], ref["ay"], ref["az"])
            b.step(dt, 1)
            got = b.particles()
            for k in KEYS:
                if k != "m":
                    ref[k][:] = got[k]
        for k in KEYS:
            np.testing.assert_array_equal(state[k], ref[k], err_msg=k)
        assert a.stats().steps == 3

"""Snapshot files (output_snapshots.c:141-239) written from the device state,
against files written by the compiled reference (oracle/_ref/qz_ref_driver,
key snap) from the same particle state.

* Without observables: every byte equal (the unit conversion keeps the
  reference's expression order; the library is built without contraction).
* With observables (compute_observables_FLAG, exact pair potential energy): the
  7N particle values and the time bit-exact, energies and momentum within
  1e-12 relative (sums in another order).
* Asynchronous write: the file holds the state at the call, although the
  simulation is stepped before the write is joined.
"""
import glob
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

CM = (0.1, -0.2, 0.3, 0.01, -0.02, 0.03)


def _reference_snapshot(tmp_path, snap, steps=2):
    ic = ics.plummer(2000, a=0.05, seed=4)
    icp = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(icp, ic)
    t = 0.37
    r = O.run_reference(icp, str(tmp_path), lmin=5, steps=steps, dt=1e-4, dump=str(steps),
                        snap=snap, snap_time=t, snap_pe=0, cm=",".join(str(c) for c in CM))
    f = glob.glob(os.path.join(str(tmp_path), "output", "*", "Data", "*_0.bin"))
    assert len(f) == 1, f
    state = {k: O.read_dump(str(tmp_path), steps, k) for k in ("x", "y", "z", "vx", "vy", "vz")}
    state["m"] = ic["m"]
    units = [r["conversion_dist"], r["conversion_velocity"], r["conversion_time"], *CM]
    return np.fromfile(f[0], dtype=np.uint8), state, units, t


@pytest.mark.parametrize("snap", [1, 2])
def test_snapshot_matches_reference_file(tmp_path, snap):
    ref, state, units, t = _reference_snapshot(tmp_path, snap)
    out = os.path.join(str(tmp_path), "mine.bin")
    with core.Simulation(state, 5) as sim:
        sim.write_snapshot(out, t, units, observables_type=0 if snap == 2 else -1)
    mine = np.fromfile(out, dtype=np.uint8)
    assert mine.size == ref.size
    if snap == 1:
        assert np.array_equal(mine, ref)
        return
    n = state["x"].size
    a, b = mine.view(np.float64), ref.view(np.float64)
    assert np.array_equal(a[:7 * n], b[:7 * n])
    assert a[-1] == b[-1]
    obs_a, obs_b = a[7 * n:7 * n + 6], b[7 * n:7 * n + 6]
    assert np.all(np.abs(obs_a - obs_b) <= 1e-12 * np.maximum(np.abs(obs_b), 1e-300)), (obs_a, obs_b)


def test_async_snapshot_holds_the_state_at_the_call(tmp_path):
    ic = ics.plummer(5000, a=0.05, seed=2)
    dt = 1e-3 * ics.crossing_time(0.05)
    a_path = os.path.join(str(tmp_path), "async.bin")
    s_path = os.path.join(str(tmp_path), "sync.bin")
    with core.Simulation(ic, 5) as sim:
        sim.init_forces()
        sim.step(dt, 2)
        sim.write_snapshot(s_path, 1.0)
        sim.write_snapshot(a_path, 1.0, wait=False)
        sim.step(dt, 3)
        sim.snapshot_wait()
        moved = sim.particles()
    a = np.fromfile(a_path)
    assert np.array_equal(a, np.fromfile(s_path))
    n = ic["x"].size
    assert not np.array_equal(a[n:2 * n], moved["x"] - 0.5)

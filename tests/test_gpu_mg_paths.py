"""GPU: the persistent red-black V-cycle launch gives the same head potential,
bit for bit, as one launch per multigrid phase (QZ_MG_LAUNCHES=1), with its
coarse levels in tiled phases (every tile core of QZ_MG_TILES that fits, the
default choice) and in grid phases (mg_tile = -1).

All paths apply the same point updates in the same dependency order (one
colour of a sweep, restriction and prolongation are order-free within a
phase; a tile recomputes its halo from the same values), so the fields must
agree exactly, in FP64 and in the mixed form.  The switch is read once per
process, so each path runs in a child process.
"""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
import numpy as np
from quantizer_b200 import core, ics
L, prec, out, tile = int(sys.argv[1]), int(sys.argv[2]), sys.argv[3], int(sys.argv[4])
ic = ics.plummer(20000, a=0.05, seed=3)
with core.Simulation(ic, L, precision=prec, mg_tile=tile) as sim:
    sim.init_forces()
    sim.step(2e-4, 3)
    p = sim.particles()
    st = sim.stats()
    np.savez(out, pot=sim.field("pot"), x=p["x"], ax=p["ax"],
             vcycles=np.array([st.vcycles_total]))
"""


def _run(tmp_path, L, prec, launches, tile=0):
    out = str(tmp_path / f"mg_L{L}_p{prec}_{int(launches)}_t{tile}.npz")
    env = dict(os.environ)
    env.pop("QZ_MG_LAUNCHES", None)
    if launches:
        env["QZ_MG_LAUNCHES"] = "1"
    env["PYTHONPATH"] = ROOT + os.pathsep + env.get("PYTHONPATH", "")
    subprocess.run([sys.executable, "-c", CHILD, str(L), str(prec), out, str(tile)], check=True,
                   env=env, cwd=ROOT, timeout=300)
    with np.load(out) as z:
        return {k: z[k] for k in z.files}


@pytest.mark.parametrize("L", [5, 6, 7])
@pytest.mark.parametrize("prec", [0, 1])
def test_persistent_vcycles_match_launch_per_phase(tmp_path, L, prec):
    b = _run(tmp_path, L, prec, launches=True)
    # the default core, every other core, grid phases
    for tile in (0, 1, 2, 3, 4, 5, 6, 7, -1) if L == 7 else (0, 6, -1):
        a = _run(tmp_path, L, prec, launches=False, tile=tile)
        assert a["vcycles"][0] == b["vcycles"][0], tile
        for k in ("pot", "x", "ax"):
            np.testing.assert_array_equal(a[k], b[k],
                                          err_msg=f"{k} L={L} precision={prec} mg_tile={tile}")

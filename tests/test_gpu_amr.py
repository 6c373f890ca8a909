"""Refinement (lmax > lmin) on the GPU against the compiled reference.

The reference (oracle/_ref/qz_ref_driver) builds its tree with
tree_construction() at step 0 and adapts it afterwards; the library rebuilds
it every step with the construction rules.  Integer outputs -- node geometry,
cell lists in order, interior / boundary / simulation-boundary grid-point lists
in order, box statuses, particle counts -- are compared bit for bit.  Fields
are compared at every listed grid point of every node, within tolerances:
  density 1e-12, potential 1e-8, grid accelerations 1e-6 (relative to the
  field's max magnitude in the node), particle accelerations 1e-6, positions
  after 3 steps 1e-10 box units.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

CASES = [
    # n, a, lmin, lmax, ref_ptcl, seed
    (20000, 0.05, 5, 8, 9, 3),
    (60000, 0.03, 6, 8, 9, 4),
]


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _run_ref(tmp, ic, dt, steps, **kw):
    p = os.path.join(tmp, "ic.bin")
    ics.write_ic(p, ic)
    O.run_reference(p, tmp, steps=steps, dt=dt, dump=f"0,{steps}", **kw)


def _level_coords(info, g):
    sx = info["rd"][0] + 1
    sxy = sx * (info["rd"][1] + 1)
    gz = g // sxy
    gy = (g - gz * sxy) // sx
    gx = g - gz * sxy - gy * sx
    return np.stack([gx + info["ts"][0], gy + info["ts"][1], gz + info["ts"][2]], axis=1)


@pytest.mark.parametrize("case", CASES)
def test_tree_and_fields_at_step0(tmp_path, case):
    n, a, lmin, lmax, rp, seed = case
    assert os.path.exists(O.REF_DRIVER)
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    _run_ref(str(tmp_path), ic, dt, 1, lmin=lmin, lmax=lmax, ref_ptcl=rp)
    ref = O.read_nodes(str(tmp_path), 0)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
        sim.init_forces()
        p = sim.particles()
        levels = sim.levels()
        assert levels == max(nd["level"] for nd in ref) + 1
        for nd in ref:
            L, i = nd["level"], nd["idx"]
            if L == 0:
                continue
            info = sim.node_info(L, i)
            for k in ("ts", "rd", "bmin", "bmax", "ncells", "nintr", "nbdry", "nsimb"):
                assert info[k] == nd[k], (L, i, k, info[k], nd[k])
            assert info["nptcl"] == nd["nptcl"]
            assert info["parent"] == nd["parent"]
            cells = sim.node_cells(L, i)
            for c, nm in enumerate(("cx", "cy", "cz")):
                np.testing.assert_array_equal(cells[:, c], O.node_dump(str(tmp_path), 0, L, i, nm))
            for which, nm in (("intr", "intr"), ("bdry", "bdry"), ("simb", "simbdry")):
                np.testing.assert_array_equal(sim.node_list(L, i, which),
                                              O.node_dump(str(tmp_path), 0, L, i, nm))
            np.testing.assert_array_equal(sim.node_box(L, i), O.node_dump(str(tmp_path), 0, L, i, "box"))
            pts = np.concatenate([sim.node_list(L, i, w) for w in ("intr", "bdry", "simb")])
            for f, tol in (("d", 1e-12), ("pot", 1e-8), ("ax", 1e-6), ("ay", 1e-6), ("az", 1e-6)):
                mine = sim.node_field(L, i, f)[pts]
                theirs = O.node_dump(str(tmp_path), 0, L, i, f)[pts]
                assert _rel(mine, theirs) < tol, (L, i, f, _rel(mine, theirs))
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6


def test_trajectory_with_refinement(tmp_path):
    n, a, lmin, lmax, rp, seed = CASES[0]
    ic = ics.plummer(n, a=a, seed=seed)
    dt = 1e-3 * ics.crossing_time(a)
    steps = 3
    _run_ref(str(tmp_path), ic, dt, steps, lmin=lmin, lmax=lmax, ref_ptcl=rp)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
        sim.init_forces()
        sim.step(dt, steps)
        p = sim.particles()
        st = sim.stats()
        # the refined cells of every level agree with the reference's (adapted) tree
        ref = O.read_nodes(str(tmp_path), steps)
        for L in range(1, sim.levels()):
            mine = set()
            for i in range(sim.num_nodes(L)):
                mine |= set(map(tuple, sim.node_cells(L, i)))
            theirs = set()
            for nd in ref:
                if nd["level"] == L:
                    cx = [O.node_dump(str(tmp_path), steps, L, nd["idx"], c) for c in ("cx", "cy", "cz")]
                    theirs |= set(zip(*[v.tolist() for v in cx]))
            assert mine == theirs, L
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - O.read_dump(str(tmp_path), steps, k)).max() < 1e-10
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], O.read_dump(str(tmp_path), steps, k)) < 1e-6
    assert st.levels == lmax - lmin + 1

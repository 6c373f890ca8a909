"""Full-size checks on the bench workloads' sizes.

* The default workload (Plummer N = 1,048,576, a = 0.02, head 128^3, three
  refinement levels above the head, refine above 8 particles) against the
  compiled reference after the step-0 forces and one step: particle
  accelerations within 1e-6 of the largest, positions within 1e-10 box units,
  the head potential within 1e-9 of its largest value.
* Size-independent properties at that size over 10 steps: two runs are equal
  bit for bit (deterministic reductions), the total momentum and the energy
  (observables.c, exact pair potential) change by less than a bound set by the
  leapfrog step.
* The 4.2 M-particle merger on a 256^3 head with four levels: two steps run,
  the tree has its five levels, momentum is conserved to the same bound.
* The same merger against the compiled reference (all host threads) after the
  step-0 forces and one step: head potential 1e-9 of its largest value,
  particle accelerations 1e-6 of the largest, positions 1e-10 box units; at
  step 0 every node's geometry and particle count equal the reference's, after
  the step the nodes per level, the particles per node and the refined cells.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_default_workload_one_step_against_reference(tmp_path):
    n, a, lmin, lmax, rp = 1048576, 0.02, 7, 10, 9
    ic = ics.plummer(n, a=a, seed=1)
    dt = 1e-3 * ics.crossing_time(a)
    p = os.path.join(str(tmp_path), "ic.bin")
    ics.write_ic(p, ic)
    O.run_reference(p, str(tmp_path), steps=1, dt=dt, dump="0,1", lmin=lmin, lmax=lmax,
                    ref_ptcl=rp)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
        sim.init_forces()
        p0 = sim.particles()
        pot0 = sim.field("pot")
        sim.step(dt, 1)
        p1 = sim.particles()
    assert _rel(pot0, O.read_dump(str(tmp_path), 0, "pot")) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], O.read_dump(str(tmp_path), 0, k)) < 1e-6, k
        assert _rel(p1[k], O.read_dump(str(tmp_path), 1, k)) < 1e-6, k
    for k in ("x", "y", "z"):
        assert np.abs(p1[k] - O.read_dump(str(tmp_path), 1, k)).max() < 1e-10, k


def _momentum(p, m):
    return np.array([np.sum(m * p[k]) for k in ("vx", "vy", "vz")])


def test_default_workload_determinism_and_conservation():
    n, a, lmin, lmax, rp = 1048576, 0.02, 7, 10, 9
    ic = ics.plummer(n, a=a, seed=2)
    dt = 1e-3 * ics.crossing_time(a)
    runs = []
    for _ in range(2):
        with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
            sim.init_forces()
            e0 = sim.observables(0)["total"]
            sim.step(dt, 10)
            e1 = sim.observables(0)["total"]
            runs.append((sim.particles(), e0, e1))
    (pa, e0, e1), (pb, _, _) = runs
    for k in pa:
        assert np.array_equal(pa[k], pb[k]), k
    m = ic["m"]
    vscale = np.sqrt(np.mean(ic["vx"] ** 2 + ic["vy"] ** 2 + ic["vz"] ** 2))
    # mesh forces are not exactly antisymmetric: momentum moves by O(dt |a| / N^(1/2))
    dp = np.abs(_momentum(pa, m) - _momentum(ic, m)).max()
    assert dp < 1e-3 * vscale * m.sum()
    assert abs(e1 - e0) < 1e-3 * abs(e0)


def test_merger_two_steps():
    ic = ics.merger(2097152, a=0.03, seed=1)
    dt = 1e-3 * ics.crossing_time(0.03)
    with core.Simulation(ic, 8, lmax=12, ref_ptcl=9) as sim:
        sim.init_forces()
        sim.step(dt, 2)
        p = sim.particles()
        assert sim.levels() == 5
    m = ic["m"]
    vscale = np.sqrt(np.mean(ic["vx"] ** 2 + ic["vy"] ** 2 + ic["vz"] ** 2))
    dp = np.abs(_momentum(p, m) - _momentum(ic, m)).max()
    assert dp < 1e-3 * vscale * m.sum()
    assert np.all((p["x"] > 0) & (p["x"] < 1))


def test_merger_one_step_against_reference(tmp_path):
    lmin, lmax, rp = 8, 12, 9
    ic = ics.merger(2097152, a=0.03, seed=1)
    dt = 1e-3 * ics.crossing_time(0.03)
    out = str(tmp_path)
    path = os.path.join(out, "ic.bin")
    ics.write_ic(path, ic)
    O.run_reference(path, out, steps=1, dt=dt, dump="0,1", lmin=lmin, lmax=lmax, ref_ptcl=rp,
                    threads=os.cpu_count() or 1)
    ref0, ref1 = O.read_nodes(out, 0), O.read_nodes(out, 1)
    with core.Simulation(ic, lmin, lmax=lmax, ref_ptcl=rp) as sim:
        sim.init_forces()
        p0 = sim.particles()
        pot0 = sim.field("pot")
        assert sim.levels() == max(nd["level"] for nd in ref0) + 1 == 5
        for nd in ref0:
            if nd["level"] == 0:
                continue
            info = sim.node_info(nd["level"], nd["idx"])
            for k in ("ts", "rd", "bmin", "bmax", "ncells", "nintr", "nbdry", "nsimb", "nptcl"):
                assert info[k] == nd[k], (nd["level"], nd["idx"], k, info[k], nd[k])
        sim.step(dt, 1)
        p1 = sim.particles()
        for L in range(1, sim.levels()):
            theirs = [nd for nd in ref1 if nd["level"] == L]
            assert sim.num_nodes(L) == len(theirs), L
            mine_n = sorted(sim.node_info(L, i)["nptcl"] for i in range(sim.num_nodes(L)))
            assert mine_n == sorted(nd["nptcl"] for nd in theirs), L
            mine = set()
            for i in range(sim.num_nodes(L)):
                mine |= set(map(tuple, sim.node_cells(L, i)))
            cells = set()
            for nd in theirs:
                cx = [O.node_dump(out, 1, L, nd["idx"], c) for c in ("cx", "cy", "cz")]
                cells |= set(zip(*[v.tolist() for v in cx]))
            assert mine == cells, L
    assert _rel(pot0, O.read_dump(out, 0, "pot")) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p0[k], O.read_dump(out, 0, k)) < 1e-6, k
        assert _rel(p1[k], O.read_dump(out, 1, k)) < 1e-6, k
    for k in ("x", "y", "z"):
        assert np.abs(p1[k] - O.read_dump(out, 1, k)).max() < 1e-10, k

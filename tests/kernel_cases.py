"""Kernel-level measurement cases of libqzb200 at chosen sizes, used to make
the ncu summaries under profiles/ (device time by CUDA events on the library
stream; the per-launch profiler books algorithmic bytes per kernel category).

    python -m tests.kernel_cases smooth    --n 257 --iters 4
    python -m tests.kernel_cases multigrid --n 257 --cycles 2
    python -m tests.kernel_cases step      --particles 1048576 --lmin 7 --levels 3 --steps 3

`smooth` and `multigrid` run the array-level routines (gauss_saidel /
multigrid, red-black order) on seeded random grids of n^3 points, which is
how the smoother is profiled at sizes whose fields exceed the 126 MB L2.
`step` runs whole leapfrog steps of a Plummer sphere on a 2^lmin head grid
with `--levels` refinement levels above it (0: head only); `--precision 1`
selects the mixed-precision form, `--node-solver 1` the node multigrid.  These are kernel-level cases, not the
timed workload of bench.py.
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from quantizer_b200 import core, ics  # noqa: E402


def _smooth(args) -> dict:
    n = args.n
    rng = np.random.default_rng(0)
    phi = rng.standard_normal(n ** 3)
    rho = rng.standard_normal(n ** 3)
    core.gauss_saidel(phi, rho, 1)  # warm-up (context, module load)
    t0 = time.perf_counter()
    core.gauss_saidel(phi, rho, args.iters)
    t = time.perf_counter() - t0
    return {"kernel": "smooth", "n": n, "iters": args.iters, "wall_s_incl_copies": t}


def _multigrid(args) -> dict:
    n = args.n
    rng = np.random.default_rng(0)
    phi = np.zeros(n ** 3)
    rho = rng.standard_normal(n ** 3)
    core.multigrid(phi, rho)
    t0 = time.perf_counter()
    for _ in range(args.cycles):
        phi = core.multigrid(phi, rho)
    t = time.perf_counter() - t0
    return {"kernel": "multigrid", "n": n, "cycles": args.cycles, "wall_s_incl_copies": t}


def _step(args) -> dict:
    ic = ics.plummer(args.particles, a=args.a, seed=1)
    dt = 1e-3 * ics.crossing_time(args.a)
    with core.Simulation(ic, args.lmin, lmax=args.lmin + args.levels, ref_ptcl=args.ref_ptcl,
                         precision=args.precision, node_solver=args.node_solver,
                         cg_variant=args.cg_variant) as sim:
        sim.init_forces()
        sim.step(dt, 1)
        st0 = sim.stats()
        t0 = time.perf_counter()
        sim.step(dt, args.steps)  # timed, profiler off
        sim.synchronize()
        t = time.perf_counter() - t0
        st1 = sim.stats()
        core.profile_reset(sim)  # separate profiled pass (per-launch events)
        core.profile_enable(sim, True)
        sim.step(dt, args.steps)
        prof = core.profile_read(sim)
        st2 = sim.stats()
    kern = {c: {"launches": v[0], "ms": round(v[1], 4),
                "GBps": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[1] > 0 else 0.0}
            for c, v in prof.items() if v[0]}
    return {"kernel": "step", "particles": args.particles, "lmin": args.lmin,
            "levels": st2.levels, "nodes": st2.nodes,
            "cg_iterations_per_step": (st1.cg_iterations - st0.cg_iterations) / args.steps,
            "steps": args.steps, "wall_ms_per_step": 1e3 * t / args.steps,
            "vcycles_per_step": (st1.vcycles_total - st0.vcycles_total) / args.steps,
            "launches_per_step": (st1.kernel_launches - st0.kernel_launches) / args.steps,
            "kernels": kern}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=("smooth", "multigrid", "step"))
    ap.add_argument("--n", type=int, default=257)
    ap.add_argument("--iters", type=int, default=4)
    ap.add_argument("--cycles", type=int, default=2)
    ap.add_argument("--particles", type=int, default=1_000_000)
    ap.add_argument("--lmin", type=int, default=7)
    ap.add_argument("--a", type=float, default=0.02)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", type=int, default=0)
    ap.add_argument("--levels", type=int, default=0, help="refinement levels above the head")
    ap.add_argument("--node-solver", type=int, default=0,
                    help="refinement nodes: 0 conjugate gradient, 1 FP32 node multigrid")
    ap.add_argument("--ref-ptcl", type=int, default=9)
    ap.add_argument("--cg-variant", type=int, default=0,
                    help="node conjugate gradient: 0 two reductions, 1 single reduction, "
                         "2 pipelined")
    args = ap.parse_args()
    fn = {"smooth": _smooth, "multigrid": _multigrid, "step": _step}[args.what]
    print(json.dumps(fn(args)))


if __name__ == "__main__":
    main()

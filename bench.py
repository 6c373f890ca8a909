"""Benchmark of the particle-mesh step on B200: prints ONE JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload NAME]

A step is one leapfrog step of QUANTIZER's main loop (main.c:375-481 with a
fixed dt): kick-drift, reset, refinement-tree rebuild, CIC deposit on every
level, Poisson solves to the reference's thresholds (head multigrid, then the
refinement levels by conjugate gradient), gradients, CIC gather from each
particle's finest node, kick.  Metric: particle-steps/s.  Other workloads
(--workload): the 4.2M-particle Hernquist merger on a 256^3 head with four
refinement levels, and the 512-member batching form (ensemble512: value is
the members stepped concurrently, beside the same members stepped one after
another).  The default workload
is the 1M-particle Plummer sphere on a 128^3 head with 3 refinement levels in
FP64 (the reference's arithmetic); the mixed-precision form (FP32 multigrid
cycles inside FP64 defect correction on the head and on every refinement node)
is timed on the same workload and reported with its force error against FP64
in "variant".

* value  -- whole-job throughput with the state resident in HBM; the device
  time of exactly K steps (CUDA events on the library stream), L2 flushed
  between steps by writing a 256 MiB buffer (outside the timed events).
* e2e    -- the same metric through the C ABI with HOST buffers: every step
  copies the particle state (x, v, a, m) from pinned host memory to the device
  and reads the advanced state (x, v, a) back, as the drop-in does for the
  reference's main loop.
* roofline -- the dominant kernel category from a profiled pass of the same
  workload (per-launch CUDA events), algorithmic bytes / device time against
  the measured HBM copy bandwidth of MEASURED_PEAKS.json.
* cpu_baseline -- the reference's own FP64 code (compiled unmodified,
  oracle/_ref/qz_ref_driver) on the box's host, 1 thread (its default).

--impl reference times the reference's CPU implementation of the same workload
with all host threads (OpenMP), on rank 0 only.

Multi-GPU (torchrun): the step has no exchange between independent
simulations, so each rank runs its own replica (different seed); value = all
ranks' particle steps / max-over-ranks device time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # Plummer N=10,000, a=0.05, head 32^3, no refinement, FP64, dt = 1e-3 t_cr
    "plummer10k_head32": dict(n=10000, a=0.05, lmin=5, levels=0, ref_ptcl=4, steps=100,
                              precision=0, cpu_steps=100, ref_steps=100),
    # Plummer N=1,048,576, a=0.02, head 128^3, refinement up to 3 levels above the head,
    # a cell refines when it holds more than 8 particles; FP64, with the mixed-precision
    # form (FP32 multigrid inside FP64 defect correction) timed beside it
    "plummer1m_head128_amr3": dict(n=1048576, a=0.02, lmin=7, levels=3, ref_ptcl=9, steps=100,
                                   precision=0, variant=1, cpu_steps=3, ref_steps=10),
}
WORKLOADS.update({
    # two Hernquist spheres of N = 2,097,152 each (a = 0.03, truncated at r <= 0.14,
    # centres 0.35 / 0.65 on x, approaching at half the mutual escape speed), head
    # 256^3, refinement up to 4 levels above the head, FP64
    "merger4m_head256_amr4": dict(ic="merger", n=2 * 2097152, a=0.03, lmin=8, levels=4,
                                  ref_ptcl=9, steps=20, precision=0, cpu_steps=1,
                                  ref_steps=1),
    # batching form: 512 Plummer members, N log-uniform in [2048, 65536], a uniform in
    # [0.02, 0.08], head 32^3 below N = 16384 else 64^3, two refinement levels, each
    # member with dt = 1e-3 of its own crossing time; stepped concurrently
    "ensemble512": dict(ic="ensemble", members=512, n=0, a=0.0, lmin=5, levels=2, ref_ptcl=9,
                        steps=10, precision=1, cpu_steps=2, ref_steps=2, threads=16,
                        cg_chunk_min=2048),
    # differentiation form: Plummer N = 262,144, a = 0.04, head 128^3 with the tree fixed
    # to the head node, FP64, 200 steps; loss = mean squared distance of the final
    # positions to targets from a forward run of ICs perturbed by N(0, 1e-3^2);
    # gradients with respect to x0, v0, m with a checkpoint every 20 steps, checked
    # against central differences on 64 random coordinates
    "adjoint262k_head128": dict(ic="adjoint", n=262144, a=0.04, lmin=7, levels=0, ref_ptcl=9,
                                steps=200, precision=0, cpu_steps=2, ref_steps=2, every=20,
                                fd_coords=64, tol=1e-11),
    # the same with two refinement levels above the head frozen to the tree built at
    # the initial positions (a cell refines above 8 particles)
    "adjoint262k_head128_amr2": dict(ic="adjoint", n=262144, a=0.04, lmin=7, levels=2,
                                     ref_ptcl=9, steps=200, precision=0, cpu_steps=2,
                                     ref_steps=2, every=20, fd_coords=64, tol=1e-11),
})
DEFAULT_WORKLOAD = "plummer1m_head128_amr3"


def make_ic(wl: dict, seed: int) -> dict:
    from quantizer_b200 import ics
    if wl.get("ic") == "merger":
        return ics.merger(wl["n"] // 2, a=wl["a"], seed=seed)
    return ics.plummer(wl["n"], a=wl["a"], seed=seed)


def ensemble_members(wl: dict, seed: int = 0) -> list:
    """(n, a, lmin) of each ensemble member (seeded)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    m = wl["members"]
    ns = np.exp(rng.uniform(np.log(2048.0), np.log(65536.0), m)).astype(int)
    As = rng.uniform(0.02, 0.08, m)
    return [(int(n), float(a), 5 if n < 16384 else 6) for n, a in zip(ns, As)]
METRIC = "particle-steps/s"
MIXED_DESC = ("fp32 head multigrid cycles in fp64 defect correction (convergence test in the "
              "launch, every iteration); refinement nodes by the fp64 node conjugate gradient")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def run_reference_cpu(wl: dict, steps: int, threads: int, seed: int) -> dict:
    """The reference's FP64 path (oracle/_ref/qz_ref_driver) on this host."""
    from oracle import oracle as O
    from quantizer_b200 import ics
    if not os.path.exists(O.REF_DRIVER):
        return {"kind": "port"} | run_port_cpu(wl, steps, seed)
    ic = make_ic(wl, seed)
    dt = 1e-3 * ics.crossing_time(wl["a"])
    with tempfile.TemporaryDirectory() as td:
        p = os.path.join(td, "ic.bin")
        ics.write_ic(p, ic)
        r = O.run_reference(p, td, lmin=wl["lmin"], lmax=wl["lmin"] + wl["levels"],
                            ref_ptcl=wl["ref_ptcl"], steps=steps, dt=dt, threads=threads)
    return {"kind": "reference", "value": wl["n"] * steps / r["loop_s"], "seconds": r["loop_s"],
            "steps": steps}


def run_port_cpu(wl: dict, steps: int, seed: int) -> dict:
    if wl["levels"]:
        raise RuntimeError("the CPU restatement covers the head-only path; refinement needs "
                           "the compiled reference (oracle/_ref)")
    import numpy as np
    from oracle import oracle as O
    from quantizer_b200 import ics
    ic = ics.plummer(wl["n"], a=wl["a"], seed=seed)
    dt = 1e-3 * ics.crossing_time(wl["a"])
    s = O.OracleSim(ic, O.params(wl["lmin"], total_mass=float(np.cumsum(ic["m"])[-1])))
    t0 = time.perf_counter()
    for _ in range(steps):
        s.step(dt)
    t = time.perf_counter() - t0
    return {"value": wl["n"] * steps / t, "seconds": t, "steps": steps}


def run_ensemble(args, wl: dict, K: int, W: int) -> int:
    """The batching form: all members stepped together (qz_ensemble_step) against the
    same members stepped one after another (one host thread, the single-instance
    path).  Time = device makespan over the members' streams (CUDA events)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    members = ensemble_members(wl, seed=rank)
    total = sum(n for n, _, _ in members)
    config = {"workload": args.workload, "members": len(members), "particles": total,
              "particles_per_member": "log-uniform in [2048, 65536]", "head_grid": "32 or 64",
              "lmax_minus_lmin": wl["levels"], "refine_above_particles": wl["ref_ptcl"] - 1,
              "dt": "1e-3 crossing time of each member",
              "precision": "fp32 head multigrid cycles in fp64 defect correction, fp64 node "
                           "conjugate gradient" if wl["precision"] else "fp64",
              "threads": wl["threads"], "replicas": world,
              "l2": "aggregate member state above L2, members interleave (no flush)"}
    if args.impl == "reference":
        if rank != 0:
            return 0
        r = ensemble_reference(wl, members, min(K, wl["ref_steps"]), os.cpu_count() or 1)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": r["steps"], "warmup": 0,
                "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
                "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": r["cores"],
                                 "kind": "reference", "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    import torch
    import torch.distributed as dist
    from quantizer_b200 import core, ics, replicas
    replicas.init("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sims, dts = [], []
    for k, (n, a, lmin) in enumerate(members):
        s = core.Simulation(ics.plummer(n, a=a, seed=1000 * rank + k), lmin,
                            lmax=lmin + wl["levels"], ref_ptcl=wl["ref_ptcl"],
                            precision=wl["precision"], cg_chunk_min=wl["cg_chunk_min"])
        s.init_forces()
        sims.append(s)
        dts.append(1e-3 * ics.crossing_time(a))
    streams = [torch.cuda.ExternalStream(s.stream, device=dev) for s in sims]

    def makespan(fn) -> float:
        starts, ends = [], []
        for st in streams:
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            starts.append(e)
        fn()
        for st in streams:
            e = torch.cuda.Event(enable_timing=True)
            e.record(st)
            ends.append(e)
        torch.cuda.synchronize()
        return max(starts[0].elapsed_time(e) for e in ends)

    core.ensemble_step(sims, dts, W, threads=wl["threads"])
    # autotuner: host threads x multigrid points per thread x tile core of the
    # tiled multigrid phases, one trial step each, states put back (untimed)
    threads, ppt, tile, tune_ms = core.ensemble_autotune(sims, dts)
    config["threads"] = threads
    config["mg_points_per_thread"] = ppt
    config["mg_tile"] = tile
    config["cg_chunk_min"] = wl["cg_chunk_min"]
    st0 = [s.stats() for s in sims]
    with ClockSampler(local) as clk:
        ms = makespan(lambda: core.ensemble_step(sims, dts, K, threads=threads))
    launches = sum(s.stats().kernel_launches - a.kernel_launches for s, a in zip(sims, st0))
    t_max = replicas.max_over_ranks(ms, dev)
    ms_max = t_max
    value = world * total * K / (ms_max / 1e3)
    Kl = min(K, 2)
    ms_loop = makespan(lambda: core.ensemble_step(sims, dts, Kl, threads=1))
    loop_value = total * Kl / (ms_loop / 1e3)
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        r = ensemble_reference(wl, members[:4], wl["cpu_steps"], 1)
        cpu = {"value": r["value"], "unit": METRIC, "cores": 1, "kind": "reference",
               "sample": r["sample"]}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64 (f32 head multigrid cycles)" if wl["precision"] else "f64",
                "data": "synthetic", "config": config, "e2e": None,
                "single_instance_loop": {"value": loop_value, "steps": Kl,
                                         "speedup_of_batching": value / world / loop_value},
                "autotune": {"threads": threads, "mg_points_per_thread": ppt, "mg_tile": tile,
                             "best_trial_ms": tune_ms,
                             "grid": "threads {4, 8, 16, 32, 64} x points per thread {2, 4, 8}"
                                     " x tile core {grid phases, 8x4x4, 8x8x8, 16x8x8}"},
                "cpu_baseline": cpu, "gpu_launches": int(launches), "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    for s in sims:
        s.close()
    replicas.finish()
    return 0


def run_adjoint(args, wl: dict, K: int, W: int) -> int:
    """Differentiation form: a plain forward of K steps against the gradient of the
    final-position loss (forward with checkpoints + reverse sweep), both device
    time (CUDA events); the gradient is checked against central differences of the
    forward on random coordinates (positions and velocities eps = 1e-6 box units,
    masses eps = 1e-3 m_p)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": args.workload, "particles": wl["n"], "head_grid": 2 ** wl["lmin"],
              "tree": "head node only (fixed)" if wl["levels"] == 0 else
              f"{wl['levels']} refinement levels frozen to the tree of the initial positions",
              "dt": "1e-3 crossing time", "precision": "fp64",
              "residual_tol": wl["tol"], "adjoint_tol": wl["tol"],
              "checkpoint_every": wl["every"], "loss": "mean_p |x_T - x*_T|^2",
              "targets": "forward run of ICs perturbed by N(0, 1e-3^2) in x, y, z",
              "replicas": world}
    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = os.cpu_count() or 1
        r = run_reference_cpu(wl, min(K, wl["ref_steps"]), threads, seed=1)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": r["steps"], "warmup": 0,
                "ms_per_step": 1e3 * r["seconds"] / r["steps"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config, "note": "the reference has no adjoint: its forward only",
                "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": threads,
                                 "kind": "reference", "sample": f"{r['steps']} forward steps"},
                "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0
    import numpy as np
    import torch
    import torch.distributed as dist
    from quantizer_b200 import core, ics, replicas
    replicas.init("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n, L = wl["n"], wl["lmin"]
    cfg = dict(tol=wl["tol"], tol2=wl["tol"], adjoint_tol=wl["tol"])
    if wl["levels"] > 0:
        cfg.update(lmax=wl["lmin"] + wl["levels"], ref_ptcl=wl["ref_ptcl"], freeze_tree=1)
    ic = ics.plummer(n, a=wl["a"], seed=replicas.seed_for(rank))
    dt = 1e-3 * ics.crossing_time(wl["a"])
    rng = np.random.default_rng(100 + rank)
    pert = {k: v.copy() for k, v in ic.items()}
    for k in ("x", "y", "z"):
        pert[k] = pert[k] + rng.normal(0.0, 1e-3, n)

    def forward(c, steps, base=None, record=False, replay=None):
        # a frozen tree is built at `base` (the unperturbed positions) and the run
        # starts from `c` on it, as the gradient assumes.  record / replay: the
        # solver schedule (iteration count of every Poisson solve), so that the
        # +eps and -eps runs apply the same map as the unperturbed run
        with core.Simulation(c if base is None else base, L, **cfg) as sm:
            if record:
                sm.record_schedule()
            if replay is not None:
                sm.replay_schedule(replay)
            sm.init_forces()
            if base is not None:
                sm.set_particles(c)
                sm.init_forces()
            sm.step(dt, steps)
            sched = sm.take_schedule() if record else None
            return sm.particles(), sched

    pt, _ = forward(pert, K, ic if wl["levels"] > 0 else None)
    tgt = {k: pt[k] for k in ("x", "y", "z")}

    def loss_of(c, base=None, replay=None):
        p, _ = forward(c, K, base, replay=replay)
        d = sum((p[k] - tgt[k]) ** 2 for k in ("x", "y", "z"))
        return float(d.sum() / n)

    # plain forward timing (warm-up runs first, then W+1 timed repetitions; the median)
    sim = core.Simulation(ic, L, **cfg)
    ext = torch.cuda.ExternalStream(sim.stream, device=dev)
    fwd_ms = []
    for rep_i in range(W + 1):
        sim.set_particles(ic)
        sim.init_forces()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        sim.step(dt, K)
        e1.record(ext)
        torch.cuda.synchronize()
        if rep_i > 0 or W == 0:
            fwd_ms.append(e0.elapsed_time(e1))
    forward_ms = statistics.median(fwd_ms)
    # gradient (after one untimed warm-up call)
    runs = []
    st0 = sim.stats()
    with ClockSampler(local) as clk:
        for rep_i in range(2):
            sim.set_particles(ic)
            sim.init_forces()
            g = sim.adjoint_final_loss(K, dt, tgt, checkpoint_every=wl["every"])
            runs.append(g["stats"])
    st1 = sim.stats()
    sa = runs[-1]
    adj_ms = sa["forward_ms"] + sa["reverse_ms"]
    t_max = replicas.max_over_ranks(adj_ms, dev)
    adj_ms_max = t_max
    free, total_mem = torch.cuda.mem_get_info(dev)
    # finite differences on random coordinates
    kinds = [("x", "gx", 1e-6)] * 12 + [("y", "gy", 1e-6)] * 6 + [("z", "gz", 1e-6)] * 6 + \
            [("vx", "gvx", 1e-6)] * 8 + [("vy", "gvy", 1e-6)] * 8 + [("vz", "gvz", 1e-6)] * 8 + \
            [("m", "gm", None)] * 16
    kinds = kinds[:wl["fd_coords"]]
    picks = rng.choice(n, len(kinds), replace=False)
    errs, rels = [], []
    # the unperturbed run's solver schedule: every +-eps run replays it
    _, sched = forward(ic, K, ic if wl["levels"] > 0 else None, record=True)
    for (field, key, eps), p in zip(kinds, picks):
        h = eps if eps is not None else 1e-3 * ic["m"][p]
        cp, cm = {k: v.copy() for k, v in ic.items()}, {k: v.copy() for k, v in ic.items()}
        cp[field][p] += h
        cm[field][p] -= h
        if wl["levels"] > 0:
            # positions and velocities on the tree of ic; mass runs on their own
            # masses (the total mass and the shell follow them; the tree is ic's)
            bp = cp if field == "m" else ic
            bm = cm if field == "m" else ic
            fd = (loss_of(cp, bp, sched) - loss_of(cm, bm, sched)) / (2 * h)
        else:
            fd = (loss_of(cp, replay=sched) - loss_of(cm, replay=sched)) / (2 * h)
        scale = float(np.abs(g[key]).max())
        errs.append(abs(fd - g[key][p]) / scale)
        rels.append(abs(fd - g[key][p]) / max(abs(fd), 1e-300))
    sim.close()
    value = world * n * K / (adj_ms_max / 1e3)
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": adj_ms_max / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config, "e2e": None,
                "adjoint": {"forward_ms": forward_ms, "gradient_ms": adj_ms,
                            "gradient_over_forward": adj_ms / forward_ms,
                            "reverse_over_forward": sa["reverse_ms"] / forward_ms,
                            "checkpointed_forward_ms": sa["forward_ms"],
                            "reverse_ms": sa["reverse_ms"],
                            "adjoint_cycles_per_step": sa["adjoint_cycles"] / K,
                            "recomputed_steps": sa["recomputed_steps"],
                            "checkpoints": sa["checkpoints"],
                            "pool_peak_bytes": sa["pool_peak_bytes"],
                            "stored_state_bytes": sa["stored_bytes"],
                            "device_bytes_in_use_after": total_mem - free,
                            "loss": runs[-1]["loss"]},
                "finite_differences": {"coords": len(kinds),
                                       "max_err_over_gradient_max": float(max(errs)),
                                       "median_err_over_gradient_max": float(np.median(errs)),
                                       "median_rel_err": float(np.median(rels)),
                                       "max_rel_err": float(max(rels)),
                                       "eps": "1e-6 (x, v), 1e-3 m_p (m)",
                                       "solver_schedule": "replayed from the unperturbed run"},
                "gpu_launches": int(st1.kernel_launches - st0.kernel_launches) // 2,
                "clocks": clk.summary(), "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    replicas.finish()
    return 0


def ensemble_reference(wl: dict, members: list, steps: int, threads: int) -> dict:
    """The reference on ensemble members one after another (host)."""
    from oracle import oracle as O
    from quantizer_b200 import ics
    parts, secs = 0, 0.0
    for k, (n, a, lmin) in enumerate(members):
        ic = ics.plummer(n, a=a, seed=k)
        with tempfile.TemporaryDirectory() as td:
            p = os.path.join(td, "ic.bin")
            ics.write_ic(p, ic)
            r = O.run_reference(p, td, lmin=lmin, lmax=lmin + wl["levels"], ref_ptcl=wl["ref_ptcl"],
                                steps=steps, dt=1e-3 * ics.crossing_time(a), threads=threads)
        parts += n * steps
        secs += r["loop_s"]
    return {"value": parts / secs, "steps": steps, "cores": threads, "seconds": secs,
            "sample": f"{len(members)} members x {steps} steps after their step-0 forces, "
                      f"one after another, {threads} thread(s)"}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cg-variant", type=int, default=None,
                    help="refinement conjugate gradient: 0 two reductions per iteration "
                         "(the reference's order), 1 one reduction")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    K = args.steps if args.steps is not None else wl["steps"]
    W = max(3, args.warmup)
    if wl.get("ic") == "ensemble":
        return run_ensemble(args, wl, K, W)
    if wl.get("ic") == "adjoint":
        return run_adjoint(args, wl, K, W)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    config = {"workload": args.workload, "particles": wl["n"], "head_grid": 2 ** wl["lmin"],
              "lmax_minus_lmin": wl["levels"], "refine_above_particles": wl["ref_ptcl"] - 1,
              "dt": "1e-3 crossing time", "precision":
              "fp64" if wl["precision"] == 0 else MIXED_DESC,
              "residual_tol": 1e-10, "l2": "flushed between timed steps (256 MiB write)",
              "replicas": world}

    if args.impl == "reference":
        if rank != 0:
            return 0
        threads = os.cpu_count() or 1
        Kr = min(K, wl["ref_steps"])
        r = run_reference_cpu(wl, Kr, threads, seed=1)
        line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": METRIC,
                "n_gpus": args.gpus, "steps": Kr, "warmup": 0,
                "ms_per_step": 1e3 * r["seconds"] / Kr, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config,
                "cpu_baseline": {"value": r["value"], "unit": METRIC, "cores": threads,
                                 "kind": r.get("kind", "reference"),
                                 "sample": f"{Kr} steps of the workload after its step-0 "
                                           "forces (whole step loop, OpenMP threads)"},
                "e2e": {"value": r["value"], "unit": METRIC, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    import numpy as np
    import torch
    import torch.distributed as dist
    from quantizer_b200 import core, ics, replicas

    replicas.init("nccl")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    ic = make_ic(wl, replicas.seed_for(rank))
    dt = 1e-3 * ics.crossing_time(wl["a"])
    simcfg = dict(lmax=wl["lmin"] + wl["levels"], ref_ptcl=wl["ref_ptcl"])
    if args.cg_variant is not None:
        simcfg["cg_variant"] = args.cg_variant
        config["cg_variant"] = args.cg_variant
    sim = core.Simulation(ic, wl["lmin"], precision=wl["precision"], **simcfg)
    ext = torch.cuda.ExternalStream(sim.stream, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    sim.init_forces()
    for _ in range(W):
        sim.step(dt, 1)

    def timed_steps_on(sm, fn, k):
        st = torch.cuda.ExternalStream(sm.stream, device=dev)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(k)]
        for i in range(k):
            with torch.cuda.stream(st):
                flush.add_(1.0)
                evs[i][0].record(st)
            fn()
            evs[i][1].record(st)
        torch.cuda.synchronize()
        return sum(a.elapsed_time(b) for a, b in evs)

    def timed_steps(fn, k):
        return timed_steps_on(sim, fn, k)

    # ---- device-resident timed region -------------------------------------------------
    st0 = sim.stats()
    barrier()
    with ClockSampler(local) as clk:
        ms = timed_steps(lambda: sim.step(dt, 1), K)
    barrier()
    st1 = sim.stats()
    launches = int(st1.kernel_launches - st0.kernel_launches)
    vcycles = int(st1.vcycles_total - st0.vcycles_total)
    cgit = int(st1.cg_iterations - st0.cg_iterations)
    t_max = replicas.max_over_ranks(ms, dev)
    ms_max = t_max
    value = world * wl["n"] * K / (ms_max / 1e3)

    # ---- end to end through the C ABI with host buffers --------------------------------
    p = sim.particles()
    host = {}
    for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m"):
        buf = torch.empty(wl["n"], dtype=torch.float64, pin_memory=True).numpy()
        buf[:] = p[k] if k != "m" else ic["m"]
        host[k] = buf
    Ke = K
    barrier()
    ms_e2e = timed_steps(lambda: sim.step_host(host, dt), Ke)
    barrier()
    t_max = replicas.max_over_ranks(ms_e2e, dev)
    e2e_value = world * wl["n"] * Ke / (t_max / 1e3)

    # ---- profiled pass: per-kernel-category device time --------------------------------
    Kp = min(K, 5)
    core.profile_reset(sim)
    core.profile_enable(sim, True)
    sim.set_particles({**p, "m": ic["m"]})
    sim.set_accelerations(p["ax"], p["ay"], p["az"])
    sim.step(dt, Kp)
    sim.synchronize()
    prof = core.profile_read(sim)
    core.profile_enable(sim, False)
    dom = max(prof, key=lambda c: prof[c][1])
    n_l, ms_l, by_l = prof[dom]
    pk = peaks()
    achieved = (by_l / (ms_l / 1e3)) / 1e9 if ms_l > 0 else 0.0
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic_per_launch.txt")
    if os.path.exists(tf):
        for ln in open(tf):
            f = ln.split()
            if len(f) >= 3 and f[0] == args.workload and f[1] == dom:
                traffic = float(f[2])
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk["hbm_gbs"],
                "unit": "GB/s", "frac": achieved / pk["hbm_gbs"], "traffic": traffic,
                "peak_source": pk["source"], "launches": n_l,
                "avg_launch_us": 1e3 * ms_l / max(n_l, 1),
                "algorithmic_bytes_per_launch": by_l / max(n_l, 1)}
    kernels = {c: {"launches": v[0], "ms": round(v[1], 4),
                   "GBps": round((v[2] / (v[1] / 1e3)) / 1e9, 1) if v[1] > 0 else 0.0}
               for c, v in prof.items() if v[0]}

    # the other precision form on the same workload, and the force error of the
    # mixed-precision form against FP64 after one step from the same state
    plain = None
    if wl.get("variant") is not None:
        st_pos = sim.particles()
        ref_sim = core.Simulation(ic, wl["lmin"], precision=wl["variant"], **simcfg)
        ref_sim.init_forces()
        for _ in range(W):
            ref_sim.step(dt, 1)
        barrier()
        sv0 = ref_sim.stats()
        ms_plain = timed_steps_on(ref_sim, lambda: ref_sim.step(dt, 1), K)
        sv1 = ref_sim.stats()
        t_max = replicas.max_over_ranks(ms_plain, dev)
        plain_value = world * wl["n"] * K / (t_max / 1e3)
        # force error: both forms from one state, one step
        state = {**st_pos, "m": ic["m"]}
        errs = []
        outs = []
        for sm in (sim, ref_sim):
            sm.set_particles(state)
            sm.set_accelerations(state["ax"], state["ay"], state["az"])
            sm.step(dt, 1)
            outs.append(sm.particles())
        f64 = outs[0] if wl["precision"] == 0 else outs[1]
        mix = outs[1] if wl["precision"] == 0 else outs[0]
        a_p = np.sqrt(sum(f64[k] ** 2 for k in ("ax", "ay", "az")))
        diff = np.sqrt(sum((mix[k] - f64[k]) ** 2 for k in ("ax", "ay", "az")))
        errs = diff / np.maximum(a_p, 1e-300)
        plain = {"precision": "fp64" if wl["variant"] == 0 else MIXED_DESC,
                 "node_mg_iterations_per_step":
                     (sv1.node_mg_iterations - sv0.node_mg_iterations) / K,
                 "vcycles_per_step": (sv1.vcycles_total - sv0.vcycles_total) / K,
                 "value": plain_value, "ms_per_step": t_max / K,
                 "max_rel_force_err_mixed_vs_fp64": float(errs.max()),
                 "median_rel_force_err_mixed_vs_fp64": float(np.median(errs))}
        ref_sim.close()
        def extra_form(**kw) -> dict:
            """The variant's form with other node-solve settings: K timed steps and
            the force error against FP64 after one step from `state`."""
            xs = core.Simulation(ic, wl["lmin"], precision=wl["variant"], **kw, **simcfg)
            xs.init_forces()
            for _ in range(W):
                xs.step(dt, 1)
            barrier()
            s0 = xs.stats()
            ms_x = timed_steps_on(xs, lambda: xs.step(dt, 1), K)
            s1 = xs.stats()
            t_x = replicas.max_over_ranks(ms_x, dev)
            xs.set_particles(state)
            xs.set_accelerations(state["ax"], state["ay"], state["az"])
            xs.step(dt, 1)
            px = xs.particles()
            xs.close()
            ex = np.sqrt(sum((px[k] - f64[k]) ** 2 for k in ("ax", "ay", "az"))) / \
                np.maximum(a_p, 1e-300)
            return {"value": world * wl["n"] * K / (t_x / 1e3), "ms_per_step": t_x / K,
                    "node_mg_iterations_per_step":
                        (s1.node_mg_iterations - s0.node_mg_iterations) / K,
                    "cg_iterations_per_step": (s1.cg_iterations - s0.cg_iterations) / K,
                    "max_rel_force_err_vs_fp64": float(ex.max()),
                    "median_rel_force_err_vs_fp64": float(np.median(ex))}

        # the refinement nodes solved by the FP32 node multigrid (flexible conjugate
        # gradient preconditioned by V-cycles) instead of the FP64 node CG
        plain["node_multigrid"] = extra_form(node_solver=core.QZ_NODE_MG)
        # the node CG started from the previous step's solution (node_warm)
        plain["warm_nodes"] = extra_form(node_warm=1)

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            r = run_reference_cpu(wl, wl["cpu_steps"], 1, seed=1)
            cpu = {"value": r["value"], "unit": METRIC, "cores": 1, "kind": r.get("kind", "reference"),
                   "sample": f"{r['steps']} steps of the same workload after its step-0 forces, "
                             "reference default 1 thread"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": METRIC, "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        n = wl["n"]
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": K,
                "warmup": W, "ms_per_step": ms_max / K, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None,
                "dtype": "f64" if wl["precision"] == 0 else "f64 (f32 multigrid cycles)",
                "data": "synthetic",
                "config": config,
                "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 80 * n,
                        "d2h_bytes_per_step": 72 * n},
                "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": launches,
                "vcycles_per_step": vcycles / K, "cg_iterations_per_step": cgit / K,
                "tree": {"levels": st1.levels, "nodes": st1.nodes},
                "variant": plain, "clocks": clk.summary(), "kernels": kernels}
        print(json.dumps(line), flush=True)
    sim.close()
    replicas.finish()
    return 0


if __name__ == "__main__":
    sys.exit(main())

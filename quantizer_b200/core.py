"""Python host mirror of the reference's hot-path interface over libqzb200.

``Simulation`` exposes the reference's per-step entry points by their own
names (grid_density, potential, grid_acceleration, particle_acceleration,
particle_updating_A/B, reset; main.c:369-481) on device-resident state, and
``step`` runs whole leapfrog steps.  Module functions mirror the array-level
force_methods routines (gauss_saidel, jacobi, multigrid) and
ptcl_idx_to_box_idx.  Every call goes through the C ABI of
include/qz_b200.h; there is no CPU fallback -- a missing library or a
machine without a CUDA device raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libqzb200.so")

QZ_GS_REDBLACK = 0
QZ_GS_LEX = 1
QZ_PREC_FP64 = 0
QZ_PREC_MIXED = 1
QZ_NODE_CG = 0
QZ_NODE_MG = 1
FIELDS = {"pot": 0, "pot_old": 1, "d": 2, "ax": 3, "ay": 4, "az": 5}

_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class Config(C.Structure):
    _fields_ = [
        ("lmin", C.c_int), ("lmax", C.c_int), ("G", C.c_double), ("total_mass", C.c_double),
        ("bdry", C.c_int), ("smoother", C.c_int), ("gs_order", C.c_int), ("cycle", C.c_int),
        ("n_pre", C.c_int), ("n_post", C.c_int), ("n_coarse", C.c_int), ("w_sor", C.c_double),
        ("tol", C.c_double), ("tol2", C.c_double), ("check_every", C.c_int),
        ("max_iter", C.c_int), ("check_method", C.c_int), ("precision", C.c_int),
        ("inner_cycles", C.c_int), ("force_stencil", C.c_int), ("ref_ptcl", C.c_int),
        ("box_extra", C.c_int), ("branch_cg_cells", C.c_int), ("branch_sor_sweeps", C.c_int),
        ("w_sor_branch", C.c_double), ("cfl", C.c_double), ("max_dt", C.c_double),
        ("time_step_method", C.c_int), ("head_pot_method", C.c_int),
        ("adjoint_tol", C.c_double), ("cg_variant", C.c_int),
        ("mg_points_per_thread", C.c_int), ("freeze_tree", C.c_int),
        ("node_solver", C.c_int), ("mg_tile", C.c_int), ("node_warm", C.c_int),
        ("tree_overlap", C.c_int), ("cg_chunk_min", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("vcycles_total", C.c_longlong), ("last_vcycles", C.c_int), ("last_converged", C.c_int),
        ("kernel_launches", C.c_longlong), ("steps", C.c_longlong), ("error_flags", C.c_int),
        ("cg_iterations", C.c_longlong), ("levels", C.c_int), ("nodes", C.c_int),
        ("last_dt", C.c_double), ("sim_time", C.c_double),
        ("adjoint_cycles", C.c_longlong), ("node_mg_iterations", C.c_longlong),
    ]


class AdjointStats(C.Structure):
    _fields_ = [
        ("loss", C.c_double), ("forward_ms", C.c_double), ("reverse_ms", C.c_double),
        ("adjoint_cycles", C.c_longlong), ("recomputed_steps", C.c_longlong),
        ("checkpoints", C.c_int), ("pool_peak_bytes", C.c_double),
        ("stored_bytes", C.c_double),
    ]


class QZError(RuntimeError):
    pass


_lib = None


def load() -> C.CDLL:
    """Load libqzb200.so (built in-tree by quantizer_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise QZError(f"{LIB_PATH} is missing: run `python -m quantizer_b200.build` "
                      "(the CUDA library has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    sig = {
        "qz_default_config": ([C.POINTER(Config), C.c_int], C.c_int),
        "qz_create": ([C.POINTER(Config), C.c_long, C.POINTER(vp)], C.c_int),
        "qz_destroy": ([vp], C.c_int),
        "qz_set_particles": ([vp, C.c_long] + [_P] * 7, C.c_int),
        "qz_get_particles": ([vp] + [_P] * 9, C.c_int),
        "qz_set_particle_accel": ([vp] + [_P] * 3, C.c_int),
        "qz_num_particles": ([vp], C.c_long),
        "qz_head_grid_points": ([vp], C.c_long),
        "qz_get_head_field": ([vp, C.c_int, _P], C.c_int),
        "qz_set_head_field": ([vp, C.c_int, _P], C.c_int),
        "qz_initial_potential_head": ([vp], C.c_int),
        "qz_reset": ([vp], C.c_int),
        "qz_grid_density": ([vp], C.c_int),
        "qz_potential": ([vp], C.c_int),
        "qz_potential_head_node": ([vp], C.c_int),
        "qz_outflow_removed": ([vp, C.POINTER(C.c_long), _I, _I], C.c_int),
        "qz_head_mass": ([vp], C.c_double),
        "qz_potential_branches": ([vp], C.c_int),
        "qz_grid_acceleration": ([vp], C.c_int),
        "qz_particle_acceleration": ([vp], C.c_int),
        "qz_particle_updating_A": ([vp, C.c_double], C.c_int),
        "qz_particle_updating_B": ([vp, C.c_double], C.c_int),
        "qz_init_forces": ([vp], C.c_int),
        "qz_step": ([vp, C.c_double, C.c_int], C.c_int),
        "qz_synchronize": ([vp], C.c_int),
        "qz_get_stats": ([vp, C.POINTER(Stats)], C.c_int),
        "qz_stream": ([vp], vp),
        "qz_last_error": ([], C.c_char_p),
        "qz_gauss_saidel": ([_P, _P, C.c_int, C.c_int, C.c_double, C.c_int], C.c_int),
        "qz_jacobi": ([_P, _P, C.c_int, C.c_int, C.c_double], C.c_int),
        "qz_multigrid": ([C.POINTER(Config), _P, _P, C.c_int, C.c_int], C.c_int),
        "qz_conjugate_gradient_multigrid": ([_P, _P, C.c_int, C.c_int], C.c_int),
        "qz_timestep": ([vp, _P], C.c_int),
        "qz_observables": ([vp, C.c_int, _P, _P], C.c_int),
        "qz_ensemble_step": ([C.POINTER(vp), C.c_int, _P, C.c_int, C.c_int], C.c_int),
        "qz_step_host": ([vp, C.c_double] + [_P] * 10, C.c_int),
        "qz_ensemble_autotune": ([C.POINTER(vp), C.c_int, _P, _I, C.c_int, _I, C.c_int, _I,
                                  C.c_int, _I, _I, _I, _P], C.c_int),
        "qz_force_vjp": ([vp] + [_P] * 7, C.c_int),
        "qz_write_snapshot": ([vp, C.c_char_p, C.c_double, _P, C.c_int, C.c_int], C.c_int),
        "qz_snapshot_wait": ([vp], C.c_int),
        "qz_adjoint_final_loss": ([vp, C.c_int, C.c_double, C.c_int] + [_P] * 10 +
                                  [C.POINTER(AdjointStats)], C.c_int),
        "qz_ptcl_idx_to_box_idx": ([C.c_int] * 6 + [C.c_long, _P, _P, _P, _I], C.c_int),
        "qz_tree_adaptation": ([vp], C.c_int),
        "qz_poisson_error": ([vp, _I], C.c_int),
        "qz_amr_levels": ([vp], C.c_int),
        "qz_amr_num_nodes": ([vp, C.c_int], C.c_int),
        "qz_amr_node_info": ([vp, C.c_int, C.c_int, _I, _P], C.c_int),
        "qz_amr_node_cells": ([vp, C.c_int, C.c_int, _I], C.c_int),
        "qz_amr_node_box": ([vp, C.c_int, C.c_int, _I], C.c_int),
        "qz_amr_node_list": ([vp, C.c_int, C.c_int, C.c_int, _I], C.c_int),
        "qz_amr_node_field": ([vp, C.c_int, C.c_int, C.c_int, _P], C.c_int),
        "qz_test_scan": ([vp, _I, _I, C.c_long, C.c_int, C.c_uint], C.c_int),
        "qz_solve_schedule": ([vp, C.c_int, _I, C.c_long, C.POINTER(C.c_long)], C.c_int),
        "qz_node_conjugate_gradient": ([vp] + [C.c_int] * 5 + [_I, C.c_double, C.c_int] +
                                       [_P] * 3, C.c_int),
        "qz_test_wait_gives_up": ([vp, C.c_int, _I], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return [n for n in dir(load()) if n.startswith("qz_")]


def _check(rc: int) -> None:
    if rc != 0:
        msg = load().qz_last_error().decode(errors="replace")
        raise QZError(msg or "libqzb200 call failed")


def _p(a: np.ndarray):
    if a.dtype == np.float64:
        return a.ctypes.data_as(_P)
    return a.ctypes.data_as(_I)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def config(lmin: int, **kw) -> Config:
    c = Config()
    _check(load().qz_default_config(C.byref(c), lmin))
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def sequential_mass(m: np.ndarray) -> float:
    """Total mass summed in index order, as the reference's input stage does."""
    return float(np.cumsum(np.asarray(m, dtype=np.float64))[-1]) if len(m) else 0.0


class Simulation:
    """Head-node particle-mesh simulation held on the current CUDA device."""

    def __init__(self, ic: dict, lmin: int, capacity: int | None = None, **cfg):
        self.lib = load()
        n = len(ic["x"])
        cfg.setdefault("total_mass", sequential_mass(ic["m"]))
        self.cfg = config(lmin, **cfg)
        h = C.c_void_p()
        _check(self.lib.qz_create(C.byref(self.cfg), capacity or n, C.byref(h)))
        self.h = h
        self.lmin = lmin
        self.set_particles(ic)

    # -- state ---------------------------------------------------------------------
    def set_particles(self, ic: dict) -> None:
        arrs = [_f64(ic[k]) for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        _check(self.lib.qz_set_particles(self.h, arrs[0].size, *[_p(a) for a in arrs]))

    def set_accelerations(self, ax, ay, az) -> None:
        a = [_f64(v) for v in (ax, ay, az)]
        _check(self.lib.qz_set_particle_accel(self.h, *[_p(v) for v in a]))

    def step_host(self, state: dict, dt: float) -> None:
        """One leapfrog step on host arrays (qz_step_host), as the reference's
        main loop keeps its state: x..vz, m, ax..az are copied to the device,
        advanced, and x..vz, ax..az are copied back into `state` (contiguous
        float64 arrays of length n; page-locked ones overlap the copies with
        the step)."""
        for k in ("x", "y", "z", "vx", "vy", "vz", "m", "ax", "ay", "az"):
            a = state[k]
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.size != self.n:
                raise QZError(f"step_host: {k} must be a contiguous float64 array of length n")
        _check(self.lib.qz_step_host(self.h, dt, *[_p(state[k]) for k in
                                                   ("x", "y", "z", "vx", "vy", "vz", "m", "ax",
                                                    "ay", "az")]))

    @property
    def n(self) -> int:
        return int(self.lib.qz_num_particles(self.h))

    def particles(self) -> dict:
        n = self.n
        out = {k: np.empty(n) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
        _check(self.lib.qz_get_particles(self.h, *[_p(out[k]) for k in
                                                   ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")]))
        return out

    def field(self, name: str) -> np.ndarray:
        g = int(self.lib.qz_head_grid_points(self.h))
        out = np.empty(g)
        _check(self.lib.qz_get_head_field(self.h, FIELDS[name], _p(out)))
        return out

    def set_field(self, name: str, values: np.ndarray) -> None:
        a = _f64(values)
        _check(self.lib.qz_set_head_field(self.h, FIELDS[name], _p(a)))

    def stats(self) -> Stats:
        s = Stats()
        _check(self.lib.qz_get_stats(self.h, C.byref(s)))
        return s

    @property
    def stream(self) -> int:
        return int(self.lib.qz_stream(self.h) or 0)

    # -- the reference's entry points ------------------------------------------------
    def reset(self): _check(self.lib.qz_reset(self.h))
    def grid_density(self): _check(self.lib.qz_grid_density(self.h))
    def potential(self): _check(self.lib.qz_potential(self.h))
    def grid_acceleration(self): _check(self.lib.qz_grid_acceleration(self.h))
    def particle_acceleration(self): _check(self.lib.qz_particle_acceleration(self.h))
    def particle_updating_A(self, dt): _check(self.lib.qz_particle_updating_A(self.h, dt))
    def particle_updating_B(self, dt): _check(self.lib.qz_particle_updating_B(self.h, dt))
    def initial_potential_head(self): _check(self.lib.qz_initial_potential_head(self.h))

    def tree_adaptation(self): _check(self.lib.qz_tree_adaptation(self.h))

    # -- refinement tree -------------------------------------------------------------------
    NODE_KEYS = ("lv", "parent", "ts", "rd", "bmin", "bmax", "ncells", "nintr", "nbdry",
                 "nsimb", "nptcl", "zone_base", "nzones", "contact")

    def levels(self) -> int:
        return int(self.lib.qz_amr_levels(self.h))

    def num_nodes(self, level: int) -> int:
        return int(self.lib.qz_amr_num_nodes(self.h, level))

    def node_info(self, level: int, node: int) -> dict:
        info = np.zeros(22, dtype=np.int32)
        mass = C.c_double()
        _check(self.lib.qz_amr_node_info(self.h, level, node, _p(info), C.byref(mass)))
        v = [int(a) for a in info]
        return {"lv": v[0], "parent": v[1], "ts": tuple(v[2:5]), "rd": tuple(v[5:8]),
                "bmin": tuple(v[8:11]), "bmax": tuple(v[11:14]), "ncells": v[14],
                "nintr": v[15], "nbdry": v[16], "nsimb": v[17], "nptcl": v[18],
                "zone_base": v[19], "nzones": v[20], "contact": v[21], "mass": mass.value}

    def node_cells(self, level: int, node: int) -> np.ndarray:
        n = self.node_info(level, node)["ncells"]
        out = np.zeros(3 * n, dtype=np.int32)
        _check(self.lib.qz_amr_node_cells(self.h, level, node, _p(out)))
        return out.reshape(n, 3)

    def node_box(self, level: int, node: int) -> np.ndarray:
        rd = self.node_info(level, node)["rd"]
        out = np.zeros(rd[0] * rd[1] * rd[2], dtype=np.int32)
        _check(self.lib.qz_amr_node_box(self.h, level, node, _p(out)))
        return out

    def node_list(self, level: int, node: int, which: str) -> np.ndarray:
        info = self.node_info(level, node)
        k = {"intr": 0, "bdry": 1, "simb": 2}[which]
        out = np.zeros(info[("nintr", "nbdry", "nsimb")[k]], dtype=np.int32)
        _check(self.lib.qz_amr_node_list(self.h, level, node, k, _p(out)))
        return out

    def node_field(self, level: int, node: int, name: str) -> np.ndarray:
        rd = self.node_info(level, node)["rd"]
        out = np.zeros((rd[0] + 1) * (rd[1] + 1) * (rd[2] + 1))
        _check(self.lib.qz_amr_node_field(self.h, level, node, FIELDS[name], _p(out)))
        return out

    def timestep(self) -> float:
        """CFL step of the current state (timestep.c:589-700)."""
        dt = C.c_double()
        _check(self.lib.qz_timestep(self.h, C.byref(dt)))
        return dt.value

    def observables(self, potential_type: int = 0, units=None) -> dict:
        """Energies and momentum (observables.c:661-696); units as qz_observables."""
        out = np.zeros(6)
        u = None if units is None else _p(np.ascontiguousarray(units, dtype=np.float64))
        _check(self.lib.qz_observables(self.h, potential_type, u, _p(out)))
        return {"kinetic": out[0], "potential": out[1], "total": out[2],
                "momentum": out[3:6].copy()}

    def init_forces(self) -> None:
        _check(self.lib.qz_init_forces(self.h))

    def outflow_removed(self):
        """(count, slots, sources) of the last step's outflow removals."""
        cnt = C.c_long()
        _check(self.lib.qz_outflow_removed(self.h, C.byref(cnt), None, None))
        slots = np.zeros(max(cnt.value, 1), dtype=np.int32)
        srcs = np.zeros(max(cnt.value, 1), dtype=np.int32)
        _check(self.lib.qz_outflow_removed(self.h, C.byref(cnt), _p(slots), _p(srcs)))
        return cnt.value, slots[:cnt.value], srcs[:cnt.value]

    def head_mass(self) -> float:
        return float(self.lib.qz_head_mass(self.h))

    def write_snapshot(self, path: str, actual_time: float, units=None,
                       observables_type: int = -1, wait: bool = True) -> None:
        """Snapshot file in the layout of output_snapshots.c:141-239
        (qz_write_snapshot); units as there, observables_type -1 for none."""
        self._snap_units = None if units is None else np.ascontiguousarray(units, dtype=np.float64)
        u = None if self._snap_units is None else _p(self._snap_units)
        _check(self.lib.qz_write_snapshot(self.h, path.encode(), actual_time, u,
                                          observables_type, 0 if wait else 1))

    def snapshot_wait(self) -> None:
        _check(self.lib.qz_snapshot_wait(self.h))

    def force_vjp(self, abx, aby, abz) -> dict:
        """(dF/dx)^T abar and (dF/dm)^T abar of the head force at the current
        state (qz_force_vjp); keys gx, gy, gz, gm."""
        a = [_f64(v) for v in (abx, aby, abz)]
        n = self.n
        out = {k: np.empty(n) for k in ("gx", "gy", "gz", "gm")}
        _check(self.lib.qz_force_vjp(self.h, *[_p(v) for v in a],
                                     *[_p(out[k]) for k in ("gx", "gy", "gz", "gm")]))
        return out

    def adjoint_final_loss(self, nsteps: int, dt: float, targets: dict,
                           checkpoint_every: int = 0) -> dict:
        """Gradients of L = mean_p |x_T,p - x*_p|^2 after nsteps fixed-dt steps
        with respect to the current x, v, m (qz_adjoint_final_loss); the
        simulation is left at step nsteps.  Keys gx..gz, gvx..gvz, gm, loss,
        stats (AdjointStats as a dict)."""
        t = [_f64(targets[k]) for k in ("x", "y", "z")]
        n = self.n
        keys = ("gx", "gy", "gz", "gvx", "gvy", "gvz", "gm")
        out = {k: np.empty(n) for k in keys}
        st = AdjointStats()
        _check(self.lib.qz_adjoint_final_loss(self.h, nsteps, dt, checkpoint_every,
                                              *[_p(v) for v in t],
                                              *[_p(out[k]) for k in keys], C.byref(st)))
        out["loss"] = st.loss
        out["stats"] = {f: getattr(st, f) for f, _ in AdjointStats._fields_}
        return out

    # -- solver schedule (finite-difference checks) ---------------------------------
    def record_schedule(self) -> None:
        """Record the iteration count of every forward Poisson solve from now on."""
        _check(self.lib.qz_solve_schedule(self.h, 1, None, 0, None))

    def take_schedule(self) -> np.ndarray:
        """Stop recording (or replaying) and return the recorded counts."""
        n = C.c_long()
        _check(self.lib.qz_solve_schedule(self.h, 0, None, 0, C.byref(n)))
        out = np.zeros(max(n.value, 1), dtype=np.int32)
        _check(self.lib.qz_solve_schedule(self.h, 0, _p(out), n.value, C.byref(n)))
        return out[:n.value]

    def replay_schedule(self, counts) -> None:
        """Every forward solve from now on runs exactly the next recorded count."""
        c = np.ascontiguousarray(counts, dtype=np.int32)
        _check(self.lib.qz_solve_schedule(self.h, 2, _p(c), c.size, None))

    def step(self, dt: float, nsteps: int = 1) -> None:
        _check(self.lib.qz_step(self.h, dt, nsteps))

    def synchronize(self) -> None:
        _check(self.lib.qz_synchronize(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.qz_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


# -- array-level routines ---------------------------------------------------------------
def ensemble_step(sims: list, dt, nsteps: int = 1, threads: int = 8) -> None:
    """Steps independent Simulations concurrently (qz_ensemble_step); dt is one
    step for all, one per member, or None for CFL steps."""
    arr = (C.c_void_p * len(sims))(*[s.h for s in sims])
    if dt is None:
        d = None
    else:
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(sims),)))
    _check(load().qz_ensemble_step(arr, len(sims), None if d is None else _p(d), nsteps, threads))


def ensemble_autotune(sims: list, dt, thread_opts=(4, 8, 16, 32, 64), ppt_opts=(2, 4, 8),
                      tile_opts=(-1, 1, 5, 6)):
    """Picks the host thread count, multigrid points per thread and tile core of
    the tiled multigrid phases (mg_tile) of the batching form by timing one
    ensemble step per combination (qz_ensemble_autotune; the members' states are
    put back).  Returns (threads, points_per_thread, mg_tile, ms)."""
    arr = (C.c_void_p * len(sims))(*[s.h for s in sims])
    d = None if dt is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(dt, dtype=np.float64), (len(sims),)))
    to = (C.c_int * len(thread_opts))(*thread_opts)
    po = (C.c_int * len(ppt_opts))(*ppt_opts)
    go = (C.c_int * len(tile_opts))(*tile_opts)
    bt, bp, bg, bms = C.c_int(), C.c_int(), C.c_int(), C.c_double()
    _check(load().qz_ensemble_autotune(arr, len(sims), None if d is None else _p(d), to,
                                       len(thread_opts), po, len(ppt_opts), go, len(tile_opts),
                                       C.byref(bt), C.byref(bp), C.byref(bg), C.byref(bms)))
    return bt.value, bp.value, bg.value, bms.value


def gauss_saidel(phi: np.ndarray, rho: np.ndarray, iters: int, w: float = 1.0,
                 order: int = QZ_GS_REDBLACK) -> np.ndarray:
    n = round(phi.size ** (1 / 3))
    out = _f64(phi).copy()
    r = _f64(rho)
    _check(load().qz_gauss_saidel(_p(out), _p(r), n, iters, w, order))
    return out


def jacobi(phi: np.ndarray, rho: np.ndarray, iters: int, w: float = 1.0) -> np.ndarray:
    n = round(phi.size ** (1 / 3))
    out = _f64(phi).copy()
    r = _f64(rho)
    _check(load().qz_jacobi(_p(out), _p(r), n, iters, w))
    return out


def conjugate_gradient_multigrid(phi: np.ndarray, rho: np.ndarray, iters: int) -> np.ndarray:
    """conjugate_gradient_multigrid.c:29-176 on a gridsize^3 array (returns a copy)."""
    n = round(phi.size ** (1 / 3))
    out = _f64(phi).copy()
    r = _f64(rho)
    _check(load().qz_conjugate_gradient_multigrid(_p(out), _p(r), n, iters))
    return out


def multigrid(phi: np.ndarray, rho: np.ndarray, cycle: int = 0, **cfg) -> np.ndarray:
    n = round(phi.size ** (1 / 3))
    c = config(2, **cfg)
    out = _f64(phi).copy()
    r = _f64(rho)
    _check(load().qz_multigrid(C.byref(c), _p(out), _p(r), n, cycle))
    return out


def ptcl_idx_to_box_idx(lv: int, box_ts: tuple, box_real_dim: tuple, x, y, z) -> np.ndarray:
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.empty(x.size, dtype=np.int32)
    _check(load().qz_ptcl_idx_to_box_idx(lv, box_ts[0], box_ts[1], box_ts[2], box_real_dim[0],
                                         box_real_dim[1], x.size, _p(x), _p(y), _p(z), _p(out)))
    return out


# -- per-launch profiler ---------------------------------------------------------------
PROF_CATEGORIES = ("smooth", "restrict", "prolong", "check", "deposit", "sort", "gradient",
                   "gather", "leapfrog", "other", "tree", "cg", "node_mg")


def _prof_sig(lib):
    if getattr(lib, "_prof_ready", False):
        return
    lib.qz_profile_enable.argtypes = [C.c_void_p, C.c_int]
    lib.qz_profile_reset.argtypes = [C.c_void_p]
    lib.qz_profile_read.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_longlong),
                                    C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib._prof_ready = True


def profile_enable(sim: Simulation, on: bool = True) -> None:
    _prof_sig(sim.lib)
    _check(sim.lib.qz_profile_enable(sim.h, 1 if on else 0))


def profile_reset(sim: Simulation) -> None:
    _prof_sig(sim.lib)
    _check(sim.lib.qz_profile_reset(sim.h))


def profile_read(sim: Simulation) -> dict:
    """{category: (launches, total_ms, algorithmic_bytes)} since the last reset."""
    _prof_sig(sim.lib)
    out = {}
    for i, name in enumerate(PROF_CATEGORIES):
        n, ms, b = C.c_longlong(), C.c_double(), C.c_double()
        _check(sim.lib.qz_profile_read(sim.h, i, C.byref(n), C.byref(ms), C.byref(b)))
        out[name] = (int(n.value), float(ms.value), float(b.value))
    return out

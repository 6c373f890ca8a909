"""ctypes front end of the CPU oracle (qz_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker of the CUDA library.  Imported by
tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg, never by the
product package.  ``load()`` compiles oracle/_build/libqzoracle.so with gcc
when it is missing (gcc is present wherever the tests run).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libqzoracle.so")
REF_DRIVER = os.path.join(HERE, "_ref", "qz_ref_driver")
DROPIN_DRIVER = os.path.join(HERE, "_ref", "qz_dropin_driver")
DROPIN_AMR_DRIVER = os.path.join(HERE, "_ref", "qz_dropin_amr_driver")

_P = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class Params(C.Structure):
    _fields_ = [
        ("L", C.c_int), ("G", C.c_double), ("total_mass", C.c_double), ("bdry", C.c_int),
        ("solver", C.c_int), ("cycle", C.c_int), ("n_pre", C.c_int), ("n_post", C.c_int),
        ("n_coarse", C.c_int), ("w_sor", C.c_double), ("tol", C.c_double), ("tol2", C.c_double),
        ("check_every", C.c_int), ("max_iter", C.c_int), ("check_method", C.c_int),
        ("force_stencil", C.c_int), ("head_pot_method", C.c_int),
    ]


class Sim(C.Structure):
    _fields_ = [("p", Params), ("n", C.c_long)] + [
        (k, _P) for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az", "m",
                          "pot", "pot_old", "d", "gax", "gay", "gaz")
    ] + [("vcycles_total", C.c_long), ("last_vcycles", C.c_int), ("head_mass", C.c_double)]


_lib = None


def build(force: bool = False) -> str:
    src = os.path.join(HERE, "qz_oracle.c")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", HERE, "restate"], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        build()
        lib = C.CDLL(LIB)
        lib.qzo_default_params.argtypes = [C.POINTER(Params), C.c_int]
        lib.qzo_grid_points.restype = C.c_long
        lib.qzo_grid_points.argtypes = [C.c_int]
        lib.qzo_initial_head.argtypes = [C.POINTER(Params), _P, _P, _P, _P]
        lib.qzo_deposit_head.argtypes = [C.POINTER(Params), C.c_long, _P, _P, _P, _P, _P]
        lib.qzo_gauss_saidel.argtypes = [_P, _P, C.c_int, C.c_int, C.c_double]
        lib.qzo_jacobi.argtypes = [_P, _P, C.c_int, C.c_int, C.c_double]
        lib.qzo_cg_smooth.argtypes = [_P, _P, C.c_int, C.c_int]
        lib.qzo_timestep_head.restype = C.c_double
        lib.qzo_timestep_head.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_long] + [_P] * 6
        lib.qzo_multigrid.argtypes = [C.POINTER(Params), _P, _P, C.c_int, C.c_int]
        lib.qzo_poisson_check_head.argtypes = [C.POINTER(Params), _P, _P, _P, C.c_double]
        lib.qzo_potential_head.argtypes = [C.POINTER(Params), _P, _P, _P, C.c_double]
        lib.qzo_grid_accel_head.argtypes = [C.POINTER(Params), _P, _P, _P, _P]
        lib.qzo_gather_head.argtypes = [C.POINTER(Params), C.c_long, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        lib.qzo_update_A_head.argtypes = [C.POINTER(Params), C.c_long, C.c_double] + [_P] * 9
        lib.qzo_update_B_head.argtypes = [C.c_long, C.c_double] + [_P] * 6
        lib.qzo_box_idx_batch.argtypes = [C.c_int] * 6 + [C.c_long, _P, _P, _P, _I]
        lib.qzo_sim_init.argtypes = [C.POINTER(Sim), C.POINTER(Params), C.c_long] + [_P] * 7
        lib.qzo_sim_step.argtypes = [C.POINTER(Sim), C.c_double]
        lib.qzo_sim_free.argtypes = [C.POINTER(Sim)]
        _lib = lib
    return _lib


def ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    if a.dtype == np.float64:
        return a.ctypes.data_as(_P)
    if a.dtype == np.int32:
        return a.ctypes.data_as(_I)
    raise TypeError(a.dtype)


def params(L: int, **kw) -> Params:
    p = Params()
    load().qzo_default_params(C.byref(p), L)
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def grid_points(L: int) -> int:
    return int(load().qzo_grid_points(L))


class OracleSim:
    """Head-only simulation on the CPU oracle (main.c call order, fixed dt)."""

    def __init__(self, ic: dict, p: Params):
        self.lib = load()
        self.s = Sim()
        self._keep = [np.ascontiguousarray(ic[k], dtype=np.float64)
                      for k in ("x", "y", "z", "vx", "vy", "vz", "m")]
        n = self._keep[0].size
        rc = self.lib.qzo_sim_init(C.byref(self.s), C.byref(p), n, *[ptr(a) for a in self._keep])
        if rc:
            raise RuntimeError("oracle potential did not converge")
        self.n = n
        self.L = p.L

    def step(self, dt: float) -> None:
        if self.lib.qzo_sim_step(C.byref(self.s), dt):
            raise RuntimeError("oracle step failed")

    def particles(self) -> dict:
        n = int(self.s.n)
        return {k: np.ctypeslib.as_array(getattr(self.s, k), shape=(n,)).copy()
                for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}

    def fields(self) -> dict:
        g = grid_points(self.L)
        return {k: np.ctypeslib.as_array(getattr(self.s, k), shape=(g,)).copy()
                for k in ("pot", "pot_old", "d", "gax", "gay", "gaz")}

    @property
    def vcycles_total(self) -> int:
        return int(self.s.vcycles_total)

    @property
    def last_vcycles(self) -> int:
        return int(self.s.last_vcycles)

    def close(self) -> None:
        if self.s is not None:
            self.lib.qzo_sim_free(C.byref(self.s))
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_reference(ic_path: str, out_dir: str, driver: str = REF_DRIVER, **kw) -> dict:
    """Run a compiled driver (reference or drop-in) and return its JSON summary."""
    import json
    args = [driver, ic_path, out_dir] + [f"{k}={v}" for k, v in kw.items()]
    r = subprocess.run(args, check=True, capture_output=True, text=True)
    return json.loads(r.stdout.strip().splitlines()[-1])


def read_dump(out_dir: str, step: int, name: str, dtype=np.float64) -> np.ndarray:
    return np.fromfile(os.path.join(out_dir, f"s{step}_{name}.bin"), dtype=dtype)


def read_nodes(out_dir: str, step: int) -> list:
    """Node summary written by the drivers for refinement runs: one dict per
    node (tentacle level, index, geometry, list sizes, particles, mass, parent)."""
    nodes = []
    for line in open(os.path.join(out_dir, f"s{step}_nodes.txt")):
        if line.startswith("#"):
            continue
        f = line.split()
        v = [int(a) for a in f[:22]]
        nodes.append({
            "lv": v[0], "idx": v[1], "ID": v[2], "rd": tuple(v[3:6]), "ts": tuple(v[6:9]),
            "bmin": tuple(v[9:12]), "bmax": tuple(v[12:15]), "ncells": v[15], "nintr": v[16],
            "nbdry": v[17], "nsimb": v[18], "nptcl": v[19], "nptcl_outs": v[20],
            "nchildren": v[21], "mass": float(f[22]), "parent_level": int(f[23]),
            "parent": int(f[24]),
        })
    base = nodes[0]["lv"] if nodes else 0
    for nd in nodes:
        nd["level"] = nd["lv"] - base
    return nodes


def node_dump(out_dir: str, step: int, level: int, idx: int, what: str) -> np.ndarray:
    """Per-node arrays: intr, bdry, simbdry, box, cells, cx, cy, cz (int32) or
    pot, d, ax, ay, az (float64)."""
    dt = np.int32 if what in ("intr", "bdry", "simbdry", "box", "cells", "cx", "cy", "cz") else np.float64
    return read_dump(out_dir, step, f"L{level}_N{idx}_{what}", dt)

"""Seeded synthetic initial conditions in code units (unit box, G = 1).

QUANTIZER reads its particles from a 7-column CSV (x y z vx vy vz m) and
recentres them on the box centre (source/input.c:117-186, 280-304), aborting
if any particle falls outside (0, 1).  These generators produce the same seven
arrays directly in code units, centred at (0.5, 0.5, 0.5):

* ``plummer``  -- positions from the inverse cumulative mass
  r = a / sqrt(u^(-2/3) - 1), speeds from the Plummer distribution function by
  rejection sampling of q^2 (1 - q^2)^(7/2), q = v / v_esc (Aarseth, Henon &
  Wielen 1974), isotropic directions; truncated at ``rmax`` (resampled) so that
  every particle lies strictly inside the box.
* ``hernquist`` -- r = a sqrt(u) / (1 - sqrt(u)), speeds by rejection from the
  Hernquist (1990) isotropic distribution function f(E), truncated at ``rmax``
  and renormalised to total mass ``M``.
* ``crossing_time`` -- t_cr = 2 sqrt(2) (R_v^3 / G M)^(1/2), R_v = 16 a / (3 pi),
  the fixed-dt convention of the Plummer workloads (dt = 1e-3 t_cr).
"""
from __future__ import annotations

import math
import struct

import numpy as np


def _isotropic(rng: np.random.Generator, n: int) -> np.ndarray:
    cos_t = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * math.pi, n)
    sin_t = np.sqrt(1.0 - cos_t * cos_t)
    return np.stack([sin_t * np.cos(phi), sin_t * np.sin(phi), cos_t])


def plummer(n: int, a: float = 0.05, M: float = 1.0, G: float = 1.0,
            seed: int = 0, rmax: float = 0.45, center=(0.5, 0.5, 0.5)) -> dict:
    """Equal-mass Plummer sphere; returns dict of float64 arrays x..vz, m."""
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    filled = 0
    while filled < n:
        u = rng.uniform(0.0, 1.0, 2 * (n - filled) + 16)
        u = u[u > 0.0]
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        rr = rr[rr <= rmax]
        take = min(n - filled, rr.size)
        r[filled:filled + take] = rr[:take]
        filled += take
    pos = _isotropic(rng, n) * r
    q = np.empty(n)
    filled = 0
    while filled < n:
        m = 2 * (n - filled) + 16
        x = rng.uniform(0.0, 1.0, m)
        y = rng.uniform(0.0, 0.1, m)
        ok = x[y < x * x * (1.0 - x * x) ** 3.5]
        take = min(n - filled, ok.size)
        q[filled:filled + take] = ok[:take]
        filled += take
    vesc = np.sqrt(2.0 * G * M / np.sqrt(r * r + a * a))
    vel = _isotropic(rng, n) * (q * vesc)
    c = np.asarray(center, dtype=np.float64)[:, None]
    pos = pos + c
    return {
        "x": pos[0].copy(), "y": pos[1].copy(), "z": pos[2].copy(),
        "vx": vel[0].copy(), "vy": vel[1].copy(), "vz": vel[2].copy(),
        "m": np.full(n, M / n),
    }


def _hernquist_f(e: np.ndarray) -> np.ndarray:
    """Hernquist (1990) isotropic DF in units G = M = a = 1, e = -E in (0, 1)."""
    e = np.clip(e, 1e-300, 1.0 - 1e-15)
    s = np.sqrt(e)
    return (s / (1.0 - e) ** 2) * ((1.0 - 2.0 * e) * (8.0 * e * e - 8.0 * e - 3.0)
                                   + 3.0 * np.arcsin(s) / np.sqrt(e * (1.0 - e)))


def hernquist(n: int, a: float = 0.03, M: float = 1.0, G: float = 1.0,
              seed: int = 0, rmax: float = 0.14, center=(0.5, 0.5, 0.5),
              bulk_v=(0.0, 0.0, 0.0)) -> dict:
    """Hernquist sphere truncated at rmax, per-particle mass M/n."""
    rng = np.random.default_rng(seed)
    r = np.empty(n)
    filled = 0
    while filled < n:
        u = rng.uniform(0.0, 1.0, 2 * (n - filled) + 16)
        su = np.sqrt(u)
        rr = a * su / (1.0 - su)
        rr = rr[rr <= rmax]
        take = min(n - filled, rr.size)
        r[filled:filled + take] = rr[:take]
        filled += take
    # Dimensionless: psi = 1 / (1 + s), s = r / a; speed v = w * sqrt(2 psi) in
    # units sqrt(G M / a).  g(w) ~ w^2 f(psi (1 - w^2)).
    s = r / a
    psi = 1.0 / (1.0 + s)
    w = np.empty(n)
    todo = np.arange(n)
    while todo.size:
        ww = rng.uniform(0.0, 1.0, todo.size)
        g = ww * ww * _hernquist_f(psi[todo] * (1.0 - ww * ww))
        # envelope: w^2 f(psi(1-w^2)) <= f(psi) (f increasing in e)
        gmax = _hernquist_f(psi[todo])
        acc = rng.uniform(0.0, 1.0, todo.size) * gmax < g
        w[todo[acc]] = ww[acc]
        todo = todo[~acc]
    speed = w * np.sqrt(2.0 * psi) * math.sqrt(G * M / a)
    pos = _isotropic(rng, n) * r
    vel = _isotropic(rng, n) * speed
    c = np.asarray(center, dtype=np.float64)[:, None]
    bv = np.asarray(bulk_v, dtype=np.float64)[:, None]
    pos = pos + c
    vel = vel + bv
    return {
        "x": pos[0].copy(), "y": pos[1].copy(), "z": pos[2].copy(),
        "vx": vel[0].copy(), "vy": vel[1].copy(), "vz": vel[2].copy(),
        "m": np.full(n, M / n),
    }


def merger(n_each: int, a: float = 0.03, M: float = 1.0, G: float = 1.0, seed: int = 0,
           rmax: float = 0.14, sep: float = 0.3) -> dict:
    """Two Hernquist spheres of mass M each, centred at 0.5 -/+ sep/2 on x and
    approaching along x at half the mutual escape speed sqrt(2 G (2M) / sep)
    (each moving at a quarter of it), truncated at rmax (per-particle mass
    renormalised to M per sphere)."""
    v = 0.25 * math.sqrt(2.0 * G * 2.0 * M / sep)
    left = hernquist(n_each, a=a, M=M, G=G, seed=2 * seed, rmax=rmax,
                     center=(0.5 - sep / 2, 0.5, 0.5), bulk_v=(v, 0.0, 0.0))
    right = hernquist(n_each, a=a, M=M, G=G, seed=2 * seed + 1, rmax=rmax,
                      center=(0.5 + sep / 2, 0.5, 0.5), bulk_v=(-v, 0.0, 0.0))
    return {k: np.concatenate([left[k], right[k]]) for k in left}


def crossing_time(a: float, M: float = 1.0, G: float = 1.0) -> float:
    rv = 16.0 * a / (3.0 * math.pi)
    return 2.0 * math.sqrt(2.0) * math.sqrt(rv ** 3 / (G * M))


FIELDS = ("x", "y", "z", "vx", "vy", "vz", "m")


def write_ic(path: str, ic: dict) -> None:
    """Binary IC: int64 N then x y z vx vy vz m as float64 arrays."""
    n = ic["x"].size
    with open(path, "wb") as f:
        f.write(struct.pack("<q", n))
        for k in FIELDS:
            f.write(np.ascontiguousarray(ic[k], dtype=np.float64).tobytes())


def read_ic(path: str) -> dict:
    with open(path, "rb") as f:
        (n,) = struct.unpack("<q", f.read(8))
        out = {}
        for k in FIELDS:
            out[k] = np.frombuffer(f.read(8 * n), dtype=np.float64).copy()
    return out

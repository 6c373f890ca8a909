"""Generate the golden fixtures of tests/golden/ from the compiled reference.

QUANTIZER ships no tests or golden vectors, so every fixture here is produced
by running the reference's own FP64 code, compiled unmodified from its
sources (oracle/Makefile, target ``ref``):

* ``head_L4_plummer1000.npz`` -- oracle/_ref/qz_ref_driver (the reference's
  main-loop call order, fixed dt) on a 1000-particle Plummer sphere, head
  16^3, 3 steps: head fields and particle state at steps 0 and 3, and the
  head box index of every particle (ptcl_idx_to_box_idx).
* ``head_L3_jacobi.npz`` -- the same with the Jacobi smoother (solver 1), head
  8^3, 2 steps.
* ``head_L4_stencil5.npz`` -- the head_L4 case with the 5-point force stencil
  (force_stencil = 1).
* ``head_L4_cgsmooth.npz`` -- the head_L4 case, 2 steps, with conjugate
  gradient as the multigrid smoother (solver 2).
* ``head_L4_cghead.npz`` -- the head_L4 case with the head solved by the node
  conjugate gradient (head_pot_method = 1) instead of multigrid cycles.
* ``head_L4_periodic.npz`` / ``head_L4_periodic5.npz`` -- periodic boundaries
  (bdry_cond_type = 0; 3- and 5-point stencils) on the 1000-particle sphere
  with 48 extra particles placed 1e-6 inside the faces and moving outwards, so
  that they wrap in the first step; 3 steps.
* ``head_L4_outflow.npz`` -- outflow boundaries (bdry_cond_type = 2) on the same
  set: the particles that leave are removed (particle count and arrays after 3
  steps, in the reference's order).
* ``timestep_head_L4.npz`` -- the reference's timestep() (methods 0 and 1) on the
  states of the head_L4 case at steps 0 and 3 (_MAX_dt_ set to 1 so that the CFL
  condition decides), with its _MAX_dt_ and _CFL_.
* ``arrays.npz`` -- direct calls into oracle/_ref/libqzref.so of the
  reference's gauss_saidel, jacobi (odd sweep count), conjugate_gradient_multigrid
  and multigrid (V, F and W cycles) on seeded random arrays.
* ``node_cg.npz`` -- the reference's conjugate_gradient(struct node *)
  (force_methods/conjugate_gradient.c:322-463) called through libqzref.so on a
  synthetic node: a 30 x 32 x 34-cell box at level 7 whose interior points
  fill an ellipsoid, a smooth positive density, boundary values of -GM/r;
  inputs and the pot / pot_old it leaves.

Run in a container that has the reference source tree:
    python tests/golden/make_golden.py [fixture-name ...]   (default: all)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from quantizer_b200 import ics  # noqa: E402

FIELDS = ("pot", "d", "gax", "gay", "gaz")
PTCL = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def run_case(name: str, ic: dict, steps: int, dt: float, **kw) -> None:
    with tempfile.TemporaryDirectory() as td:
        icp = os.path.join(td, "ic.bin")
        ics.write_ic(icp, ic)
        summary = O.run_reference(icp, td, steps=steps, dt=dt, dump=f"0,{steps}", **kw)
        out = {f"ic_{k}": ic[k] for k in ics.FIELDS}
        for s in (0, steps):
            for f in FIELDS + PTCL:
                out[f"s{s}_{f}"] = O.read_dump(td, s, f)
            out[f"s{s}_bidx"] = O.read_dump(td, s, "bidx", np.int32)
        out["meta"] = np.array([kw.get("lmin", 5), steps, dt, summary["n"]], dtype=np.float64)
    np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote", name, summary)


def edge_ic(ic: dict) -> dict:
    """The sphere plus 48 particles 1e-6 inside the six faces (8 per face),
    moving outwards at speed 2 (box units per unit time)."""
    rng = np.random.default_rng(5)
    extra = {k: [] for k in ics.FIELDS}
    for axis in range(3):
        for side in (0, 1):
            for _ in range(8):
                pos = rng.uniform(0.2, 0.8, 3)
                vel = rng.normal(0.0, 0.1, 3)
                pos[axis] = 1e-6 if side == 0 else 1.0 - 1e-6
                vel[axis] = -2.0 if side == 0 else 2.0
                for q, k in enumerate(("x", "y", "z")):
                    extra[k].append(pos[q])
                for q, k in enumerate(("vx", "vy", "vz")):
                    extra[k].append(vel[q])
                extra["m"].append(ic["m"][0])
    return {k: np.concatenate([ic[k], np.array(extra[k])]) for k in ics.FIELDS}


def timestep_case(ic: dict, dt: float) -> None:
    """The reference's timestep() (both methods) on the states of the head_L4 case."""
    out = {}
    for tsm in (0, 1):
        with tempfile.TemporaryDirectory() as td:
            icp = os.path.join(td, "ic.bin")
            ics.write_ic(icp, ic)
            summary = O.run_reference(icp, td, steps=3, dt=dt, dump="0,3", lmin=4, tsm=tsm,
                                      max_dt=1.0)
            for s in (0, 3):
                out[f"m{tsm}_s{s}_dt"] = O.read_dump(td, s, "dtcfl")
            out["max_dt"] = np.array([summary["max_dt"]])
            out["cfl"] = np.array([summary["cfl"]])
    np.savez_compressed(os.path.join(HERE, "timestep_head_L4.npz"), **out)
    print("wrote timestep_head_L4.npz", {k: v.tolist() for k, v in out.items()})


def arrays_case() -> None:
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libqzref.so"))
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)
    try:
        lib.global_variables()  # sets _Onesixth_, smoother choices, sweep counts
    finally:
        os.dup2(saved, 1)
        os.close(devnull)
    P = C.POINTER(C.c_double)
    lib.gauss_saidel.argtypes = [P, P, C.c_int, C.c_int]
    lib.jacobi.argtypes = [P, P, C.c_int, C.c_int]
    lib.multigrid.argtypes = [P, P, C.c_int, C.c_int]
    rng = np.random.default_rng(1234)
    out = {}

    def fresh(n):
        # few significant bits, so the stored inputs compress well
        phi = rng.integers(-1024, 1024, n ** 3).astype(np.float64) / 256.0
        rho = rng.integers(-1024, 1024, n ** 3).astype(np.float64) / 4.0
        return phi, rho

    for n, iters in ((9, 2), (17, 3)):
        phi, rho = fresh(n)
        out[f"gs_n{n}_in_phi"], out[f"gs_n{n}_in_rho"] = phi.copy(), rho.copy()
        lib.gauss_saidel(phi.ctypes.data_as(P), rho.ctypes.data_as(P), n, iters)
        out[f"gs_n{n}_out"] = phi
        out[f"gs_n{n}_iters"] = np.array([iters])
    for n, iters in ((9, 3), (17, 2)):
        phi, rho = fresh(n)
        out[f"jac_n{n}_in_phi"], out[f"jac_n{n}_in_rho"] = phi.copy(), rho.copy()
        lib.jacobi(phi.ctypes.data_as(P), rho.ctypes.data_as(P), n, iters)
        out[f"jac_n{n}_out"] = phi
        out[f"jac_n{n}_iters"] = np.array([iters])
    lib.conjugate_gradient_multigrid.argtypes = [P, P, C.c_int, C.c_int]
    for n, iters in ((9, 4), (17, 6)):
        phi, rho = fresh(n)
        out[f"cgs_n{n}_in_phi"], out[f"cgs_n{n}_in_rho"] = phi.copy(), rho.copy()
        lib.conjugate_gradient_multigrid(phi.ctypes.data_as(P), rho.ctypes.data_as(P), n, iters)
        out[f"cgs_n{n}_out"] = phi
        out[f"cgs_n{n}_iters"] = np.array([iters])
    for n, types in ((9, (0, 1, 2)), (17, (0, 1, 2)), (33, (0,))):
        for t in types:
            phi, rho = fresh(n)
            out[f"mg_n{n}_t{t}_in_phi"], out[f"mg_n{n}_t{t}_in_rho"] = phi.copy(), rho.copy()
            lib.multigrid(phi.ctypes.data_as(P), rho.ctypes.data_as(P), n, t)
            out[f"mg_n{n}_t{t}_out"] = phi
    np.savez_compressed(os.path.join(HERE, "arrays.npz"), **out)
    print("wrote arrays.npz")


def node_struct():
    """ctypes mirror of struct node (headers/initialize_node.h:63-216), the layout
    quantizer_b200/csrc/qz_ref_abi.h declares."""
    I, D, B, PI, PD = C.c_int, C.c_double, C.c_bool, C.POINTER(C.c_int), C.POINTER(C.c_double)
    V = C.c_void_p
    fields = [("ID", I), ("lv", I), ("ptr_box", PI), ("ptr_box_old", PI), ("box_cap", I)]
    fields += [(f"box_real_dim_{a}", I) for a in "xyz"] + [(f"box_dim_{a}", I) for a in "xyz"]
    fields += [(f"box_ts_{a}", I) for a in "xyz"] + [(f"box_min_{a}", I) for a in "xyz"]
    fields += [(f"box_max_{a}", I) for a in "xyz"] + [("box_check_fit", B)]
    fields += [("ptr_cell_idx_x", PI), ("ptr_cell_idx_y", PI), ("ptr_cell_idx_z", PI),
               ("ptr_box_idx", PI), ("cell_cap", I), ("cell_size", I), ("ptr_cell_struct", V),
               ("ptr_cell_struct_old", V), ("cell_struct_old_cap", I), ("node_mass", D),
               ("no_ptcl_full_node", I), ("no_ptcl_outs_ref_zones", I)]
    for w in ("intr", "bdry", "sim_bdry"):
        fields += [(f"ptr_{w}_grid_cell_idx_{a}", PI) for a in "xyz"]
        fields += [(f"ptr_{w}_box_grid_idx", PI), (f"grid_{w}_cap", I), (f"grid_{w}_size", I)]
    fields += [(f"ptr_{f}", PD) for f in ("pot", "pot_old", "ax", "ay", "az", "d")]
    fields += [("grid_properties_cap", I), ("pptr_chn", V), ("ptr_pt", V), ("chn_cap", I),
               ("chn_size", I), ("ptr_cell_ref", PI), ("cell_ref_cap", I), ("cell_ref_size", I),
               ("pptr_zones", V), ("zones_cap", I), ("zones_size", I), ("ptr_zone_cap", PI),
               ("ptr_zone_size", PI), ("ptr_aux_idx", PI), ("aux_idx_cap", I)]
    fields += [(f"ptr_pbc_bool_bdry_anomalies_{a}", V) for a in "xyz"]
    fields += [("pbc_bool_bdry_anomalies_cap", I)]
    fields += [(f"ptr_pbc_min_subzones_{a}", PI) for a in "xyz"]
    fields += [(f"ptr_pbc_max_subzones_{a}", PI) for a in "xyz"]
    fields += [("pbc_subzones_cap", I), ("pbc_subzones_size", I)]
    fields += [(f"ptr_links_{k}", PI) for k in ("old_ord_old", "new_ord_new", "new_ord_old",
                                                 "old_ord_new")]
    fields += [("links_cap", I)]
    fields += [(n, B) for n in ("sim_bdry_contact", "sim_bdry_contact_x", "sim_bdry_contact_y",
                                "sim_bdry_contact_z", "pbc_crosses_sim_box_bdry",
                                "pbc_crosses_sim_box_bdry_x", "pbc_crosses_sim_box_bdry_y",
                                "pbc_crosses_sim_box_bdry_z", "pbc_crosses_whole_sim_box",
                                "pbc_crosses_whole_sim_box_x", "pbc_crosses_whole_sim_box_y",
                                "pbc_crosses_whole_sim_box_z", "pbc_correction_due_pbc_flag")]

    class Node(C.Structure):
        _fields_ = fields
    return Node


def node_cg_case() -> None:
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libqzref.so"))
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)
    try:
        lib.global_variables()
    finally:
        os.dup2(saved, 1)
    Node = node_struct()
    lv, rd = 7, (30, 32, 34)
    sx, sy, sz = rd[0] + 1, rd[1] + 1, rd[2] + 1
    H = 1.0 / (1 << lv)
    gz, gy, gx = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    c = np.array([rd[0] / 2, rd[1] / 2, rd[2] / 2])
    q = ((gx - c[0]) / 12.0) ** 2 + ((gy - c[1]) / 13.0) ** 2 + ((gz - c[2]) / 14.0) ** 2
    inside = (q < 1.0) & (gx > 0) & (gy > 0) & (gz > 0) & (gx < rd[0]) & (gy < rd[1]) & (gz < rd[2])
    intr = np.flatnonzero(inside.ravel()).astype(np.int32)
    # level coordinates: the box starts at cell 40 of the level (centre of mass near 0.5)
    X = (gx + 49) * H - 0.5
    Y = (gy + 48) * H - 0.5
    Z = (gz + 47) * H - 0.5
    r = np.sqrt(X * X + Y * Y + Z * Z)
    d = (4.0 * np.pi * 3.0 / (4.0 * np.pi * 0.05 ** 3) * (1 + (r / 0.05) ** 2) ** -2.5).ravel()
    d = np.where(inside.ravel(), d, 0.0)
    pot = (-1.0 / np.sqrt(r * r + 0.05 ** 2)).ravel().copy()
    pot_old = pot.copy()
    out = {"rd": np.array(rd, dtype=np.int32), "lv": np.array([lv]), "intr": intr,
           "d": d.copy(), "pot_in": pot.copy()}
    cells = int(np.count_nonzero(inside)) // 2 + 1
    mass = 0.7
    nd = Node()
    nd.ID, nd.lv = 1, lv
    nd.box_real_dim_x, nd.box_real_dim_y, nd.box_real_dim_z = rd
    nd.grid_intr_size = intr.size
    nd.ptr_intr_box_grid_idx = intr.ctypes.data_as(C.POINTER(C.c_int))
    nd.ptr_d = d.ctypes.data_as(C.POINTER(C.c_double))
    nd.ptr_pot = pot.ctypes.data_as(C.POINTER(C.c_double))
    nd.ptr_pot_old = pot_old.ctypes.data_as(C.POINTER(C.c_double))
    nd.grid_properties_cap = sx * sy * sz
    nd.node_mass = mass
    nd.cell_size = cells
    lib.conjugate_gradient.argtypes = [C.POINTER(Node)]
    lib.conjugate_gradient.restype = C.c_int
    rc = lib.conjugate_gradient(C.byref(nd))
    out.update(rc=np.array([rc]), mass=np.array([mass]), cells=np.array([cells]),
               pot_out=pot, pot_old_out=pot_old)
    np.savez_compressed(os.path.join(HERE, "node_cg.npz"), **out)
    print("wrote node_cg.npz", rc, intr.size)


def main() -> None:
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    want = set(sys.argv[1:])
    ic = ics.plummer(1000, a=0.05, seed=11)
    dt = 1e-3 * ics.crossing_time(0.05)
    cases = [
        ("head_L4_plummer1000.npz", dict(steps=3, lmin=4)),
        ("head_L3_jacobi.npz", dict(steps=2, lmin=3, solver=1)),
        ("head_L4_stencil5.npz", dict(steps=3, lmin=4, stencil=1)),
        ("head_L4_cgsmooth.npz", dict(steps=2, lmin=4, solver=2)),
        ("head_L4_cghead.npz", dict(steps=3, lmin=4, cg_head=1)),
    ]
    for name, kw in cases:
        if not want or name in want:
            run_case(name, ic, dt=dt, **kw)
    eic = edge_ic(ic)
    for name, kw in (("head_L4_periodic.npz", dict(steps=3, lmin=4, bdry=0)),
                     ("head_L4_periodic5.npz", dict(steps=3, lmin=4, bdry=0, stencil=1)),
                     ("head_L4_outflow.npz", dict(steps=3, lmin=4, bdry=2))):
        if not want or name in want:
            run_case(name, eic, dt=dt, **kw)
    if not want or "timestep_head_L4.npz" in want:
        timestep_case(ic, dt)
    if not want or "arrays.npz" in want:
        arrays_case()
    if not want or "node_cg.npz" in want:
        node_cg_case()


if __name__ == "__main__":
    main()

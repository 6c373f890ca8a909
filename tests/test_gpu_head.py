"""GPU parity of the head-node path through the C ABI (libqzb200.so).

Bit-exact where the arithmetic order is the reference's (lexicographic
Gauss-Seidel by wavefronts, Jacobi, multigrid cycles in that mode, boundary
values, gradient, gather, kick-drift, box index); within stated tolerances
where the order differs by design (deposit sums cell by cell; red-black
smoothing converges to the same discrete solution along a different path).

Tolerances (relative to the field's max magnitude unless stated):
  density            1e-13        potential (lex)   1e-12   potential (RB)  1e-9
  accelerations (RB) 1e-8         positions (RB)    1e-9 box units after 10 steps,
                                                     1e-6 after 100 steps
  mixed precision    force 1e-5 vs the FP64 oracle
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from quantizer_b200 import core, ics

pytestmark = pytest.mark.gpu

PT = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _ic(g):
    return {k: g["ic_" + k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}


def _rel(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


# ---- array-level kernels against the reference's own outputs --------------------
def test_gauss_seidel_lex_bit_exact(arrays_golden):
    g = arrays_golden
    for n in (9, 17):
        out = core.gauss_saidel(g[f"gs_n{n}_in_phi"], g[f"gs_n{n}_in_rho"],
                                int(g[f"gs_n{n}_iters"][0]), 1.0, core.QZ_GS_LEX)
        np.testing.assert_array_equal(out, g[f"gs_n{n}_out"])


def test_jacobi_bit_exact(arrays_golden):
    g = arrays_golden
    for n in (9, 17):
        out = core.jacobi(g[f"jac_n{n}_in_phi"], g[f"jac_n{n}_in_rho"],
                          int(g[f"jac_n{n}_iters"][0]), 1.0)
        np.testing.assert_array_equal(out, g[f"jac_n{n}_out"])


def test_multigrid_cycles_lex_bit_exact(arrays_golden):
    g = arrays_golden
    for key in [k for k in g if k.startswith("mg_") and k.endswith("_out")]:
        t = int(key.split("_")[2][1:])
        out = core.multigrid(g[key.replace("_out", "_in_phi")], g[key.replace("_out", "_in_rho")],
                             cycle=t, gs_order=core.QZ_GS_LEX)
        np.testing.assert_array_equal(out, g[key], err_msg=key)


def test_redblack_reaches_the_same_discrete_solution():
    n = 17
    rng = np.random.default_rng(5)
    rho = rng.standard_normal(n ** 3)
    phi0 = np.zeros(n ** 3)
    rb = phi0
    lx = phi0.copy()
    lib = O.load()
    for _ in range(40):
        rb = core.multigrid(rb, rho, cycle=0)
        lib.qzo_multigrid(C.byref(O.params(2)), O.ptr(lx), O.ptr(rho), n, 0)
    assert _rel(rb, lx) < 1e-12


def test_box_index_bit_exact(head_golden):
    L, B = 4, 18
    for step in (0, int(head_golden["meta"][1])):
        x, y, z = (head_golden[f"s{step}_{c}"] for c in "xyz")
        out = core.ptcl_idx_to_box_idx(L, (-1, -1, -1), (B, B), x, y, z)
        np.testing.assert_array_equal(out, head_golden[f"s{step}_bidx"])
    # negative coordinates take the reference's -1 floor
    out = core.ptcl_idx_to_box_idx(3, (2, 3, 4), (10, 11), [-0.01, 0.5], [0.4, 0.9999], [0.99, 0.0])
    lib = O.load()
    ref = np.empty(2, dtype=np.int32)
    xs = [np.array(v) for v in ([-0.01, 0.5], [0.4, 0.9999], [0.99, 0.0])]
    lib.qzo_box_idx_batch(3, 2, 3, 4, 10, 11, 2, *[O.ptr(a) for a in xs], O.ptr(ref))
    np.testing.assert_array_equal(out, ref)


# ---- per-stage parity on the head node -------------------------------------------
def test_initial_boundary_bit_exact(head_golden):
    ic = _ic(head_golden)
    M = core.sequential_mass(ic["m"])
    p = O.params(4, total_mass=M)
    g = O.grid_points(4)
    ref = {k: np.zeros(g) for k in ("pot", "ax", "ay", "az")}
    O.load().qzo_initial_head(C.byref(p), *[O.ptr(ref[k]) for k in ("pot", "ax", "ay", "az")])
    with core.Simulation(ic, 4) as sim:
        for k in ("pot", "ax", "ay", "az"):
            np.testing.assert_array_equal(sim.field(k), ref[k], err_msg=k)


def test_deposit_density(head_golden):
    ic = _ic(head_golden)
    with core.Simulation(ic, 4) as sim:
        sim.reset()
        sim.grid_density()
        d = sim.field("d")
    ref = head_golden["s0_d"]
    assert _rel(d, ref) < 1e-13
    # mass conservation: sum(d) H^3 / (4 pi G) = M
    H = 1.0 / 16
    assert abs(d.sum() * H ** 3 / (4 * np.pi) - ic["m"].sum()) < 1e-12


def test_deposit_is_deterministic():
    ic = ics.plummer(20000, a=0.05, seed=3)
    outs = []
    for _ in range(2):
        with core.Simulation(ic, 5) as sim:
            sim.reset()
            sim.grid_density()
            outs.append(sim.field("d"))
    np.testing.assert_array_equal(outs[0], outs[1])


def test_gradient_gather_kick_bit_exact(head_golden):
    g = head_golden
    ic = {k: g["s0_" + k] if k != "m" else g["ic_m"] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    M = core.sequential_mass(g["ic_m"])
    with core.Simulation(ic, 4, total_mass=M) as sim:
        sim.set_field("pot", g["s0_pot"])
        sim.grid_acceleration()
        for k in ("ax", "ay", "az"):
            np.testing.assert_array_equal(sim.field(k), g["s0_g" + k], err_msg=k)
        sim.reset()
        sim.particle_acceleration()
        p = sim.particles()
        for k in ("ax", "ay", "az"):
            np.testing.assert_array_equal(p[k], g["s0_" + k], err_msg=k)
        dt = float(g["meta"][2])
        sim.particle_updating_A(dt)
        p = sim.particles()
    ref = {k: np.ascontiguousarray(g["s0_" + k]).copy() for k in PT}
    O.load().qzo_update_A_head(C.byref(O.params(4)), ref["x"].size, dt,
                               *[O.ptr(ref[k]) for k in PT])
    for k in PT:
        np.testing.assert_array_equal(p[k], ref[k], err_msg=k)


def test_reflection_at_the_walls():
    n = 4
    ic = {"x": np.array([0.999, 0.001, 0.5, 0.5]), "y": np.full(n, 0.5), "z": np.full(n, 0.5),
          "vx": np.array([10.0, -10.0, 0.0, 0.0]), "vy": np.zeros(n),
          "vz": np.array([0.0, 0.0, 10.0, -10.0]), "m": np.full(n, 0.25)}
    with core.Simulation(ic, 3) as sim:
        sim.particle_updating_A(1e-3)
        p = sim.particles()
    ref = {k: np.ascontiguousarray(ic.get(k, np.zeros(n)), dtype=np.float64).copy() for k in PT}
    O.load().qzo_update_A_head(C.byref(O.params(3)), n, 1e-3, *[O.ptr(ref[k]) for k in PT])
    for k in PT:
        np.testing.assert_array_equal(p[k], ref[k], err_msg=k)
    assert p["vx"][0] < 0 and p["vx"][1] > 0


# ---- whole steps ------------------------------------------------------------------
def _gpu_run(ic, L, steps, dt, **cfg):
    with core.Simulation(ic, L, **cfg) as sim:
        sim.init_forces()
        s0 = {k: sim.field(k) for k in ("pot", "d", "ax")}
        sim.step(dt, steps)
        return s0, {k: sim.field(k) for k in ("pot", "d", "ax")}, sim.particles(), sim.stats()


def test_pipeline_lex_against_reference(head_golden):
    g = head_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    f0, f1, p, st = _gpu_run(_ic(g), 4, steps, dt, gs_order=core.QZ_GS_LEX)
    assert _rel(f0["pot"], g["s0_pot"]) < 1e-12
    assert _rel(f1["pot"], g[f"s{steps}_pot"]) < 1e-12
    assert _rel(f1["d"], g[f"s{steps}_d"]) < 1e-12
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-13
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-11


def test_pipeline_redblack_against_reference(head_golden):
    g = head_golden
    steps, dt = int(g["meta"][1]), float(g["meta"][2])
    f0, f1, p, st = _gpu_run(_ic(g), 4, steps, dt)
    assert _rel(f0["pot"], g["s0_pot"]) < 1e-9
    assert _rel(f1["pot"], g[f"s{steps}_pot"]) < 1e-9
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], g[f"s{steps}_{k}"]) < 1e-8
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - g[f"s{steps}_{k}"]).max() < 1e-9
    assert st.last_converged == 1


@pytest.mark.parametrize("steps,pos_tol", [(10, 1e-9), (100, 1e-6)])
def test_plummer_10k_head32_against_oracle(steps, pos_tol):
    ic = ics.plummer(10000, a=0.05, seed=1)
    dt = 1e-3 * ics.crossing_time(0.05)
    M = core.sequential_mass(ic["m"])
    ref = O.OracleSim(ic, O.params(5, total_mass=M))
    for _ in range(steps):
        ref.step(dt)
    rp, rf = ref.particles(), ref.fields()
    ref.close()
    f0, f1, p, st = _gpu_run(ic, 5, steps, dt)
    assert _rel(f1["d"], rf["d"]) < 1e-9
    assert _rel(f1["pot"], rf["pot"]) < 1e-8
    for k in ("x", "y", "z"):
        assert np.abs(p[k] - rp[k]).max() < pos_tol
    for k in ("ax", "ay", "az"):
        assert _rel(p[k], rp[k]) < 1e-6


def test_mixed_precision_force_error():
    ic = ics.plummer(10000, a=0.05, seed=1)
    dt = 1e-3 * ics.crossing_time(0.05)
    M = core.sequential_mass(ic["m"])
    ref = O.OracleSim(ic, O.params(5, total_mass=M))
    for _ in range(5):
        ref.step(dt)
    rp = ref.particles()
    ref.close()
    _, _, p, st = _gpu_run(ic, 5, 5, dt, precision=core.QZ_PREC_MIXED)
    amag = np.sqrt(rp["ax"] ** 2 + rp["ay"] ** 2 + rp["az"] ** 2)
    err = np.sqrt((p["ax"] - rp["ax"]) ** 2 + (p["ay"] - rp["ay"]) ** 2 + (p["az"] - rp["az"]) ** 2)
    assert (err / amag).max() < 1e-5
    assert st.last_converged == 1


def test_particle_outside_the_box_is_an_error():
    ic = ics.plummer(100, a=0.05, seed=2)
    ic["x"] = ic["x"].copy()
    ic["x"][7] = 3.5  # far outside: the reference would index out of its arrays
    with core.Simulation(ic, 3) as sim:
        with pytest.raises(core.QZError, match="bounds"):
            sim.init_forces()

"""Pins the CPU oracle (oracle/qz_oracle.c) against fixtures dumped by the
compiled reference: every comparison here is bit-exact."""
import numpy as np

from oracle import oracle as O

PT = ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")


def _ic(g):
    return {k: g["ic_" + k] for k in ("x", "y", "z", "vx", "vy", "vz", "m")}


def _run(g, L, **kw):
    ic = _ic(g)
    p = O.params(L, total_mass=float(np.cumsum(ic["m"])[-1]), **kw)
    steps = int(g["meta"][1])
    dt = float(g["meta"][2])
    s = O.OracleSim(ic, p)
    f0, p0 = s.fields(), s.particles()
    for _ in range(steps):
        s.step(dt)
    f1, p1 = s.fields(), s.particles()
    s.close()
    return steps, (f0, p0), (f1, p1)


def _assert_exact(g, steps, s0, s1):
    for step, (f, p) in ((0, s0), (steps, s1)):
        for k in ("pot", "d", "gax", "gay", "gaz"):
            np.testing.assert_array_equal(f[k], g[f"s{step}_{k}"], err_msg=f"step {step} {k}")
        for k in PT:
            np.testing.assert_array_equal(p[k], g[f"s{step}_{k}"], err_msg=f"step {step} {k}")


def test_head_pipeline_bit_exact(head_golden):
    steps, s0, s1 = _run(head_golden, 4)
    _assert_exact(head_golden, steps, s0, s1)


def test_head_pipeline_jacobi_bit_exact(jacobi_golden):
    steps, s0, s1 = _run(jacobi_golden, 3, solver=1)
    _assert_exact(jacobi_golden, steps, s0, s1)


def test_head_pipeline_five_point_stencil_bit_exact(stencil5_golden):
    steps, s0, s1 = _run(stencil5_golden, 4, force_stencil=1)
    _assert_exact(stencil5_golden, steps, s0, s1)


def test_head_pipeline_cg_smoothing_bit_exact(cgsmooth_golden):
    steps, s0, s1 = _run(cgsmooth_golden, 4, solver=2)
    _assert_exact(cgsmooth_golden, steps, s0, s1)


def test_head_pipeline_cg_head_bit_exact(cghead_golden):
    steps, s0, s1 = _run(cghead_golden, 4, head_pot_method=1)
    _assert_exact(cghead_golden, steps, s0, s1)


def test_cg_smoother_bit_exact(arrays_golden):
    g = arrays_golden
    lib = O.load()
    for n in (9, 17):
        phi, rho = g[f"cgs_n{n}_in_phi"].copy(), g[f"cgs_n{n}_in_rho"].copy()
        lib.qzo_cg_smooth(O.ptr(phi), O.ptr(rho), n, int(g[f"cgs_n{n}_iters"][0]))
        np.testing.assert_array_equal(phi, g[f"cgs_n{n}_out"])


def test_timestep_head_bit_exact(head_golden, timestep_golden):
    lib = O.load()
    g, t = head_golden, timestep_golden
    for m in (0, 1):
        for s in (0, 3):
            arr = [np.ascontiguousarray(g[f"s{s}_{k}"]) for k in ("vx", "vy", "vz", "ax", "ay", "az")]
            dt = lib.qzo_timestep_head(4, m, float(t["cfl"][0]), float(t["max_dt"][0]),
                                       arr[0].size, *[O.ptr(a) for a in arr])
            assert dt == float(t[f"m{m}_s{s}_dt"][0]), (m, s, dt)


def test_box_index_bit_exact(head_golden):
    lib = O.load()
    L = 4
    B = (1 << L) + 2
    for step in (0, int(head_golden["meta"][1])):
        x, y, z = (np.ascontiguousarray(head_golden[f"s{step}_{c}"]) for c in "xyz")
        out = np.empty(x.size, dtype=np.int32)
        lib.qzo_box_idx_batch(L, -1, -1, -1, B, B, x.size, O.ptr(x), O.ptr(y), O.ptr(z), O.ptr(out))
        np.testing.assert_array_equal(out, head_golden[f"s{step}_bidx"])


def test_array_kernels_bit_exact(arrays_golden):
    g = arrays_golden
    lib = O.load()
    for n in (9, 17):
        phi, rho = g[f"gs_n{n}_in_phi"].copy(), g[f"gs_n{n}_in_rho"].copy()
        lib.qzo_gauss_saidel(O.ptr(phi), O.ptr(rho), n, int(g[f"gs_n{n}_iters"][0]), 1.0)
        np.testing.assert_array_equal(phi, g[f"gs_n{n}_out"])
        phi, rho = g[f"jac_n{n}_in_phi"].copy(), g[f"jac_n{n}_in_rho"].copy()
        lib.qzo_jacobi(O.ptr(phi), O.ptr(rho), n, int(g[f"jac_n{n}_iters"][0]), 1.0)
        np.testing.assert_array_equal(phi, g[f"jac_n{n}_out"])
    p = O.params(2)
    import ctypes as C
    for key in [k for k in g if k.startswith("mg_") and k.endswith("_out")]:
        n = int(key.split("_")[1][1:])
        t = int(key.split("_")[2][1:])
        phi = g[key.replace("_out", "_in_phi")].copy()
        rho = g[key.replace("_out", "_in_rho")].copy()
        lib.qzo_multigrid(C.byref(p), O.ptr(phi), O.ptr(rho), n, t)
        np.testing.assert_array_equal(phi, g[key], err_msg=key)


def test_head_pipeline_periodic_bit_exact(periodic_golden):
    steps, s0, s1 = _run(periodic_golden, 4, bdry=0)
    _assert_exact(periodic_golden, steps, s0, s1)


def test_head_pipeline_periodic_five_point_bit_exact(periodic5_golden):
    steps, s0, s1 = _run(periodic5_golden, 4, bdry=0, force_stencil=1)
    _assert_exact(periodic5_golden, steps, s0, s1)


def test_head_pipeline_outflow_bit_exact(outflow_golden):
    g = outflow_golden
    steps, s0, s1 = _run(g, 4, bdry=2)
    assert s1[1]["x"].size == g[f"s{steps}_x"].size < s0[1]["x"].size
    _assert_exact(g, steps, s0, s1)

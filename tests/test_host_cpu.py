"""Host-side checks that need no GPU: the C-ABI libraries load and export every
symbol their headers declare, the configuration defaults are the reference's,
the library refuses to run without a CUDA device (no CPU fallback), and the
synthetic initial conditions have the stated properties."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from quantizer_b200 import build, core, ics

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header: str) -> list[str]:
    text = open(os.path.join(ROOT, "include", header)).read()
    return sorted(set(re.findall(r"^QZ_\w*API\s+[\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M)))


def _exports(lib: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", lib], check=True, capture_output=True,
                         text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


@pytest.fixture(scope="module")
def built():
    build.build_all()
    return os.path.join(build.LIBDIR, "libqzb200.so"), os.path.join(build.LIBDIR, "libqz_dropin.so")


def test_core_library_loads_and_exports_its_header(built):
    names = _declared("qz_b200.h")
    assert len(names) >= 25
    lib = core.load()
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= _exports(built[0])


def test_dropin_library_exports_the_reference_entry_points(built):
    names = _declared("qz_dropin.h")
    for must in ("grid_density", "potential", "potential_head_node", "potential_branches",
                 "grid_acceleration", "particle_acceleration", "particle_updating_A",
                 "particle_updating_B", "ptcl_idx_to_box_idx", "reset", "multigrid",
                 "gauss_saidel", "jacobi", "poisson_error"):
        assert must in names, must
    assert set(names) <= _exports(built[1])
    # it loads without a host program: the reference's globals are looked up lazily
    lib = C.CDLL(built[1])
    assert hasattr(lib, "grid_density")


def test_default_config_matches_reference_defaults():
    c = core.config(5)
    # global_variables.c:300-341
    assert (c.n_pre, c.n_post, c.n_coarse, c.check_every, c.max_iter) == (2, 2, 2, 5, 5000)
    assert (c.tol, c.tol2, c.w_sor, c.bdry, c.cycle, c.smoother) == (1e-10, 1e-10, 1.0, 1, 0, 0)


def test_default_config_schedule_options():
    # the last fields of qz_config, as the library fills them: a misaligned
    # ctypes mirror would read other fields' bytes here
    c = core.config(7)
    assert (c.node_warm, c.tree_overlap, c.cg_chunk_min) == (0, 1, 0)
    assert (c.mg_points_per_thread, c.mg_tile, c.freeze_tree) == (4, 0, 0)
    c2 = core.config(7, tree_overlap=0, cg_chunk_min=2048)
    assert (c2.tree_overlap, c2.cg_chunk_min) == (0, 2048)


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    ic = ics.plummer(10, seed=0)
    with pytest.raises(core.QZError, match="CUDA device"):
        core.Simulation(ic, 3)
    with pytest.raises(core.QZError, match="CUDA device"):
        core.gauss_saidel(np.zeros(27), np.zeros(27), 1)


def test_plummer_sampler():
    a = ics.plummer(20000, a=0.05, seed=4)
    b = ics.plummer(20000, a=0.05, seed=4)
    for k in ics.FIELDS:
        np.testing.assert_array_equal(a[k], b[k])
    r = np.sqrt((a["x"] - 0.5) ** 2 + (a["y"] - 0.5) ** 2 + (a["z"] - 0.5) ** 2)
    assert r.max() <= 0.45
    assert abs(a["m"].sum() - 1.0) < 1e-12
    # half-mass radius of a Plummer sphere: a / sqrt(2^(2/3) - 1) ~ 1.305 a
    assert abs(np.median(r) / 0.05 - 1.305) < 0.05
    # bound: every speed below the local escape speed
    v2 = a["vx"] ** 2 + a["vy"] ** 2 + a["vz"] ** 2
    assert np.all(v2 < 2.0 / np.sqrt(r ** 2 + 0.05 ** 2))


def test_hernquist_sampler():
    h = ics.hernquist(20000, a=0.03, seed=5, rmax=0.14, center=(0.35, 0.5, 0.5))
    r = np.sqrt((h["x"] - 0.35) ** 2 + (h["y"] - 0.5) ** 2 + (h["z"] - 0.5) ** 2)
    assert r.max() <= 0.14 and h["x"].min() > 0.0
    assert abs(h["m"].sum() - 1.0) < 1e-12


def test_ic_file_round_trip(tmp_path):
    a = ics.plummer(100, seed=1)
    p = tmp_path / "ic.bin"
    ics.write_ic(str(p), a)
    b = ics.read_ic(str(p))
    for k in ics.FIELDS:
        np.testing.assert_array_equal(a[k], b[k])


def test_crossing_time():
    # a = 0.05: R_v = 0.0849, t_cr = 2 sqrt(2) R_v^1.5 ~ 0.06995
    assert abs(ics.crossing_time(0.05) - 0.069948) < 1e-5

"""The fused red-black sweep (k_gs_rb_zm: one launch per sweep, z-marching
tiles staged in shared memory by asynchronous copies, ping-pong between two
grids) against the two launches per sweep of k_gs_rb (red, then black): the
same arithmetic on the same values, so the results must be equal bit for bit,
for grids whose interior does not divide into whole tiles (x 64, y 16, z 32),
for an odd sweep count (the result copied back from the partner grid) and for
an over-relaxation weight.  QZ_FUSED_RB selects the fused sweep; the array
entry point reads it at every call.
"""
import os

import numpy as np
import pytest

from quantizer_b200 import core

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,iters,w", [(67, 2, 1.0), (131, 3, 1.0), (100, 2, 1.3), (257, 2, 1.0)])
def test_fused_sweep_equals_two_colour_launches(n, iters, w, monkeypatch):
    rng = np.random.default_rng(n)
    phi = rng.standard_normal(n ** 3)
    rho = rng.standard_normal(n ** 3) * 50.0
    monkeypatch.delenv("QZ_FUSED_RB", raising=False)
    plain = core.gauss_saidel(phi, rho, iters, w)
    monkeypatch.setenv("QZ_FUSED_RB", "1")
    fused = core.gauss_saidel(phi, rho, iters, w)
    assert not np.array_equal(plain, phi)
    np.testing.assert_array_equal(fused, plain)

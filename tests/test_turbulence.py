"""Turbulence extrusion set-up against the reference's iterkolmo output (CPU)."""

import numpy as np
import pytest

from aob200 import turbulence as T
from oracle import turbulence as OT


@pytest.mark.parametrize("name", ["kolmo32", "kolmo64neg"])
def test_structure_function_and_stencils(name, golden):
    ref = golden(name)
    L0 = float(ref["struct_L0"])
    got = T.structure_function(np.sqrt(ref["struct_r2"]), L0)
    np.testing.assert_allclose(got, ref["struct_val"], rtol=2e-6, atol=1e-9)
    n = ref["A"].shape[0]
    assert T.stencil_size(n) == int(ref["stencil_size"])


@pytest.mark.parametrize("name,dx,dy", [("kolmo32", 0.5, 0.3), ("kolmo64neg", -0.7, -0.2)])
def test_extrusion_operators_match_reference(name, dx, dy, golden):
    ref = golden(name)
    n = ref["A"].shape[0]
    zz, xz, xx, ist = T.covariances(n, float(ref["struct_L0"]))
    A, B = OT.factor_AB(zz, xz, xx)
    # stencil indexes are integer maps: exact
    istx = ist.astype(np.uint32)
    if dx < 0:
        istx = (n * n - 1) - istx
    np.testing.assert_array_equal(istx, ref["istencilx"])
    # A is unique; B is defined up to column signs, compare B B^T
    np.testing.assert_allclose(A, ref["A"], rtol=1e-3, atol=2e-4 * np.abs(ref["A"]).max())
    bbt, rbbt = B @ B.T, ref["B"].astype(np.float64) @ ref["B"].astype(np.float64).T
    assert np.abs(bbt - rbbt).max() < 2e-3 * np.abs(rbbt).max()


def test_extrude_keeps_structure_statistics():
    """Screens grown by the oracle extrusion have the von Karman structure function."""
    n = 32
    L0 = 1e4
    zz, xz, xx, ist = T.covariances(n, L0)
    A, B = OT.factor_AB(zz, xz, xx)
    rng = np.random.default_rng(0)
    scr = np.zeros((n, n))
    d1 = []
    for it in range(3000):
        scr = OT.extrude(scr, A, B, ist, ist, 1.0, rng.standard_normal(n), 1)
        if it > 2 * n:
            d1.append(np.mean((scr[1:, :] - scr[:-1, :]) ** 2))
    # D(1 pixel) for r0 = 1 pixel is 6.88 rad^2 (Kolmogorov, L0 >> n)
    assert abs(np.mean(d1) / 6.88 - 1) < 0.15

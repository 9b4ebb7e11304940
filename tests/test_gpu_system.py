"""Closed-loop behaviour on the GPU: calibration, loop closure and Strehl."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def plain16():
    from aob200 import _lib, system

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    sysm = system.ShAoSystem(system.plain16())
    sysm.calibrate()
    return sysm


def test_interaction_matrix_is_sane(plain16):
    s = plain16
    imat = s.imat
    assert imat.shape == (2 * s.geom.nvalid, s.nactu)
    # actuators inside the pupil produce slopes; the LS inverse reproduces a poke
    resp = np.linalg.norm(imat, axis=0)
    assert np.sum(resp > 0.1 * resp.max()) > 0.7 * s.nactu
    cm = s.cmat
    rec = cm @ imat
    inner = resp > 0.5 * resp.max()
    d = np.diag(rec)[inner]
    assert np.median(d) > 0.9


def test_batched_interaction_matrix_equals_poke_by_poke():
    """aob_imat_build (all actuators in one batch, one sensor launch) gives the
    matrix of poking one actuator after the other through the separate calls,
    bit for bit, also in chunks."""
    from aob200 import system

    s = system.ShAoSystem(system.plain16())
    seq = s.calibrate(batched=False).copy()
    s2 = system.ShAoSystem(system.plain16())
    bat = s2.interaction_matrix()
    np.testing.assert_array_equal(bat, seq)
    np.testing.assert_array_equal(s2.interaction_matrix(chunk=37), seq)
    assert np.abs(seq).max() > 0


def test_closed_loop_raises_strehl(plain16):
    s = plain16
    s.target.reset_le()
    for _ in range(20):
        s.atmos.move()
        s.trace_target()
        s.target.comp_image(None, True)
    _, le_open = s.strehl()
    s.close(graph=True)
    s.target.reset_le()
    for it in range(150):
        s.next(compute_psf=it >= 50)
    se, le = s.strehl()
    assert le > 0.3, (le, le_open)
    assert le > 5 * le_open
    assert s.ls.status() == 0

"""Failure detection without a GPU fault: the bounded waits run out and report.

Every spin-wait in the library's kernels has an iteration limit; on expiry the
kernel sets a bit of a status word, skips the work that needed the wait and
returns, so the context stays usable.  Here the wait is made to run out on
purpose with a condition that nothing satisfies (a CTA that never arrives at
the fused kernel's grid barrier; MVM items that wait for one sensor item more
than their instance has), with a short poll limit, and the tests check the
status bit, that the step returns, and that the next steps are correct again.
"""

import numpy as np
import pytest

from helpers import kolmogorov_screen, sh_geometry

pytestmark = pytest.mark.gpu

GRID_TIMEOUT = 2  # aob_ls_status bit of the fused kernel's grid barrier
DEP_TIMEOUT = 4   # aob_batch_status bit of an MVM item's dependency wait


@pytest.fixture(scope="module")
def core():
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return C


def _sh16_loop(core, cm):
    g = sh_geometry("sh16")
    w = core.ShWfs.from_geometry(g, noise=-1.0, seed=5)
    c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "cog")
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    ls = core.LsController(2 * g.nvalid, cm.shape[0], delay=0.0)
    ls.set_cmat(cm)
    ls.set_gain(0.3)
    return g, w, c, ls


def test_fused_grid_wait_expires_reports_and_recovers(core):
    from aob200 import _lib

    rng = np.random.default_rng(3)
    g = sh_geometry("sh16")
    cm = (rng.standard_normal((97, 2 * g.nvalid)) * 0.01).astype(np.float32)
    _, w1, c1, l1 = _sh16_loop(core, cm)
    loop1 = core.Loop(w1, c1, l1, graph=False)
    loop1.set_mode(2, 0)
    _, w2, c2, l2 = _sh16_loop(core, cm)
    loop2 = core.Loop(w2, c2, l2, graph=False)
    loop2.set_mode(2, 0)
    screens = [np.ascontiguousarray(kolmogorov_screen(g.tel.n, 20.0, seed=s).ravel(order="F")) for s in range(3)]
    v1 = np.zeros(97, np.float32)
    v2 = np.zeros(97, np.float32)

    loop1.step(screens[0], v1, noise=False)
    loop2.step(screens[0], v2, noise=False)
    assert l1.status() == 0
    com_before = np.array(l1.buffer("com"))
    _lib.call("aob_loop_test_wait_expiry", loop1.h, 4096, None)
    assert l1.status() & GRID_TIMEOUT
    # every CTA skipped the MVM: the integrator did not move
    np.testing.assert_array_equal(np.array(l1.buffer("com")), com_before)
    l1.status(reset=True)
    assert l1.status() == 0
    # the barrier is re-armed: the next steps equal a loop that never timed out
    for ph in screens[1:]:
        loop1.step(ph, v1, noise=False)
        loop2.step(ph, v2, noise=False)
        np.testing.assert_array_equal(v1, v2)
        np.testing.assert_array_equal(np.array(l1.buffer("com")), np.array(l2.buffer("com")))
    assert l1.status() == 0 and l2.status() == 0


def test_batch_dependency_wait_expires_reports_and_recovers(core):
    from aob200 import _lib
    from aob200 import workloads as W

    insts = [W.mc_make(24, 6, 0.12, 1), W.mc_make(26, 8, 0.15, 2)]
    loops, batch = W.build_mc_batch(insts, precision="bf16", graph=False)
    batch.step(True)
    assert batch.status() == 0
    _lib.call("aob_batch_test_wait_expiry", batch.h, 2048, 1, None)
    assert batch.status() & DEP_TIMEOUT
    batch.refresh()  # a rebuild clears the status word
    batch.step(True)
    assert batch.status() == 0
    for _, _, ls, _ in loops:
        assert np.all(np.isfinite(np.array(ls.buffer("com"))))

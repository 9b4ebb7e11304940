"""The learned reconstructor's RTC iteration in one kernel against separate launches.

At the saxo40 geometry (40 x 40 SH, photon + readout noise, wCoG with a
threshold) a network of the c4 shape (2496 -> 1024 -> 1024 -> 1377 + the linear
skip initialised to the LS matrix) drives two loops fed the same phases: one
runs aob_loop_step_mlp's single cooperative kernel (rtc_mlp_kernel), the other
the separate launches (sensor image with fused centroids, the fused control
step, the voltage kernel).  Slopes, errors, commands and voltages must be equal
bit for bit at every step, on the network path and on the LS fallback (a zero
threshold), with and without a one-frame delay.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    from aob200 import _lib
    from aob200 import mlp as M
    from aob200.workloads import sh_loop_setup, von_karman_screens

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    setup = sh_loop_setup("saxo40")
    g = setup.geom
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 4, seed=13)
    phases = [np.ascontiguousarray(s.ravel(order="F"), dtype=np.float32) for s in screens]
    net = M.MlpReconstructor(setup.nslope, setup.nactu, 1024, 1024, seed=3)
    net.init_from_ls(setup.cmat, 10.0, 1.0)
    return setup, phases, net


@pytest.mark.parametrize("threshold", [3e38, 0.0])  # the network's commands; the LS fallback
@pytest.mark.parametrize("delay", [0.0, 1.0])
def test_fused_learned_step_equals_separate_launches(env, threshold, delay):
    from aob200.workloads import build_sh_loop

    setup, phases, net = env
    loops = []
    for mode in (0, 1):  # 0: the fused kernel when it fits, 1: separate launches
        wfs, c, ls, loop = build_sh_loop(setup, graph=False)
        ls.set_delay(delay)
        loop.set_mode(mode)
        loops.append((ls, loop))
    for i in range(5):
        out = []
        for ls, loop in loops:
            v = np.zeros(setup.nactu, np.float32)
            loop.step_mlp(net, threshold, phases[i % 4], v, noise=True)
            out.append([v] + [np.array(ls.buffer(b)) for b in ("com", "err", "centroids")])
        assert loops[0][1].kernels_per_step() == 1, "the fused learned iteration did not run"
        assert loops[1][1].kernels_per_step() > 1
        for a, b, name in zip(out[0], out[1], ("voltages", "com", "err", "centroids")):
            np.testing.assert_array_equal(a, b, err_msg=f"step {i}: {name}")
    assert np.abs(out[0][0]).max() > 0
    for ls, _ in loops:
        assert ls.status() == 0

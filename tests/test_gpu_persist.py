"""The persistent RTC kernel (aob_loop_persist_*) against launched steps.

The saxo40 loop (rtc_fused_kernel<float, 32, 6>, photon + readout noise,
wCoG with threshold, LS integrator) is stepped from host phases twice: once
with one kernel launch per step (aob_loop_step), once with the kernel resident
and rung once per step, with the resident kernel's buffer-clearing command
(the benchmark's L2 flush) between some steps.  Voltages must be equal bit for
bit at every step, with the kernel writing them into pinned host memory or
with a copy.  A doorbell
that never rings makes the resident kernel's bounded wait run out: it leaves,
sets bit 16 of the controller's status and the context stays usable.
"""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NSTEPS = 12


@pytest.fixture(scope="module")
def env():
    import torch

    from aob200 import _lib
    from aob200.workloads import sh_loop_setup, von_karman_screens

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    setup = sh_loop_setup("saxo40")
    g = setup.geom
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 4, seed=21)
    phases = torch.from_numpy(np.ascontiguousarray(np.stack([s.ravel(order="F") for s in screens]))).pin_memory()
    return torch, setup, phases


def _launched(setup, phases, torch):
    from aob200.workloads import build_sh_loop

    wfs, c, ls, loop = build_sh_loop(setup, graph=False)
    out = []
    v = np.zeros(setup.nactu, np.float32)
    for i in range(NSTEPS):
        loop.step(phases[i % 4].data_ptr(), v, noise=True)
        out.append(v.copy())
    return out


@pytest.mark.parametrize("direct", [True, False])
def test_persistent_steps_equal_launched_steps(env, direct):
    torch, setup, phases = env
    from aob200.workloads import build_sh_loop

    ref = _launched(setup, phases, torch)
    wfs, c, ls, loop = build_sh_loop(setup, graph=False)
    hv = torch.zeros(setup.nactu, dtype=torch.float32).pin_memory()
    scratch = torch.empty(8 * 1024 * 1024, dtype=torch.float32, device="cuda")
    loop.persist_start(noise=True, host_voltage=hv.data_ptr() if direct else None)
    try:
        v = np.zeros(setup.nactu, np.float32)
        for i in range(NSTEPS):
            if i % 2:  # the resident kernel's own flush between steps changes nothing
                loop.persist_flush(scratch.data_ptr(), scratch.numel() * 4)
            if direct:
                loop.persist_step(phases[i % 4].data_ptr(), hv.data_ptr(), noise=True, wait=True)
                got = hv.numpy().copy()
            else:
                loop.persist_step(phases[i % 4].data_ptr(), v, noise=True, wait=True)
                got = v.copy()
            np.testing.assert_array_equal(got, ref[i], err_msg=f"step {i}")
    finally:
        loop.persist_stop()
    assert ls.status() == 0
    assert wfs.frame == NSTEPS
    # launched steps continue from the persistent ones
    loop.step(phases[0].data_ptr(), np.zeros(setup.nactu, np.float32), noise=True)
    assert ls.status() == 0


def test_persistent_doorbell_wait_expires(env):
    torch, setup, phases = env
    from aob200.workloads import build_sh_loop

    wfs, c, ls, loop = build_sh_loop(setup, graph=False)
    loop.persist_start(noise=True, door_polls=2000)  # about half a millisecond
    time.sleep(0.2)  # nothing rings
    loop.persist_stop()
    assert ls.status(reset=True) & 16
    v = np.zeros(setup.nactu, np.float32)
    loop.step(phases[0].data_ptr(), v, noise=True)
    assert ls.status() == 0 and np.isfinite(v).all()

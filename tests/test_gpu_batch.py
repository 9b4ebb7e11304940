"""Batched Monte Carlo: many SH loops of uneven size advanced by one persistent
launch per step.

The batch runs every instance's sensor stages and MVM reduction in the same
order as the instance's own fused loop kernel, so slopes, images, commands
and voltages must be bit-identical to stepping each loop on its own, for any
tile shapes the autotuner may pick, with or without CUDA-graph replay and
through the host-I/O entry point.  The loops themselves are pinned to the CPU
oracle by test_gpu_core.py; one instance is also checked against the oracle
here directly (relative slope rms <= 1e-4, no noise).
"""

import numpy as np
import pytest

from helpers import rel_rms
from oracle import rtc as ortc
from oracle import sh as osh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def mods():
    from aob200 import _lib, core, workloads

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return core, workloads


# (instance, precision, centroider, readout noise) -- uneven sizes, both
# Nfft 16 and 32, 6x6 and 8x8 pixels, every precision and CoG kind
# (nxsub, npix, pixsize, phase pixels per sub-aperture): Nfft 16 and 32,
# 6 phase pixels (compiled sizes) and 5 or 8 (runtime sizes)
SMALL = [(12, 6, 0.2, 6), (16, 6, 0.2, 6), (14, 8, 0.2, 6), (16, 8, 0.25, 8), (16, 6, 0.2, 5), (22, 8, 0.36, 6)]


def _specs(W):
    insts = [W.mc_make(n, p, 0.08 + 0.02 * i, 40 + i, pixsize=ps, pd=pd) for i, (n, p, ps, pd) in enumerate(SMALL)]
    kinds = ["wcog", "cog", "tcog", "wcog", "tcog", "cog"]
    precs = ["bf16", "f32", "fp8", "bf16", "f32", "bf16"]
    noise = [0.5, -1.0, 0.5, 0.0, 0.5, 0.5]
    return [(insts[i], precs[i], kinds[i], noise[i]) for i in range(6)]


def _build(core, inst, prec, kind, noise, seed):
    s = inst.setup
    g = s.geom
    w = core.ShWfs.from_geometry(g, noise=noise, seed=seed)
    w.set_phase(inst.phase)
    c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, kind)
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    if kind in ("tcog", "wcog"):
        c.set_threshold(s.threshold)
    if kind == "wcog":
        c.load_weights(s.weights)
    ls = core.LsController(s.nslope, s.nactu, delay=0.0)
    ls.set_precision(prec)
    ls.set_cmat(s.cmat)
    ls.set_gain(0.4)
    ls.set_com_range(-2.0, 2.0)
    loop = core.Loop(w, c, ls, graph=False)
    return w, c, ls, loop


def _objects(core, specs):
    return [_build(core, inst, p, k, nz, seed=100 + i) for i, (inst, p, k, nz) in enumerate(specs)]


def _host_phases(specs):
    return np.concatenate([np.ascontiguousarray(s[0].phase.ravel(order="F")) for s in specs])


def _state(objs):
    return [
        (
            np.array(ls.buffer("centroids")),
            np.array(ls.buffer("com")),
            np.array(ls.buffer("voltage")),
            np.array(w.d_binimg),
            w.frame,
        )
        for (w, c, ls, loop) in objs
    ]


def _assert_same(a, b):
    for i, (x, y) in enumerate(zip(a, b)):
        for j, name in enumerate(("slopes", "com", "voltage", "image")):
            np.testing.assert_array_equal(x[j], y[j], err_msg=f"instance {i}: {name}")
        assert x[4] == y[4], f"instance {i}: frame"


def _reference_run(core, specs, steps):
    objs = _objects(core, specs)
    out = []
    for _ in range(steps):
        for (w, c, ls, loop) in objs:
            loop.set_mode(2)  # the fused single-kernel loop
            loop.step(None, None, noise=True)
        out.append(_state(objs))
    return out


def _batch_run(core, specs, steps, tuning=None, graph=True, host_io=False):
    objs = _objects(core, specs)
    b = core.Batch([o[3] for o in objs], graph=graph)
    if tuning:
        b.set_tuning(*tuning)
    out = []
    if host_io:
        phases = _host_phases(specs)
        info = b.info()
        volts = np.zeros(info["volt_floats"], np.float32)
    for _ in range(steps):
        if host_io:
            b.step_host(phases, volts, noise=True)
        else:
            b.step(noise=True)
        out.append(_state(objs))
    assert b.status() == 0
    if host_io:
        _, voff = b.offsets()
        for i, o in enumerate(objs):
            n = o[2].nactu
            np.testing.assert_array_equal(volts[voff[i]:voff[i] + n], out[-1][i][2])
    return out, b.info()


def test_batch_matches_each_loop(mods):
    core, W = mods
    specs = _specs(W)
    ref = _reference_run(core, specs, 3)
    got, info = _batch_run(core, specs, 3)
    assert info["instances"] == 6
    for r, g in zip(ref, got):
        _assert_same(g, r)


@pytest.mark.parametrize(
    "tuning",
    [(1, 256, 4, 0, 1, 1), (3, 64, 16, 1, 2, 0), (64, 128, 200, 5, 1, 0), (8, 32, 48, 2, 0, 1), (5, 0, 1, 0, 2, 1),
     (1024, 32, 40, 3, 4, 0), (7, 64, 24, 1, 3, 1)],
)
def test_batch_tile_shapes_do_not_change_results(mods, tuning):
    core, W = mods
    specs = _specs(W)
    ref, _ = _batch_run(core, specs, 2)
    got, info = _batch_run(core, specs, 2, tuning=tuning)
    for r, g in zip(ref, got):
        _assert_same(g, r)


def test_batch_graph_and_host_io(mods):
    core, W = mods
    specs = _specs(W)
    ref, _ = _batch_run(core, specs, 3, graph=False)
    got, _ = _batch_run(core, specs, 3, graph=True, host_io=True)
    for r, g in zip(ref, got):
        _assert_same(g, r)


def test_batch_single_instance_and_parameter_change(mods):
    """One instance; a gain change between steps rebuilds the snapshot."""
    core, W = mods
    specs = _specs(W)[:1]
    objs_a = _objects(core, specs)
    objs_b = _objects(core, specs)
    b = core.Batch([objs_b[0][3]])
    for it in range(4):
        if it == 2:
            objs_a[0][2].set_gain(0.2)
            objs_b[0][2].set_gain(0.2)
        objs_a[0][3].set_mode(2)
        objs_a[0][3].step(None, None, noise=True)
        b.step(noise=True)
        _assert_same(_state(objs_b), _state(objs_a))


def test_batch_interleaved_with_own_steps(mods):
    """A loop stepped on its own between batch steps keeps its frame sequence."""
    core, W = mods
    specs = _specs(W)[:2]
    objs_a = _objects(core, specs)
    objs_b = _objects(core, specs)
    b = core.Batch([o[3] for o in objs_b])
    for it in range(4):
        for o in objs_a:
            o[3].set_mode(2)
            o[3].step(None, None, noise=True)
        if it == 1:
            for o in objs_b:
                o[3].set_mode(2)
                o[3].step(None, None, noise=True)
        else:
            b.step(noise=True)
        _assert_same(_state(objs_b), _state(objs_a))


def test_batch_rejects_unsupported(mods):
    from aob200._lib import AobError

    core, W = mods
    specs = _specs(W)[:1]
    inst, p, k, nz = specs[0]
    w, c, ls, loop = _build(core, inst, p, k, nz, seed=1)
    ls.set_delay(1.0)
    b = core.Batch([loop])
    with pytest.raises(AobError, match="delay 0"):
        b.step()
    empty = core.Batch([])
    with pytest.raises(AobError, match="no instances"):
        empty.step()
    with pytest.raises(AobError, match="subaps_per_item"):
        empty.set_tuning(1025, 0, 0, 0, 0, 0)
    with pytest.raises(AobError, match="added twice"):
        core.Batch([loop, loop])


def test_batch_slopes_match_oracle_noiseless(mods):
    """Direct oracle check of one batched instance (no noise): relative slope rms <= 1e-4."""
    core, W = mods
    inst = W.mc_make(12, 6, 0.12, 5, pixsize=0.2)
    w, c, ls, loop = _build(core, inst, "f32", "cog", -1.0, seed=3)
    b = core.Batch([loop])
    b.step(noise=False)
    g = inst.setup.geom
    scale = 2 * np.pi / g.wavelength_um
    _, oimg, _ = osh.comp_image(inst.phase, g.tel.mpupil, g, scale, g.nphotons, noise=-1)
    ref, _, _ = ortc.centroids(oimg, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5, kind="cog")
    assert rel_rms(np.array(ls.buffer("centroids")), ref) < 1e-4
    com = -0.4 * (inst.setup.cmat.astype(np.float64) @ ref)
    assert rel_rms(np.array(ls.buffer("com")), com) < 1e-4


def test_batch_full_montecarlo_configuration(mods):
    """The 64-instance configuration (nxsub 24..40, 6x6 / 8x8 pixels, BF16 MVM,
    photon + readout noise): two batched steps equal each loop's own steps."""
    core, W = mods
    insts = W.mc_setup(64)
    specs = [(i, "bf16", "wcog", 0.5) for i in insts]
    ref = _reference_run(core, specs, 2)
    got, info = _batch_run(core, specs, 2)
    assert info["instances"] == 64
    for r, g in zip(ref, got):
        _assert_same(g, r)

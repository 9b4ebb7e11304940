"""GPU parity of the SH sensor, centroiders and LS controller against the CPU oracle.

Tolerances (stated by the project's accuracy contract):
  * slopes: relative rms error <= 1e-4 against the float64 oracle;
  * spot images / intensities: relative rms error <= 1e-5;
  * Poisson photon noise: bit-exact given the same float32 means;
  * readout noise (Box-Muller in float64, stored float32): |diff| <= 1e-5 * noise;
  * MVM float32: relative rms <= 1e-6; bf16 / fp8 within the stated quantisation bounds.
"""

import numpy as np
import pytest

from helpers import kolmogorov_screen, rel_rms, sh_geometry
from oracle import philox, rtc as ortc, sh as osh

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def core():
    from aob200 import core as C
    from aob200 import _lib

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return C


def _setup(core, name, noise=-1.0, seed=7):
    g = sh_geometry(name)
    w = core.ShWfs.from_geometry(g, noise=noise, seed=seed)
    phase = kolmogorov_screen(g.tel.n, r0_pixels=0.16 / (8.0 / g.tel.pupdiam), seed=seed)
    w.set_phase(phase)
    return g, w, phase


@pytest.mark.parametrize("name", ["sh8", "sh16", "sh40", "sh16x", "sh16fs"])
def test_sh_image_matches_oracle(core, name):
    g, w, phase = _setup(core, name)
    w.comp_image(noise=False)
    cube = np.array(w.d_bincube).reshape(g.npix * g.npix, g.nvalid, order="F")
    img = np.array(w.d_binimg)
    inten = np.array(w.d_intensities)
    scale = 2 * np.pi / g.wavelength_um
    ocube, oimg, osums = osh.comp_image(phase, g.tel.mpupil, g, scale, g.nphotons, noise=-1)
    assert rel_rms(cube, ocube) < 1e-5
    assert rel_rms(img, oimg) < 1e-5
    assert rel_rms(inten, osums) < 1e-5


@pytest.mark.parametrize("kind", ["cog", "tcog", "wcog"])
@pytest.mark.parametrize("name", ["sh16", "sh40", "sh16x", "sh16fs"])
def test_fused_and_standalone_centroids_match_oracle(core, name, kind):
    g, w, phase = _setup(core, name)
    offset, scale = g.npix / 2 - 0.5, g.pixsize
    c = core.Centroider(g.nvalid, offset, scale, kind)
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    thr = 0.05 * g.nphotons / (g.npix * g.npix)
    c.set_threshold(thr)
    wts = None
    if kind == "wcog":
        x = np.arange(g.npix) - (g.npix - 1) / 2
        wts = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * (g.npix / 2.0) ** 2)).astype(np.float32)
        c.load_weights(wts)
    ref = np.random.default_rng(3).standard_normal(2 * g.nvalid).astype(np.float32) * 0.01
    c.set_centroids_ref(ref)
    c.attach(w)
    ls = core.LsController(2 * g.nvalid, 4)
    dslopes = ls.buffer("centroids")

    w.comp_image(noise=False)
    img0 = np.array(w.d_binimg)
    c.get_cog(dslopes.ptr)  # fused path
    fused = np.array(dslopes)
    img_after = np.array(w.d_binimg)

    wflat = None if wts is None else np.tile(wts.ravel(order="F"), g.nvalid)
    os_, oint, oimg = ortc.centroids(img0, g.validsubsx, g.validsubsy, g.npix, scale, offset, ref=ref,
                                     kind=kind, threshold=thr, weights=wflat)
    assert rel_rms(fused, os_) < 1e-4
    assert rel_rms(np.array(c.buffer("intensities")), oint) < 1e-5
    # tCoG leaves its thresholded pixels in the image, like the reference
    assert rel_rms(img_after, oimg) < 1e-6

    # standalone kernel on a fresh image gives the same slopes
    c.attach(None)
    w.comp_image(noise=False)
    c2 = core.Centroider(g.nvalid, offset, scale, kind, wfs=None)
    c2.set_npix(g.npix)
    c2.load_validpos(g.validsubsx, g.validsubsy)
    c2.set_threshold(thr)
    c2.set_centroids_ref(ref)
    if wts is not None:
        c2.load_weights(wts)
    c2.load_img(np.array(w.d_binimg))
    c2.calibrate_img()
    c2.get_cog(dslopes.ptr)
    assert rel_rms(np.array(dslopes), os_) < 1e-4


def test_photon_noise_bit_exact_and_readout_noise(core):
    g, w, phase = _setup(core, "sh16", noise=0.5, seed=11)
    w.comp_image(noise=False)
    lam = np.array(w.d_bincube).reshape(-1, order="F").astype(np.float32)
    frame = w.frame
    w.comp_image(noise=True)
    noisy = np.array(w.d_bincube).reshape(-1, order="F")
    idx = np.arange(lam.size, dtype=np.uint64)
    pois = philox.poisson(lam.astype(np.float64), idx, frame, 11)
    gaus = philox.gaussian(idx, frame, 11)
    expected = pois.astype(np.float32) + np.float32(0.5) * gaus.astype(np.float32)
    # float32 rounding of (photons + noise * N): allow two ulps of the result
    assert np.all(np.abs(noisy - expected) <= 2 * np.spacing(np.abs(expected)) + 1e-5)
    # photon part alone: exact
    w.set_noise(0.0, 11)
    w.frame = frame
    w.comp_image(noise=True)
    p_gpu = np.array(w.d_bincube).reshape(-1, order="F")
    np.testing.assert_array_equal(p_gpu, pois.astype(np.float32))
    assert w.frame == frame + 1


def test_ls_mvm_integrator_precisions(core):
    rng = np.random.default_rng(5)
    nslope, nactu = 2496, 1377
    cmat = (rng.standard_normal((nactu, nslope)) * 0.01).astype(np.float32)
    s = rng.standard_normal(nslope).astype(np.float32)
    gains = rng.uniform(0.5, 1.5, nactu).astype(np.float32)
    ref = -(cmat.astype(np.float64) @ s.astype(np.float64))
    for prec, tol in (("f32", 1e-6), ("bf16", 8e-3), ("fp8", 6e-2)):
        c = core.LsController(nslope, nactu)
        c.set_precision(prec)
        c.set_cmat(cmat)
        c.set_gain(0.4)
        c.set_modal_gains(gains)
        c.set_centroids(s)
        c.comp_com()
        err = np.array(c.buffer("err"))
        com = np.array(c.buffer("com"))
        assert rel_rms(err, ref) < tol, prec
        assert rel_rms(com, 0.4 * ref * gains) < tol, prec
        c.comp_com()
        assert rel_rms(np.array(c.buffer("com")), 0.8 * ref * gains) < tol, prec


def test_ls_voltage_delay_perturb_clip_matches_oracle(core):
    rng = np.random.default_rng(9)
    nslope, nactu = 200, 60
    for delay in (0.0, 1.0, 1.3, 2.7):
        c = core.LsController(nslope, nactu, delay=delay)
        o = ortc.LsController(nslope, nactu, delay=delay, gain=0.3)
        cm = rng.standard_normal((nactu, nslope)).astype(np.float32) * 0.05
        c.set_cmat(cm)
        o.cmat = cm.astype(np.float64)
        c.set_gain(0.3)
        c.set_com_range(-0.8, 0.8)
        o.volt_min, o.volt_max = -0.8, 0.8
        pert = rng.standard_normal((3, nactu)).astype(np.float32) * 0.1
        c.add_perturb("p", pert, 3)
        o.perturb["p"] = [pert.astype(np.float64), 0, True]
        for it in range(6):
            s = rng.standard_normal(nslope).astype(np.float32)
            c.set_centroids(s)
            o.centroids = s.astype(np.float64)
            c.comp_com()
            o.comp_com()
            c.comp_voltage()
            v = o.comp_voltage()
            assert rel_rms(np.array(c.buffer("voltage")), v) < 1e-5, (delay, it)
            assert rel_rms(np.array(c.buffer("com")), o.com) < 1e-5, (delay, it)


@pytest.mark.parametrize("built,later", [(0.0, 1.5), (0.0, 2.0), (3.0, 1.0), (2.7, 0.0)])
def test_delay_set_after_construction_equals_constructor_delay(core, built, later):
    """set_delay resizes the command ring (floor(delay) + 2 buffers): a controller
    built with one delay and given another before its first step runs exactly like
    one built with the second."""
    rng = np.random.default_rng(11)
    nslope, nactu = 120, 40
    cm = rng.standard_normal((nactu, nslope)).astype(np.float32) * 0.05
    a = core.LsController(nslope, nactu, delay=built)
    a.set_delay(later)
    b = core.LsController(nslope, nactu, delay=later)
    for c in (a, b):
        c.set_cmat(cm)
        c.set_gain(0.3)
    for it in range(6):
        s = rng.standard_normal(nslope).astype(np.float32)
        for c in (a, b):
            c.set_centroids(s)
            c.comp_com()
            c.comp_voltage()
        np.testing.assert_array_equal(np.array(a.buffer("voltage")), np.array(b.buffer("voltage")), err_msg=str(it))
    assert a.status() == 0 and b.status() == 0


def test_svd_cmat_matches_numpy(core):
    rng = np.random.default_rng(4)
    nslope, nactu = 300, 120
    imat = rng.standard_normal((nslope, nactu)).astype(np.float32)
    c = core.LsController(nslope, nactu)
    c.set_imat(imat)
    c.svdec_imat()
    ev = np.array(c.buffer("eigenvals"))
    D = imat.astype(np.float64)
    w, U = np.linalg.eigh(D.T @ D)
    np.testing.assert_allclose(ev, w, rtol=1e-5)
    nfilt = 5
    c.build_cmat(nfilt)
    inv = np.zeros_like(w)
    inv[nfilt:] = 1.0 / w[nfilt:]
    cm = (U * inv) @ U.T @ D.T
    assert rel_rms(np.array(c.buffer("cmat", shape=(nactu, nslope))), cm) < 1e-5


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("delay", [0.0, 1.0, 1.4])
@pytest.mark.parametrize("fused_batch", [0, 1])
def test_loop_matches_separate_calls(core, graph, delay, mode, fused_batch):
    """The bound loop -- three kernels (mode 1) or the fused cooperative kernel
    (mode 2, whole share per round or one sub-aperture per round), with or
    without CUDA-graph replay -- equals the separate calls bit for bit in its
    slopes and images (every launch shape reduces in the same order)."""
    rng = np.random.default_rng(21)
    g = sh_geometry("sh16")
    nact = 97

    def build():
        w = core.ShWfs.from_geometry(g, noise=0.5, seed=5)
        c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "wcog")
        c.set_npix(g.npix)
        c.load_validpos(g.validsubsx, g.validsubsy)
        c.set_threshold(1.0)
        c.load_weights(np.ones((g.npix, g.npix), np.float32))
        ls = core.LsController(2 * g.nvalid, nact, delay=delay)
        ls.set_cmat(cm)
        ls.set_gain(0.3)
        ls.set_com_range(-0.5, 0.5)
        return w, c, ls

    cm = (rng.standard_normal((nact, 2 * g.nvalid)) * 0.01).astype(np.float32)
    screens = [kolmogorov_screen(g.tel.n, 20.0, seed=s) for s in range(5)]
    w1, c1, l1 = build()
    c1.attach(w1)
    w2, c2, l2 = build()
    loop = core.Loop(w2, c2, l2, graph=graph)
    loop.set_mode(mode, fused_batch)
    v2 = np.zeros(nact, np.float32)
    for it, ph in enumerate(screens):
        w1.set_phase(ph)
        w1.comp_image(noise=True)
        c1.get_cog(l1.buffer("centroids").ptr)
        l1.comp_com()
        l1.comp_voltage()
        loop.step(np.ascontiguousarray(ph.ravel(order="F")), v2, noise=True)
        v1 = np.array(l1.buffer("voltage"))
        np.testing.assert_array_equal(np.array(l2.buffer("centroids")), np.array(l1.buffer("centroids")))
        np.testing.assert_array_equal(np.array(w2.d_binimg), np.array(w1.d_binimg))
        assert rel_rms(v2, v1) < 1e-6
        assert rel_rms(np.array(l2.buffer("com")), np.array(l1.buffer("com"))) < 1e-6
    assert w1.frame == w2.frame == len(screens)
    assert l2.status() == 0
    assert loop.kernels_per_step() == (1 if mode == 2 else 3)


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("delay", [0.0, 1.4])
def test_direct_host_io_equals_copies(core, graph, delay):
    """With a pinned host voltage buffer the fused kernel's epilogue writes the
    voltages to host memory itself (set_host_io(1)); the results, the sensor's
    phase buffer and the loop state equal the copy-engine path bit for bit, also
    when such steps alternate with device-only (graph) steps."""
    import torch

    g = sh_geometry("sh16")
    nact = 97
    rng = np.random.default_rng(8)
    cm = (rng.standard_normal((nact, 2 * g.nvalid)) * 0.01).astype(np.float32)

    def build(io):
        w = core.ShWfs.from_geometry(g, noise=0.5, seed=5)
        c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "wcog")
        c.set_npix(g.npix)
        c.load_validpos(g.validsubsx, g.validsubsy)
        c.set_threshold(1.0)
        c.load_weights(np.ones((g.npix, g.npix), np.float32))
        ls = core.LsController(2 * g.nvalid, nact, delay=delay)
        ls.set_cmat(cm)
        ls.set_gain(0.3)
        ls.set_com_range(-0.5, 0.5)
        loop = core.Loop(w, c, ls, graph=graph)
        loop.set_host_io(io)
        return w, ls, loop

    wa, la, loopa = build(1)
    wb, lb, loopb = build(0)
    screens = [kolmogorov_screen(g.tel.n, 20.0, seed=40 + i).ravel(order="F") for i in range(6)]
    ph = torch.from_numpy(np.ascontiguousarray(np.stack(screens))).pin_memory()
    va = torch.zeros(nact, dtype=torch.float32).pin_memory()
    vb = torch.zeros(nact, dtype=torch.float32).pin_memory()
    for it in range(6):
        if it == 3:  # a device-only step in between (phase already on the device)
            loopa.step(None, None, noise=True)
            loopb.step(None, None, noise=True)
        else:
            loopa.step(ph[it].data_ptr(), va.data_ptr(), noise=True)
            loopb.step(ph[it].data_ptr(), vb.data_ptr(), noise=True)
            np.testing.assert_array_equal(va.numpy(), vb.numpy())
            np.testing.assert_array_equal(va.numpy(), np.array(la.buffer("voltage")))
        np.testing.assert_array_equal(np.array(wa.d_phase), np.array(wb.d_phase))
        np.testing.assert_array_equal(np.array(la.buffer("centroids")), np.array(lb.buffer("centroids")))
        np.testing.assert_array_equal(np.array(la.buffer("com")), np.array(lb.buffer("com")))
        np.testing.assert_array_equal(np.array(wa.d_binimg), np.array(wb.d_binimg))
    assert wa.frame == wb.frame == 6
    assert la.status() == 0 and loopa.kernels_per_step() == 1
    assert np.abs(va.numpy()).max() > 0
    # the asynchronous step (aob_loop_step_async) gives the same voltages once the stream has reached it
    loopa.step(ph[0].data_ptr(), va.data_ptr(), noise=True, wait=False)
    loopb.step(ph[0].data_ptr(), vb.data_ptr(), noise=True)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(va.numpy(), vb.numpy())
    np.testing.assert_array_equal(np.array(la.buffer("com")), np.array(lb.buffer("com")))


def test_sh_launch_shapes_agree(core):
    """Every autotuner launch shape of the sensor kernel gives the oracle's image,
    and all of them the same bits."""
    g, w, phase = _setup(core, "sh40", noise=0.5, seed=3)
    ocube, _, _ = osh.comp_image(phase, g.tel.mpupil, g, 2 * np.pi / g.wavelength_um, g.nphotons)
    first = None
    for batch in (1, 3, 8, 32, 0):
        w.set_tuning(batch)
        w.comp_image(noise=False)
        cube = np.array(w.d_bincube).reshape(g.npix * g.npix, g.nvalid, order="F")
        assert rel_rms(cube, ocube) < 1e-5
        w.frame = 4
        w.comp_image(noise=True)
        noisy = np.array(w.d_bincube)
        if first is None:
            first = (cube, noisy)
        np.testing.assert_array_equal(cube, first[0])
        np.testing.assert_array_equal(noisy, first[1])


@pytest.mark.parametrize("prec", ["f32", "bf16", "fp8"])
def test_mvm_kernels_agree_and_status_clean(core, prec):
    rng = np.random.default_rng(8)
    nslope, nactu = 4016, 1600
    cmat = (rng.standard_normal((nactu, nslope)) * 0.01).astype(np.float32)
    s = rng.standard_normal(nslope).astype(np.float32)
    out = {}
    for kind, nb in ((1, 0), (2, 0), (1, 300), (2, 37)):
        c = core.LsController(nslope, nactu)
        c.set_precision(prec)
        c.set_cmat(cmat)
        c.set_gain(1.0)
        c.set_centroids(s)
        c.set_tuning(kind, nb)
        c.comp_com()
        out[(kind, nb)] = np.array(c.buffer("err"))
        assert c.status() == 0
    base = out[(2, 0)]
    for k, v in out.items():
        assert rel_rms(v, base) < 1e-6, k


@pytest.mark.parametrize("graph", [False, True])
@pytest.mark.parametrize("delay", [0.0, 1.4])
@pytest.mark.parametrize("io", [1, 0])
def test_streamed_run_equals_steps(core, graph, delay, io):
    """aob_loop_run streams nsteps host phases (the next one copied while the
    current step computes) and equals nsteps aob_loop_step calls bit for bit:
    every step's voltages, the sensor images, the controller state and the noise
    frame counter, across two runs in a row (the second one asynchronous) and
    with pageable numpy buffers as well as pinned ones."""
    import torch

    g = sh_geometry("sh16")
    nact = 97
    rng = np.random.default_rng(9)
    cm = (rng.standard_normal((nact, 2 * g.nvalid)) * 0.01).astype(np.float32)

    def build():
        w = core.ShWfs.from_geometry(g, noise=0.5, seed=6)
        c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "wcog")
        c.set_npix(g.npix)
        c.load_validpos(g.validsubsx, g.validsubsy)
        c.set_threshold(1.0)
        c.load_weights(np.ones((g.npix, g.npix), np.float32))
        ls = core.LsController(2 * g.nvalid, nact, delay=delay)
        ls.set_cmat(cm)
        ls.set_gain(0.3)
        ls.set_com_range(-0.5, 0.5)
        loop = core.Loop(w, c, ls, graph=graph)
        loop.set_host_io(io)
        return w, ls, loop

    wa, la, loopa = build()
    wb, lb, loopb = build()
    nph = 3
    screens = [kolmogorov_screen(g.tel.n, 20.0, seed=60 + i).ravel(order="F") for i in range(nph)]
    ph = torch.from_numpy(np.ascontiguousarray(np.stack(screens))).pin_memory()
    n1, n2 = 7, 4
    va = torch.zeros((n1, nact), dtype=torch.float32).pin_memory()
    vb = torch.zeros(nact, dtype=torch.float32).pin_memory()
    loopa.run(ph.data_ptr(), n1, va.data_ptr(), noise=True, nphases=nph)
    for k in range(n1):
        loopb.step(ph[k % nph].data_ptr(), vb.data_ptr(), noise=True)
        np.testing.assert_array_equal(va[k].numpy(), vb.numpy())
    # a second, asynchronous run from pageable numpy buffers continues the same state
    ph_np = np.ascontiguousarray(ph.numpy()[::-1])
    va2 = np.zeros((n2, nact), np.float32)
    loopa.run(ph_np, n2, va2, noise=True, wait=False)
    torch.cuda.synchronize()
    for k in range(n2):
        loopb.step(ph_np[k % nph], vb.data_ptr(), noise=True)
        np.testing.assert_array_equal(va2[k], vb.numpy())
    np.testing.assert_array_equal(np.array(wa.d_phase), np.array(wb.d_phase))
    np.testing.assert_array_equal(np.array(wa.d_binimg), np.array(wb.d_binimg))
    np.testing.assert_array_equal(np.array(la.buffer("com")), np.array(lb.buffer("com")))
    np.testing.assert_array_equal(np.array(la.buffer("centroids")), np.array(lb.buffer("centroids")))
    assert wa.frame == wb.frame == n1 + n2
    assert la.status() == 0
    assert np.abs(va2).max() > 0
    with pytest.raises(Exception):
        loopa.run(ph_np, 0, None)

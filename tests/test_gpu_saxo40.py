"""The benchmarked configuration itself: the saxo40 loop through the fused kernel.

bench.py times one RTC iteration of the saxo40 workload (40x40 SH, 1248 valid
sub-apertures, 6x6 pixels, Nfft 32, 6 phase samples per sub-aperture, wCoG with
threshold, photon + 0.5 e- noise, 1377 x 2496 LS MVM) as one launch of
rtc_fused_kernel<T, 32, 6>.  These tests run that exact instantiation, built by
the same workload code, against the float64 oracle and against the separate
per-stage calls.

Tolerances: slopes relative rms <= 1e-4 against the oracle (the accuracy
contract for floating point); commands against float64 products of the same
slopes: 1e-6 (float32 MVM), 8e-3 (BF16) and 6e-2 (FP8 E4M3 with row scales);
noisy images: Poisson counts bit-exact, readout noise within two float32 ulps.
"""

import numpy as np
import pytest

from helpers import rel_rms
from oracle import philox, rtc as ortc, sh as osh

pytestmark = pytest.mark.gpu

TOL_COM = {"f32": 1e-6, "bf16": 8e-3, "fp8": 6e-2}


@pytest.fixture(scope="module")
def saxo():
    from aob200 import _lib
    from aob200.workloads import sh_loop_setup, von_karman_screens

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    setup = sh_loop_setup("saxo40")
    g = setup.geom
    assert (g.nvalid, g.nfft, g.pdiam, g.npix) == (1248, 32, 6, 6)
    screens = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 3, seed=11)
    return setup, screens


def _oracle_slopes(setup, img):
    g = setup.geom
    wflat = np.tile(setup.weights.ravel(order="F"), g.nvalid)
    s, _, _ = ortc.centroids(img, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5,
                             kind="wcog", threshold=setup.threshold, weights=wflat)
    return s


@pytest.mark.parametrize("precision", ["f32", "bf16", "fp8"])
def test_saxo40_fused_step_matches_oracle(saxo, precision):
    """Noise-free fused step: image, slopes and commands against the oracle."""
    from aob200.workloads import build_sh_loop

    setup, screens = saxo
    g = setup.geom
    wfs, c, ls, loop = build_sh_loop(setup, precision=precision, graph=False)
    loop.set_mode(2, 0)  # the fused kernel only (an error if it does not fit)
    volt = np.zeros(setup.nactu, np.float32)
    com_prev = np.zeros(setup.nactu)
    scale = 2 * np.pi / g.wavelength_um
    for ph in screens[:2]:
        loop.step(np.ascontiguousarray(ph.ravel(order="F")), volt, noise=False)
        assert loop.kernels_per_step() == 1
        _, oimg, _ = osh.comp_image(ph, g.tel.mpupil, g, scale, g.nphotons, noise=-1)
        img = np.array(wfs.d_binimg)
        assert rel_rms(img, oimg) < 1e-5
        s_gpu = np.array(ls.buffer("centroids"))
        s_ref = _oracle_slopes(setup, oimg)
        assert rel_rms(s_gpu, s_ref) < 1e-4
        # integrator, gain 0.4, delay 0: voltage = command
        com_ref = com_prev - 0.4 * (setup.cmat.astype(np.float64) @ s_gpu.astype(np.float64))
        com = np.array(ls.buffer("com"))
        assert rel_rms(com - com_prev, com_ref - com_prev) < TOL_COM[precision]
        np.testing.assert_array_equal(volt, com)
        # and end to end against the oracle's slopes
        com_oracle = com_prev - 0.4 * (setup.cmat.astype(np.float64) @ s_ref)
        assert rel_rms(com - com_prev, com_oracle - com_prev) < max(1e-4, TOL_COM[precision])
        com_prev = com.astype(np.float64)
    assert ls.status() == 0


def test_saxo40_fused_equals_separate_calls_with_noise(saxo):
    """Noisy fused steps equal the separate sensor / centroider / controller calls
    bit for bit (slopes, images, frames), and the noise is the oracle's."""
    from aob200 import core
    from aob200.workloads import build_sh_loop

    setup, screens = saxo
    g = setup.geom
    w1, c1, l1, _ = build_sh_loop(setup, graph=False, seed=77)
    c1.attach(w1)
    w2, c2, l2, loop = build_sh_loop(setup, graph=False, seed=77)
    loop.set_mode(2, 0)
    v2 = np.zeros(setup.nactu, np.float32)
    for it, ph in enumerate(screens):
        frame = w1.frame
        w1.set_phase(ph)
        w1.comp_image(noise=True)
        c1.get_cog(l1.buffer("centroids").ptr)
        l1.comp_com()
        l1.comp_voltage()
        loop.step(np.ascontiguousarray(ph.ravel(order="F")), v2, noise=True)
        np.testing.assert_array_equal(np.array(l2.buffer("centroids")), np.array(l1.buffer("centroids")))
        np.testing.assert_array_equal(np.array(w2.d_binimg), np.array(w1.d_binimg))
        np.testing.assert_array_equal(np.array(w2.d_bincube), np.array(w1.d_bincube))
        assert rel_rms(v2, np.array(l1.buffer("voltage"))) < 1e-6
        # the slopes of the noisy image are the oracle's centroids of that image
        assert rel_rms(np.array(l2.buffer("centroids")), _oracle_slopes(setup, np.array(w2.d_binimg))) < 1e-4
        if it == 0:
            # photon counts of the fused kernel: bit-exact Philox Poisson draws of the
            # noise-free means; readout noise within two float32 ulps
            w1.comp_image(noise=False)
            lam = np.array(w1.d_bincube).reshape(-1, order="F").astype(np.float32)
            idx = np.arange(lam.size, dtype=np.uint64)
            pois = philox.poisson(lam.astype(np.float64), idx, frame, 77).astype(np.float32)
            gaus = philox.gaussian(idx, frame, 77).astype(np.float32)
            expected = pois + np.float32(setup.noise) * gaus
            noisy = np.array(w2.d_bincube).reshape(-1, order="F")
            assert np.all(np.abs(noisy - expected) <= 2 * np.spacing(np.abs(expected)) + 1e-5)
            w1.comp_image(noise=False)  # (noise-free images do not advance the frame)
    assert w1.frame == w2.frame == len(screens)
    assert l2.status() == 0 and loop.kernels_per_step() == 1


def test_sh40_photon_noise_bit_exact(saxo):
    """Photon noise alone at the saxo40 geometry (Nfft 32, 6x6 pixels): the
    standalone sensor kernel's counts equal the oracle's Philox draws exactly."""
    from aob200 import core

    setup, screens = saxo
    g = setup.geom
    w = core.ShWfs.from_geometry(g, noise=0.0, seed=19)
    w.set_phase(screens[0])
    w.comp_image(noise=False)
    lam = np.array(w.d_bincube).reshape(-1, order="F").astype(np.float32)
    frame = w.frame
    w.comp_image(noise=True)
    got = np.array(w.d_bincube).reshape(-1, order="F")
    idx = np.arange(lam.size, dtype=np.uint64)
    np.testing.assert_array_equal(got, philox.poisson(lam.astype(np.float64), idx, frame, 19).astype(np.float32))

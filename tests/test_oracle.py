"""Pins the CPU oracle before it is trusted as the checker.

* Philox4x32-10 against the published known-answer vectors (Random123 KAT).
* Centroiders / control law / clip / latency against the same NumPy expressions
  the reference's own test-suite uses (shesha/tests/pytest/rtc/test_rtcFFF.py:
  154-163 CoG via scipy center_of_mass, 166-171 control law, 174-187 clip,
  229-247 comp_voltage, 255-285 tCoG, 324-363 wCoG), at its tolerance 1e-2
  (max error relative to the max) -- and far tighter here.
* SH spot formation by analytic properties (the reference has no golden data
  for it): a flat wavefront gives a centred spot, a tilt moves it by the
  predicted number of pixels, total flux is normalised.
"""

import numpy as np
import pytest
from scipy.ndimage import center_of_mass

from aob200 import geometry as G
from oracle import philox, rtc, sh


def test_philox_known_answers():
    kat = [
        ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
        ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
        ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
         (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
    ]
    for ctr, key, want in kat:
        got = philox.philox4x32(*ctr, *key)
        assert tuple(int(x) for x in got) == want


def test_poisson_statistics():
    for lam in (0.3, 4.0, 9.9, 10.0, 39.9, 40.0, 57.0, 3000.0):
        idx = np.arange(20000, dtype=np.uint64)
        x = philox.poisson(np.full(idx.shape, lam), idx, frame=3, seed=99)
        assert np.all(x == np.floor(x)) and np.all(x >= 0)
        assert abs(x.mean() - lam) < 5 * np.sqrt(lam / x.size) + 1e-9
        assert abs(x.var() / lam - 1) < 0.06


def test_gaussian_statistics():
    z = philox.gaussian(np.arange(200000, dtype=np.uint64), frame=1, seed=5)
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1) < 0.01


def _image_from_cube(cube, g):
    return sh.bin_image(cube, g.validsubsx, g.validsubsy, g.npix, g.nxsub)


@pytest.fixture(scope="module")
def geom16():
    return G.sh_geometry(G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7), 128)


def _cube_as_xyk(cube, npix):
    return cube.reshape(npix, npix, -1, order="F")


def test_cog_matches_center_of_mass(geom16):
    g = geom16
    rng = np.random.default_rng(0)
    cube = rng.random((g.npix * g.npix, g.nvalid))
    img = _image_from_cube(cube, g)
    offset, scale = g.npix / 2 - 0.5, g.pixsize
    s, inten, _ = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, scale, offset)
    ref = np.zeros(2 * g.nvalid)
    c3 = _cube_as_xyk(cube, g.npix)
    for k in range(g.nvalid):
        cm = center_of_mass(c3[:, :, k])
        ref[k] = (cm[0] - offset) * scale
        ref[k + g.nvalid] = (cm[1] - offset) * scale
    assert np.abs(s - ref).max() / np.abs(ref).max() < 1e-6
    np.testing.assert_allclose(inten, cube.sum(axis=0), rtol=1e-12)


def test_tcog_and_wcog_match_reference_expressions(geom16):
    g = geom16
    rng = np.random.default_rng(1)
    cube = rng.random((g.npix * g.npix, g.nvalid))
    img = _image_from_cube(cube, g)
    offset, scale, thr = g.npix / 2 - 0.5, g.pixsize, 0.1
    s, _, img2 = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, scale, offset,
                               kind="tcog", threshold=thr)
    c3 = _cube_as_xyk(cube, g.npix) - thr
    c3[c3 < 0] = 0
    ref = np.zeros(2 * g.nvalid)
    for k in range(g.nvalid):
        cm = center_of_mass(c3[:, :, k])
        ref[k], ref[k + g.nvalid] = (cm[0] - offset) * scale, (cm[1] - offset) * scale
    assert np.abs(s - ref).max() / np.abs(ref).max() < 1e-4
    # the thresholded pixels are written back into the image
    k0 = 0
    blk = img2[g.validsubsx[k0]:g.validsubsx[k0] + g.npix, g.validsubsy[k0]:g.validsubsy[k0] + g.npix]
    exp = _cube_as_xyk(cube, g.npix)[:, :, k0] - thr
    np.testing.assert_allclose(blk, np.where(exp > 0, exp, 1e-6))

    w = rng.random(g.npix * g.npix)
    wfull = np.tile(w, g.nvalid)
    s, _, _ = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, scale, offset,
                            kind="wcog", threshold=thr, weights=wfull)
    c3 = _cube_as_xyk(cube, g.npix) - thr
    c3[c3 < 0] = 1e-6
    w2 = w.reshape(g.npix, g.npix, order="F")
    for k in range(g.nvalid):
        cm = center_of_mass(c3[:, :, k] * w2)
        ref[k], ref[k + g.nvalid] = (cm[0] - offset) * scale, (cm[1] - offset) * scale
    assert np.abs(s - ref).max() / np.abs(ref).max() < 1e-4


def test_control_law_clip_and_latency():
    rng = np.random.default_rng(2)
    nslope, nactu = 60, 25
    c = rtc.LsController(nslope, nactu, delay=1.3, gain=0.4)
    c.cmat = rng.standard_normal((nactu, nslope))
    c.centroids = rng.standard_normal(nslope)
    c.comp_com()
    np.testing.assert_allclose(c.com, -0.4 * c.cmat @ c.centroids)
    # latency: a*ring[0] + b*ring[1] then perturbation then clip
    com0, com1 = c.ring[0].copy(), c.ring[1].copy()
    pert = rng.random(nactu)
    c.perturb["test"] = [pert[None, :], 0, True]
    c.volt_min, c.volt_max = -1, 1
    v = c.comp_voltage()
    exp = np.clip(0.3 * com0 + 0.7 * com1 + pert, -1, 1)
    np.testing.assert_allclose(v, exp)


def test_flat_wavefront_gives_centred_spot(geom16):
    g = geom16
    pupil = g.tel.mpupil
    phase = np.zeros_like(pupil)
    scale = 2 * np.pi / g.wavelength_um
    cube, img, sums = sh.comp_image(phase, pupil, g, scale, g.nphotons, noise=-1)
    # flux normalisation
    np.testing.assert_allclose(cube.sum(axis=0), g.fluxPerSub.astype(np.float64) * g.nphotons, rtol=1e-12)
    s, _, _ = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5)
    full = g.fluxPerSub > 0.999
    assert np.abs(s[:g.nvalid][full]).max() < 1e-9
    assert np.abs(s[g.nvalid:][full]).max() < 1e-9


def test_tilt_moves_spot_by_prediction(geom16):
    g = geom16
    pupil = g.tel.mpupil
    n = pupil.shape[0]
    # tilt of 0.1 arcsec along x: phase [um] = theta[rad] * x[m] * 1e6
    theta = 0.1 / G.RAD2ARCSEC
    dx = 8.0 / g.tel.pupdiam
    x = (np.arange(n) - n / 2) * dx
    phase = (theta * x * 1e6)[:, None] * np.ones((1, n))
    scale = 2 * np.pi / g.wavelength_um
    _, img, _ = sh.comp_image(phase, pupil, g, scale, g.nphotons, noise=-1)
    s, _, _ = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5)
    full = g.fluxPerSub > 0.999
    # spot moves by +/- 0.1 arcsec (sign follows the forward FFT convention)
    assert np.allclose(np.abs(s[:g.nvalid][full]), 0.1, atol=0.02)
    assert np.abs(s[g.nvalid:][full]).max() < 1e-6


def test_cpu_baseline_loop_matches_oracle(geom16):
    """The vectorised CPU-baseline step equals the scalar oracle (noise off)."""
    from oracle.loop_cpu import CpuShLoop

    g = geom16
    rng = np.random.default_rng(3)
    nact = 50
    cmat = rng.standard_normal((nact, 2 * g.nvalid)) * 0.01
    n = g.tel.n
    phase = (0.1 * rng.standard_normal((n, n))).astype(np.float32)
    loop = CpuShLoop(g, cmat, "cog", gain=0.5, workers=2)
    com = loop.step(phase)
    _, img, _ = sh.comp_image(phase, g.tel.mpupil, g, 2 * np.pi / g.wavelength_um, g.nphotons)
    s, _, _ = rtc.centroids(img, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5)
    np.testing.assert_allclose(com, -0.5 * cmat @ s, rtol=1e-9, atol=1e-12)


def test_float32_exp_log_accuracy():
    """The sampler's own exp / log / log1p stay within a few float32 ulps."""
    xs = np.linspace(-10.0, 0.0, 2001, dtype=np.float32)
    e = np.array([philox._expf_neg(x) for x in xs], dtype=np.float64)
    assert np.max(np.abs(e / np.exp(xs.astype(np.float64)) - 1)) < 5e-7
    ys = np.geomspace(1e-6, 1e6, 2001).astype(np.float32)
    lg = np.array([philox._logf(y) for y in ys], dtype=np.float64)
    assert np.all(np.abs(lg - np.log(ys.astype(np.float64))) < 2e-6 * np.maximum(1, np.abs(np.log(ys))))
    ds = np.linspace(-0.25, 0.5, 1001, dtype=np.float32)
    l1 = np.array([philox._log1pf(d) for d in ds], dtype=np.float64)
    assert np.max(np.abs(l1 - np.log1p(ds.astype(np.float64)))) < 3e-7


@pytest.mark.parametrize("lam", [2.5, 9.75, 37.0, 39.9, 40.0, 61.0, 400.0, 5000.0])
def test_poisson_sampler_matches_the_pmf(lam):
    """Chi-square of 40k deviates against the exact Poisson pmf (both branches)."""
    from scipy import stats

    n = 40000
    x = philox.poisson(np.full(n, lam, np.float32), np.arange(n, dtype=np.uint64), frame=17, seed=2024)
    lo, hi = int(stats.poisson.ppf(1e-4, lam)), int(stats.poisson.ppf(1 - 1e-4, lam))
    edges = np.unique(np.linspace(lo, hi + 1, 40).astype(int))
    obs = np.histogram(x, bins=np.concatenate([[-1e9], edges[1:-1], [1e9]]))[0]
    cdf = stats.poisson.cdf(edges[1:-1] - 1, lam)
    exp_p = np.diff(np.concatenate([[0.0], cdf, [1.0]]))
    chi2 = np.sum((obs - n * exp_p) ** 2 / (n * exp_p))
    p = stats.chi2.sf(chi2, len(obs) - 1)
    assert p > 1e-4, (lam, chi2, len(obs))


@pytest.fixture(scope="module")
def pyr16():
    return G.pyr_geometry(G.PyrParams(nxsub=16, wavelength_um=0.7, ampl=3.0, npts=8, pup_sep=12, fssize=3.2), 64,
                          diam=8.0, cobs=0.14)


def test_pyramid_flat_wavefront_is_balanced(pyr16):
    """Flat wavefront: the four pupil images carry equal flux and the mean slopes vanish."""
    from oracle import pyr as opyr

    g = pyr16
    n = g.tel.n
    img = opyr.comp_image(np.zeros((n, n)), g.tel.mpupil, g, g.wavelength_um, g.nphotons)
    np.testing.assert_allclose(img.sum(), g.nphotons, rtol=1e-10)
    s, flux = opyr.slopes(img, g.validsubsx, g.validsubsy, g.nvalid, 1.0)
    q = [img[g.validsubsx[k * g.nvalid:(k + 1) * g.nvalid], g.validsubsy[k * g.nvalid:(k + 1) * g.nvalid]].sum()
         for k in range(4)]
    assert max(q) / min(q) - 1 < 1e-6
    # per-sub-aperture slopes of a flat wavefront are not zero (edge diffraction,
    # hence reference slopes) but they are antisymmetric: their means vanish
    assert abs(s[:g.nvalid].mean()) < 1e-6 and abs(s[g.nvalid:].mean()) < 1e-6


def test_pyramid_tilt_response_is_linear_and_signed(pyr16):
    """A small tilt moves the x slopes, in proportion, and leaves the y slopes at zero on average."""
    from oracle import pyr as opyr

    g = pyr16
    n = g.tel.n
    x = (np.arange(n) - n / 2.0)[:, None] * np.ones((1, n))
    out = []
    for amp in (0.0005, 0.001):  # small-signal range of the modulated pyramid
        img = opyr.comp_image(amp * x, g.tel.mpupil, g, g.wavelength_um, g.nphotons)
        s, _ = opyr.slopes(img, g.validsubsx, g.validsubsy, g.nvalid, 1.0)
        out.append((s[:g.nvalid].mean(), s[g.nvalid:].mean()))
    (sx1, sy1), (sx2, sy2) = out
    assert abs(sx1) > 1e-3 and abs(sx2 / sx1 - 2) < 0.1
    assert abs(sy1) < 0.05 * abs(sx1) and abs(sy2) < 0.05 * abs(sx2)


def test_pyramid_threaded_image_equals_sequential(pyr16):
    """The multi-threaded baseline path (scipy.fft, modulation points batched) forms
    the same image as the point-by-point numpy.fft path."""
    from oracle import pyr as opyr

    g = pyr16
    n = g.tel.n
    ph = np.random.default_rng(5).standard_normal((n, n)) * 0.05
    a = opyr.comp_image(ph, g.tel.mpupil, g, g.wavelength_um, g.nphotons)
    b = opyr.comp_image(ph, g.tel.mpupil, g, g.wavelength_um, g.nphotons, workers=4)
    np.testing.assert_allclose(b, a, rtol=1e-10, atol=1e-9 * a.max())

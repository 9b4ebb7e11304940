"""GPU parity of the modulated pyramid sensor and the pyramid centroider.

Tolerances: binned images relative rms <= 1e-5 against the float64 oracle;
slopes relative rms <= 1e-4 (the accuracy contract); photon noise bit-exact
given the GPU's float32 means; readout noise within float32 rounding.
"""

import numpy as np
import pytest

from helpers import kolmogorov_screen, rel_rms
from oracle import philox
from oracle import pyr as opyr

pytestmark = pytest.mark.gpu

PYR_CASES = {
    "pyr16": (dict(nxsub=16, wavelength_um=0.7, ampl=3.0, npts=8, pup_sep=12, fssize=3.2), 64),
    "pyr50": (dict(nxsub=50, wavelength_um=1.075, ampl=3.0, npts=24, pup_sep=32, fssize=3.2), 100),
}


@pytest.fixture(scope="module")
def core():
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return C


def _geom(name):
    from aob200 import geometry as G

    kw, pup = PYR_CASES[name]
    return G.pyr_geometry(G.PyrParams(**kw), pup, diam=8.0, cobs=0.14)


def _phase(g, seed):
    # residual-like phase: 0.05 um rms von Karman-ish screen on the pupil grid
    ph = kolmogorov_screen(g.tel.n, r0_pixels=2.0, seed=seed)
    return (ph * (0.05 / max(ph.std(), 1e-12))).astype(np.float32)


@pytest.mark.parametrize("name", ["pyr16", "pyr50"])
def test_pyramid_image_matches_oracle(core, name):
    g = _geom(name)
    w = core.PyrWfs.from_geometry(g)
    ph = _phase(g, 3)
    w.set_phase(ph)
    w.comp_image(noise=False)
    got = np.array(w.d_binimg)
    ref = opyr.comp_image(ph, g.tel.mpupil, g, g.wavelength_um, g.nphotons)
    assert rel_rms(got, ref) < 1e-5
    assert abs(got.sum() / g.nphotons - 1) < 1e-5


def test_pyramid_noise_bit_exact(core):
    g = _geom("pyr16")
    w = core.PyrWfs.from_geometry(g, noise=0.3, seed=21)
    w.set_phase(_phase(g, 4))
    w.comp_image(noise=False)
    lam = np.array(w.d_binimg).ravel(order="F").astype(np.float32)
    frame = w.frame
    w.comp_image(noise=True)
    noisy = np.array(w.d_binimg).ravel(order="F")
    idx = np.arange(lam.size, dtype=np.uint64)
    pois = philox.poisson(lam, idx, frame, 21)
    gaus = philox.gaussian(idx, frame, 21)
    expected = pois.astype(np.float32) + np.float32(0.3) * gaus.astype(np.float32)
    assert np.all(np.abs(noisy - expected) <= 2 * np.spacing(np.abs(expected)) + 1e-5)
    w.set_noise(0.0, 21)
    w.frame = frame
    w.comp_image(noise=True)
    np.testing.assert_array_equal(np.array(w.d_binimg).ravel(order="F"), pois.astype(np.float32))
    assert w.frame == frame + 1


@pytest.mark.parametrize("method", [0, 1, 2, 3])
@pytest.mark.parametrize("name", ["pyr16", "pyr50"])
def test_pyramid_centroider_matches_oracle(core, name, method):
    g = _geom(name)
    w = core.PyrWfs.from_geometry(g)
    w.set_phase(_phase(g, 5))
    w.comp_image(noise=False)
    img = np.array(w.d_binimg)
    c = core.Centroider(g.nvalid, 0.0, 0.7, "pyr")
    c.load_validpos(g.validsubsx, g.validsubsy)
    c.set_pyr_method(method)
    ref = np.random.default_rng(2).standard_normal(2 * g.nvalid).astype(np.float32) * 1e-3
    c.set_centroids_ref(ref)
    c.attach(w)
    ls = core.LsController(2 * g.nvalid, 4)
    d = ls.buffer("centroids")
    c.get_cog(d.ptr)
    got = np.array(d)
    exp, flux = opyr.slopes(img, g.validsubsx, g.validsubsy, g.nvalid, 0.7, ref=ref, method=method)
    assert rel_rms(got, exp) < 1e-4
    assert rel_rms(np.array(c.buffer("intensities")), flux) < 1e-5

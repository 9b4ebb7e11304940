"""The uint16 camera path: fakecam digitisation and the Rtc_UFF centroiders.

A sensor with fakecam digitises each image into a uint16 frame
(digitalize_krnl, libsutra/src.cu/sutra_wfs.cu:2243-2255); an RTC with uint16
input (Rtc_UFF) loads such frames, calibrates them with dark, flat and a pixel
look-up table (calib_krnl, sutra_centroider.cu:108-115; calibrate_img_validPix,
sutra_centroider.cpp:194-223) and computes the slopes from the result.

Tolerances: frames equal to the float64 oracle within one count (float32
rounding before the truncation); calibrated images relative rms <= 1e-6;
slopes <= 1e-4 against the oracle's CoG of the oracle's calibrated image.
"""

import numpy as np
import pytest

from helpers import import_dropin, kolmogorov_screen, rel_rms, sh_geometry
from oracle import rtc as ortc

pytestmark = pytest.mark.gpu

MAX_FLUX, MAX_PIX = 2000, 60000


@pytest.fixture(scope="module")
def cam():
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    g = sh_geometry("sh16")
    w = C.ShWfs.from_geometry(g)
    w.set_fakecam(True, MAX_FLUX, MAX_PIX)
    side = g.npix * g.nxsub
    rng = np.random.default_rng(4)
    dark = (rng.random((side, side)) * 20).astype(np.float32)
    flat = (0.9 + 0.2 * rng.random((side, side))).astype(np.float32)
    w.set_dark(dark)
    w.set_flat(flat)
    w.set_phase(kolmogorov_screen(g.tel.n, r0_pixels=0.16 / (8.0 / g.tel.pupdiam), seed=9))
    w.comp_image(noise=False)
    return C, g, w, dark, flat


def test_fakecam_frame_matches_oracle(cam):
    C, g, w, dark, flat = cam
    img = np.array(w.d_binimg)
    frame = np.array(w.d_camimg)
    assert frame.dtype == np.uint16
    ref = ortc.digitalize(img, dark, flat, MAX_FLUX, MAX_PIX)
    d = np.abs(frame.astype(np.int64) - ref.astype(np.int64))
    assert d.max() <= 1 and np.mean(d == 0) > 0.999
    assert frame.max() == MAX_PIX  # the brightest pixels saturate at max_pix_value


@pytest.mark.parametrize("impl", ["python", "native"])
@pytest.mark.parametrize("kind", ["cog", "wcog"])
def test_uint16_rtc_calibrates_and_centroids(cam, kind, impl):
    """Rtc_UFF: load the sensor's d_camimg (device copy), calibrate with a dark, a
    flat and a pixel permutation, then CoG / wCoG -- against the oracle; through
    the Python drop-in and the compiled pair."""
    C, g, w, _, _ = cam
    carma, sutra = import_dropin(impl)
    ctx = carma.context.get_instance()
    rtc = sutra.Rtc_UFF()
    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, kind)
    rtc.add_controller(ctx, "ls", 0, 0.0, 2 * g.nvalid, 16, idx_centro=np.zeros(1), ncentro=1)
    ce = rtc.d_centro[0]
    ce.set_npix(g.npix)
    ce.load_validpos(g.validsubsx, g.validsubsy, g.nvalid)
    thr = 50.0
    wts = None
    if kind == "wcog":
        ce.set_threshold(thr)
        x = np.arange(g.npix) - (g.npix - 1) / 2
        wts = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / 8.0).astype(np.float32)
        ce.init_weights()
        ce.load_weights(wts, 2)
    frame = np.array(w.d_camimg)
    side = frame.shape[0]
    ce.load_img(w.d_camimg, side)
    assert np.array_equal(np.array(ce.d_img_raw), frame)
    rng = np.random.default_rng(5)
    dark = (rng.random((side, side)) * 5).astype(np.float32)
    flat = (0.95 + 0.1 * rng.random((side, side))).astype(np.float32)
    lut = rng.permutation(side * side).astype(np.int32)
    ce.set_dark(dark, side)
    ce.set_flat(flat, side)
    ce.set_lutPix(lut, side * side)
    rtc.do_calibrate_img(0)
    cal = ortc.calibrate(frame, dark, flat, lut)
    assert rel_rms(np.array(ce.d_img), cal) < 1e-6
    rtc.do_centroids(0)
    wflat = None if wts is None else np.tile(wts.ravel(order="F"), g.nvalid)
    s, _, _ = ortc.centroids(cal, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix / 2 - 0.5, kind=kind,
                             threshold=thr, weights=wflat)
    assert rel_rms(np.array(rtc.d_control[0].d_centroids), s) < 1e-4
    # only the valid windows
    ce.calibrate_img_validPix()
    calv = ortc.calibrate(frame, dark, flat, lut, valid=(g.validsubsx, g.validsubsy), npix=g.npix)
    assert rel_rms(np.array(ce.d_img), calv) < 1e-6
    assert np.count_nonzero(np.array(ce.d_img)) <= g.nvalid * g.npix * g.npix


def test_uint16_frame_from_host(cam):
    """A host uint16 frame (the camera's own buffer) through the core API."""
    C, g, w, _, _ = cam
    c = C.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "cog")
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    frame = np.array(w.d_camimg)
    c.load_img(frame)
    c.calibrate_img()
    ls = C.LsController(2 * g.nvalid, 8)
    c.get_cog(ls.buffer("centroids").ptr)
    s, _, _ = ortc.centroids(frame.astype(np.float64), g.validsubsx, g.validsubsy, g.npix, g.pixsize,
                             g.npix / 2 - 0.5)
    assert rel_rms(np.array(ls.buffer("centroids")), s) < 1e-4

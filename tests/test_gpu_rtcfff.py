"""The reference's own RTC tests, restated against the drop-in `sutra` module.

shesha/tests/pytest/rtc/test_rtcFFF.py and test_rtcFFF_pyramid.py build an
``Rtc_FFF`` with a centroider that is not attached to a sensor (its image is
loaded with ``load_img``) and a *generic* controller, then check centroiders,
the generic integrator, clipping, perturbation voltages and ``comp_voltage``
against NumPy, at the reference's precision (1e-2 on the maximum error
relative to the largest value).  The same module-level set-up and the same
checks run here through the drop-in modules (compass-saxoplus_b200/dropin),
with the inputs a ``CompassSupervisor`` would give made by this project's own
sensors: the SH image of test_sh.py's 16x16, 8-pixel sensor at 0.5 um on a
seeded screen (delay 3, gain 0.4) and a pyramid image for the masked-pixel
test.
The reference's ``sup.rtc.get_command_matrix`` is a seeded random matrix here;
the checks compare the drop-in against NumPy on that same matrix.
"""

import os
import sys

import numpy as np
import pytest
from scipy.ndimage import center_of_mass

from helpers import import_dropin, kolmogorov_screen

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
precision = 1e-2
DELAY, GAIN, NACTU = 3.0, 0.4, 243


def relative_array_error(array1, array2):
    return np.abs((array1 - array2) / array2.max()).max()


@pytest.fixture(scope="module", params=["python", "native"])
def sh(request):
    """Module-level set-up of test_rtcFFF.py:33-79, through the Python drop-in and
    the compiled pair."""
    from aob200 import _lib
    from aob200 import core as C
    from aob200 import geometry as G

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    carma, sutra = import_dropin(request.param)
    # test_sh.py: 16x16 sub-apertures, 8 pixels of 0.3" at 0.5 um (field of view extended: ntot 64 > nfft 32),
    # fracsub 0.8, magnitude 3, no noise
    g = G.sh_geometry(G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.5, fracsub=0.8, gsmag=3.0), 128,
                      diam=8.0, cobs=0.12, ittime=0.002)
    w = C.ShWfs.from_geometry(g)
    w.set_phase(kolmogorov_screen(g.tel.n, r0_pixels=0.16 / (8.0 / g.tel.pupdiam), seed=5, lam_um=0.5))
    w.comp_image(noise=False)
    bincube = np.array(w.d_bincube).reshape(g.npix, g.npix, g.nvalid, order="F").astype(np.float64)
    ctx = carma.context.get_instance()
    rtc = sutra.Rtc_FFF()
    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, "cog")
    rtc.add_controller(ctx, "generic", 0, DELAY, g.nvalid * 2, NACTU, idx_centro=np.zeros(1), ncentro=1)
    centro = rtc.d_centro[0]
    control = rtc.d_control[0]
    rtc.d_centro[0].set_npix(g.npix)
    xvalid, yvalid = g.validsubsx.astype(np.int32), g.validsubsy.astype(np.int32)
    rtc.d_centro[0].load_validpos(xvalid, yvalid, xvalid.size)
    cmat = (np.random.default_rng(7).standard_normal((NACTU, 2 * g.nvalid)) * 1e-2).astype(np.float32)
    rtc.d_control[0].set_cmat(cmat)
    rtc.d_control[0].set_gain(GAIN)
    frame = np.array(w.d_binimg).astype(np.float32)
    frame /= frame.max()
    rtc.d_centro[0].load_img(frame, frame.shape[0])
    rtc.d_centro[0].calibrate_img()
    rtc.do_centroids(0)
    rtc.do_control(0)
    rng = np.random.default_rng(11)
    dark = rng.random(frame.shape)
    flat = rng.random(frame.shape)
    centro.set_dark(dark, frame.shape[0])
    centro.set_flat(flat, frame.shape[0])
    return dict(g=g, ctx=ctx, rtc=rtc, centro=centro, control=control, cmat=cmat, frame=frame, dark=dark, flat=flat,
                bincube=bincube, xvalid=xvalid, yvalid=yvalid, sutra=sutra)


def test_init_and_setters(sh):
    """test_rtcFFF.py:86-148 (init values, set_npix, load_validpos, set_cmat, set_gain, load_img, set_dark /
    set_flat)."""
    g, centro, control = sh["g"], sh["centro"], sh["control"]
    assert centro.nvalid - g.nvalid < precision
    assert centro.offset - (g.npix / 2 - 0.5) < precision
    assert centro.scale - g.pixsize < precision
    assert centro.type == "cog"
    assert control.nslope - g.nvalid * 2 < precision
    assert control.nactu - NACTU < precision
    assert control.type == "generic"
    assert control.delay - DELAY < precision
    assert g.ntot > g.nfft  # the file's sensor extends its field of view
    assert centro.npix - g.npix < precision
    assert relative_array_error(np.array(centro.d_validx), sh["xvalid"]) < precision
    assert relative_array_error(np.array(centro.d_validy), sh["yvalid"]) < precision
    assert relative_array_error(np.array(control.d_cmat), sh["cmat"]) < precision
    assert control.gain - GAIN < precision
    assert relative_array_error(np.array(centro.d_img_raw), sh["frame"]) < precision
    assert relative_array_error(np.array(centro.d_dark), sh["dark"]) < precision
    assert relative_array_error(np.array(centro.d_flat), sh["flat"]) < precision


def test_calibrate_img(sh):
    """test_rtcFFF.py:148-151."""
    centro = sh["centro"]
    centro.calibrate_img()
    imgCal = (sh["frame"] - sh["dark"]) * sh["flat"]
    assert relative_array_error(np.array(centro.d_img), imgCal) < precision


def _cog_slopes(cube, g, offset, scale, f=lambda a: a):
    slopes = np.zeros(g.nvalid * 2)
    for k in range(g.nvalid):
        tmp = center_of_mass(f(cube[:, :, k]))
        slopes[k] = (tmp[0] - offset) * scale
        slopes[k + g.nvalid] = (tmp[1] - offset) * scale
    return slopes


def test_doCentroids_cog(sh):
    """test_rtcFFF.py:154-163."""
    g, centro, control = sh["g"], sh["centro"], sh["control"]
    slopes = _cog_slopes(sh["bincube"], g, centro.offset, centro.scale)
    assert relative_array_error(np.array(control.d_centroids), slopes) < precision


def test_do_control_generic(sh):
    """test_rtcFFF.py:166-171: the generic integrator from a zero command."""
    control = sh["control"]
    slopes = np.array(control.d_centroids)
    cmat = np.array(control.d_cmat)
    commands = cmat.dot(slopes) * control.gain * (-1)
    assert relative_array_error(np.array(control.d_com), commands) < precision


def test_clipping_and_perturbations(sh):
    """test_rtcFFF.py:174-226 (set_comRange, do_clipping, perturbation voltages, add_perturb)."""
    rtc, control = sh["rtc"], sh["control"]
    rng = np.random.default_rng(3)
    control.set_comRange(-1, 1)
    assert control.comRange == (-1, 1)
    C = (rng.random(NACTU) - 0.5) * 4
    control.set_com(C, C.size)
    rtc.do_clipping(0)
    C_clipped = C.copy()
    C_clipped[np.where(C > 1)] = 1
    C_clipped[np.where(C < -1)] = -1
    assert relative_array_error(np.array(control.d_com_clipped), C_clipped) < precision
    C = rng.random(NACTU)
    control.add_perturb_voltage("test", C, 1)
    assert relative_array_error(np.array(control.d_perturb_map["test"][0]), C) < precision
    control.remove_perturb_voltage("test")
    assert control.d_perturb_map == {}
    C = rng.random(NACTU)
    control.add_perturb_voltage("test", C, 1)
    com = np.array(control.d_com_clipped)
    control.add_perturb()
    assert relative_array_error(np.array(control.d_com_clipped), com + C) < precision
    control.disable_perturb_voltage("test")
    com = np.array(control.d_com)
    control.add_perturb()
    assert relative_array_error(np.array(control.d_com), com) < precision
    control.enable_perturb_voltage("test")
    com = np.array(control.d_com_clipped)
    C = np.array(control.d_perturb_map["test"][0])
    control.add_perturb()
    assert relative_array_error(np.array(control.d_com_clipped), com + C) < precision
    control.reset_perturb_voltage()
    assert control.d_perturb_map == {}


def test_comp_voltage(sh):
    """test_rtcFFF.py:229-247: latency interpolation of the delay ring, perturbation, clip."""
    control = sh["control"]
    volt_min, volt_max = -1, 1
    control.set_comRange(volt_min, volt_max)
    control.comp_voltage()
    C = np.random.default_rng(4).random(NACTU)
    control.add_perturb_voltage("test", C, 1)
    control.set_com(C, C.size)
    com0 = np.array(control.d_circularComs0)
    com1 = np.array(control.d_circularComs1)
    control.comp_voltage()
    a = DELAY - int(DELAY)
    b = 1 - a
    commands = a * com0 + b * com1
    comPertu = commands + C
    comPertu[np.where(comPertu > volt_max)] = volt_max
    comPertu[np.where(comPertu < volt_min)] = volt_min
    assert relative_array_error(np.array(control.d_voltage), comPertu) < precision
    control.reset_perturb_voltage()


def test_doCentroids_tcog_bpcog_wcog(sh):
    """test_rtcFFF.py:250-363: remove_centroider, then tCoG, bpCoG and wCoG on the loaded frame."""
    g, ctx, rtc, control = sh["g"], sh["ctx"], sh["rtc"], sh["control"]
    frame, xvalid, yvalid = sh["frame"], sh["xvalid"], sh["yvalid"]
    rtc.remove_centroider(0)
    assert rtc.d_centro == []
    bincube = sh["bincube"] / sh["bincube"].max()

    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, "tcog")
    centro = rtc.d_centro[-1]
    threshold = 0.1
    centro.set_threshold(threshold)
    centro.set_npix(g.npix)
    centro.load_validpos(xvalid, yvalid, xvalid.size)
    centro.load_img(frame, frame.shape[0])
    centro.calibrate_img()
    rtc.do_centroids(0)
    slopes = _cog_slopes(bincube, g, centro.offset, centro.scale, lambda a: np.maximum(a - threshold, 0))
    assert relative_array_error(np.array(control.d_centroids), slopes) < precision

    rtc.remove_centroider(0)
    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, "bpcog")
    centro = rtc.d_centro[-1]
    bpix = 8
    centro.set_nmax(8)
    centro.set_npix(g.npix)
    centro.load_validpos(xvalid, yvalid, xvalid.size)
    centro.load_img(frame, frame.shape[0])
    centro.calibrate_img()
    rtc.do_centroids(0)

    def brightest(imagette):
        imagette = imagette.copy()
        threshold = np.sort(imagette, axis=None)[-(bpix + 1)]
        imagette -= threshold
        imagette[np.where(imagette < 0)] = 0
        return imagette

    slopes = _cog_slopes(bincube, g, centro.offset, centro.scale, brightest)
    assert relative_array_error(np.array(control.d_centroids), slopes) < precision

    rtc.remove_centroider(0)
    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, "wcog")
    centro = rtc.d_centro[-1]
    centro.set_npix(g.npix)
    threshold = 0.1
    centro.set_threshold(threshold)
    x = np.arange(g.npix) - (g.npix - 1) / 2.0
    weights = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * 2.0**2)).astype(np.float32)
    centro.init_weights()
    centro.load_weights(weights, weights.ndim)
    centro.load_validpos(xvalid, yvalid, xvalid.size)
    centro.load_img(frame, frame.shape[0])
    centro.calibrate_img()
    rtc.do_centroids(0)

    def weighted(a):
        a = a - threshold
        a[np.where(a < 0)] = 1e-6
        return a * weights

    slopes = _cog_slopes(bincube, g, centro.offset, centro.scale, weighted).astype(np.float32)
    assert relative_array_error(np.array(control.d_centroids), slopes) < precision


def test_generic_command_laws(sh):
    """The other laws of SutraControllerGeneric::comp_com (controller_generic.cpp:219-328) against NumPy:
    leaky integrator, pseudo-open-loop integrator, modal integrator and the two-matrix law."""
    sutra, ctx = sh["sutra"], sh["ctx"]
    rng = np.random.default_rng(9)
    ns, na = 120, 40
    cmat = (rng.standard_normal((na, ns)) * 0.1).astype(np.float32)
    imat = (rng.standard_normal((ns, na)) * 0.1).astype(np.float32)
    matE = (np.eye(na) * 0.9 + rng.standard_normal((na, na)) * 0.01).astype(np.float32)
    decay = rng.uniform(0.5, 1.0, na).astype(np.float32)
    mg = rng.uniform(0.5, 1.5, na).astype(np.float32)
    s = rng.standard_normal(ns).astype(np.float32)
    rtc = sutra.Rtc_FFF()
    rtc.add_controller(ctx, "generic", 0, 0.0, ns, na, idx_centro=np.zeros(0), ncentro=0)
    c = rtc.d_control[0]
    c.set_cmat(cmat)
    c.set_imat(imat)
    c.set_gain(0.3)
    c.set_modal_gains(mg)
    c.set_matE(matE)
    c.set_decayFactor(decay)
    c.d_centroids.set(s)
    c0 = rng.standard_normal(na).astype(np.float32)
    f64 = lambda a: np.asarray(a, np.float64)  # noqa: E731

    def run(law, leaky=1.0, polc=False):
        c.set_commandlaw(law)
        c.set_leaky_factor(leaky)
        c.set_polc(polc)
        c.set_com(c0, na)
        c.comp_voltage()  # com_clipped = c0 (delay 0, no clip)
        rtc.do_control(0)
        return f64(np.array(c.d_com))

    got = run("integrator", leaky=0.95)
    exp = 0.95 * f64(c0) - 0.3 * f64(cmat) @ f64(s)
    assert relative_array_error(got, exp) < 1e-5
    got = run("integrator", leaky=0.95, polc=True)
    sol = f64(s) - f64(imat) @ f64(c0)
    exp = (1 - 0.3) * 0.95 * f64(c0) - 0.3 * f64(cmat) @ sol
    assert relative_array_error(got, exp) < 1e-5
    buff = -(f64(cmat) @ f64(s)) * f64(mg)
    got = run("modal_integrator", leaky=0.9)
    exp = 0.3 * f64(matE) @ buff + 0.9 * f64(c0)
    assert relative_array_error(got, exp) < 1e-5
    got = run("2matrices")
    exp = (f64(matE) @ f64(c0)) * f64(decay) + buff
    assert relative_array_error(got, exp) < 1e-5
    assert c.command_law == "2matrices"


@pytest.mark.parametrize("impl", ["python", "native"])
def test_doCentroids_maskedPix(impl):
    """test_rtcFFF_pyramid.py:26-87: masked-pixel centroider and generic controller on a pyramid image."""
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    carma, sutra = import_dropin(impl)
    sys.path.insert(0, GOLD)
    try:
        import ref_cases as RC
    finally:
        sys.path.remove(GOLD)
    g = RC.pyr_geometry("pyr16")
    w = C.PyrWfs.from_geometry(g)
    w.set_phase((np.random.default_rng(1).standard_normal((g.tel.n, g.tel.n)) * 0.02).astype(np.float32))
    w.comp_image(noise=False)
    ctx = carma.context.get_instance()
    rtc = sutra.Rtc_FFF()
    nslope = g.validsubsx.size
    rtc.add_centroider(ctx, g.nvalid * 4, 0, g.pixsize, False, 0, "maskedpix")
    rtc.add_controller(ctx, "generic", 0, 1.0, nslope, 97, idx_centro=np.zeros(1), ncentro=1)
    centro = rtc.d_centro[0]
    control = rtc.d_control[0]
    rtc.d_centro[0].set_npix(g.npix)
    xvalid, yvalid = g.validsubsx.astype(np.int32), g.validsubsy.astype(np.int32)
    rtc.d_centro[0].load_validpos(xvalid, yvalid, xvalid.size)
    rtc.d_control[0].set_cmat((np.random.default_rng(2).standard_normal((97, nslope)) * 1e-2).astype(np.float32))
    rtc.d_control[0].set_gain(0.5)
    frame = np.array(w.d_binimg).astype(np.float32)
    frame /= frame.max()
    rtc.d_centro[0].load_img(frame, frame.shape[0])
    rtc.d_centro[0].calibrate_img()
    rtc.do_centroids(0)
    rtc.do_control(0)
    binimg = np.array(centro.d_img)
    slopes = np.zeros(xvalid.size)
    psum = binimg[xvalid, yvalid].sum() / slopes.size
    for k in range(slopes.size):
        slopes[k] = binimg[xvalid[k], yvalid[k]] / psum - 1  # -1 for ref slopes
    assert relative_array_error(np.array(control.d_centroids), slopes) < precision

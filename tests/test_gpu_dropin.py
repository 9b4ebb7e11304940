"""The drop-in `carma` / `sutra` modules drive the same kernels as the core API.

A supervisor-style loop (shesha's sequence: set the guide-star phase, comp_image,
do_centroids, do_control, apply_control) over one Shack-Hartmann and one
pyramid sensor feeding one LS controller must equal, bit for bit, the same
loop written with ``aob200.core`` calls; the controller reads the two
centroiders' slopes one block after the other.  It runs through both drop-ins:
the Python modules (dropin/) and the compiled pybind11 pair (dropin_native/).
"""

import numpy as np
import pytest

from helpers import import_dropin, kolmogorov_screen, sh_geometry

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["python", "native"])
def mods(request):
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    carma, sutra = import_dropin(request.param)
    return C, carma, sutra


def _pyr_geom():
    from aob200 import geometry as G

    return G.pyr_geometry(G.PyrParams(nxsub=16, wavelength_um=0.7, ampl=3.0, npts=8, pup_sep=12, fssize=3.2), 64,
                          diam=8.0, cobs=0.14)


@pytest.mark.parametrize("delay", [0.0, 1.0])
def test_supervisor_loop_equals_core_calls(mods, delay):
    C, carma, sutra = mods
    gs, gp = sh_geometry("sh16"), _pyr_geom()
    nact = 120
    nslope = 2 * (gs.nvalid + gp.nvalid)
    rng = np.random.default_rng(4)
    cm = (rng.standard_normal((nact, nslope)) * 0.01).astype(np.float32)
    ref_sh = (rng.standard_normal(2 * gs.nvalid) * 0.01).astype(np.float32)
    wts = np.ones((gs.npix, gs.npix), np.float32)

    # ---- through the drop-in modules, in shesha's call order
    ctx = carma.context.get_instance_1gpu(0)
    sens = sutra.Sensors(ctx, None, ["sh", "pyrhr"], 2,
                         np.array([gs.nxsub, gp.nxsub]), np.array([gs.nvalid, gp.nvalid]), 1,
                         np.array([gs.npix, gp.validsubsx.size]), np.array([gs.pdiam, gp.pdiam]),
                         np.array([gs.nrebin, gp.nrebin]), np.array([gs.nfft, gp.nfft]),
                         np.array([gs.ntot, gp.ntot]), np.array([gs.tel.n, gp.pyr_cx.size]),
                         np.array([gs.subapd, gp.pdiam], np.float32), np.array([gs.nphotons, gp.nphotons], np.float32),
                         np.zeros(2, np.float32), [False, False], False, 0, 0, ctx.active_device, False)
    wsh, wpy = sens.d_wfs
    wsh.load_arrays(gs.phasemap, gs.hrmap, gs.binmap, gs.halfxy, gs.fluxPerSub, gs.validsubsx, gs.validsubsy,
                    gs.validpuppixx, gs.validpuppixy)
    wsh.set_pupil(gs.tel.mpupil)
    wpy.load_arrays(gp.halfxy, gp.pyr_cx, gp.pyr_cy, None, gp.sincar, gp.submask, gp.validsubsx, gp.validsubsy,
                    gp.phasemap, gp.fluxPerSub)
    wpy.set_pupil(gp.tel.mpupil)
    z = np.zeros(2, np.float32)
    sens.initgs(z, z, np.array([gs.wavelength_um, gp.wavelength_um], np.float32), z, z, z,
                np.array([0.5, 0.3], np.float32), np.array([5, 9]), z, z, z, z)

    rtc = sutra.Rtc_FFF()
    rtc.add_centroider(ctx, gs.nvalid, gs.npix / 2 - 0.5, gs.pixsize, False, ctx.active_device, "wcog", wsh)
    rtc.add_centroider(ctx, gp.nvalid, 0.0, 0.7, False, ctx.active_device, "pyr", wpy)
    csh, cpy = rtc.d_centro
    csh.set_npix(gs.npix)
    csh.load_validpos(gs.validsubsx, gs.validsubsy, gs.validsubsx.size)
    csh.set_threshold(1.0)
    csh.load_weights(wts, 2)
    cpy.load_validpos(gp.validsubsx, gp.validsubsy, gp.validsubsx.size)
    cpy.set_pyr_method(1)
    rtc.set_centroids_ref(np.concatenate([ref_sh, np.zeros(2 * gp.nvalid, np.float32)]))
    rtc.add_controller(ctx, "ls", ctx.active_device, delay, nslope, nact)
    ctl = rtc.d_control[0]
    ctl.set_cmat(cm)
    rtc.set_gain(0, 0.3)
    ctl.set_comRange(-0.5, 0.5)

    # ---- the same loop with core calls
    w1 = C.ShWfs.from_geometry(gs, noise=0.5, seed=5)
    p1 = C.PyrWfs.from_geometry(gp, noise=0.3, seed=9)
    c1 = C.Centroider(gs.nvalid, gs.npix / 2 - 0.5, gs.pixsize, "wcog")
    c1.set_npix(gs.npix)
    c1.load_validpos(gs.validsubsx, gs.validsubsy)
    c1.set_threshold(1.0)
    c1.load_weights(wts)
    c1.set_centroids_ref(ref_sh)
    c1.attach(w1)
    q1 = C.Centroider(gp.nvalid, 0.0, 0.7, "pyr")
    q1.load_validpos(gp.validsubsx, gp.validsubsy)
    q1.set_pyr_method(1)
    q1.attach(p1)
    l1 = C.LsController(nslope, nact, delay=delay)
    l1.set_cmat(cm)
    l1.set_gain(0.3)
    l1.set_com_range(-0.5, 0.5)
    cen = l1.buffer("centroids")

    for it in range(4):
        phs = kolmogorov_screen(gs.tel.n, 20.0, seed=10 + it)
        php = kolmogorov_screen(gp.tel.n, 2.0, seed=20 + it)
        php = (php * (0.05 / max(php.std(), 1e-12))).astype(np.float32)

        wsh.d_gs.d_phase.d_screen.set(phs)
        wpy.d_gs.d_phase.d_screen.set(php)
        wsh.comp_image()
        wpy.comp_image()
        rtc.do_centroids(0)
        rtc.do_control(0)
        rtc.apply_control(0)

        w1.set_phase(phs)
        p1.set_phase(php)
        w1.comp_image(noise=True)
        p1.comp_image(noise=True)
        c1.get_cog(cen.ptr)
        q1.get_cog(cen.ptr + 4 * 2 * gs.nvalid)
        l1.comp_com()
        l1.comp_voltage()

        np.testing.assert_array_equal(np.array(wsh.d_binimg), np.array(w1.d_binimg))
        np.testing.assert_array_equal(np.array(wpy.d_binimg), np.array(p1.d_binimg))
        np.testing.assert_array_equal(np.array(ctl.d_centroids), np.array(cen))
        np.testing.assert_array_equal(np.array(ctl.d_com), np.array(l1.buffer("com")))
        np.testing.assert_array_equal(np.array(ctl.d_voltage), np.array(l1.buffer("voltage")))
    assert np.abs(np.array(ctl.d_voltage)).max() > 0



def test_native_pair_methods_equal_core_calls():
    """The compiled pair beyond the loop above: get_cog into the sensor's own
    slopes, geometric slopes, the generic controller's leaky integrator, and a
    shape error raised as RuntimeError (the reference's std::runtime_error)."""
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    carma, sutra = import_dropin("native")
    g = sh_geometry("sh16")
    ctx = carma.context.get_instance_1gpu(0)
    sens = sutra.Sensors(ctx, None, ["sh"], 1, g.nxsub, g.nvalid, 1, g.npix, g.pdiam, g.nrebin, g.nfft, g.ntot,
                         g.tel.n, np.float32(g.subapd), np.float32(g.nphotons), 0.0, False, False, 0, 0, 0, False)
    w = sens.d_wfs[0]
    assert isinstance(w, sutra.SHWFS)
    w.load_arrays(g.phasemap, g.hrmap, g.binmap, g.halfxy, g.fluxPerSub, g.validsubsx, g.validsubsy,
                  g.validpuppixx, g.validpuppixy, g.ttprojmat)
    w.set_pupil(g.tel.mpupil)
    sens.initgs(0, 0, g.wavelength_um, 0, 0, 0, -1.0, 3, 0, 0, 0, 0)
    ph = kolmogorov_screen(g.tel.n, 20.0, seed=31)
    w.d_gs.d_phase.d_screen.set(ph)
    w.comp_image(False)
    rtc = sutra.Rtc_FFF()
    rtc.add_centroider(ctx, g.nvalid, g.npix / 2 - 0.5, g.pixsize, False, 0, "cog", w)
    cen = rtc.d_centro[0]
    cen.set_npix(g.npix)
    cen.load_validpos(g.validsubsx, g.validsubsy, g.nvalid)
    nact = 40
    rtc.add_controller(ctx, "generic", 0, 0.0, 2 * g.nvalid, nact)
    ctl = rtc.d_control[0]
    assert isinstance(ctl, sutra.ControllerGENERIC)
    cm = (np.random.default_rng(6).standard_normal((nact, 2 * g.nvalid)) * 0.01).astype(np.float32)
    ctl.set_cmat(cm)
    ctl.set_commandlaw("integrator")
    ctl.set_leaky_factor(0.95)
    rtc.set_gain(0, 0.4)
    with pytest.raises(RuntimeError):
        ctl.set_cmat(cm.T)

    w1 = C.ShWfs.from_geometry(g)
    w1.set_phase(ph)
    w1.comp_image(noise=False)
    c1 = C.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, "cog")
    c1.set_npix(g.npix)
    c1.load_validpos(g.validsubsx, g.validsubsy)
    c1.attach(w1)
    l1 = C.LsController(2 * g.nvalid, nact, kind="generic")
    l1.set_cmat(cm)
    l1.set_commandlaw("integrator")
    l1.set_leaky_factor(0.95)
    l1.set_gain(0.4)
    for _ in range(3):
        rtc.do_centroids(0)
        rtc.do_control(0)
        rtc.apply_control(0)
        c1.get_cog(l1.buffer("centroids").ptr)
        l1.comp_com()
        l1.comp_voltage()
    np.testing.assert_array_equal(np.array(ctl.d_centroids), np.array(l1.buffer("centroids")))
    np.testing.assert_array_equal(np.array(ctl.d_com), np.array(l1.buffer("com")))
    np.testing.assert_array_equal(np.array(ctl.d_voltage), np.array(l1.buffer("voltage")))
    assert ctl.command_law == "integrator"

    cen.get_cog()  # into the sensor's d_slopes
    np.testing.assert_array_equal(np.array(w.d_slopes), np.array(ctl.d_centroids))
    for kind in (0, 1, 2):
        w.slopes_geom(kind)
        w1.slopes_geom(kind)
        np.testing.assert_array_equal(np.array(w.d_slopes), np.array(w1.buffer("slopes")))

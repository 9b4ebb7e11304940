"""Sensor methods beside the image path, against the oracle and the reference run.

* geometric slopes (SutraWfs::slopes_geom, all three methods) of the SH and the
  pyramid sensor;
* the pyramid focal-plane image (compute_pyrfocalplane) and the setters of its
  field stop and pyramid mask;
* the drop-in ``Rtc_FFF.do_imat`` with a ``Dms`` built from the reference's own
  DM arrays (dm17: influence functions and pixel lists from its dm_init),
  against the interaction matrix the reference's SutraRtc::do_imat computed;
* the drop-in centroider's ``get_cog`` into the sensor's ``d_slopes``.

tests/golden/ref_extras_{sh16,pyr16}.npz come from the reference's sutra build
run on a B200 (make_ref_fixtures.py extras).

Tolerances: geometric slopes relative rms <= 1e-5 against the float64 oracle
and the reference (sums of float32 differences in another order); the focal
plane <= 1e-4 against the oracle (the FFT of this project against numpy's)
and the reference (cuFFT); the interaction matrix <= 1e-4 (slopes of two
float32 sensors, the accuracy contract for floating point).
"""

import os
import sys

import numpy as np
import pytest

from helpers import import_dropin, rel_rms

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
import ref_cases as RC  # noqa: E402

pytestmark = pytest.mark.gpu



@pytest.fixture(scope="module")
def core():
    from aob200 import _lib
    from aob200 import core as C

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return C


def _ref(name):
    return np.load(os.path.join(GOLD, f"ref_extras_{name}.npz"))


@pytest.mark.parametrize("name", ["sh16", "saxo40"])
@pytest.mark.parametrize("kind", [0, 1, 2])
def test_sh_slopes_geom_matches_oracle(core, name, kind):
    from aob200.workloads import von_karman_screens
    from oracle import sh as osh

    g = RC.sh_geometry(name)
    w = core.ShWfs.from_geometry(g)
    ph = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, 0.14, 25.0, 1, seed=7 + kind)[0]
    w.set_phase(ph)
    w.slopes_geom(kind)
    s = np.array(w.buffer("slopes"))
    ref = osh.slopes_geom(ph, g.tel.mpupil, g.phasemap, g.fluxPerSub, g.subapd, g.pdiam, kind, g.ttprojmat)
    assert rel_rms(s, ref) < 1e-5


def test_sh_slopes_geom_matches_reference_run(core):
    d = _ref("sh16")
    g = RC.sh_geometry("sh16")
    w = core.ShWfs.from_geometry(g)
    w.set_phase(d["phase"])
    for kind in (0, 1, 2):
        w.slopes_geom(kind)
        assert rel_rms(np.array(w.buffer("slopes")), d[f"geom{kind}"]) < 1e-5, kind


def test_sh_slopes_geom_into_caller_buffer(core):
    g = RC.sh_geometry("sh16")
    w = core.ShWfs.from_geometry(g)
    w.set_phase(np.random.default_rng(2).standard_normal((g.tel.n, g.tel.n)).astype(np.float32) * 0.1)
    w.slopes_geom(0)
    own = np.array(w.buffer("slopes"))
    ls = core.LsController(2 * g.nvalid, 8)
    dst = ls.buffer("centroids")
    w.slopes_geom(0, dst.ptr)
    np.testing.assert_array_equal(np.array(dst), own)


def test_pyr_focal_plane_and_geom_slopes_match_reference_run(core):
    from oracle import pyr as opyr

    d = _ref("pyr16")
    g = RC.pyr_geometry("pyr16")
    w = core.PyrWfs.from_geometry(g)
    w.set_phase(d["phase"])
    w.set_compute_focalplane(True)
    w.comp_image(False)
    n = g.nfft
    focal = np.array(w.buffer("pyrfocalplane", shape=(n, n)))
    assert rel_rms(focal, d["focal"]) < 1e-4
    assert rel_rms(focal, opyr.focal_plane(d["phase"], g.tel.mpupil, g, g.wavelength_um)) < 1e-4
    assert rel_rms(np.array(w.d_binimg), d["binimg"]) < 1e-5
    for kind in (0, 1):
        w.slopes_geom(kind)
        assert rel_rms(np.array(w.buffer("slopes")), d[f"geom{kind}"]) < 1e-5, kind


def test_pyr_focal_plane_off_leaves_image_unchanged(core):
    g = RC.pyr_geometry("pyr16")
    ph = (np.random.default_rng(3).standard_normal((g.tel.n, g.tel.n)) * 0.02).astype(np.float32)
    imgs = []
    for on in (False, True):
        w = core.PyrWfs.from_geometry(g)
        w.set_phase(ph)
        w.set_compute_focalplane(on)
        w.comp_image(False)
        imgs.append(np.array(w.d_binimg))
    np.testing.assert_array_equal(imgs[0], imgs[1])


def test_pyr_setters_equal_load_arrays(core):
    """set_submask / set_phalfxy overwrite what load_arrays loaded: setting the
    same arrays again leaves the image bit for bit equal, a changed field stop
    changes it."""
    g = RC.pyr_geometry("pyr16")
    ph = (np.random.default_rng(4).standard_normal((g.tel.n, g.tel.n)) * 0.02).astype(np.float32)
    w = core.PyrWfs.from_geometry(g)
    w.set_phase(ph)
    w.comp_image(False)
    a = np.array(w.d_binimg)
    mask = np.exp(1j * np.asarray(g.halfxy, np.float64)).astype(np.complex64).T
    w.set_phalfxy(mask)
    w.set_submask(g.submask)
    w.comp_image(False)
    np.testing.assert_array_equal(np.array(w.d_binimg), a)
    sm = g.submask.copy()
    sm[: g.nfft // 2] = 0
    w.set_submask(sm)
    w.comp_image(False)
    assert rel_rms(np.array(w.d_binimg), a) > 1e-3


@pytest.fixture(scope="module", params=["python", "native"])
def mods(core, request):
    return import_dropin(request.param)


def _dropin_sh(carma, sutra, g):
    ctx = carma.context.get_instance_1gpu(0)
    i64 = lambda v: np.array([v], dtype=np.int64)  # noqa: E731
    f32 = lambda v: np.array([v], dtype=np.float32)  # noqa: E731
    sens = sutra.Sensors(ctx, None, ["sh"], 1, i64(g.nxsub), i64(g.nvalid), i64(1), i64(g.npix), i64(g.pdiam),
                         i64(g.nrebin), i64(g.nfft), i64(g.ntot), i64(g.tel.n), f32(g.subapd), f32(g.nphotons),
                         f32(g.nphotons), np.zeros(1, np.int32), np.zeros(1, bool), np.zeros(1, np.int32),
                         np.zeros(1, np.int32), ctx.active_device, False)
    w = sens.d_wfs[0]
    w.load_arrays(g.phasemap, g.hrmap, g.binmap, g.halfxy, g.fluxPerSub, g.validsubsx, g.validsubsy,
                  g.validpuppixx, g.validpuppixy, g.ttprojmat)
    w.set_pupil(g.tel.mpupil)
    one = lambda v, t=np.float32: np.array([v], dtype=t)  # noqa: E731
    sens.initgs(one(0), one(0), one(g.wavelength_um), one(8.0), 1e11, one(g.tel.n, np.int64), one(-1.0),
                one(1234, np.int64), one(1.0), one(0), one(0), one(0))
    return ctx, sens, w


def test_dropin_do_imat_matches_reference_run(mods):
    carma, sutra = mods
    d = _ref("sh16")
    dm = dict(np.load(os.path.join(GOLD, "dm17.npz")))
    g = RC.sh_geometry("sh16")
    ctx, sens, w = _dropin_sh(carma, sutra, g)
    dms = sutra.Dms()
    dim = int(dm["dim"])
    dms.add_dm(ctx, "pzt", 0.0, dim, int(dm["ntotact"]), int(dm["influsize"]), int(dm["influpos"].size),
               int(dm["ninflu"].size), float(d["push4imat"]), 0, ctx.active_device)
    dms.d_dms[0].pzt_loadarrays(dm["influ"], dm["influpos"], dm["ninflu"], dm["influstart"], dm["i1"], dm["j1"])
    w.d_gs.add_layer("pzt", 0, float(d["dm_offset"]), float(d["dm_offset"]))
    rtc = sutra.Rtc_FFF()
    rtc.add_centroider(ctx, g.nvalid, g.npix // 2.0 - 0.5, g.pixsize, False, ctx.active_device, "cog", w)
    c = rtc.d_centro[0]
    c.load_validpos(g.validsubsx, g.validsubsy, g.nvalid)
    c.set_npix(g.npix)
    nactu = int(dm["ntotact"])
    rtc.add_controller(ctx, "ls", ctx.active_device, 0.0, 2 * g.nvalid, nactu, dms=dms,
                       idx_dms=np.zeros(1, np.int32), ndm=1, idx_centro=np.zeros(1, np.int32), ncentro=1)
    rtc.do_imat(0, dms, False)
    imat = np.array(rtc.d_control[0].d_imat)
    assert imat.shape == d["imat"].shape
    assert rel_rms(imat, d["imat"]) < 1e-4
    # the poke leaves the DM flat and the commands untouched
    assert not np.array(dms.d_dms[0].d_com).any()


def test_dropin_get_cog_writes_sensor_slopes(mods):
    carma, sutra = mods
    g = RC.sh_geometry("sh16")
    ctx, sens, w = _dropin_sh(carma, sutra, g)
    w.d_gs.d_phase.d_screen.set((np.random.default_rng(5).standard_normal((g.tel.n, g.tel.n)) * 0.05)
                                .astype(np.float32))
    w.comp_image(False)
    rtc = sutra.Rtc_FFF()
    rtc.add_centroider(ctx, g.nvalid, g.npix // 2.0 - 0.5, g.pixsize, False, ctx.active_device, "cog", w)
    c = rtc.d_centro[0]
    c.load_validpos(g.validsubsx, g.validsubsy, g.nvalid)
    c.set_npix(g.npix)
    rtc.add_controller(ctx, "ls", ctx.active_device, 0.0, 2 * g.nvalid, 4)
    rtc.do_centroids(0)
    c.get_cog()
    np.testing.assert_array_equal(np.array(w.d_slopes), np.array(rtc.d_control[0].d_centroids))


def test_dropin_sh_comp_nphot(mods):
    carma, sutra = mods
    g = RC.sh_geometry("sh16")
    ctx, sens, w = _dropin_sh(carma, sutra, g)
    w.comp_nphot(0.001, 0.5, 8.0, 16, zerop=1e11, gsmag=8.0)
    expect = np.float32(1e11 * 10 ** (-0.4 * 8.0) * 0.001 * 0.5 * (8.0 / 16) ** 2)
    assert w.nphot == pytest.approx(float(expect), rel=1e-7)

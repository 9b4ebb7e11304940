"""The reference's own GPU implementation of the SH loop, driven through its API.

Test and baseline infrastructure: the reference's ``carma`` / ``sutra`` modules
built from its sources by oracle/build_ref.py (oracle/_ref/) are driven the
way shesha's supervisor drives them (shesha/shesha/init/geom_init.py:94-101
Telescope; wfs_init.py:100-234 Sensors / initgs / load_arrays;
rtc_init.py:272-358 add_centroider / load_validpos / set_npix /
set_threshold / init_weights / load_weights; add_controller "ls" with
set_cmat / set_gain / set_modal_gains), then stepped in the supervisor's
order (compassSupervisor.py:175-289): the guide-star phase from the host,
comp_image, do_centroids, do_control, comp_voltage, and the voltages read
back to the host (np.array of the carma object).

Used by tests/golden/make_ref_fixtures.py (noise-free fixtures) and by
bench.py --impl reference (the reference arm timed on the same GPU).  Nothing
in the package imports this module.
"""

import os
import sys

import numpy as np

REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref")


def modules():
    """The reference's (carma, sutra) modules; ImportError when not built."""
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import carma
    import sutra

    return carma, sutra


def available() -> bool:
    try:
        modules()
        return True
    except ImportError:
        return False


def telescope(sutra, ctx, tel):
    sp = tel.spupil.astype(np.float32)
    return sutra.Telescope(ctx, sp.shape[0], int(np.where(sp > 0)[0].size), sp, tel.mpupil.shape[0],
                           tel.mpupil.astype(np.float32))


def initgs(sensors, n, lam, mag, noise=-1.0, seed=1234):
    one = lambda v, t=np.float32: np.array([v], dtype=t)  # noqa: E731
    sensors.initgs(one(0.0), one(0.0), one(lam), one(mag), 1e11, one(n, np.int64), one(noise),
                   one(seed, np.int64), one(1.0), one(0.0), one(0.0), one(0.0))


def sh_sensors(sutra, ctx, tel, g, noise=-1.0, seed=1234, mag=8.0):
    """SutraSensors with one SH sensor of geometry ``g`` (wfs_init.py:100-234)."""
    i64 = lambda v: np.array([v], dtype=np.int64)  # noqa: E731
    f32 = lambda v: np.array([v], dtype=np.float32)  # noqa: E731
    sensors = sutra.Sensors(ctx, tel, ["sh"], 1, i64(g.nxsub), i64(g.nvalid), i64(1), i64(g.npix), i64(g.pdiam),
                            i64(g.nrebin), i64(g.nfft), i64(g.ntot), i64(g.tel.n), f32(g.subapd), f32(g.nphotons),
                            f32(g.nphotons), np.zeros(1, np.int32), np.zeros(1, bool), np.zeros(1, np.int32),
                            np.zeros(1, np.int32), ctx.active_device, False)
    initgs(sensors, g.tel.n, g.wavelength_um, mag, noise, seed)
    wfs = sensors.d_wfs[0]
    kernel = np.zeros((g.ntot, g.ntot), np.complex64)  # used only by the kernel convolution (off)
    wfs.load_arrays(g.phasemap, g.hrmap, g.binmap, g.halfxy, g.fluxPerSub, g.validsubsx, g.validsubsy,
                    g.validpuppixx, g.validpuppixy, g.ttprojmat, kernel)
    if getattr(g, "submask", None) is not None:  # wfs_init.py:233-234
        sensors.set_field_stop(0, g.submask.astype(np.float32), g.submask.shape[0])
    return sensors, wfs


def add_centroider(ctx, rtc, wfs, g, kind, threshold=0.0, weights=None):
    rtc.add_centroider(ctx, g.nvalid, g.npix // 2.0 - 0.5, g.pixsize, False, ctx.active_device, kind, wfs)
    ce = rtc.d_centro[-1]
    ce.load_validpos(g.validsubsx, g.validsubsy, g.nvalid)
    ce.set_npix(g.npix)
    if kind in ("tcog", "wcog"):
        ce.set_threshold(float(threshold))
    if kind == "wcog":
        ce.init_weights()
        ce.load_weights(weights, weights.ndim)
    return ce


def add_ls(ctx, rtc, nslope, cmat, gain, delay=0.0):
    nactu = cmat.shape[0]
    rtc.add_controller(ctx, "ls", ctx.active_device, float(delay), nslope, nactu,
                       idx_centro=np.zeros(1, np.int32), ncentro=1)
    c = rtc.d_control[-1]
    c.set_cmat(cmat)
    c.set_gain(float(gain))
    c.set_modal_gains(np.ones(nactu, np.float32))
    return c


class RefShLoop:
    """One SH RTC loop on the reference's own GPU code: sensor, one centroider,
    LS controller; ``step(phase)`` runs one supervisor-order iteration and returns
    the voltages on the host."""

    def __init__(self, g, cmat, kind="wcog", threshold=0.0, weights=None, noise=-1.0, seed=1234, gain=0.4):
        carma, sutra = modules()
        self.ctx = carma.context.get_instance_1gpu(0)
        self.tel = telescope(sutra, self.ctx, g.tel)
        self.sensors, self.wfs = sh_sensors(sutra, self.ctx, self.tel, g, noise=noise, seed=seed)
        self.rtc = sutra.Rtc_FFF()
        add_centroider(self.ctx, self.rtc, self.wfs, g, kind, threshold, weights)
        self.control = add_ls(self.ctx, self.rtc, 2 * g.nvalid, cmat, gain)
        self.noise = noise > -1

    def step(self, phase):
        self.wfs.d_gs.set_phase(phase)
        self.wfs.comp_image(self.noise)
        self.rtc.do_centroids(0)
        self.rtc.do_control(0)
        self.rtc.comp_voltage(0)
        return np.array(self.control.d_voltage)

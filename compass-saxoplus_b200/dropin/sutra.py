"""Drop-in `sutra` module for COMPASS's shesha: the hot-path classes of the
reference's pybind11 `sutra` module (python_module/sutra/src/sutra.cpp:62-103)
with their names, constructor arguments and method names, over libaob200.

Covered (the calls shesha's supervisor makes on the RTC path):

* ``Sensors`` (sensors.cpp:28-107, initgs :159-191, set_field_stop :200-210)
  holding Shack-Hartmann (``SHWFS``, wfs_sh.cpp:41-148) and pyramid
  (``PYRWFS``, wfs_pyrhr.cpp:131-163) sensors: ``load_arrays``,
  ``comp_image``, ``slopes_geom`` (wfs.cpp:242-262), ``set_noise``,
  ``set_pupil``, ``set_binimg``, ``fill_binimage``, ``comp_nphot``,
  ``set_bincube``, ``set_dark`` / ``set_flat`` (SH camera), ``set_phalfxy`` /
  ``set_submask`` / ``set_pyrimg`` / ``compute_pyrfocalplane`` (pyramid),
  ``d_binimg`` / ``d_bincube`` / ``d_binmap`` / ``d_intensities`` /
  ``d_slopes`` / ``d_validsubsx`` / ``d_validsubsy`` /
  ``d_pyrfocalplane`` / ``d_gs.d_phase.d_screen``, ``d_gs.add_layer``;
* ``Dms`` / ``Dm`` (dms.cpp:120-600) for piezo-stack DMs: ``add_dm``,
  ``pzt_loadarrays``, ``set_com``, ``comp_shape``, ``comp_oneactu``,
  ``reset_shape``, ``d_shape`` / ``d_com``;
* ``Rtc_FFF`` (rtc.cpp:100-485): ``add_centroider`` (cog, tcog, wcog, bpcog,
  pyr, maskedpix), ``add_controller`` (ls, generic), ``do_imat`` (one batched
  push-pull evaluation per DM), ``do_centroids``, ``do_control``, ``apply_control``,
  ``comp_voltage``, ``do_clipping``, ``set_gain``, ``set_modal_gains``,
  ``imat_svd``, ``build_cmat``, ``set_centroids_ref``, ``do_calibrate_img``,
  ``d_centro`` / ``d_control``;
* ``Rtc_UFF``, the camera path: centroiders that load uint16 frames (a
  sensor's ``d_camimg`` under ``fakecam``) and calibrate them with dark, flat and
  a pixel look-up table (``set_lutPix``, ``calibrate_img_validPix``);
* the centroiders (centroider.cpp:83-352), the LS controller (controller.cpp,
  controller_ls.cpp) and the generic controller (controller_generic.cpp) with
  their ``d_*`` buffers and setters.

Errors raise ``aob200._lib.AobError`` with the library's message, where the
reference raises ``RuntimeError`` from its C++ layer.  Everything else of the
reference (atmosphere, targets, other DM, sensor and controller families) is
not part of this path; ``aob200.optics`` / ``aob200.turbulence`` have the
layers and targets the closed-loop tests use.
"""

from __future__ import annotations

import os
import sys

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if _PKG not in sys.path:
    sys.path.insert(0, _PKG)

from aob200 import core as _core  # noqa: E402


def _arr(a, n=None):
    a = np.asarray(a)
    return a.ravel() if n is None else a.ravel()[:n]


# ---------------------------------------------------------------------------
class _Phase:
    """``wfs.d_gs.d_phase``: the guide-star phase screen (``d_screen``)."""

    def __init__(self, wfs):
        self._w = wfs

    @property
    def d_screen(self):
        return self._w.d_phase


class _GuideStar:
    """``wfs.d_gs``: the guide star's phase and the DM layers it sees
    (SutraSource::add_layer, source.cpp; the offsets shesha's wfs_init gives)."""

    def __init__(self, wfs, lambda_um):
        self.d_phase = _Phase(wfs)
        self.Lambda = float(lambda_um)
        self.dm_layers = {}  # DM index -> (xoff, yoff) on the sensor's phase grid

    def add_layer(self, type, idx, xoff, yoff):
        if str(type) in ("pzt", "tt", "kl"):
            self.dm_layers[int(idx)] = (float(xoff), float(yoff))
        return 0


class _WfsBase:
    """Properties shared by the sensor wrappers (wfs.cpp:54-225)."""

    def __init__(self, impl, kind):
        self._w = impl
        self.type = kind
        self.d_gs = None

    nvalid = property(lambda self: self._w.nvalid)
    npix = property(lambda self: self._w.npix)
    nfft = property(lambda self: self._w.nfft)
    ntot = property(lambda self: self._w.ntot)
    nphase = property(lambda self: self._w.nphase)
    nrebin = property(lambda self: self._w.nrebin)
    nxsub = property(lambda self: self._w.nxsub)
    nphot = property(lambda self: self._w.nphot)
    noise = property(lambda self: self._w.noise)
    d_binimg = property(lambda self: self._w.d_binimg)
    d_validsubsx = property(lambda self: self._w.buffer("validsubsx", np.int32))
    d_validsubsy = property(lambda self: self._w.buffer("validsubsy", np.int32))
    d_fluxPerSub = property(lambda self: self._w.buffer("fluxPerSub"))

    d_slopes = property(lambda self: self._w.buffer("slopes"))

    def comp_image(self, noise=True):
        self._w.comp_image(noise=bool(noise))

    def slopes_geom(self, *args, **kw):
        """slopes_geom(type=0) into d_slopes, or slopes_geom(slopes, type=0) into the
        given float32 host array (wfs.cpp:242-262): 0 edge differences, 1 derivative
        weighted by the pupil, 2 tip/tilt projection."""
        slopes = kw.pop("slopes", None)
        if args and isinstance(args[0], np.ndarray):
            slopes, args = args[0], args[1:]
        t = int(args[0]) if args else int(kw.pop("type", 0))
        self._w.slopes_geom(t)
        if slopes is not None:
            slopes[...] = np.array(self.d_slopes).reshape(slopes.shape, order="F")
        return 0

    def set_binimg(self, binimg, nElem):
        a = np.asarray(binimg, np.float32)
        if a.size != int(nElem):
            raise ValueError("set_binimg: nElem does not match the array")
        self._w.set_binimg(a)
        return 0

    def set_noise(self, noise, seed):
        self._w.set_noise(float(noise), int(seed))

    def set_pupil(self, pupil):
        self._w.set_pupil(np.asarray(pupil, np.float32))


class SHWFS(_WfsBase):
    """SutraWfsSH (wfs_sh.cpp:41-148)."""

    def __init__(self, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npup, pdiam, nphot, nphot4imat, device):
        super().__init__(_core.ShWfs(nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npup, pdiam, nphot,
                                     nphot4imat, device=device), "sh")

    def load_arrays(self, phasemap, hrmap, binmap, offsets, fluxPerSub, validsubsx, validsubsy, istart, jstart,
                    ttprojmat=None, kernel=None):
        self._w.load_arrays(phasemap, hrmap, binmap, offsets, fluxPerSub, validsubsx, validsubsy, istart, jstart,
                            ttprojmat)

    d_bincube = property(lambda self: self._w.d_bincube)
    d_intensities = property(lambda self: self._w.d_intensities)
    d_binmap = property(lambda self: self._w.buffer("binmap", np.int32))
    d_validpuppixx = property(lambda self: self._w.buffer("istart", np.int32))
    d_validpuppixy = property(lambda self: self._w.buffer("jstart", np.int32))

    def fill_binimage(self, async_=False):
        self._w.fill_binimage()

    def comp_nphot(self, ittime, optthroughput, diam, nxsub, zerop=0, gsmag=0, lgsreturnperwatt=0, laserpower=0):
        """Photons per sub-aperture and frame (sutra_wfs_sh.cpp:645-663)."""
        if laserpower == 0:
            zp = 1e11 if zerop == 0 else float(zerop)
            nphot = zp * 10.0 ** (-0.4 * float(gsmag)) * ittime * optthroughput * (diam / nxsub) ** 2
        else:
            nphot = lgsreturnperwatt * laserpower * optthroughput * (diam / nxsub) ** 2 * 1e4 * ittime
        self._w.set_nphot(np.float32(nphot))
        return 0

    def set_bincube(self, bincube, nElem):
        a = np.asarray(bincube, np.float32)
        if a.size != int(nElem):
            raise ValueError("set_bincube: nElem does not match the array")
        self._w.set_bincube(a)
        return 0

    # fakecam (Sensors(..., fakecam, max_flux_per_pix, max_pix_value)): the uint16 frame
    d_camimg = property(lambda self: self._w.d_camimg)

    def set_dark(self, dark, n):
        self._w.set_dark(np.asarray(dark, np.float32), int(n))

    def set_flat(self, flat, n):
        self._w.set_flat(np.asarray(flat, np.float32), int(n))


class PYRWFS(_WfsBase):
    """SutraWfs_PyrHR (wfs_pyrhr.cpp:131-163); npup here is the reference's number of
    modulation points (its constructor's npup)."""

    def __init__(self, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts, pdiam, nphot, nphot4imat, device):
        super().__init__(_core.PyrWfs(nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts, pdiam, nphot, nphot4imat,
                                      device=device), "pyrhr")

    def load_arrays(self, halfxy, cx, cy, weights, sincar, submask, validsubsx, validsubsy, phasemap=None,
                    fluxPerSub=None, ttprojmat=None):
        self._w.load_arrays(halfxy, cx, cy, weights, sincar, submask, validsubsx, validsubsy, phasemap, fluxPerSub,
                            ttprojmat)
        self._compute_focal = False

    def set_pyr_modulation_points(self, cx, cy, weights=None, npts=None):
        self._w.set_modulation(cx, cy, weights)

    d_submask = property(lambda self: self._w.buffer("submask", shape=(self._w.nfft, self._w.nfft)))
    d_hrimg = property(lambda self: self._w.buffer("hrimg", shape=(self._w.nfft, self._w.nfft)))
    d_pyrfocalplane = property(lambda self: self._w.buffer("pyrfocalplane", shape=(self._w.nfft, self._w.nfft)))

    @property
    def d_phalfxy(self):
        a = self._w.buffer("phalfxy")
        n = self._w.nfft
        return _core.DeviceArray(a.ptr, n * n, np.complex64, (n, n), owner=a)

    @property
    def compute_pyrfocalplane(self):
        return getattr(self, "_compute_focal", False)

    @compute_pyrfocalplane.setter
    def compute_pyrfocalplane(self, on):
        """When set, every comp_image also forms d_pyrfocalplane (wfs_pyrhr.cpp:83-90)."""
        self._compute_focal = bool(on)
        self._w.set_compute_focalplane(bool(on))

    def set_phalfxy(self, phalfxy):
        """The pyramid mask exp(i phase), nfft x nfft complex64 (wfs_pyrhr.cpp:235-242)."""
        self._w.set_phalfxy(phalfxy)
        return 0

    def set_submask(self, submask):
        self._w.set_submask(np.asarray(submask, np.float32))
        return 0

    def set_pyrimg(self, img):
        self._w.set_binimg(np.asarray(img, np.float32))
        return 0

    def comp_nphot(self, ittime, optthroughput, diam, cobs, zerop=0, gsmag=0):
        """Photons per frame over the pupil (sutra_wfs_pyr_pyrhr.cpp:722-729)."""
        nphot = zerop * 10.0 ** (-0.4 * gsmag) * ittime * optthroughput * np.pi / 4.0 * (1 - cobs * cobs) * diam * diam
        self._w.set_nphot(np.float32(nphot))
        return 0


class Sensors:
    """SutraSensors (sensors.cpp:28-107): one sensor per entry of ``type``."""

    def __init__(self, context, d_tel, type, nwfs, nxsub, nvalid, npupils, npix, nphase, nrebin, nfft, ntot, npup,
                 pdiam, nphot, nphot4imat, lgs, fakecam, max_flux_per_pix, max_pix_value, device, roket):
        self.device = int(device)
        self._wfs = []
        for i in range(int(nwfs)):
            args = (int(_arr(nxsub)[i]), int(_arr(nvalid)[i]), int(_arr(npix)[i]), int(_arr(nphase)[i]),
                    int(_arr(nrebin)[i]), int(_arr(nfft)[i]), int(_arr(ntot)[i]), int(_arr(npup)[i]),
                    float(_arr(pdiam)[i]), float(_arr(nphot)[i]), float(_arr(nphot4imat)[i]), self.device)
            if type[i] == "sh":
                self._wfs.append(SHWFS(*args))
                if bool(_arr(fakecam)[i]):
                    self._wfs[-1]._w.set_fakecam(True, int(_arr(max_flux_per_pix)[i]), int(_arr(max_pix_value)[i]))
            elif type[i] == "pyrhr":
                self._wfs.append(PYRWFS(*args))
            else:
                raise ValueError(f"Sensors: sensor type {type[i]!r} is not supported (sh, pyrhr)")

    @property
    def d_wfs(self):
        return self._wfs

    def set_field_stop(self, nwfs, field_stop, N):
        """SutraSensors::set_field_stop (sensors.cpp:200-210): SH sensors only."""
        w = self.d_wfs[int(nwfs)]
        if isinstance(w, SHWFS):
            w._w.set_field_stop(np.asarray(field_stop, np.float32).reshape(int(N), int(N)))
        return 0

    def initgs(self, xpos, ypos, lambda_um, mag, zerop, sizes, noise, seeds, G, thetaML, dx, dy):
        """Guide stars (sensors.cpp:159-191): wavelength, noise level and noise seed per sensor."""
        for i, w in enumerate(self._wfs):
            w._w.set_lambda(float(_arr(lambda_um)[i]))
            w._w.set_noise(float(_arr(noise)[i]), int(_arr(seeds)[i]))
            w.d_gs = _GuideStar(w._w, float(_arr(lambda_um)[i]))
        return 0


# ---------------------------------------------------------------------------
class Dm:
    """SutraDm of the piezo-stack type (python_module/sutra/src/dms.cpp:270-600):
    the command vector, the shape on its dim x dim support and the single-actuator
    poke that do_imat uses."""

    def __init__(self, type, alt, dim, nactus, influsize, push4imat, device):
        if type != "pzt":
            raise ValueError(f"add_dm: DM type {type!r} is not supported (pzt)")
        self.type, self.altitude = type, float(alt)
        self.dim, self.nactus, self.influsize = int(dim), int(nactus), int(influsize)
        self.push4imat = float(push4imat)
        self.device = int(device)
        self._d = None
        self._one = None

    def _need(self):
        if self._d is None:
            raise ValueError("Dm: pzt_loadarrays has not been called")
        return self._d

    def pzt_loadarrays(self, influ, influpos, npoints, istart, xoff, yoff):
        """The influence functions [influsize, influsize, nactus] and each
        actuator's corner (xoff, yoff) on the support, as dm_init.py:186-193 passes
        them; influpos / npoints / istart (the reference's pixel lists) are
        rebuilt from these by the library."""
        from aob200 import optics

        influ = np.asarray(influ, np.float32)
        i1, j1 = np.asarray(xoff, np.int64), np.asarray(yoff, np.int64)
        # comp_dmgeom (dm_init.py:902-955) places actuator a's sample (x, y) at
        # screen pixel (offs + i1[a] + x) + dim (offs + j1[a] + y), offs > 0 when
        # the DM support is smaller than the screen: read offs off the first
        # listed sample
        off = 0
        npts, ist, pos = np.asarray(npoints), np.asarray(istart), np.asarray(influpos)
        nz = np.flatnonzero(npts[: self.dim * self.dim]) if npts.size else np.empty(0, np.int64)
        if nz.size:
            p = int(nz[0])
            q = int(pos[int(ist[p])])
            s = influ.shape[0]
            a, y, x = q // (s * s), (q // s) % s, q % s
            off = p % self.dim - x - int(i1[a])
            if p // self.dim - y - int(j1[a]) != off:
                raise ValueError("pzt_loadarrays: influpos does not match xoff / yoff")
        self._d = optics.Dm(self.dim, influ, i1 + off, j1 + off, device=self.device)
        return 0

    @property
    def d_shape(self):
        return self._need().d_shape

    @property
    def d_com(self):
        return self._need().buffer("com")

    def set_com(self, com, shape_dm=True):
        self._need().set_com(np.asarray(com, np.float32))
        if shape_dm:
            self.comp_shape()
        return 0

    def comp_shape(self, com=None):
        d = self._need()
        if com is not None:
            d.set_com(np.asarray(com, np.float32))
        d.comp_shape()
        return 0

    def reset_shape(self):
        self._need()
        self.d_shape.set(np.zeros((self.dim, self.dim), np.float32))
        return 0

    def comp_oneactu(self, nactu, ampli):
        """The shape of actuator ``nactu`` alone at ``ampli`` volts; d_com is left as it is."""
        d = self._need()
        if self._one is None:
            self._one = _core.OwnedDeviceArray(self.nactus, np.float32, device=self.device)
        v = np.zeros(self.nactus, np.float32)
        v[int(nactu)] = ampli
        self._one.set(v)
        d.comp_shape(self._one.ptr)
        return 0


class Dms:
    """SutraDms (dms.cpp:120-260): the list of DMs."""

    def __init__(self):
        self._dms = []

    @property
    def d_dms(self):
        return self._dms

    def add_dm(self, context, type, alt, dim, nactus, influsize, ninflupos, n_npoints, push4imat, nord, *rest):
        """Both reference overloads: (..., nord, device) and (..., nord, dx, dy,
        thetaML, G, device); only a registration of dx = dy = thetaML = 0, G = 1 is
        supported."""
        if len(rest) == 5:
            dx, dy, theta, G, device = rest
            if (dx, dy, theta, G) != (0, 0, 0, 1):
                raise ValueError("add_dm: DM mis-registration is not supported")
        elif len(rest) == 1:
            (device,) = rest
        else:
            raise TypeError("add_dm: expected (..., nord, device) or (..., nord, dx, dy, thetaML, G, device)")
        self._dms.append(Dm(type, alt, dim, nactus, influsize, push4imat, device))
        return 0

    def remove_dm(self, idx):
        del self._dms[int(idx)]
        return 0


# ---------------------------------------------------------------------------
class Centroider:
    """SutraCentroider{Cog,Tcog,Wcog,Pyr} (centroider.cpp:83-352)."""

    def __init__(self, nvalid, offset, scale, typec, device, wfs=None, tin=np.float32):
        self._tin = tin  # image type of load_img: float32 (Rtc_FFF) or uint16 (Rtc_UFF)
        if typec == "maskedpix" and wfs is not None:
            nvalid = 4 * wfs._w.nvalid  # one slope per valid pixel (maskedPix.cpp:35-36)
        self._c = _core.Centroider(int(nvalid), float(offset), float(scale), typec, device=int(device))
        self.type = typec
        self.device = int(device)
        self.offset, self.scale = float(offset), float(scale)
        self.npix = 0
        self.threshold = 0.0
        self.nmax = 0
        self.wfs = wfs
        self._img_shape = None  # (m, n) of the loaded image (the carma objects are 2-D)
        self._raw_dtype = np.float32  # type of the loaded frame
        if wfs is not None:
            self._c.attach(wfs._w)

    nvalid = property(lambda self: self._c.nvalid)
    nslopes = property(lambda self: self._c.nslopes)
    d_dark = property(lambda self: self._c.buffer("dark", shape=self._img_shape))
    d_flat = property(lambda self: self._c.buffer("flat", shape=self._img_shape))
    d_img = property(lambda self: self._c.buffer("img", shape=self._img_shape))
    d_img_raw = property(lambda self: self._c.buffer("img_raw", dtype=self._raw_dtype, shape=self._img_shape))
    d_centroids_ref = property(lambda self: self._c.buffer("centroids_ref"))
    d_intensities = property(lambda self: self._c.buffer("intensities"))
    d_validx = property(lambda self: self._c.buffer("validx", np.int32))
    d_validy = property(lambda self: self._c.buffer("validy", np.int32))
    d_weights = property(lambda self: self._c.buffer("weights"))

    def get_cog(self):
        """Centroids of the sensor's current image into its d_slopes (centroider.cpp:186-188)."""
        if self.wfs is None:
            raise ValueError("get_cog: the centroider has no sensor (use Rtc.do_centroids)")
        self._c.get_cog(self.wfs._w.buffer("slopes").ptr)
        return 0

    def load_validpos(self, validx, validy, N):
        self._c.load_validpos(_arr(validx, int(N)), _arr(validy, int(N)))

    def set_npix(self, npix):
        self.npix = int(npix)
        self._c.set_npix(int(npix))

    def set_scale(self, scale):
        self.scale = float(scale)
        self._c.set_scale(float(scale))

    def set_offset(self, offset):
        self.offset = float(offset)
        self._c.set_offset(float(offset))

    def set_threshold(self, threshold):
        self.threshold = float(threshold)
        self._c.set_threshold(float(threshold))

    def set_nmax(self, nmax):
        """bpCoG (centroider_bpcog.cpp): rank of the threshold pixel."""
        self.nmax = int(nmax)
        self._c.set_nmax(int(nmax))

    def init_weights(self):
        """wCoG (centroider_wcog.cpp:61-62): the weights are allocated by load_weights."""
        return 0

    def set_pyr_method(self, method):
        """Pyramid slopes as the reference's Method_CoG decodes them (sutra_centroider_pyr.hpp:27-34):
        0 sinus global, 1 nosinus global (default), 2 sinus local, 3 nosinus local."""
        self._c.set_pyr_method(int(method))

    def set_pyr_thresh(self, thresh):
        self._c.set_pyr_thresh(float(thresh))

    def load_weights(self, weights, ndim):
        self._c.load_weights(np.asarray(weights, np.float32), int(ndim))

    def set_centroids_ref(self, refslopes):
        self._c.set_centroids_ref(np.asarray(refslopes, np.float32))

    def load_img(self, img, *args):
        """A frame from the host (cast to the RTC's input type, as the reference's
        pybind11 binding does) or, for a uint16 RTC, a uint16 device array such as
        a sensor's ``d_camimg``."""
        if isinstance(img, _core.DeviceArray):
            self._img_shape = tuple(img.shape)
            self._raw_dtype = img.dtype
            self._c.load_img(img)
            return 0
        img = np.asarray(img, self._tin)
        self._img_shape = img.shape if img.ndim == 2 else None
        self._raw_dtype = img.dtype
        self._c.load_img(img)
        return 0

    def calibrate_img_validPix(self):
        self._c.calibrate_img_validpix()
        return 0

    def set_lutPix(self, lutPix, n=None):
        self._c.set_lut_pix(np.asarray(lutPix, np.int32))
        return 0

    def calibrate_img(self):
        self._c.calibrate_img()

    def set_dark(self, dark, n):
        self._img_shape = self._img_shape or (int(n), int(n))
        self._c.set_dark(np.asarray(dark, np.float32), int(n))

    def set_flat(self, flat, n):
        self._img_shape = self._img_shape or (int(n), int(n))
        self._c.set_flat(np.asarray(flat, np.float32), int(n))


class _Controller:
    """SutraController (controller.cpp:65-330): the buffers, delay ring,
    perturbation voltages, clip and comp_voltage common to every controller."""

    _kind = "ls"

    def __init__(self, nslope, nactu, delay, device):
        self._l = _core.LsController(int(nslope), int(nactu), delay=float(delay), device=int(device), kind=self._kind)
        self.type = self._kind
        self.nslope, self.nactu = int(nslope), int(nactu)
        self.delay = float(delay)
        self.gain = 0.0
        self.comRange = (-1.0e6, 1.0e6)
        self.centro_idx = []
        self._perturb = {}  # name -> (voltages, counter, enabled)
        self._perturb_n = {}  # name -> number of rows

    d_centroids = property(lambda self: self._l.buffer("centroids"))
    d_com = property(lambda self: self._l.buffer("com"))
    d_com_clipped = property(lambda self: self._l.buffer("com_clipped"))
    d_voltage = property(lambda self: self._l.buffer("voltage"))
    d_err = property(lambda self: self._l.buffer("err"))
    d_cmat = property(lambda self: self._l.buffer("cmat", shape=(self.nactu, self.nslope)))
    d_imat = property(lambda self: self._l.buffer("imat", shape=(self.nslope, self.nactu)))
    d_gain = property(lambda self: self._l.buffer("gain"))
    d_circularComs0 = property(lambda self: self._l.buffer("com0"))
    d_circularComs1 = property(lambda self: self._l.buffer("com1"))

    @property
    def d_perturb_map(self):
        """name -> (perturbation voltages [N, nactu], counter, enabled), as the reference's map."""
        return dict(self._perturb)

    def set_cmat(self, cmat):
        self._l.set_cmat(np.asarray(cmat, np.float32))

    def set_imat(self, imat):
        self._l.set_imat(np.asarray(imat, np.float32))

    def set_gain(self, gain):
        self.gain = float(gain)
        self._l.set_gain(float(gain))

    def set_modal_gains(self, mgain):
        self._l.set_modal_gains(np.asarray(mgain, np.float32))

    def set_delay(self, delay):
        self.delay = float(delay)
        self._l.set_delay(float(delay))

    def set_com(self, com, nElem=None):
        self._l.set_com(np.asarray(com, np.float32))

    def set_comRange(self, comMin, comMax):
        self.comRange = (comMin, comMax)
        self._l.set_com_range(float(comMin), float(comMax))

    def set_open_loop(self, open_loop, reset=True):
        self._l.set_open_loop(bool(open_loop), bool(reset))

    def _advance_perturb(self):
        for k, (a, cpt, on) in self._perturb.items():
            if on:
                self._perturb[k] = (a, (cpt + 1) % self._perturb_n[k], on)

    def comp_voltage(self):
        self._l.comp_voltage()
        self._advance_perturb()

    def clip_commands(self):
        self._l.clip()

    def add_perturb(self):
        """com_clipped += the current row of every enabled perturbation (controller.cpp add_perturb)."""
        self._l.apply_perturb()
        self._advance_perturb()

    def add_perturb_voltage(self, name, perturb, N):
        a = np.array(perturb, np.float32)
        self._l.add_perturb(name, a, int(N))
        self._perturb[name] = (a, 0, True)
        self._perturb_n[name] = int(N)

    def remove_perturb_voltage(self, name):
        self._l.remove_perturb(name)
        self._perturb.pop(name, None)
        self._perturb_n.pop(name, None)

    def enable_perturb_voltage(self, name):
        self._l.enable_perturb(name, True)
        a, cpt, _ = self._perturb[name]
        self._perturb[name] = (a, cpt, True)

    def disable_perturb_voltage(self, name):
        self._l.enable_perturb(name, False)
        a, cpt, _ = self._perturb[name]
        self._perturb[name] = (a, cpt, False)

    def reset_perturb_voltage(self):
        self._l.reset_perturb()
        self._perturb, self._perturb_n = {}, {}


class ControllerLS(_Controller):
    """SutraControllerLs (controller_ls.cpp)."""

    _kind = "ls"
    d_eigenvals = property(lambda self: self._l.buffer("eigenvals"))


class ControllerGENERIC(_Controller):
    """SutraControllerGeneric (controller_generic.cpp): command laws integrator
    (leaky factor, pseudo-open-loop slopes), modal_integrator and 2matrices."""

    _kind = "generic"

    def set_commandlaw(self, law):
        self._l.set_commandlaw(str(law))

    @property
    def command_law(self):
        return self._l.law()["law"]

    def set_leaky_factor(self, factor):
        self._l.set_leaky_factor(float(factor))

    def set_polc(self, polc):
        self._l.set_polc(bool(polc))

    def set_decayFactor(self, decay):
        self._l.set_decay_factor(np.asarray(decay, np.float32))

    def set_matE(self, matE):
        self._l.set_matE(np.asarray(matE, np.float32))


class Rtc_FFF:
    """SutraRtc<float, float, float> (rtc.cpp:100-485).  A controller reads the
    slopes of the centroiders listed in its ``centro_idx`` (all of them, in
    order, by default), one block of 2 nvalid after the other."""

    _tin = np.float32  # image type the centroiders load

    def __init__(self):
        self.d_centro = []
        self.d_control = []

    def add_centroider(self, context, nvalid, offset, scale, filter_TT, device, typec, wfs=None):
        if typec not in ("cog", "tcog", "wcog", "bpcog", "pyr", "maskedpix"):
            raise ValueError(f"add_centroider: centroider type {typec!r} is not supported "
                             "(cog, tcog, wcog, bpcog, pyr, maskedpix)")
        self.d_centro.append(Centroider(nvalid, offset, scale, typec, device, wfs, tin=self._tin))
        return 0

    def add_controller(self, context, typec, device, delay, nslope, nactu, nslope_buffers=0, nstates=0,
                       nstate_buffers=0, nmodes=0, niir_in=0, niir_out=0, polc=False, is_modal=False, dms=None,
                       idx_dms=None, ndm=0, idx_centro=None, ncentro=0, Nphi=0, wfs_direction=False):
        if typec not in ("ls", "generic"):
            raise ValueError(f"add_controller: controller type {typec!r} is not supported (ls, generic)")
        c = (ControllerLS if typec == "ls" else ControllerGENERIC)(nslope, nactu, delay, device)
        c.centro_idx = ([int(i) for i in _arr(idx_centro)][: int(ncentro)] if idx_centro is not None and ncentro
                        else list(range(len(self.d_centro))))
        # the DMs the controller drives (d_dmseen): indexes into ``dms``
        c.dm_idx = ([int(i) for i in _arr(idx_dms)][: int(ndm)] if idx_dms is not None and ndm else None)
        self.d_control.append(c)
        return 0

    def do_imat(self, ncontrol, dms, kernconv=False):
        """Push-pull interaction matrix (sutra_rtc.cpp:150-292): every actuator of
        every DM the controller drives, pushed and pulled by its push4imat, seen
        by the controller's SH sensors (noise-free, nphot4imat photons), the
        slopes (s_push - s_pull) / (2 push) as the columns of the controller's
        d_imat.  All actuators of a DM go through one batched evaluation
        (aob_imat_build) per sensor."""
        from aob200._lib import call

        if kernconv:
            raise ValueError("do_imat: the spot convolution kernel is not supported")
        c = self.d_control[int(ncontrol)]
        if c._kind != "ls":
            raise ValueError("do_imat: the controller must be ls")
        seen = [dms.d_dms[i] for i in c.dm_idx] if c.dm_idx is not None else list(dms.d_dms)
        idx_of = {id(d): i for i, d in enumerate(dms.d_dms)}
        if sum(d.nactus for d in seen) != c.nactu:
            raise ValueError("do_imat: the DMs' actuators do not add up to the controller's nactu")
        imat = np.zeros((c.nslope, c.nactu), np.float32)
        a0 = 0
        for dm in seen:
            d = dm._need()
            off = 0
            for i in c.centro_idx:
                cen = self.d_centro[i]
                ns = cen.nslopes
                w = cen.wfs
                if not isinstance(w, SHWFS):
                    raise ValueError("do_imat: only Shack-Hartmann sensors are supported")
                n = w._w.npup
                layer = w.d_gs.dm_layers.get(idx_of[id(dm)]) if w.d_gs is not None else None
                xoff, yoff = layer if layer is not None else ((dm.dim - n) / 2.0,) * 2
                cen._c.attach(w._w)
                tmp = _core.OwnedDeviceArray(ns * dm.nactus, np.float32, (ns, dm.nactus), device=dm.device)
                call("aob_imat_build", w._w.h, cen._c.h, d.h, float(xoff), float(yoff), float(dm.push4imat), 0,
                     tmp.ptr, None)
                imat[off:off + ns, a0:a0 + dm.nactus] = np.array(tmp)
                off += ns
            a0 += dm.nactus
        c.set_imat(imat)
        return 0

    def remove_controller(self, ncontrol):
        del self.d_control[int(ncontrol)]

    def remove_centroider(self, ncentro):
        del self.d_centro[int(ncentro)]

    def _slopes_of(self, ncontrol):
        c = self.d_control[int(ncontrol)]
        base = c.d_centroids
        off = 0
        for i in c.centro_idx:
            yield self.d_centro[i], base.ptr + 4 * off
            off += self.d_centro[i].nslopes

    def do_calibrate_img(self, ncontrol):
        for cen, _ in self._slopes_of(ncontrol):
            if cen.wfs is None:
                cen.calibrate_img()
        return 0

    def do_centroids(self, ncontrol):
        for cen, ptr in self._slopes_of(ncontrol):
            cen._c.get_cog(ptr)
        return 0

    def do_control(self, ncontrol):
        self.d_control[int(ncontrol)]._l.comp_com()
        return 0

    def comp_voltage(self, ncontrol):
        self.d_control[int(ncontrol)]._l.comp_voltage()
        return 0

    def apply_control(self, ncontrol, compVoltage=True):
        """The voltages of controller ``ncontrol`` (comp_voltage when asked); the DM
        shapes they drive are computed by the caller's DM objects."""
        if compVoltage:
            self.comp_voltage(ncontrol)
        return 0

    def do_clipping(self, ncontrol):
        self.d_control[int(ncontrol)]._l.clip()
        return 0

    def set_gain(self, ncontrol, gain):
        self.d_control[int(ncontrol)].set_gain(gain)
        return 0

    def set_modal_gains(self, ncontrol, mgain):
        self.d_control[int(ncontrol)].set_modal_gains(mgain)
        return 0

    def imat_svd(self, ncontrol):
        self.d_control[int(ncontrol)]._l.svdec_imat()
        return 0

    def build_cmat(self, ncontrol, nfilt, filt_tt=False):
        if filt_tt:
            raise ValueError("build_cmat: tip-tilt filtering is not supported")
        self.d_control[int(ncontrol)]._l.build_cmat(int(nfilt))
        return 0

    def set_centroids_ref(self, centroidsRef):
        ref = np.asarray(centroidsRef, np.float32).ravel()
        off = 0
        for cen in self.d_centro:
            n = cen.nslopes
            cen.set_centroids_ref(ref[off:off + n])
            off += n
        return 0


class Rtc_UFF(Rtc_FFF):
    """SutraRtc<uint16_t, float, float> (rtc.cpp; sutra.cpp:62-103): the camera
    path -- the centroiders load uint16 frames (load_img from the host or a
    sensor's d_camimg), calibrate them to float with dark, flat and the pixel
    look-up table, then compute as Rtc_FFF does."""

    _tin = np.uint16

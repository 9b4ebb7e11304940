"""Python objects over the C ABI: SH and pyramid sensors, centroider, LS controller.

These are the host-side mirror of the reference's SutraWfsSH /
SutraCentroider* / SutraControllerLs (see include/aob200.h for the file:line
of each replaced interface).  Host arrays follow the reference's convention:
numpy arrays indexed [x, y] with x the fastest device index (Fortran order).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import addr, call, d2h, h2d, host_array

CENTRO_TYPES = {"cog": 0, "tcog": 1, "wcog": 2, "pyr": 3, "pyrhr": 3, "maskedpix": 4, "bpcog": 5}
COMMAND_LAWS = {"integrator": 1, "modal_integrator": 2, "2matrices": 3}
PRECISIONS = {"f32": 0, "fp32": 0, "float32": 0, "bf16": 1, "bfloat16": 1, "fp8": 2, "e4m3": 2}


def _device_ok() -> bool:
    """True when a synchronisation of the legacy default stream succeeds (a
    sticky CUDA error makes it fail)."""
    try:
        call("aob_stream_sync", None)
        return True
    except _lib.AobError:
        return False


class DeviceArray:
    """View of a device buffer owned by the library (the carma object role).

    ``np.array(obj)`` / ``obj.host()`` copy it to the host, reshaped to
    ``shape`` in Fortran order like the reference's carma arrays.
    """

    def __init__(self, ptr: int, n: int, dtype, shape=None, owner=None):
        self.ptr = int(ptr or 0)
        self.n = int(n)
        self.dtype = np.dtype(dtype)
        self.shape = tuple(shape) if shape is not None else (self.n,)
        self._owner = owner

    def host(self) -> np.ndarray:
        if self.ptr == 0 or self.n == 0:
            return np.zeros(self.shape, dtype=self.dtype)
        return d2h(self.ptr, self.n, self.dtype).reshape(self.shape, order="F")

    def __array__(self, dtype=None, copy=None):
        a = self.host()
        return a.astype(dtype) if dtype is not None else a

    def set(self, a) -> None:
        a = host_array(a, self.dtype)
        if a.size != self.n:
            raise ValueError(f"size mismatch: {a.size} != {self.n}")
        h2d(self.ptr, a)

    def get_dims(self):
        return self.shape

    @property
    def __cuda_array_interface__(self):
        """The buffer as a CUDA array (Fortran order, no copy), e.g. for
        ``torch.as_tensor(buf, device="cuda")``."""
        st, acc = [], self.dtype.itemsize
        for d in self.shape:
            st.append(acc)
            acc *= int(d)
        return {"shape": tuple(int(d) for d in self.shape), "typestr": self.dtype.str, "data": (self.ptr, False),
                "strides": tuple(st), "version": 3}


class OwnedDeviceArray(DeviceArray):
    """A device buffer allocated here (aob_malloc) and freed with the object."""

    def __init__(self, n: int, dtype=np.float32, shape=None, device=0):
        p = ctypes.c_void_p()
        nbytes = max(int(n), 1) * np.dtype(dtype).itemsize
        call("aob_malloc", ctypes.addressof(p), nbytes, int(device))
        super().__init__(p.value, n, dtype, shape)
        call("aob_memcpy_h2d", self.ptr, np.zeros(nbytes, np.uint8).ctypes.data, nbytes, None)

    def __del__(self):
        try:
            if self.ptr and _lib._lib is not None:
                _lib.lib().aob_free(ctypes.c_void_p(self.ptr))
        except (AttributeError, TypeError):  # interpreter shutdown
            pass
        self.ptr = 0

    def __len__(self):
        return self.shape[0]


def _buffer(fn: str, handle, which: str, dtype, shape=None, owner=None) -> DeviceArray:
    p = ctypes.c_void_p()
    n = ctypes.c_int64()
    call(fn, handle, which.encode(), ctypes.addressof(p), ctypes.addressof(n))
    if shape is not None and int(np.prod(shape)) != n.value:
        shape = None
    return DeviceArray(p.value or 0, n.value, dtype, shape, owner)


class ShWfs:
    """Shack-Hartmann sensor on one GPU (SutraWfsSH)."""

    def __init__(self, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npup, pdiam, nphot,
                 nphot4imat=0.0, device=0, lambda_um=0.5):
        self.h = ctypes.c_void_p()
        call("aob_sh_create", ctypes.addressof(self.h), int(device), int(nxsub), int(nvalid), int(npix),
             int(nphase), int(nrebin), int(nfft), int(ntot), int(npup), float(pdiam), float(nphot),
             float(nphot4imat))
        self.nxsub, self.nvalid, self.npix, self.nphase = int(nxsub), int(nvalid), int(npix), int(nphase)
        self.nrebin, self.nfft, self.ntot, self.npup = int(nrebin), int(nfft), int(ntot), int(npup)
        self.pdiam, self.nphot, self.nphot4imat = float(pdiam), float(nphot), float(nphot4imat)
        self.device = int(device)
        self.noise = -1.0
        self.lambda_um = float(lambda_um)
        call("aob_sh_set_lambda", self.h, float(lambda_um))

    @classmethod
    def from_geometry(cls, g, device=0, noise=-1.0, seed=1234):
        w = cls(g.nxsub, g.nvalid, g.npix, g.pdiam, g.nrebin, g.nfft, g.ntot, g.tel.n, g.subapd,
                g.nphotons, device=device, lambda_um=g.wavelength_um)
        w.load_arrays(g.phasemap, g.hrmap, g.binmap, g.halfxy, g.fluxPerSub, g.validsubsx, g.validsubsy,
                      g.validpuppixx, g.validpuppixy, g.ttprojmat)
        w.set_pupil(g.tel.mpupil)
        w.set_noise(noise, seed)
        if getattr(g, "submask", None) is not None:
            w.set_field_stop(g.submask)
        return w

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_sh_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def load_arrays(self, phasemap, hrmap, binmap, offsets, fluxPerSub, validsubsx, validsubsy,
                    istart, jstart, ttprojmat=None, kernel=None):
        i32, f32 = np.int32, np.float32
        keep = [host_array(binmap, i32), host_array(offsets, f32), host_array(fluxPerSub, f32),
                host_array(validsubsx, i32), host_array(validsubsy, i32), host_array(istart, i32),
                host_array(jstart, i32)]
        # hrmap is read when the field of view is extended (ntot != nfft)
        hr = host_array(hrmap, i32) if (hrmap is not None and self.ntot != self.nfft) else None
        # phasemap and ttprojmat are kept for the geometric slopes (slopes_geom)
        pm = host_array(phasemap, i32) if phasemap is not None else None
        tt = host_array(ttprojmat, f32) if ttprojmat is not None else None
        call("aob_sh_load_arrays", self.h, None if pm is None else pm.ctypes.data,
             None if hr is None else hr.ctypes.data, *[k.ctypes.data for k in keep],
             None if tt is None else tt.ctypes.data, None)

    def slopes_geom(self, type=0, dev_slopes=None, stream=None):
        """Geometric slopes of the phase (SutraWfs::slopes_geom): 0 edge
        differences, 1 pupil-weighted finite differences, 2 tip/tilt projection
        (needs ttprojmat).  Into ``dev_slopes`` or the sensor's "slopes" buffer."""
        call("aob_sh_slopes_geom", self.h, int(type), dev_slopes, stream)

    def set_pupil(self, pupil):
        a = host_array(pupil, np.float32)
        if a.size != self.npup * self.npup:
            raise ValueError("pupil must be npup x npup")
        call("aob_sh_set_pupil", self.h, a.ctypes.data)

    def set_fakecam(self, enable=True, max_flux_per_pix=0, max_pix_value=0):
        """Digitise every image into the uint16 frame ``d_camimg`` (fakecam)."""
        call("aob_sh_set_fakecam", self.h, 1 if enable else 0, int(max_flux_per_pix), int(max_pix_value))

    def set_dark(self, dark, n=None):
        a = host_array(dark, np.float32)
        call("aob_sh_set_dark", self.h, a.ctypes.data, int(np.sqrt(a.size)))

    def set_flat(self, flat, n=None):
        a = host_array(flat, np.float32)
        call("aob_sh_set_flat", self.h, a.ctypes.data, int(np.sqrt(a.size)))

    @property
    def d_camimg(self):
        side = self.npix * self.nxsub
        return self.buffer("camimg", dtype=np.uint16, shape=(side, side))

    def set_field_stop(self, mask):
        """Focal-plane field stop of the full pupil (n x n, fftshifted; None removes it)."""
        if mask is None:
            call("aob_sh_set_field_stop", self.h, None, 0)
            return
        m = np.asarray(mask)
        a = host_array(m, np.float32)
        call("aob_sh_set_field_stop", self.h, a.ctypes.data, int(m.shape[0]))

    def set_noise(self, noise, seed=1234):
        self.noise = float(noise)
        call("aob_sh_set_noise", self.h, float(noise), int(seed))

    def set_lambda(self, lam):
        self.lambda_um = float(lam)
        call("aob_sh_set_lambda", self.h, float(lam))

    def set_nphot(self, nphot):
        self.nphot = float(nphot)
        call("aob_sh_set_nphot", self.h, float(nphot))

    def set_bincube(self, cube):
        """Overwrite the sub-aperture images (npix x npix x nvalid, Fortran order)."""
        a = host_array(cube, np.float32)
        call("aob_sh_set_bincube", self.h, a.ctypes.data, int(a.size))

    def set_binimg(self, img):
        a = host_array(img, np.float32)
        call("aob_sh_set_binimg", self.h, a.ctypes.data, int(a.size))

    @property
    def frame(self) -> int:
        f = ctypes.c_uint64()
        call("aob_sh_get_frame", self.h, ctypes.addressof(f))
        return f.value

    @frame.setter
    def frame(self, v):
        call("aob_sh_set_frame", self.h, int(v))

    def buffer(self, which, dtype=np.float32, shape=None) -> DeviceArray:
        return _buffer("aob_sh_buffer", self.h, which, dtype, shape, self)

    @property
    def d_phase(self):
        return self.buffer("phase", shape=(self.npup, self.npup))

    @property
    def d_bincube(self):
        return self.buffer("bincube", shape=(self.npix, self.npix, self.nvalid))

    @property
    def d_binimg(self):
        n = self.npix * self.nxsub
        return self.buffer("binimg", shape=(n, n))

    @property
    def d_intensities(self):
        return self.buffer("intensities")

    def set_phase(self, phase):
        self.d_phase.set(phase)

    def comp_image(self, noise=True, stream=None):
        call("aob_sh_comp_image", self.h, 1 if noise else 0, stream)

    def fill_binimage(self, stream=None):
        call("aob_sh_fill_binimage", self.h, stream)

    def set_tuning(self, subaps_per_cta=0):
        """Sub-apertures per CTA batch of the sensor kernel (0 = heuristic); results are unchanged."""
        call("aob_sh_set_tuning", self.h, int(subaps_per_cta))


class PyrWfs:
    """High-resolution modulated pyramid sensor on one GPU (SutraWfs_PyrHR)."""

    def __init__(self, nxsub, nvalid, npix, nphase, nrebin, nfft, ntot, npts, pdiam, nphot,
                 nphot4imat=0.0, device=0, lambda_um=0.5):
        self.h = ctypes.c_void_p()
        call("aob_pyr_create", ctypes.addressof(self.h), int(device), int(nxsub), int(nvalid), int(npix),
             int(nphase), int(nrebin), int(nfft), int(ntot), int(npts), float(pdiam), float(nphot),
             float(nphot4imat))
        self.nxsub, self.nvalid, self.npix, self.nphase = int(nxsub), int(nvalid), int(npix), int(nphase)
        self.nrebin, self.nfft, self.ntot, self.npts = int(nrebin), int(nfft), int(ntot), int(npts)
        self.pdiam, self.nphot = float(pdiam), float(nphot)
        self.device = int(device)
        self.noise = -1.0
        self.lambda_um = float(lambda_um)
        call("aob_pyr_set_lambda", self.h, float(lambda_um))

    @classmethod
    def from_geometry(cls, g, device=0, noise=-1.0, seed=1234, weights=None):
        subapd = g.tel.diam / g.nxsub if g.tel is not None else float(g.pdiam)
        w = cls(g.nxsub, g.nvalid, g.npix, g.pdiam, g.nrebin, g.nfft, g.ntot, g.pyr_cx.size, subapd,
                g.nphotons, device=device, lambda_um=g.wavelength_um)
        w.load_arrays(g.halfxy, g.pyr_cx, g.pyr_cy, weights, g.sincar, g.submask, g.validsubsx, g.validsubsy,
                      g.phasemap, g.fluxPerSub)
        w.set_pupil(g.tel.mpupil)
        w.set_noise(noise, seed)
        return w

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_pyr_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def load_arrays(self, halfxy, cx, cy, weights, sincar, submask, validsubsx, validsubsy, phasemap=None,
                    fluxPerSub=None, ttprojmat=None):
        """``halfxy``: the pyramid phase (float) as the geometry gives it; it is passed on as
        exp(i halfxy), transposed, like the reference's wfs_init (wfs_init.py:203)."""
        f32 = np.float32
        ph = np.exp(1j * np.asarray(halfxy, np.float64)).astype(np.complex64).T
        hx = np.asfortranarray(ph).ravel(order="F").view(np.float32).copy()
        w = np.ones(np.asarray(cx).size, f32) if weights is None else weights
        keep = [hx, host_array(cx, f32), host_array(cy, f32), host_array(w, f32), host_array(sincar, f32),
                host_array(submask, f32), host_array(validsubsx, np.int32), host_array(validsubsy, np.int32)]
        flux = host_array(fluxPerSub, f32) if fluxPerSub is not None else None
        pm = host_array(phasemap, np.int32) if phasemap is not None else None
        tt = host_array(ttprojmat, f32) if ttprojmat is not None else None
        call("aob_pyr_load_arrays", self.h, *[k.ctypes.data for k in keep], None if pm is None else pm.ctypes.data,
             flux.ctypes.data if flux is not None else None, None if tt is None else tt.ctypes.data)

    def set_submask(self, submask):
        a = host_array(submask, np.float32)
        call("aob_pyr_set_submask", self.h, a.ctypes.data, int(a.size))

    def set_phalfxy(self, phalfxy):
        """The pyramid mask exp(i phase) as nfft x nfft complex64 (already in the
        sensor's layout, as the reference's set_phalfxy takes it)."""
        a = np.ascontiguousarray(np.asarray(phalfxy, np.complex64).ravel(order="F"))
        call("aob_pyr_set_phalfxy", self.h, a.view(np.float32).ctypes.data, int(a.size))

    def set_binimg(self, img):
        a = host_array(img, np.float32)
        call("aob_pyr_set_binimg", self.h, a.ctypes.data, int(a.size))

    def set_compute_focalplane(self, on=True):
        call("aob_pyr_set_compute_focalplane", self.h, 1 if on else 0)

    def slopes_geom(self, type=0, dev_slopes=None, stream=None):
        """Geometric slopes of the phase (SutraWfs::slopes_geom), see ShWfs.slopes_geom."""
        call("aob_pyr_slopes_geom", self.h, int(type), dev_slopes, stream)

    def set_modulation(self, cx, cy, weights=None):
        f32 = np.float32
        a, b = host_array(cx, f32), host_array(cy, f32)
        w = host_array(np.ones(a.size, f32) if weights is None else weights, f32)
        call("aob_pyr_set_modulation", self.h, a.ctypes.data, b.ctypes.data, w.ctypes.data, int(a.size))
        self.npts = int(a.size)

    def set_pupil(self, pupil):
        a = host_array(pupil, np.float32)
        if a.size != self.ntot * self.ntot:
            raise ValueError("pupil must be ntot x ntot")
        call("aob_pyr_set_pupil", self.h, a.ctypes.data)

    def set_noise(self, noise, seed=1234):
        self.noise = float(noise)
        call("aob_pyr_set_noise", self.h, float(noise), int(seed))

    def set_lambda(self, lam):
        self.lambda_um = float(lam)
        call("aob_pyr_set_lambda", self.h, float(lam))

    def set_nphot(self, nphot):
        self.nphot = float(nphot)
        call("aob_pyr_set_nphot", self.h, float(nphot))

    @property
    def frame(self) -> int:
        f = ctypes.c_uint64()
        call("aob_pyr_get_frame", self.h, ctypes.addressof(f))
        return f.value

    @frame.setter
    def frame(self, v):
        call("aob_pyr_set_frame", self.h, int(v))

    def buffer(self, which, dtype=np.float32, shape=None) -> DeviceArray:
        return _buffer("aob_pyr_buffer", self.h, which, dtype, shape, self)

    @property
    def d_phase(self):
        return self.buffer("phase", shape=(self.ntot, self.ntot))

    @property
    def d_binimg(self):
        n = self.nfft // self.nrebin
        return self.buffer("binimg", shape=(n, n))

    @property
    def d_hrimg(self):
        return self.buffer("hrimg", shape=(self.nfft, self.nfft))

    def set_phase(self, phase):
        self.d_phase.set(phase)

    def comp_image(self, noise=True, stream=None):
        call("aob_pyr_comp_image", self.h, 1 if noise else 0, stream)


class Centroider:
    """CoG / tCoG / wCoG / bpCoG / pyramid / masked-pixel centroider (SutraCentroider*).

    A masked-pixel centroider (``maskedpix``) takes ``nvalid`` = the number of
    valid pixels (4 x the pyramid's sub-apertures) and writes one slope per pixel."""

    def __init__(self, nvalid, offset, scale, typec="cog", device=0, wfs: ShWfs | None = None):
        self.h = ctypes.c_void_p()
        self.type = typec
        call("aob_centro_create", ctypes.addressof(self.h), int(device), CENTRO_TYPES[typec], int(nvalid),
             float(offset), float(scale))
        self.nvalid = int(nvalid)
        self.wfs = None
        if wfs is not None:
            self.attach(wfs)

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_centro_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def attach(self, wfs):
        self.wfs = wfs
        if isinstance(wfs, PyrWfs):
            call("aob_centro_attach_pyr", self.h, wfs.h)
        else:
            call("aob_centro_attach_wfs", self.h, wfs.h if wfs is not None else None)

    def set_pyr_method(self, method):
        """The reference's encoding (Method_CoG, sutra_centroider_pyr.hpp:27-34): 0 sinus global,
        1 nosinus global (the default), 2 sinus local, 3 nosinus local."""
        call("aob_centro_set_pyr_method", self.h, int(method))

    def set_pyr_thresh(self, thresh):
        call("aob_centro_set_pyr_thresh", self.h, float(thresh))

    def set_nmax(self, nmax):
        """bpCoG: the pixel of rank nmax (0 = the brightest) sets the threshold."""
        call("aob_centro_set_nmax", self.h, int(nmax))

    @property
    def nslopes(self) -> int:
        return self.nvalid if self.type == "maskedpix" else 2 * self.nvalid

    def set_npix(self, npix):
        call("aob_centro_set_npix", self.h, int(npix))

    def set_scale(self, v):
        call("aob_centro_set_scale", self.h, float(v))

    def set_offset(self, v):
        call("aob_centro_set_offset", self.h, float(v))

    def set_threshold(self, v):
        call("aob_centro_set_threshold", self.h, float(v))

    def set_slope_order(self, order):
        call("aob_centro_set_slope_order", self.h, int(order))

    def load_validpos(self, vx, vy, n=None):
        a, b = host_array(vx, np.int32), host_array(vy, np.int32)
        call("aob_centro_load_validpos", self.h, a.ctypes.data, b.ctypes.data, int(a.size))

    def set_centroids_ref(self, ref):
        a = host_array(ref, np.float32)
        call("aob_centro_set_centroids_ref", self.h, a.ctypes.data)

    def load_weights(self, w, ndim=None):
        a = host_array(w, np.float32)
        call("aob_centro_load_weights", self.h, a.ctypes.data, int(a.size))

    def load_img(self, img, m=None, n=None):
        """A float32 image, or a uint16 camera frame (host array, or a uint16
        DeviceArray such as a sensor's ``d_camimg``, copied on the device)."""
        if isinstance(img, DeviceArray):
            if img.dtype != np.uint16:
                raise TypeError("load_img from device memory takes a uint16 frame")
            m_, n_ = img.shape
            call("aob_centro_load_img_u16", self.h, img.ptr, int(m_), int(n_), 1, None)
            return
        img = np.asarray(img)
        if img.dtype == np.uint16:
            a = host_array(img, np.uint16)
            call("aob_centro_load_img_u16", self.h, a.ctypes.data, int(img.shape[0]), int(img.shape[1]), 0, None)
            return
        img = np.asarray(img, dtype=np.float32)
        a = host_array(img, np.float32)
        call("aob_centro_load_img", self.h, a.ctypes.data, int(img.shape[0]), int(img.shape[1]))

    def set_lut_pix(self, lut):
        a = host_array(lut, np.int32)
        call("aob_centro_set_lut_pix", self.h, a.ctypes.data, int(a.size))

    def calibrate_img_validpix(self, stream=None):
        call("aob_centro_calibrate_img_validpix", self.h, stream)

    def set_dark(self, d, n=None):
        a = host_array(d, np.float32)
        call("aob_centro_set_dark", self.h, a.ctypes.data, int(np.sqrt(a.size)))

    def set_flat(self, f, n=None):
        a = host_array(f, np.float32)
        call("aob_centro_set_flat", self.h, a.ctypes.data, int(np.sqrt(a.size)))

    def calibrate_img(self, stream=None):
        call("aob_centro_calibrate_img", self.h, stream)

    def get_cog(self, dev_slopes: int, stream=None):
        call("aob_centro_get_cog", self.h, dev_slopes, stream)

    def buffer(self, which, dtype=np.float32, shape=None):
        return _buffer("aob_centro_buffer", self.h, which, dtype, shape, self)

    def params(self):
        t, nv, npx = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        o, s, th = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        call("aob_centro_get_params", self.h, *[ctypes.addressof(x) for x in (t, nv, npx, o, s, th)])
        return dict(type=t.value, nvalid=nv.value, npix=npx.value, offset=o.value, scale=s.value,
                    threshold=th.value)


class LsController:
    """Least-squares controller (SutraControllerLs + SutraController), or with
    ``kind="generic"`` the generic controller (SutraControllerGeneric): the same
    buffers and voltage stage, its command laws ("integrator" with a leaky
    factor and optional pseudo-open-loop slopes, "modal_integrator",
    "2matrices") instead of the LS integrator."""

    def __init__(self, nslope, nactu, delay=0.0, device=0, kind="ls"):
        self.h = ctypes.c_void_p()
        if kind not in ("ls", "generic"):
            raise ValueError(f"controller kind must be 'ls' or 'generic', not {kind!r}")
        fn = "aob_ls_create" if kind == "ls" else "aob_generic_create"
        call(fn, ctypes.addressof(self.h), int(device), int(nslope), int(nactu), float(delay))
        self.kind = kind
        self.nslope, self.nactu = int(nslope), int(nactu)
        self.precision = 0

    def set_commandlaw(self, law):
        call("aob_ls_set_commandlaw", self.h, COMMAND_LAWS[law] if isinstance(law, str) else int(law))

    def set_leaky_factor(self, f):
        call("aob_ls_set_leaky_factor", self.h, float(f))

    def set_polc(self, on):
        call("aob_ls_set_polc", self.h, 1 if on else 0)

    def set_decay_factor(self, d):
        self._vec("aob_ls_set_decay_factor", d)

    def set_matE(self, m):
        m = np.asarray(m)
        if m.shape != (self.nactu, self.nactu):
            raise ValueError(f"matE must be ({self.nactu}, {self.nactu})")
        self._vec("aob_ls_set_matE", m)

    def law(self) -> dict:
        k, l, p = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        f = ctypes.c_float()
        call("aob_ls_get_kind", self.h, *[ctypes.addressof(x) for x in (k, l, f, p)])
        names = {v: n for n, v in COMMAND_LAWS.items()}
        return dict(kind="generic" if k.value else "ls", law=names.get(l.value, "ls"), leaky=f.value,
                    polc=bool(p.value))

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_ls_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def _vec(self, fn, a, dtype=np.float32, *extra):
        a = host_array(a, dtype)
        call(fn, self.h, a.ctypes.data, *extra)
        return a

    def set_cmat(self, cmat):
        cmat = np.asarray(cmat)
        if cmat.shape != (self.nactu, self.nslope):
            raise ValueError(f"cmat must be ({self.nactu}, {self.nslope})")
        self._vec("aob_ls_set_cmat", cmat)

    def set_imat(self, imat):
        imat = np.asarray(imat)
        if imat.shape != (self.nslope, self.nactu):
            raise ValueError(f"imat must be ({self.nslope}, {self.nactu})")
        self._vec("aob_ls_set_imat", imat)

    def set_modal_gains(self, g):
        self._vec("aob_ls_set_modal_gains", g)

    def set_gain(self, g):
        call("aob_ls_set_gain", self.h, float(g))

    def set_delay(self, d):
        call("aob_ls_set_delay", self.h, float(d))

    def set_open_loop(self, ol, reset=True):
        call("aob_ls_set_open_loop", self.h, int(ol), 1 if reset else 0)

    def set_com_range(self, lo, hi):
        call("aob_ls_set_com_range", self.h, float(lo), float(hi))

    def set_com(self, com, n=None):
        a = host_array(com, np.float32)
        call("aob_ls_set_com", self.h, a.ctypes.data, int(a.size))

    def set_centroids(self, s):
        a = host_array(s, np.float32)
        call("aob_ls_set_centroids", self.h, a.ctypes.data, int(a.size))

    def set_precision(self, prec):
        p = PRECISIONS[prec] if isinstance(prec, str) else int(prec)
        call("aob_ls_set_precision", self.h, p)
        self.precision = p

    def comp_com(self, stream=None):
        call("aob_ls_comp_com", self.h, stream)

    def set_tuning(self, kind=0, nblocks=0):
        call("aob_ls_set_tuning", self.h, int(kind), int(nblocks))

    def status(self, reset=False) -> int:
        st = ctypes.c_uint32()
        call("aob_ls_status", self.h, ctypes.addressof(st), 1 if reset else 0)
        return st.value

    def clip(self, stream=None):
        call("aob_ls_clip", self.h, stream)

    def comp_voltage(self, stream=None):
        call("aob_ls_comp_voltage", self.h, stream)

    def add_perturb(self, name, pert, n):
        a = host_array(np.asarray(pert, dtype=np.float32).reshape(int(n), self.nactu, order="F"), np.float32)
        call("aob_ls_add_perturb", self.h, name.encode(), a.ctypes.data, int(n))

    def remove_perturb(self, name):
        call("aob_ls_remove_perturb", self.h, name.encode())

    def enable_perturb(self, name, on=True):
        call("aob_ls_enable_perturb", self.h, name.encode(), 1 if on else 0)

    def reset_perturb(self):
        call("aob_ls_reset_perturb", self.h)

    def apply_perturb(self, stream=None):
        """com_clipped += the current row of every enabled perturbation buffer."""
        call("aob_ls_apply_perturb", self.h, stream)

    def svdec_imat(self):
        call("aob_ls_svdec_imat", self.h)

    def build_cmat(self, nfilt):
        call("aob_ls_build_cmat", self.h, int(nfilt))

    def buffer(self, which, dtype=np.float32, shape=None):
        return _buffer("aob_ls_buffer", self.h, which, dtype, shape, self)

    def params(self):
        ns, na, ol, pr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        de, ga, lo, hi = ctypes.c_float(), ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        call("aob_ls_get_params", self.h, *[ctypes.addressof(x) for x in (ns, na, de, ga, ol, lo, hi, pr)])
        return dict(nslope=ns.value, nactu=na.value, delay=de.value, gain=ga.value, open_loop=ol.value,
                    volt_min=lo.value, volt_max=hi.value, prec=pr.value)


class Loop:
    """One RTC iteration bound to a sensor, a centroider and an LS controller."""

    def __init__(self, wfs: ShWfs, centro: Centroider, ls: LsController, graph=True):
        self.h = ctypes.c_void_p()
        call("aob_loop_create", ctypes.addressof(self.h), wfs.h, centro.h, ls.h)
        self.wfs, self.centro, self.ls = wfs, centro, ls
        centro.wfs = wfs
        self.use_graph(graph)
        # the per-iteration entry points, bound once (a step is on a real-time path)
        lib = _lib.lib()
        self._step_fns = ((lib.aob_loop_step_async, "aob_loop_step_async"), (lib.aob_loop_step, "aob_loop_step"))

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_loop_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def use_graph(self, on=True):
        call("aob_loop_use_graph", self.h, 1 if on else 0)

    def set_mode(self, mode=0, fused_batch=0):
        """0: fused cooperative kernel when it fits, 1: three kernels, 2: fused only.

        fused_batch: at most this many sub-apertures per CTA and round in the fused
        kernel (0 = a CTA's whole share at once); results are unchanged."""
        call("aob_loop_set_mode", self.h, int(mode), int(fused_batch))

    def set_host_io(self, mode=1):
        """1: a pinned host voltage buffer of ``step`` is written by the fused
        kernel itself; 0: copy-engine transfer.  Results are identical."""
        call("aob_loop_set_host_io", self.h, int(mode))

    def kernels_per_step(self) -> int:
        n = ctypes.c_int()
        call("aob_loop_kernels_per_step", self.h, ctypes.addressof(n))
        return n.value

    def step(self, host_phase=None, host_voltage=None, noise=True, stream=None, wait=True):
        """host_phase / host_voltage: numpy float32 arrays (pinned for speed) or None.
        wait=False: enqueue the step and return (aob_loop_step_async); the voltages
        are valid once the stream has reached the step."""
        hp = host_phase if host_phase is None or type(host_phase) is int else addr(host_phase)
        hv = host_voltage if host_voltage is None or type(host_voltage) is int else addr(host_voltage)
        fn, name = self._step_fns[1 if wait else 0]
        if fn(self.h, hp, hv, 1 if noise else 0, stream) != 0:
            raise _lib.AobError(f"{name}: {_lib.lib().aob_last_error().decode()}")

    def run(self, host_phases, nsteps, host_voltages=None, noise=True, stream=None, wait=True, nphases=None):
        """``nsteps`` iterations streamed from the host (aob_loop_run): step k
        takes row ``k % nphases`` of ``host_phases`` (a C-contiguous float32
        array, one Fortran-order phase per row, or an int host address with
        ``nphases`` given) and writes row k of ``host_voltages`` (nsteps x nactu
        float32, or None).  The voltages equal ``nsteps`` calls of ``step``; the
        next phase crosses the bus while the current step computes, so pinned
        buffers give the overlap."""
        if type(host_phases) is int:
            if nphases is None:
                raise ValueError("Loop.run: nphases is required with a host address")
            hp = host_phases
        else:
            a = host_phases
            if not isinstance(a, np.ndarray) or a.dtype != np.float32 or not a.flags.c_contiguous or a.ndim < 2:
                raise ValueError("Loop.run: host_phases must be a C-contiguous float32 array, one phase per row")
            nphases, hp = a.shape[0], a.ctypes.data
        hv = host_voltages
        if isinstance(hv, np.ndarray):
            if hv.dtype != np.float32 or not hv.flags.c_contiguous or hv.shape[0] < nsteps:
                raise ValueError("Loop.run: host_voltages must be a C-contiguous float32 array with nsteps rows")
            hv = hv.ctypes.data
        call("aob_loop_run", self.h, hp, int(nphases), int(nsteps), hv, 1 if noise else 0, stream, 1 if wait else 0)

    def step_mlp(self, net, threshold, host_phase=None, host_voltage=None, noise=True, stream=None, wait=True):
        """One iteration with the learned reconstructor ``net`` (an
        ``aob200.mlp.MlpReconstructor``) in place of the LS matrix: sensor image
        with fused centroids, the network's control step (threshold test, LS
        fallback on this loop's controller), voltages -- one fused kernel when it
        fits (aob_loop_step_mlp)."""
        fn = "aob_loop_step_mlp" if wait else "aob_loop_step_mlp_async"
        call(fn, self.h, net.h, float(threshold), addr(host_phase), addr(host_voltage), 1 if noise else 0, stream)

    def persist_start(self, noise=True, host_voltage=None, door_polls=0):
        """Keep the fused kernel resident (matrix rows, tables and the integrator
        state in shared memory); each ``persist_step`` then rings it once.
        host_voltage: a pinned host array the kernel writes at every step."""
        call("aob_loop_persist_start", self.h, 1 if noise else 0, addr(host_voltage), int(door_polls))

    def persist_step(self, host_phase=None, host_voltage=None, noise=True, stream=None, wait=True):
        call("aob_loop_persist_step", self.h, addr(host_phase), addr(host_voltage), 1 if noise else 0, stream,
             1 if wait else 0)

    def persist_stop(self):
        call("aob_loop_persist_stop", self.h)

    def persist_stats(self):
        """(RTC steps rung, summed busy nanoseconds measured by the resident kernel)."""
        n, t = ctypes.c_uint64(), ctypes.c_uint64()
        call("aob_loop_persist_stats", self.h, ctypes.addressof(n), ctypes.addressof(t))
        return n.value, t.value

    def persist_flush(self, dev_buf, nbytes, stream=None):
        """The resident kernel writes nbytes of zeros at dev_buf (an L2 flush
        between timed steps; no other kernel runs beside it)."""
        call("aob_loop_persist_flush", self.h, int(dev_buf), int(nbytes), stream)

    def time(self, noise=True, warmup=3, iters=20) -> float:
        """Device milliseconds of one step (device phase, no host copies)."""
        ms = ctypes.c_float()
        call("aob_loop_time", self.h, 1 if noise else 0, int(warmup), int(iters), ctypes.addressof(ms))
        return float(ms.value)

    def healthy(self) -> bool:
        """False when the device context is broken (a sticky CUDA error makes the
        synchronisation fail) or a bounded wait of the controller's kernels expired."""
        return _device_ok() and self.ls.status() == 0


class Batch:
    """Many SH loops advanced together by one persistent kernel launch per step.

    The batched Monte Carlo mode (no counterpart in the reference, where each
    simulation is a separate process): loops of uneven size -- sub-aperture
    count, pixels, Nfft 16 or 32, any MVM precision -- are stepped by a single
    launch, replayed from a CUDA graph, with results bit-identical to stepping
    each ``Loop`` on its own.  Controllers must have delay 0 and no
    perturbation.  The loops must outlive the batch.
    """

    INFO_KEYS = ("instances", "items", "ctas", "smem_bytes", "rows_per_item", "alg_bytes",
                 "phase_floats", "volt_floats")

    def __init__(self, loops, device=0, graph=True):
        self.h = ctypes.c_void_p()
        call("aob_batch_create", ctypes.addressof(self.h), int(device))
        self.loops = list(loops)
        for l in self.loops:
            call("aob_batch_add", self.h, l.h)
        self.use_graph(graph)

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_batch_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def use_graph(self, on=True):
        call("aob_batch_use_graph", self.h, 1 if on else 0)

    def set_tuning(self, subaps_per_item=0, team_threads=0, mvm_kb=0, lag=2, ctas_per_sm=0, order=0):
        """Tile shapes: sub-apertures per sensor item, threads per sensor team,
        command-matrix KB per MVM item, lag (instances) between an instance's
        sensor and MVM items, CTAs per SM, instance order (0 largest first,
        1 as added).  Results do not depend on them."""
        call("aob_batch_set_tuning", self.h, int(subaps_per_item), int(team_threads), int(mvm_kb), int(lag),
             int(ctas_per_sm), int(order))

    def refresh(self):
        """Re-snapshot every loop's parameters at the next step."""
        call("aob_batch_refresh", self.h)

    def step(self, noise=True, stream=None):
        call("aob_batch_step", self.h, 1 if noise else 0, stream)

    def step_host(self, host_phases=None, host_volts=None, noise=True, stream=None):
        """host_phases: all sensors' phases (each npup*npup, Fortran order as in
        ``Loop.step``) concatenated in insertion order, or None for the device
        phases; host_volts receives all voltages concatenated.  Waits for the stream."""
        call("aob_batch_step_host", self.h, addr(host_phases), addr(host_volts), 1 if noise else 0, stream)

    def info(self) -> dict:
        v = (ctypes.c_int64 * 8)()
        call("aob_batch_info", self.h, ctypes.addressof(v), 8)
        return dict(zip(self.INFO_KEYS, (int(x) for x in v)))

    def offsets(self):
        n = len(self.loops)
        p = (ctypes.c_int64 * n)()
        q = (ctypes.c_int64 * n)()
        call("aob_batch_offsets", self.h, ctypes.addressof(p), ctypes.addressof(q))
        return np.array(p[:], dtype=np.int64), np.array(q[:], dtype=np.int64)

    def status(self) -> int:
        s = ctypes.c_uint32()
        call("aob_batch_status", self.h, ctypes.addressof(s))
        return int(s.value)

    def time(self, noise=True, warmup=3, iters=10) -> float:
        """Device milliseconds of one step (CUDA events on a private stream)."""
        ms = ctypes.c_float()
        call("aob_batch_time", self.h, 1 if noise else 0, int(warmup), int(iters), ctypes.addressof(ms))
        return float(ms.value)

    def healthy(self) -> bool:
        """False when the device context is broken or a bounded wait expired."""
        return _device_ok() and self.status() == 0

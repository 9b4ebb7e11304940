"""Deformable mirror, raytracing and science target on the GPU (C ABI wrappers).

SutraDm (libsutra/src.cpp/sutra_dm.cpp, sutra_dm.cu), SutraSource::raytrace
(sutra_source.cpp:222-320) and SutraSource::comp_image / comp_strehl
(sutra_source.cpp:397-515).
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call, host_array
from .core import DeviceArray, _buffer


class Dm:
    """Piezo-stack DM: shape = sum over actuators of command x influence patch."""

    def __init__(self, dim, influ, i1, j1, device=0):
        influ = np.asarray(influ, dtype=np.float32)
        self.dim, self.influsize, self.nact = int(dim), int(influ.shape[0]), int(influ.shape[2])
        self.h = ctypes.c_void_p()
        a = host_array(influ, np.float32)
        ii, jj = host_array(i1, np.int32), host_array(j1, np.int32)
        call("aob_dm_create", ctypes.addressof(self.h), int(device), self.dim, self.nact, self.influsize,
             a.ctypes.data, ii.ctypes.data, jj.ctypes.data)

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_dm_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def buffer(self, which, shape=None) -> DeviceArray:
        return _buffer("aob_dm_buffer", self.h, which, np.float32, shape, self)

    @property
    def d_shape(self):
        return self.buffer("shape", (self.dim, self.dim))

    def set_com(self, com):
        self.buffer("com").set(com)

    def comp_shape(self, dev_com=None, stream=None):
        call("aob_dm_comp_shape", self.h, dev_com, stream)


def raytrace(dev_out, nx, ny, sources, reset=True, stream=None):
    """sources: list of (dev_ptr, dim, xoff, yoff); out = (0 or out) + bilinear sum."""
    n = len(sources)
    ptrs = (ctypes.c_void_p * max(n, 1))(*[s[0] for s in sources])
    dims = (ctypes.c_int * max(n, 1))(*[int(s[1]) for s in sources])
    xo = (ctypes.c_float * max(n, 1))(*[float(s[2]) for s in sources])
    yo = (ctypes.c_float * max(n, 1))(*[float(s[3]) for s in sources])
    call("aob_raytrace", dev_out, int(nx), int(ny), n, ctypes.addressof(ptrs), ctypes.addressof(dims),
         ctypes.addressof(xo), ctypes.addressof(yo), 1 if reset else 0, stream)


class Target:
    """Science target PSF and Strehl ratio at one wavelength."""

    def __init__(self, pupil, lambda_um, nfft, device=0):
        pupil = np.asarray(pupil, dtype=np.float32)
        self.npup, self.nfft, self.lambda_um = int(pupil.shape[0]), int(nfft), float(lambda_um)
        self.h = ctypes.c_void_p()
        p = host_array(pupil, np.float32)
        call("aob_target_create", ctypes.addressof(self.h), int(device), self.npup, self.nfft, p.ctypes.data,
             float(lambda_um))

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_target_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def buffer(self, which, shape=None) -> DeviceArray:
        return _buffer("aob_target_buffer", self.h, which, np.float32, shape, self)

    @property
    def d_phase(self):
        return self.buffer("phase", (self.npup, self.npup))

    @property
    def d_image_se(self):
        return self.buffer("image_se", (self.nfft, self.nfft))

    @property
    def d_image_le(self):
        return self.buffer("image_le", (self.nfft, self.nfft))

    def comp_image(self, dev_phase=None, comp_le=True, stream=None):
        call("aob_target_comp_image", self.h, dev_phase, 1 if comp_le else 0, stream)

    def strehl(self, stream=None, fit=False):
        """(short, long exposure) Strehl: the image peaks, or with ``fit`` the
        reference's sinc fit of the peak (comp_strehl(do_fit))."""
        se, le = ctypes.c_float(), ctypes.c_float()
        call("aob_target_strehl_fit" if fit else "aob_target_strehl", self.h, ctypes.addressof(se),
             ctypes.addressof(le), stream)
        return se.value, le.value

    def reset_le(self, stream=None):
        call("aob_target_reset_le", self.h, stream)


def fft2d(dev_ptr, n, batch=1, inverse=False, device=0, stream=None):
    call("aob_fft2d_c64", dev_ptr, int(n), int(batch), 1 if inverse else 0, int(device), stream)

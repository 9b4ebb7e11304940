"""Von Karman turbulent layers: extrusion operators and the layer set-up.

Restates the reference's iterative screen extrusion set-up (Fried & Clark,
JOSA A 25(2):463, 2008) from shesha/shesha/util/iterkolmo.py:
  create_stencil :35-75, stencil_size :78-100, Czz/Cxz/Cxx :125-198, AB :201-267
and the layer parameters of shesha/shesha/init/atmos_init.py:29-120.
The covariances are formed on the host in float64; their factorisation (the
pseudo-inverse of Czz and the square root of the innovation covariance) runs
in float64 on the GPU through aob_kolmo_factor_ab.  The von Karman phase
structure function is evaluated from its closed form with the modified Bessel
function K_{5/6} (scipy.special.kv).
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
from scipy.special import gamma, kv

from . import _lib
from ._lib import call, host_array

# 2 Gamma(11/6) 2^(-5/6) pi^(-8/3) (24 Gamma(6/5) / 5)^(5/6)
_K1 = 2 * gamma(11.0 / 6) * 2 ** (-5.0 / 6) * np.pi ** (-8.0 / 3) * (24 * gamma(6.0 / 5) / 5.0) ** (5.0 / 6)
_K2 = gamma(5.0 / 6) * 2 ** (-1.0 / 6)


def structure_function(r, L0=None):
    """Phase structure function D(r) for separation r (pixels, radians^2 at r0 = 1 pixel)."""
    r = np.asarray(r, dtype=np.float64)
    if L0 is None:
        return 6.88 * r ** (5.0 / 6.0)
    x = 2 * np.pi * r / L0
    out = np.zeros_like(x)
    nz = x > 0
    xn = x[nz]
    out[nz] = _K2 - xn ** (5.0 / 6) * kv(5.0 / 6, xn)
    return _K1 * L0 ** (5.0 / 3.0) * out


def _stencil_mask(n):
    st = np.zeros((n, n))
    ns = int(np.log2(n + 1) + 1)
    st[:, 0] = 1
    for i in range(2, ns):
        st[:: 2 ** (i - 1), 2 ** (i - 2)] = 1
        k = 2 ** (i - 1) - 1
        st[k // n, k % n] = 1
    k = 2 ** (ns - 1) - 1
    st[k // n, k % n] = 1
    for i in range(0, n, 2 ** (ns - 1)):
        k = 2 ** (ns - 2) + i * n
        st[k // n, k % n] = 1
    k = 2 ** ns - 1
    st[k // n, k % n] = 1
    for i in range(0, n, 2 ** ns):
        k = 2 ** (ns - 1) + i * n
        st[k // n, k % n] = 1
    return st


def stencil_size(n: int) -> int:
    return int(np.sum(_stencil_mask(n)))


def create_stencil(n):
    """Grid coordinates, new-column coordinates and the stencil indexes."""
    zx, zy = np.meshgrid(np.arange(n) + 1, np.arange(n) + 1, indexing="xy")
    xx = np.full(n, n + 1, dtype=np.float64)
    xy = np.arange(n) + 1
    st = _stencil_mask(n)
    st = np.roll(st, n // 2, axis=0)
    st = np.fliplr(st)
    ist = np.where(st.flatten() != 0)[0]
    return zx, zy, xx, xy, ist


def covariances(n, L0):
    """Czz, Cxz, Cxx (float64) for extruding an n x n screen."""
    zx, zy, xx, xy, ist = create_stencil(n)
    D = lambda d2: structure_function(np.sqrt(d2), L0)  # noqa: E731
    zxs = zx.flatten()[ist].astype(np.float64)
    zys = zy.flatten()[ist].astype(np.float64)
    x0, y0 = float(zx[0, n - 1]), float(zy[0, n - 1])
    # Czz
    t = D((x0 - zxs) ** 2 + (y0 - zys) ** 2)
    zz = 0.5 * (-D((zxs[:, None] - zxs[None, :]) ** 2 + (zys[:, None] - zys[None, :]) ** 2) + t[:, None] + t[None, :])
    # Cxz
    tx = D((x0 - xx) ** 2 + (y0 - xy) ** 2)
    xz = 0.5 * (-D((xx[:, None] - zxs[None, :]) ** 2 + (xy[:, None] - zys[None, :]) ** 2) + tx[:, None] + t[None, :])
    # Cxx
    xxm = 0.5 * (-D((xx[:, None] - xx[None, :]) ** 2 + (xy[:, None] - xy[None, :]) ** 2) + tx[:, None] + tx[None, :])
    return zz, xz, xxm, ist


def extrusion_operators(n, L0, deltax=1.0, deltay=1.0, device=0):
    """A (n x nst), B (n x n) float32 and the x / y stencil indexes (uint32), like iterkolmo.AB."""
    zz, xz, xxm, ist = covariances(n, L0)
    nst = ist.size
    A = np.zeros((n, nst), dtype=np.float32, order="F")
    B = np.zeros((n, n), dtype=np.float32, order="F")
    # keep the host copies alive for the duration of the call
    zzf, xzf, xxf = host_array(zz, np.float64), host_array(xz, np.float64), host_array(xxm, np.float64)
    call("aob_kolmo_factor_ab", int(device), int(n), int(nst), zzf.ctypes.data, xzf.ctypes.data, xxf.ctypes.data,
         A.ctypes.data, B.ctypes.data)
    test = np.zeros(n * n, np.float32)
    test[ist] = np.arange(nst) + 1
    test = np.reshape(test, (n, n), "C")
    isty = np.argsort(test.T.flatten("C")).astype(np.uint32)[n * n - nst:]
    istx = ist.copy()
    if deltay < 0:
        isty = (n * n - 1) - isty
    if deltax < 0:
        istx = (n * n - 1) - istx
    return A, B, istx.astype(np.uint32), isty.astype(np.uint32)


@dataclass
class LayerParams:
    r0_pix: float
    alt: float
    deltax: float
    deltay: float
    dim: int
    L0_pix: float
    seed: int


def layer_params(r0, fracs, alts, winds, dirs, L0s, pupdiam, diam, n_mpupil, ittime, seeds=None):
    """Per-layer r0 (pixels), screen size and per-iteration shifts (atmos_init.py:70-110), on axis."""
    fracs = np.asarray(fracs, dtype=np.float32)
    fracs = fracs / fracs.sum()
    pupixsize = np.float32(diam) / pupdiam
    dim = n_mpupil + 4
    dim += dim % 2
    out = []
    for i in range(len(fracs)):
        lin = pupdiam / diam * winds[i] * ittime
        dx = lin * np.sin(np.pi / 180 * dirs[i] + np.pi)
        dy = lin * np.cos(np.pi / 180 * dirs[i] + np.pi)
        r0l = r0 / (fracs[i] ** (3.0 / 5.0) * pupixsize)
        out.append(LayerParams(float(r0l), float(alts[i]), float(dx), float(dy), int(dim),
                               float(L0s[i] * pupdiam / diam), int(seeds[i] if seeds is not None else 1234 + i)))
    return out


class Atmosphere:
    """Set of extruded von Karman layers on the GPU (SutraAtmos)."""

    def __init__(self, layers, device=0):
        self.h = ctypes.c_void_p()
        call("aob_atmos_create", ctypes.addressof(self.h), int(device))
        self.layers = layers
        self.device = device
        self.offsets = []
        for lp in layers:
            A, B, istx, isty = extrusion_operators(lp.dim, lp.L0_pix, lp.deltax, lp.deltay, device)
            self.add_screen(lp, A, B, istx, isty)
            self.refresh(len(self.offsets) - 1)

    def add_screen(self, lp, A, B, istx, isty):
        idx = ctypes.c_int()
        a, b = host_array(A, np.float32), host_array(B, np.float32)
        ix, iy = host_array(istx, np.uint32), host_array(isty, np.uint32)
        call("aob_atmos_add_screen", self.h, int(lp.dim), int(ix.size), float(lp.r0_pix), float(lp.alt),
             float(lp.deltax), float(lp.deltay), a.ctypes.data, b.ctypes.data, ix.ctypes.data, iy.ctypes.data,
             int(lp.seed), ctypes.addressof(idx))
        self.offsets.append(idx.value)
        return idx.value

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_atmos_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def refresh(self, idx, stream=None):
        call("aob_atmos_refresh_screen", self.h, int(idx), stream)

    def move(self, stream=None):
        call("aob_atmos_move", self.h, stream)

    def screen(self, idx):
        p = ctypes.c_void_p()
        dim = ctypes.c_int()
        ax, ay = ctypes.c_float(), ctypes.c_float()
        call("aob_atmos_screen", self.h, int(idx), ctypes.addressof(p), ctypes.addressof(dim), ctypes.addressof(ax),
             ctypes.addressof(ay))
        return p.value, dim.value, ax.value, ay.value

    def screen_host(self, idx):
        p, dim, _, _ = self.screen(idx)
        return _lib.d2h(p, dim * dim, np.float32).reshape(dim, dim, order="F")

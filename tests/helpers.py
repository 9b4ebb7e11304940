"""Shared test inputs: seeded phase screens, geometry builders and the drop-in modules."""

import os

import numpy as np

from aob200 import geometry as G

SH_CASES = {
    "sh8": (G.ShParams(nxsub=8, npix=2, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0), 48),
    "sh16": (G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0), 128),
    "sh40": (G.ShParams(nxsub=40, npix=6, pixsize=0.36, wavelength_um=0.7, fracsub=0.5, gsmag=8.0), 240),
    # shesha/tests/pytest/par/test_sh.py's sensor: field of view extended (ntot 64 > nfft 32)
    "sh16x": (G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.5, fracsub=0.8, gsmag=3.0), 128),
    # a round focal-plane field stop of 1.6 arcsec over the full pupil
    "sh16fs": (G.ShParams(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0, fssize=1.6), 128),
}
SH_TEL = {"sh16x": dict(cobs=0.12, ittime=0.002)}


def sh_geometry(name):
    p, pup = SH_CASES[name]
    return G.sh_geometry(p, pup, diam=8.0, **SH_TEL.get(name, dict(cobs=0.14, ittime=0.001)))


def kolmogorov_screen(n, r0_pixels, seed, lam_um=0.5):
    """FFT-filtered Kolmogorov phase screen in micron (test input only)."""
    rng = np.random.default_rng(seed)
    f = np.fft.fftfreq(n)
    fx, fy = np.meshgrid(f, f, indexing="ij")
    k = np.hypot(fx, fy)
    k[0, 0] = 1.0
    psd = 0.023 * r0_pixels ** (-5.0 / 3.0) * k ** (-11.0 / 3.0)
    psd[0, 0] = 0.0
    noise = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    ph = np.fft.ifft2(noise * np.sqrt(psd)).real * n  # radians at 0.5 um
    return (ph * lam_um / (2 * np.pi)).astype(np.float32)


def rel_rms(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b**2)), 1e-300))


_PKG = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "compass-saxoplus_b200")
DROPIN_DIRS = {"python": os.path.join(_PKG, "dropin"), "native": os.path.join(_PKG, "dropin_native")}


def import_dropin(kind):
    """(carma, sutra) of the Python drop-in (``kind="python"``) or of the compiled
    pybind11 pair (``"native"``).  Both are named carma / sutra, so whatever
    those names held in sys.modules before is put back afterwards."""
    import sys

    path = DROPIN_DIRS[kind]
    saved = {k: sys.modules.pop(k) for k in ("carma", "sutra") if k in sys.modules}
    sys.path.insert(0, path)
    try:
        import carma
        import sutra
    finally:
        sys.path.remove(path)
        for k in ("carma", "sutra"):
            sys.modules.pop(k, None)
        sys.modules.update(saved)
    if kind == "native":
        assert sutra.__file__.endswith(".so") and carma.__file__.endswith(".so"), "the compiled drop-in is not built"
    return carma, sutra

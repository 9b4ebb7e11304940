"""Cases of the reference-run fixtures (tests/golden/ref_*.npz).

Shared by the script that makes the fixtures with the reference's own GPU
code (make_ref_fixtures.py) and the tests that read them: the geometry
parameters, the seeded command matrix and the wCoG weights.
"""

import numpy as np

from aob200 import geometry as G

SH_CASES = {
    "sh16": (dict(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0), 128),
    "saxo40": (dict(nxsub=40, npix=6, pixsize=0.36, wavelength_um=0.7, fracsub=0.5, gsmag=8.0), 240),
    # shesha/tests/pytest/par/test_sh.py's sensor: field of view extended (ntot 64 > nfft 32)
    "sh16x": (dict(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.5, fracsub=0.8, gsmag=3.0), 128),
    # a round focal-plane field stop of 1.6 arcsec (Sensors.set_field_stop)
    "sh16fs": (dict(nxsub=16, npix=8, pixsize=0.3, wavelength_um=0.7, fracsub=0.5, gsmag=8.0, fssize=1.6), 128),
}
SH_TEL = {"sh16x": dict(cobs=0.12, ittime=0.002)}
PYR_CASES = {
    "pyr16": (dict(nxsub=16, wavelength_um=0.7, ampl=3.0, npts=8, pup_sep=12, fssize=3.2), 64),
    "pyr50": (dict(nxsub=50, wavelength_um=1.075, ampl=3.0, npts=24, pup_sep=32, fssize=3.2), 100),
}
NACTU = 97
GAIN = 0.4


def command_matrix(nslope, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal((NACTU, nslope)) / np.sqrt(nslope)).astype(np.float32)


def wcog_weights(npix):
    x = np.arange(npix) - (npix - 1) / 2.0
    return np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * (npix / 2.35) ** 2)).astype(np.float32)


def sh_geometry(name):
    kw, pup = SH_CASES[name]
    return G.sh_geometry(G.ShParams(**kw), pup, diam=8.0, **SH_TEL.get(name, dict(cobs=0.14, ittime=0.001)))


def pyr_geometry(name):
    kw, pup = PYR_CASES[name]
    return G.pyr_geometry(G.PyrParams(**kw), pup, diam=8.0, cobs=0.14)

"""The CPU oracle pinned against the reference's own GPU code.

tests/golden/ref_*.npz hold what the reference's sutra build (its carma /
sutra modules compiled from source, driven through its Python API as
shesha's supervisor does; tests/golden/make_ref_fixtures.py) computed on a
B200 for seeded inputs: SH spot cubes, images, intensities, CoG / tCoG / wCoG
slopes and LS commands, pyramid images and slopes for all four methods.

The float64 oracle must reproduce them within the reference's own float32
arithmetic: it is compiled with -use_fast_math (libcarma/CMakeLists.txt:45)
and computes in float32 with cuFFT, so the stated bounds are relative rms
1e-6 for images and intensities, 1e-5 for slopes, 1e-6 for commands from
the reference's own slopes.
"""

import os
import sys

import numpy as np
import pytest

from helpers import rel_rms
from oracle import pyr as opyr
from oracle import rtc as ortc
from oracle import sh as osh

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
sys.path.insert(0, GOLD)
import ref_cases as RC  # noqa: E402


def _load(name):
    return np.load(os.path.join(GOLD, f"ref_{name}.npz"))


@pytest.mark.parametrize("name", list(RC.SH_CASES))
def test_sh_oracle_matches_reference_run(name):
    d = _load(name)
    g = RC.sh_geometry(name)
    cube, img, sums = osh.comp_image(d["phase"], g.tel.mpupil, g, 2 * np.pi / g.wavelength_um, g.nphotons)
    assert rel_rms(d["bincube"].reshape(g.npix * g.npix, g.nvalid, order="F"), cube) < 1e-6
    assert rel_rms(d["binimg"], img) < 1e-6
    assert rel_rms(d["intensities"], sums) < 1e-6
    thr = float(d["threshold"])
    w = RC.wcog_weights(g.npix)
    cm = RC.command_matrix(2 * g.nvalid, int(d["cmat_seed"])).astype(np.float64)
    for kind in ("cog", "wcog", "tcog"):
        wflat = np.tile(w.ravel(order="F"), g.nvalid) if kind == "wcog" else None
        s, _, _ = ortc.centroids(img, g.validsubsx, g.validsubsy, g.npix, g.pixsize, g.npix // 2.0 - 0.5, kind=kind,
                                 threshold=thr, weights=wflat)
        assert rel_rms(d[f"slopes_{kind}"], s) < 1e-5, kind
        com = -RC.GAIN * (cm @ d[f"slopes_{kind}"].astype(np.float64))
        assert rel_rms(d[f"com_{kind}"], com) < 1e-6, kind


@pytest.mark.parametrize("name", list(RC.PYR_CASES))
def test_pyramid_oracle_matches_reference_run(name):
    d = _load(name)
    g = RC.pyr_geometry(name)
    img = opyr.comp_image(d["phase"], g.tel.mpupil, g, g.wavelength_um, g.nphotons)
    assert rel_rms(d["binimg"], img) < 1e-6
    for m in range(4):
        s, _ = opyr.slopes(img, g.validsubsx, g.validsubsy, g.nvalid, float(d["scale"]), thresh=1e-4, method=m)
        assert rel_rms(d[f"slopes_m{m}"], s) < 1e-5, m

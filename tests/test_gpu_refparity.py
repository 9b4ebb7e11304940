"""This project's kernels against the reference's own GPU output.

tests/golden/ref_*.npz were computed by the reference's sutra build on a
B200 from seeded inputs (tests/golden/make_ref_fixtures.py).  The same inputs
go through this project's C ABI here: the standalone SH sensor kernel, the
fused and standalone CoG / tCoG / wCoG centroiders, the LS controller, the
fused single-kernel RTC step at the benchmarked saxo40 geometry
(rtc_fused_kernel<float, 32, 6>), and the pyramid sensor with all four slope
methods.

Tolerances: images and intensities relative rms <= 1e-5 (both sides compute in
float32; the reference with -use_fast_math and cuFFT, this project with its
pruned DFT); slopes and commands <= 1e-4 (the accuracy contract for floating
point).
"""

import os
import sys

import numpy as np
import pytest

from helpers import rel_rms

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


def _load(name):
    return np.load(os.path.join(GOLD, f"ref_{name}.npz"))


def _centroider(core, g, kind, thr):
    c = core.Centroider(g.nvalid, g.npix // 2.0 - 0.5, g.pixsize, kind)
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    if kind in ("tcog", "wcog"):
        c.set_threshold(thr)
    if kind == "wcog":
        c.load_weights(RC.wcog_weights(g.npix))
    return c


@pytest.mark.parametrize("name", list(RC.SH_CASES))
def test_sh_sensor_centroiders_and_ls_match_reference_run(core, name):
    d = _load(name)
    g = RC.sh_geometry(name)
    w = core.ShWfs.from_geometry(g)
    w.set_phase(d["phase"])
    w.comp_image(noise=False)
    assert rel_rms(np.array(w.d_bincube).reshape(-1, order="F"), d["bincube"].reshape(-1, order="F")) < 1e-5
    assert rel_rms(np.array(w.d_binimg), d["binimg"]) < 1e-5
    assert rel_rms(np.array(w.d_intensities), d["intensities"]) < 1e-5
    thr = float(d["threshold"])
    cm = RC.command_matrix(2 * g.nvalid, int(d["cmat_seed"]))
    for kind in ("cog", "wcog", "tcog"):
        c = _centroider(core, g, kind, thr)
        c.attach(w)
        ls = core.LsController(2 * g.nvalid, RC.NACTU)
        ls.set_cmat(cm)
        ls.set_gain(RC.GAIN)
        w.comp_image(noise=False)
        c.get_cog(ls.buffer("centroids").ptr)  # slopes fused into the sensor kernel
        ls.comp_com()
        assert rel_rms(np.array(ls.buffer("centroids")), d[f"slopes_{kind}"]) < 1e-4, kind
        assert rel_rms(np.array(ls.buffer("com")), d[f"com_{kind}"]) < 1e-4, kind
        c.attach(None)


def test_saxo40_fused_step_matches_reference_run(core):
    """The benchmarked instantiation, rtc_fused_kernel<float, 32, 6>, against the
    reference's wCoG slopes and LS commands for the same phase and matrix."""
    d = _load("saxo40")
    g = RC.sh_geometry("saxo40")
    w = core.ShWfs.from_geometry(g)
    c = _centroider(core, g, "wcog", float(d["threshold"]))
    ls = core.LsController(2 * g.nvalid, RC.NACTU)
    ls.set_cmat(RC.command_matrix(2 * g.nvalid, int(d["cmat_seed"])))
    ls.set_gain(RC.GAIN)
    loop = core.Loop(w, c, ls, graph=False)
    loop.set_mode(2, 0)
    volt = np.zeros(RC.NACTU, np.float32)
    loop.step(np.ascontiguousarray(d["phase"].ravel(order="F")), volt, noise=False)
    assert loop.kernels_per_step() == 1
    assert rel_rms(np.array(w.d_binimg), d["binimg"]) < 1e-5
    assert rel_rms(np.array(ls.buffer("centroids")), d["slopes_wcog"]) < 1e-4
    assert rel_rms(volt, d["com_wcog"]) < 1e-4
    assert ls.status() == 0


@pytest.mark.parametrize("name", list(RC.PYR_CASES))
def test_pyramid_image_and_slopes_match_reference_run(core, name):
    d = _load(name)
    g = RC.pyr_geometry(name)
    w = core.PyrWfs.from_geometry(g)
    w.set_phase(d["phase"])
    w.comp_image(noise=False)
    assert rel_rms(np.array(w.d_binimg), d["binimg"]) < 1e-5
    for m in range(4):
        c = core.Centroider(g.nvalid, 0.0, float(d["scale"]), "pyr")
        c.load_validpos(g.validsubsx, g.validsubsy)
        c.set_pyr_method(m)
        c.set_pyr_thresh(1e-4)
        c.attach(w)
        ls = core.LsController(2 * g.nvalid, 4)
        c.get_cog(ls.buffer("centroids").ptr)
        assert rel_rms(np.array(ls.buffer("centroids")), d[f"slopes_m{m}"]) < 1e-4, m

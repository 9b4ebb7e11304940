"""Golden fixtures computed by the reference's own sutra GPU code.

Run on a machine with a GPU after ``python oracle/build_ref.py`` built the
reference's ``carma`` / ``sutra`` modules into ``oracle/_ref/``:

    python tests/golden/make_ref_fixtures.py [OUT_DIR [CASE ...]]

For each case the script builds the sensor, centroiders and least-squares
controller through the reference's Python API in the order shesha's
supervisor uses (shesha/shesha/init/geom_init.py:94-101 Telescope,
shesha/shesha/init/wfs_init.py:100-234 Sensors / initgs / load_arrays,
shesha/shesha/init/rtc_init.py:272-358 add_centroider / load_validpos /
set_npix / set_threshold / init_weights / load_weights), with the geometry
arrays of this project's ``aob200.geometry`` (which equal the reference's own
``geom_init`` output bit for bit, tests/test_geometry.py), a seeded von Karman
phase screen and a seeded command matrix.  It stores the inputs and what the
reference computes -- ``d_bincube``, ``d_binimg``, ``d_intensities``, the
CoG / tCoG / wCoG slopes and the LS commands (SH), the pyramid image and its
slopes -- as ``ref_<case>.npz``.  The sensors are noise-free (noise -1), the
path where the reference's output is deterministic.

The tests (tests/test_gpu_refparity.py) compare this project's kernels, and
the CPU oracle, with these files; nothing reads the reference at test time.
"""

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (os.path.join(ROOT, "oracle", "_ref"), os.path.join(ROOT, "compass-saxoplus_b200"), ROOT, HERE):
    if p not in sys.path:
        sys.path.insert(0, p)

from oracle import ref_sutra  # noqa: E402

carma, sutra = ref_sutra.modules()  # the reference's modules, built by oracle/build_ref.py

from aob200.workloads import von_karman_screens  # noqa: E402

from ref_cases import (GAIN, NACTU, PYR_CASES, SH_CASES, command_matrix, pyr_geometry,  # noqa: E402
                       sh_geometry, wcog_weights)


def phase_screen(n, pupdiam, seed):
    """Seeded von Karman screen (r0 0.14 m at 0.5 um, L0 25 m) in micron."""
    return von_karman_screens(n, 8.0 / pupdiam, 0.14, 25.0, 1, seed=seed)[0]


def _telescope(ctx, tel):
    return ref_sutra.telescope(sutra, ctx, tel)


def _initgs(sensors, n, lam, mag):
    ref_sutra.initgs(sensors, n, lam, mag)


def _ls(ctx, rtc, nslope, cmat):
    return ref_sutra.add_ls(ctx, rtc, nslope, cmat, GAIN)


def run_sh(ctx, name, seed):
    g = sh_geometry(name)
    tel = _telescope(ctx, g.tel)
    sensors, wfs = ref_sutra.sh_sensors(sutra, ctx, tel, g)
    phase = phase_screen(g.tel.n, g.tel.pupdiam, seed)
    wfs.d_gs.set_phase(phase)
    nslope = 2 * g.nvalid
    cmat = command_matrix(nslope, seed + 1)
    thr = float(0.02 * g.nphotons / (g.npix * g.npix))
    out = dict(phase=phase, cmat_seed=seed + 1, threshold=thr)
    for kind in ("cog", "wcog", "tcog"):  # tcog last: it writes the thresholded pixels back
        wfs.comp_image(False)
        if kind == "cog":
            out["bincube"] = np.array(wfs.d_bincube)
            out["binimg"] = np.array(wfs.d_binimg)
            out["intensities"] = np.array(wfs.d_intensities)
        rtc = sutra.Rtc_FFF()
        ref_sutra.add_centroider(ctx, rtc, wfs, g, kind, thr, wcog_weights(g.npix))
        c = _ls(ctx, rtc, nslope, cmat)
        rtc.do_centroids(0)
        rtc.do_control(0)
        out[f"slopes_{kind}"] = np.array(c.d_centroids)
        out[f"com_{kind}"] = np.array(c.d_com)
    return out


def run_pyr(ctx, name, seed):
    g = pyr_geometry(name)
    tel = _telescope(ctx, g.tel)
    i64 = lambda v: np.array([v], dtype=np.int64)  # noqa: E731
    f32 = lambda v: np.array([v], dtype=np.float32)  # noqa: E731
    npts = int(g.pyr_cx.size)
    sensors = sutra.Sensors(ctx, tel, ["pyrhr"], 1, i64(g.nxsub), i64(g.nvalid), i64(4),
                            i64(int(g.validsubsx.size)), i64(g.pdiam), i64(g.nrebin), i64(g.nfft), i64(g.ntot),
                            i64(npts), f32(g.pdiam), f32(g.nphotons), f32(g.nphotons), np.zeros(1, np.int32),
                            np.zeros(1, bool), np.zeros(1, np.int32), np.zeros(1, np.int32), ctx.active_device,
                            False)
    _initgs(sensors, g.tel.n, g.wavelength_um, 6.0)
    wfs = sensors.d_wfs[0]
    halfxy = np.exp(1j * g.halfxy).astype(np.complex64).T.copy()
    wfs.compute_pyrfocalplane = False
    ttproj = np.zeros((g.pdiam * g.pdiam, 2 * g.nvalid), np.float32)
    wfs.load_arrays(halfxy, g.pyr_cx, g.pyr_cy, np.ones(npts, np.float32), g.sincar, g.submask, g.validsubsx,
                    g.validsubsy, g.phasemap, g.fluxPerSub, ttproj)
    phase = (np.random.default_rng(seed).standard_normal((g.tel.n, g.tel.n)) * 0.02).astype(np.float32)
    wfs.d_gs.set_phase(phase)
    wfs.comp_image(False)
    out = dict(phase=phase, binimg=np.array(wfs.d_binimg))
    scale = (g.wavelength_um * 1e-6 / 8.0) * 3.0 * 206264.80624709636
    for method in (0, 1, 2, 3):
        rtc = sutra.Rtc_FFF()
        rtc.add_centroider(ctx, g.nvalid, 0.0, scale, False, ctx.active_device, "pyr", wfs)
        ce = rtc.d_centro[0]
        ce.load_validpos(g.validsubsx, g.validsubsy, int(g.validsubsx.size))
        ce.set_npix(g.npix)
        ce.set_pyr_method(method)
        ce.set_pyr_thresh(1e-4)
        c = _ls(ctx, rtc, 2 * g.nvalid, command_matrix(2 * g.nvalid, seed + 1))
        rtc.do_centroids(0)
        out[f"slopes_m{method}"] = np.array(c.d_centroids)
    out["scale"] = scale
    return out


def main(out_dir, only=None):
    os.makedirs(out_dir, exist_ok=True)
    ctx = carma.context.get_instance_1gpu(0)
    for i, name in enumerate(SH_CASES):
        if only and name not in only:
            continue
        d = run_sh(ctx, name, seed=100 + i)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), **d)
        print(name, {k: getattr(v, "shape", v) for k, v in d.items()})
    for i, name in enumerate(PYR_CASES):
        if only and name not in only:
            continue
        d = run_pyr(ctx, name, seed=200 + i)
        np.savez_compressed(os.path.join(out_dir, f"ref_{name}.npz"), **d)
        print(name, {k: getattr(v, "shape", v) for k, v in d.items()})


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else HERE, sys.argv[2:])

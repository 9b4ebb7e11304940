"""Golden fixtures computed by the reference's own sutra GPU code.

Run on a machine with a GPU after ``python oracle/build_ref.py`` built the
reference's ``carma`` / ``sutra`` modules into ``oracle/_ref/``:

    python tests/golden/make_ref_fixtures.py [OUT_DIR [CASE ...]]
    python tests/golden/make_ref_fixtures.py extras [OUT_DIR]

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
path where the reference's output is deterministic.  ``extras`` stores the
geometric slopes, the 17x17-DM interaction matrix (do_imat) and the pyramid
focal plane as ``ref_extras_sh16.npz`` / ``ref_extras_pyr16.npz``.

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


def run_sh_extras(ctx, name, seed):
    """Geometric slopes (SutraWfs::slopes_geom, all three methods) and the
    push-pull interaction matrix of the 17x17 DM (SutraRtc::do_imat with a CoG
    centroider and an LS controller), on the reference's own objects."""
    g = sh_geometry(name)
    tel = _telescope(ctx, g.tel)
    sensors, wfs = ref_sutra.sh_sensors(sutra, ctx, tel, g)
    phase = phase_screen(g.tel.n, g.tel.pupdiam, seed)
    wfs.d_gs.set_phase(phase)
    out = dict(phase=phase)
    for t in (0, 1, 2):
        wfs.slopes_geom(t)
        out[f"geom{t}"] = np.array(wfs.d_slopes)
    dm = dict(np.load(os.path.join(HERE, "dm17.npz")))
    dms = sutra.Dms()
    dim = int(dm["dim"])
    push = 0.05
    dms.add_dm(ctx, "pzt", 0.0, dim, int(dm["ntotact"]), int(dm["influsize"]), int(dm["influpos"].size),
               int(dm["ninflu"].size), push, 0, ctx.active_device)
    dms.d_dms[0].pzt_loadarrays(dm["influ"], dm["influpos"], dm["ninflu"], dm["influstart"], dm["i1"], dm["j1"])
    off = (dim - g.tel.n) / 2.0
    wfs.d_gs.add_layer("pzt", 0, off, off)
    rtc = sutra.Rtc_FFF()
    ref_sutra.add_centroider(ctx, rtc, wfs, g, "cog")
    nactu = int(dm["ntotact"])
    rtc.add_controller(ctx, "ls", ctx.active_device, 0.0, 2 * g.nvalid, nactu, dms=dms,
                       idx_dms=np.zeros(1, np.int32), ndm=1, idx_centro=np.zeros(1, np.int32), ncentro=1)
    rtc.do_imat(0, dms, False)
    out["imat"] = np.array(rtc.d_control[0].d_imat)
    out["push4imat"] = push
    out["dm_offset"] = off
    return out


def run_pyr_extras(ctx, name, seed):
    """The pyramid focal plane (compute_pyrfocalplane) and geometric slopes
    (methods 0 and 1) on the reference's own sensor."""
    g = pyr_geometry(name)
    tel = _telescope(ctx, g.tel)
    i64 = lambda v: np.array([v], dtype=np.int64)  # noqa: E731
    f32 = lambda v: np.array([v], dtype=np.float32)  # noqa: E731
    npts = int(g.pyr_cx.size)
    subapd = float(g.tel.diam) / g.nxsub
    sensors = sutra.Sensors(ctx, tel, ["pyrhr"], 1, i64(g.nxsub), i64(g.nvalid), i64(4),
                            i64(int(g.validsubsx.size)), i64(g.pdiam), i64(g.nrebin), i64(g.nfft), i64(g.ntot),
                            i64(npts), f32(subapd), f32(g.nphotons), f32(g.nphotons), np.zeros(1, np.int32),
                            np.zeros(1, bool), np.zeros(1, np.int32), np.zeros(1, np.int32), ctx.active_device,
                            False)
    _initgs(sensors, g.tel.n, g.wavelength_um, 6.0)
    wfs = sensors.d_wfs[0]
    halfxy = np.exp(1j * g.halfxy).astype(np.complex64).T.copy()
    ttproj = np.zeros((g.pdiam * g.pdiam, 2 * g.nvalid), np.float32)
    wfs.load_arrays(halfxy, g.pyr_cx, g.pyr_cy, np.ones(npts, np.float32), g.sincar, g.submask, g.validsubsx,
                    g.validsubsy, g.phasemap, g.fluxPerSub, ttproj)
    phase = (np.random.default_rng(seed).standard_normal((g.tel.n, g.tel.n)) * 0.02).astype(np.float32)
    wfs.d_gs.set_phase(phase)
    wfs.compute_pyrfocalplane = True
    wfs.comp_image(False)
    out = dict(phase=phase, focal=np.array(wfs.d_pyrfocalplane), binimg=np.array(wfs.d_binimg), subapd=subapd)
    for t in (0, 1):
        wfs.slopes_geom(t)
        out[f"geom{t}"] = np.array(wfs.d_slopes)
    return out


def main_extras(out_dir):
    os.makedirs(out_dir, exist_ok=True)
    ctx = carma.context.get_instance_1gpu(0)
    d = run_sh_extras(ctx, "sh16", seed=300)
    np.savez_compressed(os.path.join(out_dir, "ref_extras_sh16.npz"), **d)
    print("sh16 extras", {k: getattr(v, "shape", v) for k, v in d.items()})
    d = run_pyr_extras(ctx, "pyr16", seed=301)
    np.savez_compressed(os.path.join(out_dir, "ref_extras_pyr16.npz"), **d)
    print("pyr16 extras", {k: getattr(v, "shape", v) for k, v in d.items()})


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
    args = sys.argv[1:]
    if args and args[0] == "extras":
        main_extras(args[1] if len(args) > 1 else HERE)
    else:
        main(args[0] if args else HERE, args[1:])

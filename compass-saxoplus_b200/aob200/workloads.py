"""Named workloads used by the benchmark and the smoke test.

``saxo40``: the SAXO-scale Shack-Hartmann loop -- 8 m telescope with a 0.14
central obstruction, 40x40 sub-apertures over a 240-pixel pupil (6 phase
pixels per sub-aperture), 6x6 binned pixels, 0.36 arcsec requested pixels at
0.7 um (so the reference geometry gives Nfft = 32, nrebin = 3 and 1248 valid
sub-apertures), guide star magnitude 8 with photon noise and 0.5 e- readout
noise, weighted CoG with threshold, 1377 actuators.

``plain16``: the plain 16x16 loop (128-pixel pupil, 8x8 pixels, no noise,
plain CoG, 241 actuators).

Phase screens for the standalone benchmark are seeded von Karman screens made
by FFT filtering (the synthetic stand-in for the turbulence the reference
extrudes; the GPU extrusion lives in the atmosphere module).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import geometry as G

WORKLOADS = {
    "saxo40": dict(nxsub=40, npix=6, pixsize=0.36, lam=0.7, pupdiam=240, gsmag=8.0, noise=0.5,
                   centroider="wcog", nactu=1377, r0=0.14, L0=25.0),
    "plain16": dict(nxsub=16, npix=8, pixsize=0.3, lam=0.7, pupdiam=128, gsmag=8.0, noise=-1.0,
                    centroider="cog", nactu=241, r0=0.16, L0=25.0),
}


def von_karman_screens(n, pixsize_m, r0_m, L0_m, count, seed, lam_um=0.5):
    """``count`` independent n x n von Karman phase screens in micron (FFT method)."""
    rng = np.random.default_rng(seed)
    m = 2 * n  # oversize to reduce the periodicity of the FFT method
    f = np.fft.fftfreq(m, d=pixsize_m)
    fx, fy = np.meshgrid(f, f, indexing="ij")
    k2 = fx**2 + fy**2 + 1.0 / L0_m**2
    psd = 0.023 * r0_m ** (-5.0 / 3.0) * k2 ** (-11.0 / 6.0)
    psd[0, 0] = 0.0
    df = 1.0 / (m * pixsize_m)
    out = np.empty((count, n, n), dtype=np.float32)
    for i in range(count):
        c = (rng.standard_normal((m, m)) + 1j * rng.standard_normal((m, m))) * np.sqrt(psd) * df
        ph = np.fft.ifft2(c).real * m * m  # radians at 0.5 um
        out[i] = (ph[:n, :n] * lam_um / (2 * np.pi)).astype(np.float32)
    return out


@dataclass
class ShLoopSetup:
    name: str
    geom: G.ShGeometry
    cmat: np.ndarray
    threshold: float
    weights: np.ndarray
    noise: float
    centroider: str

    @property
    def nslope(self):
        return 2 * self.geom.nvalid

    @property
    def nactu(self):
        return self.cmat.shape[0]


def sh_loop_setup(name="saxo40", seed=0) -> ShLoopSetup:
    """Geometry, command matrix (seeded, least-squares scaled) and centroider settings."""
    w = WORKLOADS[name]
    p = G.ShParams(nxsub=w["nxsub"], npix=w["npix"], pixsize=w["pixsize"], wavelength_um=w["lam"],
                   fracsub=0.5, gsmag=w["gsmag"], noise=w["noise"])
    g = G.sh_geometry(p, w["pupdiam"], diam=8.0, cobs=0.14, ittime=0.001)
    rng = np.random.default_rng(seed)
    cmat = (rng.standard_normal((w["nactu"], 2 * g.nvalid)) / np.sqrt(2 * g.nvalid)).astype(np.float32)
    x = np.arange(g.npix) - (g.npix - 1) / 2.0
    weights = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * (g.npix / 2.35) ** 2)).astype(np.float32)
    thr = 0.02 * g.nphotons / (g.npix * g.npix)
    return ShLoopSetup(name, g, cmat, float(thr), weights, w["noise"], w["centroider"])


def build_sh_loop(setup: ShLoopSetup, precision="f32", device=0, graph=True, seed=1234):
    """Construct (sensor, centroider, controller, loop) on the GPU for ``setup``."""
    from . import core

    g = setup.geom
    wfs = core.ShWfs.from_geometry(g, device=device, noise=setup.noise, seed=seed)
    c = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, setup.centroider, device=device)
    c.set_npix(g.npix)
    c.load_validpos(g.validsubsx, g.validsubsy)
    if setup.centroider in ("tcog", "wcog"):
        c.set_threshold(setup.threshold)
    if setup.centroider == "wcog":
        c.load_weights(setup.weights)
    ls = core.LsController(setup.nslope, setup.nactu, delay=0.0, device=device)
    ls.set_precision(precision)
    ls.set_cmat(setup.cmat)
    ls.set_gain(0.4)
    loop = core.Loop(wfs, c, ls, graph=graph)
    return wfs, c, ls, loop


# ---------------------------------------------------------------------------
# Second-stage input: the residual of the saxo40 closed loop
def saxo40_residual(niter=200, device=0):
    """Residual phase (micron) on the target's pupil grid after ``niter``
    seeded iterations of the saxo40 closed loop (3-layer von Karman turbulence,
    photon + readout noise, its own push-pull LS command matrix)."""
    from . import system as S

    sy = S.ShAoSystem(S.saxo40(), device)
    sy.calibrate()
    sy.close(graph=False)
    for _ in range(niter):
        sy.next(compute_psf=False, noise=True)
    sy.trace_target()
    ph = np.array(sy.target.d_phase, dtype=np.float64)
    pup = sy.geom.tel.spupil > 0
    ph = np.where(pup, ph - ph[pup].mean(), 0.0)
    return ph.astype(np.float32), float(sy.geom.tel.pupdiam)


def resample_pupil(phase, pupdiam_in, n_out, pupdiam_out):
    """Bilinear resampling of a phase given on a pupil grid of ``pupdiam_in``
    pixels across (the pupil filling the array, centred) onto an ``n_out`` x
    ``n_out`` grid whose centred pupil is ``pupdiam_out`` pixels across."""
    n_in = phase.shape[0]
    off_in = (n_in - pupdiam_in) / 2.0
    off_out = (n_out - pupdiam_out) / 2.0
    r = pupdiam_in / pupdiam_out
    u = np.clip((np.arange(n_out) - off_out + 0.5) * r - 0.5 + off_in, 0.0, n_in - 1.0)
    i0 = np.minimum(np.floor(u).astype(np.int64), n_in - 2)
    t = u - i0
    p = phase.astype(np.float64)
    rows = p[i0] * (1 - t)[:, None] + p[i0 + 1] * t[:, None]
    out = rows[:, i0] * (1 - t)[None, :] + rows[:, i0 + 1] * t[None, :]
    return out.astype(np.float32)


# ---------------------------------------------------------------------------
# Batched Monte Carlo: independent SH instances of uneven size
@dataclass
class McInstance:
    index: int
    nxsub: int
    npix: int
    r0: float
    seed: int
    setup: ShLoopSetup
    phase: np.ndarray  # npup x npup von Karman screen at 0.5 um [um]


def mc_instance_list(count=64, seed=0):
    """(nxsub, npix, r0, seed) of each instance: nxsub uniform in [24, 40],
    6x6 or 8x8 binned pixels, r0 uniform in [0.08, 0.20] m, seeds 0..count-1."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        nxsub = int(rng.integers(24, 41))
        npix = int(rng.choice([6, 8]))
        r0 = float(rng.uniform(0.08, 0.20))
        out.append((nxsub, npix, r0, i))
    return out


def mc_make(nxsub, npix, r0, seed, pixsize=0.36, pd=6):
    """One SAXO-like instance: ``pd`` phase pixels per sub-aperture (pupil
    pd * nxsub), ``pixsize`` arcsec pixels at 0.7 um, guide star magnitude 8
    with 0.5 e- readout noise and a weighted CoG; the DM has about
    1377 * ((nxsub + 1) / 41)^2 actuators (the saxo40 count scaled by the
    actuator grid); seeded command matrix and von Karman phase screen."""
    p = G.ShParams(nxsub=nxsub, npix=npix, pixsize=pixsize, wavelength_um=0.7, fracsub=0.5, gsmag=8.0,
                   noise=0.5)
    g = G.sh_geometry(p, pd * nxsub, diam=8.0, cobs=0.14, ittime=0.001)
    nact = int(round(1377 * ((nxsub + 1) / 41.0) ** 2))
    rng = np.random.default_rng(1000 + seed)
    cmat = (rng.standard_normal((nact, 2 * g.nvalid)) / np.sqrt(2 * g.nvalid)).astype(np.float32)
    x = np.arange(g.npix) - (g.npix - 1) / 2.0
    weights = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * (g.npix / 2.35) ** 2)).astype(np.float32)
    thr = 0.02 * g.nphotons / (g.npix * g.npix)
    setup = ShLoopSetup(f"mc{seed}", g, cmat, float(thr), weights, 0.5, "wcog")
    phase = von_karman_screens(g.tel.n, 8.0 / g.tel.pupdiam, r0, 25.0, 1, seed=2000 + seed)[0]
    return McInstance(seed, nxsub, npix, r0, seed, setup, phase)


def mc_setup(count=64, seed=0):
    """The batched Monte Carlo workload: ``count`` instances from mc_instance_list."""
    return [mc_make(nxsub, npix, r0, s) for nxsub, npix, r0, s in mc_instance_list(count, seed)]


def build_mc_batch(instances, precision="bf16", device=0, graph=True):
    """Loops of every instance (phases loaded) and the batch that steps them."""
    from . import core

    loops = []
    for inst in instances:
        wfs, c, ls, loop = build_sh_loop(inst.setup, precision=precision, device=device, graph=graph,
                                         seed=1234 + inst.seed)
        wfs.set_phase(inst.phase)
        loops.append((wfs, c, ls, loop))
    batch = core.Batch([l[3] for l in loops], device=device, graph=graph)
    return loops, batch

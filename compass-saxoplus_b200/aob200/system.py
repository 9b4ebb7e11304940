"""A single-conjugate SH adaptive-optics system driven on one GPU.

The iteration order is the reference supervisor's (CompassSupervisor.next,
shesha/shesha/supervisor/compassSupervisor.py:175-289): move the layers, trace
the target (layers + DM) and the sensor (layers + DM), form the sensor image
with its fused centroids, run the LS control law and voltages, shape the DM,
then the target PSF and Strehl.  Calibration follows the reference's push-pull
interaction matrix (libsutra/src.cpp/sutra_rtc.cpp:150-292) and the filtered
least-squares inverse (sutra_controller_ls.cpp:116-217, float64 on the GPU).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import core, dm_geometry, optics, turbulence
from . import geometry as G
from ._lib import call


@dataclass
class AoConfig:
    nxsub: int = 40
    npix: int = 6
    pixsize: float = 0.36
    wfs_lambda: float = 0.7
    pupdiam: int = 240
    diam: float = 8.0
    cobs: float = 0.14
    gsmag: float = 8.0
    noise: float = 0.5
    centroider: str = "wcog"
    threshold_frac: float = 0.02
    nact: int = 41
    coupling: float = 0.3
    dm_margin_out: float | None = 1.0
    r0: float = 0.14
    fracs: tuple = (0.5, 0.3, 0.2)
    alts: tuple = (0.0, 0.0, 0.0)
    winds: tuple = (8.0, 15.0, 25.0)
    dirs: tuple = (0.0, 45.0, 90.0)
    L0: float = 25.0
    ittime: float = 0.001
    gain: float = 0.4
    delay: float = 0.0
    target_lambda: float = 1.65
    push4imat: float = 0.05
    maxcond: float = 1500.0
    precision: str = "f32"
    seeds: tuple = field(default=(1234, 1235, 1236))


def saxo40() -> AoConfig:
    return AoConfig()


def plain16() -> AoConfig:
    # maxcond 30 filters the weakly sensed edge-actuator modes (LE Strehl 0.83
    # at 1.65 um instead of 0.33 with 1500 on this geometry)
    return AoConfig(nxsub=16, npix=8, pixsize=0.3, pupdiam=128, noise=-1.0, centroider="cog", nact=17,
                    dm_margin_out=None, r0=0.16, fracs=(1.0,), alts=(0.0,), winds=(10.0,), dirs=(0.0,),
                    seeds=(1234,), maxcond=30.0)


class ShAoSystem:
    def __init__(self, cfg: AoConfig, device: int = 0):
        self.cfg = cfg
        self.device = device
        p = G.ShParams(nxsub=cfg.nxsub, npix=cfg.npix, pixsize=cfg.pixsize, wavelength_um=cfg.wfs_lambda,
                       fracsub=0.5, gsmag=cfg.gsmag, noise=cfg.noise)
        self.geom = g = G.sh_geometry(p, cfg.pupdiam, diam=cfg.diam, cobs=cfg.cobs, ittime=cfg.ittime)
        tel = g.tel
        self.n = tel.n
        # sensor, centroider
        self.wfs = core.ShWfs.from_geometry(g, device=device, noise=cfg.noise, seed=1234)
        self.centro = core.Centroider(g.nvalid, g.npix / 2 - 0.5, g.pixsize, cfg.centroider, device=device)
        self.centro.set_npix(g.npix)
        self.centro.load_validpos(g.validsubsx, g.validsubsy)
        if cfg.centroider in ("tcog", "wcog"):
            self.centro.set_threshold(cfg.threshold_frac * g.nphotons / (g.npix * g.npix))
        if cfg.centroider == "wcog":
            x = np.arange(g.npix) - (g.npix - 1) / 2.0
            w = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / (2 * (g.npix / 2.35) ** 2)).astype(np.float32)
            self.centro.load_weights(w)
        # DM
        self.dmg = dmg = dm_geometry.pzt_dm_geometry(cfg.nact, tel.pupdiam, tel.cent, tel.ssize, tel.n, cfg.cobs,
                                                      coupling=cfg.coupling, margin_out=cfg.dm_margin_out)
        self.dm = optics.Dm(dmg.dim, dmg.influ, dmg.i1, dmg.j1, device=device)
        self.dm_off = (dmg.dim - tel.n) / 2.0
        self.nactu = dmg.ntotact
        # controller
        self.ls = core.LsController(2 * g.nvalid, self.nactu, delay=cfg.delay, device=device)
        self.ls.set_precision(cfg.precision)
        self.ls.set_gain(cfg.gain)
        # layers
        self.layer_params = turbulence.layer_params(cfg.r0, cfg.fracs, cfg.alts, cfg.winds, cfg.dirs,
                                                    [cfg.L0] * len(cfg.fracs), tel.pupdiam, cfg.diam, tel.n,
                                                    cfg.ittime, seeds=cfg.seeds)
        self.atmos = turbulence.Atmosphere(self.layer_params, device=device)
        # target on the spupil grid
        self.target = optics.Target(tel.spupil, cfg.target_lambda, tel.ssize, device=device)
        self.pupdiff = (tel.n - tel.pupdiam) / 2.0
        self.loop = None
        self.iter = 0

    # ------------------------------------------------------------- raytracing
    def _layer_sources(self, extra=0.0):
        out = []
        for i, lp in enumerate(self.layer_params):
            p, dim, ax, ay = self.atmos.screen(i)
            off = (dim - self.n) / 2.0 + extra
            out.append((p, dim, off + ax, off + ay))
        return out

    def trace_wfs(self, stream=None, with_atmos=True, with_dm=True):
        srcs = (self._layer_sources() if with_atmos else [])
        if with_dm:
            srcs.append((self.dm.d_shape.ptr, self.dm.dim, self.dm_off, self.dm_off))
        optics.raytrace(self.wfs.d_phase.ptr, self.n, self.n, srcs, reset=True, stream=stream)

    def trace_target(self, stream=None):
        srcs = self._layer_sources(extra=self.pupdiff)
        srcs.append((self.dm.d_shape.ptr, self.dm.dim, self.dm_off + self.pupdiff, self.dm_off + self.pupdiff))
        npup = self.target.npup
        optics.raytrace(self.target.d_phase.ptr, npup, npup, srcs, reset=True, stream=stream)

    # ------------------------------------------------------------ calibration
    def measure_slopes(self, stream=None):
        self.wfs.comp_image(noise=False, stream=stream)
        dst = self.ls.buffer("centroids")
        self.centro.attach(self.wfs)
        self.centro.get_cog(dst.ptr, stream)
        return np.array(dst)

    def interaction_matrix(self, push=None, chunk=0):
        """Push-pull interaction matrix of the DM seen by the sensor, every actuator
        poked in one batch (aob_imat_build: four launches per chunk of actuators)."""
        push = self.cfg.push4imat if push is None else push
        self.centro.attach(self.wfs)
        imat = np.zeros((self.ls.nslope, self.nactu), dtype=np.float32)
        self.ls.set_imat(imat)  # allocates the controller's imat buffer
        out = self.ls.buffer("imat")
        call("aob_imat_build", self.wfs.h, self.centro.h, self.dm.h, float(self.dm_off), float(self.dm_off),
             float(push), int(chunk), out.ptr, None)
        return np.array(self.ls.buffer("imat", shape=(self.ls.nslope, self.nactu)))

    def calibrate(self, push=None, maxcond=None, batched=True):
        """Push-pull interaction matrix through DM -> sensor, then the filtered LS inverse.

        ``batched``: all actuators in one batch (interaction_matrix), else one poke
        after the other through the separate calls.  Modes whose singular value is
        below the largest over ``maxcond`` are filtered (the eigenvalues of
        imat^T imat are squared singular values).
        """
        push = self.cfg.push4imat if push is None else push
        maxcond = self.cfg.maxcond if maxcond is None else maxcond
        if batched:
            imat = self.interaction_matrix(push)
            self.dm.set_com(np.zeros(self.nactu, dtype=np.float32))
            self.dm.comp_shape()
            return self._finish_calibration(imat, maxcond)
        imat = np.zeros((self.ls.nslope, self.nactu), dtype=np.float32)
        com = np.zeros(self.nactu, dtype=np.float32)
        for a in range(self.nactu):
            com[a] = push
            self.dm.set_com(com)
            self.dm.comp_shape()
            self.trace_wfs(with_atmos=False)
            sp = self.measure_slopes()
            com[a] = -push
            self.dm.set_com(com)
            self.dm.comp_shape()
            self.trace_wfs(with_atmos=False)
            sm = self.measure_slopes()
            com[a] = 0.0
            imat[:, a] = (sp - sm) / (2 * push)
        self.dm.set_com(com)
        self.dm.comp_shape()
        return self._finish_calibration(imat, maxcond)

    def _finish_calibration(self, imat, maxcond):
        self.imat = imat
        self.ls.set_imat(imat)
        self.ls.svdec_imat()
        ev = np.array(self.ls.buffer("eigenvals"))
        nfilt = int(np.sum(ev < ev.max() / maxcond**2))
        self.nfilt = nfilt
        self.ls.build_cmat(nfilt)
        self.cmat = np.array(self.ls.buffer("cmat", shape=(self.nactu, self.ls.nslope)))
        # reload the packed copies used by the MVM
        self.ls.set_cmat(self.cmat)
        return imat

    # ------------------------------------------------------------------ loop
    def close(self, graph=False, mode=0):
        self.loop = core.Loop(self.wfs, self.centro, self.ls, graph=graph)
        self.loop.set_mode(mode)
        return self.loop

    def next(self, stream=None, compute_psf=True, noise=True, mlp=None, threshold=np.inf):
        """One closed-loop iteration (the supervisor's order).  With ``mlp`` the
        commands come from the learned reconstructor (aob_mlp_comp_com), with the
        LS MVM as fallback when the predicted command norm exceeds ``threshold``."""
        self.atmos.move(stream)
        if compute_psf:
            self.trace_target(stream)
        self.trace_wfs(stream)
        if mlp is None:
            self.loop.step(None, None, noise, stream)
        else:
            self.wfs.comp_image(noise, stream)
            self.centro.get_cog(self.ls.buffer("centroids").ptr, stream)
            mlp.comp_com(self.ls, float(min(threshold, 3.0e38)), stream)
            self.ls.comp_voltage(stream)
        self.dm.comp_shape(self.ls.buffer("voltage").ptr, stream)
        if compute_psf:
            self.target.comp_image(None, True, stream)
        self.iter += 1

    def strehl(self, stream=None):
        return self.target.strehl(stream)

    def residual_rms(self):
        """Pupil-averaged rms of the target phase (micron) over the pupil."""
        ph = np.array(self.target.d_phase)
        m = self.geom.tel.spupil > 0
        v = ph[m] - ph[m].mean()
        return float(np.sqrt(np.mean(v**2)))

"""Precision of the command-matrix MVM against a float64 reconstruction.

The LS command of the reference is computed in float32 (SutraControllerLs::
comp_com, libsutra/src.cpp/sutra_controller_ls.cpp:251-285).  This build also
runs it with the matrix in BF16 or FP8 (E4M3) with one float32 scale per row
and float32 accumulation.  This module measures what that costs on a real
system: the LS command matrix comes from the system's own push-pull
interaction matrix and the float64 filtered inverse (aob_ls_build_cmat), and
the yardstick is the same inverse recomputed in float64 on the host with the
command evaluated in float64.

Two measurements:

* ``command_errors`` -- the relative error ||c_p - c_64|| / ||c_64|| of the
  command of one MVM, for slope vectors taken from the closed loop;
* ``closed_loop`` -- the same seeded closed loop (turbulence, the sensor in
  float32) run once per reconstruction: the float64 host reconstruction, then
  the device MVM in each precision.  It reports the time-averaged
  residual-wavefront rms on the target and the long-exposure Strehl (sinc
  fit), so the relative residual-rms change of each precision is stated
  against the float64 loop.

The comparison is made noise-free, where two loops that differ only by the
rounding of their commands stay on neighbouring trajectories.  With photon
noise they do not: a Poisson draw is a step function of the pixel's mean, so
a change in the last bit of one command (even rounding the float64 command
matrix to float32) selects other counts in some pixel within a few frames,
and from there the two loops see different noise.  With noise the study
therefore compares statistics of whole runs (mean residual, long-exposure
Strehl), not trajectories.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import core
from . import system as S


def fp64_cmat(imat, nfilt):
    """cmat = V diag(1/ev) V^T imat^T with imat^T imat = V diag(ev) V^T, the
    ``nfilt`` smallest eigenvalues dropped (sutra_controller_ls.cpp:116-217),
    entirely in float64 on the host."""
    D = np.asarray(imat, dtype=np.float64)
    ev, V = np.linalg.eigh(D.T @ D)
    inv = np.zeros_like(ev)
    keep = np.arange(ev.size) >= max(int(nfilt), 0)
    keep &= np.abs(ev) > 1e-9
    inv[keep] = 1.0 / ev[keep]
    return (V * inv) @ (V.T @ D.T)


def command_errors(cmat32, cmat64, slopes, precisions=("f32", "bf16", "fp8"), device=0):
    """Relative command error of one device MVM per precision.

    ``slopes``: (k, nslope) float32 slope vectors.  The device command is
    -(cmat @ s) (integrator from zero, gain 1); the float64 one is
    -(cmat64 @ s) with s in float64.  Returns {precision: array of k errors}.
    """
    nactu, nslope = cmat32.shape
    ls = core.LsController(nslope, nactu, device=device)
    ls.set_cmat(cmat32)
    ls.set_gain(1.0)
    zero = np.zeros(nactu, np.float32)
    ref = -(np.asarray(slopes, np.float64) @ cmat64.T)
    out = {}
    for p in precisions:
        ls.set_precision(p)
        err = np.empty(len(slopes))
        for k, s in enumerate(slopes):
            ls.set_com(zero)
            ls.set_centroids(np.ascontiguousarray(s, dtype=np.float32))
            ls.comp_com()
            c = np.array(ls.buffer("com"), dtype=np.float64)
            err[k] = np.linalg.norm(c - ref[k]) / np.linalg.norm(ref[k])
        out[p] = err
    return out


@dataclass
class LoopRun:
    name: str
    residual: np.ndarray  # residual-wavefront rms per iteration (micron)
    slopes: list = field(default_factory=list)  # sampled slope vectors
    strehl_le: float = 0.0  # long exposure at the target wavelength, sinc fit
    strehl_le_peak: float = 0.0  # long exposure, plain peak ratio
    seconds: float = 0.0

    def mean_residual(self, nskip):
        return float(np.mean(self.residual[nskip:]))


def closed_loop(cfg, cmat32, recon, niter, nskip, cmat64=None, sample_every=0, device=0, noise=True):
    """One seeded closed loop of ``niter`` iterations with the given command matrix.

    ``recon``: "fp64" (slopes read back, the integrator evaluated on the host
    in float64 with ``cmat64``, the command written back; every
    ``sample_every``-th slope vector is kept) or a device precision "f32" /
    "bf16" / "fp8" (the loop's own MVM).  The long-exposure image is
    accumulated from iteration ``nskip`` on; ``noise``: the sensor's photon and
    readout noise on or off.
    """
    sy = S.ShAoSystem(cfg, device)
    sy.ls.set_cmat(cmat32)
    res = np.empty(niter)
    run = LoopRun(recon, res)
    gain = float(cfg.gain)
    t0 = time.perf_counter()
    if recon == "fp64":
        if cmat64 is None:
            raise ValueError("closed_loop: the float64 reconstruction needs cmat64")
        com = np.zeros(cmat64.shape[0])
        sy.centro.attach(sy.wfs)
        cen = sy.ls.buffer("centroids")
        volt = sy.ls.buffer("voltage")
    else:
        sy.ls.set_precision(recon)
        sy.close(graph=False)
    for it in range(niter):
        if it == nskip:
            sy.target.reset_le()
        if recon == "fp64":
            sy.atmos.move()
            sy.trace_target()
            sy.trace_wfs()
            sy.wfs.comp_image(noise)
            sy.centro.get_cog(cen.ptr)
            s = np.array(cen, dtype=np.float64)
            com -= gain * (cmat64 @ s)
            sy.ls.set_com(com.astype(np.float32))
            sy.ls.comp_voltage()
            sy.dm.comp_shape(volt.ptr)
            sy.target.comp_image(None, True)
            sy.iter += 1
            if sample_every and it % sample_every == 0:
                run.slopes.append(s.astype(np.float32))
        else:
            sy.next(compute_psf=True, noise=noise)
        res[it] = sy.residual_rms()
    run.seconds = time.perf_counter() - t0
    run.strehl_le = sy.target.strehl(fit=True)[1]
    run.strehl_le_peak = sy.target.strehl(fit=False)[1]
    return run


def study(cfg=None, niter=1000, nskip=200, precisions=("f32", "bf16", "fp8"), sample_every=50, device=0,
          noise_modes=(False, True)):
    """Calibrate ``cfg`` (push-pull imat in one batch, float64 inverse on the
    device), then the command errors and, for each entry of ``noise_modes``,
    the closed loops.  Returns a dict of plain numbers."""
    cfg = cfg or S.saxo40()
    t0 = time.perf_counter()
    sy = S.ShAoSystem(cfg, device)
    sy.calibrate()
    t_cal = time.perf_counter() - t0
    cmat32 = np.ascontiguousarray(sy.cmat, dtype=np.float32)
    cmat64 = fp64_cmat(sy.imat, sy.nfilt)
    cmat_err = float(np.linalg.norm(cmat32 - cmat64) / np.linalg.norm(cmat64))
    nfilt, nslope, nactu = sy.nfilt, sy.ls.nslope, sy.nactu
    del sy
    out = dict(nslope=nslope, nactu=nactu, nfilt=nfilt, niter=niter, nskip=nskip, calib_s=round(t_cal, 3),
               cmat_f32_vs_fp64=cmat_err)
    slopes = None
    for noise in noise_modes:
        key = "noisy" if noise else "noiseless"
        runs = {"fp64": closed_loop(cfg, cmat32, "fp64", niter, nskip, cmat64=cmat64, sample_every=sample_every,
                                    device=device, noise=noise)}
        for p in precisions:
            runs[p] = closed_loop(cfg, cmat32, p, niter, nskip, device=device, noise=noise)
        if noise or slopes is None:
            slopes = runs["fp64"].slopes  # command errors on the slopes of the noisy loop when it runs
        r64 = runs["fp64"].mean_residual(nskip)
        res = dict(fp64=dict(residual_rms_um=r64, strehl_le=runs["fp64"].strehl_le,
                             strehl_le_peak=runs["fp64"].strehl_le_peak, loop_s=round(runs["fp64"].seconds, 3)))
        for p in precisions:
            r = runs[p]
            rp = r.mean_residual(nskip)
            d = r.residual[nskip:] - runs["fp64"].residual[nskip:]
            res[p] = dict(residual_rms_um=rp, residual_rel_change=(rp - r64) / r64,
                          residual_per_iter_rel_rms=float(np.sqrt(np.mean(d**2)) / r64),
                          strehl_le=r.strehl_le, strehl_le_peak=r.strehl_le_peak, loop_s=round(r.seconds, 3))
        out[key] = res
    cerr = command_errors(cmat32, cmat64, slopes, precisions, device=device)
    out["nsamples"] = len(slopes)
    out["command"] = {p: dict(rel_err_median=float(np.median(cerr[p])), rel_err_max=float(np.max(cerr[p])))
                      for p in precisions}
    return out

"""Vectorised float64 NumPy/SciPy restatement of one SH RTC iteration -- the CPU baseline.

Same algorithm as the GPU loop step (and as the reference's comp_image ->
do_centroids -> do_control -> comp_voltage chain, see oracle/sh.py and
oracle/rtc.py for the file:line citations): sub-aperture fields, batched
2-D FFT (scipy.fft, all host cores), |E|^2, binning, flux normalisation,
photon + readout noise (NumPy's generator: the CPU baseline times the
algorithm, it does not reproduce the GPU's Philox stream), weighted CoG with
threshold, float64 MVM (multithreaded BLAS), integrator and clip.
Test infrastructure only (used by the benchmark's CPU-baseline arm).
"""

import os

import numpy as np
import scipy.fft


class CpuShLoop:
    def __init__(self, geom, cmat, centroider="cog", threshold=0.0, weights=None, noise=-1.0,
                 gain=0.4, seed=0, workers=None):
        g = geom
        self.g = g
        self.workers = workers or len(os.sched_getaffinity(0))
        self.cmat = np.asarray(cmat, dtype=np.float64)
        self.kind = centroider
        self.thr = float(threshold)
        npix2 = g.npix * g.npix
        self.w = None if weights is None else np.tile(np.asarray(weights, np.float64).ravel(order="F")[:, None],
                                                      (1, g.nvalid))
        self.noise = float(noise)
        self.gain = float(gain)
        self.rng = np.random.default_rng(seed)
        self.com = np.zeros(self.cmat.shape[0])
        x = np.arange(g.pdiam)
        self.ix = g.validpuppixx[None, None, :] + x[:, None, None]
        self.iy = g.validpuppixy[None, None, :] + x[None, :, None]
        self.amp = g.tel.mpupil[self.ix, self.iy].astype(np.float64)
        self.off = g.halfxy.astype(np.float64)[:, :, None]
        self.scale = 2 * np.pi / g.wavelength_um
        self.flux = g.fluxPerSub.astype(np.float64) * g.nphotons
        p = np.arange(npix2)
        self.px = (p % g.npix).astype(np.float64)[:, None]
        self.py = (p // g.npix).astype(np.float64)[:, None]
        self.cube = np.zeros((g.nvalid, g.nfft, g.nfft), dtype=np.complex128)

    def step(self, phase):
        g = self.g
        ph = phase[self.ix, self.iy].astype(np.float64) * self.scale - self.off
        self.cube[:, :g.pdiam, :g.pdiam] = np.moveaxis(self.amp * np.exp(1j * ph), 2, 0)
        F = scipy.fft.fft2(self.cube, axes=(1, 2), workers=self.workers)
        hr = (F.real**2 + F.imag**2).reshape(g.nvalid, -1)  # [k, y*nfft + x] C-order
        # binmap holds x + y*nfft indexes (Fortran order of the x, y plane)
        hr_f = np.ascontiguousarray(np.swapaxes(hr.reshape(g.nvalid, g.nfft, g.nfft), 1, 2)).reshape(g.nvalid, -1)
        b = hr_f[:, g.binmap].sum(axis=1).T  # [npix2, nvalid]
        s = b.sum(axis=0)
        b = np.where(s != 0, b * self.flux / np.where(s != 0, s, 1.0), b)
        if self.noise > -1:
            b = self.rng.poisson(b).astype(np.float64)
        if self.noise > 0:
            b = b + self.noise * self.rng.standard_normal(b.shape)
        d = b
        if self.kind in ("tcog", "wcog"):
            d = np.where(d > self.thr, d - self.thr, 1e-6)
        if self.kind == "wcog":
            d = d * self.w
        tot = d.sum(axis=0) + 1e-6
        off = g.npix / 2 - 0.5
        sx = ((self.px * d).sum(axis=0) / tot - off) * g.pixsize
        sy = ((self.py * d).sum(axis=0) / tot - off) * g.pixsize
        slopes = np.concatenate([sx, sy])
        err = -(self.cmat @ slopes)
        self.com += self.gain * err
        return np.clip(self.com, -1e6, 1e6)

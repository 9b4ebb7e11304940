"""Centroiders and the least-squares controller in float64 (oracle).

Centre of gravity (CoG)       libsutra/src.cu/sutra_centroider_cog.cu:28-81
Thresholded CoG (tCoG)        libsutra/src.cu/sutra_centroider_tcog.cu:27-81
Weighted CoG (wCoG)           libsutra/src.cu/sutra_centroider_wcog.cu:58-113
Slope ordering                libsutra/src.cu/sutra_centroider_utils.cuh:31-51
LS control law                libsutra/src.cpp/sutra_controller_ls.cpp:251-285
Integrator with modal gains   libsutra/src.cu/sutra_utils.cu:631-639 (mult_int_krnl)
Command delay ring            libsutra/src.cpp/sutra_controller.cpp:26-66,205-218
Latency interpolation         sutra_controller.cpp:232-242
Perturbation voltages         sutra_controller.cpp:266-285
Clip                          sutra_controller.cpp:221-229, libcarma/src.cu/carma_obj.cu:111-131
"""

import numpy as np

UNTIED = 0       # x0..xn, y0..yn (the reference's default)
INTERLEAVED = 1  # x0, y0, x1, y1, ...


def _slot(k, nvalid, order):
    if order == UNTIED:
        return k, k + nvalid
    return 2 * k, 2 * k + 1


def centroids(img, validx, validy, npix, scale, offset, ref=None, kind="cog",
              threshold=0.0, weights=None, order=UNTIED):
    """Slopes and intensities from the sensor image.

    Returns (slopes[2*nvalid], intensities[nvalid], image) where ``image`` is the
    input with the tCoG thresholding written back (the reference kernel stores the
    thresholded pixels into the image, sutra_centroider_tcog.cu:63).
    """
    img = np.array(img, dtype=np.float64, copy=True)
    size = img.shape[0]
    nvalid = len(validx)
    if ref is None:
        ref = np.zeros(2 * nvalid)
    slopes = np.zeros(2 * nvalid)
    inten = np.zeros(nvalid)
    p = np.arange(npix * npix)
    x, y = p % npix, p // npix
    flat = img.reshape(-1, order="F")
    for k in range(nvalid):
        idim = (x + validx[k]) + (y + validy[k]) * size
        ok = idim < size * size
        d = flat[idim[ok]]
        xx, yy = x[ok], y[ok]
        if kind in ("tcog", "wcog"):
            d = np.where(d > threshold, d - threshold, 1e-6)
            if kind == "tcog":
                flat[idim[ok]] = d
        if kind == "wcog":
            d = d * weights[(xx + yy * npix) + k * npix * npix]
        s = d.sum()
        sx = (d * xx).sum()
        sy = (d * yy).sum()
        ix, iy = _slot(k, nvalid, order)
        slopes[ix] = (sx / (s + 1e-6) - offset) * scale - ref[ix]
        slopes[iy] = (sy / (s + 1e-6) - offset) * scale - ref[iy]
        inten[k] = s
    return slopes, inten, flat.reshape(img.shape, order="F")


class LsController:
    """State machine of SutraControllerLs + SutraController (float64)."""

    def __init__(self, nslope, nactu, delay=0.0, gain=0.0):
        self.nslope = nslope
        self.nactu = nactu
        self.cmat = np.zeros((nactu, nslope))
        self.gains = np.ones(nactu)
        self.gain = gain
        self.volt_min, self.volt_max = -1.0e6, 1.0e6
        self.open_loop = False
        self.set_delay(delay)
        self.centroids = np.zeros(nslope)
        nring = 1 if delay <= 0 else int(delay) + 2
        self.ring = [np.zeros(nactu) for _ in range(nring)]
        self.com_clipped = np.zeros(nactu)
        self.perturb = {}  # name -> [array(N, nactu), counter, enabled]

    @property
    def com(self):
        return self.ring[-1]

    def set_delay(self, delay):
        self.delay = delay
        fl = int(delay)
        self.a = delay - fl
        self.b = 1 - self.a

    def comp_com(self):
        if self.open_loop:
            return
        err = -(self.cmat @ self.centroids)
        self.ring[-1] = self.ring[-1] + self.gain * (err * self.gains)

    def clip(self):
        if self.volt_min < self.volt_max:
            self.com_clipped = np.clip(self.com_clipped, self.volt_min, self.volt_max)

    def comp_voltage(self):
        if self.delay > 0:
            self.com_clipped = self.a * self.ring[0] + self.b * self.ring[1]
            # rotate: the oldest buffer receives a copy of the current command
            oldest = self.ring.pop(0)
            oldest[:] = self.ring[-1]
            self.ring.append(oldest)
        else:
            self.com_clipped = self.ring[-1].copy()
        for name in sorted(self.perturb):
            buf, cpt, on = self.perturb[name]
            if on:
                self.com_clipped = self.com_clipped + buf[cpt]
                self.perturb[name][1] = cpt + 1 if cpt < buf.shape[0] - 1 else 0
        self.clip()
        return self.com_clipped


def digitalize(img, dark, flat, max_flux_per_pix, max_pix_value):
    """uint16 camera frame of a sensor image (digitalize_krnl,
    libsutra/src.cu/sutra_wfs.cu:2243-2255): min((img * flat + dark) /
    max_flux_per_pix, 1) * max_pix_value, truncated, saturating at 0 and 65535."""
    v = (np.asarray(img, np.float64) * flat + dark) / float(max_flux_per_pix)
    v = np.minimum(v, 1.0) * float(max_pix_value)
    return np.clip(np.trunc(v), 0, 65535).astype(np.uint16)


def calibrate(raw, dark, flat, lut=None, valid=None, npix=None):
    """Calibrated image (raw[lut] - dark) * flat (calib_krnl,
    libsutra/src.cu/sutra_centroider.cu:108-115), arrays in [x, y] order with the
    lut over the flattened Fortran-order image.  valid = (validx, validy): only
    those windows (npix x npix, or single pixels when npix is None) are
    calibrated, the rest is zero (calibrate_img_validPix,
    sutra_centroider.cpp:194-223)."""
    raw = np.asarray(raw)
    m, n = raw.shape
    flat_raw = raw.ravel(order="F").astype(np.float64)
    idx = np.arange(m * n) if lut is None else np.asarray(lut).ravel()
    cal = (flat_raw[idx] - np.asarray(dark, np.float64).ravel(order="F")) * np.asarray(flat, np.float64).ravel(order="F")
    if valid is None:
        return cal.reshape(m, n, order="F")
    keep = np.zeros(m * n, bool)
    vx, vy = valid
    w = 1 if npix is None else npix
    for x0, y0 in zip(vx, vy):
        xs = (np.arange(w)[:, None] + x0 + (np.arange(w)[None, :] + y0) * m).ravel()
        keep[xs[xs < m * n]] = True
    out = np.where(keep, cal, 0.0)
    return out.reshape(m, n, order="F")

"""Modulated pyramid image formation and slopes in float64 (oracle).

Follows the reference's SutraWfs_PyrHR::comp_generic / comp_modulation
(libsutra/src.cpp/sutra_wfs_pyr_pyrhr.cpp:379-627) and kernels:
  pyrgetpup_krnl  libsutra/src.cu/sutra_wfs.cu:1191-1233  padded field with the modulation tilt
  CarmaFFT dir -1 (cuFFT inverse), libcarma/src.cpp/carma_fft.cpp:175-179
  submask_krnl, submaskpyr_krnl   sutra_wfs.cu:1864-1958  field stop, pyramid phase
  CarmaFFT dir +1 (cuFFT forward), abs2_krnl with factor   sutra_utils.cu:118-142
  pixel transfer: inverse FFT, x sincar, forward FFT, real part
  pyr_bimg_krnl   sutra_wfs.cu:1580-1630   nrebin x nrebin binning
  pyr_fact        normalisation to nphot by the image sum
and SutraCentroiderPyr::get_pyr (libsutra/src.cpp/sutra_centroider_pyr.cpp:101-130,
pyr2slopes_krnl libsutra/src.cu/sutra_centroider_pyr.cu:27-69).

Arrays are indexed [x, y] with x the fastest device index.  The pyramid
phase mask is exp(i halfxy) transposed, as the reference's wfs_init passes it
(shesha/shesha/init/wfs_init.py:203).
"""

import numpy as np

from . import philox


def hr_image(phase, pupil, g, lam_um, weights=None, workers=None):
    """High-resolution modulated image (before the pixel transfer function).

    ``workers``: None runs one modulation point after the other through
    numpy.fft; an integer batches the points through scipy.fft on that many
    threads (the same sums, for the multi-core CPU baseline)."""
    n_fft = g.nfft
    n = phase.shape[0]
    off = int((n_fft - n) / 2.0)
    xx = np.arange(n) - n / 2.0
    mask = g.submask.astype(np.float64) * np.exp(1j * g.halfxy.astype(np.float64)).T
    w = np.ones(g.pyr_cx.size) if weights is None else np.asarray(weights, np.float64)
    mic2rad = 2 * np.pi / lam_um
    hr = np.zeros((n_fft, n_fft))
    base = phase.astype(np.float64) * mic2rad
    amp = pupil.astype(np.float64)
    npts = g.pyr_cx.size
    chunk = 1 if workers is None else max(1, min(npts, 8))
    for p0 in range(0, npts, chunk):
        pts = range(p0, min(p0 + chunk, npts))
        f = np.zeros((len(pts), n_fft, n_fft), dtype=np.complex128)
        for k, p in enumerate(pts):
            phi = float(g.pyr_cx[p]) * xx[:, None] + float(g.pyr_cy[p]) * xx[None, :]
            f[k, off:off + n, off:off + n] = amp * np.exp(1j * (base + phi))
        if workers is None:
            F = np.fft.ifft2(f) * (n_fft * n_fft)
            G = np.fft.fft2(F * mask)
        else:
            import scipy.fft as sf

            F = sf.ifft2(f, workers=workers) * (n_fft * n_fft)
            G = sf.fft2(F * mask, workers=workers)
        for k, p in enumerate(pts):
            hr += w[p] * (G[k].real ** 2 + G[k].imag ** 2)
    return hr


def focal_plane(phase, pupil, g, lam_um, weights=None):
    """The focal plane image of compute_pyrfocalplane: sum over the modulation
    points of w_p |submask x F_p|^2, F_p the inverse FFT of the tilted pupil field
    (abs2 of d_camplifoc after apply_submask, sutra_wfs_pyr_pyrhr.cpp:384-401)."""
    n_fft = g.nfft
    n = phase.shape[0]
    off = int((n_fft - n) / 2.0)
    xx = np.arange(n) - n / 2.0
    sm = g.submask.astype(np.float64)
    w = np.ones(g.pyr_cx.size) if weights is None else np.asarray(weights, np.float64)
    base = phase.astype(np.float64) * (2 * np.pi / lam_um)
    amp = pupil.astype(np.float64)
    out = np.zeros((n_fft, n_fft))
    for p in range(g.pyr_cx.size):
        phi = float(g.pyr_cx[p]) * xx[:, None] + float(g.pyr_cy[p]) * xx[None, :]
        f = np.zeros((n_fft, n_fft), dtype=np.complex128)
        f[off:off + n, off:off + n] = amp * np.exp(1j * (base + phi))
        F = np.fft.ifft2(f) * (n_fft * n_fft) * sm
        out += w[p] * (F.real ** 2 + F.imag ** 2)
    return out


def comp_image(phase, pupil, g, lam_um, nphot, weights=None, noise=-1.0, frame=0, seed=1234, workers=None):
    """Binned, normalised (and optionally noisy) pyramid image [nb, nb]."""
    n_fft = g.nfft
    hr = hr_image(phase, pupil, g, lam_um, weights, workers)
    if workers is None:
        T = np.fft.ifft2(hr) * (n_fft * n_fft)
        hr2 = np.fft.fft2(T * g.sincar.astype(np.float64)).real
    else:
        import scipy.fft as sf

        T = sf.ifft2(hr, workers=workers) * (n_fft * n_fft)
        hr2 = sf.fft2(T * g.sincar.astype(np.float64), workers=workers).real
    r = g.nrebin
    nb = n_fft // r
    b = hr2.reshape(nb, r, nb, r).sum(axis=(1, 3)) / (r * r)
    b = b * (nphot / b.sum())
    if noise > -1:
        lam = b.astype(np.float32).ravel(order="F")
        idx = np.arange(lam.size, dtype=np.uint64)
        v = philox.poisson(lam, idx, frame, seed)
        if noise > 0:
            v = v + noise * philox.gaussian(idx, frame, seed).astype(np.float64)
        b = v.reshape(nb, nb, order="F")
    return b


def slopes(img, validsubsx, validsubsy, nvalid, scale, ref=None, thresh=1e-4, method=1):
    """Pyramid slopes (untied order) and the flux used for each sub-aperture.

    ``method`` as the reference decodes it (Method_CoG(uint8_t),
    libsutra/include/sutra_centroider_pyr.hpp:27-34): 0 sinus global, 1 nosinus
    global (the default, sutra_centroider_pyr.cpp:43), 2 sinus local, 3 nosinus
    local."""
    b = np.asarray(img, np.float64)
    q = [b[validsubsx[k * nvalid:(k + 1) * nvalid], validsubsy[k * nvalid:(k + 1) * nvalid]] for k in range(4)]
    flux = q[0] + q[1] + q[2] + q[3]
    f = flux if method > 1 else np.full(nvalid, flux.sum() / nvalid)
    tx = ((q[0] + q[3]) - (q[1] + q[2])) / f
    ty = ((q[0] + q[2]) - (q[1] + q[3])) / f
    if method % 2 == 0:
        tx, ty = np.sin(np.pi * tx / 2), np.sin(np.pi * ty / 2)
    s = np.concatenate([scale * tx, scale * ty])
    s[np.concatenate([f < thresh, f < thresh])] = 0.0
    if ref is not None:
        s = s - ref
    return s, f

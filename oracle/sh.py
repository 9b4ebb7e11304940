"""Shack-Hartmann image formation in float64 (oracle).

Follows the reference's SutraWfsSH::comp_generic / fill_binimage
(libsutra/src.cpp/sutra_wfs_sh.cpp:337-621) and its kernels:
  camplipup_krnl   libsutra/src.cu/sutra_wfs.cu:27-53   field in each sub-aperture
  cuFFT forward    sutra_wfs_sh.cpp:393 (carma_fft.cpp:175-179, dir=1 -> CUFFT_FORWARD)
  abs2c_krnl       libsutra/src.cu/sutra_utils.cu:144-168
  fillbincube_krnl sutra_wfs.cu:369-414   binning through ``binmap``
  reduce2          sutra_wfs.cu:556-590   per-sub-aperture sum
  subapnorm_krnl   sutra_utils.cu:170-193 flux normalisation (skipped when the sum is 0)
  prng('P'), prng('N', noise, 1)  sutra_wfs_sh.cpp:580-587 photon + readout noise
  bimg_krnl        sutra_wfs.cu:183-229   scatter to the 2-D image
The natural-guide-star path is restated, with the field of view extended
(Ntot > Nfft) or not, with or without the focal-plane field stop; the kernel
convolution is not.

Array convention: every 2-D numpy array ``a`` here is indexed ``a[x, y]`` with
``x`` the fastest-varying device index (the reference passes F-ordered arrays).
"""

import numpy as np

from . import philox


def field_stop_field(phase, pupil, scale, submask):
    """Full-pupil field filtered by the focal-plane field stop, normalised.

    fsamplipup_krnl (libsutra/src.cu/sutra_wfs.cu:148-166) puts pupil *
    exp(i phase scale) in the top-left npup x npup corner of an n x n array;
    a forward FFT, the fftshifted mask (submask_krnl, :1868-1876) and an
    unnormalised inverse FFT follow (sutra_wfs_sh.cpp:366-391); the complex
    camplipup_krnl (:87-117) divides by n^2."""
    n = submask.shape[0]
    npup = phase.shape[0]
    f = np.zeros((n, n), dtype=np.complex128)
    f[:npup, :npup] = pupil.astype(np.float64) * np.exp(1j * phase.astype(np.float64) * scale)
    return np.fft.ifft2(np.fft.fft2(f) * submask)  # = unnormalised inverse / n^2


def spot_field(phase, pupil, puppixx, puppixy, offsets, scale, pdiam, nfft, field=None):
    """Complex field cube [nfft, nfft, nvalid], non-zero in the top-left pdiam x pdiam.

    ``field``: the field-stop-filtered full-pupil field; the sub-aperture field is
    then field * exp(-i offset) (camplipup_krnl, sutra_wfs.cu:87-117)."""
    nvalid = len(puppixx)
    x = np.arange(pdiam)
    ix = puppixx[None, None, :] + x[:, None, None]
    iy = puppixy[None, None, :] + x[None, :, None]
    cube = np.zeros((nfft, nfft, nvalid), dtype=np.complex128)
    if field is not None:
        cube[:pdiam, :pdiam, :] = field[ix, iy] * np.exp(-1j * offsets.astype(np.float64)[:, :, None])
        return cube
    ph = phase[ix, iy].astype(np.float64) * scale - offsets.astype(np.float64)[:, :, None]
    amp = pupil[ix, iy].astype(np.float64)
    cube[:pdiam, :pdiam, :] = amp * np.exp(1j * ph)
    return cube


def hr_images(field):
    """|FFT|^2 of every sub-aperture (forward transform, unnormalised)."""
    return np.abs(np.fft.fft2(field, axes=(0, 1))) ** 2


def bin_cube(hr, binmap, hrmap=None, ntot=None):
    """bincube[p, k] = sum_r hr_flat[binmap[r, p], k] with hr_flat[x + y*nfft].

    With an extended field of view (ntot > nfft) the spot is first written into
    an ntot x ntot image at ``hrmap`` (indexfill_krnl, libsutra/src.cu/
    sutra_wfs.cu:462-473: element i of the spot goes to hrmap[i], the rest of
    the image is zero; sutra_wfs_sh.cpp:409-481) and binmap indexes that image."""
    nfft = hr.shape[0]
    flat = hr.reshape(nfft * nfft, -1, order="F")
    if ntot is not None and int(ntot) != nfft:
        big = np.zeros((int(ntot) * int(ntot), flat.shape[1]), dtype=flat.dtype)
        big[np.asarray(hrmap).ravel(), :] = flat
        flat = big
    return flat[binmap, :].sum(axis=0)


def normalise(bincube, flux_per_sub, nphot):
    """Scale each sub-aperture to flux_per_sub * nphot photons; returns (cube, raw sums)."""
    sums = bincube.sum(axis=0)
    out = bincube.copy()
    nz = sums != 0
    out[:, nz] = bincube[:, nz] * flux_per_sub[nz] / sums[nz] * nphot
    return out, sums


def add_noise(bincube, noise, seed, frame):
    """Photon noise when noise > -1, then readout noise of rms ``noise`` when noise > 0."""
    out = bincube.astype(np.float64)
    idx = np.arange(out.size, dtype=np.uint64).reshape(out.shape, order="F")
    if noise > -1:
        # the device samples the float32 mean, as the reference's curand_poisson does
        out = philox.poisson(out.astype(np.float32).astype(np.float64), idx, frame, seed)
    if noise > 0:
        out = out.astype(np.float32).astype(np.float64) + np.float32(noise) * philox.gaussian(idx, frame, seed)
    return out


def bin_image(bincube, validsubsx, validsubsy, npix, nxsub):
    """Scatter sub-aperture cubes into the npix*nxsub square sensor image."""
    size = npix * nxsub
    img = np.zeros((size, size), dtype=bincube.dtype)
    p = np.arange(npix * npix)
    px, py = p % npix, p // npix
    for k in range(bincube.shape[1]):
        img[validsubsx[k] + px, validsubsy[k] + py] = bincube[:, k]
    return img


def comp_image(phase, pupil, g, scale, nphot, noise=-1.0, seed=1234, frame=0):
    """Full SH image: returns (bincube, binimg, intensities) in float64.

    ``g`` is an object/dict with the SH geometry fields (validpuppixx/y,
    halfxy, binmap, fluxPerSub, validsubsx/y, pdiam, nfft, npix, nxsub).
    """
    get = (lambda k: g[k]) if isinstance(g, dict) else (lambda k: getattr(g, k))
    try:
        submask = get("submask")
    except (KeyError, AttributeError):
        submask = None
    fs = None if submask is None else field_stop_field(phase, pupil, scale, np.asarray(submask, np.float64))
    field = spot_field(phase, pupil, get("validpuppixx"), get("validpuppixy"), get("halfxy"),
                       scale, int(get("pdiam")), int(get("nfft")), field=fs)
    cube = bin_cube(hr_images(field), get("binmap"), get("hrmap"), int(get("ntot")))
    cube, sums = normalise(cube, get("fluxPerSub").astype(np.float64), nphot)
    cube = add_noise(cube, noise, seed, frame)
    img = bin_image(cube, get("validsubsx"), get("validsubsy"), int(get("npix")), int(get("nxsub")))
    return cube, img, sums


def slopes_geom(phase, pupil, phasemap, flux_per_sub, subapd, nphase, kind=0, ttprojmat=None):
    """Geometric slopes of the phase (SutraWfs::slopes_geom, libsutra/src.cpp/
    sutra_wfs.cpp:199-251) in float64; the reference's float alpha is kept.

    ``phase`` / ``pupil``: the sensor's n x n screen and pupil ([x, y]);
    ``phasemap``: [nphase^2, nvalid] indexes into the Fortran-flattened screen;
    ``ttprojmat``: [nphase^2, 2 nvalid].
      kind 0  reduce_phasex / reduce_phasey (sutra_wfs.cu:866-910)
      kind 1  derive_phasex / derive_phasey (sutra_wfs.cu:912-970)
      kind 2  project_gather + two strided-batched GEMMs (sutra_wfs.cu:1049-1082)
    """
    n = int(nphase)
    ph = np.asarray(phase, np.float64).ravel(order="F")
    pup = np.asarray(pupil, np.float64).ravel(order="F")
    pm = np.asarray(phasemap)
    nvalid = pm.shape[1]
    alpha = float(np.float32(0.206265 / float(np.float32(subapd)) * n / (n - 1)))
    v = ph[pm]  # [n^2, nvalid]
    if kind == 0:
        rows = v.reshape(n, n, nvalid, order="F")  # rows[a, b, k]: sample a + b n
        sx = (rows[n - 1, :, :] - rows[0, :, :]).sum(axis=0) / n * alpha
        sy = (rows[:, n - 1, :] - rows[:, 0, :]).sum(axis=0) / n * alpha
    elif kind == 1:
        m = pup[pm]
        a = np.arange(n * n) % n
        i = np.arange(n * n)
        ip1, im1 = np.minimum(i + 1, n * n - 1), np.maximum(i - 1, 0)
        dx = np.where((a == 0)[:, None], v[ip1] - v, np.where((a == n - 1)[:, None], v - v[im1], v[ip1] - v[im1]))
        ipn, imn = np.minimum(i + n, n * n - 1), np.maximum(i - n, 0)
        dy = np.where((i < n)[:, None], v[ipn] - v,
                      np.where((i >= n * (n - 1))[:, None], v - v[imn], v[ipn] - v[imn]))
        f = np.asarray(flux_per_sub, np.float64)
        sx = (dx * m).sum(axis=0) / n * alpha / f / 2
        sy = (dy * m).sum(axis=0) / n / 2 * alpha / f
    elif kind == 2:
        M = np.asarray(ttprojmat, np.float64)
        sx = (M[:, :nvalid] * v).sum(axis=0)
        sy = (M[:, nvalid:] * v).sum(axis=0)
    else:
        raise ValueError("slopes_geom: kind must be 0, 1 or 2")
    return np.concatenate([sx, sy])

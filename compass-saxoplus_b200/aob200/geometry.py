"""Host-side geometry builder for Shack-Hartmann and pyramid wavefront sensors.

This runs once at initialisation and produces the integer maps and float
tables that the GPU kernels consume (valid sub-apertures, pixel binning maps,
phase offsets, flux per sub-aperture, pyramid masks and modulation points).
It restates the reference's geometry initialisation so that every integer map
is identical to the reference's output on the same parameters:

  shesha/shesha/init/geom_init.py   geom_init            :999-1052
                                    init_wfs_size        :176-392
                                    compute_nphotons     :394-470
                                    init_pyrhr_geom      :472-732
                                    init_sh_geom         :735-996
  shesha/shesha/util/make_pupil.py  make_pupil_generic   :144-238 (no spiders)
  shesha/shesha/util/utilities.py   fft_goodsize :33, pad_array :86, dist :100,
                                    rebin :23

Array conventions follow the reference: 2-D maps are numpy arrays whose first
index is the fastest-varying index of the device buffer (the reference hands
them to the GPU in Fortran order).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

RAD2ARCSEC = 3600.0 * 360.0 / (2 * np.pi)
ARCSEC2RAD = 2.0 * np.pi / (360.0 * 3600.0)

# The reference stores every user float parameter as a numpy float32 scalar
# (config_setter_utils.py enforce_float), so the size arithmetic below runs in
# float32 exactly as it does there.
f32 = np.float32


def fft_goodsize(s: int) -> int:
    """Next power of two strictly above ``s`` (utilities.py:33)."""
    return 2 ** (int(np.log2(s)) + 1)


def radial_distance(dim: int, xc: float = -1, yc: float = -1) -> np.ndarray:
    """Euclidean distance of each pixel to (xc, yc); columns run along x (utilities.py:100)."""
    if xc < 0:
        xc = int(dim / 2.0)
    if yc < 0:
        yc = int(dim / 2.0)
    dx = np.tile(np.arange(dim) - xc, (dim, 1))
    dy = np.tile(np.arange(dim) - yc, (dim, 1)).T
    return np.sqrt(dx**2 + dy**2)


def pad_center(a: np.ndarray, n: int) -> np.ndarray:
    """Embed ``a`` in an n x n float64 zero array, offset by (n - size)//2 (utilities.py:86)."""
    d1 = (n - a.shape[0]) // 2
    d2 = (n - a.shape[1]) // 2
    out = np.zeros((n, n))
    out[d1:d1 + a.shape[0], d2:d2 + a.shape[1]] = a
    return out


def block_mean(a: np.ndarray, shape) -> np.ndarray:
    """Mean over non-overlapping blocks down to ``shape`` (utilities.py:23)."""
    sh = shape[0], a.shape[0] // shape[0], shape[1], a.shape[1] // shape[1]
    return np.mean(a.reshape(sh), axis=(1, 3))


def disc_pupil(dim: int, pupd: float, cobs: float, xc: float, yc: float) -> np.ndarray:
    """Binary circular aperture with a central obstruction (make_pupil.py:144-188)."""
    d = radial_distance(dim, xc, yc)
    pup = (d < (pupd + 1.0) / 2).astype(np.float32)
    if cobs > 0:
        pup -= (radial_distance(dim, xc, yc) < (pupd * cobs + 1.0) * 0.5).astype(np.float32)
    return pup


@dataclass
class TelescopeGeometry:
    """Pupil arrays shared by every sensor (geom_init.py:999-1052)."""

    pupdiam: int
    ssize: int
    cent: float
    p1: int
    p2: int
    n: int
    n1: int
    n2: int
    spupil: np.ndarray
    ipupil: np.ndarray
    mpupil: np.ndarray
    diam: float
    cobs: float

    @property
    def pixsize(self) -> float:
        return self.diam / self.pupdiam


def telescope_geometry(pupdiam: int, diam: float, cobs: float, padding: int = 2) -> TelescopeGeometry:
    ssize = int(2 ** np.ceil(np.log2(pupdiam) + 1))
    cent = ssize / 2 - 0.5
    p1 = int(np.ceil(cent - pupdiam / 2.0))
    p2 = int(np.floor(cent + pupdiam / 2.0))
    pupdiam = p2 - p1 + 1
    n = pupdiam + 2 * padding
    c = pupdiam / 2.0 - 0.5
    spupil = disc_pupil(pupdiam, pupdiam, cobs, c, c).astype(np.float32)
    return TelescopeGeometry(
        pupdiam=pupdiam, ssize=ssize, cent=cent, p1=p1, p2=p2, n=n,
        n1=p1 - padding, n2=p2 + padding, spupil=spupil,
        ipupil=pad_center(spupil, ssize).astype(np.float32),
        mpupil=pad_center(spupil, n).astype(np.float32), diam=diam, cobs=cobs,
    )


def compute_nphotons(kind: str, ittime: float, optthroughput: float, diam: float,
                     cobs: float = 0.0, nxsub: int = 0, zerop: float = 0.0,
                     gsmag: float = 0.0) -> float:
    """Photons per sub-aperture (SH) or per pupil (pyramid) per frame (geom_init.py:394-470)."""
    ittime, optthroughput, diam, cobs = f32(ittime), f32(optthroughput), f32(diam), f32(cobs)
    zerop, gsmag = f32(zerop), f32(gsmag)
    if kind == "pyrhr":
        surface = np.pi / 4.0 * (1 - cobs**2.0) * diam**2.0
    elif kind == "sh":
        if zerop == 0:
            zerop = f32(1e11)
        surface = (diam / nxsub) ** 2.0
    else:
        raise ValueError(f"unknown sensor kind {kind!r}")
    return float(zerop * 10.0 ** (-0.4 * gsmag) * ittime * optthroughput * surface)


@dataclass
class ShParams:
    """User-facing SH parameters (the subset of ParamWfs the hot path reads)."""

    nxsub: int
    npix: int
    pixsize: float
    wavelength_um: float
    fracsub: float = 0.5
    gsmag: float = 8.0
    zerop: float = 1e11
    optthroughput: float = 0.5
    noise: float = -1.0
    fssize: float = 0.0   # field-stop size in arcsec (0: no field stop)
    fstop: str = "round"  # field-stop shape: "round" or "square"


@dataclass
class ShGeometry:
    """Everything ``SHWFS.load_arrays`` takes, plus the derived sizes."""

    nxsub: int
    npix: int
    pdiam: int
    nfft: int
    ntot: int
    nrebin: int
    nvalid: int
    pixsize: float
    qpixsize: float
    subapd: float
    nphotons: float
    isvalid: np.ndarray
    fluxPerSub_grid: np.ndarray
    fluxPerSub: np.ndarray
    validsubsx: np.ndarray
    validsubsy: np.ndarray
    validpuppixx: np.ndarray
    validpuppixy: np.ndarray
    phasemap: np.ndarray
    binmap: np.ndarray
    halfxy: np.ndarray
    hrmap: np.ndarray
    ttprojmat: np.ndarray
    wavelength_um: float
    tel: Optional[TelescopeGeometry] = field(default=None, repr=False)
    submask: Optional[np.ndarray] = None  # field-stop mask (fftshifted), None without field stop


def _sh_sizes(p: ShParams, pdiam: int, diam: float):
    """FFT support, rebin factor and pixel scale for a SH sensor (geom_init.py:296-349)."""
    lam = p.wavelength_um * 1.0e-6
    pdiam = np.int32(pdiam)  # the reference holds it as an int32 scalar
    pix_req = f32(p.pixsize)
    subapdiam = f32(diam) / float(p.nxsub)
    nrebin = int(2 * subapdiam * pix_req / lam / RAD2ARCSEC) + 1
    nrebin = max(2, nrebin)
    nfft = fft_goodsize(int(pdiam / subapdiam * nrebin / pix_req * RAD2ARCSEC * lam))
    qpixsize = (pdiam * lam / subapdiam * RAD2ARCSEC) / nfft
    ratio = pix_req / qpixsize
    nrebin = int(ratio) + 1 if ratio - int(ratio) > 0.5 else int(ratio)
    pixsize = nrebin * qpixsize
    if pixsize * p.npix > qpixsize * nfft:
        ntot = fft_goodsize(int(pixsize * p.npix / qpixsize) + 1)
    else:
        ntot = nfft
    if ntot % 2 != nfft % 2:
        ntot += 1
    return nfft, ntot, nrebin, float(pixsize), float(qpixsize)


def _focal_mask(size: int, radius: int, shape: str) -> np.ndarray:
    """Round or square field stop of ``radius`` pixels centred in a size x size
    focal plane (geom_init.py:513-520 for the pyramid, :978-988 for the SH)."""
    if shape == "round":
        return radial_distance(size, xc=size / 2.0 - 0.5, yc=size / 2.0 - 0.5) < radius
    if shape == "square":
        ij = np.indices((size, size)) + 1
        fx = ij[1] - (size + 1.0) / 2.0
        fy = ij[0] - (size + 1.0) / 2.0
        return (np.abs(fx) <= radius) * (np.abs(fy) <= radius)
    raise ValueError("field stop must be 'round' or 'square'")


def _tt_projection(mask_t: np.ndarray, i0: int, j0: int, nph: int):
    """Tip/tilt slope projection vectors of one sub-aperture (geom_init.py:790-807)."""
    sub = mask_t[i0:i0 + nph, j0:j0 + nph]
    sx = np.zeros((nph, nph), dtype=np.float32)
    sy = np.zeros((nph, nph), dtype=np.float32)
    left = np.zeros_like(sub)
    right = np.zeros_like(sub)
    up = np.zeros_like(sub)
    down = np.zeros_like(sub)
    left[:, 1:] = sub[:, :-1]
    right[:, :-1] = sub[:, 1:]
    up[1:, :] = sub[:-1, :]
    down[:-1, :] = sub[1:, :]
    sx[:] = (left - right) * sub
    sy[:] = (up - down) * sub
    den_x = -sx.cumsum(axis=1).sum()
    den_y = -sy.cumsum(axis=0).sum()
    if den_x == 0 or den_y == 0:
        return None
    return (sx / den_x).flatten(), (sy / den_y).flatten()


def sh_geometry(p: ShParams, pupdiam: int, diam: float = 8.0, cobs: float = 0.14,
                ittime: float = 0.001, tel: Optional[TelescopeGeometry] = None) -> ShGeometry:
    """Build the full SH geometry for a sensor whose sub-apertures tile ``pupdiam`` pixels.

    Mirrors ``init_wfs_geom`` -> ``init_wfs_size`` -> ``init_sh_geom`` for the case where
    the pupil diameter in pixels is given (geom_init.py:140-169,176-392,735-996).
    """
    pdiam = pupdiam // p.nxsub
    if (pdiam * p.nxsub) % 2:
        pdiam += 1
    nfft, ntot, nrebin, pixsize, qpixsize = _sh_sizes(p, pdiam, diam)
    if tel is None:
        tel = telescope_geometry(pdiam * p.nxsub, diam, cobs)
    nx = p.nxsub

    starts = np.linspace(0, tel.pupdiam, nx + 1)[:-1].astype(np.int64) + 2
    flux = np.zeros((nx, nx), dtype=np.float32)
    for i in range(nx):
        for j in range(nx):
            flux[i, j] = np.sum(tel.mpupil[starts[i]:starts[i] + pdiam, starts[j]:starts[j] + pdiam])
    flux = flux / pdiam**2.0
    isvalid = (flux >= f32(p.fracsub)).astype(np.int32)
    nvalid = int(isvalid.sum())
    vy, vx = np.where(isvalid.T)
    vx = vx.astype(np.int32)
    vy = vy.astype(np.int32)

    grid = np.arange(tel.n)[None, :] + np.arange(tel.n)[:, None] * tel.n
    phasemap = np.zeros((pdiam * pdiam, nvalid), dtype=np.int32)
    ttproj = np.zeros((pdiam * pdiam, 2 * nvalid), dtype=np.float32)
    mask_t = tel.mpupil.T
    for k in range(nvalid):
        i0 = starts[vy[k]]
        j0 = starts[vx[k]]
        phasemap[:, k] = grid[i0:i0 + pdiam, j0:j0 + pdiam].flatten()
        tt = _tt_projection(mask_t, i0, j0, pdiam)
        if tt is not None:
            ttproj[:, k] = tt[0]
            ttproj[:, k + nvalid] = tt[1]
    ttproj = ttproj * tel.pupdiam / diam * RAD2ARCSEC * 1e-6

    # half-pixel phase ramp so that the spot is centred between 4 pixels
    ramp = np.linspace(0, 2 * np.pi, nfft + 1)[0:pdiam] / 2.0
    ramp = np.tile(ramp, (pdiam, 1))
    ramp = ramp + ramp.T
    if p.npix % 2 == 1 and nrebin % 2 == 1:
        halfxy = np.zeros((pdiam, pdiam), dtype=np.float32)
    else:
        halfxy = ramp.astype(np.float32)

    if ntot != nfft:
        # extended field of view (geom_init.py:847-867): the nfft x nfft spot sits
        # in the middle of an ntot x ntot image, both centred on pixel 0 by the
        # half-size rolls; hrmap lists the spot's pixel positions in that image
        # (row-major order, which is the order the reference's indexfill reads)
        lo = int((ntot - nfft) / 2.0)
        block = np.zeros((ntot, ntot))
        block[lo:lo + nfft, lo:lo + nfft] = 1
        block = np.roll(np.roll(block, ntot // 2, axis=0), ntot // 2, axis=1)
        hrmap = np.flatnonzero(block).astype(np.int32).reshape(-1, 1)
    else:
        hrmap = np.zeros((2, 2), dtype=np.int32)  # set even if unused, as the reference does

    span = nrebin * p.npix
    lo = int((ntot - span) / 2.0) + (1 if span % 2 != ntot % 2 else 0)
    # binned pixel label of each high-resolution pixel, 0 = outside the sensor field
    label = np.zeros((ntot, ntot))
    iy, ix = np.indices((span, span))
    label[lo:lo + span, lo:lo + span] = (ix // nrebin) + (iy // nrebin) * p.npix + 1
    label = np.roll(label, ntot // 2, axis=0)
    label = np.roll(label, ntot // 2, axis=1)
    flat = np.arange(ntot)[None, :] + np.arange(ntot)[:, None] * ntot
    binmap = np.zeros((nrebin * nrebin, p.npix * p.npix))
    for q in range(p.npix * p.npix):
        binmap[:, q] = flat[label == q + 1]
    binmap = binmap.astype(np.int32)

    nphot = compute_nphotons("sh", ittime, p.optthroughput, diam, nxsub=nx,
                             zerop=p.zerop, gsmag=p.gsmag)
    submask = None
    if p.fssize != 0:
        # field stop in the focal plane of the full pupil (geom_init.py:973-995)
        fftsize = fft_goodsize(tel.mpupil.shape[0])
        fspixsize = (tel.pupdiam * (p.wavelength_um * 1.0e-6) / diam * RAD2ARCSEC) / fftsize
        rf = int(p.fssize / fspixsize / 2.0)
        submask = np.fft.fftshift(_focal_mask(fftsize, rf, p.fstop) * 1.0)
    return ShGeometry(
        nxsub=nx, npix=p.npix, pdiam=pdiam, nfft=nfft, ntot=ntot, nrebin=nrebin,
        nvalid=nvalid, pixsize=pixsize, qpixsize=qpixsize, subapd=diam / nx,
        nphotons=nphot, isvalid=isvalid, fluxPerSub_grid=flux,
        fluxPerSub=flux.T[np.where(isvalid.T > 0)].copy(),
        validsubsx=(vx * p.npix).astype(np.int32), validsubsy=(vy * p.npix).astype(np.int32),
        validpuppixx=(vx * pdiam + 2).astype(np.int32),
        validpuppixy=(vy * pdiam + 2).astype(np.int32),
        phasemap=phasemap, binmap=binmap, halfxy=halfxy, hrmap=hrmap, ttprojmat=ttproj,
        wavelength_um=p.wavelength_um, tel=tel, submask=submask,
    )


@dataclass
class PyrParams:
    nxsub: int
    wavelength_um: float
    ampl: float = 3.0
    npts: int = 24
    pup_sep: int = -1
    fssize: float = 0.0
    fstop: str = "round"
    fracsub: float = 0.0001
    gsmag: float = 6.0
    zerop: float = 1e11
    optthroughput: float = 0.5
    noise: float = -1.0
    npupils: int = 4


@dataclass
class PyrGeometry:
    nxsub: int
    pdiam: int
    nfft: int
    ntot: int
    nrebin: int
    nvalid: int
    qpixsize: float
    pixsize: float
    nphotons: float
    npix: int
    halfxy: np.ndarray
    pyr_cx: np.ndarray
    pyr_cy: np.ndarray
    sincar: np.ndarray
    submask: np.ndarray
    validsubsx: np.ndarray
    validsubsy: np.ndarray
    isvalid: np.ndarray
    fluxPerSub: np.ndarray
    phasemap: np.ndarray
    wavelength_um: float
    tel: Optional[TelescopeGeometry] = field(default=None, repr=False)


def pyr_geometry(p: PyrParams, pupdiam: int, diam: float = 8.0, cobs: float = 0.14,
                 ittime: float = 0.001) -> PyrGeometry:
    """Build the high-resolution pyramid geometry (geom_init.py:140-169,356-375,472-732)."""
    lam = p.wavelength_um * 1.0e-6
    diam = f32(diam)
    pdiam = pupdiam // p.nxsub
    if (pdiam * p.nxsub) % 2:
        pdiam += 1
    ptot = pdiam * p.nxsub
    m = 3
    nfft = int(2 ** np.ceil(np.log2(m * ptot)))
    nrebin = ptot // p.nxsub
    while nfft % nrebin != 0:
        nrebin += 1
        ptot = nrebin * p.nxsub
        nfft = int(2 ** np.ceil(np.log2(m * ptot)))
    qpix64 = (np.int32(ptot) * lam / diam * RAD2ARCSEC) / nfft
    # stored as float32 scalars by the reference's parameter setters
    qpixsize = f32(qpix64)
    pixsize = f32(qpix64 * nrebin)
    pdiam = ptot // p.nxsub
    tel = telescope_geometry(pdiam * p.nxsub, diam, cobs, padding=nrebin)
    npix = pdiam
    ntot = tel.n
    size = nfft

    rf = int(f32(p.fssize) / qpixsize / 2.0)
    submask = np.fft.fftshift(_focal_mask(size, rf, p.fstop) * 1.0)

    pup_sep = int(p.nxsub) if p.pup_sep == -1 else p.pup_sep
    gy = np.tile(np.arange(size) - size / 2, (size, 1))
    gx = gy.T
    pangle = pup_sep * nrebin
    k = np.arange(p.npupils)
    centers = pangle / np.sin(np.pi / p.npupils) * np.c_[
        np.cos((2 * k + 1) * np.pi / p.npupils), np.sin((2 * k + 1) * np.pi / p.npupils)]
    if p.npupils == 4:
        centers = np.round(centers[[1, 0, 2, 3], :]).astype(np.int32)
    mis = np.zeros((p.npupils, 2), dtype=np.float32)
    faces = np.asarray([(c[0] + mm[0]) * gx + (c[1] + mm[1]) * gy for c, mm in zip(centers, mis)])
    pyr = 2 * np.pi / size * np.min(faces, axis=0)
    halfxy = np.fft.fftshift(pyr.T)

    pup = np.zeros((size, size))
    h = tel.n // 2
    pup[size // 2 - h:size // 2 + h, size // 2 - h:size // 2 + h] = tel.mpupil
    stacked = None
    for q in range(p.npupils):
        shifted = np.roll(pup, tuple((centers[q] + mis[q]).astype(np.int32)), (0, 1))
        lowres = block_mean(shifted.copy(), [size // nrebin, size // nrebin])
        back = np.roll(lowres >= f32(p.fracsub), tuple((-centers[q] / nrebin).astype(np.int32)), (0, 1))
        stacked = back if stacked is None else stacked + back
    if p.npupils == 4:
        centers = centers[[2, 1, 3, 0], :]
    rows, cols = [], []
    for q in range(p.npupils):
        wh = np.where(np.roll(stacked, tuple((centers[q] / nrebin).astype(np.int32)), (0, 1)))
        rows.append(wh[0].astype(np.int32))
        cols.append(wh[1].astype(np.int32))
    nvalid = rows[0].size
    rows = np.asarray(rows).flatten()
    cols = np.asarray(cols).flatten()
    _, first = np.unique(np.c_[rows, cols], axis=0, return_index=True)
    order = np.sort(first)
    validsubsx = rows[order]
    validsubsy = cols[order]

    scale = 2 * np.pi / np.int32(size) * (lam / diam) / ((np.pi * qpixsize) / (3600 * 180)) * f32(p.ampl)
    ang = np.arange(p.npts) * 2.0 * np.pi / p.npts
    cx = scale * np.sin(ang)
    cy = scale * np.cos(ang)

    nphot = compute_nphotons("pyrhr", ittime, p.optthroughput, diam, cobs=cobs,
                             zerop=p.zerop, gsmag=p.gsmag)

    sy = np.tile(np.arange(size) - size // 2, (size, 1))
    sx = sy.T
    sincar = np.fft.fftshift(np.sinc(sx * 1.0 / size) * np.sinc(sy * 1.0 / size)).astype(np.float32)

    a = size // nrebin
    b = tel.n // nrebin
    pupvalid = stacked[a // 2 - b // 2:a // 2 + b // 2, a // 2 - b // 2:a // 2 + b // 2]
    isvalid = pupvalid.T.astype(np.int32)
    vsx = np.where(pupvalid)[0].astype(np.int32)
    vsy = np.where(pupvalid)[1].astype(np.int32)

    starts = np.arange(p.nxsub + 2) * npix
    flux = np.zeros((p.nxsub + 2, p.nxsub + 2), dtype=np.float32)
    for i in range(p.nxsub + 2):
        for j in range(p.nxsub + 2):
            flux[i, j] = np.sum(tel.mpupil[starts[i]:starts[i] + npix, starts[j]:starts[j] + npix])
    flux = flux / p.nxsub**2.0

    grid = np.arange(tel.n)[None, :] + np.arange(tel.n)[:, None] * tel.n
    phasemap = np.zeros((npix * npix, nvalid), dtype=np.int32)
    for k2 in range(len(vsx)):
        i0 = starts[vsy[k2]]
        j0 = starts[vsx[k2]]
        phasemap[:, k2] = grid[i0:i0 + npix, j0:j0 + npix].flatten("C")

    return PyrGeometry(
        nxsub=p.nxsub, pdiam=pdiam, nfft=nfft, ntot=ntot, nrebin=nrebin, nvalid=nvalid,
        qpixsize=float(qpixsize), pixsize=float(pixsize), nphotons=nphot, npix=npix,
        halfxy=halfxy.astype(np.float32), pyr_cx=cx.astype(np.float32),
        pyr_cy=cy.astype(np.float32), sincar=sincar, submask=submask.astype(np.float32),
        validsubsx=validsubsx,
        validsubsy=validsubsy, isvalid=isvalid,
        fluxPerSub=flux.T[np.where(isvalid.T > 0)].copy(), phasemap=phasemap,
        wavelength_um=p.wavelength_um, tel=tel,
    )

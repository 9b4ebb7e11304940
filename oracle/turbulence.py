"""Turbulence extrusion, raytrace, DM shape and PSF in float64 (oracle).

extrusion_AB   shesha/shesha/util/iterkolmo.py:201-267 (numpy SVD factorisation)
extrude        libsutra/src.cpp/sutra_tscreen.cpp:137-220 (direction conventions)
raytrace       libsutra/src.cu/sutra_target.cu:25-70 (bilinear, G = 1, no rotation)
dm_shape       libsutra/src.cu/sutra_dm.cu:83-133 (sum of influence patches)
psf / strehl   libsutra/src.cpp/sutra_source.cpp:397-515 (peak, no sinc fit)
"""

import numpy as np


def factor_AB(zz, xz, xx):
    """A, B from the covariances exactly as iterkolmo.AB does (SVD pseudo-inverse)."""
    U, s, V = np.linalg.svd(zz)
    s1 = s.copy()
    s1[-1] = 1
    s1 = 1.0 / s1
    s1[-1] = 0
    zz1 = (U * s1) @ V
    A = xz @ zz1
    bbt = xx - A @ xz.T
    U1, sv, _ = np.linalg.svd(bbt)
    B = U1 * np.sqrt(sv)
    return A, B


def extrude(screen, A, B, istx, isty, amplitude, noise, direction):
    """One extrusion of ``screen`` (numpy [x, y], x fastest) with the given N(0,1) noise."""
    n = screen.shape[0]
    flat = screen.reshape(-1, order="F").astype(np.float64)
    ist = istx if direction in (1, -1) else isty
    x0 = n - 1 if direction in (1, -2) else n * (n - 1)
    z = flat[ist] - flat[x0]
    y = A.astype(np.float64) @ z + amplitude * (B.astype(np.float64) @ noise) + flat[x0]
    out = np.empty_like(screen, dtype=np.float64)
    s = screen.astype(np.float64)
    if direction == 1:
        out[:-1, :] = s[1:, :]
        out[-1, :] = y
    elif direction == -1:
        out[1:, :] = s[:-1, :]
        out[0, :] = y[::-1]
    elif direction == 2:
        out[:, :-1] = s[:, 1:]
        out[:, -1] = y
    else:
        out[:, 1:] = s[:, :-1]
        out[:, 0] = y[::-1]
    return out


def raytrace(nx, ny, screens, xoffs, yoffs):
    out = np.zeros((nx, ny))
    x = np.arange(nx, dtype=np.float32)[:, None] * np.ones((1, ny), np.float32)
    y = np.arange(ny, dtype=np.float32)[None, :] * np.ones((nx, 1), np.float32)
    for scr, xo, yo in zip(screens, xoffs, yoffs):
        N = scr.shape[0]
        xr = (x - nx / 2.0) + nx / 2.0 + np.float32(xo)
        yr = (y - ny / 2.0) + ny / 2.0 + np.float32(yo)
        ir, jr = xr.astype(np.int64), yr.astype(np.int64)
        xs, ys = xr - ir, yr - jr
        ok = (ir + 1 < N) & (jr + 1 < N)
        irc, jrc = np.where(ok, ir, 0), np.where(ok, jr, 0)
        s = scr.astype(np.float64)
        v = ((1 - xs) * (1 - ys) * s[irc, jrc] + xs * (1 - ys) * s[irc + 1, jrc] + (1 - xs) * ys * s[irc, jrc + 1]
             + xs * ys * s[irc + 1, jrc + 1])
        out += np.where(ok, v, 0.0)
    return out


def dm_shape(dim, influ, i1, j1, com):
    shape = np.zeros((dim, dim))
    isz = influ.shape[0]
    for a in range(influ.shape[2]):
        x0, y0 = int(i1[a]), int(j1[a])
        xs = slice(max(x0, 0), min(x0 + isz, dim))
        ys = slice(max(y0, 0), min(y0 + isz, dim))
        shape[xs, ys] += com[a] * influ[xs.start - x0:xs.stop - x0, ys.start - y0:ys.stop - y0, a]
    return shape


def psf(phase, pupil, lam_um, nfft):
    npup = phase.shape[0]
    amp = np.zeros((nfft, nfft), dtype=np.complex128)
    m = pupil > 0
    amp[:npup, :npup][m] = np.exp(1j * 2 * np.pi / lam_um * phase[m])
    img = np.abs(np.fft.fft2(amp)) ** 2
    return img / float(m.sum()) ** 2


def strehl_sinc_fit(img, half=3):
    """Peak of a well-sampled PSF by sinc interpolation at its sub-pixel maximum
    (SutraSource::fitmax2x1dSinc, libsutra/src.cpp/sutra_source.cpp:451-488):
    parabolas through the 3-pixel cross around the brightest pixel (first one on
    ties) give the offset (x0, y0); the (2 half + 1)^2 window, read
    periodically (extract_krnl with roll, libcarma/src.cu/carma_obj.cu:454-488),
    is summed with weights sinc(x0 - i) sinc(y0 - j).  ``img`` is [x, y]."""
    n = img.shape[0]
    flat = np.asarray(img, np.float64).ravel(order="F")
    c = int(np.argmax(flat))
    cx, cy = c % n, c // n
    w = 2 * half + 1
    win = np.empty(w * w)
    for t in range(w * w):
        y = (cy + t // w - half) % n
        x = (cx + t % w - half) % n
        win[t] = flat[x + y * n]
    ctr = (w * w - 1) // 2
    A = 0.5 * (win[ctr - w] + win[ctr + w]) - win[ctr]
    B = 0.5 * (win[ctr - 1] + win[ctr + 1]) - win[ctr]
    if A * B == 0:
        return 0.0
    x0 = -0.5 * (win[ctr + w] - win[ctr - w]) / 2.0 / A
    y0 = -0.5 * (win[ctr + 1] - win[ctr - 1]) / 2.0 / B
    val, ind = 0.0, 0
    for i in range(-half, half + 1):
        for j in range(-half, half + 1):
            val += np.sinc(x0 - i) * np.sinc(y0 - j) * win[ind]
            ind += 1
    return float(val)

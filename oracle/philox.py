"""Philox4x32-10 counter-based generator and the noise samplers built on it.

Philox is the published generator of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of a
multiply-xor bijection over a 128-bit counter, keyed by a 64-bit key bumped
by the golden-ratio Weyl constants each round.  The GPU kernels use the same
stream, so the raw 32-bit words are bit-identical between this module and the
device.  This replaces the reference's cuRAND XORWOW states
(libcarma/src.cu/carma_rng.cu:35-141), whose streams cannot be reproduced.

Counter layout used by the sensors (one 128-bit block per pixel and draw):
  c0 = pixel index, c1 = frame number, c2 = stream tag, c3 = draw number
  key = (seed & 0xffffffff, seed >> 32)
Stream tags: 0 = photon (Poisson) noise, 1 = readout (Gaussian) noise.

Poisson sampling (replaces curand_poisson, carma_rng.cu:135-141):
  lambda < 10: sequential-search inversion (Devroye 1986, ch. X.3) on one
               uniform, in float64 with no fused multiply-add (1/k from a table);
  lambda >= 10: PTRS transformed rejection (Hoermann 1993, "The transformed
               rejection method for generating Poisson random variables") with
               its acceptance test in product form and log(k!) from a table of
               cumulative log sums (two-term Stirling series beyond 4095).
Gaussian: Box-Muller in float32 on one block (u1 from word 0, u2 from word 2).
"""

import math

import numpy as np

M0 = 0xD2511F53
M1 = 0xCD9E8D57
W0 = 0x9E3779B9
W1 = 0xBB67AE85
MASK = 0xFFFFFFFF

TAG_POISSON = 0
TAG_GAUSS = 1
POISSON_SMALL = 10.0
POISSON_MAX_DRAWS = 64


def philox4x32(c0, c1, c2, c3, k0, k1):
    """Ten Philox rounds on uint32 numpy arrays (broadcasting); returns 4 uint32 arrays."""
    c0 = np.asarray(c0, dtype=np.uint64) & MASK
    c1 = np.asarray(c1, dtype=np.uint64) & MASK
    c2 = np.asarray(c2, dtype=np.uint64) & MASK
    c3 = np.asarray(c3, dtype=np.uint64) & MASK
    k0 = np.asarray(k0, dtype=np.uint64) & MASK
    k1 = np.asarray(k1, dtype=np.uint64) & MASK
    for r in range(10):
        p0 = c0 * np.uint64(M0)
        p1 = c2 * np.uint64(M1)
        hi0, lo0 = p0 >> np.uint64(32), p0 & np.uint64(MASK)
        hi1, lo1 = p1 >> np.uint64(32), p1 & np.uint64(MASK)
        c0, c1, c2, c3 = (hi1 ^ c1 ^ k0) & np.uint64(MASK), lo1, (hi0 ^ c3 ^ k1) & np.uint64(MASK), lo0
        if r < 9:
            k0 = (k0 + np.uint64(W0)) & np.uint64(MASK)
            k1 = (k1 + np.uint64(W1)) & np.uint64(MASK)
    return (c0.astype(np.uint32), c1.astype(np.uint32), c2.astype(np.uint32), c3.astype(np.uint32))


def key_of(seed):
    seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    return seed & MASK, seed >> 32


def u01(x):
    """Open-interval uniform from one 32-bit word, exact in float64."""
    return (np.asarray(x, dtype=np.float64) + 0.5) * (1.0 / 4294967296.0)


LOGFACT_N = 4096
RK_N = 1024


def _tables():
    """log(k!) by cumulative sums of log(i) and 1/k -- the same tables the device uses."""
    lf = [0.0] * LOGFACT_N
    for k in range(1, LOGFACT_N):
        lf[k] = lf[k - 1] + math.log(k)
    rk = [0.0] + [1.0 / k for k in range(1, RK_N)]
    return lf, rk


LOGFACT, RK = _tables()


def log_factorial(k):
    if k < LOGFACT_N:
        return LOGFACT[int(k)]
    x = k + 1.0
    ix = 1.0 / x
    r = (x + -0.5) * math.log(x)
    r = (r + -x) + 0.91893853320467274178
    c = 0.08333333333333333 * ix + -((0.002777777777777778 * ix) * (ix * ix))
    return r + c


def _ptrs(lam, words_of_draw):
    """PTRS transformed rejection with the acceptance test in product form."""
    slam = math.sqrt(lam)
    loglam = math.log(lam)
    b = 0.931 + 2.53 * slam
    a = -0.059 + 0.02483 * b
    invalpha = 1.1239 + 1.1328 / (b + -3.4)
    vr = 0.9277 + -(3.6224 / (b + -2.0))
    a2 = 2.0 * a
    for d in range(POISSON_MAX_DRAWS):
        w = words_of_draw(d)
        u = float(u01(w[0])) + -0.5
        v = float(u01(w[1]))
        us = 0.5 + -abs(u)
        k = math.floor((((a2 / us) + b) * u + lam) + 0.43)
        if us >= 0.07 and v <= vr:
            return k
        if k < 0 or (us < 0.013 and v > us):
            continue
        lhs = (v * invalpha) / ((a / (us * us)) + b)
        rhs = math.exp(((k * loglam) + -lam) + -log_factorial(k))
        if lhs <= rhs:
            return k
    return math.floor(lam + 0.5)


def _inversion(lam, u):
    p = math.exp(-lam)
    f = p
    k = 0
    while u > f and k < RK_N - 1:
        k += 1
        p = p * (lam * RK[k])
        f = f + p
    return k


def poisson(lam, index, frame, seed):
    """Poisson deviates for an array of means ``lam`` at pixel ``index``; float64 out."""
    lam = np.asarray(lam, dtype=np.float64)
    index = np.asarray(index, dtype=np.uint64)
    k0, k1 = key_of(seed)
    out = np.zeros(lam.shape, dtype=np.float64)
    flat_l = lam.ravel()
    flat_i = np.broadcast_to(index, lam.shape).ravel()
    w0 = philox4x32(flat_i, frame, TAG_POISSON, 0, k0, k1)
    res = out.ravel()
    for j in range(flat_l.size):
        m = float(flat_l[j])
        if not (m > 0.0):
            res[j] = 0.0
        elif m < POISSON_SMALL:
            res[j] = _inversion(m, float(u01(w0[0][j])))
        else:
            ij = int(flat_i[j])

            def words(d, ij=ij, j=j):
                if d == 0:
                    return (w0[0][j], w0[1][j])
                w = philox4x32(ij, frame, TAG_POISSON, d, k0, k1)
                return (w[0], w[1])

            res[j] = _ptrs(m, words)
    return res.reshape(lam.shape)


def gaussian(index, frame, seed):
    """Standard normal deviates (float32 Box-Muller, 24-bit uniforms) for pixel indices."""
    index = np.asarray(index, dtype=np.uint64)
    k0, k1 = key_of(seed)
    w = philox4x32(index, frame, TAG_GAUSS, 0, k0, k1)
    u1 = ((w[0] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    u2 = ((w[2] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    return np.sqrt(np.float32(-2.0) * np.log(u1)) * np.cos(np.float32(2.0 * np.pi) * u2.astype(np.float64)).astype(np.float32)


def normal_f32(c0, c1, c2, c3, seed):
    """float32 Box-Muller deviate from the Philox block (c0, c1, c2, c3) (words 0 and 2)."""
    k0, k1 = key_of(seed)
    w = philox4x32(c0, c1, c2, c3, k0, k1)
    u1 = ((w[0] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    u2 = ((w[2] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    return np.sqrt(np.float32(-2.0) * np.log(u1)) * np.cos(np.float32(2.0 * np.pi) * u2.astype(np.float64)).astype(np.float32)

"""Philox4x32-10 counter-based generator and the noise samplers built on it.

Philox is the published generator of Salmon, Moraes, Dror and Shaw,
"Parallel random numbers: as easy as 1, 2, 3" (SC'11): ten rounds of a
multiply-xor bijection over a 128-bit counter, keyed by a 64-bit key bumped
by the golden-ratio Weyl constants each round.  The GPU kernels use the same
stream, so the raw 32-bit words are bit-identical between this module and the
device.  This replaces the reference's cuRAND XORWOW states
(libcarma/src.cu/carma_rng.cu:35-141), whose streams cannot be reproduced.

Counter layout used by the sensors (one 128-bit block per pixel and draw):
  c0 = pixel index, c1 = frame number, c2 = stream tag (0 = sensor noise),
  c3 = block number; key = (seed & 0xffffffff, seed >> 32).
Block 0 of a pixel gives the first Poisson draw (words 0, 1) and the readout
noise (words 2, 3); rejected Poisson draws continue with block 1 (words 0, 1,
then 2, 3), block 2, ...
(The turbulence extrusion uses tag 2, c3 = layer.)

Poisson sampling (replaces curand_poisson, carma_rng.cu:135-141), restating
the device sampler operation for operation, all in float32 on 24-bit uniforms:
  lambda < 40: sequential-search inversion (Devroye 1986, ch. X.3, at most
               160 steps) with
               p0 = exp(-lambda) from the project's own exp (Cody-Waite
               reduction, degree-7 Taylor polynomial);
  lambda >= 40: PTRS transformed rejection (Hoermann 1993, "The transformed
               rejection method for generating Poisson random variables"):
               the published fast acceptance test, and the exact test in the
               log domain with log(k!) in Stirling form arranged so that no
               large terms cancel (own log / log1p by the atanh series).
Gaussian: Box-Muller in float32 on words 2 (u1) and 3 (u2) of draw 0.
"""

import math

import numpy as np

M0 = 0xD2511F53
M1 = 0xCD9E8D57
W0 = 0x9E3779B9
W1 = 0xBB67AE85
MASK = 0xFFFFFFFF

TAG_POISSON = 0
POISSON_SMALL = 40.0
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


F32 = np.float32
INV_KMAX = 160


def _u01f(x):
    """24-bit uniform ((x >> 8) + 0.5) / 2^24, exact in float32."""
    return (F32(int(x) >> 8) + F32(0.5)) * F32(5.9604644775390625e-08)


# Every helper below uses single correctly rounded NumPy float32 scalar operations
# in the device's order, so results equal the GPU's bit for bit.
def _expf_neg(x):
    """exp(x), x in [-88, 0]: Cody-Waite reduction by ln2, degree-7 Taylor polynomial."""
    n = np.rint(x * F32(1.44269502))
    r = (x + -(n * F32(0.693145752))) + -(n * F32(1.42860677e-06))
    p = F32(1.98412701e-04)
    for c in (1.38888892e-03, 8.33333377e-03, 4.16666679e-02, 1.66666672e-01, 0.5, 1.0, 1.0):
        p = p * r + F32(c)
    return p * np.ldexp(F32(1.0), int(n))


def _log_series(s):
    """log((1+s)/(1-s)) = 2 s + 2 s^3/3 + ... + 2 s^11/11."""
    s2 = s * s
    t = F32(0.181818187)
    for c in (0.222222224, 0.285714298, 0.400000006, 0.666666687):
        t = t * s2 + F32(c)
    return s * F32(2.0) + (s * s2) * t


def _logf(x):
    """log(x), normal x > 0, from x = m 2^e with m in [sqrt(1/2), sqrt(2)]."""
    bits = int(np.asarray(F32(x)).view(np.int32))
    e = ((bits >> 23) & 0xFF) - 127
    m = np.asarray(np.int32((bits & 0x007FFFFF) | 0x3F800000)).view(np.float32)[()]
    if m > F32(1.41421354):
        m = m * F32(0.5)
        e += 1
    s = (m + F32(-1.0)) / (m + F32(1.0))
    fe = F32(e)
    return fe * F32(0.693145752) + (fe * F32(1.42860677e-06) + _log_series(s))


def _log1pf(d):
    return _log_series(d / (F32(2.0) + d))


_LOGFACT_SMALL = [F32(math.lgamma(k + 1)) for k in range(10)]


def _ptrs(lamf, words_of_draw):
    """PTRS transformed rejection in float32; exact test in the log domain (Stirling form)."""
    slam = np.sqrt(lamf)
    b = F32(0.931) + F32(2.53) * slam
    a = F32(-0.059) + F32(0.02483) * b
    vr = F32(0.9277) + -(F32(3.6224) / (b + F32(-2.0)))
    a2 = F32(2.0) * a
    invalpha = F32(1.1239) + F32(1.1328) / (b + F32(-3.4))
    for d in range(POISSON_MAX_DRAWS):
        w = words_of_draw(d)
        u = _u01f(w[0]) + F32(-0.5)
        v = _u01f(w[1])
        us = F32(0.5) + -abs(u)
        k = np.floor((((a2 / us) + b) * u + lamf) + F32(0.43))
        if us >= F32(0.07) and v <= vr:
            return float(k)
        if k < 0 or (us < F32(0.013) and v > us):
            continue
        lhs = _logf((v * invalpha) / ((a / (us * us)) + b))
        if k < F32(10.0):
            rhs = (k * _logf(lamf) + -lamf) + -_LOGFACT_SMALL[int(k)]
        else:
            x = k + F32(1.0)
            dd = (lamf + -x) / x
            lr = _log1pf(dd) if (F32(-0.25) <= dd <= F32(0.5)) else _logf(lamf / x)
            ix = F32(1.0) / x
            corr = F32(0.0833333358) * ix + -((F32(0.00277777785) * ix) * (ix * ix))
            rhs = k * lr + -(F32(0.5) * _logf(x))
            rhs = rhs + (x + -lamf)
            rhs = (rhs + F32(-0.918938518)) + -corr
        if lhs <= rhs:
            return float(k)
    return float(np.floor(lamf + F32(0.5)))


def _inversion(lamf, u):
    p = _expf_neg(-lamf)
    f = p
    k = 0
    while u > f and k < INV_KMAX:
        k += 1
        p = p * (lamf * (F32(1.0) / F32(k)))
        f = f + p
    return float(k)


def poisson(lam, index, frame, seed):
    """Poisson deviates for an array of float32 means ``lam`` at pixel ``index``; float64 out."""
    lam = np.asarray(lam, dtype=np.float32)
    index = np.asarray(index, dtype=np.uint64)
    k0, k1 = key_of(seed)
    out = np.zeros(lam.shape, dtype=np.float64)
    flat_l = lam.ravel()
    flat_i = np.broadcast_to(index, lam.shape).ravel()
    w0 = philox4x32(flat_i, frame, TAG_POISSON, 0, k0, k1)
    res = out.ravel()
    for j in range(flat_l.size):
        m = flat_l[j]
        if not (m > 0):
            res[j] = 0.0
        elif m < POISSON_SMALL:
            res[j] = _inversion(m, _u01f(w0[0][j]))
        else:
            ij = int(flat_i[j])

            def words(d, ij=ij, j=j):
                if d == 0:
                    return (w0[0][j], w0[1][j])
                w = philox4x32(ij, frame, TAG_POISSON, (d + 1) // 2, k0, k1)
                return (w[0], w[1]) if d % 2 == 1 else (w[2], w[3])

            res[j] = _ptrs(m, words)
    return res.reshape(lam.shape)


def gaussian(index, frame, seed):
    """Readout-noise deviates: float32 Box-Muller on words 2 (u1) and 3 (u2) of each
    pixel's draw-0 Poisson block (24-bit uniforms)."""
    index = np.asarray(index, dtype=np.uint64)
    k0, k1 = key_of(seed)
    w = philox4x32(index, frame, TAG_POISSON, 0, k0, k1)
    u1 = ((w[2] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    u2 = ((w[3] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    return np.sqrt(np.float32(-2.0) * np.log(u1)) * np.cos(np.float32(2.0 * np.pi) * u2.astype(np.float64)).astype(np.float32)


def normal_f32(c0, c1, c2, c3, seed):
    """float32 Box-Muller deviate from the Philox block (c0, c1, c2, c3) (words 0 and 2)."""
    k0, k1 = key_of(seed)
    w = philox4x32(c0, c1, c2, c3, k0, k1)
    u1 = ((w[0] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    u2 = ((w[2] >> np.uint32(8)).astype(np.float32) + np.float32(0.5)) * np.float32(5.9604644775390625e-08)
    return np.sqrt(np.float32(-2.0) * np.log(u1)) * np.cos(np.float32(2.0 * np.pi) * u2.astype(np.float64)).astype(np.float32)

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
  c3 = draw number; key = (seed & 0xffffffff, seed >> 32).
Draw 0 of a pixel gives the first Poisson draw (words 0, 1) and the readout
noise (words 2, 3); rejected Poisson draws continue with draws 1, 2, ...
(The turbulence extrusion uses tag 2, c3 = layer.)

Poisson sampling (replaces curand_poisson, carma_rng.cu:135-141), restating
the device sampler operation for operation:
  lambda < 10: sequential-search inversion (Devroye 1986, ch. X.3) on one
               32-bit uniform, in float64 with no fused multiply-add (1/k as
               the IEEE quotient);
  lambda >= 10: PTRS transformed rejection (Hoermann 1993, "The transformed
               rejection method for generating Poisson random variables"):
               the fast acceptance path in float32 on 24-bit uniforms, the
               exact acceptance test in float64 in product form with log(k!)
               from a table of cumulative log sums (two-term Stirling series
               beyond 4095).
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
    """log(k!) by cumulative sums of log(i) (the device table) and 1/k (the device computes the
    same correctly rounded value with __drcp_rn)."""
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


F32 = np.float32


def _u01f(x):
    """24-bit uniform ((x >> 8) + 0.5) / 2^24, exact in float32."""
    return (F32(int(x) >> 8) + F32(0.5)) * F32(5.9604644775390625e-08)


def _ptrs(lamf, words_of_draw):
    """PTRS transformed rejection: float32 fast path, float64 exact test in product form.

    Every float32 operation is a single correctly rounded NumPy float32 scalar
    operation, in the device's order.
    """
    slam = np.sqrt(lamf)
    b = F32(0.931) + F32(2.53) * slam
    a = F32(-0.059) + F32(0.02483) * b
    vr = F32(0.9277) + -(F32(3.6224) / (b + F32(-2.0)))
    a2 = F32(2.0) * a
    loglam = math.log(float(lamf))
    invalpha = 1.1239 + 1.1328 / (float(b) + -3.4)
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
        usd = float(us)
        lhs = (float(v) * invalpha) / ((float(a) / (usd * usd)) + float(b))
        rhs = math.exp(((float(k) * loglam) + -float(lamf)) + -log_factorial(float(k)))
        if lhs <= rhs:
            return float(k)
    return float(np.floor(lamf + F32(0.5)))


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
            res[j] = _inversion(float(m), float(u01(w0[0][j])))
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

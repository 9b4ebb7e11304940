"""GPU parity of the closed-loop support: FFT, extrusion, raytrace, DM shape, PSF.

Tolerances: float32 kernels against float64 NumPy -- relative rms <= 1e-5
unless stated; the FP64 A/B factorisation against NumPy's SVD form <= 1e-9.
"""

import numpy as np
import pytest

from helpers import rel_rms
from oracle import philox
from oracle import turbulence as OT

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    from aob200 import _lib

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return _lib


@pytest.mark.parametrize("n,batch", [(16, 3), (64, 2), (256, 1), (512, 2)])
@pytest.mark.parametrize("inverse", [False, True])
def test_fft2d_matches_numpy(lib, n, batch, inverse):
    import torch

    from aob200 import optics

    rng = np.random.default_rng(n + batch)
    x = (rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))).astype(np.complex64)
    d = torch.from_numpy(x).cuda()
    optics.fft2d(d.data_ptr(), n, batch, inverse)
    torch.cuda.synchronize()
    got = d.cpu().numpy()
    ref = np.fft.ifft2(x.astype(np.complex128)) * n * n if inverse else np.fft.fft2(x.astype(np.complex128))
    assert rel_rms(got.view(np.float32), ref.astype(np.complex64).view(np.float32)) < 2e-6


def test_kolmo_factorisation_fp64(lib):
    from aob200 import turbulence as T

    n = 48
    A, B, istx, isty = T.extrusion_operators(n, 300.0, 1.0, 1.0)
    zz, xz, xx, ist = T.covariances(n, 300.0)
    Ao, Bo = OT.factor_AB(zz, xz, xx)
    assert rel_rms(A, Ao) < 1e-6
    assert rel_rms(B.astype(np.float64) @ B.T.astype(np.float64), Bo @ Bo.T) < 1e-6


@pytest.mark.parametrize("dx,dy", [(0.7, 0.4), (-1.3, -0.6)])
def test_atmosphere_extrusion_matches_oracle(lib, dx, dy):
    from aob200 import turbulence as T

    n = 40
    lp = T.LayerParams(r0_pix=3.0, alt=0.0, deltax=dx, deltay=dy, dim=n, L0_pix=200.0, seed=77)
    A, B, istx, isty = T.extrusion_operators(n, lp.L0_pix, dx, dy)
    atm = T.Atmosphere([], device=0)
    atm.add_screen(lp, A, B, istx, isty)
    amp = np.float32(lp.r0_pix) ** np.float32(-5.0 / 6.0) * np.float32(0.5) / np.float32(2 * np.pi)
    scr = np.zeros((n, n))
    counter = 0
    # refresh: zero then 2n extrusions in x
    atm.refresh(0)
    d = 1 if dx > 0 else -1
    for _ in range(2 * n):
        xi = philox.normal_f32(np.arange(n, dtype=np.uint64), counter, 2, 0, lp.seed).astype(np.float64)
        scr = OT.extrude(scr, A, B, istx, isty, float(amp), xi, d)
        counter += 1
    assert rel_rms(atm.screen_host(0), scr) < 1e-4
    # a few moves: accumulate shifts in float32 like the reference's float accumx/accumy
    # (sutra_atmos.cpp:100-119), extrude along x then y
    ax = ay = np.float32(0.0)
    for _ in range(5):
        atm.move()
        ax = np.float32(ax + np.float32(dx))
        ay = np.float32(ay + np.float32(dy))
        for axis, acc in ((1, ax), (2, ay)):
            k = int(acc)
            c = 1 if k > 0 else -1
            for _ in range(c * k):
                xi = philox.normal_f32(np.arange(n, dtype=np.uint64), counter, 2, 0, lp.seed).astype(np.float64)
                scr = OT.extrude(scr, A, B, istx, isty, float(amp), xi, axis * c)
                counter += 1
            if axis == 1:
                ax = np.float32(ax - np.float32(k))
            else:
                ay = np.float32(ay - np.float32(k))
    assert rel_rms(atm.screen_host(0), scr) < 1e-4
    _, _, gax, gay = atm.screen(0)
    assert gax == ax and gay == ay


def test_raytrace_and_dm_shape_match_oracle(lib, golden):
    import torch

    from aob200 import optics

    dm = golden("dm17")
    rng = np.random.default_rng(2)
    d = optics.Dm(int(dm["dim"]), dm["influ"], dm["i1"], dm["j1"])
    com = rng.standard_normal(int(dm["ntotact"])).astype(np.float32)
    d.set_com(com)
    d.comp_shape()
    shape = np.array(d.d_shape)
    oshape = OT.dm_shape(int(dm["dim"]), dm["influ"].astype(np.float64), dm["i1"], dm["j1"], com.astype(np.float64))
    assert rel_rms(shape, oshape) < 1e-6
    # raytrace: two random layers plus the DM shape into a 132 x 132 pupil grid
    n = int(dm["n_mpupil"])
    l1 = rng.standard_normal((140, 140)).astype(np.float32)
    l2 = rng.standard_normal((150, 150)).astype(np.float32)
    t1, t2 = torch.from_numpy(np.asfortranarray(l1).ravel(order="F")).cuda(), torch.from_numpy(
        np.asfortranarray(l2).ravel(order="F")).cuda()
    out = torch.zeros(n * n, device="cuda")
    xoff_dm = (int(dm["dim"]) - n) / 2.0
    srcs = [(t1.data_ptr(), 140, 4.0 + 0.37, 4.0 + 0.81), (t2.data_ptr(), 150, 9.0 + 0.5, 9.0),
            (d.d_shape.ptr, int(dm["dim"]), xoff_dm, xoff_dm)]
    optics.raytrace(out.data_ptr(), n, n, srcs)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(n, n, order="F")
    ref = OT.raytrace(n, n, [l1, l2, shape], [4.37, 9.5, xoff_dm], [4.81, 9.0, xoff_dm])
    assert rel_rms(got, ref) < 1e-6


def test_target_psf_and_strehl(lib):
    from aob200 import geometry as G
    from aob200 import optics

    tel = G.telescope_geometry(120, 8.0, 0.14)
    pup = tel.spupil
    t = optics.Target(pup, 1.65, 256)
    rng = np.random.default_rng(5)
    ph = (0.05 * rng.standard_normal(pup.shape)).astype(np.float32)
    t.d_phase.set(ph)
    t.comp_image()
    se, le = t.strehl()
    ref = OT.psf(ph.astype(np.float64), pup, 1.65, 256)
    assert rel_rms(np.array(t.d_image_se), ref) < 1e-5
    assert abs(se - ref.max()) < 1e-5
    # flat wavefront: Strehl 1
    t.d_phase.set(np.zeros_like(ph))
    t.reset_le()
    t.comp_image()
    se, le = t.strehl()
    assert abs(se - 1.0) < 1e-5 and abs(le - 1.0) < 1e-5
    sf, lf = t.strehl(fit=True)
    assert abs(sf - 1.0) < 1e-4 and abs(lf - 1.0) < 1e-4


def test_target_strehl_sinc_fit_matches_oracle(lib):
    """comp_strehl(do_fit): the sinc fit of a tilted (off-pixel) PSF peak, short and
    long exposure, against the oracle's restatement."""
    from aob200 import geometry as G
    from aob200 import optics

    tel = G.telescope_geometry(120, 8.0, 0.14)
    pup = tel.spupil
    t = optics.Target(pup, 1.65, 256)
    rng = np.random.default_rng(6)
    x = np.arange(pup.shape[0])
    imgs = []
    for k in range(3):
        tilt = 1.65 * (0.37 + 0.1 * k) / pup.shape[0] * 2.13  # a fraction of a pixel in the focal plane
        ph = (tilt * x[:, None] + 0.03 * rng.standard_normal(pup.shape)).astype(np.float32)
        t.d_phase.set(ph)
        t.comp_image()
        imgs.append(np.array(t.d_image_se).astype(np.float64))
    sf, lf = t.strehl(fit=True)
    ref_se = OT.strehl_sinc_fit(imgs[-1])
    ref_le = OT.strehl_sinc_fit(sum(imgs)) / len(imgs)
    assert abs(sf - ref_se) < 1e-5 * max(ref_se, 1e-3) + 1e-6
    assert abs(lf - ref_le) < 1e-4 * ref_le
    se, le = t.strehl()
    assert sf >= se - 1e-6  # the fitted peak is at least the brightest pixel

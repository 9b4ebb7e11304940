"""The learned reconstructor on the GPU: its BF16 tensor-core GEMMs and
gradients against the float64 oracle, training, batch-1 inference, and the
closed loop against the least-squares reconstructor it falls back to.

Tolerances: forward outputs relative rms <= 5e-3 and gradients <= 3e-2
against the oracle (BF16 storage of activations and gradients on both sides,
float32 against float64 accumulation); batch-1 inference equals the batched
forward within 3e-3.
"""

import numpy as np
import pytest

from helpers import rel_rms
from oracle import mlp as omlp

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def M():
    import torch

    from aob200 import _lib, mlp

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    return mlp, torch


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


@pytest.mark.parametrize("gemm", [0, 1])
@pytest.mark.parametrize("dims,batch", [((40, 32, 24, 20), 16), ((2496, 1024, 1024, 1377), 64), ((131, 70, 45, 33), 37),
                                        ((200, 256, 136, 72), 300)])
def test_forward_and_gradients_match_oracle(M, dims, batch, gemm):
    """Both GEMM kernels (0: mma.sync, 1: tcgen05 with TMA tensor loads and a
    TMEM accumulator) against the oracle, every operand layout and epilogue."""
    mlp, torch = M
    nin, nh1, nh2, nout = dims
    net = mlp.MlpReconstructor(nin, nout, nh1, nh2, seed=3)
    net.set_gemm(gemm)
    rng = np.random.default_rng(4)
    params = [(w, rng.standard_normal(w.shape[0]).astype(np.float32) * 0.1) for w, _ in net.get_params()[:3]]
    params.append((rng.standard_normal((nout, nin)).astype(np.float32) * 0.05, None))  # skip path
    net.set_params(params)
    net.set_scales(0.5, 2.0)
    x = rng.standard_normal((batch, nin)).astype(np.float32)
    t = rng.standard_normal((batch, nout)).astype(np.float32)
    dx, dt = _dev(torch, x), _dev(torch, t)
    dy = torch.zeros((batch, nout), device="cuda")
    loss = torch.zeros(1, device="cuda")
    net.forward(dx.data_ptr(), batch, dy.data_ptr())
    net.backward(dt.data_ptr(), batch, loss.data_ptr())
    torch.cuda.synchronize()
    y_ref, _ = omlp.forward(params, x, 0.5)
    assert rel_rms(dy.cpu().numpy(), 2.0 * y_ref) < 5e-3
    loss_ref, g = omlp.backward(params, x, t, 0.5, 2.0)
    assert abs(float(loss.item()) / loss_ref - 1) < 5e-3
    pin, ph1, ph2, pout = net.padded_dims()
    shapes = {"dW1": (ph1, pin), "dW2": (ph2, ph1), "dW3": (pout, ph2), "dWs": (pout, pin)}
    real = {"dW1": (nh1, nin), "dW2": (nh2, nh1), "dW3": (nout, nh2), "dWs": (nout, nin), "db1": nh1, "db2": nh2,
            "db3": nout}
    from aob200 import _lib

    for name, ref in g.items():
        ptr, n = net.buffer(name)
        got = _lib.d2h(ptr, n, np.float32)
        if name.startswith("dW"):
            got = got.reshape(shapes[name])[: real[name][0], : real[name][1]]
        else:
            got = got[: real[name]]
        assert rel_rms(got, ref) < 3e-2, name
    assert net.gemm_status() == 0


def test_infer_equals_batched_forward(M):
    mlp, torch = M
    net = mlp.MlpReconstructor(2496, 1377, seed=5)
    net.set_scales(3.0, 0.5)
    rng = np.random.default_rng(6)
    x = rng.standard_normal((8, 2496)).astype(np.float32)
    dx = _dev(torch, x)
    dyb = torch.zeros((8, 1377), device="cuda")
    net.forward(dx.data_ptr(), 8, dyb.data_ptr())
    y1 = torch.zeros(1377, device="cuda")
    for i in range(8):
        net.infer(dx[i].data_ptr(), y1.data_ptr())
        torch.cuda.synchronize()
        # the GEMV and the tensor-core GEMM sum in different orders, so a hidden
        # activation occasionally rounds to the neighbouring bfloat16
        assert rel_rms(y1.cpu().numpy(), dyb[i].cpu().numpy()) < 3e-3


@pytest.mark.parametrize("gemm", [0, 1])
def test_training_learns_a_linear_reconstructor(M, gemm):
    """On a noiseless linear map slopes -> commands the loss falls by 20x
    (bfloat16 storage sets the floor), with either GEMM kernel."""
    mlp, torch = M
    rng = np.random.default_rng(7)
    nin, nout, n = 200, 60, 16384
    R = rng.standard_normal((nout, nin)).astype(np.float32) / np.sqrt(nin)
    X = rng.standard_normal((n, nin)).astype(np.float32)
    T = X @ R.T
    net = mlp.MlpReconstructor(nin, nout, 256, 256, seed=8)
    net.set_gemm(gemm)
    hist = net.fit(_dev(torch, X), _dev(torch, T), epochs=40, batch=512, lr=2e-3, lr_decay=0.93)
    assert hist[-1] < hist[0] / 20, hist


def test_learned_reconstructor_closes_the_loop(M):
    """plain16.  The network starts as the LS reconstructor (skip path = cmat)
    and is trained on pseudo-open-loop pairs (the atmosphere alone at several
    turbulence strengths, its slopes, the DM-projected phase as the target).
    Gain: on held-out pairs it predicts the DM-projected phase with a smaller
    error than LS.  In closed loop its long-exposure Strehl stays within 10 % of
    the LS loop's; with a zero threshold every step falls back to LS and the
    result is the LS loop's exactly."""
    mlp, torch = M
    from aob200 import system

    def fresh():
        s = system.ShAoSystem(system.plain16())
        s.calibrate()
        s.close(graph=False, mode=1)
        return s

    s = fresh()
    P, mask = mlp.dm_projector(s)
    X, T = mlp.collect_open_loop(s, 12000, P, mask)
    n = 10000
    net = mlp.MlpReconstructor(X.shape[1], T.shape[1], 256, 256, seed=9)
    net.init_from_ls(s.cmat, 1.0 / float(X.std()), float(T.std()))
    net.fit(_dev(torch, X[:n]), _dev(torch, T[:n]), epochs=12, batch=256, lr=3e-4, lr_decay=0.85,
            scales_from_data=False)
    dx = _dev(torch, X[n:])
    dy = torch.zeros((X.shape[0] - n, T.shape[1]), device="cuda")
    net.forward(dx.data_ptr(), X.shape[0] - n, dy.data_ptr())
    torch.cuda.synchronize()
    err_mlp = rel_rms(dy.cpu().numpy(), T[n:])
    err_ls = rel_rms(X[n:] @ s.cmat.T, T[n:])
    assert err_mlp < err_ls, (err_mlp, err_ls)

    def run(sysm, **kw):
        for _ in range(20):
            sysm.next(compute_psf=False, **kw)
        sysm.target.reset_le()
        for _ in range(150):
            sysm.next(**kw)
        return sysm.strehl()[1]

    le_ls = run(fresh())
    le_mlp = run(fresh(), mlp=net, threshold=np.inf)
    assert le_mlp > 0.9 * le_ls, (le_mlp, le_ls, err_mlp, err_ls)
    net.fallbacks(reset=True)
    le_fb = run(fresh(), mlp=net, threshold=0.0)
    assert net.fallbacks() == 170
    assert abs(le_fb - le_ls) < 1e-6 * max(le_ls, 1e-6)


@pytest.mark.parametrize("prec", ["f32", "bf16", "fp8"])
@pytest.mark.parametrize("dims", [(2496, 1024, 1024, 1377), (131, 70, 45, 33)])
def test_fused_control_step_equals_multi_kernel_path(M, prec, dims):
    """The single-launch control step (all layers, the threshold test, the LS
    fallback) gives the same commands, errors and fallback count as the
    GEMV-per-layer path, bit for bit: network path (threshold inf) and LS
    fallback (threshold 0), over several steps of the integrator."""
    mlp, torch = M
    from aob200 import core

    nin, nh1, nh2, nout = dims
    rng = np.random.default_rng(11)
    cm = (rng.standard_normal((nout, nin)) / np.sqrt(nin)).astype(np.float32)

    w3 = (rng.standard_normal((nout, nh2)) * 0.05).astype(np.float32)

    def make(mode):
        net = mlp.MlpReconstructor(nin, nout, nh1, nh2, seed=4)
        net.init_from_ls(cm, 2.0, 0.5)
        P = net.get_params()
        P[2] = (w3, P[2][1] + 0.01)  # a non-zero last layer: the hidden path counts too
        net.set_params(P)
        net.set_mode(mode)
        ls = core.LsController(nin, nout)
        ls.set_precision(prec)
        ls.set_cmat(cm)
        ls.set_gain(0.4)
        return net, ls

    a_net, a_ls = make(0)
    b_net, b_ls = make(1)
    for it, thr in enumerate([np.inf, np.inf, 0.0, np.inf, 0.0]):
        s = rng.standard_normal(nin).astype(np.float32)
        a_ls.set_centroids(s)
        b_ls.set_centroids(s)
        a_net.comp_com(a_ls, thr)
        b_net.comp_com(b_ls, thr)
        for name in ("com", "err"):
            np.testing.assert_array_equal(np.array(a_ls.buffer(name)), np.array(b_ls.buffer(name)),
                                          err_msg=f"step {it}: {name}")
    assert a_net.fallbacks() == b_net.fallbacks() == 2
    assert a_ls.status() == 0

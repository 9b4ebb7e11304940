"""The learned reconstructor at its configured scale, against least squares.

The saxo40 system (40 x 40 SH, 1352 actuators) calibrated by its push-pull
interaction matrix; pairs of (noisy slopes, DM-projected residual phase) taken
from closed LS loops at five turbulence strengths (r0 0.08-0.20 m) and
guide-star magnitudes drawn in 6-10; the MLP 2496 -> 1024 -> 1024 -> 1352 (+ a
linear skip path initialised to the LS matrix) trained on them by the
project's GPU kernels; then both reconstructors drive the same closed loop
(held-out turbulence seeds, r0 0.14 m, magnitude 8) and their long-exposure
Strehl at 1.65 um (the reference's sinc fit) is compared.

The network's output scale is its loop gain.  Fitted in the mean-square sense
to noise-dominated closed-loop slopes, its response to a DM shape is below the
LS reconstructor's unit response (it shrinks), which in an integrator lowers
the loop gain.  The output is therefore scaled by f / g, g the measured
response to the slopes of known DM shapes and f chosen on a validation loop
with other seeds; the held-out loop is run once with the chosen f.
"""

from __future__ import annotations

import dataclasses
import time

import numpy as np

from . import mlp as M
from . import system as S

R0S = (0.08, 0.11, 0.14, 0.17, 0.20)
FACTORS = (1.0, 1.2, 1.35, 1.5, 1.75, 2.0)


def c4_experiment(pairs=200000, epochs=16, loop_iters=3000, settle=100, device=0):
    import torch

    t0 = time.perf_counter()
    base = S.saxo40()
    cal = S.ShAoSystem(base, device)
    cal.calibrate()
    cmat, imat = cal.cmat, cal.imat
    P, mask = M.dm_projector(cal)
    probe = M.dm_probe(cal)
    del cal
    systems = []
    for j, r0 in enumerate(R0S):
        sy = S.ShAoSystem(dataclasses.replace(base, r0=r0, seeds=(500 + 3 * j, 501 + 3 * j, 502 + 3 * j)), device)
        sy.imat = imat
        sy.ls.set_cmat(cmat)
        sy.close(graph=False)
        systems.append(sy)
    t_setup = time.perf_counter() - t0
    t0 = time.perf_counter()
    X, T = M.collect_closed_loop(systems, pairs, P, mask, seed=3)
    t_pairs = time.perf_counter() - t0
    del systems
    n = X.shape[0]
    ntr = int(0.95 * n)
    net = M.MlpReconstructor(X.shape[1], T.shape[1], 1024, 1024, device=device, seed=1)
    net.set_gemm(1)
    net.init_from_ls(cmat, 1.0 / float(X[:ntr].std()), float(T[:ntr].std()))
    t0 = time.perf_counter()
    hist = net.fit(X[:ntr], T[:ntr], epochs=epochs, batch=1024, lr=2e-4, lr_decay=0.85, scales_from_data=False)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    # held-out pairs: error of each reconstructor against the target
    Y = torch.zeros((n - ntr, T.shape[1]), device="cuda")
    net.forward(X[ntr:].data_ptr(), n - ntr, Y.data_ptr())
    torch.cuda.synchronize()
    Tv = T[ntr:].double()
    ct = torch.as_tensor(np.asarray(cmat, np.float32), device="cuda")
    err_mlp = float(torch.linalg.norm(Y.double() - Tv) / torch.linalg.norm(Tv))
    err_ls = float(torch.linalg.norm((X[ntr:] @ ct.T).double() - Tv) / torch.linalg.norm(Tv))
    del X, T, Y

    def closed(cfg, niter, mlp=None):
        sy = S.ShAoSystem(cfg, device)
        sy.ls.set_cmat(cmat)
        sy.close(graph=False)
        for _ in range(settle):
            sy.next(compute_psf=False, mlp=mlp, threshold=np.inf)
        sy.target.reset_le()
        res = []
        for _ in range(niter):
            sy.next(mlp=mlp, threshold=np.inf)
            res.append(sy.residual_rms())
        return dict(strehl_le=sy.target.strehl(fit=True)[1], residual_rms_um=float(np.mean(res)))

    gain = M.response_gain(net, probe)
    o0 = net.out_scale
    val_cfg = dataclasses.replace(base, seeds=(700, 701, 702))
    val = {}
    for f in FACTORS:
        net.set_scales(net.in_scale, o0 * f / gain)
        val[f] = closed(val_cfg, loop_iters // 2, net)["strehl_le"]
    f_best = max(val, key=val.get)
    net.set_scales(net.in_scale, o0)
    raw = closed(base, loop_iters, net)
    net.set_scales(net.in_scale, o0 * f_best / gain)
    ls = closed(base, loop_iters)
    mlp = closed(base, loop_iters, net)
    mlp.update(response_gain=gain, factor=f_best, validation_strehl={str(k): v for k, v in val.items()})
    return dict(ls=ls, mlp=mlp, mlp_unscaled=raw, rel_diff=(mlp["strehl_le"] - ls["strehl_le"]) / ls["strehl_le"],
                heldout_rel_err={"mlp": err_mlp, "ls": err_ls}, loss_per_epoch=hist, pairs=n, train_pairs=ntr,
                seconds={"setup": round(t_setup, 1), "pairs": round(t_pairs, 1), "train": round(t_train, 1)},
                net=net)

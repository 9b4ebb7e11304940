"""Learned reconstructor: MLP slopes -> DM commands trained on the GPU.

The network (include/aob200.h, aob_mlp_*) has no counterpart in the reference.
This module holds its Python object, the seeded initialisation, a training
loop over device-resident data, the least-squares DM projector that turns a
residual pupil phase into the training target (the DM commands that best fit
it), and the collection of (slopes, projected residual) pairs from the
closed-loop simulator.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import call, host_array


class MlpReconstructor:
    """3-layer MLP nin -> nh1 -> nh2 -> nout (GELU hidden layers) plus a linear skip
    path nin -> nout, BF16 on the GPU.  ``init_from_ls`` sets the skip path to the
    least-squares command matrix and the last layer to zero, so that the network
    starts as the LS reconstructor and training learns the correction."""

    def __init__(self, nin, nout, nh1=1024, nh2=1024, device=0, seed=0):
        self.h = ctypes.c_void_p()
        call("aob_mlp_create", ctypes.addressof(self.h), int(device), int(nin), int(nh1), int(nh2), int(nout))
        self.nin, self.nh1, self.nh2, self.nout = int(nin), int(nh1), int(nh2), int(nout)
        self.device = int(device)
        self.in_scale, self.out_scale = 1.0, 1.0
        rng = np.random.default_rng(seed)
        dims = [(nh1, nin), (nh2, nh1), (nout, nh2)]
        params = []
        for i, (o, k) in enumerate(dims):
            lim = np.sqrt(6.0 / k) if i < 2 else np.sqrt(3.0 / k)  # He-uniform for GELU layers
            params.append((rng.uniform(-lim, lim, (o, k)).astype(np.float32), np.zeros(o, np.float32)))
        params.append((np.zeros((nout, nin), np.float32), None))  # skip path
        self.set_params(params)

    def __del__(self):
        h = getattr(self, "h", None)
        try:
            if h is not None and h.value and _lib._lib is not None:
                _lib.lib().aob_mlp_destroy(h)
        except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
            pass
        self.h = None

    def set_params(self, params):
        """params: [(W1, b1), (W2, b2), (W3, b3)] and optionally (Ws, None) for the skip path."""
        for l, (w, b) in enumerate(params):
            w = np.ascontiguousarray(w, np.float32)
            b = None if b is None else np.ascontiguousarray(b, np.float32)
            call("aob_mlp_set_params", self.h, l, w.ctypes.data, None if b is None else b.ctypes.data)

    def get_params(self):
        out = []
        dims = [(self.nh1, self.nin), (self.nh2, self.nh1), (self.nout, self.nh2), (self.nout, self.nin)]
        for l, (o, k) in enumerate(dims):
            w, b = np.zeros((o, k), np.float32), np.zeros(o, np.float32)
            call("aob_mlp_get_params", self.h, l, w.ctypes.data, b.ctypes.data)
            out.append((w, b if l < 3 else None))
        return out

    def init_from_ls(self, cmat, in_scale, out_scale):
        """Start as the LS reconstructor: skip path = cmat in the network's scaled
        units, last layer and its bias zero."""
        self.set_scales(in_scale, out_scale)
        p = self.get_params()
        p[2] = (np.zeros_like(p[2][0]), np.zeros_like(p[2][1]))
        p[3] = (np.asarray(cmat, np.float64) / (in_scale * out_scale), None)
        self.set_params(p)

    def set_scales(self, in_scale, out_scale):
        self.in_scale, self.out_scale = float(in_scale), float(out_scale)
        call("aob_mlp_set_scales", self.h, float(in_scale), float(out_scale))

    def forward(self, dev_x, batch, dev_y=None, stream=None):
        call("aob_mlp_forward", self.h, dev_x, int(batch), dev_y, stream)

    def backward(self, dev_t, batch, dev_loss=None, stream=None):
        call("aob_mlp_backward", self.h, dev_t, int(batch), dev_loss, stream)

    def train_step(self, dev_x, dev_t, batch, lr, dev_loss=None, stream=None):
        call("aob_mlp_train_step", self.h, dev_x, dev_t, int(batch), float(lr), dev_loss, stream)

    def infer(self, dev_x, dev_y, stream=None):
        call("aob_mlp_infer", self.h, dev_x, dev_y, stream)

    def set_gemm(self, kind=0):
        """Training GEMMs: 0 the mma.sync kernel, 1 the tcgen05 / TMEM kernel."""
        call("aob_mlp_set_gemm", self.h, int(kind))

    def gemm_status(self, reset=False) -> int:
        s = ctypes.c_uint32()
        call("aob_mlp_gemm_status", self.h, ctypes.addressof(s), 1 if reset else 0)
        return int(s.value)

    def set_mode(self, mode=0):
        """0: one cooperative kernel per control step when it fits, 1: the multi-kernel path."""
        call("aob_mlp_set_mode", self.h, int(mode))

    def comp_com(self, ls, threshold, stream=None):
        call("aob_mlp_comp_com", self.h, ls.h, float(threshold), stream)

    def fallbacks(self, reset=False) -> int:
        n = ctypes.c_uint32()
        call("aob_mlp_fallbacks", self.h, ctypes.addressof(n), 1 if reset else 0)
        return n.value

    def buffer(self, which):
        p, n = ctypes.c_void_p(), ctypes.c_int64()
        call("aob_mlp_buffer", self.h, which.encode(), ctypes.addressof(p), ctypes.addressof(n))
        return p.value, n.value

    def padded_dims(self):
        d = (ctypes.c_int * 4)()
        call("aob_mlp_get_dims", self.h, d)
        return tuple(d)

    def fit(self, X, T, epochs=10, batch=1024, lr=1e-3, seed=0, lr_decay=1.0, scales_from_data=True):
        """Train on device tensors X [n][nin] (slopes) and T [n][nout] (commands);
        returns the mean loss of every epoch.  Scales are set from the data unless
        ``scales_from_data`` is False (keep those of ``init_from_ls``)."""
        import torch

        n = X.shape[0]
        if scales_from_data:
            self.set_scales(1.0 / float(X.std()), float(T.std()))
        gen = torch.Generator(device="cpu").manual_seed(seed)
        loss = torch.zeros(1, device=X.device)
        hist = []
        for ep in range(epochs):
            perm = torch.randperm(n, generator=gen).to(X.device)
            tot, cnt = 0.0, 0
            for i in range(0, n - batch + 1, batch):
                idx = perm[i:i + batch]
                xb = X.index_select(0, idx).contiguous()
                tb = T.index_select(0, idx).contiguous()
                self.train_step(xb.data_ptr(), tb.data_ptr(), batch, lr, loss.data_ptr(),
                                torch.cuda.current_stream().cuda_stream)
                tot += float(loss.item())
                cnt += 1
            hist.append(tot / max(cnt, 1))
            lr *= lr_decay
        return hist


def dm_projector(sys, maxcond=None, rcond=1e-2, sensed_only=False):
    """Projector from the sensor's phase grid to DM commands (float64): the
    least-squares DM fit of a pupil phase, F^+ (influence functions F seen by
    the sensor inside the pupil, singular values below rcond * max dropped),
    restricted to the command modes the interaction matrix senses -- the
    right singular vectors of imat kept by the same condition limit as the LS
    inverse -- so that the target holds no component the slopes cannot see
    (waffle and other unsensed DM patterns).  ``sensed_only``: fit only the
    phase samples inside valid sub-apertures (the sensor's phasemap), not the
    pupil's edge pixels that no slope sees."""
    if sensed_only:
        mask = np.zeros(sys.n * sys.n, bool)
        mask[np.unique(np.asarray(sys.geom.phasemap).ravel())] = True
        mask &= (sys.geom.tel.mpupil > 0).ravel(order="F")
    else:
        mask = (sys.geom.tel.mpupil > 0).ravel(order="F")
    F = np.zeros((int(mask.sum()), sys.nactu))
    com = np.zeros(sys.nactu, np.float32)
    for a in range(sys.nactu):
        com[a] = 1.0
        sys.dm.set_com(com)
        sys.dm.comp_shape()
        sys.trace_wfs(with_atmos=False)
        F[:, a] = np.array(sys.wfs.d_phase).ravel(order="F")[mask]
        com[a] = 0.0
    sys.dm.set_com(com)
    sys.dm.comp_shape()
    F -= F.mean(axis=0, keepdims=True)  # piston is invisible to the sensor
    maxcond = sys.cfg.maxcond if maxcond is None else maxcond
    _, S, Vt = np.linalg.svd(np.asarray(sys.imat, np.float64), full_matrices=False)
    Vk = Vt[S >= S.max() / maxcond].T
    # F^+ through the normal equations (F has many more pupil pixels than
    # actuators): F^T F = V diag(s^2) V^T, singular values below rcond * max dropped
    ev, V = np.linalg.eigh(F.T @ F)
    keep = ev >= (rcond**2) * ev.max()
    Fp = (V[:, keep] / ev[keep]) @ (V[:, keep].T @ F.T)
    return Vk @ (Vk.T @ Fp), mask


def collect_pairs(sys, nsamples, projector, mask, settle=20, nphot_scales=(1.0,)):
    """Run the closed LS loop and record (slopes, DM-projected residual phase) pairs:
    at every step the sensor's phase is the residual the slopes measure, and the
    target is the command vector whose DM shape best fits it."""
    X = np.zeros((nsamples, sys.ls.nslope), np.float32)
    T = np.zeros((nsamples, sys.nactu), np.float32)
    for _ in range(settle):
        sys.next(compute_psf=False)
    base_nphot = sys.geom.nphotons
    for i in range(nsamples):
        sys.wfs.set_nphot(base_nphot * nphot_scales[i % len(nphot_scales)])
        sys.next(compute_psf=False)
        X[i] = np.array(sys.ls.buffer("centroids"))
        phase = np.array(sys.wfs.d_phase).ravel(order="F")[mask].astype(np.float64)
        T[i] = (projector @ (phase - phase.mean())).astype(np.float32)
    sys.wfs.set_nphot(base_nphot)
    return X, T


def collect_open_loop(sys, nsamples, projector, mask, strengths=(0.5, 1.0, 1.5, 2.0), noise=True):
    """Pseudo-open-loop pairs: the atmosphere alone (no DM) at several
    turbulence strengths (the traced phase scaled by each factor in turn), its
    noisy slopes, and the DM-projected phase as the target."""
    X = np.zeros((nsamples, sys.ls.nslope), np.float32)
    T = np.zeros((nsamples, sys.nactu), np.float32)
    d = sys.ls.buffer("centroids")
    for i in range(nsamples):
        sys.atmos.move()
        sys.trace_wfs(with_dm=False)
        ph = np.array(sys.wfs.d_phase) * np.float32(strengths[i % len(strengths)])
        sys.wfs.d_phase.set(ph)
        sys.wfs.comp_image(noise=noise)
        sys.centro.get_cog(d.ptr)
        X[i] = np.array(d)
        v = ph.ravel(order="F")[mask].astype(np.float64)
        T[i] = (projector @ (v - v.mean())).astype(np.float32)
    return X, T


def dm_probe(sys, count=32, amplitude=0.02, seed=11):
    """Noise-free slopes of ``count`` random DM commands (the atmosphere off):
    (commands [count][nactu] float64, slopes [count][nslope] float32).  The LS
    reconstructor returns the commands with unit gain on these."""
    rng = np.random.default_rng(seed)
    C, Sl = [], []
    for _ in range(count):
        c = (rng.standard_normal(sys.nactu) * amplitude).astype(np.float32)
        sys.dm.set_com(c)
        sys.dm.comp_shape()
        sys.trace_wfs(with_atmos=False)
        C.append(c)
        Sl.append(sys.measure_slopes().astype(np.float32))
    sys.dm.set_com(np.zeros(sys.nactu, np.float32))
    sys.dm.comp_shape()
    return np.array(C, np.float64), np.array(Sl, np.float32)


def response_gain(net, probe):
    """Mean response of the network to the probe's slopes, relative to the
    probe's commands (1 for the LS reconstructor)."""
    import torch

    C, Sl = probe
    x = torch.as_tensor(Sl, device="cuda")
    y = torch.zeros((x.shape[0], net.nout), device="cuda")
    net.forward(x.data_ptr(), x.shape[0], y.data_ptr())
    torch.cuda.synchronize()
    Y = y.double().cpu().numpy()
    return float((Y * C).sum() / (C * C).sum())


def collect_closed_loop(systems, nsamples, projector, mask, mags=(6.0, 10.0), segment=100, settle=20, seed=0,
                        batch=256):
    """(slopes, DM-projected residual phase) pairs from closed LS loops, on the
    device (torch tensors X [n][nslope], T [n][nactu]).

    ``systems``: closed ShAoSystem loops of one geometry at several turbulence
    strengths; the pairs cycle through them in segments of ``segment`` steps,
    each segment at a guide-star magnitude drawn uniformly in ``mags`` (the
    photon count scaled from the geometry's, the wCoG threshold kept).  At
    every step the sensor's phase is the residual its slopes measure; the
    target is the command vector whose DM shape best fits it (``projector``,
    applied on the device in batches)."""
    import torch

    rng = np.random.default_rng(seed)
    s0 = systems[0]
    nslope, nactu = s0.ls.nslope, s0.nactu
    X = torch.empty((nsamples, nslope), device="cuda", dtype=torch.float32)
    T = torch.empty((nsamples, nactu), device="cuda", dtype=torch.float32)
    Pt = torch.as_tensor(np.asarray(projector, np.float32), device="cuda")
    idx = torch.as_tensor(np.flatnonzero(mask), device="cuda", dtype=torch.int64)
    PH = torch.empty((batch, idx.numel()), device="cuda", dtype=torch.float32)
    for sy in systems:
        for _ in range(settle):
            sy.next(compute_psf=False)
    views = [(torch.as_tensor(sy.ls.buffer("centroids"), device="cuda"),
              torch.as_tensor(sy.wfs.buffer("phase"), device="cuda")) for sy in systems]
    nph0 = [sy.geom.nphotons for sy in systems]
    i, j0, seg = 0, 0, 0
    while i < nsamples:
        k = seg % len(systems)
        sy = systems[k]
        sy.wfs.set_nphot(nph0[k] * 10.0 ** (-0.4 * (rng.uniform(*mags) - 8.0)))
        cen, ph = views[k]
        for _ in range(min(segment, nsamples - i)):
            sy.next(compute_psf=False)
            X[i].copy_(cen)
            v = ph.index_select(0, idx)
            PH[i - j0].copy_(v - v.mean())
            i += 1
            if i - j0 == batch or i == nsamples:
                T[j0:i] = PH[: i - j0] @ Pt.T
                j0 = i
        sy.wfs.set_nphot(nph0[k])
        seg += 1
    torch.cuda.synchronize()
    return X, T

"""The project's autotuner: picks launch shapes by timing candidates on the device.

Tuned objects and their knobs (none of them changes results -- every kernel
reduces in a fixed order -- only the time):

* ``Batch`` (batched Monte Carlo): sub-apertures per sensor item, threads
  per sensor team, command-matrix KB per MVM item, lag between an
  instance's sensor and MVM items, CTAs per SM, instance order;
* ``Loop`` (one SH loop): sub-apertures per CTA and round in the fused
  single-kernel step.

Each candidate is timed with CUDA events on a private stream (``warmup``
untimed steps, then the mean of ``iters`` steps); timing steps the objects,
so their loop state (commands, noise frame) advances.  A candidate the
library rejects (for instance one whose tiles do not fit in shared memory) is
recorded with its error and skipped; only when no candidate runs does the
search raise.  A failure that leaves the device broken (a sticky CUDA error,
or an expired bounded wait in the object's status word) is raised at once.  The winner is cached
in a JSON file -- ``$AOB_AUTOTUNE_CACHE``, default
``~/.cache/aob200/autotune.json`` -- under a key made of the device name, its
SM count and a signature of the workload's shapes, so a later run with the
same shapes on the same kind of GPU skips the search.
"""

from __future__ import annotations

import ctypes
import hashlib
import json
import os
import time

from ._lib import AobError, call

DEFAULT_BATCH_SPACE = dict(subaps=(16, 32, 64), team=(64, 256), mvm_kb=(48, 96), lag=(16,), ctas_per_sm=(2, 3),
                           order=(0,))
_BATCH_KEYS = ("subaps", "team", "mvm_kb", "lag", "ctas_per_sm", "order")
DEFAULT_LOOP_SPACE = dict(fused_batch=(0, 1, 2, 4, 8))


def cache_path() -> str:
    return os.environ.get("AOB_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "aob200", "autotune.json"))


def _load() -> dict:
    try:
        with open(cache_path()) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(store: dict) -> None:
    p = cache_path()
    try:
        os.makedirs(os.path.dirname(p), exist_ok=True)
        tmp = p + f".{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(store, f, indent=1, sort_keys=True)
        os.replace(tmp, p)
    except OSError:
        pass  # a read-only home only costs the next run a search


def device_key(device: int = 0) -> str:
    buf = ctypes.create_string_buffer(256)
    sms = ctypes.c_int()
    call("aob_device_name", int(device), ctypes.addressof(buf), 256, ctypes.addressof(sms))
    return f"{buf.value.decode()}|{sms.value}sm"


def _sig(parts) -> str:
    return hashlib.sha1(repr(parts).encode()).hexdigest()[:16]


def batch_signature(batch) -> str:
    shapes = []
    for loop in batch.loops:
        w, ls = loop.wfs, loop.ls
        shapes.append((w.nvalid, w.npix, w.nfft, w.nphase, ls.nactu, ls.precision))
    return _sig(shapes)


def _grid(space: dict):
    keys = list(space)
    out = [[]]
    for k in keys:
        out = [o + [v] for o in out for v in space[k]]
    return [dict(zip(keys, o)) for o in out]


def _reraise_if_broken(obj, err):
    """A candidate the library refused on the host leaves the device usable and is
    skipped.  A failure that left a sticky CUDA error or an expired bounded wait
    (``obj.healthy()`` is False) would make every later timing meaningless: it is
    raised at once."""
    healthy = getattr(obj, "healthy", None)
    if healthy is not None and not healthy():
        raise AobError(f"autotune: the device failed while timing a candidate: {err}") from err


def _fastest(trials, what):
    ran = [r for r in trials if r["ms"] is not None]
    if not ran:
        raise AobError(f"autotune: no {what} tuning candidate ran ({trials[0].get('error') if trials else 'empty space'})")
    return min(ran, key=lambda r: r["ms"])


def tune_batch(batch, noise=True, space=None, warmup=3, iters=10, use_cache=True, device=0, log=None):
    """Time every tuning in ``space`` (a dict of candidate lists, see
    DEFAULT_BATCH_SPACE) on ``batch``, apply the fastest and return
    {"tuning": {...}, "ms": t, "trials": [...], "cached": bool}."""
    space = space or DEFAULT_BATCH_SPACE
    key = f"{device_key(device)}|batch|{batch_signature(batch)}|noise={int(bool(noise))}"
    store = _load() if use_cache else {}
    if use_cache and key in store:
        t = store[key]["tuning"]
        batch.set_tuning(*(t.get(k, 0) for k in _BATCH_KEYS))
        return dict(store[key], cached=True)
    trials = []
    for cand in _grid(space):
        cand = {k: cand.get(k, 0) for k in _BATCH_KEYS}
        t0 = time.perf_counter()
        try:
            batch.set_tuning(*(cand[k] for k in _BATCH_KEYS))
            ms = batch.time(noise=noise, warmup=warmup, iters=iters)
        except AobError as e:
            _reraise_if_broken(batch, e)
            trials.append(dict(cand, ms=None, error=str(e)))
            if log:
                log(f"batch tuning {cand}: rejected ({e})")
            continue
        trials.append(dict(cand, ms=ms))
        if log:
            log(f"batch tuning {cand}: {ms * 1e3:.1f} us/step ({time.perf_counter() - t0:.2f} s)")
    best = _fastest(trials, "batch")
    tuning = {k: best[k] for k in _BATCH_KEYS}
    batch.set_tuning(*(tuning[k] for k in _BATCH_KEYS))
    res = dict(tuning=tuning, ms=best["ms"], trials=trials)
    if use_cache:
        store = _load()
        store[key] = res
        _save(store)
    return dict(res, cached=False)


def tune_loop(loop, noise=True, space=None, warmup=3, iters=20, use_cache=True, device=0, log=None):
    """Pick the fused kernel's sub-apertures per CTA and round for ``loop``
    (the loop must fit the fused kernel); returns like tune_batch."""
    from . import core  # noqa: F401  (loop is a core.Loop)

    space = space or DEFAULT_LOOP_SPACE
    w, ls = loop.wfs, loop.ls
    key = (f"{device_key(device)}|loop|"
           f"{_sig((w.nvalid, w.npix, w.nfft, w.nphase, ls.nactu, ls.precision))}|noise={int(bool(noise))}")
    store = _load() if use_cache else {}
    if use_cache and key in store:
        loop.set_mode(0, store[key]["tuning"]["fused_batch"])
        return dict(store[key], cached=True)
    trials = []
    for cand in _grid(space):
        try:
            loop.set_mode(2, cand["fused_batch"])
            ms = loop.time(noise=noise, warmup=warmup, iters=iters)
        except AobError as e:
            _reraise_if_broken(loop, e)
            trials.append(dict(cand, ms=None, error=str(e)))
            if log:
                log(f"loop tuning {cand}: rejected ({e})")
            continue
        trials.append(dict(cand, ms=ms))
        if log:
            log(f"loop tuning {cand}: {ms * 1e3:.1f} us/step")
    best = _fastest(trials, "loop")
    loop.set_mode(0, best["fused_batch"])
    res = dict(tuning={"fused_batch": best["fused_batch"]}, ms=best["ms"], trials=trials)
    if use_cache:
        store = _load()
        store[key] = res
        _save(store)
    return dict(res, cached=False)

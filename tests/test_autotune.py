"""The autotuner on CPU, with stand-in objects for the tuned batch and loop: it
times every candidate, skips the ones the library rejects (AobError), applies
and caches the fastest, and raises only when no candidate runs."""

import types

import pytest

from aob200 import autotune
from aob200._lib import AobError


class FakeBatch:
    """set_tuning / time like aob200.core.Batch; tilings with 256-thread teams
    are rejected, the time is lowest for subaps 32 and 3 CTAs per SM."""

    def __init__(self, reject_all=False):
        w = types.SimpleNamespace(nvalid=1248, npix=6, nfft=32, nphase=6)
        ls = types.SimpleNamespace(nactu=1377, precision=1)
        self.loops = [types.SimpleNamespace(wfs=w, ls=ls)]
        self.reject_all = reject_all
        self.tuning = None
        self.timed = []

    def set_tuning(self, subaps, team, mvm_kb, lag, ctas_per_sm, order):
        self.tuning = (subaps, team, mvm_kb, lag, ctas_per_sm, order)

    def time(self, noise=True, warmup=3, iters=10):
        subaps, team, mvm_kb, lag, ctas, order = self.tuning
        if self.reject_all or team == 256:
            raise AobError("aob_batch_set_tuning: shared memory per CTA exceeds 227 KB")
        self.timed.append(self.tuning)
        return 1.0 + abs(subaps - 32) / 100 + abs(ctas - 3) / 10 + mvm_kb / 1000


@pytest.fixture
def cache(tmp_path, monkeypatch):
    monkeypatch.setenv("AOB_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    monkeypatch.setattr(autotune, "device_key", lambda device=0: "fake|148sm")
    return tmp_path / "autotune.json"


def test_skips_rejected_candidates_and_caches_the_fastest(cache):
    b = FakeBatch()
    res = autotune.tune_batch(b, space=dict(subaps=(16, 32), team=(64, 256), mvm_kb=(48, 96), lag=(16,),
                                            ctas_per_sm=(2, 3), order=(0,)))
    assert not res["cached"]
    assert res["tuning"] == dict(subaps=32, team=64, mvm_kb=48, lag=16, ctas_per_sm=3, order=0)
    assert b.tuning == (32, 64, 48, 16, 3, 0)  # the winner is applied
    rejected = [t for t in res["trials"] if t["ms"] is None]
    assert len(rejected) == 8 and all("227 KB" in t["error"] for t in rejected)
    assert all(t[1] == 64 for t in b.timed)
    assert cache.exists()
    b2 = FakeBatch()
    res2 = autotune.tune_batch(b2)  # same shapes and device: from the cache, nothing timed
    assert res2["cached"] and b2.timed == [] and b2.tuning == (32, 64, 48, 16, 3, 0)


def test_raises_when_no_candidate_runs(cache):
    with pytest.raises(AobError, match="no batch tuning candidate ran"):
        autotune.tune_batch(FakeBatch(reject_all=True), use_cache=False)


def test_a_failure_that_breaks_the_device_is_raised_at_once(cache):
    class BrokenBatch(FakeBatch):
        """The first timing fails and leaves the object unhealthy (as a sticky
        CUDA error or an expired bounded wait would)."""

        def time(self, noise=True, warmup=3, iters=10):
            raise AobError("aob_batch_time: an illegal memory access was encountered")

        def healthy(self):
            return False

    b = BrokenBatch()
    with pytest.raises(AobError, match="device failed while timing"):
        autotune.tune_batch(b, use_cache=False)
    assert b.timed == []

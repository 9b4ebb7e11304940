"""The learned reconstructor at the saxo40 geometry against least squares.

100 k training pairs from closed LS loops at r0 0.08-0.20 m and guide-star
magnitudes 6-10, 16 epochs on the project's tcgen05 GEMM, the output gain
chosen on a validation loop, then both reconstructors on the same held-out
closed loop (r0 0.14 m, magnitude 8, 2000 iterations after 100 settling ones).

Bounds (the accuracy target of the learned reconstructor): the learned loop's long-exposure Strehl at
1.65 um within 1 % of the LS loop's (or above it); on held-out pairs the
network predicts the DM-projected residual with a smaller error than LS.
"""

import pytest

pytestmark = pytest.mark.gpu


def test_learned_reconstructor_matches_ls_strehl_at_saxo40():
    from aob200 import _lib, learned

    if _lib.device_count() < 1:
        pytest.fail("no CUDA device visible to libaob200")
    r = learned.c4_experiment(pairs=100000, epochs=16, loop_iters=2000)
    print(f"LS LE SR {r['ls']['strehl_le']:.4f}, learned {r['mlp']['strehl_le']:.4f} "
          f"(unscaled {r['mlp_unscaled']['strehl_le']:.4f}, response gain {r['mlp']['response_gain']:.3f}, "
          f"factor {r['mlp']['factor']}), held-out error {r['heldout_rel_err']}")
    assert r["heldout_rel_err"]["mlp"] < r["heldout_rel_err"]["ls"]
    assert r["ls"]["strehl_le"] > 0.8
    assert r["rel_diff"] > -0.01, r

"""Workload-level autotuner over the library's speed knobs.

The library's knobs (include/troy_b200.h, "tuning"): the NTT launch variant per
direction for 2^12..2^14 blocks, the key-switch scratch budget (how many
ciphertexts one key-switch launch sequence takes) and whether launches of at most half
the SM count of limbs take the two-CTA form. Every setting computes the same
words, so the tuner may pick any of them: it times the caller's own step function
with CUDA events under each candidate setting and keeps the fastest. Results are
process-wide settings of the library.
"""
from __future__ import annotations

import ctypes

import tb_capi

# NTT launch variants of 2^12..2^14 blocks: 0-2 one CTA per limb at 1, 1/2, 1/4 of the
# default thread count; 3-5 the same thread counts on a two-CTA cluster per limb
NTT_VARIANTS = 6


def _set(logn, fwd, inv, budget, pairs=1):
    lib = tb_capi.lib()
    if 12 <= logn <= 14:
        tb_capi.check(lib.tb_ntt_set_variant(1, logn, fwd))
        tb_capi.check(lib.tb_ntt_set_variant(0, logn, inv))
    lib.tb_keyswitch_set_budget.argtypes = [ctypes.c_uint64]
    tb_capi.check(lib.tb_keyswitch_set_budget(budget))
    tb_capi.check(lib.tb_ntt_set_small_launch_pairs(int(pairs)))


def tune_step(step, logn, stream, reps=3, budgets=(0, 256 << 20, 8 << 30)):
    """Times `step()` (which launches one workload step on `stream`, a torch stream)
    under candidate settings of the NTT variants, the key-switch budget (0 = the
    default) and the small-launch pair rule, one knob at a time (forward variant,
    inverse variant, budget, pair rule), keeps the fastest setting (a change must gain
    at least 1%) and returns {"forward", "inverse", "ks_budget", "small_launch_pairs",
    "ms", "default_ms"}."""
    import torch

    variants = tuple(range(NTT_VARIANTS)) if 12 <= logn <= 14 else (0,)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(setting):
        _set(logn, *setting)
        step()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(reps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    best = (0, 0, 0, 1)
    _set(logn, *best)
    for _ in range(3):   # first calls grow the device pools; keep them out of every timing
        step()
    torch.cuda.synchronize()
    default_ms = best_ms = timed(best)
    for axis, choices in ((0, variants), (1, variants), (2, budgets), (3, (1, 0))):
        for v in choices:
            cand = best[:axis] + (v,) + best[axis + 1:]
            if cand == best:
                continue
            t = timed(cand)
            if t < 0.99 * best_ms:   # a setting must beat the current one by 1% (above noise)
                best, best_ms = cand, t
    fwd, inv, budget, pairs = best
    ms = best_ms
    _set(logn, fwd, inv, budget, pairs)
    return {"forward": fwd, "inverse": inv, "ks_budget": budget or "default", "small_launch_pairs": bool(pairs),
            "ms": round(ms, 4), "default_ms": round(default_ms, 4)}

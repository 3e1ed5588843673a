"""The workload autotuner (seal-cuda_b200/python/tuning.py) times a caller's step under
every candidate setting of the library's speed knobs — NTT launch variants per
direction, key-switch scratch budget, the small-launch pair rule — and keeps the
fastest. Every setting computes the same words: a relinearization step gives the
oracle's words before tuning, under the tuned setting, and under each pair rule."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
import tuning  # noqa: E402
from oracle import Oracle  # noqa: E402


def _rand(rng, moduli, n, lead):
    out = np.empty(tuple(lead) + (len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = rng.integers(0, q, tuple(lead) + (n,), dtype=np.uint64)
    return out


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def test_tuned_settings_give_the_same_words():
    orc = Oracle("orc")
    n, batch = 4096, 6
    moduli = orc.coeff_modulus_create(n, [60, 40, 40, 60])
    ctx = tb_capi.Context(tb_capi.SCHEME_CKKS, n, moduli, 0)
    K = len(moduli)
    L = K - 1
    rng = np.random.default_rng(77)
    hkey = _rand(rng, moduli, n, (K - 1, 2))
    key = _dev(hkey)
    ct3 = _rand(rng, moduli[:L], n, (batch, 3))
    src = _dev(ct3)
    work = torch.empty_like(src)
    stream = torch.cuda.current_stream()

    def step():
        work.copy_(src)
        ctx("relinearize", L, work, 0, key, batch, None)

    def words():
        step()
        torch.cuda.synchronize()
        return work.cpu().numpy().view(np.uint64)[:, :2].copy()

    before = words()
    for b in (0, batch - 1):
        exp = orc.keyswitch(tb_capi.SCHEME_CKKS, n.bit_length() - 1, moduli, 0, ct3[b, 2], ct3[b, :2], hkey)
        assert np.array_equal(before[b], exp), b
    try:
        res = tuning.tune_step(step, n.bit_length() - 1, stream, reps=1)
        assert set(res) == {"forward", "inverse", "ks_budget", "small_launch_pairs", "ms", "default_ms"}
        assert 0 <= res["forward"] < tuning.NTT_VARIANTS and 0 <= res["inverse"] < tuning.NTT_VARIANTS
        assert res["ms"] <= res["default_ms"]
        assert np.array_equal(words(), before)
        for pairs in (0, 1):
            tuning._set(n.bit_length() - 1, res["forward"], res["inverse"], 0, pairs)
            assert np.array_equal(words(), before), pairs
    finally:
        tuning._set(n.bit_length() - 1, 0, 0, 0, 1)   # the library's defaults for later tests

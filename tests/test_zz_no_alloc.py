"""tb_relinearize_noalloc — relinearization for callers that cannot allocate device
memory at call time (a serving loop that reserved all of HBM up front, code running
while another allocator owns the free memory) — gives the same words as
tb_relinearize and as the oracle's key switch, on two calls in a row (the second
reuses the static scratch the first one left behind), for CKKS, BFV and BGV.

This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from oracle import Oracle  # noqa: E402


def _rand(rng, moduli, n, lead):
    out = np.empty(tuple(lead) + (len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = rng.integers(0, q, tuple(lead) + (n,), dtype=np.uint64)
    return out


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


@pytest.mark.parametrize("scheme,n,bits,t,batch", [
    (tb_capi.SCHEME_CKKS, 16384, [60] + [40] * 7 + [60], 0, 3),   # one ciphertext per scratch chunk
    (tb_capi.SCHEME_BFV, 4096, [36, 36, 37], 65537, 5),            # whole batch in one chunk
    (tb_capi.SCHEME_BGV, 4096, [40, 40, 41, 41], 65537, 4),        # BGV's own mod-down
])
def test_noalloc_matches_relinearize_twice(scheme, n, bits, t, batch):
    orc = Oracle("orc")
    moduli = orc.coeff_modulus_create(n, bits)
    ctx = tb_capi.Context(scheme, n, moduli, t)
    K = len(moduli)
    L = K - 1
    logn = n.bit_length() - 1
    rng = np.random.default_rng(n + batch)
    hkey = _rand(rng, moduli, n, (K - 1, 2))
    key = _dev(hkey)
    for call in range(2):
        ct3 = _rand(rng, moduli[:L], n, (batch, 3))
        ref = _dev(ct3)
        got = _dev(ct3)
        ctx("relinearize", L, ref, 0, key, batch, None)
        ctx("relinearize_noalloc", L, got, 0, key, batch, None)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"call {call}"
        # and word for word against the oracle's key switch of c2 into (c0, c1)
        words = got.cpu().numpy().view(np.uint64)
        for b in (0, batch - 1):
            exp = orc.keyswitch(scheme, logn, moduli, t, ct3[b, 2], ct3[b, :2], hkey)
            assert np.array_equal(words[b, :2], exp), f"call {call}, ciphertext {b}"


def test_noalloc_rejects_levels_beyond_its_scratch():
    orc = Oracle("orc")
    n = 16384
    moduli = orc.coeff_modulus_create(n, [60] + [40] * 9 + [60])   # L = 10 needs > 16 MiB per ciphertext
    ctx = tb_capi.Context(tb_capi.SCHEME_CKKS, n, moduli)
    K = len(moduli)
    ct = torch.zeros((1, 3, K - 1, n), dtype=torch.int64, device="cuda")
    key = torch.zeros((K - 1, 2, K, n), dtype=torch.int64, device="cuda")
    with pytest.raises(tb_capi.TroyError) as e:
        ctx("relinearize_noalloc", K - 1, ct, 0, key, 1, None)
    assert e.value.status == 1 and "static scratch" in str(e.value)

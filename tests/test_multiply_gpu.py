"""Parity of batched ciphertext multiplication (BFV BEHZ, BGV, CKKS) with the oracle,
bit-exact, through the C ABI."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402

BFV, CKKS, BGV = 1, 2, 3


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _rand(rng, moduli, n, lead):
    shape = tuple(lead) + (len(moduli), n)
    out = np.empty(shape, np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = rng.integers(0, q, tuple(lead) + (n,), dtype=np.uint64)
    return out


@pytest.mark.parametrize("n,bits,t", [
    (4096, [36, 36, 37], 65537),
    (8192, [43, 43, 44, 44, 44], None),
    (16384, [48] * 9, None),
    (64, [40, 40, 40, 40], None),
    (4096, [50] * 41, 65537),   # 40 and 41 data limbs: the wide run-time form
])
def test_bfv_multiply(orc, n, bits, t):
    moduli = orc.coeff_modulus_create(n, bits)
    if t is None:
        t = orc.plain_modulus_batching(n, 20)
    ctx = tb_capi.Context(BFV, n, moduli, t)
    rng = np.random.default_rng(n)
    K = len(moduli)
    for L in sorted({K - 1, 1 if K > 2 else K - 1, K}):
        data = moduli[:L]
        B = 2
        a = _rand(rng, data, n, (B, 2))
        b = _rand(rng, data, n, (B, 2))
        out = torch.empty((B, 3, L, n), dtype=torch.int64, device="cuda")
        ctx("multiply", L, _dev(a), 0, _dev(b), 0, out, 0, B, None)
        got = _host(out)
        for i in range(B):
            exp = orc.bfv_multiply(n, data, t, a[i], b[i])
            assert np.array_equal(got[i], exp), (L, i)


def test_bgv_and_ckks_multiply(orc):
    n = 4096
    logn = 12
    moduli = orc.coeff_modulus_create(n, [40, 40, 41, 41])
    t = orc.plain_modulus_batching(n, 20)
    rng = np.random.default_rng(5)
    L, B = 3, 2
    data = moduli[:L]
    a = _rand(rng, data, n, (B, 2))
    b = _rand(rng, data, n, (B, 2))
    for scheme in (BGV, CKKS):
        ctx = tb_capi.Context(scheme, n, moduli, t if scheme == BGV else 0)
        out = torch.empty((B, 3, L, n), dtype=torch.int64, device="cuda")
        ctx("multiply", L, _dev(a), 0, _dev(b), 0, out, 0, B, None)
        got = _host(out)
        for i in range(B):
            x, y = a[i], b[i]
            if scheme == BGV:
                x = orc.ntt_forward_rns(logn, data, x)
                y = orc.ntt_forward_rns(logn, data, y)
            d0 = orc.dyadic_rns(data, x[0], y[0])
            d2 = orc.dyadic_rns(data, x[1], y[1])
            s1 = orc.dyadic_rns(data, x[0], y[1]).astype(object) + orc.dyadic_rns(data, x[1], y[0]).astype(object)
            d1 = np.stack([(s1[l] % data[l]).astype(np.uint64) for l in range(L)])
            exp = np.stack([d0, d1, d2])
            if scheme == BGV:
                exp = orc.ntt_inverse_rns(logn, data, exp)
            assert np.array_equal(got[i], exp), (scheme, i)


@pytest.mark.parametrize("bits", [[60, 60, 60, 60], [20, 30, 50, 60], [30, 41, 40, 60]])
def test_ckks_multiply_extreme_words(orc, bits):
    """The CKKS tensor reduces its products with the one-product Barrett reduction (valid
    below 2^(2n+1)); its extremes: every word q - 1 (products (q - 1)^2, sums 2 (q - 1)^2),
    zeros, and words near q, for moduli of 20 .. 60 bits. Checked against the oracle's
    dyadic products."""
    n = 4096
    moduli = orc.coeff_modulus_create(n, bits)
    L, B = len(moduli) - 1, 3
    data = moduli[:L]
    qs = np.asarray(data, np.uint64)[None, None, :, None]
    rng = np.random.default_rng(61)
    a = np.broadcast_to(qs - 1, (B, 2, L, n)).copy()
    b = a.copy()
    a[1] = 0
    a[2] = (qs - 1 - (rng.integers(0, 1 << 16, (2, L, n), dtype=np.uint64) % qs))[0]
    b[2] = (qs - 1 - (rng.integers(0, 1 << 16, (2, L, n), dtype=np.uint64) % qs))[0]
    ctx = tb_capi.Context(CKKS, n, moduli, 0)
    out = torch.empty((B, 3, L, n), dtype=torch.int64, device="cuda")
    ctx("multiply", L, _dev(a), 0, _dev(b), 0, out, 0, B, None)
    got = _host(out)
    for i in range(B):
        x, y = a[i], b[i]
        d0 = orc.dyadic_rns(data, x[0], y[0])
        d2 = orc.dyadic_rns(data, x[1], y[1])
        s1 = orc.dyadic_rns(data, x[0], y[1]).astype(object) + orc.dyadic_rns(data, x[1], y[0]).astype(object)
        d1 = np.stack([(s1[l] % data[l]).astype(np.uint64) for l in range(L)])
        assert np.array_equal(got[i], np.stack([d0, d1, d2])), i

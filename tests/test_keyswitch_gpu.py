"""Parity of batched key switching, relinearization, Galois automorphisms, rescale /
modulus switching and the tensor product with the oracle (bit-exact), through the
C ABI, on random residues at several levels for BFV, CKKS and BGV."""
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


def _rand(rng, moduli, n, lead=()):
    return np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli], axis=-2) if not lead else \
        np.stack([_rand(rng, moduli, n, lead[1:]) for _ in range(lead[0])])


PARAMS = [
    (BFV, 4096, [36, 36, 37], 65537),
    (BGV, 4096, [40, 40, 41, 41], None),
    (CKKS, 4096, [60, 40, 40, 60], 0),
    (CKKS, 16384, [60, 40, 40, 40, 40, 40, 40, 40, 60], 0),
    (BFV, 8192, [43, 43, 44, 44, 44], None),
]


def _setup(orc, scheme, n, bits, t):
    moduli = orc.coeff_modulus_create(n, bits)
    if t is None:
        t = orc.plain_modulus_batching(n, 20)
    return moduli, t, tb_capi.Context(scheme, n, moduli, t)


def _key_sub(key, L):
    return np.ascontiguousarray(np.concatenate([key[:L, :, :L], key[:L, :, -1:]], axis=2))


@pytest.mark.parametrize("scheme,n,bits,t", PARAMS)
def test_keyswitch_batch(orc, scheme, n, bits, t):
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    logn = n.bit_length() - 1
    rng = np.random.default_rng(n + scheme)
    key = _rand(rng, moduli, n, (K - 1, 2))
    dkey = _dev(key)
    for L in sorted({K - 1, max(1, K - 3)}):
        B = 3
        data = moduli[:L]
        target = _rand(rng, data, n, (B,))
        ct = _rand(rng, data, n, (B, 2))
        dct = _dev(ct)
        ctx("keyswitch", L, _dev(target), 0, dct, 0, dkey, B, None)
        got = _host(dct)
        km = data + [moduli[-1]]
        for b in range(B):
            exp = orc.keyswitch(scheme, logn, km, t, target[b], ct[b], _key_sub(key, L))
            assert np.array_equal(got[b], exp), (L, b)


@pytest.mark.parametrize("scheme,n,bits,t", PARAMS[:3])
def test_relinearize_strided(orc, scheme, n, bits, t):
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    logn = n.bit_length() - 1
    rng = np.random.default_rng(7)
    key = _rand(rng, moduli, n, (K - 1, 2))
    L = K - 1
    B = 2
    ct3 = _rand(rng, moduli[:L], n, (B, 3))
    d = _dev(ct3)
    ctx("relinearize", L, d, 0, _dev(key), B, None)
    got = _host(d)
    km = moduli[:L] + [moduli[-1]]
    for b in range(B):
        exp = orc.keyswitch(scheme, logn, km, t, ct3[b, 2], ct3[b, :2], _key_sub(key, L))
        assert np.array_equal(got[b, :2], exp)
        assert np.array_equal(got[b, 2], ct3[b, 2])


@pytest.mark.parametrize("scheme,n,bits,t", PARAMS[:4])
@pytest.mark.parametrize("inplace", [False, True])
def test_apply_galois(orc, scheme, n, bits, t, inplace):
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    logn = n.bit_length() - 1
    rng = np.random.default_rng(11)
    key = _rand(rng, moduli, n, (K - 1, 2))
    L = K - 1
    B = 2
    data = moduli[:L]
    ct = _rand(rng, data, n, (B, 2))
    for step in (1, -3, 0):
        elt = orc.galois_elt_from_step(logn, step)
        import ctypes
        e = ctypes.c_uint32()
        ctx("galois_elt_from_step", step, ctypes.byref(e))
        assert e.value == elt
        din = _dev(ct)
        dout = din if inplace else torch.empty_like(din)
        ctx("apply_galois", L, elt, din, 0, dout, 0, _dev(key), B, None)
        got = _host(dout)
        for b in range(B):
            if scheme == CKKS:
                c0 = np.stack([orc.apply_galois_ntt(logn, elt, ct[b, 0, i]) for i in range(L)])
                tg = np.stack([orc.apply_galois_ntt(logn, elt, ct[b, 1, i]) for i in range(L)])
            else:
                c0 = np.stack([orc.apply_galois(logn, elt, data[i], ct[b, 0, i]) for i in range(L)])
                tg = np.stack([orc.apply_galois(logn, elt, data[i], ct[b, 1, i]) for i in range(L)])
            base = np.stack([c0, np.zeros_like(c0)])
            exp = orc.keyswitch(scheme, logn, data + [moduli[-1]], t, tg, base, _key_sub(key, L))
            assert np.array_equal(got[b], exp), (step, b)


@pytest.mark.parametrize("scheme,n,bits,t", PARAMS)
def test_rescale_mod_switch(orc, scheme, n, bits, t):
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    rng = np.random.default_rng(13)
    op = {BFV: "div_round_last", CKKS: "div_round_last_ntt", BGV: "mod_t_div_last"}[scheme]
    for L in sorted({K - 1, 2}):
        data = moduli[:L]
        P = 4
        x = _rand(rng, data, n, (P,))
        out = torch.empty((P, L - 1, n), dtype=torch.int64, device="cuda")
        ctx("rescale_to_next", L, _dev(x), 0, out, 0, 1, P, None)
        got = _host(out)
        for p in range(P):
            exp = orc.rns_op(op, n, data, t, x[p], L)[: L - 1]
            assert np.array_equal(got[p], exp), (L, p)
        # strided: size-3 ciphertexts, first two polynomials
        x3 = _rand(rng, data, n, (2, 3))
        out2 = torch.empty((2, 2, L - 1, n), dtype=torch.int64, device="cuda")
        ctx("rescale_to_next", L, _dev(x3), 3 * L * n, out2, 0, 2, 2, None)
        got = _host(out2)
        for b in range(2):
            for k in range(2):
                exp = orc.rns_op(op, n, data, t, x3[b, k], L)[: L - 1]
                assert np.array_equal(got[b, k], exp)


def test_tensor_product(orc):
    n = 8192
    moduli = orc.coeff_modulus_create(n, [60, 40, 40, 40, 60])
    ctx = tb_capi.Context(CKKS, n, moduli)
    rng = np.random.default_rng(17)
    L, B = 4, 3
    a = _rand(rng, moduli[:L], n, (B, 2))
    b = _rand(rng, moduli[:L], n, (B, 2))
    out = torch.empty((B, 3, L, n), dtype=torch.int64, device="cuda")
    ctx("tensor_product", 0, L, _dev(a), 0, _dev(b), 0, out, 0, B, None)
    got = _host(out)
    data = moduli[:L]
    for i in range(B):
        d0 = orc.dyadic_rns(data, a[i, 0], b[i, 0])
        d2 = orc.dyadic_rns(data, a[i, 1], b[i, 1])
        x = orc.dyadic_rns(data, a[i, 0], b[i, 1]).astype(object) + orc.dyadic_rns(data, a[i, 1], b[i, 0]).astype(object)
        d1 = np.stack([(x[l] % data[l]).astype(np.uint64) for l in range(L)])
        assert np.array_equal(got[i, 0], d0) and np.array_equal(got[i, 1], d1) and np.array_equal(got[i, 2], d2)


@pytest.mark.parametrize("scheme,n,bits,t", [PARAMS[0], PARAMS[2]])
def test_apply_galois_groups(orc, scheme, n, bits, t):
    """Several rotation steps with different keys in one batched call."""
    import ctypes
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    logn = n.bit_length() - 1
    rng = np.random.default_rng(19)
    L = K - 1
    data = moduli[:L]
    steps = [1, 2, -5]
    counts = [2, 1, 3]
    B = sum(counts)
    keys = [_rand(rng, moduli, n, (K - 1, 2)) for _ in steps]
    dkeys = [_dev(k) for k in keys]
    elts = [orc.galois_elt_from_step(logn, s_) for s_ in steps]
    ct = _rand(rng, data, n, (B, 2))
    din = _dev(ct)
    dout = torch.empty_like(din)
    E = (ctypes.c_uint32 * 3)(*elts)
    C = (ctypes.c_uint64 * 3)(*counts)
    P = (ctypes.c_void_p * 3)(*[k.data_ptr() for k in dkeys])
    ctx("apply_galois_groups", L, 3, E, C, din, 0, dout, 0, P, None)
    got = _host(dout)
    b = 0
    for g, cnt in enumerate(counts):
        for _ in range(cnt):
            if scheme == CKKS:
                c0 = np.stack([orc.apply_galois_ntt(logn, elts[g], ct[b, 0, i]) for i in range(L)])
                tg = np.stack([orc.apply_galois_ntt(logn, elts[g], ct[b, 1, i]) for i in range(L)])
            else:
                c0 = np.stack([orc.apply_galois(logn, elts[g], data[i], ct[b, 0, i]) for i in range(L)])
                tg = np.stack([orc.apply_galois(logn, elts[g], data[i], ct[b, 1, i]) for i in range(L)])
            exp = orc.keyswitch(scheme, logn, data + [moduli[-1]], t, tg, np.stack([c0, np.zeros_like(c0)]),
                                _key_sub(keys[g], L))
            assert np.array_equal(got[b], exp), (g, b)
            b += 1


@pytest.mark.parametrize("scheme,n,bits,t", [p for p in PARAMS if p[1] >= 4096])
def test_persistent_keyswitch_matches_oracle(orc, scheme, n, bits, t):
    """The persistent form (one launch per key-switch step, CTAs taking the next limb
    from a device counter) gives the oracle's words too, for a relinearization and a
    grouped multi-key rotation batch."""
    moduli, t, ctx = _setup(orc, scheme, n, bits, t)
    K = len(moduli)
    logn = n.bit_length() - 1
    rng = np.random.default_rng(n * 3 + scheme)
    key = _rand(rng, moduli, n, (K - 1, 2))
    lib = tb_capi.lib()
    lib.tb_keyswitch_set_persistent(1)
    try:
        assert lib.tb_keyswitch_get_persistent() == 1
        L = K - 1
        B = 5
        ct3 = _rand(rng, moduli[:L], n, (B, 3))
        d = _dev(ct3)
        ctx("relinearize", L, d, 0, _dev(key), B, None)
        got = _host(d)
        for b in (0, 2, B - 1):
            exp = orc.keyswitch(scheme, logn, moduli, t, ct3[b, 2], ct3[b, :2], key)
            assert np.array_equal(got[b, :2], exp), b
    finally:
        lib.tb_keyswitch_set_persistent(0)
    assert lib.tb_keyswitch_get_persistent() == 0


@pytest.mark.parametrize("scheme", [CKKS, BFV])
def test_keyswitch_slack_bounds(orc, scheme):
    """The mod-up transforms defer their reductions and hand the inner product unreduced
    digits: key moduli below 2^57 run no subtraction with estimated quotients (digits
    below 2^61 + 56 q), those below 2^60 subtract at two stages (digits below 16 q).
    Worst cases of those bounds: N = 16384, 57-bit and 58-bit data primes (the largest of
    each form) with random residues near q (products near q^2), 15 digits (the most
    summed unreduced) and 16 digits, where the digits are reduced before the sum; a 60-bit
    special prime in the same launches. Bit-exact against the oracle."""
    n = 16384
    logn = n.bit_length() - 1
    moduli = orc.coeff_modulus_create(n, [57] * 8 + [58] * 8 + [60])
    assert all(q < (1 << 57) for q in moduli[:8]) and all((1 << 57) <= q < (1 << 58) for q in moduli[8:16])
    t = 0 if scheme == CKKS else orc.plain_modulus_batching(n, 20)
    ctx = tb_capi.Context(scheme, n, moduli, t)
    K = len(moduli)
    rng = np.random.default_rng(58)
    key = rng.integers(0, 1, (K - 1, 2, K, n), dtype=np.uint64)
    for j, q in enumerate(moduli):
        key[:, :, j] = rng.integers(q - (q >> 4), q, (K - 1, 2, n), dtype=np.uint64)
    dkey = _dev(key)
    for L in (15, 16):
        data = moduli[:L]
        target = np.stack([rng.integers(q - (q >> 4), q, n, dtype=np.uint64) for q in data])[None]
        ct = _rand(rng, data, n, (1, 2))
        dct = _dev(ct)
        ctx("keyswitch", L, _dev(target), 0, dct, 0, dkey, 1, None)
        exp = orc.keyswitch(scheme, logn, data + [moduli[-1]], t, target[0], ct[0], _key_sub(key, L))
        assert np.array_equal(_host(dct)[0], exp), L


def test_wide_form_takes_unreduced_inputs(orc):
    """Limbs of moduli below 2^57 run the one-CTA forward transforms with no subtraction
    (estimated quotients) and take their inputs unreduced: the mod-up the digit of a larger modulus, the CKKS
    mod-down and rescale the 60-bit residue being dropped. Chain {57, 57, 60} + a 60-bit
    special prime at N = 16384: key switching (60-bit digit into 57-bit moduli, special
    residue into 57-bit limbs) and rescaling (the 60-bit last limb into 57-bit limbs),
    with residues near q, bit-exact against the oracle."""
    n = 16384
    logn = n.bit_length() - 1
    moduli = orc.coeff_modulus_create(n, [57, 57, 60, 60])
    assert moduli[0] < (1 << 57) and moduli[2] >= (1 << 59)
    ctx = tb_capi.Context(CKKS, n, moduli, 0)
    K, L = len(moduli), len(moduli) - 1
    rng = np.random.default_rng(57)

    def near_q(mods, lead):
        return np.stack([rng.integers(q - (q >> 6), q, tuple(lead) + (n,), dtype=np.uint64) for q in mods], axis=-2)

    key = near_q(moduli, (K - 1, 2))
    data = moduli[:L]
    target = near_q(data, (2,))
    ct = near_q(data, (2, 2))
    dct = _dev(ct)
    ctx("keyswitch", L, _dev(target), 0, dct, 0, _dev(key), 2, None)
    got = _host(dct)
    for b in range(2):
        exp = orc.keyswitch(CKKS, logn, data + [moduli[-1]], 0, target[b], ct[b], _key_sub(key, L))
        assert np.array_equal(got[b], exp), b
    x = near_q(data, (3,))
    out = torch.empty((3, L - 1, n), dtype=torch.int64, device="cuda")
    ctx("rescale_to_next", L, _dev(x), 0, out, 0, 1, 3, None)
    got = _host(out)
    for p in range(3):
        assert np.array_equal(got[p], orc.rns_op("div_round_last_ntt", n, data, 0, x[p], L)[: L - 1]), p

"""Parity of the CUDA NTT / inverse NTT / dyadic product with the oracle, through the C ABI.

Bit-exact for full and lazy outputs (the lazy ranges are reproduced exactly).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.parametrize("logn", list(range(1, 18)))
def test_ntt_roundtrip_all_sizes(orc, logn):
    n = 1 << logn
    bits = [50, 50, 40] if logn >= 4 else [30, 30, 30]
    moduli = orc.coeff_modulus_create(n, bits)
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(logn)
    polys = 2 if logn < 15 else 1
    x = np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(polys)])
    d = _dev(x)
    out = torch.empty_like(d)
    for lazy in (0, 1):
        ctx("ntt_forward", d, out, polys, 0, len(moduli), lazy, None)
        got = _host(out)
        exp = orc.ntt_forward_rns(logn, moduli, x, lazy=bool(lazy))
        assert np.array_equal(got, exp), f"forward lazy={lazy}"
        ctx("ntt_inverse", d, out, polys, 0, len(moduli), lazy, None)
        got = _host(out)
        exp = orc.ntt_inverse_rns(logn, moduli, x, lazy=bool(lazy))
        assert np.array_equal(got, exp), f"inverse lazy={lazy}"
    # in-place round trip returns the input
    y = d.clone()
    ctx("ntt_forward", y, y, polys, 0, len(moduli), 0, None)
    ctx("ntt_inverse", y, y, polys, 0, len(moduli), 0, None)
    assert torch.equal(y, d)


def _is_prime(q):
    """Deterministic Miller-Rabin for 64-bit q."""
    if q < 2 or q % 2 == 0:
        return q == 2
    d, r = q - 1, 0
    while d % 2 == 0:
        d, r = d // 2, r + 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, q)
        if x in (1, q - 1):
            continue
        for _ in range(r - 1):
            x = x * x % q
            if x == q - 1:
                break
        else:
            return False
    return True


def _ntt_prime(bits, m):
    """The largest prime below 2^bits that is 1 mod m."""
    q = ((1 << bits) - 1) // m * m + 1
    while not _is_prime(q):
        q -= m
    return q


@pytest.mark.parametrize("logn", [12, 14, 15, 17])
def test_ntt_full_forward_deferred_bounds(orc, logn):
    """Full forward outputs of primes just below 2^60 (the largest whose transforms
    defer their reductions to a bound of 16 q) and of a 61-bit prime (Harvey stages
    throughout), from inputs anywhere in [0, 4q): bit-exact against the oracle."""
    n = 1 << logn
    moduli = orc.coeff_modulus_create(n, [60, 60]) + [_ntt_prime(61, 2 * n)]
    assert moduli[0] >= (1 << 59) and moduli[-1] >= (1 << 60)
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(logn + 60)
    x = np.stack([rng.integers(4 * q - (q >> 3), 4 * q, n, dtype=np.uint64) for q in moduli])
    x[:, ::7] = np.asarray(moduli, np.uint64)[:, None] * 4 - 1
    d = _dev(x)
    out = torch.empty_like(d)
    ctx("ntt_forward", d, out, 1, 0, len(moduli), 0, None)
    assert np.array_equal(_host(out), orc.ntt_forward_rns(logn, moduli, x, lazy=False))


def test_ntt_lazy_input_range(orc):
    """Forward accepts [0, 4q) inputs and inverse [0, 2q) inputs, as the reference."""
    logn, n = 12, 4096
    moduli = orc.coeff_modulus_create(n, [60, 60])
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(3)
    x = np.stack([rng.integers(0, 4 * q, n, dtype=np.uint64) for q in moduli])
    d = _dev(x)
    out = torch.empty_like(d)
    ctx("ntt_forward", d, out, 1, 0, 2, 1, None)
    assert np.array_equal(_host(out), orc.ntt_forward_rns(logn, moduli, x, lazy=True))
    y = np.stack([rng.integers(0, 2 * q, n, dtype=np.uint64) for q in moduli])
    d = _dev(y)
    ctx("ntt_inverse", d, out, 1, 0, 2, 0, None)
    assert np.array_equal(_host(out), orc.ntt_inverse_rns(logn, moduli, y))


def test_dyadic_product(orc):
    n = 8192
    moduli = orc.coeff_modulus_create(n, [60, 50, 40, 36])
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(4)
    a = np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(3)])
    b = np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(3)])
    out = torch.empty(a.shape, dtype=torch.int64, device="cuda")
    ctx("dyadic_product", _dev(a), _dev(b), out, 3, 0, 4, None)
    assert np.array_equal(_host(out), orc.dyadic_rns(moduli, a, b))


def test_batched_ntt_sweep_shapes(orc):
    """The raw NTT sweep: B polynomials x 8 limbs of 50-bit primes, forward, dyadic, inverse."""
    for n, B in ((4096, 16), (16384, 4), (32768, 2)):
        logn = n.bit_length() - 1
        moduli = orc.coeff_modulus_create(n, [50] * 8)
        ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
        rng = np.random.default_rng(n)
        x = np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(B)])
        y = np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(B)])
        dx, dy = _dev(x), _dev(y)
        ctx("ntt_forward", dx, dx, B, 0, 8, 0, None)
        ctx("ntt_forward", dy, dy, B, 0, 8, 0, None)
        dz = torch.empty_like(dx)
        ctx("dyadic_product", dx, dy, dz, B, 0, 8, None)
        ctx("ntt_inverse", dz, dz, B, 0, 8, 0, None)
        ex = orc.ntt_forward_rns(logn, moduli, x)
        ey = orc.ntt_forward_rns(logn, moduli, y)
        ez = orc.ntt_inverse_rns(logn, moduli, orc.dyadic_rns(moduli, ex, ey))
        assert np.array_equal(_host(dz), ez), n


@pytest.mark.parametrize("logn", [12, 13, 14, 15, 16])
def test_ntt_launch_variants_are_identical(orc, logn):
    """Every launch variant of the 2^12..2^14 block kernels (thread counts, one CTA or a
    two-CTA cluster per limb; the split transform of longer limbs takes the one-CTA form)
    gives the oracle's words, and the autotuner keeps a valid choice."""
    lib = tb_capi.lib()
    n = 1 << logn
    moduli = orc.coeff_modulus_create(n, [50, 50, 40])
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(100 + logn)
    x = np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli])[None]
    d = _dev(x)
    out = torch.empty_like(d)
    exp_f = orc.ntt_forward_rns(logn, moduli, x, lazy=False)
    exp_i = orc.ntt_inverse_rns(logn, moduli, x, lazy=False)
    try:
        tb_capi.check(lib.tb_ntt_set_small_launch_pairs(0))   # every launch takes the set variant
        for v in range(6):
            for b in (12, 13, 14):
                tb_capi.check(lib.tb_ntt_set_variant(1, b, v))
                tb_capi.check(lib.tb_ntt_set_variant(0, b, v))
            ctx("ntt_forward", d, out, 1, 0, len(moduli), 0, None)
            assert np.array_equal(_host(out), exp_f), v
            ctx("ntt_inverse", d, out, 1, 0, len(moduli), 0, None)
            assert np.array_equal(_host(out), exp_i), v
        import ctypes
        f, i = ctypes.c_int(-1), ctypes.c_int(-1)
        ctx("autotune_ntt", 64, None, ctypes.byref(f), ctypes.byref(i))
        assert f.value in range(6) and i.value in range(6)
        ctx("ntt_forward", d, out, 1, 0, len(moduli), 0, None)
        assert np.array_equal(_host(out), exp_f)
    finally:
        lib.tb_ntt_set_small_launch_pairs(1)
        for b in (12, 13, 14):
            lib.tb_ntt_set_variant(1, b, 0)
            lib.tb_ntt_set_variant(0, b, 0)


@pytest.mark.parametrize("logn", [12, 13, 14, 15])
def test_raw_ntt_dyadic_sweep_configuration(orc, logn):
    """The raw NTT / dyadic / inverse NTT workload: L = 8 distinct 50-bit primes
    = 1 mod 2N, batches of 1 and 16 polynomials checked word for word against the
    oracle (forward, dyadic product of pairs, inverse); a batch of 256 checked by
    size-independent properties (round trip, linearity of the transform) and spot
    polynomials against the oracle."""
    n = 1 << logn
    moduli = orc.coeff_modulus_create(n, [50] * 8)
    ctx = tb_capi.Context(tb_capi.SCHEME_RAW, n, moduli)
    rng = np.random.default_rng(7000 + logn)

    def rand(b):
        return np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli]) for _ in range(b)])

    for B in (1, 16):
        x, y = rand(B), rand(B)
        dx, dy = _dev(x), _dev(y)
        ctx("ntt_forward", dx, dx, B, 0, 8, 0, None)
        ctx("ntt_forward", dy, dy, B, 0, 8, 0, None)
        fx = orc.ntt_forward_rns(logn, moduli, x)
        assert np.array_equal(_host(dx), fx)
        z = torch.empty_like(dx)
        ctx("dyadic_product", dx, dy, z, B, 0, 8, None)
        fz = np.stack([orc.dyadic_rns(moduli, fx[b], orc.ntt_forward_rns(logn, moduli, y[b:b + 1])[0])
                       for b in range(B)])
        assert np.array_equal(_host(z), fz)
        ctx("ntt_inverse", z, z, B, 0, 8, 0, None)
        assert np.array_equal(_host(z), orc.ntt_inverse_rns(logn, moduli, fz))
    B = 256 if logn <= 14 else 64
    x = torch.remainder(torch.randint(0, 2 ** 62, (B, 8, n), dtype=torch.int64, device="cuda"),
                        torch.tensor(moduli, dtype=torch.int64, device="cuda").view(8, 1))
    y = x.clone()
    ctx("ntt_forward", y, y, B, 0, 8, 0, None)
    for b in (0, B // 2, B - 1):
        assert np.array_equal(_host(y[b]), orc.ntt_forward_rns(logn, moduli, _host(x[b])[None])[0])
    # linearity: NTT(x + x') = NTT(x) + NTT(x') limb-wise mod q
    x2 = torch.roll(x, 1, 0)
    s = torch.remainder(x + x2, torch.tensor(moduli, dtype=torch.int64, device="cuda").view(8, 1))
    ctx("ntt_forward", s, s, B, 0, 8, 0, None)
    y2 = torch.roll(y, 1, 0)
    assert torch.equal(s, torch.remainder(y + y2, torch.tensor(moduli, dtype=torch.int64, device="cuda").view(8, 1)))
    ctx("ntt_inverse", y, y, B, 0, 8, 0, None)
    assert torch.equal(y, x)


def test_integer_ceiling_is_measured():
    """The butterfly-rate microbenchmarks run and report plausible rates (between 1e10
    and 1e14 butterflies per second on one GPU); the butterfly without the conditional
    subtraction is not slower than the one with it, nor the estimated-quotient one than
    that."""
    import ctypes
    lib = tb_capi.lib()
    rates = []
    for fn in (lib.tb_measure_butterfly_rate, lib.tb_measure_slack_butterfly_rate, lib.tb_measure_wide_butterfly_rate):
        fn.argtypes = [ctypes.c_uint64, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
        r = ctypes.c_double(0)
        tb_capi.check(fn((1 << 60) - 93, None, ctypes.byref(r)))
        assert 1e10 < r.value < 1e14
        rates.append(r.value)
    assert rates[1] > 0.95 * rates[0] and rates[2] > 0.95 * rates[1]
    # the machine's 64-bit multiply throughputs bound the exact-quotient butterflies: one
    # high and two low 64-bit products each (the wide form estimates its quotient from
    # 32-bit products and is not bound by this)
    mul = lib.tb_measure_mul64_rate
    mul.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    lo, hi = ctypes.c_double(0), ctypes.c_double(0)
    tb_capi.check(mul(0, None, ctypes.byref(lo)))
    tb_capi.check(mul(1, None, ctypes.byref(hi)))
    bound = 1.0 / (1.0 / hi.value + 2.0 / lo.value)
    assert max(rates[:2]) <= 1.05 * bound, (rates, lo.value, hi.value)

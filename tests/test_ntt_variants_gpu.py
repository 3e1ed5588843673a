"""Every NTT launch variant inside the fused operations: with variants 0..5 forced for
the ring degree's block size (one CTA or a two-CTA cluster per limb, three thread counts
each), and with the default (variant 0, launches smaller than the SM count on CTA
pairs), seeded BFV and CKKS chains (encrypt, multiply, relinearize, rotate, mod-switch /
rescale) give the reference CPU path's words at every step."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
import tb_capi  # noqa: E402
from oracle import RefSession, available  # noqa: E402

SEED = [int(x) for x in range(101, 109)]
S = pytroy.SchemeType


def _words(x):
    return np.asarray(x.data(), np.uint64).reshape(-1)


def _same(ref, rid, ct):
    return np.array_equal(ref.ct(rid)["data"].reshape(-1), _words(ct))


def _context(scheme, n, bits, t=None):
    p = pytroy.EncryptionParameters(scheme)
    p.set_poly_modulus_degree(n)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(n, bits))
    if t is not None:
        p.set_plain_modulus(t)
    p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    return pytroy.SEALContext(p)


def _set_variant(logn, v):
    """Variant v for every launch (the small-launch rule off); v = None restores the
    default: variant 0 with small launches on CTA pairs."""
    lib = tb_capi.lib()
    tb_capi.check(lib.tb_ntt_set_variant(1, logn, v or 0))
    tb_capi.check(lib.tb_ntt_set_variant(0, logn, v or 0))
    tb_capi.check(lib.tb_ntt_set_small_launch_pairs(1 if v is None else 0))


VARIANTS = list(range(6)) + [None]


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("variant", VARIANTS)
def test_bfv_chain_under_each_variant(variant):
    n, bits = 8192, [50, 50, 50, 50]
    t = pytroy.PlainModulus.batching(n, 20)
    ctx = _context(S.bfv, n, bits, t)
    ref = RefSession(1, n, [m.value() for m in pytroy.CoeffModulus.create(n, bits)], t.value(),
                     np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    rlk = keygen.create_relin_keys()
    gk = keygen.create_galois_keys([1])
    enc = pytroy.BatchEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(40 + (variant or 0))
    a = rng.integers(0, t.value(), n, dtype=np.uint64)
    b = rng.integers(0, t.value(), n, dtype=np.uint64)
    ra, rb = ref.encrypt_slots(a), ref.encrypt_slots(b)
    try:
        _set_variant(13, variant)
        ea, eb = encryptor.encrypt(enc.encode(a)), encryptor.encrypt(enc.encode(b))
        assert _same(ref, ra, ea) and _same(ref, rb, eb)
        m = ev.multiply(ea, eb)
        rm = ref.multiply(ra, rb)
        assert _same(ref, rm, m)
        ev.relinearize_inplace(m, rlk)
        rm = ref.relinearize(rm)
        assert _same(ref, rm, m)
        r = ev.rotate_rows(m, 1, gk)
        rr = ref.rotate_rows(rm, 1)
        assert _same(ref, rr, r)
        ms = ev.mod_switch_to_next(r)
        assert _same(ref, ref.mod_switch(rr), ms)
    finally:
        _set_variant(13, None)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("variant", VARIANTS)
def test_ckks_chain_under_each_variant(variant):
    n, bits, scale = 16384, [60] + [40] * 5 + [60], 2.0 ** 40
    ctx = _context(S.ckks, n, bits)
    ref = RefSession(2, n, [m.value() for m in pytroy.CoeffModulus.create(n, bits)], 0, np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    rlk = keygen.create_relin_keys()
    gk = keygen.create_galois_keys([1])
    enc = pytroy.CKKSEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(50 + (variant or 0))
    v = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    w = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ra, rb = ref.encrypt_ckks(v, scale), ref.encrypt_ckks(w, scale)
    try:
        _set_variant(14, variant)
        ea, eb = encryptor.encrypt(enc.encode(v, scale)), encryptor.encrypt(enc.encode(w, scale))
        assert _same(ref, ra, ea) and _same(ref, rb, eb)
        m = ev.multiply(ea, eb)
        rm = ref.multiply(ra, rb)
        assert _same(ref, rm, m)
        ev.relinearize_inplace(m, rlk)
        rm = ref.relinearize(rm)
        assert _same(ref, rm, m)
        ev.rescale_to_next_inplace(m)
        rm = ref.rescale(rm)
        assert _same(ref, rm, m)
        r = ev.rotate_vector(m, 1, gk)
        assert _same(ref, ref.rotate_vector(rm, 1), r)
        got = enc.decode(pytroy.Decryptor(ctx, keygen.secret_key()).decrypt(r))
        assert np.abs(got - np.roll(v * w, -1)).max() < 1e-4
    finally:
        _set_variant(14, None)

"""Ring degrees 32768, 65536 and 131072 through the fused operations (each limb on a
cluster of two, four or eight CTAs exchanging the stages that join their blocks
through distributed shared memory): seeded BFV, BGV and CKKS chains (encrypt,
multiply, relinearize, rotate, mod-switch / rescale) give the reference CPU path's
words at every step. Degrees above 32768 have no 128-bit security table in the
reference, so every context here is made with SecurityLevel.none, as the reference
session is."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
from oracle import RefSession, available  # noqa: E402

N = 32768   # the BFV test with more than 16 data limbs
DEGREES = [32768, 65536, 131072]
SEED = [int(x) for x in range(101, 109)]
S = pytroy.SchemeType


def _words(x):
    return np.asarray(x.data(), np.uint64).reshape(-1)


def _same(ref, rid, ct):
    return np.array_equal(ref.ct(rid)["data"].reshape(-1), _words(ct))


def _context(scheme, bits, t=None, n=N):
    p = pytroy.EncryptionParameters(scheme)
    p.set_poly_modulus_degree(n)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(n, bits))
    if t is not None:
        p.set_plain_modulus(t)
    p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    return pytroy.SEALContext(p, True, pytroy.SecurityLevel.none)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("N", DEGREES)
@pytest.mark.parametrize("scheme", [S.bfv, S.bgv], ids=["bfv", "bgv"])
def test_batched_schemes_at_large_degrees_match_reference_words(scheme, N):
    bits = [50, 50, 50, 50, 60]
    t = pytroy.PlainModulus.batching(N, 20)
    ctx = _context(scheme, bits, t, N)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(N, bits)]
    ref = RefSession(int(scheme.value), N, moduli, t.value(), np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    rlk = keygen.create_relin_keys()
    gk = keygen.create_galois_keys([1])
    enc = pytroy.BatchEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(32)
    a = rng.integers(0, t.value(), N, dtype=np.uint64)
    b = rng.integers(0, t.value(), N, dtype=np.uint64)
    ea, eb = encryptor.encrypt(enc.encode(a)), encryptor.encrypt(enc.encode(b))
    ra, rb = ref.encrypt_slots(a), ref.encrypt_slots(b)
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
    rs = ref.mod_switch(rr)
    assert _same(ref, rs, ms)
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    prod = (a.astype(object) * b.astype(object)) % t.value()
    half = N // 2
    want = np.concatenate([np.roll(prod[:half], -1), np.roll(prod[half:], -1)]).astype(np.uint64)
    assert np.array_equal(enc.decode(dec.decrypt(ms)), want)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("N", DEGREES)
def test_ckks_at_large_degrees_matches_reference_words(N):
    bits = [60, 40, 40, 40, 60]
    scale = 2.0 ** 40
    ctx = _context(S.ckks, bits, None, N)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(N, bits)]
    ref = RefSession(2, N, moduli, 0, np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    rlk = keygen.create_relin_keys()
    gk = keygen.create_galois_keys([1])
    enc = pytroy.CKKSEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(33)
    v = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    w = rng.uniform(-1, 1, N // 2) + 1j * rng.uniform(-1, 1, N // 2)
    ea, eb = encryptor.encrypt(enc.encode(v, scale)), encryptor.encrypt(enc.encode(w, scale))
    ra, rb = ref.encrypt_ckks(v, scale), ref.encrypt_ckks(w, scale)
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
    rr = ref.rotate_vector(rm, 1)
    assert _same(ref, rr, r)
    got = enc.decode(pytroy.Decryptor(ctx, keygen.secret_key()).decrypt(r))
    want = np.roll(v * w, -1)
    assert np.abs(got - want).max() < 1e-4
    assert np.abs(got - ref.decrypt_ckks(rr, N // 2)).max() < 2.0 ** -20


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_bfv_multiply_with_more_than_16_data_limbs():
    """17 data limbs: past the limb counts the BEHZ kernels are specialised for, the
    run-time form gives the reference's words too."""
    bits = [48] * 18   # 864 bits, within the 128-bit security bound at N = 32768
    t = pytroy.PlainModulus.batching(N, 20)
    ctx = _context(S.bfv, bits, t)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(N, bits)]
    ref = RefSession(1, N, moduli, t.value(), np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    enc = pytroy.BatchEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(34)
    a = rng.integers(0, t.value(), N, dtype=np.uint64)
    b = rng.integers(0, t.value(), N, dtype=np.uint64)
    ea, eb = encryptor.encrypt(enc.encode(a)), encryptor.encrypt(enc.encode(b))
    ra, rb = ref.encrypt_slots(a), ref.encrypt_slots(b)
    m = ev.multiply(ea, eb)
    assert _same(ref, ref.multiply(ra, rb), m)
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    want = ((a.astype(object) * b.astype(object)) % t.value()).astype(np.uint64)
    assert np.array_equal(enc.decode(dec.decrypt(m)), want)

"""Products of unrelinearized ciphertexts (sizes above 2): size 3 x 2 -> 4 and the square of
a size-3 ciphertext -> 5 give the reference CPU path's words for BFV, BGV and CKKS on
seeded parameters, and decrypt to the plaintext products."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
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


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("scheme", [S.bfv, S.bgv], ids=["bfv", "bgv"])
def test_batched_products_of_larger_ciphertexts(scheme):
    n, bits = 8192, [50, 50, 50, 50]   # 200 bits: within the 128-bit security bound
    t = pytroy.PlainModulus.batching(n, 20)
    ctx = _context(scheme, n, bits, t)
    ref = RefSession(int(scheme.value), n, [m.value() for m in pytroy.CoeffModulus.create(n, bits)], t.value(),
                     np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    enc = pytroy.BatchEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(7)
    a = rng.integers(0, t.value(), n, dtype=np.uint64)
    b = rng.integers(0, t.value(), n, dtype=np.uint64)
    ea, eb = encryptor.encrypt(enc.encode(a)), encryptor.encrypt(enc.encode(b))
    ra, rb = ref.encrypt_slots(a), ref.encrypt_slots(b)
    m3 = ev.multiply(ea, eb)
    r3 = ref.multiply(ra, rb)
    assert _same(ref, r3, m3)
    m4 = ev.multiply(m3, eb)
    r4 = ref.multiply(r3, rb)
    assert m4.size() == 4 and _same(ref, r4, m4)
    m5 = ev.square(m3)
    r5 = ref.multiply(r3, r3)
    assert m5.size() == 5 and _same(ref, r5, m5)
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    tv = t.value()
    ab = (a.astype(object) * b.astype(object)) % tv
    assert np.array_equal(enc.decode(dec.decrypt(m4)), (ab * b.astype(object) % tv).astype(np.uint64))
    assert np.array_equal(enc.decode(dec.decrypt(m5)), (ab * ab % tv).astype(np.uint64))


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_ckks_products_of_larger_ciphertexts():
    n, bits, scale = 8192, [60, 50, 50, 50], 2.0 ** 30
    ctx = _context(S.ckks, n, bits)
    ref = RefSession(2, n, [m.value() for m in pytroy.CoeffModulus.create(n, bits)], 0, np.array(SEED, np.uint64))
    keygen = pytroy.KeyGenerator(ctx)
    enc = pytroy.CKKSEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key())
    ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(8)
    v = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    w = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ea, eb = encryptor.encrypt(enc.encode(v, scale)), encryptor.encrypt(enc.encode(w, scale))
    ra, rb = ref.encrypt_ckks(v, scale), ref.encrypt_ckks(w, scale)
    m3 = ev.multiply(ea, eb)
    r3 = ref.multiply(ra, rb)
    m4 = ev.multiply(m3, eb)
    r4 = ref.multiply(r3, rb)
    assert m4.size() == 4 and _same(ref, r4, m4)
    assert m4.scale() == pytest.approx(scale ** 3, rel=1e-15)
    got = enc.decode(pytroy.Decryptor(ctx, keygen.secret_key()).decrypt(m4))
    assert np.abs(got - v * w * w).max() < 1e-3

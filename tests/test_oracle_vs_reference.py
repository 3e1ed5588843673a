"""Random cross-checks of the oracle restatement against the compiled reference
(oracle/_ref). CPU only; skipped where the reference library is not built."""
import numpy as np
import pytest

from oracle import Oracle, RefSession, available
from session import OracleSession

pytestmark = pytest.mark.skipif(not available("ref"), reason="reference library not built")


@pytest.fixture(scope="module")
def ref():
    return Oracle("ref")


@pytest.mark.parametrize("logn,bits", [(3, 20), (10, 36), (12, 50), (13, 60), (14, 40)])
def test_ntt_tables_and_transforms(orc, ref, logn, bits):
    n = 1 << logn
    q = ref.coeff_modulus_create(n, [bits])[0]
    for a, b in zip(orc.ntt_tables(logn, q), ref.ntt_tables(logn, q)):
        assert np.array_equal(a, b)
    rng = np.random.default_rng(logn)
    x = rng.integers(0, q, n, dtype=np.uint64)
    y = rng.integers(0, 4 * q, n, dtype=np.uint64)
    for lazy in (False, True):
        assert np.array_equal(orc.ntt_forward(logn, q, x, lazy), ref.ntt_forward(logn, q, x, lazy))
        assert np.array_equal(orc.ntt_forward(logn, q, y, lazy), ref.ntt_forward(logn, q, y, lazy))
        assert np.array_equal(orc.ntt_inverse(logn, q, x, lazy), ref.ntt_inverse(logn, q, x, lazy))
    assert np.array_equal(orc.dyadic_product(q, x, y % q), ref.dyadic_product(q, x, y % q))


def test_prng_stream_and_samplers(orc, ref):
    seed = np.arange(1, 9, dtype=np.uint64)
    assert np.array_equal(orc.prng_bytes(seed, 0, 9000), ref.prng_bytes(seed, 0, 9000))
    assert np.array_equal(orc.prng_bytes(seed, 4090, 20), ref.prng_bytes(seed, 4090, 20))
    q = ref.coeff_modulus_create(4096, [60, 40, 40, 60])
    for kind in range(3):
        assert np.array_equal(orc.sample(kind, seed, 4096, q), ref.sample(kind, seed, 4096, q)), kind


def test_bsk_61bit_transforms(orc, ref):
    q = ref.coeff_modulus_create(4096, [60, 40, 40, 60])
    _, _, bsk = ref.rns_bases(4096, q, 0)
    rng = np.random.default_rng(9)
    for p in bsk[:2]:
        x = rng.integers(0, p, 4096, dtype=np.uint64)
        for lazy in (False, True):
            assert np.array_equal(orc.ntt_forward(12, p, x, lazy), ref.ntt_forward(12, p, x, lazy))
            assert np.array_equal(orc.ntt_inverse(12, p, x, lazy), ref.ntt_inverse(12, p, x, lazy))


def test_galois(orc, ref):
    for logn in (3, 12):
        n = 1 << logn
        q = ref.coeff_modulus_create(n, [40])[0]
        x = np.random.default_rng(2).integers(0, q, n, dtype=np.uint64)
        for step in ((0, 1, -1) if n == 8 else (0, 1, -1, 2, n // 4 - 1, -(n // 4 - 1))):
            e = orc.galois_elt_from_step(logn, step)
            assert e == ref.galois_elt_from_step(logn, step)
            assert np.array_equal(orc.apply_galois(logn, e, q, x), ref.apply_galois(logn, e, q, x))
            assert np.array_equal(orc.apply_galois_ntt(logn, e, x), ref.apply_galois_ntt(logn, e, x))


@pytest.mark.parametrize("scheme,n,bits,t", [(1, 64, [40, 40, 41, 41], None), (3, 128, [40, 40, 40, 40], None),
                                              (2, 128, [60, 40, 40, 40, 60], 0)])
def test_sessions_level_chain(scheme, n, bits, t):
    """Seeded sessions of another shape: encryption through two levels of the chain."""
    ref = Oracle("ref")
    moduli = ref.coeff_modulus_create(n, bits)
    if t is None:
        t = ref.plain_modulus_batching(n, 20)
    seed = np.arange(7, 15, dtype=np.uint64)
    R = RefSession(scheme, n, moduli, t, seed)
    O = OracleSession(scheme, n, moduli, t, seed)
    rlk = R.relin_key()
    assert np.array_equal(O.relin_key(), rlk)
    rng = np.random.default_rng(1)
    if scheme == 2:
        v = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
        ia = R.encrypt_ckks(v, 2.0 ** 30)
    else:
        ia = R.encrypt_slots(rng.integers(0, t, n, dtype=np.uint64))
    c = R.ct(ia)["data"]
    for _ in range(2):
        im = R.multiply(ia, ia)
        ir = R.relinearize(im)
        assert np.array_equal(O.relinearize(O.multiply(c, c), rlk), R.ct(ir)["data"])
        nxt = R.rescale(ir) if scheme == 2 else R.mod_switch(ir)
        assert np.array_equal(O.rescale(R.ct(ir)["data"]), R.ct(nxt)["data"])
        ia, c = nxt, R.ct(nxt)["data"]

"""Host-side parts of the `pytroy` module (no GPU): parameter identifiers, prime
selection and the security table agree with the reference."""
import hashlib

import numpy as np
import pytest

pytroy = pytest.importorskip("pytroy")
from oracle import Oracle, available  # noqa: E402


def _words_hash(words):
    d = hashlib.blake2b(np.asarray(words, np.uint64).tobytes(), digest_size=32).digest()
    return [int(x) for x in np.frombuffer(d, np.uint64)]


@pytest.mark.parametrize("scheme,n,bits,t", [(pytroy.SchemeType.bfv, 4096, [36, 36, 37], 65537),
                                             (pytroy.SchemeType.ckks, 16384, [60] + [40] * 7 + [60], 0),
                                             (pytroy.SchemeType.bgv, 64, [40, 40, 41], 1048193)])
def test_parms_id_is_blake2b_of_the_parameter_words(scheme, n, bits, t):
    q = pytroy.CoeffModulus.create(n, bits)
    p = pytroy.EncryptionParameters(scheme)
    p.set_poly_modulus_degree(n)
    p.set_coeff_modulus(q)
    if t:
        p.set_plain_modulus(t)
    words = [int(scheme.value), n] + [m.value() for m in q] + [t]
    assert p.parms_id() == _words_hash(words)
    if available("ref"):
        assert p.parms_id() == Oracle("ref").parms_id(int(scheme.value), n, [m.value() for m in q], t)


@pytest.mark.parametrize("n,bits", [(64, [40, 40, 41]), (4096, [36, 36, 37]), (8192, [43, 43, 44, 44, 44]),
                                    (16384, [60] + [40] * 7 + [60]), (32768, [50] * 8)])
def test_coeff_modulus_create_matches_oracle(orc, n, bits):
    assert [m.value() for m in pytroy.CoeffModulus.create(n, bits)] == orc.coeff_modulus_create(n, bits)


def test_plain_modulus_and_prime_factor():
    orc = Oracle("orc")
    assert pytroy.PlainModulus.batching(16384, 20).value() == orc.plain_modulus_batching(16384, 20)
    t = pytroy.Modulus(65537)
    for m in pytroy.CoeffModulus.create(4096, t, [40, 40]):
        v = m.value()
        assert m.is_prime() and v % 8192 == 1 and v % 65537 == 1 and v.bit_length() == 40


def test_security_table_and_errors():
    assert pytroy.CoeffModulus.max_bit_count(4096) == 109
    assert pytroy.CoeffModulus.max_bit_count(16384, pytroy.SecurityLevel.tc256) == 237
    with pytest.raises(ValueError):
        pytroy.CoeffModulus.create(4096, [61])
    with pytest.raises(ValueError):
        pytroy.CoeffModulus.create(3000, [40])


def test_invalid_parameters_are_reported_without_a_device():
    p = pytroy.EncryptionParameters(pytroy.SchemeType.bfv)
    p.set_poly_modulus_degree(4096)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(4096, [60, 60]))  # 120 bits > 109
    p.set_plain_modulus(65537)
    ctx = pytroy.SEALContext(p)
    assert not ctx.parameters_set()
    assert ctx.parameter_error_name() == "invalid_parameters_insecure"
    with pytest.raises(ValueError):
        pytroy.KeyGenerator(ctx)


def test_bfv_default_primes_match_the_reference():
    ref = Oracle("ref") if available("ref") else None
    L = pytroy.SecurityLevel
    for sec, bits in ((L.tc128, 128), (L.tc192, 192), (L.tc256, 256)):
        for n in (1024, 2048, 4096, 8192, 16384, 32768):
            got = [m.value() for m in pytroy.CoeffModulus.bfv_default(n, sec)]
            assert sum(q.bit_length() for q in got) <= pytroy.CoeffModulus.max_bit_count(n, sec)
            assert all(pytroy.Modulus(q).is_prime() and q % (2 * n) == 1 for q in got)
            if ref is not None:
                assert got == ref.bfv_default(n, bits), (n, bits)
    with pytest.raises(ValueError):
        pytroy.CoeffModulus.bfv_default(4096, L.none)
    with pytest.raises(ValueError):
        pytroy.CoeffModulus.bfv_default(3000)

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


# valid parameters create the device context, so those cases run on the GPU
_G = pytest.mark.gpu


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("scheme,n,bits,t,sec", [
    pytest.param(pytroy.SchemeType.bfv, 4096, [36, 36, 37], 65537, 128, marks=_G),
    pytest.param(pytroy.SchemeType.bfv, 8192, [43, 43, 44, 44, 44], "batch20", 128, marks=_G),
    pytest.param(pytroy.SchemeType.bgv, 4096, [30, 30, 30], "prime40", 128, marks=_G),   # t above every q_i
    pytest.param(pytroy.SchemeType.ckks, 16384, [60] + [40] * 7 + [60], 0, 128, marks=_G),
    pytest.param(pytroy.SchemeType.bfv, 4096, [60, 60], 65537, 0, marks=_G),              # security none
    (pytroy.SchemeType.ckks, 4096, [60, 60], 0, 128),                                     # insecure
    pytest.param(pytroy.SchemeType.bfv, 4096, [36, 36, 37], 1 << 20, 128, marks=_G),       # no batching
    pytest.param(pytroy.SchemeType.bgv, 4096, [36, 36, 37], 3 * 8191, 128, marks=_G),      # no batching
    (pytroy.SchemeType.bfv, 4096, [36, 36, 37], "q0", 128),                               # t shares a prime
])
def test_context_qualifiers_and_constants_match_the_reference(scheme, n, bits, t, sec):
    q = [m.value() for m in pytroy.CoeffModulus.create(n, bits)]
    if t == "batch20":
        t = pytroy.PlainModulus.batching(n, 20).value()
    elif t == "prime40":
        t = pytroy.CoeffModulus.create(n, [40])[0].value()
    elif t == "q0":
        t = q[0]
    ref = Oracle("ref").context_consts(int(scheme.value), n, q, t, sec)
    p = pytroy.EncryptionParameters(scheme)
    p.set_poly_modulus_degree(n)
    p.set_coeff_modulus([pytroy.Modulus(x) for x in q])
    if scheme != pytroy.SchemeType.ckks:
        p.set_plain_modulus(t)
    levels = {0: pytroy.SecurityLevel.none, 128: pytroy.SecurityLevel.tc128}
    ctx = pytroy.SEALContext(p, True, levels[sec])
    d = ctx.first_context_data()
    qual = d.qualifiers()
    assert int(qual.parameter_error.value) == ref["error"], qual.parameter_error_name()
    for f in ("using_fft", "using_ntt", "using_batching", "using_fast_plain_lift", "using_descending_modulus_chain"):
        assert int(getattr(qual, f)) == ref[f], f
    assert int(qual.sec_level.value) == ref["sec_level"]
    if not qual.parameters_set():
        return
    L = len(d.parms().coeff_modulus())
    assert list(d.total_coeff_modulus()) == ref["total"][:L]
    assert d.plain_upper_half_threshold() == ref["plain_upper_half_threshold"]
    assert list(d.plain_upper_half_increment()) == ref["plain_upper_half_increment"][:L]
    if scheme == pytroy.SchemeType.ckks:
        assert list(d.upper_half_threshold()) == ref["upper_half_threshold"][:L]
    else:
        assert d.coeff_modulus_mod_plain_modulus() == ref["q_mod_t"]
        assert [a for a, _ in d.coeff_div_plain_modulus()] == ref["delta"][:L]
        assert [b for _, b in d.coeff_div_plain_modulus()] == ref["delta_quotient"][:L]
        assert list(d.upper_half_increment()) == ref["upper_half_increment"][:L]

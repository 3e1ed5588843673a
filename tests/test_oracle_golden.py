"""The oracle restatement reproduces every golden fixture generated from the reference
(tests/golden/gen_golden.py) and the reference unit tests' known answers. CPU only."""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle import Oracle
from session import CkksCodec, OracleSession

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SEED = np.arange(101, 109, dtype=np.uint64)


@pytest.fixture(scope="module")
def kat():
    with open(os.path.join(G, "kat.json")) as f:
        return json.load(f)


def test_ntt_known_answers(orc, kat):
    q = kat["ntt_q"]
    for logn, key in ((1, "root_powers_logn1"), (2, "root_powers_logn2")):
        rop, _, iop, _, extra = orc.ntt_tables(logn, q)
        assert [int(x) for x in rop] == kat[key]
        if logn == 1:  # inverse root power 1 inverts root power 1 (test/utils/ntt.cpp:62-64)
            assert int(iop[1]) == pow(int(rop[1]), -1, q)
    for x, y in zip(kat["ntt_logn1"]["in"], kat["ntt_logn1"]["out"]):
        assert [int(v) for v in orc.ntt_forward(1, q, np.array(x, np.uint64))] == y
    # inverse round trip of the reference test at N = 8 (test/utils/ntt.cpp:101-132)
    rng = np.random.default_rng(0)
    x = rng.integers(0, q, 8, dtype=np.uint64)
    assert np.array_equal(orc.ntt_inverse(3, q, orc.ntt_forward(3, q, x)), x)


def test_primes_and_plain_modulus(orc, kat):
    for k, v in kat["coeff_modulus"].items():
        n, bits = k.split(":")
        assert orc.coeff_modulus_create(int(n), [int(b) for b in bits.split(",")]) == v
    for k, v in kat["plain_batching"].items():
        assert orc.plain_modulus_batching(int(k.split(":")[0]), 20) == v


def test_rns_operations(orc):
    z = np.load(os.path.join(G, "rns_n64.npz"))
    for tag in ("bfv", "ckks"):
        q = [int(x) for x in z[f"{tag}_q"]]
        t = int(z[f"{tag}_t"][0])
        bsk = [int(x) for x in z[f"{tag}_bsk"]]
        assert orc.rns_bases(64, q, t)[2] == bsk
        xq, xbm = z[f"{tag}_xq"], z[f"{tag}_xbm"]
        B = len(bsk)
        ops = [("fastbconv_mtilde", xq, B + 1), ("sm_mrq", xbm, B), ("fast_floor", np.concatenate([xq, xbm[:B]]), B),
               ("fastbconv_sk", xbm[:B], len(q)), ("div_round_last", xq, len(q)), ("div_round_last_ntt", xq, len(q))]
        if t:
            ops += [("decrypt_scale_round", xq, 1), ("mod_t_div_last", xq, len(q)), ("decrypt_mod_t", xq, 1)]
        for name, data, ol in ops:
            assert np.array_equal(orc.rns_op(name, 64, q, t, data, ol), z[f"{tag}_{name}"]), (tag, name)


def _session(z, prefix, scheme):
    moduli = [int(x) for x in z[prefix + "moduli"]]
    t = int(z[prefix + "t"][0])
    return OracleSession(scheme, 64, moduli, t, SEED), moduli, t


@pytest.mark.parametrize("name,scheme", [("bfv", 1), ("bgv", 3)])
def test_seeded_bfv_bgv_sessions(name, scheme):
    z = np.load(os.path.join(G, "sessions_n64.npz"))
    p = name + "_"
    s, moduli, t = _session(z, p, scheme)
    assert np.array_equal(s.sk, z[p + "sk"])
    assert np.array_equal(s.pk, z[p + "pk"])
    rlk = s.relin_key()
    assert np.array_equal(rlk, z[p + "rlk"])
    elt = int(z[p + "elt"][0])
    assert np.array_equal(s.galois_key(elt), z[p + "gk"])
    assert np.array_equal(s.encode_slots(z[p + "a"]), z[p + "plain_a"])
    assert np.array_equal(s.encrypt_slots(z[p + "a"]), z[p + "enc_a"])
    mul = s.multiply(z[p + "enc_a"], z[p + "enc_b"])
    assert np.array_equal(mul, z[p + "mul"])
    rel = s.relinearize(z[p + "mul"], rlk)
    assert np.array_equal(rel, z[p + "relin"])
    rot = s.apply_galois(z[p + "relin"], elt, z[p + "gk"])
    assert np.array_equal(rot, z[p + "rot"])
    assert np.array_equal(s.rescale(z[p + "rot"]), z[p + "modswitch"])
    corr = int(z[p + "correction"][0])
    assert np.array_equal(s.decrypt_slots(z[p + "rot"], corr), z[p + "dec"])
    # the decrypted slots are the rotated product
    exp = (z[p + "a"].astype(object) * z[p + "b"].astype(object)) % t
    exp = np.roll(np.array(exp, np.uint64).reshape(2, 32), -1, axis=1).reshape(-1)
    assert np.array_equal(z[p + "dec"], exp)


def test_seeded_ckks_session():
    z = np.load(os.path.join(G, "sessions_n64.npz"))
    p = "ckks_"
    s, moduli, t = _session(z, p, 2)
    assert np.array_equal(s.sk, z[p + "sk"]) and np.array_equal(s.pk, z[p + "pk"])
    rlk = s.relin_key()
    assert np.array_equal(rlk, z[p + "rlk"])
    elt = int(z[p + "elt"][0])
    assert np.array_equal(s.galois_key(elt), z[p + "gk"])
    codec = CkksCodec(64, moduli)
    scale = float(z[p + "scale"][0])
    plain = codec.encode(z[p + "v"], scale, len(moduli) - 1)
    assert np.array_equal(plain.reshape(-1), z[p + "plain_v"])
    assert np.array_equal(s.encrypt_plain(plain), z[p + "enc_a"])
    assert np.array_equal(s.multiply(z[p + "enc_a"], z[p + "enc_b"]), z[p + "mul"])
    assert np.array_equal(s.relinearize(z[p + "mul"], rlk), z[p + "relin"])
    assert np.array_equal(s.rescale(z[p + "relin"]), z[p + "rescale"])
    assert np.array_equal(s.apply_galois(z[p + "rescale"], elt, z[p + "gk"]), z[p + "rot"])
    dec = codec.decode(s.decrypt_plain(z[p + "rot"]), float(z[p + "rot_scale"][0]))
    assert np.abs(dec - z[p + "dec"]).max() < 2.0 ** -20
    exact = np.roll(z[p + "v"] * z[p + "w"], -1)
    assert np.abs(dec - exact).max() < 1e-3


def test_bfv_single_op_configuration_hashes():
    """The full seeded chain at N=4096 {36,36,37}, t=65537 matches the reference's hashes."""
    with open(os.path.join(G, "bfv_n4096.json")) as f:
        ref = json.load(f)
    moduli = ref["moduli"]
    h = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    s = OracleSession(1, 4096, moduli, 65537, SEED)
    assert h(s.sk) == ref["sk"] and h(s.pk) == ref["pk"]
    rlk = s.relin_key()
    assert h(rlk) == ref["rlk"]
    rng = np.random.default_rng(7)
    a = rng.integers(0, 65537, 4096, dtype=np.uint64)
    b = rng.integers(0, 65537, 4096, dtype=np.uint64)
    assert h(a) == ref["a"] and h(b) == ref["b"]
    ea, eb = s.encrypt_slots(a), s.encrypt_slots(b)
    assert h(ea) == ref["enc_a"] and h(eb) == ref["enc_b"]
    m = s.multiply(ea, eb)
    assert h(m) == ref["mul"]
    r = s.relinearize(m, rlk)
    assert h(r) == ref["relin"]
    elt = Oracle("orc").galois_elt_from_step(12, 1)
    gk = s.galois_key(elt)
    assert h(gk) == ref["gk"]
    o = s.apply_galois(r, elt, gk)
    assert h(o) == ref["rot"]
    assert h(s.decrypt_slots(o)) == ref["dec"]

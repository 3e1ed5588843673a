"""The whole seeded chain on the GPU through the C ABI — key generation, batch encoding,
encryption, multiply, relinearize, rotate, modulus switch / rescale, decryption —
reproduces the reference's words (golden fixtures generated from the reference:
tests/golden/gen_golden.py), and the plaintext-side operations match the oracle."""
import ctypes
import hashlib
import json
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from oracle import Oracle  # noqa: E402
from session import OracleSession  # noqa: E402

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SEED = np.arange(101, 109, dtype=np.uint64)
SEEDP = (ctypes.c_uint64 * 8)(*[int(x) for x in SEED])


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.uint64)).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _empty(*shape):
    return torch.empty(shape, dtype=torch.int64, device="cuda")


class GpuSession:
    """Seeded key generation on the device, like the reference's seeded factory."""

    def __init__(self, scheme, n, moduli, t):
        self.ctx = tb_capi.Context(scheme, n, moduli, t)
        self.n, self.K, self.scheme, self.t = n, len(moduli), scheme, t
        self.sk = _empty(self.K, n)
        self.ctx("keygen_secret", SEEDP, self.sk, None)
        self.pk = _empty(2, self.K, n)
        self.ctx("keygen_public", SEEDP, self.sk, self.pk, None)

    def relin_key(self):
        k = _empty(self.K - 1, 2, self.K, self.n)
        self.ctx("keygen_relin", SEEDP, self.sk, k, None)
        return k

    def galois_key(self, elt):
        k = _empty(self.K - 1, 2, self.K, self.n)
        self.ctx("keygen_galois", SEEDP, self.sk, elt, k, None)
        return k


def _chain_bfv_bgv(z, p, scheme):
    moduli = [int(x) for x in z[p + "moduli"]]
    t = int(z[p + "t"][0])
    n = 64
    s = GpuSession(scheme, n, moduli, t)
    assert np.array_equal(_host(s.sk), z[p + "sk"])
    assert np.array_equal(_host(s.pk), z[p + "pk"])
    rlk = s.relin_key()
    assert np.array_equal(_host(rlk), z[p + "rlk"])
    elt = int(z[p + "elt"][0])
    gk = s.galois_key(elt)
    assert np.array_equal(_host(gk), z[p + "gk"])
    L = len(moduli) - 1
    plain = _empty(2, n)
    slots = _dev(np.stack([z[p + "a"], z[p + "b"]]))
    s.ctx("batch_encode", slots, n, n, plain, 2, None)
    assert np.array_equal(_host(plain)[0], z[p + "plain_a"])
    ct = _empty(2, 2, L, n)
    s.ctx("encrypt", SEEDP, s.pk, L, plain, n, n, ct, 0, 2, None)
    assert np.array_equal(_host(ct)[0], z[p + "enc_a"]) and np.array_equal(_host(ct)[1], z[p + "enc_b"])
    m = _empty(1, 3, L, n)
    s.ctx("multiply", L, ct[0:1], 0, ct[1:2], 0, m, 0, 1, None)
    assert np.array_equal(_host(m)[0], z[p + "mul"])
    s.ctx("relinearize", L, m, 0, rlk, 1, None)
    assert np.array_equal(_host(m)[0, :2], z[p + "relin"])
    rot = _empty(1, 2, L, n)
    s.ctx("apply_galois", L, elt, m, 3 * L * n, rot, 0, gk, 1, None)
    assert np.array_equal(_host(rot)[0], z[p + "rot"])
    ms = _empty(1, 2, L - 1, n)
    s.ctx("rescale_to_next", L, rot, 0, ms, 0, 2, 1, None)
    assert np.array_equal(_host(ms)[0], z[p + "modswitch"])
    dec = _empty(1, n)
    s.ctx("decrypt", s.sk, L, 2, rot, 0, dec, 0, int(z[p + "correction"][0]), 1, None)
    out = _empty(1, n)
    s.ctx("batch_decode", dec, out, 0, 1, None)
    assert np.array_equal(_host(out)[0], z[p + "dec"])


def test_bfv_chain_matches_reference_words():
    _chain_bfv_bgv(np.load(os.path.join(G, "sessions_n64.npz")), "bfv_", 1)


def test_bgv_chain_matches_reference_words():
    _chain_bfv_bgv(np.load(os.path.join(G, "sessions_n64.npz")), "bgv_", 3)


def test_ckks_chain_matches_reference_words():
    z = np.load(os.path.join(G, "sessions_n64.npz"))
    p = "ckks_"
    moduli = [int(x) for x in z[p + "moduli"]]
    n = 64
    s = GpuSession(2, n, moduli, 0)
    assert np.array_equal(_host(s.sk), z[p + "sk"]) and np.array_equal(_host(s.pk), z[p + "pk"])
    rlk = s.relin_key()
    assert np.array_equal(_host(rlk), z[p + "rlk"])
    elt = int(z[p + "elt"][0])
    gk = s.galois_key(elt)
    assert np.array_equal(_host(gk), z[p + "gk"])
    L = len(moduli) - 1
    plain = _dev(z[p + "plain_v"].reshape(L, n))
    ct = _empty(1, 2, L, n)
    s.ctx("encrypt", SEEDP, s.pk, L, plain, 0, n, ct, 0, 1, None)
    assert np.array_equal(_host(ct)[0], z[p + "enc_a"])
    m = _empty(1, 3, L, n)
    s.ctx("multiply", L, ct, 0, _dev(z[p + "enc_b"][None]), 0, m, 0, 1, None)
    assert np.array_equal(_host(m)[0], z[p + "mul"])
    s.ctx("relinearize", L, m, 0, rlk, 1, None)
    r = _empty(1, 2, L - 1, n)
    s.ctx("rescale_to_next", L, m, 3 * L * n, r, 0, 2, 1, None)
    assert np.array_equal(_host(r)[0], z[p + "rescale"])
    o = _empty(1, 2, L - 1, n)
    s.ctx("apply_galois", L - 1, elt, r, 0, o, 0, gk, 1, None)
    assert np.array_equal(_host(o)[0], z[p + "rot"])
    ph = _empty(1, L - 1, n)
    s.ctx("decrypt", s.sk, L - 1, 2, o, 0, ph, 0, 1, 1, None)
    O = OracleSession(2, n, moduli, 0, SEED)
    assert np.array_equal(_host(ph)[0], O.decrypt_plain(z[p + "rot"]))


def test_bfv_single_op_configuration_hashes():
    """N=4096 {36,36,37}, t=65537: every array of the seeded chain hashes to the reference's."""
    with open(os.path.join(G, "bfv_n4096.json")) as f:
        ref = json.load(f)
    h = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()
    moduli = ref["moduli"]
    n, L = 4096, 2
    s = GpuSession(1, n, moduli, 65537)
    assert h(_host(s.sk)) == ref["sk"] and h(_host(s.pk)) == ref["pk"]
    rlk = s.relin_key()
    assert h(_host(rlk)) == ref["rlk"]
    elt = Oracle("orc").galois_elt_from_step(12, 1)
    gk = s.galois_key(elt)
    assert h(_host(gk)) == ref["gk"]
    rng = np.random.default_rng(7)
    a = rng.integers(0, 65537, n, dtype=np.uint64)
    b = rng.integers(0, 65537, n, dtype=np.uint64)
    plain = _empty(2, n)
    s.ctx("batch_encode", _dev(np.stack([a, b])), n, n, plain, 2, None)
    ct = _empty(2, 2, L, n)
    s.ctx("encrypt", SEEDP, s.pk, L, plain, n, n, ct, 0, 2, None)
    assert h(_host(ct)[0]) == ref["enc_a"] and h(_host(ct)[1]) == ref["enc_b"]
    m = _empty(1, 3, L, n)
    s.ctx("multiply", L, ct[0:1], 0, ct[1:2], 0, m, 0, 1, None)
    assert h(_host(m)[0]) == ref["mul"]
    s.ctx("relinearize", L, m, 0, rlk, 1, None)
    assert h(_host(m)[0, :2]) == ref["relin"]
    rot = _empty(1, 2, L, n)
    s.ctx("apply_galois", L, elt, m, 3 * L * n, rot, 0, gk, 1, None)
    assert h(_host(rot)[0]) == ref["rot"]
    dec = _empty(1, n)
    s.ctx("decrypt", s.sk, L, 2, rot, 0, dec, 0, 1, 1, None)
    out = _empty(1, n)
    s.ctx("batch_decode", dec, out, 0, 1, None)
    assert h(_host(out)[0]) == ref["dec"]


@pytest.mark.parametrize("scheme,n,bits", [(1, 4096, [36, 36, 37]), (3, 4096, [40, 40, 41])])
def test_plain_ops_and_symmetric_encryption(orc, scheme, n, bits):
    moduli = orc.coeff_modulus_create(n, bits)
    t = orc.plain_modulus_batching(n, 20)
    s = GpuSession(scheme, n, moduli, t)
    O = OracleSession(scheme, n, moduli, t, SEED)
    L = len(moduli) - 1
    rng = np.random.default_rng(n + scheme)
    a = rng.integers(0, t, n, dtype=np.uint64)
    w = rng.integers(0, t, n, dtype=np.uint64)
    ca = O.encrypt_slots(a)
    # multiply_plain with a shared plaintext, two ciphertexts
    pw = O.encode_slots(w)
    cts = _dev(np.stack([ca, ca]))
    out = torch.empty_like(cts)
    s.ctx("multiply_plain", L, 2, cts, 0, _dev(pw), 0, n, out, 0, 2, None)
    exp = O.multiply_plain_slots(ca, w)
    assert np.array_equal(_host(out)[0], exp) and np.array_equal(_host(out)[1], exp)
    # add / sub / negate
    c2 = O.encrypt_slots(w)
    moduli_l = moduli[:L]
    o2 = _empty(1, 2, L, n)
    s.ctx("add", L, 2, _dev(ca[None]), 0, _dev(c2[None]), 0, o2, 0, 1, None)
    assert np.array_equal(_host(o2)[0], np.stack([O._add(moduli_l, ca[k], c2[k]) for k in range(2)]))
    s.ctx("sub", L, 2, _dev(ca[None]), 0, _dev(c2[None]), 0, o2, 0, 1, None)
    dsub = _host(o2)[0]
    s.ctx("negate", L, 2, _dev(ca[None]), 0, o2, 0, 1, None)
    assert np.array_equal(_host(o2)[0], np.stack([O._neg(moduli_l, ca[k]) for k in range(2)]))
    # decrypt(a - w) = a - w slot-wise
    dec = _empty(1, n)
    s.ctx("decrypt", s.sk, L, 2, _dev(dsub[None]), 0, dec, 0, 1, 1, None)
    sl = _empty(1, n)
    s.ctx("batch_decode", dec, sl, 0, 1, None)
    assert np.array_equal(_host(sl)[0], ((a.astype(np.int64) - w.astype(np.int64)) % t).astype(np.uint64))
    # add_plain then decrypt
    ct = _dev(ca[None])
    s.ctx("add_plain", L, ct, 0, _dev(pw), 0, n, 1, None)
    s.ctx("decrypt", s.sk, L, 2, ct, 0, dec, 0, 1, 1, None)
    s.ctx("batch_decode", dec, sl, 0, 1, None)
    assert np.array_equal(_host(sl)[0], ((a + w) % t).astype(np.uint64))
    # symmetric encryption decrypts correctly
    pa = _dev(O.encode_slots(a))
    cs = _empty(1, 2, L, n)
    s.ctx("encrypt_symmetric", None, s.sk, L, pa, 0, n, cs, 0, 1, None)
    s.ctx("decrypt", s.sk, L, 2, cs, 0, dec, 0, 1, 1, None)
    s.ctx("batch_decode", dec, sl, 0, 1, None)
    assert np.array_equal(_host(sl)[0], a)

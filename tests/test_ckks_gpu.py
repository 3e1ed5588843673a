"""CKKS encode / decode on the GPU: encoded plaintext words match the reference's,
decoded values are within 2^-20 of the reference's decode, and a full batched
evaluation decodes to the FP64 plaintext product."""
import ctypes
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from oracle import Oracle, RefSession, available  # noqa: E402
from session import CkksCodec, OracleSession  # noqa: E402

G = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SEED = np.arange(101, 109, dtype=np.uint64)
SEEDP = (ctypes.c_uint64 * 8)(*[int(x) for x in SEED])


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.uint64)).view(np.int64)).cuda()


def _devc(v):
    a = np.ascontiguousarray(np.stack([np.real(v), np.imag(v)], -1).astype(np.float64))
    return torch.from_numpy(a).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def test_encode_decode_match_reference_n64():
    z = np.load(os.path.join(G, "sessions_n64.npz"))
    p = "ckks_"
    moduli = [int(x) for x in z[p + "moduli"]]
    n, L = 64, len(moduli) - 1
    ctx = tb_capi.Context(2, n, moduli)
    scale = float(z[p + "scale"][0])
    plain = torch.empty((1, L, n), dtype=torch.int64, device="cuda")
    ctx("ckks_encode", L, _devc(z[p + "v"]), 0, n // 2, scale, plain, 1, None)
    assert np.array_equal(_host(plain).reshape(-1), z[p + "plain_v"])
    # decode the decrypted rotated product
    O = OracleSession(2, n, moduli, 0, SEED)
    ph = O.decrypt_plain(z[p + "rot"])
    out = torch.empty((1, n // 2, 2), dtype=torch.float64, device="cuda")
    ctx("ckks_decode", L - 1, _dev(ph[None]), float(z[p + "rot_scale"][0]), out, 0, 1, None)
    got = out.cpu().numpy()[0]
    got = got[:, 0] + 1j * got[:, 1]
    assert np.abs(got - z[p + "dec"]).max() < 2.0 ** -20


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_encode_matches_reference_n16384():
    r = Oracle("ref")
    n = 16384
    moduli = r.coeff_modulus_create(n, [60] + [40] * 7 + [60])
    R = RefSession(2, n, moduli, 0, SEED)
    rng = np.random.default_rng(3)
    v = rng.uniform(-1, 1, n // 2) + 1j * rng.uniform(-1, 1, n // 2)
    ref = R.encode_ckks(v, 2.0 ** 40).reshape(len(moduli) - 1, n)
    ctx = tb_capi.Context(2, n, moduli)
    plain = torch.empty((1, len(moduli) - 1, n), dtype=torch.int64, device="cuda")
    ctx("ckks_encode", len(moduli) - 1, _devc(v), 0, n // 2, 2.0 ** 40, plain, 1, None)
    got = _host(plain)[0]
    assert np.array_equal(got, ref)


def test_batched_ckks_evaluation_decodes_to_the_product():
    """Config-style chain at N=16384: encode, encrypt, multiply, relinearize, rescale,
    rotate, decrypt, decode; compared with the FP64 plaintext result and with the
    oracle's decode of the same ciphertext."""
    orc = Oracle("orc")
    n = 16384
    moduli = orc.coeff_modulus_create(n, [60] + [40] * 7 + [60])
    K, L = len(moduli), len(moduli) - 1
    ctx = tb_capi.Context(2, n, moduli)
    sk = torch.empty((K, n), dtype=torch.int64, device="cuda")
    pk = torch.empty((2, K, n), dtype=torch.int64, device="cuda")
    ctx("keygen_secret", SEEDP, sk, None)
    ctx("keygen_public", SEEDP, sk, pk, None)
    rlk = torch.empty((K - 1, 2, K, n), dtype=torch.int64, device="cuda")
    ctx("keygen_relin", SEEDP, sk, rlk, None)
    steps = [1, 2, 4096]
    B = len(steps)
    elts = [orc.galois_elt_from_step(14, k) for k in steps]
    gks = []
    for e in elts:
        g = torch.empty((K - 1, 2, K, n), dtype=torch.int64, device="cuda")
        ctx("keygen_galois", SEEDP, sk, e, g, None)
        gks.append(g)
    rng = np.random.default_rng(11)
    v = rng.uniform(-1, 1, (B, n // 2)) + 1j * rng.uniform(-1, 1, (B, n // 2))
    w = rng.uniform(-1, 1, (B, n // 2)) + 1j * rng.uniform(-1, 1, (B, n // 2))
    scale = 2.0 ** 40
    pv = torch.empty((B, L, n), dtype=torch.int64, device="cuda")
    pw = torch.empty_like(pv)
    ctx("ckks_encode", L, _devc(v), 0, n // 2, scale, pv, B, None)
    ctx("ckks_encode", L, _devc(w), 0, n // 2, scale, pw, B, None)
    ca = torch.empty((B, 2, L, n), dtype=torch.int64, device="cuda")
    cb = torch.empty_like(ca)
    ctx("encrypt", None, pk, L, pv, L * n, 0, ca, 0, B, None)
    ctx("encrypt", None, pk, L, pw, L * n, 0, cb, 0, B, None)
    t3 = torch.empty((B, 3, L, n), dtype=torch.int64, device="cuda")
    ctx("multiply", L, ca, 0, cb, 0, t3, 0, B, None)
    ctx("relinearize", L, t3, 0, rlk, B, None)
    r = torch.empty((B, 2, L - 1, n), dtype=torch.int64, device="cuda")
    ctx("rescale_to_next", L, t3, 3 * L * n, r, 0, 2, B, None)
    o = torch.empty_like(r)
    E = (ctypes.c_uint32 * B)(*elts)
    C = (ctypes.c_uint64 * B)(*([1] * B))
    P = (ctypes.c_void_p * B)(*[g.data_ptr() for g in gks])
    ctx("apply_galois_groups", L - 1, B, E, C, r, 0, o, 0, P, None)
    ph = torch.empty((B, L - 1, n), dtype=torch.int64, device="cuda")
    ctx("decrypt", sk, L - 1, 2, o, 0, ph, 0, 1, B, None)
    out = torch.empty((B, n // 2, 2), dtype=torch.float64, device="cuda")
    new_scale = scale * scale / moduli[L - 1]
    ctx("ckks_decode", L - 1, ph, new_scale, out, 0, B, None)
    got = out.cpu().numpy()
    got = got[..., 0] + 1j * got[..., 1]
    codec = CkksCodec(n, moduli)
    for b, k in enumerate(steps):
        exact = np.roll(v[b] * w[b], -k)
        assert np.abs(got[b] - exact).max() < 2.0 ** -14, b
        ref_dec = codec.decode(_host(ph)[b], new_scale)
        assert np.abs(got[b] - ref_dec).max() < 2.0 ** -20, b


def _cround(x):
    """C round(): halves away from zero (Python's round() rounds halves to even)."""
    import math
    f = math.floor(x)
    d = x - f
    return int(f + 1) if (d > 0.5 or (d == 0.5 and x > 0)) else int(f)


def test_constant_and_coefficient_encoders():
    """Constant encoders write round(value*scale) (or the integer) mod q_l into every
    NTT coefficient (src/ckks.cpp:279-440), negative values negated mod q; the
    coefficient encoder is exact after an inverse NTT and round-trips through
    decode_polynomial."""
    orc = Oracle("orc")
    n = 4096
    moduli = orc.coeff_modulus_create(n, [60, 40, 40, 60])
    L = len(moduli) - 1
    ctx = tb_capi.Context(2, n, moduli)
    plain = torch.empty((L, n), dtype=torch.int64, device="cuda")
    for value, scale in [(-1.5, 2.0 ** 40), (0.3, 2.0 ** 30), (12345.678, 2.0 ** 60)]:
        ctx("ckks_encode_double", L, value, scale, plain, None)
        c = _cround(value * scale)
        exp = np.array([[c % q] * n for q in moduli[:L]], np.uint64)
        assert np.array_equal(_host(plain), exp), (value, scale)
    for value in [-7, 0, 2 ** 40 + 3]:
        ctx("ckks_encode_int64", L, value, plain, None)
        exp = np.array([[((value + q) % 2 ** 64 if value < 0 else value) % q] * n for q in moduli[:L]], np.uint64)
        assert np.array_equal(_host(plain), exp), value
    rng = np.random.default_rng(21)
    coeffs = rng.uniform(-1000, 1000, (2, n))
    pp = torch.empty((2, L, n), dtype=torch.int64, device="cuda")
    ctx("ckks_encode_polynomial", L, torch.from_numpy(coeffs).cuda(), 0, n, 2.0 ** 40, pp, 2, None)
    out = torch.empty((2, n), dtype=torch.float64, device="cuda")
    ctx("ckks_decode_polynomial", L, pp, 2.0 ** 40, out, 0, 2, None)
    assert np.abs(out.cpu().numpy() - coeffs).max() < 2.0 ** -25
    raw = _host(pp)[0]
    coef = np.stack([orc.ntt_inverse(12, q, raw[l].copy()) for l, q in enumerate(moduli[:L])])
    exp = np.array([[_cround(x * 2.0 ** 40) % q for x in coeffs[0]] for q in moduli[:L]], np.uint64)
    assert np.array_equal(coef, exp)

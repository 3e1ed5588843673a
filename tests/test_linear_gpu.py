"""Linear layers on encrypted data on the GPU (Plain2d, Cipher2d, MatmulHelper,
Conv2dHelper of the reference's app/LinearHelper.cuh).

* Word parity with the reference CPU path: the encoded plaintexts equal the numpy
  restatement of the reference's layouts, the symmetric encryptions of the inputs and
  every fused sum of products (conv2d, and matmul with ciphertext weights) equal the
  reference's own encryptSymmetric / multiplyPlain / addInplace words on the same
  seeded parameters, for an unblocked image with channel groups and a blocked one.
* Every product form (ciphertext x plaintext, ciphertext x ciphertext, plaintext x
  ciphertext) decrypts to the product mod t; encoded outputs add in; outputs, encoded
  weights and Cipher2d survive their wire formats; shape errors raise ValueError."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
from linear_layout import Conv2dLayout, MatmulLayout  # noqa: E402
from oracle import RefSession, available  # noqa: E402

S = pytroy.SchemeType
N = 8192
BITS = [43, 43, 44, 44, 44]
SEED = [int(x) for x in range(101, 109)]


def _setup(seeded):
    t = pytroy.PlainModulus.batching(N, 20)
    p = pytroy.EncryptionParameters(S.bfv)
    p.set_poly_modulus_degree(N)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(N, BITS))
    p.set_plain_modulus(t)
    if seeded:
        p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    ns = type("NS", (), {})()
    ns.ctx = pytroy.SEALContext(p)
    ns.t = t.value()
    ns.keygen = pytroy.KeyGenerator(ns.ctx)
    ns.enc = pytroy.BatchEncoder(ns.ctx)
    ns.encryptor = pytroy.Encryptor(ns.ctx, ns.keygen.create_public_key(), ns.keygen.secret_key())
    ns.dec = pytroy.Decryptor(ns.ctx, ns.keygen.secret_key())
    ns.ev = pytroy.Evaluator(ns.ctx)
    return ns


@pytest.fixture(scope="module")
def plain_ctx():
    return _setup(seeded=False)


def _words(c):
    return np.asarray(c.data(), np.uint64)


def _same_poly(pt, vec):
    d = np.asarray(pt.data(), np.uint64)
    v = np.zeros(max(d.size, vec.size), np.uint64)
    v[:vec.size] = vec
    e = np.zeros_like(v)
    e[:d.size] = d
    return np.array_equal(e, v)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("shape", [(1, 30, 30, 3, 3, 12, 2), (1, 100, 100, 3, 3, 2, 2)],
                         ids=["channel-groups", "blocked"])
def test_conv2d_matches_reference_cpu_words(shape):
    ns = _setup(seeded=True)
    lay = Conv2dLayout(*shape, N)
    batch, ih, iw, kh, kw, ic, oc = shape
    rng = np.random.default_rng(ih + ic)
    x = rng.integers(0, ns.t, batch * ic * ih * iw, dtype=np.uint64)
    w = rng.integers(0, ns.t, oc * ic * kh * kw, dtype=np.uint64)
    h = pytroy.Conv2dHelper(*shape, N)
    assert h.total_batch_size() == lay.total
    px, pw = h.encode_inputs(ns.enc, x), h.encode_weights(ns.enc, w)
    xin, win = lay.inputs(x), lay.weights(w)
    for b in range(lay.total):
        assert all(_same_poly(p, v) for p, v in zip(px[b], xin[b])), b
    for o in range(oc):
        assert all(_same_poly(p, v) for p, v in zip(pw[o], win[o])), o
    cts = px.encrypt(ns.encryptor)
    out = h.conv2d(ns.ev, cts, pw)
    ref = RefSession(1, N, [m.value() for m in pytroy.CoeffModulus.create(N, BITS)], ns.t,
                     np.array(SEED, np.uint64))
    for b in range(lay.total):
        ids = [ref.encrypt_poly(v, symmetric=True) for v in xin[b]]
        for g, rid in enumerate(ids):
            assert np.array_equal(ref.ct(rid)["data"].reshape(-1), _words(cts[b][g])), (b, g)
        for o in range(oc):
            acc = None
            for g, rid in enumerate(ids):
                prod = ref.multiply_plain_poly(rid, win[o][g])
                acc = prod if acc is None else ref.add(acc, prod)
            assert np.array_equal(ref.ct(acc)["data"].reshape(-1), _words(out[b][o])), (b, o)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, out), lay.expected(x, w, ns.t).reshape(-1))


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_matmul_with_encrypted_weights_matches_reference_cpu_words():
    """matmul(plain inputs, cipher weights): the fused pass against the reference's
    multiplyPlain(weight ciphertext, input plaintext) + addInplace."""
    ns = _setup(seeded=True)
    batch, inp, out = 2, 700, 24
    lay = MatmulLayout(batch, inp, out, N)
    h = pytroy.MatmulHelper(batch, inp, out, N)
    assert (h.batch_block, h.input_block, h.output_block) == (lay.bb, lay.ib, lay.ob)
    rng = np.random.default_rng(5)
    x = rng.integers(0, ns.t, batch * inp, dtype=np.uint64)
    w = rng.integers(0, ns.t, inp * out, dtype=np.uint64)
    px, pw = h.encode_inputs(ns.enc, x), h.encode_weights(ns.enc, w)
    xin, win = lay.inputs(x), lay.weights(w)
    assert all(_same_poly(p, v) for r, rv in zip(px, xin) for p, v in zip(r, rv))
    assert all(_same_poly(p, v) for r, rv in zip(pw, win) for p, v in zip(r, rv))
    cw = pw.encrypt(ns.encryptor)
    res = h.matmul(ns.ev, px, cw)
    ref = RefSession(1, N, [m.value() for m in pytroy.CoeffModulus.create(N, BITS)], ns.t,
                     np.array(SEED, np.uint64))
    wid = [[ref.encrypt_poly(v, symmetric=True) for v in row] for row in win]
    for bi in range(len(xin)):
        for bj in range(len(win[0])):
            acc = None
            for i in range(len(win)):
                prod = ref.multiply_plain_poly(wid[i][bj], xin[bi][i])
                acc = prod if acc is None else ref.add(acc, prod)
            assert np.array_equal(ref.ct(acc)["data"].reshape(-1), _words(res[bi][bj])), (bi, bj)
    want = (x.reshape(batch, inp).astype(object) @ w.reshape(inp, out).astype(object) % ns.t).astype(np.uint64)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, res), want.reshape(-1))


def test_matmul_forms_outputs_and_wire_formats(plain_ctx):
    ns = plain_ctx
    batch, inp, out = 3, 300, 40
    h = pytroy.MatmulHelper(batch, inp, out, N)
    rng = np.random.default_rng(11)
    x = rng.integers(0, ns.t, batch * inp, dtype=np.uint64)
    w = rng.integers(0, ns.t, inp * out, dtype=np.uint64)
    y = rng.integers(0, ns.t, batch * out, dtype=np.uint64)
    want = (x.reshape(batch, inp).astype(object) @ w.reshape(inp, out).astype(object) % ns.t).astype(np.uint64)
    want = want.reshape(-1)
    pw = h.encode_weights(ns.enc, w)
    cts = h.encrypt_inputs(ns.encryptor, ns.enc, x)
    r1 = h.matmul(ns.ev, cts, pw)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r1), want)
    cw = pw.encrypt(ns.encryptor)
    r2 = h.matmul(ns.ev, cts, cw)                  # ciphertext x ciphertext: size-3 outputs
    assert r2[0][0].size() == 3
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r2), want)
    r3 = h.matmul(ns.ev, h.encode_inputs(ns.enc, x), cw)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r3), want)
    # encoded outputs add in at the output coefficients
    r1.add_plain_inplace(ns.ev, h.encode_outputs(ns.enc, y))
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r1), (want + y) % ns.t)
    # only the output coefficients travel; they decrypt the same
    blob = h.serialize_outputs(ns.ev, r1)
    assert len(blob) < len(r1.save())
    back = h.deserialize_outputs(ns.ev, blob)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, back), (want + y) % ns.t)
    # encoded weights and Cipher2d round trips give identical words
    pw2 = h.deserialize_encoded_weights(h.serialize_encoded_weights(pw))
    r4 = h.matmul(ns.ev, cts, pw2)
    r5 = h.matmul(ns.ev, cts, pw)
    c2 = pytroy.Cipher2d()
    c2.load(r5.save(), ns.ctx)
    for b in range(len(r4)):
        for j in range(len(r4[b])):
            assert np.array_equal(_words(r4[b][j]), _words(r5[b][j]))
            assert np.array_equal(_words(c2[b][j]), _words(r5[b][j]))
    # Cipher2d arithmetic and modulus switching
    s = r5.add_plain(ns.ev, h.encode_outputs(ns.enc, y))
    s.add_inplace(ns.ev, c2)
    s.mod_switch_to_next(ns.ev)
    assert s[0][0].coeff_modulus_size() == len(BITS) - 2
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, s), (2 * want + y) % ns.t)
    with pytest.raises(ValueError):
        s.add_inplace(ns.ev, pytroy.Cipher2d())
    with pytest.raises(ValueError):
        h.matmul(ns.ev, pytroy.Cipher2d([list(cts[0])] * (len(cts) + 1)), pw)   # a batch block too many


@pytest.mark.parametrize("shape", [(2, 12, 12, 3, 3, 4, 3), (1, 100, 96, 5, 3, 2, 2)], ids=["small", "blocked"])
def test_conv2d_forms_outputs_and_wire_formats(plain_ctx, shape):
    ns = plain_ctx
    lay = Conv2dLayout(*shape, N)
    batch, ih, iw, kh, kw, ic, oc = shape
    rng = np.random.default_rng(ih * iw)
    x = rng.integers(0, ns.t, batch * ic * ih * iw, dtype=np.uint64)
    w = rng.integers(0, ns.t, oc * ic * kh * kw, dtype=np.uint64)
    yshape = batch * oc * (ih - kh + 1) * (iw - kw + 1)
    y = rng.integers(0, ns.t, yshape, dtype=np.uint64)
    want = lay.expected(x, w, ns.t).reshape(-1)
    h = pytroy.Conv2dHelper(*shape, N)
    pw = h.encode_weights(ns.enc, w)
    cts = h.encrypt_inputs(ns.encryptor, ns.enc, x)
    r1 = h.conv2d(ns.ev, cts, pw)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r1), want)
    cw = pw.encrypt(ns.encryptor)
    r2 = h.conv2d(ns.ev, cts, cw)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r2), want)
    r3 = h.conv2d(ns.ev, h.encode_inputs(ns.enc, x), cw)
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r3), want)
    h.add_plain_inplace(ns.ev, r1, h.encode_outputs(ns.enc, y))
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, r1), (want + y) % ns.t)
    h.add_inplace(ns.ev, r1, r3)
    back = h.deserialize_outputs(ns.ev, h.serialize_outputs(ns.ev, r1))
    assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, back), (2 * want + y) % ns.t)
    with pytest.raises(ValueError):
        h.encode_weights(ns.enc, w[:-1])
    with pytest.raises(ValueError):
        h.encode_outputs(ns.enc, y[:-1])

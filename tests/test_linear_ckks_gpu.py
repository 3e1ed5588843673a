"""CKKS linear layers on the GPU (the reference's app/LinearHelperCKKS.cuh helpers and
the diagonal matrix-vector product of app/matmul.cuh).

* Word parity with the reference CPU path on the same seeded parameters: the inputs'
  symmetric encryptions, every fused sum of NTT-form products (matmul, conv2d) and the
  diagonal product's rotations, products, rescale and folds equal the reference's own
  encryptSymmetric / multiplyPlain / addInplace / rotateVector / rescaleToNext words,
  given the same encoded plaintext words.
* Decryptions are within 1e-6 (coefficient helpers, scale 2^40 squared) or 1e-4 (after
  a rescale) of the FP64 product; encoded outputs add in; outputs survive their wire
  format; a diagonal step without its own Galois key takes the reference's NAF chain."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
from linear_layout import Conv2dLayout, DiagonalLayout  # noqa: E402
from oracle import RefSession, available  # noqa: E402

N = 8192
BITS = [60, 40, 40, 60]
SEED = [int(x) for x in range(101, 109)]
SCALE = 2.0 ** 40


def _setup():
    p = pytroy.EncryptionParameters(pytroy.SchemeType.ckks)
    p.set_poly_modulus_degree(N)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(N, BITS))
    p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    ns = type("NS", (), {})()
    ns.ctx = pytroy.SEALContext(p)
    ns.keygen = pytroy.KeyGenerator(ns.ctx)
    ns.enc = pytroy.CKKSEncoder(ns.ctx)
    ns.encryptor = pytroy.Encryptor(ns.ctx, ns.keygen.create_public_key(), ns.keygen.secret_key())
    ns.dec = pytroy.Decryptor(ns.ctx, ns.keygen.secret_key())
    ns.ev = pytroy.Evaluator(ns.ctx)
    ns.first = ns.ctx.first_parms_id()
    ns.L = len(BITS) - 1
    return ns


@pytest.fixture(scope="module")
def ns():
    return _setup()


def _ref():
    moduli = [m.value() for m in pytroy.CoeffModulus.create(N, BITS)]
    return RefSession(2, N, moduli, 0, np.array(SEED, np.uint64))


def _words(c):
    return np.asarray(c.data(), np.uint64)


def _same(ref, rid, c):
    return np.array_equal(ref.ct(rid)["data"].reshape(-1), _words(c))


def _ref_sums(ref, cts, pts, terms):
    """The reference's multiplyPlain + addInplace over (input id, plaintext) pairs."""
    acc = None
    for i, pt in terms:
        prod = ref.multiply_plain_words(cts[i], np.asarray(pt.data(), np.uint64), pt.scale())
        acc = prod if acc is None else ref.add(acc, prod)
    return acc


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_ckks_matmul_matches_reference_words_and_decrypts(ns):
    batch, inp, out = 2, 300, 20
    h = pytroy.CkksMatmulHelper(batch, inp, out, N // 2)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, batch * inp)
    w = rng.uniform(-1, 1, inp * out)
    y = rng.uniform(-1, 1, batch * out)
    h.encode_weights(ns.enc, ns.first, w, SCALE)
    px = h.encode_inputs(ns.enc, ns.first, x, SCALE)
    cts = px.encrypt(ns.encryptor)
    res = h.matmul(ns.ev, cts)
    ref = _ref()
    W = h.encoded_weights
    for b in range(batch):
        ids = []
        for i in range(len(px[b])):
            pt = px[b][i]
            ids.append(ref.encrypt_plain_words(np.asarray(pt.data(), np.uint64), pt.scale(), symmetric=True))
            assert _same(ref, ids[-1], cts[b][i]), (b, i)
        for j in range(len(W[0])):
            acc = _ref_sums(ref, ids, None, [(i, W[i][j]) for i in range(len(W))])
            assert _same(ref, acc, res[b][j]), (b, j)
            assert ref.ct(acc)["scale"] == res[b][j].scale()
    want = x.reshape(batch, inp) @ w.reshape(inp, out)
    got = h.decrypt_outputs(ns.enc, ns.dec, res)
    assert np.abs(got - want.reshape(-1)).max() < 1e-6
    h.add_plain_inplace(ns.ev, res, h.encode_outputs(ns.enc, ns.first, y, SCALE * SCALE))
    assert np.abs(h.decrypt_outputs(ns.enc, ns.dec, res) - (want.reshape(-1) + y)).max() < 1e-6
    back = h.deserialize_outputs(ns.ev, h.serialize_outputs(ns.ev, res))
    assert np.abs(h.decrypt_outputs(ns.enc, ns.dec, back) - (want.reshape(-1) + y)).max() < 1e-6
    with pytest.raises(ValueError):
        h.encode_weights(ns.enc, ns.first, w[:-1], SCALE)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
@pytest.mark.parametrize("shape", [(1, 20, 20, 3, 3, 25, 2), (1, 100, 100, 3, 3, 1, 2)], ids=["groups", "blocked"])
def test_ckks_conv2d_matches_reference_words_and_decrypts(ns, shape):
    lay = Conv2dLayout(*shape, N)
    batch, ih, iw, kh, kw, ic, oc = shape
    rng = np.random.default_rng(ih + ic)
    x = rng.uniform(-1, 1, batch * ic * ih * iw)
    w = rng.uniform(-1, 1, oc * ic * kh * kw)
    h = pytroy.CkksConv2dHelper(*shape, N // 2)
    assert h.total_batch_size() == lay.total
    h.encode_weights(ns.enc, ns.first, w, SCALE)
    px = h.encode_inputs(ns.enc, ns.first, x, SCALE)
    cts = px.encrypt(ns.encryptor)
    res = h.conv2d(ns.ev, cts)
    ref = _ref()
    W = h.encoded_weights
    for b in range(lay.total):
        ids = [ref.encrypt_plain_words(np.asarray(pt.data(), np.uint64), pt.scale(), symmetric=True) for pt in px[b]]
        for o in range(oc):
            acc = _ref_sums(ref, ids, None, [(g, W[o][g]) for g in range(len(ids))])
            assert _same(ref, acc, res[b][o]), (b, o)
    # the float convolution, computed as the integer layout's expectation in float64
    X = x.reshape(batch, ic, ih, iw)
    K = w.reshape(oc, ic, kh, kw)
    oyh, oyw = ih - kh + 1, iw - kw + 1
    want = np.zeros((batch, oc, oyh, oyw))
    for ki in range(kh):
        for kj in range(kw):
            want += np.einsum("bchw,oc->bohw", X[:, :, ki:ki + oyh, kj:kj + oyw], K[:, :, ki, kj])
    got = h.decrypt_outputs(ns.enc, ns.dec, res)
    assert np.abs(got - want.reshape(-1)).max() < 1e-6
    yv = rng.uniform(-1, 1, want.size)
    h.add_plain_inplace(ns.ev, res, h.encode_outputs(ns.enc, ns.first, yv, SCALE * SCALE))
    back = h.deserialize_outputs(ns.ev, h.serialize_outputs(ns.ev, res))
    assert np.abs(h.decrypt_outputs(ns.enc, ns.dec, back) - (want.reshape(-1) + yv)).max() < 1e-6


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_diagonal_matmul_matches_reference_words_and_decrypts(ns):
    height, width = 500, 30
    lay = DiagonalLayout(height, width, N // 2)
    assert lay.count == 4
    rng = np.random.default_rng(9)
    m = rng.uniform(-1, 1, (height, width)) + 1j * rng.uniform(-1, 1, (height, width))
    v = rng.uniform(-1, 1, width) + 1j * rng.uniform(-1, 1, width)
    h = pytroy.DiagonalMatmulHelper(height, width, N // 2)
    h.encode(m, ns.enc, SCALE)
    ct = ns.encryptor.encrypt(h.prepare_input(v, ns.enc, SCALE))
    steps = list(range(1, lay.count)) + [lay.count * 2 ** k for k in range(8) if lay.count * 2 ** k < lay.p2]
    gk = ns.keygen.create_galois_keys(steps)
    res = h.multiply(ct, ns.ev, gk, True)
    want = m @ v
    got = h.decode_result(ns.dec.decrypt(res), ns.enc)
    assert np.abs(got - want).max() < 1e-4
    # the reference's sequence on the same input words and diagonals
    ref = _ref()
    rid = ref.ct_from_words(_words(ct), 2, ns.L, True, ct.scale())
    diags = lay.diagonals(m)
    acc = None
    for i in range(lay.count):
        r = rid if i == 0 else ref.rotate_vector(rid, i)
        prod = ref.multiply_plain_words(r, ref.encode_ckks(diags[i], SCALE), SCALE)
        acc = prod if acc is None else ref.add(acc, prod)
    acc = ref.rescale(acc)
    rot = lay.count
    while rot < lay.p2:
        acc = ref.add(acc, ref.rotate_vector(acc, rot))
        rot *= 2
    assert _same(ref, acc, res)
    # without a key for step 3 the rotation goes through its NAF chain (4, then -1)
    gk2 = ns.keygen.create_galois_keys([-1, 1, 2, 4, 8, 16])
    got2 = h.decode_result(ns.dec.decrypt(h.multiply(ct, ns.ev, gk2, True)), ns.enc)
    assert np.abs(got2 - want).max() < 1e-4
    # no rescale: the product keeps scale^2
    res3 = h.multiply(ct, ns.ev, gk, False)
    assert res3.scale() == ct.scale() * SCALE
    assert np.abs(h.decode_result(ns.dec.decrypt(res3), ns.enc) - want).max() < 1e-4

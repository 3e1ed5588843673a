"""Encrypted vector x matrix products and the continuous-batching server on the GPU.

* MatmulHelper (the reference's app/LinearHelper.cuh encodings, products fused into
  one device pass) gives the reference CPU path's words: the reference's own
  multiplyPlain + addInplace per block pair on the same seeded ciphertexts.
* MatmulServer returns, for every request, the same words whether the request ran
  alone or arrived in a Poisson stream and was batched with others, and every result
  decrypts to the plaintext product mod t.
* Admission keeps the device footprint under the budget; a failed wave is reported
  per request and the server keeps serving (host-side fault injection)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")
from oracle import RefSession, available  # noqa: E402

S = pytroy.SchemeType
N = 8192
BITS = [43, 43, 44, 44, 44]
SEED = [int(x) for x in range(101, 109)]


def _context(seeded):
    t = pytroy.PlainModulus.batching(N, 20)
    p = pytroy.EncryptionParameters(S.bfv)
    p.set_poly_modulus_degree(N)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(N, BITS))
    p.set_plain_modulus(t)
    if seeded:
        p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    return pytroy.SEALContext(p), t.value()


def _expected(x, w, t, inp, out):
    return (x.astype(object) @ w.reshape(inp, out).astype(object) % t).astype(np.uint64)


def _ct_bytes(ctx, words):
    """A first-level size-2 coefficient-form ciphertext in the reference's wire format."""
    L = len(BITS) - 1
    head = np.array(ctx.first_parms_id(), np.uint64).tobytes() + b"\x00"
    head += np.array([2, N, L], np.uint64).tobytes() + np.array([1.0]).tobytes()
    head += np.array([1, 0], np.uint64).tobytes() + b"\x00" + np.array([words.size], np.uint64).tobytes()
    return head + np.ascontiguousarray(words, np.uint64).tobytes()


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_matmul_helper_matches_reference_cpu_words():
    ctx, t = _context(seeded=True)
    keygen = pytroy.KeyGenerator(ctx)
    enc = pytroy.BatchEncoder(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.create_public_key(), keygen.secret_key())
    ev = pytroy.Evaluator(ctx)
    inp, out = 300, 40
    h = pytroy.MatmulHelper(1, inp, out, N)
    ib, ob = h.input_block, h.output_block
    rng = np.random.default_rng(17)
    x = rng.integers(0, t, inp, dtype=np.uint64)
    w = rng.integers(0, t, inp * out, dtype=np.uint64)
    cts = h.encrypt_inputs(encryptor, enc, x)
    res = h.matmul(ev, cts, h.encode_weights(enc, w))
    ref = RefSession(1, N, [m.value() for m in pytroy.CoeffModulus.create(N, BITS)], t, np.array(SEED, np.uint64))
    ni, no = (inp + ib - 1) // ib, (out + ob - 1) // ob
    ids = []
    for bi in range(ni):  # encodeInputs layout (app/LinearHelper.cuh:279-300)
        vec = np.zeros(N, np.uint64)
        seg = x[bi * ib:(bi + 1) * ib]
        vec[:seg.size] = seg
        ids.append(ref.encrypt_poly(vec, symmetric=True))  # Plain2d::encrypt is symmetric
        assert np.array_equal(ref.ct(ids[-1])["data"].reshape(-1), np.asarray(cts[0][bi].data(), np.uint64))
    W = w.reshape(inp, out)
    for bj in range(no):
        acc = None
        for bi in range(ni):  # encodeWeightSmall layout (app/LinearHelper.cuh:230-247)
            vec = np.zeros(ib * ob, np.uint64)
            for j in range(bj * ob, min((bj + 1) * ob, out)):
                for i in range(bi * ib, min((bi + 1) * ib, inp)):
                    vec[(j - bj * ob) * ib + ib - (i - bi * ib) - 1] = W[i, j]
            prod = ref.multiply_plain_poly(ids[bi], vec)
            acc = prod if acc is None else ref.add(acc, prod)
        assert np.array_equal(ref.ct(acc)["data"].reshape(-1), np.asarray(res[0][bj].data(), np.uint64)), bj
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    assert np.array_equal(h.decrypt_outputs(enc, dec, res), _expected(x, w, t, inp, out))


@pytest.fixture(scope="module")
def serving():
    ctx, t = _context(seeded=False)
    keygen = pytroy.KeyGenerator(ctx)
    ns = type("NS", (), {})()
    ns.ctx, ns.t = ctx, t
    ns.enc = pytroy.BatchEncoder(ctx)
    ns.encryptor = pytroy.Encryptor(ctx, keygen.create_public_key(), keygen.secret_key())
    ns.dec = pytroy.Decryptor(ctx, keygen.secret_key())
    ns.ev = pytroy.Evaluator(ctx)
    rng = np.random.default_rng(29)
    ns.reqs = []
    for _ in range(24):
        inp = int(rng.integers(1, 17)) * 64
        out = int(rng.integers(1, 17)) * 16
        x = rng.integers(0, t, inp, dtype=np.uint64)
        w = rng.integers(0, t, inp * out, dtype=np.uint64)
        h = pytroy.MatmulHelper(1, inp, out, N)
        cts = h.encrypt_inputs(ns.encryptor, ns.enc, x)
        words = np.concatenate([np.asarray(c.data(), np.uint64) for c in cts[0]])
        ns.reqs.append((inp, out, x, w, h, cts, words))
    return ns


def _run_alone(ns, server):
    outs = []
    for inp, out, x, w, h, cts, words in ns.reqs:
        rid = server.submit(inp, out, words, w, pytroy.MatmulServer.now())
        assert server.drain(60.0)
        o, _, _, ok = server.result(rid)
        assert ok
        outs.append(np.asarray(o))
    return outs


def _out_buffer(k, size):
    """Result buffers given to the server: plain memory for even k, page-locked for odd."""
    if k % 2 == 0:
        return np.zeros(size, np.uint64)
    return torch.zeros(size, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)


def _run_poisson(ns, server, rate, seed, outs=None):
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, len(ns.reqs))
    start = pytroy.MatmulServer.now()
    due = start + np.cumsum(gaps)
    ids, k = [], 0
    deadline = start + 60.0
    while k < len(ns.reqs) or not server.idle():
        now = pytroy.MatmulServer.now()
        while k < len(ns.reqs) and due[k] <= now:
            inp, out, x, w, h, cts, words = ns.reqs[k]
            dst = None if outs is None else outs[k]
            ids.append(server.submit(inp, out, words, w, float(due[k]), outputs=dst))
            k += 1
        server.step()
        assert now < deadline
    return ids


def test_server_results_identical_alone_and_in_the_mix(serving):
    ns = serving
    alone = _run_alone(ns, pytroy.MatmulServer(ns.ctx, slots=3))
    server = pytroy.MatmulServer(ns.ctx, slots=3)
    ids = _run_poisson(ns, server, rate=5000.0, seed=3)
    st = server.stats()
    assert st["completed"] == len(ns.reqs) and st["failed"] == 0
    assert st["max_wave"] > 1  # requests really were batched together
    L = len(BITS) - 1
    # the same stream with caller-owned result buffers (plain and page-locked memory)
    outs = [_out_buffer(k, a.size) for k, a in enumerate(alone)]
    server2 = pytroy.MatmulServer(ns.ctx, slots=3)
    ids2 = _run_poisson(ns, server2, rate=5000.0, seed=4, outs=outs)
    for k, rid in enumerate(ids2):
        o, _, _, ok = server2.take(rid)
        assert ok and np.asarray(o).size == 0
        assert np.array_equal(outs[k], alone[k]), k
    for k, rid in enumerate(ids):
        o, arrival, done, ok = server.result(rid)
        assert ok and done >= arrival
        assert np.array_equal(np.asarray(o), alone[k]), k
        inp, out, x, w, h, cts, words = ns.reqs[k]
        # word-identical to the helper's products, and decrypts to x @ W mod t
        ref = h.matmul(ns.ev, cts, h.encode_weights(ns.enc, w))
        assert np.array_equal(np.concatenate([np.asarray(c.data(), np.uint64) for c in ref[0]]), alone[k])
        per = 2 * L * N
        outs = []
        for j in range(alone[k].size // per):
            c = pytroy.Ciphertext()
            c.load(_ct_bytes(ns.ctx, alone[k][j * per:(j + 1) * per]), ns.ctx)
            outs.append(c)
        assert np.array_equal(h.decrypt_outputs(ns.enc, ns.dec, pytroy.Cipher2d([outs])), _expected(x, w, ns.t, inp, out)), k


def test_admission_by_memory_footprint(serving):
    ns = serving
    inp, out = 512, 128
    h = pytroy.MatmulHelper(1, inp, out, N)
    rng = np.random.default_rng(41)
    reqs = []
    for _ in range(3):
        x = rng.integers(0, ns.t, inp, dtype=np.uint64)
        w = rng.integers(0, ns.t, inp * out, dtype=np.uint64)
        cts = h.encrypt_inputs(ns.encryptor, ns.enc, x)
        reqs.append((x, w, cts, np.concatenate([np.asarray(c.data(), np.uint64) for c in cts[0]])))
    L = len(BITS) - 1
    ni, no = (inp + h.input_block - 1) // h.input_block, (out + h.output_block - 1) // h.output_block
    size = 8 * (ni * 2 * L * N + inp * out + ni * no * N + ni * no * L * N + no * 2 * L * N) + (64 << 10)
    budget = int(size * 1.5)  # one request fits, two do not
    server = pytroy.MatmulServer(ns.ctx, memory_budget=budget, slots=3)
    ids = [server.submit(inp, out, words, w, pytroy.MatmulServer.now()) for x, w, cts, words in reqs]
    assert server.drain(60.0)
    st = server.stats()
    assert st["peak_bytes"] <= budget and st["max_wave"] == 1 and st["completed"] == len(reqs)
    for rid, (x, w, cts, words) in zip(ids, reqs):
        o, _, _, ok = server.result(rid)
        ref = h.matmul(ns.ev, cts, h.encode_weights(ns.enc, w))
        assert ok and np.array_equal(np.asarray(o), np.concatenate([np.asarray(c.data(), np.uint64) for c in ref[0]]))
    with pytest.raises(ValueError):
        pytroy.MatmulServer(ns.ctx, memory_budget=1 << 20).submit(inp, out, reqs[0][3], reqs[0][1], 0.0)


def test_failed_wave_is_reported_and_the_server_keeps_serving(serving):
    ns = serving
    server = pytroy.MatmulServer(ns.ctx, slots=1)
    server.inject_wave_failure()
    bad = [server.submit(r[0], r[1], r[6], r[3], pytroy.MatmulServer.now()) for r in ns.reqs[:2]]
    assert server.drain(60.0)
    for rid in bad:
        o, _, _, ok = server.result(rid)
        assert not ok and np.asarray(o).size == 0
    inp, out, x, w, h, cts, words = ns.reqs[2]
    rid = server.submit(inp, out, words, w, pytroy.MatmulServer.now())
    assert server.drain(60.0)
    o, _, _, ok = server.result(rid)
    assert ok
    st = server.stats()
    assert st["failed"] == 2 and st["completed"] == 1

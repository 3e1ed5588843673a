"""The benchmark's timed step, run exactly as the benchmark runs it, checked word for
word against the reference.

Workload: CKKS, N = 16384, chain {60, 40 x 7, 60}, scale 2^40, 64 ciphertext pairs
through multiply -> relinearize -> rescale_to_next -> rotate_vector over 13 Galois
keys (k = 1, 2, 4, ..., 4096), as two concurrent sub-batches on two streams with the
pairs of each step grouped into one tb_apply_galois_groups call per sub-batch
(seal-cuda_b200/python/ckks_step.py, the class bench.py times).

Inputs are real seeded encryptions made by the reference's own CPU path (compiled
under oracle/_ref); the relinearization and Galois keys come from this library's
device key generator and are first checked equal to the reference's. Every one of
the 64 outputs must equal the reference's multiply -> relinearize -> rescaleToNext ->
rotateVector words (src/evaluator.cpp:626, 1113, 2153-2251), and every pair must
decode within 2^-20 of the reference's decode and within 2^-14 of the FP64 product.
The same step as one batch on one stream (the benchmark's per-kernel timing pass) is
checked on one pair per rotation step."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from ckks_step import BatchedCkksStep  # noqa: E402
from oracle import Oracle, RefSession, available  # noqa: E402

SEED = np.arange(101, 109, dtype=np.uint64)
SEEDP = (ctypes.c_uint64 * 8)(*[int(x) for x in SEED])
N = 16384
BITS = [60] + [40] * 7 + [60]
PAIRS = 64
SUB = 2   # bench.py's HEADLINE_SUB_BATCHES
STEPS_K = [1 << i for i in range(13)]
SCALE = 2.0 ** 40


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.uint64)).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def _empty(*shape):
    return torch.empty(shape, dtype=torch.int64, device="cuda")


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_benchmark_step_matches_reference_words_and_decodes():
    orc = Oracle("orc")
    moduli = orc.coeff_modulus_create(N, BITS)
    K, L = len(moduli), len(moduli) - 1
    logn = N.bit_length() - 1
    R = RefSession(2, N, moduli, 0, SEED)
    free = R.lib.ref_ct_free
    free.argtypes = [ctypes.c_void_p, ctypes.c_int]

    # keys from the device generator, equal to the reference's
    ctx = tb_capi.Context(tb_capi.SCHEME_CKKS, N, moduli)
    sk = _empty(K, N)
    ctx("keygen_secret", SEEDP, sk, None)
    rlk = _empty(K - 1, 2, K, N)
    ctx("keygen_relin", SEEDP, sk, rlk, None)
    assert np.array_equal(_host(rlk), R.relin_key())
    elts = [orc.galois_elt_from_step(logn, k) for k in STEPS_K]
    gks = []
    for e in elts:
        g = _empty(K - 1, 2, K, N)
        ctx("keygen_galois", SEEDP, sk, e, g, None)
        assert np.array_equal(_host(g), R.galois_key(e)), e
        gks.append(g)

    # 64 pairs of real encryptions by the reference
    rng = np.random.default_rng(2025)
    v = rng.uniform(-1, 1, (PAIRS, N // 2)) + 1j * rng.uniform(-1, 1, (PAIRS, N // 2))
    w = rng.uniform(-1, 1, (PAIRS, N // 2)) + 1j * rng.uniform(-1, 1, (PAIRS, N // 2))
    ia, ib = [], []
    A = np.empty((PAIRS, 2, L, N), np.uint64)
    B = np.empty_like(A)
    for i in range(PAIRS):
        ia.append(R.encrypt_ckks(v[i], SCALE))
        ib.append(R.encrypt_ckks(w[i], SCALE))
        A[i] = R.ct(ia[-1])["data"].reshape(2, L, N)
        B[i] = R.ct(ib[-1])["data"].reshape(2, L, N)

    # the benchmark's step: two sub-batches on two streams
    step = BatchedCkksStep(torch, ctx, L, N, PAIRS, rlk, elts, gks, SUB)
    dA, dB = _dev(A), _dev(B)
    out = _empty(PAIRS, 2, L - 1, N)
    stream = torch.cuda.current_stream()
    step(dA, dB, out, stream)
    torch.cuda.synchronize()
    got = _host(out)
    # a second step over the same inputs gives the same words (no state kept between steps)
    out2 = _empty(PAIRS, 2, L - 1, N)
    step(dA, dB, out2, stream)
    torch.cuda.synchronize()
    assert np.array_equal(_host(out2), got)

    groups = step.row_groups()
    assert sorted(set(groups)) == list(range(len(STEPS_K)))
    ref_dec = {}

    def reference(i, g):
        """The reference chain of pair i rotated by STEPS_K[g]: words and decode."""
        m = R.multiply(ia[i], ib[i])
        r = R.relinearize(m)
        rs = R.rescale(r)
        o = R.rotate_vector(rs, STEPS_K[g])
        words = R.ct(o)["data"].reshape(2, L - 1, N)
        dec = R.decrypt_ckks(o, N // 2)
        for x in (m, r, rs, o):
            free(R.h, x)
        return words, dec

    for i in range(PAIRS):
        words, dec = reference(i, groups[i])
        assert np.array_equal(got[i], words), (i, STEPS_K[groups[i]])
        ref_dec[i] = dec

    # decode every output on the device: within 2^-20 of the reference's decode and
    # 2^-14 of the FP64 product rotated by the pair's step
    ph = _empty(PAIRS, L - 1, N)
    ctx("decrypt", sk, L - 1, 2, out, 0, ph, 0, 1, PAIRS, None)
    vals = torch.empty((PAIRS, N // 2, 2), dtype=torch.float64, device="cuda")
    ctx("ckks_decode", L - 1, ph, SCALE * SCALE / moduli[L - 1], vals, 0, PAIRS, None)
    dec = vals.cpu().numpy()
    dec = dec[..., 0] + 1j * dec[..., 1]
    for i in range(PAIRS):
        k = STEPS_K[groups[i]]
        assert np.abs(dec[i] - ref_dec[i]).max() <= 2.0 ** -20, i
        assert np.abs(dec[i] - np.roll(v[i] * w[i], -k)).max() <= 2.0 ** -14, i

    # the same workload as one batch on one stream (steps assigned over the whole batch)
    whole = _empty(PAIRS, 2, L - 1, N)
    step(dA, dB, whole, stream, sub=1)
    torch.cuda.synchronize()
    got1 = _host(whole)
    g1 = step.row_groups(sub=1)
    for g in range(len(STEPS_K)):
        i = g1.index(g)
        words, _ = reference(i, g)
        assert np.array_equal(got1[i], words), (i, STEPS_K[g])

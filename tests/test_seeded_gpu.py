"""Seed-compressed ciphertexts on the wire: the reference's GPU path saves a symmetric
encryption as c0 plus a 64-bit seed and regenerates c1 with cuRAND on load. Bytes made
by the reference's own CUDA build (oracle/_ref/libtroyref_gpu.so, run in a child
process) load here to the same words its loader produces, and decrypt with the same
seeded secret key to the encrypted values; without a context the load is refused as
in the reference."""
import ctypes
import multiprocessing as mp
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
pytroy = pytest.importorskip("pytroy")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_GPU = os.path.join(ROOT, "oracle", "_ref", "libtroyref_gpu.so")
SEED = [int(x) for x in range(101, 109)]


def _ref_gpu_seeded(args):
    """Child process: the reference CUDA build's seeded symmetric encryption."""
    scheme, n, moduli, t, values, reals, scale = args
    lib = ctypes.CDLL(REF_GPU)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    lib.ref_gpu_seeded_ct.argtypes = [ctypes.c_int, ctypes.c_size_t, u64p, ctypes.c_int, ctypes.c_uint64, u64p, u64p,
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_size_t, ctypes.c_double,
                                      ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t), u64p, u64p]
    L = len(moduli) - 1
    mods = (ctypes.c_uint64 * len(moduli))(*moduli)
    seed = (ctypes.c_uint64 * 8)(*SEED)
    vals = (ctypes.c_uint64 * max(1, len(values)))(*values)
    rl = (ctypes.c_double * max(1, len(reals)))(*reals)
    cap = 16 * L * n + 4096
    buf = ctypes.create_string_buffer(cap)
    ln = ctypes.c_size_t(0)
    words = (ctypes.c_uint64 * (2 * L * n))()
    sd = ctypes.c_uint64(0)
    rc = lib.ref_gpu_seeded_ct(scheme, n, mods, len(moduli), t, seed, vals, rl, max(len(values), len(reals)), scale,
                               buf, cap, ctypes.byref(ln), words, ctypes.byref(sd))
    return rc, buf.raw[:ln.value], np.frombuffer(bytes(words), np.uint64).copy(), sd.value


def _from_reference(args):
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.apply(_ref_gpu_seeded, (args,))


def _context(scheme, n, bits, t=None):
    p = pytroy.EncryptionParameters(scheme)
    p.set_poly_modulus_degree(n)
    p.set_coeff_modulus(pytroy.CoeffModulus.create(n, bits))
    if t is not None:
        p.set_plain_modulus(t)
    p.set_random_generator(pytroy.Blake2xbPRNGFactory(SEED))
    return pytroy.SEALContext(p)


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference CUDA build not present")
def test_bfv_seeded_ciphertext_from_the_reference_loads_and_decrypts():
    n, bits, t = 4096, [36, 36, 37], 65537
    ctx = _context(pytroy.SchemeType.bfv, n, bits, t)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(n, bits)]
    values = np.random.default_rng(5).integers(0, t, n, dtype=np.uint64)
    rc, blob, words, seed = _from_reference((1, n, moduli, t, [int(v) for v in values], [], 1.0))
    assert rc in (0, 2) and seed != 0
    L = len(bits) - 1
    assert len(blob) < 16 * L * n   # only c0 travels
    ct = pytroy.Ciphertext()
    ct.load(blob, ctx)
    assert ct.size() == 2 and np.array_equal(np.asarray(ct.data(), np.uint64), words)
    keygen = pytroy.KeyGenerator(ctx)
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    assert np.array_equal(pytroy.BatchEncoder(ctx).decode(dec.decrypt(ct)), values)
    with pytest.raises(ValueError):
        pytroy.Ciphertext().load(blob)            # the reference also needs the context
    back = pytroy.Ciphertext()
    back.load(ct.save(), ctx)                     # saved here in full (seed 0)
    assert np.array_equal(np.asarray(back.data(), np.uint64), words)


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference CUDA build not present")
def test_ckks_seeded_ciphertext_from_the_reference_loads_and_decrypts():
    n, bits, scale = 8192, [60, 40, 60], 2.0 ** 40
    ctx = _context(pytroy.SchemeType.ckks, n, bits)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(n, bits)]
    reals = np.random.default_rng(6).uniform(-1, 1, n // 2)
    rc, blob, words, seed = _from_reference((2, n, moduli, 0, [], [float(x) for x in reals], scale))
    assert rc in (0, 2) and seed != 0
    ct = pytroy.Ciphertext()
    ct.load(blob, ctx)
    assert ct.is_ntt_form() and np.array_equal(np.asarray(ct.data(), np.uint64), words)
    keygen = pytroy.KeyGenerator(ctx)
    got = pytroy.CKKSEncoder(ctx).decode(pytroy.Decryptor(ctx, keygen.secret_key()).decrypt(ct))
    assert np.abs(got - reals).max() < 1e-5


def _ref_gpu_load(args):
    """Child process: the reference CUDA build loads bytes made here with its own loader,
    decrypts them with the secret key of the same seeded factory and decodes."""
    scheme, n, moduli, t, blob, nvalues = args
    lib = ctypes.CDLL(REF_GPU)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    lib.ref_gpu_load_decrypt.argtypes = [ctypes.c_int, ctypes.c_size_t, u64p, ctypes.c_int, ctypes.c_uint64, u64p,
                                         ctypes.c_char_p, ctypes.c_size_t, u64p, ctypes.POINTER(ctypes.c_double),
                                         ctypes.c_size_t, u64p]
    L = len(moduli) - 1
    mods = (ctypes.c_uint64 * len(moduli))(*moduli)
    seed = (ctypes.c_uint64 * 8)(*SEED)
    vals = (ctypes.c_uint64 * nvalues)()
    reals = (ctypes.c_double * nvalues)()
    words = (ctypes.c_uint64 * (2 * L * n))()
    rc = lib.ref_gpu_load_decrypt(scheme, n, mods, len(moduli), t, seed, blob, len(blob), vals, reals, nvalues, words)
    return (rc, np.frombuffer(bytes(vals), np.uint64).copy(), np.frombuffer(bytes(reals), np.float64).copy(),
            np.frombuffer(bytes(words), np.uint64).copy())


def _in_reference(args):
    with mp.get_context("spawn").Pool(1) as pool:
        return pool.apply(_ref_gpu_load, (args,))


@pytest.mark.skipif(not os.path.exists(REF_GPU), reason="reference CUDA build not present")
@pytest.mark.parametrize("scheme", ["bfv", "ckks"])
def test_seeded_ciphertext_written_here_loads_and_decrypts_in_the_reference(scheme):
    """encrypt_symmetric_seeded writes c0 plus a seed; the reference's own loader
    regenerates the same second polynomial from the seed and its decryptor recovers the
    values. The bytes also load back here to the same words."""
    if scheme == "bfv":
        n, bits, t = 4096, [36, 36, 37], 65537
        st = pytroy.SchemeType.bfv
    else:
        n, bits, t = 8192, [60, 40, 60], 0
        st = pytroy.SchemeType.ckks
    ctx = _context(st, n, bits, t if t else None)
    moduli = [m.value() for m in pytroy.CoeffModulus.create(n, bits)]
    L = len(bits) - 1
    keygen = pytroy.KeyGenerator(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.secret_key())
    rng = np.random.default_rng(71)
    if scheme == "bfv":
        values = rng.integers(0, t, n, dtype=np.uint64)
        plain = pytroy.BatchEncoder(ctx).encode(values)
        count = n
    else:
        reals = rng.uniform(-1, 1, n // 2)
        plain = pytroy.CKKSEncoder(ctx).encode(reals, 2.0 ** 40)
        count = n // 2
    ct = encryptor.encrypt_symmetric_seeded(plain)
    assert ct.seed() != 0
    words = np.asarray(ct.data(), np.uint64)
    blob = ct.save()
    assert len(blob) < 8 * L * n + 1024             # c0 and the seed only
    rc, vals, got_reals, ref_words = _in_reference((1 if scheme == "bfv" else 2, n, moduli, t, blob, count))
    assert rc in (0, 2)                              # 2: a pending CUDA error of the reference, results kept
    assert np.array_equal(ref_words, words)          # the reference regenerated the same c1
    dec = pytroy.Decryptor(ctx, keygen.secret_key())
    back = pytroy.Ciphertext()
    back.load(blob, ctx)
    assert back.seed() == 0 and np.array_equal(np.asarray(back.data(), np.uint64), words)
    if scheme == "bfv":
        assert np.array_equal(vals, values)
        assert np.array_equal(pytroy.BatchEncoder(ctx).decode(dec.decrypt(back)), values)
    else:
        assert np.abs(got_reals - reals).max() < 1e-5
        assert np.abs(pytroy.CKKSEncoder(ctx).decode(dec.decrypt(back)) - reals).max() < 1e-5
    # an evaluation clears the seed: the result travels in full
    ev = pytroy.Evaluator(ctx)
    ev.add_inplace(ct, ct)
    assert ct.seed() == 0 and len(ct.save()) > 16 * L * n


def test_seeded_bgv_encryption_is_refused():
    n, bits = 4096, [36, 36, 37]
    t = pytroy.PlainModulus.batching(n, 20)
    ctx = _context(pytroy.SchemeType.bgv, n, bits, t)
    keygen = pytroy.KeyGenerator(ctx)
    encryptor = pytroy.Encryptor(ctx, keygen.secret_key())
    plain = pytroy.BatchEncoder(ctx).encode(np.zeros(n, np.uint64))
    with pytest.raises(Exception, match="NTT domain"):
        encryptor.encrypt_symmetric_seeded(plain)


@pytest.mark.parametrize("scheme,inverse", [(2, 0), (1, 1)])
def test_batched_seed_expansion_equals_one_per_call(orc, scheme, inverse):
    """tb_expand_seeded_batch writes, for every ciphertext of a batch, the second
    polynomial tb_expand_seeded (the reference loader's cuRAND expansion) gives it."""
    import tb_capi
    n = 4096
    moduli = orc.coeff_modulus_create(n, [36, 36, 37])
    ctx = tb_capi.Context(scheme, n, moduli, 65537 if scheme == 1 else 0)
    L, B = 2, 5
    seeds = [0x1234567890abcdef + 977 * b for b in range(B)]
    dseeds = torch.tensor(np.array(seeds, np.uint64).view(np.int64), device="cuda")
    cts = torch.zeros((B, 2, L, n), dtype=torch.int64, device="cuda")
    ctx("expand_seeded_batch", L, dseeds, B, inverse, cts[:, 1], 2 * L * n, None)
    one = torch.zeros((L, n), dtype=torch.int64, device="cuda")
    for b in range(B):
        ctx("expand_seeded", L, seeds[b], inverse, one, None)
        torch.cuda.synchronize()
        assert torch.equal(cts[b, 1], one), b
        assert not cts[b, 0].any()

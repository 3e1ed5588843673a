"""Uneven batches (ring degree 4096 / 8192 / 16384, chains of 3 / 5 / 9 primes, BFV and
BGV, one 20-bit batching plain modulus) through multiply, relinearize and rotate_rows(1):
the captured CUDA graph (one launch for the whole batch), the stream-overlapped run and
the one-ciphertext-per-call path give identical words, and sample ciphertexts equal the
reference CPU path's."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from oracle import Oracle, RefSession, available  # noqa: E402
from uneven import ShapeGroup, UnevenBatch  # noqa: E402

SEED = np.arange(101, 109, dtype=np.uint64)
SHAPES = [(1, 4096, [36, 36, 37]), (3, 8192, [43, 43, 44, 44, 44]), (1, 16384, [48] * 9)]


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(np.asarray(a, np.uint64)).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


@pytest.mark.skipif(not available("ref"), reason="reference library not built")
def test_uneven_batch_graph_streams_per_op_and_reference_agree():
    orc = Oracle("orc")
    t = orc.plain_modulus_batching(16384, 20)
    rng = np.random.default_rng(404)
    # the benchmark's 512 ciphertexts with degrees drawn uniformly; the first two of each
    # group are real encryptions made by the reference, the rest uniform residues
    draws = rng.integers(0, len(SHAPES), 512)
    groups, checks = [], []
    for gi, (scheme, n, bits) in enumerate(SHAPES):
        moduli = orc.coeff_modulus_create(n, bits)
        K, L = len(moduli), len(moduli) - 1
        ref = RefSession(scheme, n, moduli, t, SEED)
        elt = orc.galois_elt_from_step(n.bit_length() - 1, 1)
        rlk, gk = ref.relin_key(), ref.galois_key(elt)
        count = max(2, int((draws == gi).sum()))
        A = np.stack([np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli[:L]])
                                for _ in range(2)]) for _ in range(count)])
        Bm = np.stack([np.stack([np.stack([rng.integers(0, q, n, dtype=np.uint64) for q in moduli[:L]])
                                 for _ in range(2)]) for _ in range(count)])
        ids = []
        for i in range(2):
            ia = ref.encrypt_slots(rng.integers(0, t, n, dtype=np.uint64))
            ib = ref.encrypt_slots(rng.integers(0, t, n, dtype=np.uint64))
            A[i], Bm[i] = ref.ct(ia)["data"].reshape(2, L, n), ref.ct(ib)["data"].reshape(2, L, n)
            ids.append(ref.rotate_rows(ref.relinearize(ref.multiply(ia, ib)), 1))
        ctx = tb_capi.Context(scheme, n, moduli, t)
        groups.append(ShapeGroup(ctx, L, _dev(A), _dev(Bm), _dev(rlk), _dev(gk), elt))
        checks.append((ref, ids))
    batch = UnevenBatch(groups)
    batch.run()
    torch.cuda.synchronize()
    streams = [g.out.clone() for g in groups]
    for g in groups:
        g.out.zero_()
    # every group's key switches in one persistent launch per step
    batch.set_shapes(True)
    batch.run()
    torch.cuda.synchronize()
    for gi, g in enumerate(groups):
        assert torch.equal(g.out, streams[gi]), gi
        g.out.zero_()
    batch.set_shapes(False)
    batch.run_per_op()
    torch.cuda.synchronize()
    per_op = [g.out.clone() for g in groups]
    for g in groups:
        g.out.zero_()
    batch.set_shapes(True)
    batch.capture()
    batch.replay()
    batch.replay()  # twice: replays are repeatable
    torch.cuda.synchronize()
    for gi, g in enumerate(groups):
        got = _host(g.out)
        assert np.array_equal(got, _host(streams[gi])), gi
        assert np.array_equal(got, _host(per_op[gi])), gi
        ref, ids = checks[gi]
        for i, rid in enumerate(ids):
            assert np.array_equal(got[i], ref.ct(rid)["data"].reshape(got[i].shape)), (gi, i)

"""tb_relinearize_noalloc — relinearization for callers that cannot allocate device
memory at call time (a serving loop that reserved all of HBM up front, code running
while another allocator owns the free memory) — gives the same words as
tb_relinearize and as the oracle's key switch, on two calls in a row (the second
reuses the static scratch the first one left behind), for CKKS, BFV and BGV.

This file is named to be collected last."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

import tb_capi  # noqa: E402
from oracle import Oracle  # noqa: E402


def _rand(rng, moduli, n, lead):
    out = np.empty(tuple(lead) + (len(moduli), n), np.uint64)
    for i, q in enumerate(moduli):
        out[..., i, :] = rng.integers(0, q, tuple(lead) + (n,), dtype=np.uint64)
    return out


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int64)).cuda()


@pytest.mark.parametrize("scheme,n,bits,t,batch", [
    (tb_capi.SCHEME_CKKS, 16384, [60] + [40] * 7 + [60], 0, 3),   # one ciphertext per scratch chunk
    (tb_capi.SCHEME_BFV, 4096, [36, 36, 37], 65537, 5),            # whole batch in one chunk
    (tb_capi.SCHEME_BGV, 4096, [40, 40, 41, 41], 65537, 4),        # BGV's own mod-down
])
def test_noalloc_matches_relinearize_twice(scheme, n, bits, t, batch):
    orc = Oracle("orc")
    moduli = orc.coeff_modulus_create(n, bits)
    ctx = tb_capi.Context(scheme, n, moduli, t)
    K = len(moduli)
    L = K - 1
    logn = n.bit_length() - 1
    rng = np.random.default_rng(n + batch)
    hkey = _rand(rng, moduli, n, (K - 1, 2))
    key = _dev(hkey)
    for call in range(2):
        ct3 = _rand(rng, moduli[:L], n, (batch, 3))
        ref = _dev(ct3)
        got = _dev(ct3)
        ctx("relinearize", L, ref, 0, key, batch, None)
        ctx("relinearize_noalloc", L, got, 0, key, batch, None)
        torch.cuda.synchronize()
        assert torch.equal(got, ref), f"call {call}"
        # and word for word against the oracle's key switch of c2 into (c0, c1)
        words = got.cpu().numpy().view(np.uint64)
        for b in (0, batch - 1):
            exp = orc.keyswitch(scheme, logn, moduli, t, ct3[b, 2], ct3[b, :2], hkey)
            assert np.array_equal(words[b, :2], exp), f"call {call}, ciphertext {b}"


def test_noalloc_rejects_levels_beyond_its_scratch():
    orc = Oracle("orc")
    n = 16384
    moduli = orc.coeff_modulus_create(n, [60] + [40] * 9 + [60])   # L = 10 needs > 16 MiB per ciphertext
    ctx = tb_capi.Context(tb_capi.SCHEME_CKKS, n, moduli)
    K = len(moduli)
    ct = torch.zeros((1, 3, K - 1, n), dtype=torch.int64, device="cuda")
    key = torch.zeros((K - 1, 2, K, n), dtype=torch.int64, device="cuda")
    with pytest.raises(tb_capi.TroyError) as e:
        ctx("relinearize_noalloc", K - 1, ct, 0, key, 1, None)
    assert e.value.status == 1 and "static scratch" in str(e.value)


_CHILD = r"""
import sys
import numpy as np
import torch
import tb_capi
from oracle import Oracle
orc = Oracle("orc")
n, batch = 4096, 3
moduli = orc.coeff_modulus_create(n, [60, 40, 40, 60])
ctx = tb_capi.Context(tb_capi.SCHEME_CKKS, n, moduli)
K = len(moduli)
L = K - 1
rng = np.random.default_rng(4096)
def rand(mods, lead):
    out = np.empty(tuple(lead) + (len(mods), n), np.uint64)
    for i, q in enumerate(mods):
        out[..., i, :] = rng.integers(0, q, tuple(lead) + (n,), dtype=np.uint64)
    return torch.from_numpy(out.view(np.int64)).cuda()
key = rand(moduli, (K - 1, 2))
src = rand(moduli[:L], (batch, 3))
got = torch.empty_like(src)
graph = torch.cuda.CUDAGraph()
side = torch.cuda.Stream()
side.wait_stream(torch.cuda.current_stream())
torch.cuda.synchronize()
with torch.cuda.graph(graph, stream=side):   # the process's first library call
    got.copy_(src)
    ctx("relinearize_noalloc", L, got, 0, key, batch, side)
graph.replay()
ref = src.clone()
ctx("relinearize", L, ref, 0, key, batch, None)
torch.cuda.synchronize()
assert torch.equal(got[:, :2], ref[:, :2])
print("CAPTURED-OK")
"""


def test_noalloc_first_call_inside_a_graph_capture():
    """The static scratch's device address is taken when the context is created, so in a
    fresh process the first relinearize_noalloc call loads and allocates nothing: it can
    be the process's first library call, inside a CUDA graph capture (a call that loaded
    the module or allocated would break the capture). The replayed graph gives the words
    of tb_relinearize. Runs in a child process so that no earlier test has loaded the
    module."""
    import os
    import subprocess
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    env = dict(os.environ)
    env["PYTHONPATH"] = os.pathsep.join([os.path.join(root, "seal-cuda_b200", "python"), os.path.join(root, "oracle"),
                                         os.path.join(root, "seal-cuda_b200", "lib"), env.get("PYTHONPATH", "")])
    r = subprocess.run([sys.executable, "-c", _CHILD], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "CAPTURED-OK" in r.stdout, r.stdout[-2000:] + r.stderr[-2000:]

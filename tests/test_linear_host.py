"""Linear-layer coefficient layouts (no GPU).

The numpy restatement of the reference's MatmulHelper / Conv2dHelper encodings
(oracle/linear_layout.py) is pinned against the operations themselves: multiplying the
encoded polynomials negacyclically mod (X^N + 1, t), summing over input blocks and
reading the reference's output coefficients gives x W and the valid 2-d
cross-correlation, for unblocked and blocked (image larger than sqrt(slots)) shapes.
The module's host-only parts (block plans, blocked batch counts, shape errors) agree
with the restatement."""
import numpy as np
import pytest

from linear_layout import Conv2dLayout, DiagonalLayout, MatmulLayout, negacyclic_mul

T = 65537


@pytest.mark.parametrize("batch,ih,iw,kh,kw,ic,oc,slots", [
    (2, 5, 6, 3, 2, 3, 2, 64),      # unblocked, several channels per polynomial
    (1, 7, 7, 3, 3, 5, 2, 64),      # unblocked, channel groups
    (1, 10, 11, 3, 3, 2, 2, 64),    # blocked: 8 x 8 blocks overlapping by the kernel
    (2, 20, 9, 2, 4, 1, 3, 256),    # blocked along one axis
])
def test_conv2d_layout_computes_the_convolution(batch, ih, iw, kh, kw, ic, oc, slots):
    lay = Conv2dLayout(batch, ih, iw, kh, kw, ic, oc, slots)
    rng = np.random.default_rng(batch * 1000 + ih * 10 + ic)
    x = rng.integers(0, T, batch * ic * ih * iw, dtype=np.uint64)
    w = rng.integers(0, T, oc * ic * kh * kw, dtype=np.uint64)
    xin, win = lay.inputs(x), lay.weights(w)
    assert len(xin) == lay.total and all(len(r) == len(win[0]) for r in xin)
    got = np.zeros((batch, oc, ih - kh + 1, iw - kw + 1), np.uint64)
    seen = np.zeros(got.shape, bool)
    for b in range(lay.total):
        for o in range(oc):
            acc = np.zeros(slots, np.uint64)
            for g in range(len(xin[b])):
                acc = (acc + negacyclic_mul(xin[b][g], win[o][g], slots, T)) % T
            for img, i, j, mi in lay.output_positions(b):
                got[img, o, i, j] = acc[mi]
                seen[img, o, i, j] = True
    assert seen.all()
    assert np.array_equal(got, lay.expected(x, w, T))


@pytest.mark.parametrize("batch,inp,out,slots", [(1, 40, 7, 64), (3, 10, 6, 64), (2, 100, 3, 128)])
def test_matmul_layout_computes_the_product(batch, inp, out, slots):
    lay = MatmulLayout(batch, inp, out, slots)
    rng = np.random.default_rng(inp + out)
    x = rng.integers(0, T, batch * inp, dtype=np.uint64)
    w = rng.integers(0, T, inp * out, dtype=np.uint64)
    xin, win = lay.inputs(x), lay.weights(w)
    got = np.zeros((batch, out), np.uint64)
    for bi, li in enumerate(range(0, batch, lay.bb)):
        for bj, lj in enumerate(range(0, out, lay.ob)):
            acc = np.zeros(slots, np.uint64)
            for k in range(len(win)):
                acc = (acc + negacyclic_mul(xin[bi][k], win[k][bj], slots, T)) % T
            for i, j, c in lay.output_positions(li, lj):
                got[i, j] = acc[c]
    want = (x.reshape(batch, inp).astype(object) @ w.reshape(inp, out).astype(object) % T).astype(np.uint64)
    assert np.array_equal(got, want)


def test_conv2d_helper_host_parts():
    pytroy = pytest.importorskip("pytroy")
    for shape in [(1, 30, 30, 3, 3, 12, 2, 8192), (1, 100, 100, 3, 3, 2, 2, 8192), (3, 200, 95, 5, 4, 1, 1, 8192)]:
        h = pytroy.Conv2dHelper(*shape)
        assert h.total_batch_size() == Conv2dLayout(*shape).total
    with pytest.raises(ValueError):
        pytroy.Conv2dHelper(1, 8, 8, 9, 3, 1, 1, 8192)   # kernel taller than the image
    with pytest.raises(ValueError):
        pytroy.Conv2dHelper(0, 8, 8, 3, 3, 1, 1, 8192)
    assert len(pytroy.Cipher2d()) == 0 and len(pytroy.Plain2d()) == 0


@pytest.mark.parametrize("height,width,slots", [(20, 30, 256), (500, 30, 4096), (60, 7, 64), (64, 64, 64)])
def test_diagonal_layout_computes_the_matrix_vector_product(height, width, slots):
    lay = DiagonalLayout(height, width, slots)
    rng = np.random.default_rng(height * width)
    m = rng.uniform(-1, 1, (height, width)) + 1j * rng.uniform(-1, 1, (height, width))
    v = rng.uniform(-1, 1, width) + 1j * rng.uniform(-1, 1, width)
    assert np.allclose(lay.apply(m, v), m @ v, atol=1e-12)
    pytroy = pytest.importorskip("pytroy")
    h = pytroy.DiagonalMatmulHelper(height, width, slots)
    assert (h.pack_num, h.cipher_count) == (lay.pack, lay.count)


def test_diagonal_helper_rejects_shapes_the_packing_cannot_hold():
    """More diagonals than next_pow2(width) slots (here 16 > 8) lose rows in the packing
    (the repacked diagonal index never reaches them), so such shapes are refused."""
    pytroy = pytest.importorskip("pytroy")
    lay = DiagonalLayout(100, 7, 64)
    assert lay.count > lay.p2
    with pytest.raises(ValueError):
        pytroy.DiagonalMatmulHelper(100, 7, 64)
    with pytest.raises(ValueError):
        pytroy.DiagonalMatmulHelper(4, 100, 64)   # width beyond the slots

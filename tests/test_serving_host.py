"""Block planning of the matrix helper (no GPU): MatmulHelper picks the reference's
block shape (MatmulHelper::determineBlock, app/LinearHelper.cuh:206-228), restated
here as a plain loop."""
import pytest

pytroy = pytest.importorskip("pytroy")


def _plan(batch, inp, out, slots):
    cdiv = lambda a, b: (a + b - 1) // b
    best, res = 2147483647, None
    for b in range(batch, 0, -1):
        bc = cdiv(batch, b)
        if b >= slots or bc * 2 > best:
            continue
        for i in range(1, slots // b):
            o = min(slots // b // i, out)
            if i > inp or o < 1:
                continue
            c = bc * (cdiv(inp, i) + cdiv(out, o))
            if c >= best:
                continue
            best, res = c, (b, i, o)
    return res


@pytest.mark.parametrize("batch,inp,out", [(1, 1024, 256), (1, 64, 16), (1, 320, 48), (1, 1000, 250),
                                           (4, 128, 32), (16, 784, 10), (3, 5, 7)])
def test_block_plan_matches_the_reference_rule(batch, inp, out):
    h = pytroy.MatmulHelper(batch, inp, out, 8192)
    assert (h.batch_block, h.input_block, h.output_block) == _plan(batch, inp, out, 8192)


def test_block_plan_rejects_empty_shapes():
    with pytest.raises(ValueError):
        pytroy.MatmulHelper(1, 0, 16, 8192)

"""Test infrastructure, not part of the library: a numpy restatement of the reference's
linear-layer encodings (app/LinearHelper.cuh) used to check MatmulHelper and
Conv2dHelper. Each function returns the coefficient vectors that the reference feeds
to BatchEncoder::encodePolynomial, so the reference's own CPU evaluator
(oracle.RefSession) can encrypt and multiply the same polynomials, and
`negacyclic_mul` lets the layouts be checked against a direct product on the CPU."""
import math

import numpy as np


def cdiv(a, b):
    return (a + b - 1) // b


def matmul_plan(batch, inp, out, slots):
    """MatmulHelper::determineBlock (app/LinearHelper.cuh:206-228)."""
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


class MatmulLayout:
    """Coefficient layouts of MatmulHelper (app/LinearHelper.cuh:230-420)."""

    def __init__(self, batch, inp, out, slots):
        self.batch, self.inp, self.out, self.slots = batch, inp, out, slots
        self.bb, self.ib, self.ob = matmul_plan(batch, inp, out, slots)

    def inputs(self, x):
        """encodeInputs (app/LinearHelper.cuh:279-311): rows [batch block][input block]."""
        x = np.asarray(x, np.uint64).reshape(self.batch, self.inp)
        rows = []
        for li in range(0, self.batch, self.bb):
            row = []
            for lj in range(0, self.inp, self.ib):
                v = np.zeros(self.slots, np.uint64)
                for i in range(li, min(li + self.bb, self.batch)):
                    seg = x[i, lj:lj + self.ib]
                    base = (i - li) * self.ib * self.ob
                    v[base:base + seg.size] = seg
                row.append(v)
            rows.append(row)
        return rows

    def weights(self, w):
        """encodeWeights / encodeWeightSmall (app/LinearHelper.cuh:230-277): rows
        [input block][output block], each block's columns reversed within the block."""
        W = np.asarray(w, np.uint64).reshape(self.inp, self.out)
        rows = []
        for li in range(0, self.inp, self.ib):
            row = []
            for lj in range(0, self.out, self.ob):
                v = np.zeros(self.ib * self.ob, np.uint64)
                for j in range(lj, min(lj + self.ob, self.out)):
                    for i in range(li, min(li + self.ib, self.inp)):
                        v[(j - lj) * self.ib + self.ib - (i - li) - 1] = W[i, j]
                row.append(v)
            rows.append(row)
        return rows

    def output_positions(self, li, lj):
        """(row, column, coefficient) of each output held by block (li, lj)
        (decryptOutputs, app/LinearHelper.cuh:422-451)."""
        out = []
        for i in range(li, min(li + self.bb, self.batch)):
            for j in range(lj, min(lj + self.ob, self.out)):
                out.append((i, j, (i - li) * self.ib * self.ob + (j - lj) * self.ib + self.ib - 1))
        return out


class Conv2dLayout:
    """Coefficient layouts of Conv2dHelper (app/LinearHelper.cuh:531-930): batch x ic x
    ih x iw images, oc x ic x kh x kw kernels, "valid" cross-correlation outputs."""

    def __init__(self, batch, ih, iw, kh, kw, ic, oc, slots):
        self.batch, self.ih, self.iw, self.kh, self.kw, self.ic, self.oc, self.slots = \
            batch, ih, iw, kh, kw, ic, oc, slots
        m = int(np.sqrt(slots))
        self.blocked = ih > m or iw > m
        self.bh, self.bw = (m, m) if self.blocked else (ih, iw)
        self.block = self.bh * self.bw
        self.cs = slots // self.block                     # channels per polynomial
        self.sh = cdiv(ih - (kh - 1), self.bh - (kh - 1))
        self.sw = cdiv(iw - (kw - 1), self.bw - (kw - 1))
        self.total = batch * self.sh * self.sw if self.blocked else batch

    def inputs(self, x):
        """encodeInputs (app/LinearHelper.cuh:674-742): rows [block][channel group]."""
        x = np.asarray(x, np.uint64).reshape(self.batch, self.ic, self.ih, self.iw)
        blocks = []
        for b in range(self.batch):
            for i in range(self.sh):
                for j in range(self.sw):
                    si, sj = i * (self.bh - self.kh + 1), j * (self.bw - self.kw + 1)
                    t = np.zeros((self.ic, self.bh, self.bw), np.uint64)
                    part = x[b, :, si:si + self.bh, sj:sj + self.bw]
                    t[:, :part.shape[1], :part.shape[2]] = part
                    blocks.append(t)
        rows = []
        for t in blocks:
            row = []
            for c in range(0, self.ic, self.cs):
                v = np.zeros(self.slots, np.uint64)
                for k in range(min(self.cs, self.ic - c)):
                    v[k * self.block:(k + 1) * self.block] = t[c + k].reshape(-1)
                row.append(v)
            rows.append(row)
        return rows

    def weights(self, w):
        """encodeWeights (app/LinearHelper.cuh:626-661): rows [output channel][channel
        group], each kernel flipped and placed in reversed channel order."""
        w = np.asarray(w, np.uint64).reshape(self.oc, self.ic, self.kh, self.kw)
        rows = []
        for o in range(self.oc):
            row = []
            for lic in range(0, self.ic, self.cs):
                v = np.zeros(self.cs * self.block, np.uint64)
                for j in range(lic, min(lic + self.cs, self.ic)):
                    base = (self.cs - 1 - (j - lic)) * self.block
                    for ki in range(self.kh):
                        v[base + ki * self.bw:base + ki * self.bw + self.kw] = w[o, j, self.kh - 1 - ki, ::-1]
                row.append(v)
            rows.append(row)
        return rows

    def output_positions(self, b):
        """(image, output row, output column, coefficient) of each output read from
        block b (decryptOutputs, app/LinearHelper.cuh:886-930)."""
        yh, yw = self.bh - self.kh + 1, self.bw - self.kw + 1
        oyh, oyw = self.ih - self.kh + 1, self.iw - self.kw + 1
        ob, si, sj = b // (self.sh * self.sw), (b % (self.sh * self.sw)) // self.sw, b % self.sw
        out = []
        for i in range(yh):
            for j in range(yw):
                if si * yh + i < oyh and sj * yw + j < oyw:
                    mi = (self.cs - 1) * self.block + (self.bh - yh + i) * self.bw + (self.bw - yw + j)
                    out.append((ob, si * yh + i, sj * yw + j, mi))
        return out

    def expected(self, x, w, t):
        """The convolution itself, mod t."""
        x = np.asarray(x, np.uint64).reshape(self.batch, self.ic, self.ih, self.iw).astype(object)
        w = np.asarray(w, np.uint64).reshape(self.oc, self.ic, self.kh, self.kw).astype(object)
        oyh, oyw = self.ih - self.kh + 1, self.iw - self.kw + 1
        y = np.zeros((self.batch, self.oc, oyh, oyw), object)
        for ki in range(self.kh):
            for kj in range(self.kw):
                patch = x[:, :, ki:ki + oyh, kj:kj + oyw]
                y += np.einsum("bchw,oc->bohw", patch, w[:, :, ki, kj])
        return (y % t).astype(np.uint64)


def negacyclic_mul(a, b, n, t):
    """a(X) b(X) mod (X^n + 1, t) with exact integers (small n only)."""
    a = np.concatenate([np.asarray(a, np.uint64).astype(object), np.zeros(n - len(a), object)])
    b = np.concatenate([np.asarray(b, np.uint64).astype(object), np.zeros(n - len(b), object)])
    full = np.convolve(a, b)
    res = full[:n].copy()
    res[:len(full) - n] -= full[n:]
    return (res % t).astype(np.uint64)


def next_pow2(v):
    """nextPow2 (app/matmul.cuh:15): 2^ceil(log(v) / log(2)) in double precision."""
    return int(2.0 ** math.ceil(math.log(v) / math.log(2.0)))


class DiagonalLayout:
    """Slot layout of the diagonal CKKS matrix-vector product (app/matmul.cuh:5-123)."""

    def __init__(self, height, width, slots):
        self.height, self.width, self.slots = height, width, slots
        self.p2 = next_pow2(width)
        self.pack = slots // self.p2
        self.count = int(math.ceil(np.float32(next_pow2(height)) / np.float32(self.pack)))

    def input(self, v):
        """prepareInput (app/matmul.cuh:19-32): v repeated pack times, p2 slots apart."""
        out = np.zeros(self.slots, np.complex128)
        for idx in range(self.pack):
            out[idx * self.p2:idx * self.p2 + self.width] = v
        return out

    def diagonals(self, m):
        """encode (app/matmul.cuh:45-90): rows packed count at a time, then repacked
        into generalized diagonals."""
        m = np.asarray(m, np.complex128)
        pack = np.zeros((self.count, self.slots), np.complex128)
        for row in range(self.height):
            c = row // self.count
            pack[row % self.count, c * self.p2:c * self.p2 + self.width] = m[row]
        mod_mask, wrap_mask = self.count - 1, self.p2 - 1
        diag = np.zeros_like(pack)
        for ct in range(self.count):
            for col in range(self.slots):
                dl = (col - ct) & wrap_mask & mod_mask
                dh = (col ^ ct) & self.slots & mod_mask
                cl = (col - dl) & wrap_mask
                ch = (self.p2 * (col // self.p2)) ^ dh
                diag[dh + dl, ch + cl] = pack[ct, col]
        return diag

    def rows(self, slots):
        """decodeResult (app/matmul.cuh:34-43)."""
        return np.array([slots[(i % self.count) + self.p2 * (i // self.count)] for i in range(self.height)])

    def apply(self, m, v):
        """The product on plain slot vectors: sum_i rotate(x, i) * diag_i, then the
        rotate-and-add folds (rotate by k: slot j takes slot j + k)."""
        x = self.input(v)
        d = self.diagonals(m)
        r = sum(np.roll(x, -i) * d[i] for i in range(self.count))
        rot = self.count
        while rot < self.p2:
            r = r + np.roll(r, -rot)
            rot *= 2
        return self.rows(r)

"""The batched CKKS evaluation step: many ciphertext pairs through multiply ->
relinearize -> rescale_to_next -> rotate_vector, each pair rotated by its own step,
as a few concurrent sub-batches on streams of their own.

This is the step the benchmark times (N = 16384, 64 pairs, 13 rotation steps, four
sub-batches) and the step its GPU parity test runs word for word against the
reference's own evaluator (multiply, relinearize, rescaleToNext, rotateVector per
ciphertext: src/evaluator.cpp:626, 1113, 2153-2251; on the GPU
src/evaluator_cuda.cu:384-432, 703-744, 749-824, 2106-2163), so both use this one
implementation.

Rotation steps are assigned in runs: inside a sub-batch as many pairs take step g as
pairs i of the sub-batch have i mod len(steps) == g, and those pairs are consecutive
rows, so one ``tb_apply_galois_groups`` call serves every step of the sub-batch with
its own Galois key (row_groups() gives each row's step).
"""
from __future__ import annotations

import ctypes


def rotation_runs(first, count, nsteps):
    """Rotation groups of pairs first .. first + count - 1, pair i taking step
    i mod nsteps, laid out as contiguous runs (group g, start within the sub-batch,
    count), empty groups left out."""
    runs, at = [], 0
    for g in range(nsteps):
        cnt = sum(1 for i in range(first, first + count) if i % nsteps == g)
        if cnt:
            runs.append((g, at, cnt))
            at += cnt
    return runs


def row_groups(pairs, sub_batches, nsteps):
    """Rotation step index of every pair (row) of a step run as `sub_batches`
    sub-batches: the runs of rotation_runs, one sub-batch after another."""
    pc = pairs // sub_batches
    out = []
    for c in range(sub_batches):
        for g, _, cnt in rotation_runs(c * pc, pc, nsteps):
            out += [g] * cnt
    return out


class BatchedCkksStep:
    """One step of the batched evaluation over device tensors (torch, int64 words).

    ctx: a tb_capi.Context (CKKS); L: data limbs of the inputs; n: degree; pairs: pairs
    per step; rlk: relinearization key [K-1][2][K][n]; elts / gks: the Galois element
    and key of each rotation step; sub_batches: concurrent sub-batches (one stream
    each; 1 runs the whole batch on the caller's stream).

    step(a, b, out, stream): a, b [pairs][2][L][n]; out [pairs][2][L-1][n], row r the
    product of pair r rotated by step row_groups()[r]. sub=1 runs the same workload as
    one batch on the caller's stream (steps then assigned in runs over the whole
    batch: row_groups(sub=1))."""

    def __init__(self, torch, ctx, L, n, pairs, rlk, elts, gks, sub_batches=1):
        self.torch, self.ctx, self.L, self.n, self.pairs = torch, ctx, L, n, pairs
        self.rlk, self.elts, self.gks = rlk, list(elts), list(gks)
        self.sub = sub_batches if sub_batches >= 1 and pairs % sub_batches == 0 else 1
        self.T3 = torch.empty((pairs, 3, L, n), dtype=torch.int64, device="cuda")
        self.R = torch.empty((pairs, 2, L - 1, n), dtype=torch.int64, device="cuda")
        self.whole = self.runs(0, pairs)
        self.pc = pairs // self.sub
        self.parts = [self.runs(c * self.pc, self.pc) for c in range(self.sub)]
        self.streams = [torch.cuda.Stream() for _ in range(self.sub)] if self.sub > 1 else []

    def runs(self, first, count):
        """C-ABI arrays (elements, counts, keys, groups) of the rotation runs of pairs
        first .. first + count - 1."""
        runs = rotation_runs(first, count, len(self.elts))
        return ((ctypes.c_uint32 * len(runs))(*[self.elts[g] for g, _, _ in runs]),
                (ctypes.c_uint64 * len(runs))(*[cnt for _, _, cnt in runs]),
                (ctypes.c_void_p * len(runs))(*[self.gks[g].data_ptr() for g, _, _ in runs]),
                len(runs))

    def row_groups(self, sub=None):
        return row_groups(self.pairs, sub or self.sub, len(self.elts))

    def chain(self, runs, count, rows, a, b, out, st):
        """multiply -> relinearize -> rescale -> grouped rotations of `count` pairs."""
        L, n, ctx = self.L, self.n, self.ctx
        e_, c_, p_, nr = runs
        ctx("multiply", L, a, 0, b, 0, self.T3[rows], 0, count, st)
        ctx("relinearize", L, self.T3[rows], 0, self.rlk, count, st)
        ctx("rescale_to_next", L, self.T3[rows], 3 * L * n, self.R[rows], 0, 2, count, st)
        ctx("apply_galois_groups", L - 1, nr, e_, c_, self.R[rows], 0, out, 0, p_, st)

    def __call__(self, a, b, out, stream, sub=None):
        torch = self.torch
        if (sub or self.sub) == 1:
            self.chain(self.whole, self.pairs, slice(0, self.pairs), a, b, out, stream)
            return
        fork = torch.cuda.Event()
        fork.record(stream)
        for c, sc in enumerate(self.streams):
            sc.wait_event(fork)
            rows = slice(c * self.pc, (c + 1) * self.pc)
            self.chain(self.parts[c], self.pc, rows, a[rows], b[rows], out[rows], sc)
        for sc in self.streams:
            join = torch.cuda.Event()
            join.record(sc)
            stream.wait_event(join)

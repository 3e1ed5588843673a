"""Batches of ciphertexts with different ring degrees and modulus chains in one launch.

A batch is split into shape groups (one parameter context each). Every group runs
its whole pipeline — multiply, relinearize, rotate (apply_galois) — as batched C-ABI
calls on a stream of its own, so the groups overlap on the device; the fork/join of
all groups is captured once into a CUDA graph, after which one graph launch runs the
entire uneven batch. The arithmetic per ciphertext is the same as the one-call-per-
ciphertext path, so the results are identical word for word.
"""
from __future__ import annotations

import torch

import tb_capi


class ShapeGroup:
    """Ciphertext pairs of one parameter set: a, b are [count][2][L][N] device tensors
    (int64 view of uint64 words); rlk and gk the relinearization and Galois keys
    ([K-1][2][K][N]); elt the Galois element of the rotation."""

    def __init__(self, ctx: tb_capi.Context, L: int, a, b, rlk, gk, elt: int):
        self.ctx, self.L, self.a, self.b, self.rlk, self.gk, self.elt = ctx, L, a, b, rlk, gk, elt
        self.count, n = a.shape[0], ctx.n
        self.t3 = torch.empty((self.count, 3, L, n), dtype=torch.int64, device=a.device)
        self.out = torch.empty((self.count, 2, L, n), dtype=torch.int64, device=a.device)

    def run(self, stream):
        ctx, L, n, c = self.ctx, self.L, self.ctx.n, self.count
        ctx("multiply", L, self.a, 0, self.b, 0, self.t3, 0, c, stream)
        ctx("relinearize", L, self.t3, 0, self.rlk, c, stream)
        ctx("apply_galois", L, self.elt, self.t3, 3 * L * n, self.out, 0, self.gk, c, stream)

    def run_per_op(self, stream):
        """The same pipeline one ciphertext per call (the reference's usage pattern)."""
        ctx, L, n = self.ctx, self.L, self.ctx.n
        for i in range(self.count):
            t3, out = self.t3[i:i + 1], self.out[i:i + 1]
            ctx("multiply", L, self.a[i:i + 1], 0, self.b[i:i + 1], 0, t3, 0, 1, stream)
            ctx("relinearize", L, t3, 0, self.rlk, 1, stream)
            ctx("apply_galois", L, self.elt, t3, 3 * L * n, out, 0, self.gk, 1, stream)


class UnevenBatch:
    """All shape groups of one batch: run() issues them on one stream each (joined back
    to the caller's stream); capture() records that fork/join once as a CUDA graph and
    replay() then launches the whole batch with a single graph launch."""

    def __init__(self, groups):
        self.groups = list(groups)
        self.streams = [torch.cuda.Stream() for _ in self.groups]
        self.graph = None

    def run(self, stream=None):
        stream = stream or torch.cuda.current_stream()
        start = torch.cuda.Event()
        start.record(stream)
        ends = []
        for g, s in zip(self.groups, self.streams):
            s.wait_event(start)
            g.run(s)
            e = torch.cuda.Event()
            e.record(s)
            ends.append(e)
        for e in ends:
            stream.wait_event(e)

    def run_per_op(self, stream=None):
        stream = stream or torch.cuda.current_stream()
        for g in self.groups:
            g.run_per_op(stream)

    def capture(self):
        """Records the batch as one CUDA graph. Run the batch once uncaptured first: the
        library builds per-element tables on first use."""
        self.graph = torch.cuda.CUDAGraph()
        cap = torch.cuda.Stream()
        cap.wait_stream(torch.cuda.current_stream())
        with torch.cuda.graph(self.graph, stream=cap, capture_error_mode="relaxed"):
            self.run(cap)
        torch.cuda.current_stream().wait_stream(cap)
        return self.graph

    def replay(self):
        self.graph.replay()

    @property
    def count(self):
        return sum(g.count for g in self.groups)

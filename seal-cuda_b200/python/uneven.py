"""Batches of ciphertexts with different ring degrees and modulus chains (Python side
of the C ABI's uneven batches, ``tb_uneven_*`` in include/troy_b200.h).

A batch is split into shape groups (one parameter context each). The library runs
every group's pipeline — multiply, relinearize, rotate (apply_galois) — as batched
calls on a stream of its own, so the groups overlap on the device; ``capture()``
records that fork/join once as a CUDA graph, after which one graph launch runs the
entire uneven batch. The arithmetic per ciphertext is the same as the
one-call-per-ciphertext path, so the results are identical word for word.
"""
from __future__ import annotations

import ctypes

import torch

import tb_capi


class _Group(ctypes.Structure):
    """tb_uneven_group."""
    _fields_ = [("ctx", ctypes.c_void_p), ("L", ctypes.c_int), ("count", ctypes.c_uint64),
                ("a", ctypes.c_void_p), ("b", ctypes.c_void_p), ("relin_key", ctypes.c_void_p),
                ("galois_key", ctypes.c_void_p), ("galois_elt", ctypes.c_uint32), ("out", ctypes.c_void_p)]


class ShapeGroup:
    """Ciphertext pairs of one parameter set: a, b are [count][2][L][N] device tensors
    (int64 view of uint64 words); rlk and gk the relinearization and Galois keys
    ([K-1][2][K][N]); elt the Galois element of the rotation. out receives the results."""

    def __init__(self, ctx: tb_capi.Context, L: int, a, b, rlk, gk, elt: int):
        self.ctx, self.L, self.a, self.b, self.rlk, self.gk, self.elt = ctx, L, a, b, rlk, gk, elt
        self.count = a.shape[0]
        self.out = torch.empty((self.count, 2, L, ctx.n), dtype=torch.int64, device=a.device)

    def descriptor(self):
        return _Group(self.ctx.h.value if hasattr(self.ctx.h, "value") else self.ctx.h, self.L, self.count,
                      self.a.data_ptr(), self.b.data_ptr(), self.rlk.data_ptr(), self.gk.data_ptr(), self.elt,
                      self.out.data_ptr())


class UnevenBatch:
    """All shape groups of one batch (a ``tb_uneven`` handle): run() issues them on one
    stream each, joined back to the caller's stream; run_per_op() one ciphertext per
    call; capture() records run() once as a CUDA graph and replay() then launches the
    whole batch with a single graph launch."""

    def __init__(self, groups):
        self.groups = list(groups)
        self._lib = tb_capi.lib()
        arr = (_Group * len(self.groups))(*[g.descriptor() for g in self.groups])
        self.h = ctypes.c_void_p()
        self._lib.tb_uneven_create.argtypes = [ctypes.POINTER(_Group), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
        tb_capi.check(self._lib.tb_uneven_create(arr, len(self.groups), ctypes.byref(self.h)))
        self._lib.tb_uneven_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._lib.tb_uneven_run_per_op.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._lib.tb_uneven_capture.argtypes = [ctypes.c_void_p]
        self._lib.tb_uneven_replay.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        self._lib.tb_uneven_destroy.argtypes = [ctypes.c_void_p]

    @staticmethod
    def _s(stream):
        return (stream or torch.cuda.current_stream()).cuda_stream

    def set_shapes(self, on=True):
        """Relinearizations and rotations of every group with one persistent launch per
        key-switch step (tb_uneven_set_shapes); set before capture()."""
        self._lib.tb_uneven_set_shapes.argtypes = [ctypes.c_void_p, ctypes.c_int]
        tb_capi.check(self._lib.tb_uneven_set_shapes(self.h, int(bool(on))))

    def run(self, stream=None):
        tb_capi.check(self._lib.tb_uneven_run(self.h, self._s(stream)))

    def run_per_op(self, stream=None):
        tb_capi.check(self._lib.tb_uneven_run_per_op(self.h, self._s(stream)))

    def capture(self):
        tb_capi.check(self._lib.tb_uneven_capture(self.h))

    def replay(self, stream=None):
        tb_capi.check(self._lib.tb_uneven_replay(self.h, self._s(stream)))

    def close(self):
        if self.h:
            self._lib.tb_uneven_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def count(self):
        return sum(g.count for g in self.groups)

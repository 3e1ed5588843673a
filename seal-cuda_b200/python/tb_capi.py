"""Python binding of the C ABI in include/troy_b200.h (ctypes over lib/libtroy_b200.so).

Device memory, streams and host staging come from PyTorch; every call goes
through the C entry points. There is no fallback: if the CUDA library is missing
or a call fails, a ``TroyError`` is raised.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "lib", "libtroy_b200.so")
HEADER = os.path.join(os.path.dirname(PKG), "include", "troy_b200.h")

SCHEME_RAW, SCHEME_BFV, SCHEME_CKKS, SCHEME_BGV = 0, 1, 2, 3


class TroyError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"troy_b200 status {status}: {msg}")
        self.status = status


_lib = None


def declared_functions(header: str = HEADER):
    """Names of the functions include/troy_b200.h declares."""
    text = open(header).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tb_\w+)\s*\(", text)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TroyError(-1, f"CUDA library not built: {LIB_PATH} (run seal-cuda_b200/build.py)")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.tb_last_error.restype = ctypes.c_char_p
    return _lib


def _ptr(x):
    if x is None:
        return None
    if isinstance(x, int):
        return ctypes.c_void_p(x)
    return ctypes.c_void_p(x.data_ptr())


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return ctypes.c_void_p(s)
    return ctypes.c_void_p(s.cuda_stream)


def check(status):
    if status != 0:
        raise TroyError(status, lib().tb_last_error().decode())
    return status


def call(name, *args):
    """Calls tb_<name>; pointer-like args (tensors) are converted."""
    fn = getattr(lib(), "tb_" + name)
    conv = []
    for a in args:
        if hasattr(a, "data_ptr"):
            conv.append(ctypes.c_void_p(a.data_ptr()))
        elif hasattr(a, "cuda_stream"):
            conv.append(ctypes.c_void_p(a.cuda_stream))
        elif isinstance(a, float):
            conv.append(ctypes.c_double(a))
        elif isinstance(a, bool):
            conv.append(ctypes.c_int(int(a)))
        elif isinstance(a, int):
            conv.append(ctypes.c_uint64(a) if a >= 2 ** 31 or a < -(2 ** 31) else ctypes.c_longlong(a))
        else:
            conv.append(a)
    return check(fn(*conv))


class Context:
    """A parameter context (tb_context_create)."""

    def __init__(self, scheme, n, moduli, plain_modulus=0):
        L = lib()
        L.tb_context_create.argtypes = [ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64), ctypes.c_int,
                                        ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p)]
        arr = (ctypes.c_uint64 * len(moduli))(*[int(m) for m in moduli])
        h = ctypes.c_void_p()
        check(L.tb_context_create(scheme, n, arr, len(moduli), int(plain_modulus), ctypes.byref(h)))
        self.h = h
        self.n = n
        self.logn = n.bit_length() - 1
        self.moduli = [int(m) for m in moduli]
        self.scheme = scheme
        self.t = int(plain_modulus)

    def close(self):
        if self.h:
            lib().tb_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def table_moduli(self):
        L = lib()
        cnt = ctypes.c_int()
        out = (ctypes.c_uint64 * 256)()
        check(L.tb_context_moduli(self.h, out, 256, ctypes.byref(cnt)))
        return [int(out[i]) for i in range(cnt.value)]

    # raw calls: (name, *args) with the context handle prepended
    def __call__(self, name, *args):
        L = lib()
        fn = getattr(L, "tb_" + name)
        conv = [self.h]
        for a in args:
            if hasattr(a, "data_ptr"):
                conv.append(ctypes.c_void_p(a.data_ptr()))
            elif hasattr(a, "cuda_stream"):
                conv.append(ctypes.c_void_p(a.cuda_stream))
            elif a is None:
                conv.append(ctypes.c_void_p(0))
            elif isinstance(a, float):
                conv.append(ctypes.c_double(a))
            elif isinstance(a, bool):
                conv.append(ctypes.c_int(int(a)))
            elif isinstance(a, ctypes._SimpleCData) or isinstance(a, ctypes.Array):
                conv.append(a)
            elif isinstance(a, int):
                conv.append(ctypes.c_uint64(a) if (a >= 2 ** 31 or a < -(2 ** 31)) else ctypes.c_longlong(a))
            else:
                conv.append(a)
        return check(fn(*conv))

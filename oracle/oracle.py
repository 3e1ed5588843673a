"""ctypes front end for the two CPU checkers under oracle/.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
bench.py's CPU-baseline leg, never by the product.

* ``Oracle("orc")`` loads ``oracle/liboracle.so``, the plain-C restatement of the
  reference's hot-path algorithms (troy_oracle.c, each function citing the
  reference file it follows).
* ``Oracle("ref")`` loads ``oracle/_ref/libtroyref.so``, the reference's own CPU
  implementation compiled from its sources plus a C shim (ref_shim.cpp). It
  exposes the same primitive entry points and, in addition, seeded end-to-end
  sessions used to pin ciphertext words.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {
    "orc": os.path.join(HERE, "liboracle.so"),
    "ref": os.path.join(HERE, "_ref", "libtroyref.so"),
}

_u64 = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
_i32 = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64 = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_sz = ctypes.c_size_t
_c = ctypes


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind])


def _arr(x, dtype=np.uint64):
    return np.ascontiguousarray(np.asarray(x, dtype=dtype))


class Oracle:
    """Primitive entry points shared by the restatement and the compiled reference."""

    def __init__(self, kind: str = "orc"):
        if kind not in LIBS:
            raise ValueError(kind)
        self.kind = kind
        self.lib = ctypes.CDLL(LIBS[kind])
        p = kind + "_"
        L = self.lib
        self._f = {}

        def bind(name, res, args):
            fn = getattr(L, p + name)
            fn.restype = res
            fn.argtypes = args
            self._f[name] = fn

        bind("ntt_tables", _c.c_int, [_c.c_int, _c.c_uint64, _u64, _u64, _u64, _u64, _u64])
        bind("ntt_forward", _c.c_int, [_c.c_int, _c.c_uint64, _u64, _c.c_int])
        bind("ntt_inverse", _c.c_int, [_c.c_int, _c.c_uint64, _u64, _c.c_int])
        bind("dyadic_product", None, [_c.c_uint64, _u64, _u64, _u64, _sz])
        bind("coeff_modulus_create", _c.c_int, [_sz, _i32, _c.c_int, _u64])
        bind("plain_modulus_batching", _c.c_int, [_sz, _c.c_int, _u64])
        bind("prng_bytes", None, [_u64, _sz, _sz, _u8])
        bind("sample", _c.c_int, [_c.c_int, _u64, _sz, _u64, _c.c_int, _u64])
        bind("rns_op", _c.c_int, [_c.c_int, _sz, _u64, _c.c_int, _c.c_uint64, _u64, _u64])
        bind("rns_bases", _c.c_int, [_sz, _u64, _c.c_int, _c.c_uint64, _u64])
        bind("galois_elt_from_step", _c.c_uint32, [_c.c_int, _c.c_int])
        bind("apply_galois", None, [_c.c_int, _c.c_uint32, _c.c_uint64, _u64, _u64])
        bind("apply_galois_ntt", None, [_c.c_int, _c.c_uint32, _u64, _u64])
        if kind == "orc":
            bind("keyswitch", _c.c_int, [_c.c_int, _c.c_int, _u64, _c.c_int, _c.c_uint64, _u64, _u64, _u64])
            bind("bfv_multiply", _c.c_int, [_sz, _u64, _c.c_int, _c.c_uint64, _u64, _u64, _u64])
            bind("sample_at", _c.c_int, [_c.c_int, _u64, _c.POINTER(_sz), _sz, _u64, _c.c_int, _u64])
            bind("poly_add", None, [_u64, _c.c_int, _sz, _u64, _u64, _u64])
            bind("poly_sub", None, [_u64, _c.c_int, _sz, _u64, _u64, _u64])
            bind("poly_negate", None, [_u64, _c.c_int, _sz, _u64, _u64])
            bind("poly_dyadic", None, [_u64, _c.c_int, _sz, _u64, _u64, _u64])
            bind("poly_mul_scalar", None, [_u64, _c.c_int, _sz, _u64, _c.c_uint64, _u64])
            bind("ntt_forward_rns", _c.c_int, [_c.c_int, _u64, _c.c_int, _u64, _c.c_int])
            bind("ntt_inverse_rns", _c.c_int, [_c.c_int, _u64, _c.c_int, _u64, _c.c_int])
        if kind == "ref":
            bind("parms_id", _c.c_int, [_c.c_int, _sz, _u64, _c.c_int, _c.c_uint64, _u64])
            bind("bfv_default", _c.c_int, [_sz, _c.c_int, _u64, _c.c_int])
            bind("context_consts", _c.c_int, [_c.c_int, _sz, _u64, _c.c_int, _c.c_uint64, _c.c_int, _u64])

    # ------------------------------------------------------------ primitives
    def ntt_tables(self, logn, q):
        n = 1 << logn
        a, b, c, d = (np.zeros(n, np.uint64) for _ in range(4))
        e = np.zeros(3, np.uint64)
        if self._f["ntt_tables"](logn, q, a, b, c, d, e):
            raise ValueError("no NTT tables for this modulus")
        return a, b, c, d, e

    def ntt_forward(self, logn, q, data, lazy=False):
        x = _arr(data).copy()
        if self._f["ntt_forward"](logn, q, x, int(lazy)):
            raise ValueError("ntt failed")
        return x

    def ntt_inverse(self, logn, q, data, lazy=False):
        x = _arr(data).copy()
        if self._f["ntt_inverse"](logn, q, x, int(lazy)):
            raise ValueError("ntt failed")
        return x

    def ntt_forward_rns(self, logn, moduli, data, lazy=False):
        """[..., L, n] forward transform, limb l with moduli[l]."""
        x = _arr(data).copy()
        L = len(moduli)
        flat = x.reshape(-1, L, 1 << logn)
        for p in range(flat.shape[0]):
            for l in range(L):
                row = np.ascontiguousarray(flat[p, l])
                self._f["ntt_forward"](logn, int(moduli[l]), row, int(lazy))
                flat[p, l] = row
        return flat.reshape(x.shape)

    def ntt_inverse_rns(self, logn, moduli, data, lazy=False):
        x = _arr(data).copy()
        L = len(moduli)
        flat = x.reshape(-1, L, 1 << logn)
        for p in range(flat.shape[0]):
            for l in range(L):
                row = np.ascontiguousarray(flat[p, l])
                self._f["ntt_inverse"](logn, int(moduli[l]), row, int(lazy))
                flat[p, l] = row
        return flat.reshape(x.shape)

    def dyadic_product(self, q, a, b):
        a, b = _arr(a), _arr(b)
        out = np.zeros_like(a)
        self._f["dyadic_product"](q, a, b, out, a.size)
        return out

    def dyadic_rns(self, moduli, a, b):
        a, b = _arr(a), _arr(b)
        L = len(moduli)
        n = a.shape[-1]
        fa, fb = a.reshape(-1, L, n), b.reshape(-1, L, n)
        out = np.zeros_like(fa)
        for p in range(fa.shape[0]):
            for l in range(L):
                o = np.zeros(n, np.uint64)
                self._f["dyadic_product"](int(moduli[l]), np.ascontiguousarray(fa[p, l]),
                                          np.ascontiguousarray(fb[p, l]), o, n)
                out[p, l] = o
        return out.reshape(a.shape)

    def coeff_modulus_create(self, n, bits):
        out = np.zeros(len(bits), np.uint64)
        if self._f["coeff_modulus_create"](n, _arr(bits, np.int32), len(bits), out):
            raise ValueError("cannot create coeff modulus")
        return [int(x) for x in out]

    def parms_id(self, scheme, n, moduli, t):
        """EncryptionParameters::parmsID of the compiled reference (kind "ref" only)."""
        out = np.zeros(4, np.uint64)
        if self._f["parms_id"](scheme, n, _arr(moduli), len(moduli), t, out):
            raise ValueError("invalid parameters")
        return [int(x) for x in out]

    def bfv_default(self, n, sec):
        """CoeffModulus::BFVDefault of the compiled reference (kind "ref" only); sec is
        128, 192 or 256. None when the reference rejects the arguments."""
        out = np.zeros(64, np.uint64)
        k = self._f["bfv_default"](n, sec, out, 64)
        return None if k < 0 else [int(x) for x in out[:k]]

    def context_consts(self, scheme, n, moduli, t, sec):
        """The reference's first-level qualifiers and constants (kind "ref" only), as a
        dict; None when the reference throws."""
        out = np.zeros(9 + 6 * len(moduli), np.uint64)
        L = self._f["context_consts"](scheme, n, _arr(moduli), len(moduli), t, sec, out)
        if L < 0:
            return None
        head = [int(x) for x in out[:9]]
        rows = out[9:9 + 6 * L].reshape(6, L)
        keys = ("total", "delta", "delta_quotient", "upper_half_increment", "plain_upper_half_increment",
                "upper_half_threshold")
        d = {k: [int(x) for x in r] for k, r in zip(keys, rows)}
        d.update(error=np.int64(np.uint64(head[0])).item(), using_fft=head[1], using_ntt=head[2],
                 using_batching=head[3], using_fast_plain_lift=head[4], using_descending_modulus_chain=head[5],
                 sec_level=head[6], q_mod_t=head[7], plain_upper_half_threshold=head[8])
        return d

    def plain_modulus_batching(self, n, bits):
        out = np.zeros(1, np.uint64)
        if self._f["plain_modulus_batching"](n, bits, out):
            raise ValueError("no batching prime")
        return int(out[0])

    def prng_bytes(self, seed8, offset, count):
        out = np.zeros(count, np.uint8)
        self._f["prng_bytes"](_arr(seed8), offset, count, out)
        return out

    def sample(self, kind, seed8, n, moduli):
        out = np.zeros(len(moduli) * n, np.uint64)
        if self._f["sample"](kind, _arr(seed8), n, _arr(moduli), len(moduli), out):
            raise ValueError("sampling failed")
        return out.reshape(len(moduli), n)

    def sample_at(self, kind, seed8, offset, n, moduli):
        """Sample from stream position `offset`; returns (values [L][n], new offset)."""
        out = np.zeros(len(moduli) * n, np.uint64)
        off = _sz(offset)
        if self._f["sample_at"](kind, _arr(seed8), ctypes.byref(off), n, _arr(moduli), len(moduli), out):
            raise ValueError("sampling failed")
        return out.reshape(len(moduli), n), off.value

    RNS_OPS = {
        "fastbconv_mtilde": 0, "sm_mrq": 1, "fast_floor": 2, "fastbconv_sk": 3,
        "div_round_last": 4, "div_round_last_ntt": 5, "decrypt_scale_round": 6,
        "mod_t_div_last": 7, "decrypt_mod_t": 8,
    }

    def rns_bases(self, n, q, t):
        out = np.zeros(70, np.uint64)
        bsk = self._f["rns_bases"](n, _arr(q), len(q), t, out)
        if bsk < 0:
            raise ValueError("rns tool")
        return int(out[0]), int(out[1]), [int(x) for x in out[2:2 + bsk]]

    def rns_op(self, op, n, q, t, data, out_limbs):
        data = _arr(data)
        out = np.zeros(out_limbs * n, np.uint64)
        if self._f["rns_op"](self.RNS_OPS[op], n, _arr(q), len(q), t, data, out):
            raise ValueError("rns op failed")
        return out.reshape(out_limbs, n)

    def galois_elt_from_step(self, logn, step):
        return int(self._f["galois_elt_from_step"](logn, step))

    def apply_galois(self, logn, elt, q, data):
        out = np.zeros(1 << logn, np.uint64)
        self._f["apply_galois"](logn, elt, q, _arr(data), out)
        return out

    def apply_galois_ntt(self, logn, elt, data):
        out = np.zeros(1 << logn, np.uint64)
        self._f["apply_galois_ntt"](logn, elt, _arr(data), out)
        return out

    # ---------------------------------------------------- restatement only
    def keyswitch(self, scheme, logn, key_moduli, t, target, ct, key):
        """Key switching; returns the updated [2][L][n] ciphertext."""
        L = len(key_moduli) - 1
        ct = _arr(ct).copy()
        if self._f["keyswitch"](scheme, logn, _arr(key_moduli), L, t, _arr(target), ct, _arr(key)):
            raise ValueError("keyswitch failed")
        return ct

    def bfv_multiply(self, n, q, t, ct1, ct2):
        out = np.zeros(3 * len(q) * n, np.uint64)
        if self._f["bfv_multiply"](n, _arr(q), len(q), t, _arr(ct1), _arr(ct2), out):
            raise ValueError("bfv multiply failed")
        return out.reshape(3, len(q), n)


class RefSession:
    """A seeded end-to-end session of the compiled reference (oracle/_ref).

    scheme: 1 bfv, 2 ckks, 3 bgv; moduli: the key-level chain, special prime last.
    """

    def __init__(self, scheme, n, moduli, t, seed8):
        self.lib = ctypes.CDLL(LIBS["ref"])
        L = self.lib
        L.ref_session_new.restype = ctypes.c_void_p
        L.ref_session_new.argtypes = [_c.c_int, _sz, _u64, _c.c_int, _c.c_uint64, _u64]
        L.ref_session_free.argtypes = [_c.c_void_p]
        for nm in ("ref_secret_key", "ref_public_key", "ref_relin_key"):
            getattr(L, nm).restype = _sz
            getattr(L, nm).argtypes = [_c.c_void_p, _c.c_void_p]
        L.ref_galois_key.restype = _sz
        L.ref_galois_key.argtypes = [_c.c_void_p, _c.c_uint32, _c.c_void_p]
        L.ref_ct_encrypt_slots.argtypes = [_c.c_void_p, _u64, _sz]
        L.ref_encode_slots.argtypes = [_c.c_void_p, _u64, _sz, _u64]
        L.ref_ct_encrypt_ckks.argtypes = [_c.c_void_p, _f64, _f64, _sz, _c.c_double]
        L.ref_encode_ckks.argtypes = [_c.c_void_p, _f64, _f64, _sz, _c.c_double, _u64]
        L.ref_ct_get.restype = _sz
        L.ref_ct_get.argtypes = [_c.c_void_p, _c.c_int, _c.c_void_p, _c.c_void_p, _c.c_void_p]
        L.ref_ct_multiply.argtypes = [_c.c_void_p, _c.c_int, _c.c_int]
        L.ref_ct_add.argtypes = [_c.c_void_p, _c.c_int, _c.c_int]
        L.ref_ct_encrypt_poly.argtypes = [_c.c_void_p, _u64, _sz, _c.c_int]
        L.ref_ct_multiply_plain_poly.argtypes = [_c.c_void_p, _c.c_int, _u64, _sz]
        L.ref_ct_from_words.argtypes = [_c.c_void_p, _u64, _sz, _sz, _c.c_int, _c.c_double, _c.c_uint64]
        L.ref_ct_encrypt_plain_words.argtypes = [_c.c_void_p, _u64, _sz, _c.c_double, _c.c_int]
        L.ref_ct_multiply_plain_words.argtypes = [_c.c_void_p, _c.c_int, _u64, _sz, _c.c_double]
        L.ref_ct_relinearize.argtypes = [_c.c_void_p, _c.c_int]
        L.ref_ct_rotate.argtypes = [_c.c_void_p, _c.c_int, _c.c_int, _c.c_int]
        L.ref_ct_rescale.argtypes = [_c.c_void_p, _c.c_int]
        L.ref_ct_mod_switch.argtypes = [_c.c_void_p, _c.c_int]
        L.ref_ct_multiply_plain_slots.argtypes = [_c.c_void_p, _c.c_int, _u64, _sz]
        L.ref_ct_decrypt_slots.argtypes = [_c.c_void_p, _c.c_int, _u64, _sz]
        L.ref_ct_decrypt_ckks.argtypes = [_c.c_void_p, _c.c_int, _f64, _f64, _sz]
        self.n = n
        self.moduli = list(moduli)
        self.h = L.ref_session_new(scheme, n, _arr(moduli), len(moduli), t, _arr(seed8))
        if not self.h:
            raise ValueError("reference rejected the parameters")

    def close(self):
        if self.h:
            self.lib.ref_session_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _dump(self, fn, *args):
        words = fn(self.h, *args, None)
        out = np.zeros(words, np.uint64)
        fn(self.h, *args, out.ctypes.data_as(ctypes.c_void_p))
        return out

    def secret_key(self):
        return self._dump(self.lib.ref_secret_key).reshape(len(self.moduli), self.n)

    def public_key(self):
        return self._dump(self.lib.ref_public_key).reshape(2, len(self.moduli), self.n)

    def relin_key(self):
        K = len(self.moduli)
        return self._dump(self.lib.ref_relin_key).reshape(K - 1, 2, K, self.n)

    def galois_key(self, elt):
        K = len(self.moduli)
        return self._dump(self.lib.ref_galois_key, elt).reshape(K - 1, 2, K, self.n)

    def _check(self, i):
        if i < 0:
            raise ValueError("reference operation failed")
        return i

    def encrypt_slots(self, slots):
        s = _arr(slots)
        return self._check(self.lib.ref_ct_encrypt_slots(self.h, s, s.size))

    def encode_slots(self, slots):
        s = _arr(slots)
        out = np.zeros(self.n, np.uint64)
        k = self.lib.ref_encode_slots(self.h, s, s.size, out)
        return out[:k]

    def encrypt_ckks(self, values, scale):
        v = np.asarray(values, np.complex128)
        re, im = _arr(v.real, np.float64), _arr(v.imag, np.float64)
        return self._check(self.lib.ref_ct_encrypt_ckks(self.h, re, im, v.size, scale))

    def encode_ckks(self, values, scale):
        v = np.asarray(values, np.complex128)
        re, im = _arr(v.real, np.float64), _arr(v.imag, np.float64)
        out = np.zeros(self.n * len(self.moduli), np.uint64)
        k = self.lib.ref_encode_ckks(self.h, re, im, v.size, scale, out)
        return out[:k]

    def ct(self, i):
        info = np.zeros(4, np.uint64)
        scale = np.zeros(1, np.float64)
        words = self.lib.ref_ct_get(self.h, i, None, None, None)
        out = np.zeros(words, np.uint64)
        self.lib.ref_ct_get(self.h, i, out.ctypes.data_as(ctypes.c_void_p), info.ctypes.data_as(ctypes.c_void_p),
                            scale.ctypes.data_as(ctypes.c_void_p))
        size, limbs = int(info[0]), int(info[1])
        return {"data": out.reshape(size, limbs, self.n), "ntt": bool(info[2]), "correction": int(info[3]),
                "scale": float(scale[0])}

    def multiply(self, a, b):
        return self._check(self.lib.ref_ct_multiply(self.h, a, b))

    def add(self, a, b):
        return self._check(self.lib.ref_ct_add(self.h, a, b))

    def relinearize(self, a):
        return self._check(self.lib.ref_ct_relinearize(self.h, a))

    def rotate_rows(self, a, step):
        return self._check(self.lib.ref_ct_rotate(self.h, a, 0, step))

    def rotate_columns(self, a):
        return self._check(self.lib.ref_ct_rotate(self.h, a, 1, 0))

    def rotate_vector(self, a, step):
        return self._check(self.lib.ref_ct_rotate(self.h, a, 2, step))

    def rescale(self, a):
        return self._check(self.lib.ref_ct_rescale(self.h, a))

    def mod_switch(self, a):
        return self._check(self.lib.ref_ct_mod_switch(self.h, a))

    def encrypt_poly(self, coeffs, symmetric=False):
        """Encryption of the coefficient-encoded plaintext (encodePolynomial), with the
        public key or (symmetric) the secret key."""
        c = _arr(coeffs)
        return self._check(self.lib.ref_ct_encrypt_poly(self.h, c, c.size, int(bool(symmetric))))

    def multiply_plain_poly(self, a, coeffs):
        c = _arr(coeffs)
        return self._check(self.lib.ref_ct_multiply_plain_poly(self.h, a, c, c.size))

    def ct_from_words(self, words, size, limbs, ntt, scale=1.0, correction=1):
        """A ciphertext given as words (size x limbs x n) at the level with `limbs` primes."""
        w = _arr(words)
        return self._check(self.lib.ref_ct_from_words(self.h, w, size, limbs, int(bool(ntt)), scale, correction))

    def encrypt_plain_words(self, words, scale=1.0, symmetric=False):
        """Encryption of a plaintext given as words at the first level (CKKS: NTT form)."""
        w = _arr(words)
        return self._check(self.lib.ref_ct_encrypt_plain_words(self.h, w, w.size, scale, int(bool(symmetric))))

    def multiply_plain_words(self, a, words, scale=1.0):
        """multiplyPlain by a plaintext given as words at the ciphertext's level."""
        w = _arr(words)
        return self._check(self.lib.ref_ct_multiply_plain_words(self.h, a, w, w.size, scale))

    def multiply_plain_slots(self, a, slots):
        s = _arr(slots)
        return self._check(self.lib.ref_ct_multiply_plain_slots(self.h, a, s, s.size))

    def decrypt_slots(self, a):
        out = np.zeros(self.n, np.uint64)
        if self.lib.ref_ct_decrypt_slots(self.h, a, out, self.n):
            raise ValueError("decrypt failed")
        return out

    def decrypt_ckks(self, a, count):
        re, im = np.zeros(count), np.zeros(count)
        if self.lib.ref_ct_decrypt_ckks(self.h, a, re, im, count):
            raise ValueError("decrypt failed")
        return re + 1j * im

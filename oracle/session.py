"""End-to-end CPU restatement of the reference's scheme layer, on the C oracle.

TEST INFRASTRUCTURE ONLY (imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg). ``OracleSession`` mirrors a seeded reference
session: key generation (src/keygenerator.cpp), zero encryption
(src/utils/rlwe.cpp), encryption (src/encryptor.cpp), the evaluator operations on
the hot path (src/evaluator.cpp), decryption (src/decryptor.cpp) and both
encoders (src/batchencoder.cpp, src/ckks.cpp). The heavy per-limb arithmetic is
done by oracle/liboracle.so; Python composes the steps in the reference's order,
including the order in which the seeded PRNG stream is consumed.

Seeded PRNG semantics (src/randomgen.h:412-427): a Blake2xbPRNGFactory built with
a seed gives every PRNG it creates that same seed, so every create() restarts the
stream at offset 0.
"""
from __future__ import annotations

import numpy as np

from oracle import Oracle

BFV, CKKS, BGV = 1, 2, 3


def _bitrev(x: int, bits: int) -> int:
    r = 0
    for _ in range(bits):
        r = (r << 1) | (x & 1)
        x >>= 1
    return r


def matrix_reps_index_map(n: int, slots: int) -> np.ndarray:
    """BatchEncoder/CKKSEncoder slot -> coefficient map (src/batchencoder.cpp:64-82,
    src/ckks.cpp:45-60)."""
    logn = n.bit_length() - 1
    m = n << 1
    out = np.zeros(2 * slots, np.int64)
    pos = 1
    for i in range(slots):
        out[i] = _bitrev((pos - 1) >> 1, logn)
        out[slots + i] = _bitrev((m - pos - 1) >> 1, logn)
        pos = (pos * 3) & (m - 1)
    return out


class OracleSession:
    """scheme: 1 bfv, 2 ckks, 3 bgv. moduli: key-level chain, special prime last."""

    def __init__(self, scheme, n, moduli, t, seed8, o: Oracle | None = None):
        self.o = o or Oracle("orc")
        self.scheme, self.n, self.t = scheme, n, int(t)
        self.logn = n.bit_length() - 1
        self.moduli = [int(x) for x in moduli]
        self.K = len(self.moduli)
        self.seed = np.ascontiguousarray(np.asarray(seed8, np.uint64))
        # KeyGenerator::generateSk (src/keygenerator.cpp:47-74): ternary over the key
        # level from a fresh PRNG, then NTT
        sk, _ = self.o.sample_at(0, self.seed, 0, n, self.moduli)
        self.sk = self.o.ntt_forward_rns(self.logn, self.moduli, sk)
        self.pk = self.encrypt_zero_symmetric(self.moduli, True)
        self.index_map = matrix_reps_index_map(n, n // 2)
        self._plain_tables = None

    # ------------------------------------------------------------ helpers
    def level_moduli(self, L):
        return self.moduli[:L]

    def _rand_poly(self, kind, offset, moduli):
        return self.o.sample_at(kind, self.seed, offset, self.n, moduli)

    # ------------------------------------------------------ zero encryption
    def encrypt_zero_symmetric(self, moduli, is_ntt):
        """util::encryptZeroSymmetric (src/utils/rlwe.cpp:232-357)."""
        o, n, L = self.o, self.n, len(moduli)
        public_seed = o.prng_bytes(self.seed, 0, 64).view(np.uint64).copy()
        c1, _ = o.sample_at(2, public_seed, 0, n, moduli)
        e, _ = self._rand_poly(1, 64, moduli)
        sk = self.sk[:L]
        c0 = o.dyadic_rns(moduli, sk, c1)
        if is_ntt:
            e = o.ntt_forward_rns(self.logn, moduli, e)
        else:
            c0 = o.ntt_inverse_rns(self.logn, moduli, c0)
        if self.scheme == BGV:
            e = self._mul_scalar(moduli, e, self.t)
        c0 = self._add(moduli, e, c0)
        c0 = self._neg(moduli, c0)
        if not is_ntt:
            c1 = o.ntt_inverse_rns(self.logn, moduli, c1)
        return np.stack([c0, c1])

    def encrypt_zero_asymmetric(self, moduli, is_ntt):
        """util::encryptZeroAsymmetric (src/utils/rlwe.cpp:152-230), u and e from one PRNG."""
        o, n, L = self.o, self.n, len(moduli)
        u, off = self._rand_poly(0, 0, moduli)
        u = o.ntt_forward_rns(self.logn, moduli, u)
        pk = self.pk[:, :L] if L == self.K else np.stack([self.pk[0][:L], self.pk[1][:L]])
        dest = np.stack([o.dyadic_rns(moduli, u, pk[j]) for j in range(2)])
        if not is_ntt:
            dest = o.ntt_inverse_rns(self.logn, moduli, dest)
        for j in range(2):
            e, off = self._rand_poly(1, off, moduli)
            if self.scheme == BGV:
                if is_ntt:
                    e = o.ntt_forward_rns(self.logn, moduli, e, lazy=True)
                e = self._mul_scalar(moduli, e, self.t)
            elif is_ntt:
                e = o.ntt_forward_rns(self.logn, moduli, e)
            dest[j] = self._add(moduli, e, dest[j])
        return dest

    # -------------------------------------------------------------- keys
    def _kswitch_key(self, new_key):
        """KeyGenerator::generateOneKswitchKey (src/keygenerator.cpp:294-322)."""
        K = self.K
        out = np.zeros((K - 1, 2, K, self.n), np.uint64)
        qk = self.moduli[-1]
        for i in range(K - 1):
            ek = self.encrypt_zero_symmetric(self.moduli, True)
            qi = self.moduli[i]
            tmp = self._mul_scalar([qi], new_key[i:i + 1], qk % qi)
            ek[0][i] = self._add([qi], ek[0][i:i + 1], tmp)[0]
            out[i] = ek
        return out

    def relin_key(self):
        s2 = self.o.dyadic_rns(self.moduli, self.sk, self.sk)
        return self._kswitch_key(s2)

    def galois_key(self, elt):
        rot = np.stack([self.o.apply_galois_ntt(self.logn, elt, self.sk[i]) for i in range(self.K)])
        return self._kswitch_key(rot)

    # ---------------------------------------------------------- encoding
    def encode_slots(self, values):
        """BatchEncoder::encode (src/batchencoder.cpp:104-128)."""
        n, t = self.n, self.t
        dest = np.zeros(n, np.uint64)
        v = np.asarray(values, np.uint64)
        dest[self.index_map[:len(v)]] = v
        return self.o.ntt_inverse(self.logn, t, dest)

    def decode_slots(self, plain):
        """BatchEncoder::decode (src/batchencoder.cpp:155-182)."""
        tmp = np.zeros(self.n, np.uint64)
        p = np.asarray(plain, np.uint64)[: self.n]
        tmp[: len(p)] = p
        tmp = self.o.ntt_forward(self.logn, self.t, tmp)
        return tmp[self.index_map]

    # -------------------------------------------------------- encryption
    def _q_products(self, moduli):
        Q = 1
        for m in moduli:
            Q *= m
        return Q

    def encrypt_slots(self, values):
        return self.encrypt_plain(self.encode_slots(values))

    def encrypt_plain(self, plain):
        """Encryptor::encryptInternal, asymmetric (src/encryptor.cpp:92-237)."""
        K = self.K
        first = self.moduli[:K - 1]
        is_ntt = self.scheme == CKKS
        tmp = self.encrypt_zero_asymmetric(self.moduli, is_ntt)
        op = {BFV: "div_round_last", CKKS: "div_round_last_ntt", BGV: "mod_t_div_last"}[self.scheme]
        ct = np.stack([self.o.rns_op(op, self.n, self.moduli, self.t, tmp[j], K)[: K - 1] for j in range(2)])
        if self.scheme == BFV:
            ct[0] = self._multiply_add_plain_scaling_variant(first, ct[0], plain)
        elif self.scheme == BGV:
            p = np.asarray(plain, np.uint64)
            for j, qj in enumerate(first):
                m = np.array([int(x) % qj for x in p], np.uint64)
                ct[0][j][: len(p)] = (ct[0][j][: len(p)].astype(object) + m.astype(object)) % qj
        else:
            ct[0] = self._add(first, ct[0], plain)
        return ct

    def _multiply_add_plain_scaling_variant(self, moduli, c0, plain):
        """util::multiplyAddPlainWithScalingVariant (src/utils/scalingvariant.cpp:51-81)."""
        t = self.t
        Q = self._q_products(moduli)
        q_mod_t = Q % t
        q_div_t = Q // t
        thr = (t + 1) >> 1
        out = c0.copy()
        p = [int(x) for x in np.asarray(plain, np.uint64)]
        for j, qj in enumerate(moduli):
            cd = q_div_t % qj
            row = out[j].astype(object)
            for i, m in enumerate(p):
                fix = (m * q_mod_t + thr) // t
                row[i] = (int(row[i]) + (m * cd + fix) % qj) % qj
            out[j] = np.array(row, dtype=np.uint64)
        return out

    # -------------------------------------------------------- evaluator
    def multiply(self, a, b):
        L = a.shape[1]
        moduli = self.moduli[:L]
        if self.scheme == BFV:
            return self.o.bfv_multiply(self.n, moduli, self.t, a, b)
        if self.scheme == CKKS:
            return self._tensor(moduli, a, b)
        # BGV (src/evaluator.cpp:704-794)
        an = self.o.ntt_forward_rns(self.logn, moduli, a)
        bn = self.o.ntt_forward_rns(self.logn, moduli, b)
        return self.o.ntt_inverse_rns(self.logn, moduli, self._tensor(moduli, an, bn))

    def _tensor(self, moduli, a, b):
        d0 = self.o.dyadic_rns(moduli, a[0], b[0])
        d1 = self._add(moduli, self.o.dyadic_rns(moduli, a[0], b[1]), self.o.dyadic_rns(moduli, a[1], b[0]))
        d2 = self.o.dyadic_rns(moduli, a[1], b[1])
        return np.stack([d0, d1, d2])

    def _key_for_level(self, key, L):
        """Digits and key limbs a level-L key switch reads: limbs 0..L-1 and the special prime."""
        sub = np.concatenate([key[:L, :, :L], key[:L, :, -1:]], axis=2)
        return np.ascontiguousarray(sub)

    def keyswitch(self, ct2, target, key):
        L = ct2.shape[1]
        km = self.moduli[:L] + [self.moduli[-1]]
        return self.o.keyswitch(self.scheme, self.logn, km, self.t, target, ct2, self._key_for_level(key, L))

    def relinearize(self, ct3, rlk):
        """Evaluator::relinearizeInternal for size 3 (src/evaluator.cpp:1113-1163)."""
        return self.keyswitch(ct3[:2].copy(), ct3[2], rlk)

    def apply_galois(self, ct, elt, gk):
        """Evaluator::applyGaloisInplace (src/evaluator.cpp:2153-2249)."""
        L = ct.shape[1]
        moduli = self.moduli[:L]
        if self.scheme == CKKS:
            c0 = np.stack([self.o.apply_galois_ntt(self.logn, elt, ct[0][i]) for i in range(L)])
            tgt = np.stack([self.o.apply_galois_ntt(self.logn, elt, ct[1][i]) for i in range(L)])
        else:
            c0 = np.stack([self.o.apply_galois(self.logn, elt, moduli[i], ct[0][i]) for i in range(L)])
            tgt = np.stack([self.o.apply_galois(self.logn, elt, moduli[i], ct[1][i]) for i in range(L)])
        base = np.stack([c0, np.zeros_like(c0)])
        return self.keyswitch(base, tgt, gk)

    def rotate(self, ct, step, gk):
        return self.apply_galois(ct, self.o.galois_elt_from_step(self.logn, step), gk)

    def rescale(self, ct):
        """Evaluator::modSwitchScaleToNext (src/evaluator.cpp:1165-1239)."""
        L = ct.shape[1]
        moduli = self.moduli[:L]
        op = {BFV: "div_round_last", CKKS: "div_round_last_ntt", BGV: "mod_t_div_last"}[self.scheme]
        return np.stack([self.o.rns_op(op, self.n, moduli, self.t, ct[j], L)[: L - 1] for j in range(ct.shape[0])])

    def multiply_plain_slots(self, ct, values):
        """Evaluator::multiplyPlainNormal for BFV/BGV (src/evaluator.cpp:1791-1930): the plain
        lift is centred (upper half gets q - t added), then NTT, dyadic, INTT."""
        plain = self.encode_slots(values)
        L = ct.shape[1]
        moduli = self.moduli[:L]
        t = self.t
        thr = (t + 1) >> 1
        lifted = np.zeros((L, self.n), np.uint64)
        for j, qj in enumerate(moduli):
            row = [(int(p) + (qj - t)) % qj if int(p) >= thr else int(p) % qj for p in plain]
            lifted[j, : len(row)] = row
        pn = self.o.ntt_forward_rns(self.logn, moduli, lifted)
        cn = self.o.ntt_forward_rns(self.logn, moduli, ct)
        prod = np.stack([self.o.dyadic_rns(moduli, cn[k], pn) for k in range(ct.shape[0])])
        return self.o.ntt_inverse_rns(self.logn, moduli, prod)

    # -------------------------------------------------------- decryption
    def phase(self, ct):
        """Decryptor::dotProductCtSkArray for size-2 ciphertexts."""
        L = ct.shape[1]
        moduli = self.moduli[:L]
        sk = self.sk[:L]
        if self.scheme == CKKS:
            return self._add(moduli, ct[0], self.o.dyadic_rns(moduli, ct[1], sk))
        c1 = self.o.ntt_forward_rns(self.logn, moduli, ct[1])
        prod = self.o.ntt_inverse_rns(self.logn, moduli, self.o.dyadic_rns(moduli, c1, sk))
        return self._add(moduli, ct[0], prod)

    def decrypt_plain(self, ct, correction=1):
        L = ct.shape[1]
        moduli = self.moduli[:L]
        ph = self.phase(ct)
        if self.scheme == BFV:
            return self.o.rns_op("decrypt_scale_round", self.n, moduli, self.t, ph, 1)[0]
        if self.scheme == BGV:
            p = self.o.rns_op("decrypt_mod_t", self.n, moduli, self.t, ph, 1)[0]
            if correction != 1:
                inv = pow(correction, -1, self.t)
                p = np.array([(int(x) * inv) % self.t for x in p], np.uint64)
            return p
        return ph

    def decrypt_slots(self, ct, correction=1):
        return self.decode_slots(self.decrypt_plain(ct, correction))

    # ----------------------------------------------------- element-wise
    def _add(self, moduli, a, b):
        a, b = np.ascontiguousarray(a, np.uint64), np.ascontiguousarray(b, np.uint64)
        out = np.zeros_like(a)
        self.o._f["poly_add"](np.asarray(moduli, np.uint64), len(moduli), self.n, a, b, out)
        return out

    def _neg(self, moduli, a):
        a = np.ascontiguousarray(a, np.uint64)
        out = np.zeros_like(a)
        self.o._f["poly_negate"](np.asarray(moduli, np.uint64), len(moduli), self.n, a, out)
        return out

    def _mul_scalar(self, moduli, a, s):
        a = np.ascontiguousarray(a, np.uint64)
        out = np.zeros_like(a)
        self.o._f["poly_mul_scalar"](np.asarray(moduli, np.uint64), len(moduli), self.n, a, int(s), out)
        return out


# ------------------------------------------------------------------ CKKS
def ckks_complex_roots(m: int):
    """ComplexRoots::getRoot table (src/utils/croots.cpp:10-59): e^(2 pi i k / m)."""
    k = np.arange(m)
    return np.exp(2j * np.pi * k / m)


class CkksCodec:
    """CKKSEncoder encode/decode (src/ckks.cpp:32-579) in FP64."""

    def __init__(self, n, moduli, o: Oracle | None = None):
        self.o = o or Oracle("orc")
        self.n, self.slots = n, n // 2
        self.logn = n.bit_length() - 1
        self.moduli = [int(x) for x in moduli]
        self.index_map = matrix_reps_index_map(n, self.slots)
        roots = ckks_complex_roots(2 * n)
        self.root_powers = np.zeros(n, np.complex128)
        self.inv_root_powers = np.zeros(n, np.complex128)
        for i in range(1, n):
            self.root_powers[i] = roots[_bitrev(i, self.logn)]
            self.inv_root_powers[i] = np.conj(roots[_bitrev(i - 1, self.logn) + 1])

    def _fft_from_rev(self, a, scalar):
        n = self.n
        gap, m, ridx = 1, n >> 1, 0
        a = a.copy()
        while m > 1:
            for i in range(m):
                ridx += 1
                r = self.inv_root_powers[ridx]
                off = 2 * gap * i
                u = a[off:off + gap].copy()
                v = a[off + gap:off + 2 * gap].copy()
                a[off:off + gap] = u + v
                a[off + gap:off + 2 * gap] = (u - v) * r
            m >>= 1
            gap <<= 1
        ridx += 1
        r = self.inv_root_powers[ridx] * scalar
        u = a[:gap].copy()
        v = a[gap:].copy()
        a[:gap] = (u + v) * scalar
        a[gap:] = (u - v) * r
        return a

    def _fft_to_rev(self, a):
        n = self.n
        gap, m, ridx = n >> 1, 1, 0
        a = a.copy()
        while m < n:
            for i in range(m):
                ridx += 1
                r = self.root_powers[ridx]
                off = 2 * gap * i
                u = a[off:off + gap].copy()
                v = a[off + gap:off + 2 * gap] * r
                a[off:off + gap] = u + v
                a[off + gap:off + 2 * gap] = u - v
            m <<= 1
            gap >>= 1
        return a

    def encode(self, values, scale, L):
        """Plaintext in NTT form at the level with L limbs."""
        n = self.n
        v = np.asarray(values, np.complex128)
        conj = np.zeros(n, np.complex128)
        conj[self.index_map[: len(v)]] = v
        conj[self.index_map[self.slots: self.slots + len(v)]] = np.conj(v)
        res = self._fft_from_rev(conj, scale / n)
        coeffs = [int(x) for x in np.round(res.real)]
        moduli = self.moduli[:L]
        out = np.zeros((L, n), np.uint64)
        for j, qj in enumerate(moduli):
            out[j] = [c % qj for c in coeffs]
        return self.o.ntt_forward_rns(self.logn, moduli, out)

    def decode(self, plain_ntt, scale):
        L = plain_ntt.shape[0]
        moduli = self.moduli[:L]
        coeff = self.o.ntt_inverse_rns(self.logn, moduli, plain_ntt)
        Q = 1
        for m in moduli:
            Q *= m
        vals = np.zeros(self.n, np.complex128)
        # CRT compose then centre (src/ckks.cpp:524-563)
        for i in range(self.n):
            x = 0
            for j, qj in enumerate(moduli):
                Qj = Q // qj
                x += int(coeff[j][i]) * Qj * pow(Qj % qj, -1, qj)
            x %= Q
            if x >= (Q + 1) >> 1:
                x -= Q
            vals[i] = float(x) / scale
        res = self._fft_to_rev(vals)
        return res[self.index_map[: self.slots]]

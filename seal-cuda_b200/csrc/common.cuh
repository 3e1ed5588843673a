// Shared device definitions: the per-modulus descriptor kept in HBM and the exact
// 64-bit modular arithmetic every kernel uses (CUDA cores, umulhi-based).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace tb {

// One NTT-friendly prime with everything the kernels need about it.
// roots[i] = psi^bitrev(i) (forward, bit-reversed order), inv_roots in the
// scrambled order of the Gentleman-Sande pass; each entry {operand, Shoup quotient}.
struct Mod {
    uint64_t value;
    uint64_t ratio_lo, ratio_hi;   // floor(2^128 / value)
    uint64_t inv_n, inv_n_quo;     // N^-1 mod value and its Shoup quotient
    uint64_t sroot, sroot_quo;     // last inverse-NTT root times N^-1, and its quotient
    const ulonglong2 *roots;
    const ulonglong2 *inv_roots;
};

__device__ __forceinline__ uint64_t mulhi(uint64_t a, uint64_t b) { return __umul64hi(a, b); }

// x * w mod q in [0, 2q) for any 64-bit x (Shoup; wq = floor(w 2^64 / q)).
__device__ __forceinline__ uint64_t mul_shoup_lazy(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) {
    return w * x - mulhi(x, wq) * q;
}

__device__ __forceinline__ uint64_t mul_shoup(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) {
    const uint64_t r = mul_shoup_lazy(x, w, wq, q);
    return min(r, r - q);
}

// x mod q for x < 2q (any x < q + 2^63): x - q wraps above x exactly when x < q, so the
// unsigned minimum picks the reduced value (a subtraction and a minimum, no compare
// and select).
__device__ __forceinline__ uint64_t csub(uint64_t x, uint64_t q) { return min(x, x - q); }

__device__ __forceinline__ uint64_t add_mod(uint64_t a, uint64_t b, uint64_t q) { return csub(a + b, q); }

__device__ __forceinline__ uint64_t sub_mod(uint64_t a, uint64_t b, uint64_t q) {
    return a >= b ? a - b : a + q - b;
}

__device__ __forceinline__ uint64_t neg_mod(uint64_t a, uint64_t q) { return a ? q - a : 0; }

// x mod q for any 64-bit x: the quotient estimate floor(x * floor(2^128/q) / 2^128)
// using only the high ratio word is off by at most one.
__device__ __forceinline__ uint64_t reduce64(uint64_t x, const Mod &m) {
    uint64_t qt = mulhi(x, m.ratio_hi);
    return csub(x - qt * m.value, m.value);
}

// (hi:lo) mod q for a 128-bit value: Barrett reduction with the 128-bit ratio;
// the truncated quotient is at most one below the true one.
__device__ __forceinline__ uint64_t reduce128(uint64_t hi, uint64_t lo, const Mod &m) {
    // quotient estimate: the high 64 bits of (hi:lo) * (ratio_hi:ratio_lo) / 2^64 over
    // the three partial products that reach them, carried in two multiply-add chains
    uint64_t qt;
    asm("{\n\t"
        ".reg .u64 c, t1, t3, t2;\n\t"
        "mul.hi.u64 c, %1, %3;\n\t"
        "mad.lo.cc.u64 t1, %1, %4, c;\n\t"
        "madc.hi.u64 t3, %1, %4, 0;\n\t"
        "mad.lo.cc.u64 t2, %2, %3, t1;\n\t"
        "madc.hi.u64 t3, %2, %3, t3;\n\t"
        "mad.lo.u64 %0, %2, %4, t3;\n\t"
        "}"
        : "=l"(qt)
        : "l"(lo), "l"(hi), "l"(m.ratio_lo), "l"(m.ratio_hi));
    return csub(lo - qt * m.value, m.value);
}

__device__ __forceinline__ uint64_t mul_mod(uint64_t a, uint64_t b, const Mod &m) {
    return reduce128(mulhi(a, b), a * b, m);
}

// (hi:lo) mod q for a value below 2^(2n+1), n the bit length of q (n <= 61): a product
// of two residues below q, or the sum of two such products. Barrett with one 64-bit
// quotient product instead of reduce128's three 128-bit ones: with s = n - 2,
// t = (hi:lo) >> s < 2^(n+3) <= 2^64 and mu = floor(2^(64+s) / q) = floor(2^128 / q) >>
// (64 - s) < 2^63, the estimate floor(t mu / 2^64) is never above floor(x / q) and at
// most 2 below it (it misses x / 2^(s+64) < 2^(n-61) <= 1, 2^s / q < 1/2 and the
// floors), so x - estimate * q lies in [0, 3q) and two conditional subtractions finish.
__device__ __forceinline__ uint64_t reduce_prod(uint64_t hi, uint64_t lo, const Mod &m) {
    const uint64_t q = m.value;
    const int s = 62 - __clzll((long long)q);
    const uint64_t t = s ? (lo >> s) | (hi << (64 - s)) : lo;
    const uint64_t mu = s ? (m.ratio_hi << s) | (m.ratio_lo >> (64 - s)) : m.ratio_hi;
    const uint64_t r = lo - mulhi(t, mu) * q;
    return csub(csub(r, 2 * q), q);
}

// a * b mod q for residues a, b < q.
__device__ __forceinline__ uint64_t mul_mod_canon(uint64_t a, uint64_t b, const Mod &m) {
    return reduce_prod(mulhi(a, b), a * b, m);
}

// 128-bit accumulator helpers for lazy inner products.
struct U128 {
    uint64_t lo, hi;
};

// acc += a * b: the low product word added with carry-out, the high word with the
// carry-in (extended-precision multiply-add, one carry chain).
__device__ __forceinline__ void mac128(U128 &acc, uint64_t a, uint64_t b) {
    asm("mad.lo.cc.u64 %0, %2, %3, %0;\n\t"
        "madc.hi.u64 %1, %2, %3, %1;"
        : "+l"(acc.lo), "+l"(acc.hi)
        : "l"(a), "l"(b));
}

// Layout helper: 64-bit coefficient index -> shared-memory slot. XOR-swizzling the
// low four index bits with the next four keeps every radix pass of the NTT and
// the contiguous copies free of bank conflicts.
__device__ __forceinline__ int swz(int e) { return e ^ ((e >> 4) & 15); }

}  // namespace tb

#define TB_CUDA_TRY(expr)                                 \
    do {                                                  \
        cudaError_t _e = (expr);                          \
        if (_e != cudaSuccess) return tb::status_from(_e); \
    } while (0)

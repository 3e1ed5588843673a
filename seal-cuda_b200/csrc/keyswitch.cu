// Batched key switching (relinearize, rotations / Galois automorphisms).
//
// Restates Evaluator::switchKeyInplace (src/evaluator.cpp:2310-2653): RNS digit
// decomposition with one digit per data limb and one special prime, per-digit
// NTT into every key modulus, inner product with the key, then division by the
// special prime with rounding ("mod-down") added into the ciphertext. A batch of
// ciphertexts goes through five launches:
//   1. (CKKS) inverse NTT of every target limb;
//   2. mod-up: one fused forward-NTT CTA per (ciphertext, digit j, key modulus i)
//      that takes digit j into key modulus i (unreduced, or reduced in its load) and
//      stores the transform's unreduced outputs;
//   3. inner product of the digits with both key components (lazy 128-bit sums) for
//      the data moduli;
//   4. inverse NTT of the special-prime accumulators, whose load runs the special
//      modulus's inner product, with the rounding offset;
//   5. mod-down: one fused NTT (CKKS) or inverse NTT (BFV/BGV) CTA per output limb
//      whose epilogue subtracts the special-prime part, scales by q_k^-1 and adds
//      into the ciphertext.
// Only exact residues matter between the steps, so the result is word-identical to
// the reference.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <string>

#include "context.hpp"
#include "hostmath.hpp"
#include "trace.cuh"

namespace tb {
size_t ks_scratch_budget();
bool ks_persistent();

unsigned grid_for(uint64_t work, int threads);

// Up to MAX_GROUPS key-switching keys in one batched launch: ciphertexts
// [first[g], first[g+1]) of the launch use key[g]. Passed by value as a kernel
// parameter, so no device-side descriptor upload is needed.
constexpr int MAX_GROUPS = 32;
struct KeyGroups {
    int count = 0;
    const uint64_t *key[MAX_GROUPS];
    uint32_t first[MAX_GROUPS + 1];
    __device__ __forceinline__ const uint64_t *of(uint32_t cb) const {
        int g = 0;
        while (g + 1 < count && cb >= first[g + 1]) g++;
        return key[g];
    }
    // The groups restricted to ciphertexts [b0, b0 + nb), rebased to start at 0.
    KeyGroups slice(uint32_t b0, uint32_t nb) const {
        KeyGroups r;
        for (int g = 0; g < count; g++) {
            const uint32_t lo = std::max(first[g], b0), hi = std::min(first[g + 1], b0 + nb);
            if (lo >= hi) continue;
            r.key[r.count] = key[g];
            r.first[r.count] = lo - b0;
            r.count++;
        }
        r.first[r.count] = nb;
        return r;
    }
};

// One shape of a multi-shape key switch: B ciphertexts of context c at level L, target
// [B][L][N] at target + b*tstride, ciphertext (2 polys, L limbs) at ct + b*cstride.
struct KsShape {
    const Context *c;
    int L;
    const uint64_t *target;
    uint64_t tstride;
    uint64_t *ct;
    uint64_t cstride;
    KeyGroups keys;
    uint64_t B;
};

namespace {

__device__ __forceinline__ uint64_t full_fwd(uint64_t v, uint64_t q) {
    return csub(csub(v, 2 * q), q);
}

// [0, q) from any value below 16 q (a forward transform with deferred reductions)
__device__ __forceinline__ uint64_t full_fwd16(uint64_t v, uint64_t q) {
    return full_fwd(csub(csub(v, 8 * q), 4 * q), q);
}

// [P][limbs] limbs at base + p*stride + l*N -> out + p*ostride + l*N.
template <bool FWD>
struct StridedNttOp {
    const uint64_t *in;
    uint64_t *out;
    uint64_t istride, ostride;
    const Mod *mods;
    int first, limbs, lazy, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
        int islack;   // full inverse outputs: the wide inverse form (outputs below 4q)
    };
    __device__ Ctx ctx(int b) const {
        const int p = b / limbs, l = b % limbs;
        Ctx c;
        c.lm = make_limb(mods[first + l], 0);
        c.islack = !FWD && !lazy;
        c.in = in + (size_t)p * istride + ((size_t)l << logn);
        c.out = out + (size_t)p * ostride + ((size_t)l << logn);
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const { return c.in[e]; }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ uint64_t fix(const Ctx &c, uint64_t v) const {
        if (lazy) return v;
        return FWD ? full_fwd(v, c.lm.q) : csub(csub(v, 2 * c.lm.q), c.lm.q);
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const { c.out[e] = fix(c, v); }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b) const {
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(fix(c, a), fix(c, b));
    }
};

// Step 2: forward NTT of digit j (coefficient form) into key modulus i. Only exact
// residues matter downstream (the inner product reduces its 128-bit sums), so the
// transform defers its reductions (ntt.cuh), takes the digit unreduced where its bound
// allows (or a Barrett remainder in [0, 2q)), and, while the sums stay below 2^128,
// the store keeps its unreduced outputs (bounds below).
struct ModUpOp {
    const uint64_t *src;      // CKKS: inverse-transformed targets [B][L][N]; else targets
    uint64_t sstride;         // words between ciphertexts in src
    uint64_t *digits;         // [B][L][L+1][N]
    const Mod *mods;
    const uint64_t *chain;    // device copy of chain values (for the reduce test)
    int L, K, ckks, logn;
    // Up to 15 digits are summed unreduced by the 128-bit inner products: below 4q (a
    // 61-bit q), below 16 q (q < 2^60, deferred reductions), or, for q < 2^57 in the
    // one-CTA transform (no subtraction, estimated quotients), below 2^61 + 56 q <
    // 2^63.2: the digit then enters unreduced (below q_j < 2^61) and the transform's 14
    // stages add at most 4q each. 15 products below 4 q * q < 2^124, 16 q * q < 2^124 or
    // 2^63.2 * 2^57 stay below 2^128. More digits are reduced to [0, q) at the store (the
    // transform then stays below 16 q).
    static constexpr int LAZY_MAX_L = 15;
    static constexpr bool wide_slack = true;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
        uint64_t ratio_hi;
        int reduce;
        int slack;
    };
    __device__ Ctx ctx(int b) const {
        const int P = ckks ? L * L : L * (L + 1);
        const int cb = b / P, p = b % P;
        int j, i;
        if (ckks) {
            j = p / L;
            const int ii = p % L;
            i = ii + (ii >= j);
        } else {
            j = p / (L + 1);
            i = p % (L + 1);
        }
        const int mi = i == L ? K - 1 : i;
        const Mod &m = mods[mi];
        Ctx c;
        c.lm = make_limb(m, 0);
        c.ratio_hi = m.ratio_hi;
        // the transform's input: any digit word in the no-subtraction form, below 4q in
        // the others (a Barrett remainder in [0, 2q) when q_j is larger)
        const bool wide = L <= LAZY_MAX_L && logn <= MAX_LOGB && m.value < (1ull << 57);
        c.slack = wide ? SLACK_WIDE : m.value < (1ull << 60) ? SLACK_M : 0;
        c.reduce = !wide && mods[j].value > 4 * m.value;
        c.in = src + (size_t)cb * sstride + ((size_t)j << logn);
        c.out = digits + ((((size_t)cb * L + j) * (L + 1) + i) << logn);
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const {
        const uint64_t x = c.in[e];
        if (!c.reduce) return x;
        return x - mulhi(x, c.ratio_hi) * c.lm.q;   // in [0, 2q)
    }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b) const {
        if (L > LAZY_MAX_L) {
            a = full_fwd16(a, c.lm.q);
            b = full_fwd16(b, c.lm.q);
        }
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(a, b);
    }
};

// Step 3: acc[b][c][i] = sum_j digit(b, j, i) * key[j][c][mi] mod q_mi, two coefficients
// (e, e+1) of output modulus i of ciphertext cb per thread.
__device__ __forceinline__ void ks_inner_pair(const uint64_t *__restrict__ digits, const uint64_t *__restrict__ target,
                                              uint64_t tstride, const KeyGroups &keys, uint64_t *__restrict__ acc,
                                              const Mod *__restrict__ mods, int L, int K, int ckks, int logn,
                                              uint32_t e, int i, size_t cb) {
    const int mi = i == L ? K - 1 : i;
    const Mod m = mods[mi];
    const uint64_t *__restrict__ key = keys.of((uint32_t)cb);
    U128 a00{0, 0}, a01{0, 0}, a10{0, 0}, a11{0, 0};
    // running pointers: digit j of output modulus i, and key digit j (polys 0 and 1) at mi
    const size_t dstep = (size_t)(L + 1) << logn, kstep = (size_t)(2 * K) << logn, kpoly = (size_t)K << logn;
    const uint64_t *d = digits + ((cb * L * (L + 1) + i) << logn) + e;
    const uint64_t *k = key + ((size_t)mi << logn) + e;
    for (int j = 0; j < L; j++, d += dstep, k += kstep) {
        const uint64_t *dj = (ckks && i == j) ? target + cb * tstride + ((size_t)j << logn) + e : d;
        const ulonglong2 dv = *reinterpret_cast<const ulonglong2 *>(dj);
        const ulonglong2 k0 = __ldg(reinterpret_cast<const ulonglong2 *>(k));
        const ulonglong2 k1 = __ldg(reinterpret_cast<const ulonglong2 *>(k + kpoly));
        mac128(a00, dv.x, k0.x);
        mac128(a01, dv.y, k0.y);
        mac128(a10, dv.x, k1.x);
        mac128(a11, dv.y, k1.y);
    }
    uint64_t *o0 = acc + (((cb * 2 + 0) * (L + 1) + i) << logn) + e;
    uint64_t *o1 = acc + (((cb * 2 + 1) * (L + 1) + i) << logn) + e;
    *reinterpret_cast<ulonglong2 *>(o0) = make_ulonglong2(reduce128(a00.hi, a00.lo, m), reduce128(a01.hi, a01.lo, m));
    *reinterpret_cast<ulonglong2 *>(o1) = make_ulonglong2(reduce128(a10.hi, a10.lo, m), reduce128(a11.hi, a11.lo, m));
}

constexpr int INNER_THREADS = 128;

__global__ void __launch_bounds__(INNER_THREADS, 8) ks_inner_kernel(const uint64_t *__restrict__ digits, const uint64_t *__restrict__ target,
                                uint64_t tstride, KeyGroups keys, uint64_t *__restrict__ acc,
                                const Mod *__restrict__ mods, int L, int K, int ckks, int logn) {
    const uint32_t e = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (e >= (1u << logn)) return;
    ks_inner_pair(digits, target, tstride, keys, acc, mods, L, K, ckks, logn, e, blockIdx.y, blockIdx.z);
}

// The inner products of several key-switch shapes (contexts of different degrees and
// levels) in one launch: blocks [first[g], first[g+1]) belong to shape g, laid out per
// ciphertext as (output modulus, coefficient chunk) like the grid of ks_inner_kernel.
struct InnerShape {
    const uint64_t *digits, *target;
    uint64_t tstride;
    KeyGroups keys;
    uint64_t *acc;
    const Mod *mods;
    int L, K, ckks, logn;
};

struct InnerTable {
    int count = 0;
    InnerShape sh[MAX_SHAPES];
    unsigned first[MAX_SHAPES + 1];
};

__global__ void __launch_bounds__(INNER_THREADS) ks_inner_shapes_kernel(InnerTable t) {
    int g = 0;
    while (g + 1 < t.count && blockIdx.x >= t.first[g + 1]) g++;
    const InnerShape &S = t.sh[g];
    const unsigned local = blockIdx.x - t.first[g];
    const unsigned chunks = ((1u << S.logn) / 2 + INNER_THREADS - 1) / INNER_THREADS;
    const unsigned per_ct = chunks * (unsigned)(S.L + 1);
    const unsigned cb = local / per_ct, r = local - cb * per_ct;
    const int i = (int)(r / chunks);
    const uint32_t e = 2 * ((r - (unsigned)i * chunks) * INNER_THREADS + threadIdx.x);
    if (e >= (1u << S.logn)) return;
    ks_inner_pair(S.digits, S.target, S.tstride, S.keys, S.acc, S.mods, S.L, S.K, S.ckks, S.logn, e, i, cb);
}

// Step 4: inverse NTT of the special-prime accumulator; CKKS/BFV add (q_k - 1)/2 for
// rounding (src/evaluator.cpp:2587-2596), BGV keeps the canonical residue.
struct SpecialInttOp {
    const uint64_t *acc;
    uint64_t *last;
    const Mod *mods;
    int L, K, bgv, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
    };
    __device__ Ctx ctx(int b) const {
        Ctx c;
        c.lm = make_limb(mods[K - 1], 0);
        c.in = acc + (((size_t)b * (L + 1) + L) << logn);
        c.out = last + ((size_t)b << logn);
        return c;
    }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const {
        const uint64_t q = c.lm.q;
        if (bgv) {
            c.out[e] = v >= q ? v - q : v;
        } else {
            uint64_t x = v + (q >> 1);
            x = x >= 2 * q ? x - 2 * q : x;
            c.out[e] = x >= q ? x - q : x;
        }
    }
};

// Steps 3 and 4 fused for the special prime: the inverse NTT whose load is the inner
// product itself, acc = sum_j digit(b, j, special) * key[j][c][K-1] (lazy 128-bit sums,
// one Barrett reduction), so the special-prime accumulator never goes through HBM;
// output as SpecialInttOp (rounding offset for CKKS/BFV, canonical for BGV).
struct SpecialInnerOp {
    const uint64_t *digits;   // [B][L][L+1][N]
    KeyGroups keys;
    uint64_t *last;           // [B][2][N]
    const Mod *mods;
    int L, K, bgv, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *d, *k;
        uint64_t *out;
        uint64_t ratio_lo, ratio_hi;
        int islack;   // the wide inverse form: outputs below 4q, reduced at the store
    };
    __device__ Ctx ctx(int b) const {
        const int cb = b >> 1, comp = b & 1;
        const Mod &m = mods[K - 1];
        Ctx c;
        c.lm = make_limb(m, 0);
        c.ratio_lo = m.ratio_lo;
        c.ratio_hi = m.ratio_hi;
        c.d = digits + (((size_t)cb * L * (L + 1) + L) << logn);
        c.k = keys.of((uint32_t)cb) + (((size_t)comp * K + K - 1) << logn);
        c.out = last + ((size_t)b << logn);
        c.islack = 1;
        return c;
    }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const size_t dstep = (size_t)(L + 1) << logn, kstep = (size_t)(2 * K) << logn;
        U128 s0{0, 0}, s1{0, 0};
        const uint64_t *d = c.d + e, *k = c.k + e;
        for (int j = 0; j < L; j++, d += dstep, k += kstep) {
            const ulonglong2 dv = *reinterpret_cast<const ulonglong2 *>(d);
            const ulonglong2 kv = __ldg(reinterpret_cast<const ulonglong2 *>(k));
            mac128(s0, dv.x, kv.x);
            mac128(s1, dv.y, kv.y);
        }
        Mod m;
        m.value = c.lm.q;
        m.ratio_lo = c.ratio_lo;
        m.ratio_hi = c.ratio_hi;
        a = reduce128(s0.hi, s0.lo, m);
        b = reduce128(s1.hi, s1.lo, m);
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const {
        const uint64_t q = c.lm.q;
        v = csub(v, 2 * q);   // [0, 2q) from the wide inverse form's [0, 4q)
        if (bgv) {
            c.out[e] = csub(v, q);
        } else {
            c.out[e] = csub(csub(v + (q >> 1), 2 * q), q);
        }
    }
};

struct ModDownBase {
    const uint64_t *acc;      // [B][2][L+1][N]
    const uint64_t *last;     // [B][2][N]
    uint64_t *ct;             // c0 at ct + b*cstride, c1 at + L*N
    uint64_t cstride;
    const Mod *mods;
    const DropC *drop;        // row for the special prime: drop[K*K + j]
    int L, K, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *acc;
        const uint64_t *last;
        uint64_t *ct;
        uint64_t ratio_hi;
        DropC d;
        int reduce;
        int slack;   // forward transform (CKKS) with deferred reductions
        uint64_t wide_off;   // (floor(2^64 / q_j) - 1) q_j: the epilogue's offset after the wide form
    };
    static constexpr bool wide_slack = true;
    __device__ Ctx make(int b) const {
        const int j = b % L, bc = b / L;  // bc = cb*2 + c
        const int cb = bc >> 1, cc = bc & 1;
        const Mod &m = mods[j];
        Ctx c;
        c.lm = make_limb(m, 0);
        c.ratio_hi = m.ratio_hi;
        c.d = drop[(size_t)K * K + j];
        c.reduce = mods[K - 1].value > m.value;
        c.slack = (logn <= MAX_LOGB && m.value < (1ull << 57)) ? SLACK_WIDE : m.value < (1ull << 60) ? SLACK_M : 0;
        c.wide_off = (m.ratio_hi - 1) * m.value;
        c.acc = acc + (((size_t)bc * (L + 1) + j) << logn);
        c.last = last + ((size_t)bc << logn);
        c.ct = ct + (size_t)cb * cstride + (((size_t)cc * L + j) << logn);
        return c;
    }
    // the special-prime residue r mod q_j: in [0, 2q) (lazy), or canonical
    __device__ uint64_t last_mod_lazy(const Ctx &c, int e) const {
        const uint64_t r = c.last[e];
        if (!c.reduce) return r;
        return r - mulhi(r, c.ratio_hi) * c.lm.q;
    }
    __device__ uint64_t last_mod(const Ctx &c, int e) const {
        const uint64_t x = last_mod_lazy(c, e);
        return x >= c.lm.q ? x - c.lm.q : x;
    }
};

// Step 5, CKKS: NTT of (r mod q_j) + fix, epilogue ct += (acc + 4 q_j - ntt) * q_k^-1.
// The transform's input only has to stay below 4 q_j: a lazy residue (< 2 q_j) plus fix
// (at most q_j). After the deferred-reduction form (ntt below 16 q_j) one subtraction of
// 8 q_j brings ntt below 8 q_j and the epilogue takes acc + 8 q_j - ntt: below 9 q_j <
// 2^64, where acc + 16 q_j - ntt would pass 2^64 for a 60-bit q_j. The no-subtraction
// form (q_j < 2^57, one CTA per limb) takes r itself (below 2^61) plus fix: ntt stays
// below 2^61 + 57 q_j < 2^63.2 < 2^64 - 2 q_j <= wide_off, and the epilogue takes
// acc + wide_off - ntt, below 2^64. The same residue each way.
struct ModDownCkksOp : ModDownBase {
    __device__ Ctx ctx(int b) const { return make(b); }
    __device__ uint64_t load(const Ctx &c, int e) const {
        return (c.slack == SLACK_WIDE ? c.last[e] : last_mod_lazy(c, e)) + c.d.fix;
    }
    // epilogue reads of a coefficient pair: the accumulator and the ciphertext limb
    struct Epi {
        ulonglong2 acc, ct;
    };
    __device__ Epi epi2(const Ctx &c, int e) const {
        return {*reinterpret_cast<const ulonglong2 *>(c.acc + e), *reinterpret_cast<const ulonglong2 *>(c.ct + e)};
    }
    __device__ uint64_t fin(const Ctx &c, uint64_t acc, uint64_t ct, uint64_t v) const {
        const uint64_t q = c.lm.q;
        const uint64_t x = c.slack == SLACK_WIDE ? acc + c.wide_off - v
                           : c.slack ? acc + (q << 3) - csub(v, q << 3) : acc + (q << 2) - v;
        return add_mod(mul_shoup(x, c.d.inv, c.d.inv_quo, q), ct, q);
    }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b, const Epi &p) const {
        *reinterpret_cast<ulonglong2 *>(c.ct + e) = make_ulonglong2(fin(c, p.acc.x, p.ct.x, a), fin(c, p.acc.y, p.ct.y, b));
    }
};

// Step 5, BFV: inverse NTT of acc, epilogue ct += (intt + 2 q_j - ((r mod q_j) + fix)) * q_k^-1.
struct ModDownBfvOp : ModDownBase {
    __device__ Ctx ctx(int b) const { return make(b); }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.acc + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const {
        const uint64_t q = c.lm.q;
        const uint64_t t = last_mod(c, e) + c.d.fix;
        const uint64_t x = v + 2 * q - t;
        c.ct[e] = add_mod(mul_shoup(x, c.d.inv, c.d.inv_quo, q), c.ct[e], q);
    }
};

// Step 5, BGV (src/evaluator.cpp:2528-2583): k = -(r mod t) q_k^-1 mod t,
// ct += (intt + 2 q_j - (k q_k mod q_j + r mod q_j)) * q_k^-1.
struct ModDownBgvOp : ModDownBase {
    Mod tm;
    uint64_t inv_qk_t;
    __device__ Ctx ctx(int b) const { return make(b); }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.acc + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const {
        const uint64_t q = c.lm.q;
        const uint64_t r = c.last[e];
        uint64_t k = neg_mod(reduce64(r, tm), tm.value);
        if (inv_qk_t != 1) k = mul_mod(k, inv_qk_t, tm);
        const uint64_t kq = k - mulhi(k, c.ratio_hi) * q;
        const uint64_t delta = mul_shoup(kq >= q ? kq - q : kq, c.d.lastmod, c.d.lastmod_quo, q);
        const uint64_t x = v + 2 * q - (delta + last_mod(c, e));
        c.ct[e] = add_mod(mul_shoup(x, c.d.inv, c.d.inv_quo, q), c.ct[e], q);
    }
};

}  // namespace

// Per-context device scratch is taken from the stream-ordered pool of the device.
struct Scratch {
    void *p = nullptr;
    cudaStream_t s;
    explicit Scratch(cudaStream_t st) : s(st) {}
    cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes, s); }
    ~Scratch() {
        if (p) cudaFreeAsync(p, s);
    }
};

void ensure_pool_retains(int device);

int keyswitch_shapes(const KsShape *shapes, int count, cudaStream_t s);

// target[b] (L limbs) at target + b*tstride; ct[b] (2 polys, L limbs) at ct + b*cstride.
int keyswitch_groups(const Context &c, int L, const uint64_t *target, uint64_t tstride, uint64_t *ct,
                     uint64_t cstride, const KeyGroups &keys, uint64_t B, cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a scheme context");
    if (K < 2) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a special prime");
    if (L < 1 || L > K - 1) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the data chain");
    if (c.logn > MAX_FUSED_LOGN) return set_error(TB_ERR_UNSUPPORTED, "fused key switching supports N <= 131072");
    if (!target || !ct || keys.count < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    for (int g = 0; g < keys.count; g++)
        if (!keys.key[g]) return set_error(TB_ERR_NO_KEY, "missing key-switching key");
    if (B == 0) return TB_OK;
    const uint64_t n = c.n;
    if (!tstride) tstride = (uint64_t)L * n;
    if (!cstride) cstride = 2ull * L * n;
    const bool ckks = c.scheme == SCHEME_CKKS;
    const int pairs = ckks ? L * L : L * (L + 1);
    const size_t per_ct = ((ckks ? (size_t)L : 0) + (size_t)L * (L + 1) + 2ull * (L + 1) + 2) * n * 8;
    // Whole batches per launch keep every stage's grid several waves deep; the batch is
    // only split when its intermediates would exceed the scratch budget.
    const size_t budget = ks_scratch_budget();
    if (ks_persistent() && c.logn >= 12 && c.logn <= MAX_LOGB && per_ct * B <= budget &&
        B <= 0x7fffffffull / ((uint64_t)L * (L + 1))) {
        const KsShape sh{&c, L, target, tstride, ct, cstride, keys, B};
        return keyswitch_shapes(&sh, 1, s);
    }
    uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(B, budget / per_ct));
    ensure_pool_retains(c.device);
    Scratch scr(s);
    cudaError_t e = scr.alloc(per_ct * chunk);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *base = (uint64_t *)scr.p;
    uint64_t *tgt = base;
    uint64_t *digits = tgt + (ckks ? chunk * L * n : 0);
    uint64_t *acc = digits + chunk * (uint64_t)L * (L + 1) * n;
    uint64_t *last = acc + chunk * 2ull * (L + 1) * n;
    const int logn = c.logn;
    for (uint64_t b0 = 0; b0 < B; b0 += chunk) {
        const uint64_t nb = std::min(chunk, B - b0);
        const uint64_t *tg = target + b0 * tstride;
        uint64_t *cc = ct + b0 * cstride;
        if (ckks) {
            StridedNttOp<false> op{tg, tgt, tstride, (uint64_t)L * n, c.d_mods, 0, L, 0, logn};
            TraceScope ts("ks_target_intt", s);
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * L), logn, 1, s);
            if (e != cudaSuccess) return status_from(e);
        }
        ModUpOp mu{ckks ? tgt : tg, ckks ? (uint64_t)L * n : tstride, digits, c.d_mods, nullptr, L, K, ckks, logn};
        {
            TraceScope ts("ks_modup_ntt", s);
            e = dispatch_ntt<true>(logn, mu, (unsigned)(nb * pairs), 0, 0, s);
        }
        if (e != cudaSuccess) return status_from(e);
        // the data moduli's inner products; the special prime's runs inside its inverse NTT
        const int threads = INNER_THREADS;
        const KeyGroups kslice = keys.slice((uint32_t)b0, (uint32_t)nb);
        dim3 grid((unsigned)((n / 2 + threads - 1) / threads), L, (unsigned)nb);
        {
            TraceScope ts("ks_inner_product", s);
            ks_inner_kernel<<<grid, threads, 0, s>>>(digits, tg, tstride, kslice, acc, c.d_mods, L, K, ckks, logn);
            e = cudaGetLastError();
        }
        if (e != cudaSuccess) return status_from(e);
        SpecialInnerOp si{digits, kslice, last, c.d_mods, L, K, c.scheme == SCHEME_BGV, logn};
        {
            TraceScope ts("ks_special_intt", s);
            e = dispatch_ntt<false>(logn, si, (unsigned)(nb * 2), logn, 1, s);
        }
        if (e != cudaSuccess) return status_from(e);
        ModDownBase mb{acc, last, cc, cstride, c.d_mods, c.d_drop, L, K, logn};
        TraceScope ts("ks_moddown", s);
        if (ckks) {
            ModDownCkksOp op{mb};
            e = dispatch_ntt<true>(logn, op, (unsigned)(nb * 2 * L), 0, 0, s);
        } else if (c.scheme == SCHEME_BFV) {
            ModDownBfvOp op{mb};
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * 2 * L), logn, 1, s);
        } else {
            ModDownBgvOp op{mb, c.t_mod, c.inv_qlast_t[K]};
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * 2 * L), logn, 1, s);
        }
        if (e != cudaSuccess) return status_from(e);
    }
    return TB_OK;
}

// ------------------------------------------------- several shapes in one launch per step
//
// Key switching of ciphertexts of several contexts (ring degrees 2^12 .. 2^14, any
// levels, any of the three schemes) with one persistent launch per step for all of
// them: the CKKS target inverse transforms, every mod-up transform, every inner
// product, every special-prime inverse transform, and the mod-downs (one launch per
// scheme present: the CKKS mod-down is a forward transform, BFV's and BGV's inverse
// ones with different epilogues). Same operations, same words as keyswitch_groups per
// shape.
int keyswitch_shapes(const KsShape *shapes, int count, cudaStream_t s) {
    if (count < 1 || count > MAX_SHAPES) return set_error(TB_ERR_INVALID_ARGUMENT, "between 1 and 8 shapes");
    size_t bytes = 0;
    for (int g = 0; g < count; g++) {
        const KsShape &sh = shapes[g];
        const Context &c = *sh.c;
        const int K = (int)c.chain.size(), L = sh.L;
        if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a scheme context");
        if (K < 2) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a special prime");
        if (L < 1 || L > K - 1) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the data chain");
        if (c.logn < 12 || c.logn > MAX_LOGB)
            return set_error(TB_ERR_UNSUPPORTED, "one-launch key switching takes degrees 4096 .. 16384");
        if (!sh.target || !sh.ct || sh.keys.count < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
        for (int k = 0; k < sh.keys.count; k++)
            if (!sh.keys.key[k]) return set_error(TB_ERR_NO_KEY, "missing key-switching key");
        if (sh.B > 0x7fffffffull / ((uint64_t)L * (L + 1))) return set_error(TB_ERR_INVALID_ARGUMENT, "batch too large");
        const bool ckks = c.scheme == SCHEME_CKKS;
        bytes += ((ckks ? (size_t)L : 0) + (size_t)L * (L + 1) + 2ull * (L + 1) + 2) * c.n * 8 * sh.B;
    }
    ensure_pool_retains(shapes[0].c->device);
    Scratch scr(s);
    cudaError_t e = scr.alloc(bytes + 256);
    if (e != cudaSuccess) return status_from(e);
    unsigned *counter = (unsigned *)scr.p;
    uint64_t *at = (uint64_t *)((char *)scr.p + 256);
    // largest degree first: the cheap limbs of small rings fill the last round
    int order[MAX_SHAPES];
    for (int g = 0; g < count; g++) order[g] = g;
    std::stable_sort(order, order + count, [&](int a, int b) { return shapes[a].c->logn > shapes[b].c->logn; });
    struct Bufs {
        uint64_t *tgt, *digits, *acc, *last;
    } buf[MAX_SHAPES];
    for (int k = 0; k < count; k++) {
        const KsShape &sh = shapes[order[k]];
        const uint64_t n = sh.c->n, L = (uint64_t)sh.L;
        const bool ckks = sh.c->scheme == SCHEME_CKKS;
        buf[k].tgt = at;
        buf[k].digits = buf[k].tgt + (ckks ? sh.B * L * n : 0);
        buf[k].acc = buf[k].digits + sh.B * L * (L + 1) * n;
        buf[k].last = buf[k].acc + sh.B * 2 * (L + 1) * n;
        at = buf[k].last + sh.B * 2 * n;
    }
    // 1. CKKS targets out of the NTT domain
    {
        ShapeTable<StridedNttOp<false>> t;
        unsigned f = 0;
        for (int k = 0; k < count; k++) {
            const KsShape &sh = shapes[order[k]];
            if (sh.c->scheme != SCHEME_CKKS || !sh.B) continue;
            const uint64_t tstride = sh.tstride ? sh.tstride : (uint64_t)sh.L * sh.c->n;
            t.op[t.count] = StridedNttOp<false>{sh.target, buf[k].tgt, tstride, (uint64_t)sh.L * sh.c->n,
                                                sh.c->d_mods, 0, sh.L, 0, sh.c->logn};
            t.logn[t.count] = sh.c->logn;
            t.first[t.count] = f;
            f += (unsigned)(sh.B * sh.L);
            t.count++;
        }
        t.first[t.count] = f;
        if (t.count) {
            TraceScope ts("ks_target_intt", s);
            e = launch_shapes<false>(t, counter, s);
            if (e != cudaSuccess) return status_from(e);
        }
    }
    // 2. mod-up transforms
    {
        ShapeTable<ModUpOp> t;
        unsigned f = 0;
        for (int k = 0; k < count; k++) {
            const KsShape &sh = shapes[order[k]];
            if (!sh.B) continue;
            const bool ckks = sh.c->scheme == SCHEME_CKKS;
            const uint64_t tstride = sh.tstride ? sh.tstride : (uint64_t)sh.L * sh.c->n;
            t.op[t.count] = ModUpOp{ckks ? buf[k].tgt : sh.target, ckks ? (uint64_t)sh.L * sh.c->n : tstride,
                                    buf[k].digits, sh.c->d_mods, nullptr, sh.L, (int)sh.c->chain.size(), ckks ? 1 : 0,
                                    sh.c->logn};
            t.logn[t.count] = sh.c->logn;
            t.first[t.count] = f;
            f += (unsigned)(sh.B * (ckks ? sh.L * sh.L : sh.L * (sh.L + 1)));
            t.count++;
        }
        t.first[t.count] = f;
        if (t.count) {
            TraceScope ts("ks_modup_ntt", s);
            e = launch_shapes<true>(t, counter, s);
            if (e != cudaSuccess) return status_from(e);
        }
    }
    // 3. inner products
    {
        InnerTable t;
        unsigned f = 0;
        for (int k = 0; k < count; k++) {
            const KsShape &sh = shapes[order[k]];
            if (!sh.B) continue;
            const uint64_t tstride = sh.tstride ? sh.tstride : (uint64_t)sh.L * sh.c->n;
            t.sh[t.count] = InnerShape{buf[k].digits, sh.target, tstride, sh.keys, buf[k].acc, sh.c->d_mods, sh.L,
                                       (int)sh.c->chain.size(), sh.c->scheme == SCHEME_CKKS ? 1 : 0, sh.c->logn};
            t.first[t.count] = f;
            const unsigned chunks = (sh.c->n / 2 + INNER_THREADS - 1) / INNER_THREADS;
            f += (unsigned)(sh.B * (sh.L + 1)) * chunks;
            t.count++;
        }
        t.first[t.count] = f;
        if (t.count && f) {
            TraceScope ts("ks_inner_product", s);
            ks_inner_shapes_kernel<<<f, INNER_THREADS, 0, s>>>(t);
            e = cudaGetLastError();
            if (e != cudaSuccess) return status_from(e);
        }
    }
    // 4. special-prime accumulators out of the NTT domain
    {
        ShapeTable<SpecialInttOp> t;
        unsigned f = 0;
        for (int k = 0; k < count; k++) {
            const KsShape &sh = shapes[order[k]];
            if (!sh.B) continue;
            t.op[t.count] = SpecialInttOp{buf[k].acc, buf[k].last, sh.c->d_mods, sh.L, (int)sh.c->chain.size(),
                                          sh.c->scheme == SCHEME_BGV ? 1 : 0, sh.c->logn};
            t.logn[t.count] = sh.c->logn;
            t.first[t.count] = f;
            f += (unsigned)(sh.B * 2);
            t.count++;
        }
        t.first[t.count] = f;
        if (t.count) {
            TraceScope ts("ks_special_intt", s);
            e = launch_shapes<false>(t, counter, s);
            if (e != cudaSuccess) return status_from(e);
        }
    }
    // 5. mod-down into the ciphertexts, one launch per scheme present
    TraceScope ts("ks_moddown", s);
    ShapeTable<ModDownCkksOp> tc;
    ShapeTable<ModDownBfvOp> tf;
    ShapeTable<ModDownBgvOp> tg;
    unsigned fc = 0, ff = 0, fg = 0;
    for (int k = 0; k < count; k++) {
        const KsShape &sh = shapes[order[k]];
        if (!sh.B) continue;
        const Context &c = *sh.c;
        const int K = (int)c.chain.size();
        const uint64_t cstride = sh.cstride ? sh.cstride : 2ull * sh.L * c.n;
        const ModDownBase mb{buf[k].acc, buf[k].last, sh.ct, cstride, c.d_mods, c.d_drop, sh.L, K, c.logn};
        const unsigned limbs = (unsigned)(sh.B * 2 * sh.L);
        if (c.scheme == SCHEME_CKKS) {
            tc.op[tc.count] = ModDownCkksOp{mb};
            tc.logn[tc.count] = c.logn;
            tc.first[tc.count++] = fc;
            fc += limbs;
        } else if (c.scheme == SCHEME_BFV) {
            tf.op[tf.count] = ModDownBfvOp{mb};
            tf.logn[tf.count] = c.logn;
            tf.first[tf.count++] = ff;
            ff += limbs;
        } else {
            tg.op[tg.count] = ModDownBgvOp{mb, c.t_mod, c.inv_qlast_t[K]};
            tg.logn[tg.count] = c.logn;
            tg.first[tg.count++] = fg;
            fg += limbs;
        }
    }
    tc.first[tc.count] = fc;
    tf.first[tf.count] = ff;
    tg.first[tg.count] = fg;
    if (tc.count && (e = launch_shapes<true>(tc, counter, s)) != cudaSuccess) return status_from(e);
    if (tf.count && (e = launch_shapes<false>(tf, counter, s)) != cudaSuccess) return status_from(e);
    if (tg.count && (e = launch_shapes<false>(tg, counter, s)) != cudaSuccess) return status_from(e);
    return TB_OK;
}

int keyswitch(const Context &c, int L, const uint64_t *target, uint64_t tstride, uint64_t *ct, uint64_t cstride,
              const uint64_t *key, uint64_t B, cudaStream_t s) {
    KeyGroups kg;
    kg.count = 1;
    kg.key[0] = key;
    kg.first[0] = 0;
    kg.first[1] = (uint32_t)B;
    return keyswitch_groups(c, L, target, tstride, ct, cstride, kg, B, s);
}

// ------------------------------------------------------------------ Galois

namespace {

// Coefficient-domain X -> X^elt with the negacyclic sign (GaloisTool::applyGalois,
// src/utils/galois.cpp:143-165): c0 -> out c0, c1 -> target, out c1 cleared.
struct GaloisGroups {
    int count = 0;
    uint32_t elt[MAX_GROUPS];
    const uint32_t *perm[MAX_GROUPS];
    uint32_t first[MAX_GROUPS + 1];
    __device__ __forceinline__ int of(uint32_t cb) const {
        int g = 0;
        while (g + 1 < count && cb >= first[g + 1]) g++;
        return g;
    }
};

__global__ void galois_coeff_kernel(const uint64_t *__restrict__ in, uint64_t istride, uint64_t *__restrict__ out0,
                                    uint64_t ostride, uint64_t *__restrict__ tgt, uint64_t tstride,
                                    uint64_t *__restrict__ out1, const Mod *__restrict__ mods, int L, int logn,
                                    GaloisGroups gg) {
    const uint32_t n = 1u << logn;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = blockIdx.y;
    const size_t cb = blockIdx.z;
    const uint32_t elt = gg.elt[gg.of((uint32_t)cb)];
    const uint64_t q = mods[j].value;
    const uint64_t raw = (uint64_t)i * elt;
    const uint32_t idx = (uint32_t)(raw & (n - 1));
    const bool neg = (raw >> logn) & 1;
    const uint64_t *src = in + cb * istride + ((size_t)j << logn);
    uint64_t v0 = src[i], v1 = src[((size_t)L << logn) + i];
    if (neg) {
        v0 = neg_mod(v0, q);
        v1 = neg_mod(v1, q);
    }
    out0[cb * ostride + ((size_t)j << logn) + idx] = v0;
    tgt[cb * tstride + ((size_t)j << logn) + idx] = v1;
    out1[cb * ostride + ((size_t)j << logn) + i] = 0;
}

// NTT-domain permutation (GaloisTool::applyGaloisNtt, src/utils/galois.cpp:167-177).
__global__ void galois_ntt_kernel(const uint64_t *__restrict__ in, uint64_t istride, uint64_t *__restrict__ out0,
                                  uint64_t ostride, uint64_t *__restrict__ tgt, uint64_t tstride,
                                  uint64_t *__restrict__ out1, GaloisGroups gg, int L, int logn) {
    const uint32_t n = 1u << logn;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = blockIdx.y;
    const size_t cb = blockIdx.z;
    const uint32_t *__restrict__ perm = gg.perm[gg.of((uint32_t)cb)];
    const uint32_t p = __ldg(&perm[i]);
    const uint64_t *src = in + cb * istride + ((size_t)j << logn);
    out0[cb * ostride + ((size_t)j << logn) + i] = src[p];
    tgt[cb * tstride + ((size_t)j << logn) + i] = src[((size_t)L << logn) + p];
    out1[cb * ostride + ((size_t)j << logn) + i] = 0;
}

}  // namespace

// Device permutation table of an element, built and uploaded on first use
// (GaloisTool::generateTableNtt, src/utils/galois.cpp:18-43).
int galois_ntt_table(Context &c, uint32_t elt, const uint32_t **out) {
    std::lock_guard<std::mutex> g(c.galois_mu);
    auto it = c.galois_ntt.find(elt);
    if (it != c.galois_ntt.end()) {
        *out = it->second;
        return TB_OK;
    }
    const uint32_t n = c.n;
    std::vector<uint32_t> t(n);
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t rev = host::bitrev(n + i, c.logn + 1);
        uint64_t raw = ((uint64_t)elt * rev) >> 1;
        raw &= (uint64_t)(n - 1);
        t[i] = host::bitrev((uint32_t)raw, c.logn);
    }
    uint32_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, n * 4);
    if (e == cudaSuccess) e = cudaMemcpy(d, t.data(), n * 4, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        if (d) cudaFree(d);
        return status_from(e);
    }
    c.galois_ntt[elt] = d;
    *out = d;
    return TB_OK;
}

// Groups of ciphertexts, group g rotated by elts[g] and key-switched with keys[g]
// (Evaluator::applyGaloisInplace, src/evaluator.cpp:2153-2249, batched over many
// elements): ciphertexts of group g follow those of group g-1 in `in` / `out`.
int apply_galois_groups(Context &c, int L, int groups, const uint32_t *elts, const uint64_t *counts,
                        const uint64_t *in, uint64_t istride, uint64_t *out, uint64_t ostride,
                        const uint64_t *const *keys, cudaStream_t s) {
    const uint32_t n = c.n;
    if (L < 1 || L > (int)c.chain.size() - 1) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the data chain");
    if (!in || !out || !elts || !counts || !keys || groups < 1)
        return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!istride) istride = 2ull * L * n;
    if (!ostride) ostride = 2ull * L * n;
    uint64_t B = 0;
    for (int g = 0; g < groups; g++) {
        if (!(elts[g] & 1) || elts[g] >= 2 * n) return set_error(TB_ERR_INVALID_ARGUMENT, "Galois element is not valid");
        if (!keys[g]) return set_error(TB_ERR_NO_KEY, "Galois key not present");
        B += counts[g];
    }
    if (B == 0) return TB_OK;
    if (groups > MAX_GROUPS) {
        // split into launches of at most MAX_GROUPS groups
        uint64_t done = 0;
        for (int g0 = 0; g0 < groups; g0 += MAX_GROUPS) {
            const int gc = std::min(MAX_GROUPS, groups - g0);
            uint64_t cnt = 0;
            for (int g = g0; g < g0 + gc; g++) cnt += counts[g];
            int st = apply_galois_groups(c, L, gc, elts + g0, counts + g0, in + done * istride, istride,
                                         out + done * ostride, ostride, keys + g0, s);
            if (st != TB_OK) return st;
            done += cnt;
        }
        return TB_OK;
    }
    if (B > 65535) return set_error(TB_ERR_INVALID_ARGUMENT, "at most 65535 ciphertexts per call");
    GaloisGroups gg;
    KeyGroups kg;
    gg.count = kg.count = groups;
    uint32_t f = 0;
    for (int g = 0; g < groups; g++) {
        gg.elt[g] = elts[g];
        gg.perm[g] = nullptr;
        if (c.scheme == SCHEME_CKKS) {
            int st = galois_ntt_table(c, elts[g], &gg.perm[g]);
            if (st != TB_OK) return st;
        }
        gg.first[g] = kg.first[g] = f;
        kg.key[g] = keys[g];
        f += (uint32_t)counts[g];
    }
    gg.first[groups] = kg.first[groups] = f;
    const bool inplace = out < in + B * istride && in < out + B * ostride;
    ensure_pool_retains(c.device);
    Scratch scr(s);
    const uint64_t tstride = (uint64_t)L * n;
    const uint64_t ostride_w = inplace ? 2ull * L * n : ostride;
    cudaError_t e = scr.alloc(B * tstride * 8 + (inplace ? B * 2ull * L * n * 8 : 0));
    if (e != cudaSuccess) return status_from(e);
    uint64_t *tgt = (uint64_t *)scr.p;
    uint64_t *dst = inplace ? tgt + B * tstride : out;
    dim3 grid((n + 255) / 256, L, (unsigned)B);
    {
        TraceScope ts("galois_permute", s);
        if (c.scheme == SCHEME_CKKS)
            galois_ntt_kernel<<<grid, 256, 0, s>>>(in, istride, dst, ostride_w, tgt, tstride, dst + (size_t)L * n, gg,
                                                   L, c.logn);
        else
            galois_coeff_kernel<<<grid, 256, 0, s>>>(in, istride, dst, ostride_w, tgt, tstride, dst + (size_t)L * n,
                                                     c.d_mods, L, c.logn, gg);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return status_from(e);
    int st = keyswitch_groups(c, L, tgt, tstride, dst, ostride_w, kg, B, s);
    if (st != TB_OK) return st;
    if (inplace) {
        e = cudaMemcpy2DAsync(out, ostride * 8, dst, ostride_w * 8, 2ull * L * n * 8, B, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return status_from(e);
    }
    return TB_OK;
}

// The relinearize -> rotate part of an uneven batch with every key-switch step in one
// launch for all shapes: t3[g] holds shape g's B products ([B][3][L][n]); they are
// relinearized in place (one keyswitch_shapes), each shape's Galois permutation writes
// out[g] (c0 permuted, c1 cleared) and its permuted c1 into scratch, and one more
// keyswitch_shapes adds the rotation key switch into out[g] (applyGaloisInplace,
// src/evaluator.cpp:2153-2249, for every shape at once).
int uneven_relin_rotate(Context *const *ctxs, const int *Ls, const uint64_t *Bs, uint64_t *const *t3,
                        const uint64_t *const *rlks, const uint64_t *const *gks, const uint32_t *elts,
                        uint64_t *const *outs, int count, cudaStream_t s) {
    if (count < 1 || count > MAX_SHAPES) return set_error(TB_ERR_INVALID_ARGUMENT, "between 1 and 8 shapes");
    KsShape sh[MAX_SHAPES];
    uint64_t words = 0;
    for (int g = 0; g < count; g++) {
        const uint64_t n = ctxs[g]->n, L = (uint64_t)Ls[g];
        KeyGroups kg;
        kg.count = 1;
        kg.key[0] = rlks[g];
        kg.first[0] = 0;
        kg.first[1] = (uint32_t)Bs[g];
        sh[g] = KsShape{ctxs[g], Ls[g], t3[g] + 2 * L * n, 3 * L * n, t3[g], 3 * L * n, kg, Bs[g]};
        words += Bs[g] * L * n;
    }
    int st = keyswitch_shapes(sh, count, s);
    if (st != TB_OK) return st;
    ensure_pool_retains(ctxs[0]->device);
    Scratch scr(s);
    cudaError_t e = scr.alloc(words * 8);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *tgt = (uint64_t *)scr.p;
    {
        TraceScope ts("galois_permute", s);
        for (int g = 0; g < count; g++) {
            Context &c = *ctxs[g];
            const uint64_t n = c.n, L = (uint64_t)Ls[g];
            GaloisGroups gg;
            gg.count = 1;
            gg.elt[0] = elts[g];
            gg.perm[0] = nullptr;
            gg.first[0] = 0;
            gg.first[1] = (uint32_t)Bs[g];
            if (c.scheme == SCHEME_CKKS) {
                st = galois_ntt_table(c, elts[g], &gg.perm[0]);
                if (st != TB_OK) return st;
            }
            dim3 grid((unsigned)((n + 255) / 256), (unsigned)L, (unsigned)Bs[g]);
            if (c.scheme == SCHEME_CKKS)
                galois_ntt_kernel<<<grid, 256, 0, s>>>(t3[g], 3 * L * n, outs[g], 2 * L * n, tgt, L * n,
                                                       outs[g] + L * n, gg, (int)L, c.logn);
            else
                galois_coeff_kernel<<<grid, 256, 0, s>>>(t3[g], 3 * L * n, outs[g], 2 * L * n, tgt, L * n,
                                                         outs[g] + L * n, c.d_mods, (int)L, c.logn, gg);
            e = cudaGetLastError();
            if (e != cudaSuccess) return status_from(e);
            KeyGroups kg;
            kg.count = 1;
            kg.key[0] = gks[g];
            kg.first[0] = 0;
            kg.first[1] = (uint32_t)Bs[g];
            sh[g] = KsShape{ctxs[g], Ls[g], tgt, L * n, outs[g], 2 * L * n, kg, Bs[g]};
            tgt += Bs[g] * L * n;
        }
    }
    return keyswitch_shapes(sh, count, s);
}

int apply_galois(Context &c, int L, uint32_t elt, const uint64_t *in, uint64_t istride, uint64_t *out,
                 uint64_t ostride, const uint64_t *key, uint64_t B, cudaStream_t s) {
    const uint64_t *keys[1] = {key};
    return apply_galois_groups(c, L, 1, &elt, &B, in, istride, out, ostride, keys, s);
}

// ------------------------------------------------- allocation-free relinearize
//
// Some callers cannot allocate device memory when they relinearize: a serving loop
// that has budgeted every byte of HBM up front and must neither stall on the
// allocator nor fail a request half-way with an out-of-memory error, or code that
// runs while another allocator owns the device's free memory. For them
// tb_relinearize_noalloc works out of a fixed scratch array that lives in the
// library's device image: every GPU that loads the library holds these
// TB_NOALLOC_SCRATCH_BYTES until the process exits. A batch is processed in as many
// ciphertexts at a time as fit; a single ciphertext that needs more than the array
// holds is rejected. Every call shares the one array, so calls that overlap on the
// GPU (different streams, or different host threads) race on it and must be
// serialised by the caller. No word of the scratch needs to start at zero: each word
// a call reads was written earlier in that same call.

constexpr size_t TB_NOALLOC_SCRATCH_BYTES = 16ull << 20;  // 16 MiB: one L=8, N=16384 CKKS ciphertext
static __device__ __align__(256) uint64_t g_noalloc_scratch[TB_NOALLOC_SCRATCH_BYTES / 8];

// Device address of g_noalloc_scratch on the current device. In host code the
// array's name only stands in for the symbol, so the address is asked for while a
// context is created (its device current) and kept in the context. With lazy module
// loading this lookup is what loads the library's device image, array included, on
// that device: the 16 MiB are taken at context creation, never inside a relinearize
// call, and a context created after a device reset gets the new address.
int noalloc_scratch_address(uint64_t **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return status_from(e);
    *out = (uint64_t *)p;
    return TB_OK;
}

int relinearize_noalloc(const Context &c, int L, uint64_t *ct3, uint64_t cstride, const uint64_t *key, uint64_t B,
                        cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a scheme context");
    if (K < 2) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a special prime");
    if (L < 1 || L > K - 1) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the data chain");
    if (c.logn > MAX_FUSED_LOGN) return set_error(TB_ERR_UNSUPPORTED, "fused key switching supports N <= 131072");
    if (!ct3 || !key) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (B == 0) return TB_OK;
    const uint64_t n = c.n;
    if (!cstride) cstride = 3ull * L * n;
    const bool ckks = c.scheme == SCHEME_CKKS;
    const int pairs = ckks ? L * L : L * (L + 1);
    const size_t per_ct = ((ckks ? (size_t)L : 0) + (size_t)L * (L + 1) + 2ull * (L + 1) + 2) * n * 8;
    if (per_ct > TB_NOALLOC_SCRATCH_BYTES)
        return set_error(TB_ERR_INVALID_ARGUMENT,
                         "relinearize without allocation needs " + std::to_string(per_ct) +
                             " bytes of scratch for one ciphertext at this level; the static scratch holds " +
                             std::to_string(TB_NOALLOC_SCRATCH_BYTES) + " bytes");
    uint64_t *base = c.noalloc_scratch;
    if (!base) return set_error(TB_ERR_CUDA, "static relinearize scratch not found on this device");
    const uint64_t chunk = std::min<uint64_t>(B, TB_NOALLOC_SCRATCH_BYTES / per_ct);
    uint64_t *tgt = base;
    uint64_t *digits = tgt + (ckks ? chunk * L * n : 0);
    uint64_t *acc = digits + chunk * (uint64_t)L * (L + 1) * n;
    uint64_t *last = acc + chunk * 2ull * (L + 1) * n;
    KeyGroups keys;
    keys.count = 1;
    keys.key[0] = key;
    keys.first[0] = 0;
    const int logn = c.logn;
    const uint64_t tstride = cstride;
    cudaError_t e;
    for (uint64_t b0 = 0; b0 < B; b0 += chunk) {
        const uint64_t nb = std::min(chunk, B - b0);
        keys.first[1] = (uint32_t)nb;
        uint64_t *cc = ct3 + b0 * cstride;
        const uint64_t *tg = cc + 2ull * L * n;   // the third polynomial is the target
        if (ckks) {
            StridedNttOp<false> op{tg, tgt, tstride, (uint64_t)L * n, c.d_mods, 0, L, 0, logn};
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * L), logn, 1, s);
            if (e != cudaSuccess) return status_from(e);
        }
        ModUpOp mu{ckks ? tgt : tg, ckks ? (uint64_t)L * n : tstride, digits, c.d_mods, nullptr, L, K, ckks, logn};
        e = dispatch_ntt<true>(logn, mu, (unsigned)(nb * pairs), 0, 0, s);
        if (e != cudaSuccess) return status_from(e);
        const int threads = 128;
        dim3 grid((unsigned)((n / 2 + threads - 1) / threads), L + 1, (unsigned)nb);
        ks_inner_kernel<<<grid, threads, 0, s>>>(digits, tg, tstride, keys, acc, c.d_mods, L, K, ckks, logn);
        e = cudaGetLastError();
        if (e != cudaSuccess) return status_from(e);
        SpecialInttOp si{acc, last, c.d_mods, L, K, c.scheme == SCHEME_BGV, logn};
        e = dispatch_ntt<false>(logn, si, (unsigned)(nb * 2), logn, 1, s);
        if (e != cudaSuccess) return status_from(e);
        ModDownBase mb{acc, last, cc, cstride, c.d_mods, c.d_drop, L, K, logn};
        if (ckks) {
            ModDownCkksOp op{mb};
            e = dispatch_ntt<true>(logn, op, (unsigned)(nb * 2 * L), 0, 0, s);
        } else if (c.scheme == SCHEME_BFV) {
            ModDownBfvOp op{mb};
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * 2 * L), logn, 1, s);
        } else {
            ModDownBgvOp op{mb, c.t_mod, c.inv_qlast_t[K]};
            e = dispatch_ntt<false>(logn, op, (unsigned)(nb * 2 * L), logn, 1, s);
        }
        if (e != cudaSuccess) return status_from(e);
    }
    return TB_OK;
}

// GaloisTool::getEltFromStep (src/utils/galois.cpp:45-88), generator 3.
int galois_elt_from_step(const Context &c, int step, uint32_t *elt) {
    const uint32_t n = c.n, m = 2 * n;
    if (step == 0) {
        *elt = m - 1;
        return TB_OK;
    }
    const bool neg = step < 0;
    uint32_t pos = (uint32_t)(neg ? -step : step);
    if (pos >= (n >> 1)) return set_error(TB_ERR_INVALID_ARGUMENT, "step count too large");
    pos &= m - 1;
    uint32_t k = neg ? (n >> 1) - pos : pos;
    uint64_t g = 1;
    while (k--) g = (g * 3) & (m - 1);
    *elt = (uint32_t)g;
    return TB_OK;
}

}  // namespace tb

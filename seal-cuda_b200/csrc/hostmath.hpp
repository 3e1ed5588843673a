// Host-side number theory for parameter precompute (runs once per context).
// Produces the same primes, roots and constants as the reference's host code:
// getPrimes (src/utils/numth.cpp:261-283), tryMinimalPrimitiveRoot
// (src/utils/numth.cpp:285-364), MultiplyUIntModOperand quotients
// (src/utils/uintarithsmallmod.h:166-184) and NTTTables (src/utils/ntt.cpp:17-66).
#pragma once

#include <cstdint>
#include <vector>

namespace tb {
namespace host {

using u128 = unsigned __int128;

inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)((u128)a * b % q); }

inline uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

// Inverse modulo m (m need not be prime); 0 when none exists.
inline uint64_t invmod(uint64_t a, uint64_t m) {
    __int128 t = 0, nt = 1, r = m, nr = a % m;
    while (nr) {
        __int128 qq = r / nr, tmp;
        tmp = t - qq * nt; t = nt; nt = tmp;
        tmp = r - qq * nr; r = nr; nr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += m;
    return (uint64_t)t;
}

inline uint64_t shoup(uint64_t w, uint64_t q) { return (uint64_t)(((u128)w << 64) / q); }

// floor(2^128 / q) for odd q (q never divides 2^128).
inline void barrett_ratio(uint64_t q, uint64_t &lo, uint64_t &hi) {
    u128 r = (~(u128)0) / q;
    lo = (uint64_t)r;
    hi = (uint64_t)(r >> 64);
}

inline bool is_prime(uint64_t n) {
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return false;
    for (uint64_t p : small) {
        if (n == p) return true;
        if (n % p == 0) return false;
    }
    uint64_t d = n - 1;
    int r = 0;
    while (!(d & 1)) { d >>= 1; r++; }
    for (uint64_t a : small) {
        uint64_t x = powmod(a, d, n);
        if (x == 1 || x == n - 1) continue;
        bool ok = false;
        for (int k = 1; k < r; k++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { ok = true; break; }
        }
        if (!ok) return false;
    }
    return true;
}

// Largest `count` primes = 1 mod factor below 2^bits, in descending order.
inline bool get_primes(uint64_t factor, int bits, size_t count, std::vector<uint64_t> &out) {
    out.clear();
    uint64_t value = ((uint64_t(1) << bits) - 1) / factor * factor + 1;
    uint64_t lower = uint64_t(1) << (bits - 1);
    while (out.size() < count && value > lower) {
        if (is_prime(value)) out.push_back(value);
        value -= factor;
    }
    return out.size() == count;
}

// Smallest primitive degree-th root of unity mod prime q (0 if none).
inline uint64_t minimal_root(uint64_t degree, uint64_t q) {
    if ((q - 1) % degree) return 0;
    uint64_t quot = (q - 1) / degree, root = 0;
    for (uint64_t x = 2; x < q; x++) {
        uint64_t r = powmod(x, quot, q);
        if (powmod(r, degree >> 1, q) == q - 1) { root = r; break; }
    }
    if (!root) return 0;
    uint64_t sq = mulmod(root, root, q), cur = root, best = root;
    for (uint64_t i = 0; i < degree; i += 2) {
        if (cur < best) best = cur;
        cur = mulmod(cur, sq, q);
    }
    return best;
}

inline uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

inline int bit_count(uint64_t x) {
    int b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}

// Product of `count` words as a little-endian multi-word integer.
inline std::vector<uint64_t> product(const uint64_t *v, size_t count) {
    std::vector<uint64_t> r{1};
    for (size_t i = 0; i < count; i++) {
        u128 carry = 0;
        for (auto &w : r) {
            u128 x = (u128)w * v[i] + carry;
            w = (uint64_t)x;
            carry = x >> 64;
        }
        if (carry) r.push_back((uint64_t)carry);
    }
    return r;
}

inline int bit_count(const std::vector<uint64_t> &v) {
    for (size_t i = v.size(); i-- > 0;)
        if (v[i]) return (int)(64 * i) + bit_count(v[i]);
    return 0;
}

// (prod of v except index skip) mod m
inline uint64_t punctured_mod(const uint64_t *v, size_t count, size_t skip, uint64_t m) {
    uint64_t p = 1 % m;
    for (size_t k = 0; k < count; k++)
        if (k != skip) p = mulmod(p, v[k] % m, m);
    return p;
}

inline uint64_t prod_mod(const uint64_t *v, size_t count, uint64_t m) {
    return punctured_mod(v, count, count, m);
}

// Multi-word integer modulo m.
inline uint64_t mod_words(const std::vector<uint64_t> &w, uint64_t m) {
    u128 r = 0;
    for (size_t i = w.size(); i-- > 0;) r = ((r << 64) | w[i]) % m;
    return (uint64_t)r;
}

// Multi-word integer divided by a word: quotient words and remainder.
inline std::vector<uint64_t> div_words(const std::vector<uint64_t> &w, uint64_t d, uint64_t &rem) {
    std::vector<uint64_t> q(w.size());
    u128 r = 0;
    for (size_t i = w.size(); i-- > 0;) {
        u128 cur = (r << 64) | w[i];
        q[i] = (uint64_t)(cur / d);
        r = cur % d;
    }
    rem = (uint64_t)r;
    return q;
}

}  // namespace host
}  // namespace tb

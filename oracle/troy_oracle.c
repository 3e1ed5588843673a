/*
 * CPU restatement of the reference's ciphertext-arithmetic hot path.
 * TEST INFRASTRUCTURE ONLY (see troy_oracle.h): the checker for the CUDA path,
 * never linked into the product.
 *
 * Citations are to the reference project (SecretHQ/seal-cuda, the "troy" port of
 * Microsoft SEAL 4.0), relative to its root.
 */
#include "troy_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------ modular basics */

static inline uint64_t mulhi64(uint64_t a, uint64_t b) { return (uint64_t)(((u128)a * b) >> 64); }
static inline uint64_t mulmod(uint64_t a, uint64_t b, uint64_t q) { return (uint64_t)(((u128)a * b) % q); }
static inline uint64_t addmod(uint64_t a, uint64_t b, uint64_t q) {
    uint64_t s = a + b;
    return s >= q ? s - q : s;
}
static inline uint64_t submod(uint64_t a, uint64_t b, uint64_t q) { return a >= b ? a - b : a + q - b; }
static inline uint64_t negmod(uint64_t a, uint64_t q) { return a ? q - a : 0; }

/* MultiplyUIntModOperand::setQuotient: floor(operand * 2^64 / q)
   (src/utils/uintarithsmallmod.h:166-184) */
static inline uint64_t shoup_quotient(uint64_t op, uint64_t q) { return (uint64_t)(((u128)op << 64) / q); }

/* multiplyUintModLazy: x*y - floor(x*y'/2^64)*q, in [0, 2q) for any 64-bit x
   (src/utils/uintarithsmallmod.h:226-240) */
static inline uint64_t mul_shoup_lazy(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) {
    return w * x - mulhi64(x, wq) * q;
}
/* multiplyUintMod with a MultiplyUIntModOperand (src/utils/uintarithsmallmod.h:205-219) */
static inline uint64_t mul_shoup(uint64_t x, uint64_t w, uint64_t wq, uint64_t q) {
    uint64_t r = mul_shoup_lazy(x, w, wq, q);
    return r >= q ? r - q : r;
}

static uint64_t powmod(uint64_t a, uint64_t e, uint64_t q) {
    uint64_t r = 1 % q;
    a %= q;
    while (e) {
        if (e & 1) r = mulmod(r, a, q);
        a = mulmod(a, a, q);
        e >>= 1;
    }
    return r;
}

/* tryInvertUintMod via the extended Euclidean algorithm (src/utils/numth.cpp:57-78); 0 if none */
static uint64_t invmod(uint64_t a, uint64_t m) {
    __int128 t = 0, newt = 1, r = m, newr = a % m;
    while (newr) {
        __int128 qq = r / newr, tmp;
        tmp = t - qq * newt; t = newt; newt = tmp;
        tmp = r - qq * newr; r = newr; newr = tmp;
    }
    if (r != 1) return 0;
    if (t < 0) t += m;
    return (uint64_t)t;
}

static uint32_t bitrev(uint32_t x, int bits) {
    uint32_t r = 0;
    for (int i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
    return r;
}

static int bit_count(uint64_t x) {
    int b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}

/* -------------------------------------------------------------- primes */

/* Deterministic Miller-Rabin for 64-bit inputs; the reference's isPrime
   (src/utils/numth.cpp:163-259) is the probabilistic form of the same test. */
static int is_prime(uint64_t n) {
    static const uint64_t small[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37};
    if (n < 2) return 0;
    for (int i = 0; i < 12; i++) {
        if (n == small[i]) return 1;
        if (n % small[i] == 0) return 0;
    }
    uint64_t d = n - 1;
    int r = 0;
    while (!(d & 1)) { d >>= 1; r++; }
    for (int i = 0; i < 12; i++) {
        uint64_t x = powmod(small[i], d, n);
        if (x == 1 || x == n - 1) continue;
        int ok = 0;
        for (int k = 1; k < r; k++) {
            x = mulmod(x, x, n);
            if (x == n - 1) { ok = 1; break; }
        }
        if (!ok) return 0;
    }
    return 1;
}

/* getPrimes: largest primes = 1 mod factor below 2^bit_size, descending (src/utils/numth.cpp:261-283) */
int orc_get_primes(uint64_t factor, int bit_size, size_t count, uint64_t *out) {
    uint64_t value = (((uint64_t)1 << bit_size) - 1) / factor * factor + 1;
    uint64_t lower = (uint64_t)1 << (bit_size - 1);
    size_t k = 0;
    while (k < count && value > lower) {
        if (is_prime(value)) out[k++] = value;
        value -= factor;
    }
    return k == count ? 0 : -1;
}

/* CoeffModulus::Create: per bit size take primes from the back of that size's list
   (src/modulus.cpp:80-118) */
int orc_coeff_modulus_create(size_t n, const int *bits, int count, uint64_t *out) {
    uint64_t lists[64][64];
    int list_len[64] = {0}, used[64] = {0};
    int need[64] = {0};
    for (int i = 0; i < count; i++) {
        if (bits[i] < 2 || bits[i] > 60) return -1;
        need[bits[i]]++;
    }
    for (int b = 0; b < 64; b++) {
        if (!need[b]) continue;
        if (orc_get_primes(2 * (uint64_t)n, b, (size_t)need[b], lists[b])) return -1;
        list_len[b] = need[b];
    }
    for (int i = 0; i < count; i++) {
        int b = bits[i];
        out[i] = lists[b][list_len[b] - 1 - used[b]];
        used[b]++;
    }
    return 0;
}

/* PlainModulus::Batching(n, bits) = CoeffModulus::Create(n, {bits})[0] (src/modulus.h:528-535) */
int orc_plain_modulus_batching(size_t n, int bits, uint64_t *out) {
    int b = bits;
    return orc_coeff_modulus_create(n, &b, 1, out);
}

/* tryMinimalPrimitiveRoot: the smallest primitive degree-th root of unity
   (src/utils/numth.cpp:285-364). Any primitive root works as a starting point
   because the minimum over all its odd powers is unique. */
uint64_t orc_minimal_root(uint64_t degree, uint64_t q) {
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

/* ---------------------------------------------------------------- NTT */

typedef struct {
    int logn;
    uint64_t q;
    uint64_t *rop, *rquo, *iop, *iquo;
    uint64_t inv_n, inv_n_quo;
} tables_t;

/* NTTTables::initialize (src/utils/ntt.cpp:17-66): root powers in bit-reversed order,
   inverse root powers in the scrambled order used by the Gentleman-Sande pass. */
static int build_tables(int logn, uint64_t q, tables_t *t) {
    size_t n = (size_t)1 << logn;
    uint64_t root = orc_minimal_root(2 * (uint64_t)n, q);
    if (!root) return -1;
    uint64_t inv_root = invmod(root, q);
    t->logn = logn;
    t->q = q;
    t->rop = malloc(8 * n); t->rquo = malloc(8 * n);
    t->iop = malloc(8 * n); t->iquo = malloc(8 * n);
    uint64_t power = root;
    for (size_t i = 1; i < n; i++) {
        size_t idx = bitrev((uint32_t)i, logn);
        t->rop[idx] = power;
        power = mulmod(power, root, q);
    }
    t->rop[0] = 1;
    power = inv_root;
    for (size_t i = 1; i < n; i++) {
        size_t idx = (size_t)bitrev((uint32_t)(i - 1), logn) + 1;
        t->iop[idx] = power;
        power = mulmod(power, inv_root, q);
    }
    t->iop[0] = 1;
    for (size_t i = 0; i < n; i++) {
        t->rquo[i] = shoup_quotient(t->rop[i], q);
        t->iquo[i] = shoup_quotient(t->iop[i], q);
    }
    t->inv_n = invmod((uint64_t)n % q, q);
    t->inv_n_quo = shoup_quotient(t->inv_n, q);
    return 0;
}

static void free_tables(tables_t *t) {
    free(t->rop); free(t->rquo); free(t->iop); free(t->iquo);
}

int orc_ntt_tables(int logn, uint64_t q, uint64_t *root_op, uint64_t *root_quo, uint64_t *inv_op,
                   uint64_t *inv_quo, uint64_t *inv_n) {
    tables_t t;
    if (build_tables(logn, q, &t)) return -1;
    size_t n = (size_t)1 << logn;
    memcpy(root_op, t.rop, 8 * n); memcpy(root_quo, t.rquo, 8 * n);
    memcpy(inv_op, t.iop, 8 * n); memcpy(inv_quo, t.iquo, 8 * n);
    inv_n[0] = t.inv_n; inv_n[1] = t.inv_n_quo;
    inv_n[2] = t.rop[bitrev(1, logn)]; /* root^1 sits at bitrev(1) */
    free_tables(&t);
    return 0;
}

/* DWTHandler::transformToRev with the lazy modular arithmetic of NTTTables
   (src/utils/dwthandler.h:88-204, src/utils/ntt.h:17-60): Cooley-Tukey, natural
   order in, bit-reversed out, values kept in [0, 4q). */
static void ntt_fwd(const tables_t *t, uint64_t *a) {
    size_t n = (size_t)1 << t->logn;
    uint64_t q = t->q, q2 = q << 1;
    size_t gap = n >> 1, m = 1, ridx = 0;
    for (; m < (n >> 1); m <<= 1) {
        size_t offset = 0;
        for (size_t i = 0; i < m; i++) {
            ++ridx;
            uint64_t w = t->rop[ridx], wq = t->rquo[ridx];
            uint64_t *x = a + offset, *y = x + gap;
            for (size_t j = 0; j < gap; j++) {
                uint64_t u = x[j] >= q2 ? x[j] - q2 : x[j];
                uint64_t v = mul_shoup_lazy(y[j], w, wq, q);
                x[j] = u + v;
                y[j] = u + q2 - v;
            }
            offset += gap << 1;
        }
        gap >>= 1;
    }
    for (size_t i = 0; i < m; i++) {
        ++ridx;
        uint64_t w = t->rop[ridx], wq = t->rquo[ridx];
        uint64_t u = a[0] >= q2 ? a[0] - q2 : a[0];
        uint64_t v = mul_shoup_lazy(a[1], w, wq, q);
        a[0] = u + v;
        a[1] = u + q2 - v;
        a += 2;
    }
}

/* DWTHandler::transformFromRev with scalar n^-1 folded into the last stage
   (src/utils/dwthandler.h:206-372): Gentleman-Sande, values kept in [0, 2q). */
static void ntt_inv(const tables_t *t, uint64_t *a) {
    size_t n = (size_t)1 << t->logn;
    uint64_t q = t->q, q2 = q << 1;
    size_t gap = 1, m = n >> 1, ridx = 0;
    for (; m > 1; m >>= 1) {
        size_t offset = 0;
        for (size_t i = 0; i < m; i++) {
            ++ridx;
            uint64_t w = t->iop[ridx], wq = t->iquo[ridx];
            uint64_t *x = a + offset, *y = x + gap;
            for (size_t j = 0; j < gap; j++) {
                uint64_t u = x[j], v = y[j];
                uint64_t s = u + v;
                x[j] = s >= q2 ? s - q2 : s;
                y[j] = mul_shoup_lazy(u + q2 - v, w, wq, q);
            }
            offset += gap << 1;
        }
        gap <<= 1;
    }
    ++ridx;
    uint64_t w = t->iop[ridx];
    uint64_t sw = mul_shoup(w, t->inv_n, t->inv_n_quo, q); /* mulRootScalar */
    uint64_t swq = shoup_quotient(sw, q);
    for (size_t j = 0; j < gap; j++) {
        uint64_t u = a[j] >= q2 ? a[j] - q2 : a[j];
        uint64_t v = a[j + gap];
        uint64_t s = u + v;
        s = s >= q2 ? s - q2 : s;
        a[j] = mul_shoup_lazy(s, t->inv_n, t->inv_n_quo, q);
        a[j + gap] = mul_shoup_lazy(u + q2 - v, sw, swq, q);
    }
}

/* nttNegacyclicHarvey / inverseNttNegacyclicHarvey final reductions (src/utils/ntt.cpp:164-213) */
static void ntt_forward_t(const tables_t *t, uint64_t *a, int lazy) {
    ntt_fwd(t, a);
    if (!lazy) {
        size_t n = (size_t)1 << t->logn;
        uint64_t q = t->q, q2 = q << 1;
        for (size_t i = 0; i < n; i++) {
            if (a[i] >= q2) a[i] -= q2;
            if (a[i] >= q) a[i] -= q;
        }
    }
}

static void ntt_inverse_t(const tables_t *t, uint64_t *a, int lazy) {
    ntt_inv(t, a);
    if (!lazy) {
        size_t n = (size_t)1 << t->logn;
        for (size_t i = 0; i < n; i++)
            if (a[i] >= t->q) a[i] -= t->q;
    }
}

int orc_ntt_forward(int logn, uint64_t q, uint64_t *data, int lazy) {
    tables_t t;
    if (build_tables(logn, q, &t)) return -1;
    ntt_forward_t(&t, data, lazy);
    free_tables(&t);
    return 0;
}

int orc_ntt_inverse(int logn, uint64_t q, uint64_t *data, int lazy) {
    tables_t t;
    if (build_tables(logn, q, &t)) return -1;
    ntt_inverse_t(&t, data, lazy);
    free_tables(&t);
    return 0;
}

int orc_ntt_forward_rns(int logn, const uint64_t *moduli, int count, uint64_t *data, int lazy) {
    size_t n = (size_t)1 << logn;
    for (int i = 0; i < count; i++)
        if (orc_ntt_forward(logn, moduli[i], data + i * n, lazy)) return -1;
    return 0;
}

int orc_ntt_inverse_rns(int logn, const uint64_t *moduli, int count, uint64_t *data, int lazy) {
    size_t n = (size_t)1 << logn;
    for (int i = 0; i < count; i++)
        if (orc_ntt_inverse(logn, moduli[i], data + i * n, lazy)) return -1;
    return 0;
}

/* ------------------------------------------------ element-wise arithmetic */

/* dyadicProductCoeffmod: a*b mod q (src/utils/polyarithsmallmod.cpp:71-104) */
void orc_dyadic_product(uint64_t q, const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n) {
    for (size_t i = 0; i < n; i++) out[i] = mulmod(a[i], b[i], q);
}

void orc_poly_dyadic(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                     uint64_t *out) {
    for (int j = 0; j < count; j++) orc_dyadic_product(moduli[j], a + j * n, b + j * n, out + j * n, n);
}

/* addPolyCoeffmod / subPolyCoeffmod / negatePolyCoeffmod / multiplyPolyScalarCoeffmod
   (src/utils/polyarithsmallmod.h) */
void orc_poly_add(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                  uint64_t *out) {
    for (int j = 0; j < count; j++)
        for (size_t i = 0; i < n; i++) out[j * n + i] = addmod(a[j * n + i], b[j * n + i], moduli[j]);
}

void orc_poly_sub(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                  uint64_t *out) {
    for (int j = 0; j < count; j++)
        for (size_t i = 0; i < n; i++) out[j * n + i] = submod(a[j * n + i], b[j * n + i], moduli[j]);
}

void orc_poly_negate(const uint64_t *moduli, int count, size_t n, const uint64_t *a, uint64_t *out) {
    for (int j = 0; j < count; j++)
        for (size_t i = 0; i < n; i++) out[j * n + i] = negmod(a[j * n + i], moduli[j]);
}

void orc_poly_mul_scalar(const uint64_t *moduli, int count, size_t n, const uint64_t *a, uint64_t scalar,
                         uint64_t *out) {
    for (int j = 0; j < count; j++) {
        uint64_t s = scalar % moduli[j];
        for (size_t i = 0; i < n; i++) out[j * n + i] = mulmod(a[j * n + i], s, moduli[j]);
    }
}

/* ------------------------------------------------------ Blake2xb stream */

/* BLAKE2b compression (RFC 7693), used by the reference through src/utils/blake2b.c */
static const uint64_t B2_IV[8] = {0x6a09e667f3bcc908ULL, 0xbb67ae8584caa73bULL, 0x3c6ef372fe94f82bULL,
                                  0xa54ff53a5f1d36f1ULL, 0x510e527fade682d1ULL, 0x9b05688c2b3e6c1fULL,
                                  0x1f83d9abfb41bd6bULL, 0x5be0cd19137e2179ULL};
static const uint8_t B2_SIGMA[12][16] = {
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3},
    {11, 8, 12, 0, 5, 2, 15, 13, 10, 14, 3, 6, 7, 1, 9, 4}, {7, 9, 3, 1, 13, 12, 11, 14, 2, 6, 5, 10, 4, 0, 15, 8},
    {9, 0, 5, 7, 2, 4, 10, 15, 14, 1, 11, 12, 6, 8, 3, 13}, {2, 12, 6, 10, 0, 11, 8, 3, 4, 13, 7, 5, 15, 14, 1, 9},
    {12, 5, 1, 15, 14, 13, 4, 10, 0, 7, 6, 3, 9, 2, 8, 11}, {13, 11, 7, 14, 12, 1, 3, 9, 5, 0, 15, 4, 8, 6, 2, 10},
    {6, 15, 14, 9, 11, 3, 0, 8, 12, 2, 13, 7, 1, 4, 10, 5}, {10, 2, 8, 4, 7, 6, 1, 5, 15, 11, 9, 14, 3, 12, 13, 0},
    {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15}, {14, 10, 4, 8, 9, 15, 13, 6, 1, 12, 0, 2, 11, 7, 5, 3}};

static inline uint64_t rotr64(uint64_t x, int c) { return (x >> c) | (x << (64 - c)); }

static void b2_compress(uint64_t h[8], const uint64_t m[16], uint64_t t, int last) {
    uint64_t v[16];
    for (int i = 0; i < 8; i++) { v[i] = h[i]; v[i + 8] = B2_IV[i]; }
    v[12] ^= t;
    if (last) v[14] = ~v[14];
#define B2G(a, b, c, d, x, y)                 \
    do {                                      \
        v[a] = v[a] + v[b] + (x);             \
        v[d] = rotr64(v[d] ^ v[a], 32);       \
        v[c] = v[c] + v[d];                   \
        v[b] = rotr64(v[b] ^ v[c], 24);       \
        v[a] = v[a] + v[b] + (y);             \
        v[d] = rotr64(v[d] ^ v[a], 16);       \
        v[c] = v[c] + v[d];                   \
        v[b] = rotr64(v[b] ^ v[c], 63);       \
    } while (0)
    for (int r = 0; r < 12; r++) {
        const uint8_t *s = B2_SIGMA[r];
        B2G(0, 4, 8, 12, m[s[0]], m[s[1]]);
        B2G(1, 5, 9, 13, m[s[2]], m[s[3]]);
        B2G(2, 6, 10, 14, m[s[4]], m[s[5]]);
        B2G(3, 7, 11, 15, m[s[6]], m[s[7]]);
        B2G(0, 5, 10, 15, m[s[8]], m[s[9]]);
        B2G(1, 6, 11, 12, m[s[10]], m[s[11]]);
        B2G(2, 7, 8, 13, m[s[12]], m[s[13]]);
        B2G(3, 4, 9, 14, m[s[14]], m[s[15]]);
    }
#undef B2G
    for (int i = 0; i < 8; i++) h[i] ^= v[i] ^ v[i + 8];
}

/* One 4096-byte refill of Blake2xbPRNG (src/randomgen.cpp:188-198): BLAKE2Xb with
   the 64-byte seed as key, the 8-byte little-endian counter as message and
   xof_length 4096. Root: keyed BLAKE2b-512 with fanout=depth=1; output block i:
   BLAKE2b of the root with leaf_length=inner_length=64, node_offset=i. */
static void blake2xb_block(const uint64_t seed[8], uint64_t counter, uint8_t out[4096]) {
    const uint32_t xof_len = 4096;
    uint64_t h[8], m[16];
    /* parameter block word 0: digest 64 | key 64 << 8 | fanout 1 << 16 | depth 1 << 24 | leaf 0 */
    for (int i = 0; i < 8; i++) h[i] = B2_IV[i];
    h[0] ^= 64ULL | (64ULL << 8) | (1ULL << 16) | (1ULL << 24);
    h[1] ^= (uint64_t)xof_len << 32; /* node_offset 0 | xof_length */
    memset(m, 0, sizeof(m));
    for (int i = 0; i < 8; i++) m[i] = seed[i];
    b2_compress(h, m, 128, 0);
    memset(m, 0, sizeof(m));
    m[0] = counter;
    b2_compress(h, m, 136, 1);
    for (uint32_t blk = 0; blk < xof_len / 64; blk++) {
        uint64_t c[8];
        for (int i = 0; i < 8; i++) c[i] = B2_IV[i];
        c[0] ^= 64ULL | (64ULL << 32); /* digest 64, key 0, fanout 0, depth 0, leaf_length 64 */
        c[1] ^= (uint64_t)blk | ((uint64_t)xof_len << 32);
        c[2] ^= 64ULL << 8; /* node_depth 0, inner_length 64 */
        memset(m, 0, sizeof(m));
        for (int i = 0; i < 8; i++) m[i] = h[i];
        b2_compress(c, m, 64, 1);
        memcpy(out + 64 * blk, c, 64);
    }
}

/* UniformRandomGenerator::generate over the refill blocks (src/randomgen.cpp:165-181):
   the stream is the concatenation of refills with counters 0, 1, 2, ... */
void orc_prng_bytes(const uint64_t *seed8, size_t offset, size_t count, uint8_t *out) {
    uint8_t block[4096];
    uint64_t cur = (uint64_t)-1;
    for (size_t i = 0; i < count; i++) {
        size_t pos = offset + i;
        uint64_t b = pos >> 12;
        if (b != cur) {
            blake2xb_block(seed8, b, block);
            cur = b;
        }
        out[i] = block[pos & 4095];
    }
}

typedef struct {
    const uint64_t *seed;
    size_t offset;
    uint64_t cur;
    uint8_t block[4096];
} stream_t;

static void stream_read(stream_t *s, void *dst, size_t count) {
    uint8_t *d = dst;
    for (size_t i = 0; i < count; i++) {
        size_t pos = s->offset + i;
        uint64_t b = pos >> 12;
        if (b != s->cur) {
            blake2xb_block(s->seed, b, s->block);
            s->cur = b;
        }
        d[i] = s->block[pos & 4095];
    }
    s->offset += count;
}

static int hw8(uint8_t x) { return __builtin_popcount(x); }

int orc_sample_at(int kind, const uint64_t *seed8, size_t *offset, size_t n, const uint64_t *moduli,
                  int count, uint64_t *out) {
    stream_t s;
    s.seed = seed8;
    s.offset = *offset;
    s.cur = (uint64_t)-1;
    if (kind == 0) {
        /* samplePolyTernary (src/utils/rlwe.cpp:21-42): uniform_int_distribution<uint64_t>(0, 2)
           over the 32-bit RandomToStandardAdapter; with a 32-bit engine libstdc++ 13 draws
           x, keeps (x*3) >> 32 and redraws while (uint32)(x*3) < (2^32 mod 3) = 1, i.e. x == 0. */
        for (size_t i = 0; i < n; i++) {
            uint32_t x;
            uint64_t prod;
            do {
                stream_read(&s, &x, 4);
                prod = (uint64_t)x * 3u;
            } while ((uint32_t)prod < 1u);
            uint64_t r = prod >> 32;
            for (int j = 0; j < count; j++)
                out[j * n + i] = r == 0 ? moduli[j] - 1 : r - 1;
        }
    } else if (kind == 1) {
        /* samplePolyCbd (src/utils/rlwe.cpp:71-107): 6 bytes per coefficient */
        for (size_t i = 0; i < n; i++) {
            uint8_t x[6];
            stream_read(&s, x, 6);
            x[2] &= 0x1F;
            x[5] &= 0x1F;
            int v = hw8(x[0]) + hw8(x[1]) + hw8(x[2]) - hw8(x[3]) - hw8(x[4]) - hw8(x[5]);
            for (int j = 0; j < count; j++)
                out[j * n + i] = v < 0 ? moduli[j] - (uint64_t)(-v) : (uint64_t)v;
        }
    } else if (kind == 2) {
        /* samplePolyUniform (src/utils/rlwe.cpp:126-149): n*count words first, then rejected
           words are replaced by further words from the same stream, in order. */
        stream_read(&s, out, 8 * n * (size_t)count);
        for (int j = 0; j < count; j++) {
            uint64_t q = moduli[j];
            uint64_t max_multiple = UINT64_MAX - (UINT64_MAX % q) - 1;
            for (size_t i = 0; i < n; i++) {
                uint64_t r = out[j * n + i];
                while (r >= max_multiple) stream_read(&s, &r, 8);
                out[j * n + i] = r % q;
            }
        }
    } else {
        return -1;
    }
    *offset = s.offset;
    return 0;
}

int orc_sample(int kind, const uint64_t *seed8, size_t n, const uint64_t *moduli, int count, uint64_t *out) {
    size_t off = 0;
    return orc_sample_at(kind, seed8, &off, n, moduli, count, out);
}

/* ------------------------------------------------------------ RNS tool */

/* BaseConverter (src/utils/rns.cpp:400-548): punctured products of the input base
   reduced into each output modulus; computed modulus by modulus, which equals
   reducing the multi-precision punctured product. */
typedef struct {
    int ni, no;
    const uint64_t *ib, *ob;
    uint64_t inv_punct[64];     /* (Q/q_i)^-1 mod q_i */
    uint64_t matrix[64][64];    /* [o][i] = (Q/q_i) mod p_o */
} conv_t;

static void conv_init(conv_t *c, const uint64_t *ib, int ni, const uint64_t *ob, int no) {
    c->ni = ni; c->no = no; c->ib = ib; c->ob = ob;
    for (int i = 0; i < ni; i++) {
        uint64_t p = 1 % ib[i];
        for (int k = 0; k < ni; k++)
            if (k != i) p = mulmod(p, ib[k] % ib[i], ib[i]);
        c->inv_punct[i] = invmod(p, ib[i]);
    }
    for (int o = 0; o < no; o++)
        for (int i = 0; i < ni; i++) {
            uint64_t p = 1 % ob[o];
            for (int k = 0; k < ni; k++)
                if (k != i) p = mulmod(p, ib[k] % ob[o], ob[o]);
            c->matrix[o][i] = p;
        }
}

/* fastConvertArray: out_o = sum_i [x_i (Q/q_i)^-1]_{q_i} (Q/q_i) mod p_o */
static void conv_fast(const conv_t *c, size_t n, const uint64_t *in, uint64_t *out) {
    uint64_t tmp[64];
    for (size_t j = 0; j < n; j++) {
        for (int i = 0; i < c->ni; i++) tmp[i] = mulmod(in[i * n + j] % c->ib[i], c->inv_punct[i], c->ib[i]);
        for (int o = 0; o < c->no; o++) {
            u128 acc = 0;
            for (int i = 0; i < c->ni; i++) acc += (u128)tmp[i] * c->matrix[o][i];
            out[o * n + j] = (uint64_t)(acc % c->ob[o]);
        }
    }
}

static uint64_t prod_mod(const uint64_t *b, int cnt, uint64_t m) {
    uint64_t p = 1 % m;
    for (int k = 0; k < cnt; k++) p = mulmod(p, b[k] % m, m);
    return p;
}

typedef struct {
    size_t n;
    int L;
    uint64_t q[64], t;
    int bB, bsk;
    uint64_t B[64], Bsk[64], Bskm[64], m_sk, gamma, m_tilde;
    conv_t q_to_bsk, q_to_mt, B_to_q, B_to_msk, q_to_tg, q_to_t;
    uint64_t tg[2];
} rns_t;

/* RNSTool::initialize (src/utils/rns.cpp:581-803) */
static int rns_init(rns_t *r, size_t n, const uint64_t *q, int L, uint64_t t) {
    r->n = n; r->L = L; r->t = t;
    memcpy(r->q, q, 8 * (size_t)L);
    /* total bit count of prod(q) */
    int total = 0;
    {
        /* multiply out prod(q) in base 2^64 limbs to count bits */
        uint64_t limbs[66] = {0};
        int len = 1;
        limbs[0] = 1;
        for (int i = 0; i < L; i++) {
            u128 carry = 0;
            for (int k = 0; k < len; k++) {
                u128 v = (u128)limbs[k] * q[i] + carry;
                limbs[k] = (uint64_t)v;
                carry = v >> 64;
            }
            if (carry) limbs[len++] = (uint64_t)carry;
        }
        total = 64 * (len - 1) + bit_count(limbs[len - 1]);
    }
    int bB = L;
    if (32 + bit_count(t) + total >= 61 * L + 61) bB++;
    r->bB = bB;
    r->bsk = bB + 1;
    uint64_t primes[66];
    if (orc_get_primes(2 * (uint64_t)n, 61, (size_t)(r->bsk + 1), primes)) return -1;
    r->m_sk = primes[0];
    r->gamma = primes[1];
    for (int i = 0; i < bB; i++) r->B[i] = primes[2 + i];
    for (int i = 0; i < bB; i++) r->Bsk[i] = r->B[i];
    r->Bsk[bB] = r->m_sk;
    r->m_tilde = (uint64_t)1 << 32;
    for (int i = 0; i < r->bsk; i++) r->Bskm[i] = r->Bsk[i];
    r->Bskm[r->bsk] = r->m_tilde;
    r->tg[0] = t;
    r->tg[1] = r->gamma;
    conv_init(&r->q_to_bsk, r->q, L, r->Bsk, r->bsk);
    conv_init(&r->q_to_mt, r->q, L, &r->m_tilde, 1);
    conv_init(&r->B_to_q, r->B, bB, r->q, L);
    conv_init(&r->B_to_msk, r->B, bB, &r->m_sk, 1);
    if (t) {
        conv_init(&r->q_to_tg, r->q, L, r->tg, 2);
        conv_init(&r->q_to_t, r->q, L, &r->t, 1);
    }
    return 0;
}

/* fastbconvmTilde (src/utils/rns.cpp:1010-1037) */
static void rns_fastbconv_mtilde(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    uint64_t *tmp = malloc(8 * n * (size_t)r->L);
    for (int i = 0; i < r->L; i++)
        for (size_t j = 0; j < n; j++) tmp[i * n + j] = mulmod(in[i * n + j], r->m_tilde % r->q[i], r->q[i]);
    conv_fast(&r->q_to_bsk, n, tmp, out);
    conv_fast(&r->q_to_mt, n, tmp, out + (size_t)r->bsk * n);
    free(tmp);
}

/* smMrq (src/utils/rns.cpp:934-975) */
static void rns_smmrq(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    uint64_t mt = r->m_tilde;
    uint64_t neg_inv_q_mt = negmod(invmod(prod_mod(r->q, r->L, mt), mt), mt);
    const uint64_t *in_mt = in + (size_t)r->bsk * n;
    for (int i = 0; i < r->bsk; i++) {
        uint64_t b = r->Bsk[i];
        uint64_t q_mod_b = prod_mod(r->q, r->L, b);
        uint64_t inv_mt_b = invmod(mt % b, b);
        for (size_t j = 0; j < n; j++) {
            uint64_t rm = mulmod(in_mt[j], neg_inv_q_mt, mt);
            uint64_t tmp = rm;
            if (tmp >= (mt >> 1)) tmp += b - mt;
            uint64_t v = addmod(mulmod(tmp % b, q_mod_b, b), in[i * n + j] % b, b);
            out[i * n + j] = mulmod(v, inv_mt_b, b);
        }
    }
}

/* fastFloor (src/utils/rns.cpp:977-1008) */
static void rns_fast_floor(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    conv_fast(&r->q_to_bsk, n, in, out);
    const uint64_t *in_bsk = in + (size_t)r->L * n;
    for (int i = 0; i < r->bsk; i++) {
        uint64_t b = r->Bsk[i];
        uint64_t inv_q_b = invmod(prod_mod(r->q, r->L, b), b);
        for (size_t j = 0; j < n; j++) {
            uint64_t x = in_bsk[i * n + j] + (b - out[i * n + j]);
            out[i * n + j] = mulmod(x % b, inv_q_b, b);
        }
    }
}

/* fastbconvSk (src/utils/rns.cpp:878-932) */
static void rns_fastbconv_sk(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    conv_fast(&r->B_to_q, n, in, out);
    uint64_t *tmp = malloc(8 * n);
    conv_fast(&r->B_to_msk, n, in, tmp);
    uint64_t msk = r->m_sk;
    uint64_t inv_pb_msk = invmod(prod_mod(r->B, r->bB, msk), msk);
    const uint64_t *in_msk = in + (size_t)r->bB * n;
    for (size_t j = 0; j < n; j++) tmp[j] = mulmod((tmp[j] + (msk - in_msk[j])) % msk, inv_pb_msk, msk);
    for (int i = 0; i < r->L; i++) {
        uint64_t b = r->q[i];
        uint64_t pb = prod_mod(r->B, r->bB, b);
        for (size_t j = 0; j < n; j++) {
            uint64_t a = tmp[j];
            uint64_t d = out[i * n + j];
            if (a > (msk >> 1)) out[i * n + j] = addmod(mulmod((msk - a) % b, pb, b), d % b, b);
            else out[i * n + j] = addmod(mulmod(a % b, negmod(pb, b), b), d % b, b);
        }
    }
    free(tmp);
}

/* divideAndRoundqLastInplace (src/utils/rns.cpp:805-829) */
static void rns_div_round_last(const rns_t *r, uint64_t *io) {
    size_t n = r->n;
    int L = r->L;
    uint64_t ql = r->q[L - 1], half = ql >> 1;
    uint64_t *last = io + (size_t)(L - 1) * n;
    for (size_t j = 0; j < n; j++) last[j] = addmod(last[j], half % ql, ql);
    for (int i = 0; i < L - 1; i++) {
        uint64_t b = r->q[i], hm = half % b, inv = invmod(ql % b, b);
        for (size_t j = 0; j < n; j++) {
            uint64_t tmp = submod(last[j] % b, hm, b);
            io[i * n + j] = mulmod(submod(io[i * n + j], tmp, b), inv, b);
        }
    }
}

/* divideAndRoundqLastNttInplace (src/utils/rns.cpp:831-876) */
static int rns_div_round_last_ntt(const rns_t *r, uint64_t *io) {
    size_t n = r->n;
    int L = r->L, logn = 0;
    while (((size_t)1 << logn) < n) logn++;
    uint64_t ql = r->q[L - 1], half = ql >> 1;
    uint64_t *last = io + (size_t)(L - 1) * n;
    tables_t tl;
    if (build_tables(logn, ql, &tl)) return -1;
    ntt_inverse_t(&tl, last, 0);
    free_tables(&tl);
    for (size_t j = 0; j < n; j++) last[j] = addmod(last[j], half % ql, ql);
    uint64_t *tmp = malloc(8 * n);
    for (int i = 0; i < L - 1; i++) {
        uint64_t b = r->q[i];
        tables_t tb;
        if (build_tables(logn, b, &tb)) { free(tmp); return -1; }
        for (size_t j = 0; j < n; j++) tmp[j] = b < ql ? last[j] % b : last[j];
        uint64_t neg_half = b - (half % b);
        for (size_t j = 0; j < n; j++) tmp[j] += neg_half;
        ntt_forward_t(&tb, tmp, 1);
        uint64_t inv = invmod(ql % b, b), invq = shoup_quotient(inv, b);
        for (size_t j = 0; j < n; j++) {
            uint64_t x = io[i * n + j] + ((b << 2) - tmp[j]);
            io[i * n + j] = mul_shoup(x, inv, invq, b);
        }
        free_tables(&tb);
    }
    free(tmp);
    return 0;
}

/* decryptScaleAndRound (src/utils/rns.cpp:1039-1095) */
static void rns_decrypt_scale_round(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    int L = r->L;
    uint64_t t = r->t, g = r->gamma;
    uint64_t *tmp = malloc(8 * n * (size_t)L), *tg = malloc(16 * n);
    for (int i = 0; i < L; i++) {
        uint64_t f = mulmod(t % r->q[i], g % r->q[i], r->q[i]);
        for (size_t j = 0; j < n; j++) tmp[i * n + j] = mulmod(in[i * n + j], f, r->q[i]);
    }
    conv_fast(&r->q_to_tg, n, tmp, tg);
    for (int k = 0; k < 2; k++) {
        uint64_t m = r->tg[k];
        uint64_t f = negmod(invmod(prod_mod(r->q, L, m), m), m);
        for (size_t j = 0; j < n; j++) tg[k * n + j] = mulmod(tg[k * n + j], f, m);
    }
    uint64_t inv_g_t = invmod(g % t, t);
    for (size_t j = 0; j < n; j++) {
        uint64_t vt = tg[j], vg = tg[n + j], d;
        if (vg > (g >> 1)) d = addmod(vt, (g - vg) % t, t);
        else d = submod(vt, vg % t, t);
        if (d) d = mulmod(d, inv_g_t, t);
        out[j] = d;
    }
    free(tmp);
    free(tg);
}

/* modTAndDivideqLastInplace (src/utils/rns.cpp:1097-1140) */
static void rns_mod_t_div_last(const rns_t *r, uint64_t *io) {
    size_t n = r->n;
    int L = r->L;
    uint64_t t = r->t, ql = r->q[L - 1];
    uint64_t inv_ql_t = invmod(ql % t, t);
    const uint64_t *last = io + (size_t)(L - 1) * n;
    uint64_t *neg = malloc(8 * n);
    for (size_t j = 0; j < n; j++) {
        neg[j] = negmod(last[j] % t, t);
        if (inv_ql_t != 1) neg[j] = mulmod(neg[j], inv_ql_t, t);
    }
    for (int i = 0; i < L - 1; i++) {
        uint64_t b = r->q[i], inv = invmod(ql % b, b);
        for (size_t j = 0; j < n; j++) {
            uint64_t delta = mulmod(neg[j] % b, ql % b, b);
            uint64_t x = io[i * n + j] + 2 * b - (last[j] % b) - delta;
            io[i * n + j] = mulmod(x % b, inv, b);
        }
    }
    free(neg);
}

/* decryptModt -> BaseConverter::exactConvertArray (src/utils/rns.cpp:461-548): the FP64
   rounding sum is accumulated in the same order as the reference. */
static void rns_decrypt_mod_t(const rns_t *r, const uint64_t *in, uint64_t *out) {
    size_t n = r->n;
    int L = r->L;
    const conv_t *c = &r->q_to_t;
    uint64_t t = r->t;
    uint64_t q_mod_t = prod_mod(r->q, L, t);
    for (size_t j = 0; j < n; j++) {
        uint64_t tmp[64];
        double agg = 0.0;
        for (int i = 0; i < L; i++) {
            uint64_t b = r->q[i];
            if (c->inv_punct[i] == 1) tmp[i] = in[i * n + j] % b;
            else tmp[i] = mulmod(in[i * n + j], c->inv_punct[i], b);
        }
        for (int i = 0; i < L; i++) agg += (double)tmp[i] / (double)r->q[i];
        agg += 0.5;
        uint64_t v = (uint64_t)agg;
        u128 acc = 0;
        for (int i = 0; i < L; i++) acc += (u128)tmp[i] * c->matrix[0][i];
        uint64_t s = (uint64_t)(acc % t);
        out[j] = submod(s, mulmod(v % t, q_mod_t, t), t);
    }
}

int orc_rns_bases(size_t n, const uint64_t *q, int count, uint64_t t, uint64_t *out) {
    rns_t r;
    if (rns_init(&r, n, q, count, t)) return -1;
    out[0] = r.m_sk;
    out[1] = r.gamma;
    for (int i = 0; i < r.bsk; i++) out[2 + i] = r.Bsk[i];
    return r.bsk;
}

int orc_rns_op(int op, size_t n, const uint64_t *q, int count, uint64_t t, const uint64_t *in, uint64_t *out) {
    rns_t r;
    if (rns_init(&r, n, q, count, t)) return -1;
    switch (op) {
    case 0: rns_fastbconv_mtilde(&r, in, out); return 0;
    case 1: rns_smmrq(&r, in, out); return 0;
    case 2: rns_fast_floor(&r, in, out); return 0;
    case 3: rns_fastbconv_sk(&r, in, out); return 0;
    case 4: memcpy(out, in, 8 * n * (size_t)count); rns_div_round_last(&r, out); return 0;
    case 5: memcpy(out, in, 8 * n * (size_t)count); return rns_div_round_last_ntt(&r, out);
    case 6: rns_decrypt_scale_round(&r, in, out); return 0;
    case 7: memcpy(out, in, 8 * n * (size_t)count); rns_mod_t_div_last(&r, out); return 0;
    case 8: rns_decrypt_mod_t(&r, in, out); return 0;
    default: return -2;
    }
}

/* Evaluator::bfvMultiply for two size-2 ciphertexts (src/evaluator.cpp:385-624): BEHZ
   steps (1)-(8): lift to q U Bsk U {m~}, Montgomery-reduce to Bsk, NTT in q and
   Bsk, tensor, INTT, multiply by t, fast floor into Bsk, Shenoy-Kumaresan to q. */
int orc_bfv_multiply(size_t n, const uint64_t *q, int count, uint64_t t, const uint64_t *ct1,
                     const uint64_t *ct2, uint64_t *out) {
    rns_t r;
    if (rns_init(&r, n, q, count, t)) return -1;
    int logn = 0;
    while (((size_t)1 << logn) < n) logn++;
    int L = count, bsk = r.bsk;
    size_t pq = n * (size_t)L, pb = n * (size_t)bsk;
    uint64_t *aq = malloc(8 * 2 * pq), *ab = malloc(8 * 2 * pb);
    uint64_t *bq = malloc(8 * 2 * pq), *bb = malloc(8 * 2 * pb);
    uint64_t *tmp = malloc(8 * n * (size_t)(bsk + 1));
    const uint64_t *src[2] = {ct1, ct2};
    uint64_t *dq[2] = {aq, bq}, *db[2] = {ab, bb};
    for (int c = 0; c < 2; c++)
        for (int p = 0; p < 2; p++) {
            const uint64_t *in = src[c] + p * pq;
            memcpy(dq[c] + p * pq, in, 8 * pq);
            orc_ntt_forward_rns(logn, q, L, dq[c] + p * pq, 1);
            rns_fastbconv_mtilde(&r, in, tmp);
            rns_smmrq(&r, tmp, db[c] + p * pb);
            orc_ntt_forward_rns(logn, r.Bsk, bsk, db[c] + p * pb, 1);
        }
    uint64_t *tq = calloc(3 * pq, 8), *tb = calloc(3 * pb, 8);
    /* tensor: d0 = a0 b0, d1 = a0 b1 + a1 b0, d2 = a1 b1 (dyadic on lazy NTT values) */
    for (int k = 0; k < 3; k++) {
        int lo = k < 1 ? 0 : k - 1, hi = k < 1 ? k : 1;
        for (int i = lo; i <= hi; i++) {
            int j = k - i;
            for (int l = 0; l < L; l++)
                for (size_t x = 0; x < n; x++) {
                    uint64_t m = q[l];
                    uint64_t v = mulmod(aq[i * pq + l * n + x], bq[j * pq + l * n + x], m);
                    tq[k * pq + l * n + x] = addmod(tq[k * pq + l * n + x], v, m);
                }
            for (int l = 0; l < bsk; l++)
                for (size_t x = 0; x < n; x++) {
                    uint64_t m = r.Bsk[l];
                    uint64_t v = mulmod(ab[i * pb + l * n + x], bb[j * pb + l * n + x], m);
                    tb[k * pb + l * n + x] = addmod(tb[k * pb + l * n + x], v, m);
                }
        }
    }
    uint64_t *qb = malloc(8 * (pq + pb)), *fl = malloc(8 * pb);
    for (int k = 0; k < 3; k++) {
        orc_ntt_inverse_rns(logn, q, L, tq + k * pq, 1);
        orc_ntt_inverse_rns(logn, r.Bsk, bsk, tb + k * pb, 1);
        for (int l = 0; l < L; l++)
            for (size_t x = 0; x < n; x++) qb[l * n + x] = mulmod(tq[k * pq + l * n + x], t % q[l], q[l]);
        for (int l = 0; l < bsk; l++)
            for (size_t x = 0; x < n; x++)
                qb[pq + l * n + x] = mulmod(tb[k * pb + l * n + x], t % r.Bsk[l], r.Bsk[l]);
        rns_fast_floor(&r, qb, fl);
        rns_fastbconv_sk(&r, fl, out + k * pq);
    }
    free(aq); free(ab); free(bq); free(bb); free(tmp); free(tq); free(tb); free(qb); free(fl);
    return 0;
}

/* ---------------------------------------------------------------- Galois */

/* GaloisTool::getEltFromStep (src/utils/galois.cpp:45-88), generator 3 */
uint32_t orc_galois_elt_from_step(int logn, int step) {
    uint32_t n = 1u << logn, m = 2 * n;
    if (step == 0) return m - 1;
    int sign = step < 0;
    uint32_t pos = (uint32_t)(step < 0 ? -step : step);
    if (pos >= (n >> 1)) return 0;
    pos &= m - 1;
    uint32_t s = sign ? (n >> 1) - pos : pos;
    uint64_t elt = 1;
    while (s--) elt = (elt * 3) & (m - 1);
    return (uint32_t)elt;
}

/* GaloisTool::applyGalois, coefficient domain X -> X^elt with negacyclic sign
   (src/utils/galois.cpp:143-165) */
void orc_apply_galois(int logn, uint32_t elt, uint64_t q, const uint64_t *in, uint64_t *out) {
    uint64_t n = (uint64_t)1 << logn, mask = n - 1, raw = 0;
    for (uint64_t i = 0; i < n; i++, raw += elt) {
        uint64_t idx = raw & mask, v = in[i];
        if ((raw >> logn) & 1) v = negmod(v, q);
        out[idx] = v;
    }
}

/* GaloisTool::applyGaloisNtt with the table of generateTableNtt (src/utils/galois.cpp:18-43,167-177) */
void orc_apply_galois_ntt(int logn, uint32_t elt, const uint64_t *in, uint64_t *out) {
    uint32_t n = 1u << logn;
    for (uint32_t i = 0; i < n; i++) {
        uint32_t rev = bitrev(n + i, logn + 1);
        uint64_t raw = ((uint64_t)elt * rev) >> 1;
        raw &= (uint64_t)(n - 1);
        out[i] = in[bitrev((uint32_t)raw, logn)];
    }
}

/* ------------------------------------------------------------ key switch */

/* Evaluator::switchKeyInplace (src/evaluator.cpp:2310-2653). The inner products are
   accumulated exactly (128-bit) and reduced once; the reference's lazy 128-bit
   accumulation with a reduction every 256 terms yields the same residues. */
int orc_keyswitch(int scheme, int logn, const uint64_t *km, int L, uint64_t t, const uint64_t *target,
                  uint64_t *ct, const uint64_t *key) {
    size_t n = (size_t)1 << logn;
    int K = L + 1;
    tables_t tb[65];
    for (int i = 0; i < K; i++)
        if (build_tables(logn, km[i], &tb[i])) return -1;
    uint64_t *tt = malloc(8 * n * (size_t)L);
    memcpy(tt, target, 8 * n * (size_t)L);
    if (scheme == 2)
        for (int j = 0; j < L; j++) ntt_inverse_t(&tb[j], tt + j * n, 0);
    uint64_t *prod = calloc(2 * (size_t)K * n, 8); /* [2][K][n] */
    uint64_t *tn = malloc(8 * n);
    u128 *acc = malloc(sizeof(u128) * 2 * n);
    for (int i = 0; i < K; i++) {
        int ki = i == L ? K - 1 : i;
        uint64_t qi = km[ki];
        memset(acc, 0, sizeof(u128) * 2 * n);
        for (int j = 0; j < L; j++) {
            const uint64_t *op;
            if (scheme == 2 && i == j) {
                op = target + j * n;
            } else {
                for (size_t x = 0; x < n; x++) tn[x] = km[j] <= qi ? tt[j * n + x] : tt[j * n + x] % qi;
                ntt_forward_t(&tb[ki], tn, 1);
                op = tn;
            }
            for (int c = 0; c < 2; c++) {
                const uint64_t *kp = key + ((size_t)j * 2 + c) * K * n + (size_t)ki * n;
                for (size_t x = 0; x < n; x++) acc[c * n + x] += ((u128)op[x] * kp[x]) % qi;
            }
        }
        for (int c = 0; c < 2; c++)
            for (size_t x = 0; x < n; x++) prod[((size_t)c * K + i) * n + x] = (uint64_t)(acc[c * n + x] % qi);
    }
    uint64_t qk = km[K - 1], qk_half = qk >> 1;
    for (int c = 0; c < 2; c++) {
        uint64_t *last = prod + ((size_t)c * K + L) * n;
        uint64_t *dst = ct + (size_t)c * L * n;
        if (scheme == 3) {
            /* BGV mod-down with the t-correction (src/evaluator.cpp:2528-2583) */
            ntt_inverse_t(&tb[K - 1], last, 0);
            uint64_t inv_qk_t = invmod(qk % t, t);
            uint64_t *k = malloc(8 * n);
            for (size_t x = 0; x < n; x++) {
                k[x] = negmod(last[x] % t, t);
                if (inv_qk_t != 1) k[x] = mulmod(k[x], inv_qk_t, t);
            }
            for (int j = 0; j < L; j++) {
                uint64_t qj = km[j];
                uint64_t *p = prod + ((size_t)c * K + j) * n;
                ntt_inverse_t(&tb[j], p, 0);
                uint64_t inv = invmod(qk % qj, qj);
                for (size_t x = 0; x < n; x++) {
                    uint64_t delta = mulmod(k[x] % qj, qk % qj, qj);
                    uint64_t cm = last[x] % qj;
                    uint64_t v = p[x] + 2 * qj - (delta + cm);
                    v = mulmod(v % qj, inv, qj);
                    dst[j * n + x] = addmod(v, dst[j * n + x], qj);
                }
            }
            free(k);
        } else {
            /* BFV / CKKS mod-down with rounding (src/evaluator.cpp:2584-2650) */
            ntt_inverse_t(&tb[K - 1], last, 1);
            for (size_t x = 0; x < n; x++) last[x] = (last[x] + qk_half) % qk;
            for (int j = 0; j < L; j++) {
                uint64_t qj = km[j];
                uint64_t *p = prod + ((size_t)c * K + j) * n;
                for (size_t x = 0; x < n; x++) tn[x] = qk > qj ? last[x] % qj : last[x];
                uint64_t fix = qj - (qk_half % qj);
                for (size_t x = 0; x < n; x++) tn[x] += fix;
                uint64_t qj_lazy = qj << 1;
                if (scheme == 2) {
                    ntt_forward_t(&tb[j], tn, 1);
                    qj_lazy = qj << 2;
                } else {
                    ntt_inverse_t(&tb[j], p, 1);
                }
                uint64_t inv = invmod(qk % qj, qj), invq = shoup_quotient(inv, qj);
                for (size_t x = 0; x < n; x++) {
                    uint64_t v = p[x] + (qj_lazy - tn[x]);
                    v = mul_shoup(v, inv, invq, qj);
                    dst[j * n + x] = addmod(v, dst[j * n + x], qj);
                }
            }
        }
    }
    for (int i = 0; i < K; i++) free_tables(&tb[i]);
    free(tt); free(prod); free(tn); free(acc);
    return 0;
}

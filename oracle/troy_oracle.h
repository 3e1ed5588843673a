/*
 * CPU restatement of the reference's ciphertext-arithmetic hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the oracle the CUDA path is checked against:
 * it is loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline leg, never by the product. Every function restates the reference
 * routine cited beside it (paths relative to the reference project). All
 * results are exact 64-bit modular integer arithmetic (unsigned __int128 for
 * products); where the reference keeps values in a lazy range, the oracle
 * reproduces the same lazy values so lazy outputs can be compared too.
 *
 * Layout conventions follow the reference: a polynomial over L moduli is
 * uint64 [L][N]; a ciphertext is [size][L][N]; a key-switching key is
 * [digit][2][L+1][N] (one PublicKey per decomposition digit).
 */
#ifndef TROY_ORACLE_H
#define TROY_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* number theory / parameters */
int orc_get_primes(uint64_t factor, int bit_size, size_t count, uint64_t *out);
int orc_coeff_modulus_create(size_t n, const int *bits, int count, uint64_t *out);
int orc_plain_modulus_batching(size_t n, int bits, uint64_t *out);
uint64_t orc_minimal_root(uint64_t degree, uint64_t q);

/* NTT */
int orc_ntt_tables(int logn, uint64_t q, uint64_t *root_op, uint64_t *root_quo, uint64_t *inv_op,
                   uint64_t *inv_quo, uint64_t *inv_n);
int orc_ntt_forward(int logn, uint64_t q, uint64_t *data, int lazy);
int orc_ntt_inverse(int logn, uint64_t q, uint64_t *data, int lazy);
/* same transforms over [count][n] with moduli[count] */
int orc_ntt_forward_rns(int logn, const uint64_t *moduli, int count, uint64_t *data, int lazy);
int orc_ntt_inverse_rns(int logn, const uint64_t *moduli, int count, uint64_t *data, int lazy);

/* element-wise polynomial arithmetic over [count][n] */
void orc_dyadic_product(uint64_t q, const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n);
void orc_poly_dyadic(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                     uint64_t *out);
void orc_poly_add(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                  uint64_t *out);
void orc_poly_sub(const uint64_t *moduli, int count, size_t n, const uint64_t *a, const uint64_t *b,
                  uint64_t *out);
void orc_poly_negate(const uint64_t *moduli, int count, size_t n, const uint64_t *a, uint64_t *out);
void orc_poly_mul_scalar(const uint64_t *moduli, int count, size_t n, const uint64_t *a, uint64_t scalar,
                         uint64_t *out);

/* PRNG stream and samplers */
void orc_prng_bytes(const uint64_t *seed8, size_t offset, size_t count, uint8_t *out);
/* kind: 0 ternary, 1 cbd, 2 uniform; *offset is the stream position, advanced by what was consumed */
int orc_sample_at(int kind, const uint64_t *seed8, size_t *offset, size_t n, const uint64_t *moduli,
                  int count, uint64_t *out);
int orc_sample(int kind, const uint64_t *seed8, size_t n, const uint64_t *moduli, int count, uint64_t *out);

/* RNS tool (BEHZ, rescale, mod-switch, decrypt); op codes as in the reference shim */
int orc_rns_bases(size_t n, const uint64_t *q, int count, uint64_t t, uint64_t *out);
int orc_rns_op(int op, size_t n, const uint64_t *q, int count, uint64_t t, const uint64_t *in, uint64_t *out);
/* BFV multiply of two size-2 ciphertexts at moduli q[count] -> size-3 */
int orc_bfv_multiply(size_t n, const uint64_t *q, int count, uint64_t t, const uint64_t *ct1,
                     const uint64_t *ct2, uint64_t *out);

/* Galois */
uint32_t orc_galois_elt_from_step(int logn, int step);
void orc_apply_galois(int logn, uint32_t elt, uint64_t q, const uint64_t *in, uint64_t *out);
void orc_apply_galois_ntt(int logn, uint32_t elt, const uint64_t *in, uint64_t *out);

/*
 * Key switching (reference src/evaluator.cpp:2310-2653).
 * scheme 1 bfv, 2 ckks, 3 bgv; key_moduli has L+1 entries (special prime last);
 * target [L][n]; ct [2][L][n] accumulates; key [L][2][L+1][n].
 */
int orc_keyswitch(int scheme, int logn, const uint64_t *key_moduli, int L, uint64_t t, const uint64_t *target,
                  uint64_t *ct, const uint64_t *key);

#ifdef __cplusplus
}
#endif
#endif

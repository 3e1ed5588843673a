/*
 * troy_b200.h - C ABI of the B200 ciphertext-arithmetic library.
 *
 * Plain C: opaque handles, raw device pointers, sizes and a cudaStream_t passed as
 * `void *` (NULL = the legacy default stream). Every function returns a status
 * (TB_OK = 0); tb_last_error() gives the message of the calling thread's last
 * failure. Polynomials are uint64 words laid out [poly][limb][N] as in the
 * reference (src/kernelutils.cu:41); limb l of a level-L ciphertext is modulus
 * chain[l]. Pointers must be 16-byte aligned device memory.
 *
 * Each entry point names the reference interface it replaces. Paths are relative
 * to the reference project (SecretHQ/seal-cuda).
 */
#ifndef TROY_B200_H
#define TROY_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TB_OK = 0,
    TB_ERR_INVALID_ARGUMENT = 1,
    TB_ERR_UNSUPPORTED = 2,
    TB_ERR_CUDA = 3,
    TB_ERR_OUT_OF_MEMORY = 4,
    TB_ERR_NO_KEY = 5,
    TB_ERR_TIMEOUT = 6
};

enum { TB_SCHEME_RAW = 0, TB_SCHEME_BFV = 1, TB_SCHEME_CKKS = 2, TB_SCHEME_BGV = 3 };

typedef struct tb_context tb_context;

/* Message of the calling thread's most recent error ("" if none). */
const char *tb_last_error(void);

/* ------------------------------------------------------------------ context */

/*
 * Creates the device-resident precompute for one parameter set: ring degree n,
 * the key-level coefficient modulus chain (special prime last) and, for BFV/BGV,
 * the plain modulus. Uploads NTT tables for every chain prime, the plain modulus
 * (when 1 mod 2n) and the 61-bit Bsk primes, plus the RNS-tool constants of every
 * chain level. Replaces SEALContextCuda construction with its NTTTablesCuda /
 * RNSToolCuda uploads (src/context_cuda.cuh:28-61, src/utils/rns_cuda.cuh:76-141).
 * scheme TB_SCHEME_RAW creates tables only (raw transforms).
 */
int tb_context_create(int scheme, uint64_t poly_degree, const uint64_t *coeff_moduli, int count,
                      uint64_t plain_modulus, tb_context **out);
int tb_context_destroy(tb_context *ctx);

/*
 * NTT-friendly primes for a chain: for each requested bit size, the largest primes
 * = 1 mod 2n below 2^bits, assigned from the smallest of each size's list first, as
 * CoeffModulus::Create does (src/modulus.cpp:80-118). Host only.
 */
int tb_coeff_modulus_create(uint64_t poly_degree, const int *bit_sizes, int count, uint64_t *out);

/* The batching plain modulus PlainModulus::Batching(n, bits) (src/modulus.h:528). Host only. */
int tb_plain_modulus_batching(uint64_t poly_degree, int bits, uint64_t *out);

/* Moduli with NTT tables, in table order: chain, then t (if batching), then Bsk primes. */
int tb_context_moduli(const tb_context *ctx, uint64_t *out, int capacity, int *count);

/* ------------------------------------------------------------------ transforms */

/*
 * Negacyclic forward NTT of [polys][limbs][n]; limb l uses table modulus first+l.
 * Bit-reversed output, lazy != 0 keeps values in [0, 4q) exactly as
 * nttNegacyclicHarveyLazy. in may equal out.
 * Replaces kernel_util::kNttNegacyclicHarvey[Lazy] (src/kernelutils.cuh:578-603).
 */
int tb_ntt_forward(tb_context *ctx, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs,
                   int lazy, void *stream);

/*
 * Inverse negacyclic NTT (bit-reversed in, natural out, N^-1 folded in); lazy != 0
 * keeps values in [0, 2q). Replaces kernel_util::kInverseNttNegacyclicHarvey[Lazy]
 * (src/kernelutils.cuh:607-632).
 */
int tb_ntt_inverse(tb_context *ctx, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs,
                   int lazy, void *stream);

/* ------------------------------------------------------------- element-wise */

/*
 * out = a * b mod q per limb over [polys][limbs][n]. Replaces
 * kernel_util::kDyadicProductCoeffmod (src/kernelutils.cuh:480-503).
 */
int tb_dyadic_product(tb_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t polys,
                      int first, int limbs, void *stream);

/*
 * Ciphertext tensor product of B pairs of size-2 ciphertexts in the NTT domain:
 * out = (a0 b0, a0 b1 + a1 b0, a1 b1), limbs first..first+L-1. Strides are words
 * between consecutive ciphertexts (0 = packed: 2*L*n in, 3*L*n out); out must not
 * overlap the inputs. This is the CKKS multiply (and the BGV multiply between its
 * transforms). Replaces EvaluatorCuda::ckksMultiply's gDyadicConvolutionCoeffmod
 * launches (src/evaluator_cuda.cu:384-432, src/kernelutils.cu:89).
 */
int tb_tensor_product(tb_context *ctx, int first, int L, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
                      uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);

/*
 * Multiplies `batch` pairs of size-2 ciphertexts at level L into size-3 outputs with
 * the context's scheme: BFV by the BEHZ RNS method (EvaluatorCuda::bfvMultiply,
 * src/evaluator_cuda.cu:283-382, over RNSToolCuda::fastbconvmTilde / smMrq /
 * fastFloor / fastbconvSk, src/utils/rns_cuda.cu:339-443), BGV by NTT-tensor-INTT
 * (src/evaluator_cuda.cu:435-501), CKKS by the NTT-domain tensor
 * (src/evaluator_cuda.cu:384-432). Strides 0 = packed (2*L*n in, 3*L*n out); out must
 * not overlap the inputs. BFV takes up to 64 data limbs.
 */
int tb_multiply(tb_context *ctx, int L, const uint64_t *a, uint64_t a_stride, const uint64_t *b, uint64_t b_stride,
                uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);
/*
 * One product of a size-a_size and a size-b_size ciphertext (2 .. 64 polynomials each,
 * packed [size][L][n]) at level L into a_size + b_size - 1 polynomials at out: the
 * reference's bfvMultiply / bgvMultiply / ckksMultiply for any operand sizes
 * (src/evaluator_cuda.cu:283-501), e.g. an unrelinearized product times another
 * ciphertext. out must not overlap the inputs.
 */
int tb_multiply_sizes(tb_context *ctx, int L, const uint64_t *a, int a_size, const uint64_t *b, int b_size,
                      uint64_t *out, void *stream);

/* ------------------------------------------------------------ key switching */

/*
 * Key-switching key layout: the key-level KSwitchKeys entry of one key, as the
 * reference stores it: [K-1 digits][2 polys][K limbs][n] words in NTT form, K =
 * chain length (src/keygenerator.cpp:294-329, src/kswitchkeys_cuda.cuh:43-56).
 *
 * tb_keyswitch: for each of `batch` ciphertexts at level L (L data limbs, 1 <= L <= K-1)
 * adds switch(target) into the ciphertext's first two polynomials. target[b] has L
 * limbs at target + b*target_stride (NTT form for CKKS, coefficient form for
 * BFV/BGV); ciphertext b at ct + b*ct_stride. Strides in words, 0 = packed.
 * Every target and ciphertext word is a residue below its limb's modulus (as in any
 * valid ciphertext; the transforms take the target words unreduced). The same holds
 * for the ciphertexts of tb_relinearize, tb_apply_galois and tb_multiply.
 * Replaces EvaluatorCuda::switchKeyInplace (src/evaluator_cuda.cu:1164-1363).
 */
int tb_keyswitch(tb_context *ctx, int L, const uint64_t *target, uint64_t target_stride, uint64_t *ct,
                 uint64_t ct_stride, const uint64_t *key, uint64_t batch, void *stream);

/*
 * Relinearizes `batch` size-3 ciphertexts [b][3][L][n] in place (the first two
 * polynomials receive the result; the third is left as is). ct_stride 0 = 3*L*n.
 * key is the RelinKeys entry for s^2. Replaces EvaluatorCuda::relinearizeInternal
 * (src/evaluator_cuda.cu:703-744).
 */
int tb_relinearize(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *key, uint64_t batch,
                   void *stream);

/*
 * tb_relinearize for callers that cannot allocate device memory at call time (for
 * example a serving loop that has budgeted all of HBM up front and must not stall on
 * the allocator or fail a request with an out-of-memory error, or code running while
 * another allocator owns the free memory). No counterpart in the reference: it is an
 * addition of this library. Same arguments and result as tb_relinearize, but it
 * calls no allocator: it works out of a 16 MiB scratch array in the library's device
 * image (held on every GPU that loads the library until exit), one chunk of the
 * batch at a time. A level whose single-ciphertext scratch exceeds 16 MiB is
 * rejected with TB_ERR_INVALID_ARGUMENT (e.g. CKKS N=16384 fits up to L=8). The
 * array's device address is looked up by tb_context_create (which, under lazy module
 * loading, is when the device takes the 16 MiB), so no call of this function loads
 * or allocates anything. All calls share the array: calls that overlap on the GPU
 * race, so serialise them (one stream, one thread at a time).
 */
int tb_relinearize_noalloc(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *key,
                           uint64_t batch, void *stream);

/*
 * Applies the Galois automorphism `galois_elt` to `batch` size-2 ciphertexts and
 * key-switches with that element's Galois key: coefficient-domain permutation for
 * BFV/BGV, NTT-domain permutation for CKKS. in may equal out. Replaces
 * EvaluatorCuda::applyGaloisInplace (src/evaluator_cuda.cu:2011-2104) with
 * GaloisToolCuda::applyGalois[Ntt] (src/utils/galois_cuda.cuh:21-25).
 */
int tb_apply_galois(tb_context *ctx, int L, uint32_t galois_elt, const uint64_t *in, uint64_t in_stride,
                    uint64_t *out, uint64_t out_stride, const uint64_t *key, uint64_t batch, void *stream);

/*
 * Batched rotations with many keys in one pass: `groups` groups of ciphertexts laid
 * out one after another in `in` / `out` (group g has counts[g] ciphertexts), group g
 * rotated by galois_elt elts[g] and key-switched with keys[g] (a host array of device
 * pointers to Galois keys). One launch sequence serves all groups, so a batch that
 * mixes rotation steps fills the GPU like a single-key batch. No counterpart call in
 * the reference (it rotates one ciphertext per call, src/evaluator_cuda.cu:2106-2163).
 */
int tb_apply_galois_groups(tb_context *ctx, int L, int groups, const uint32_t *elts, const uint64_t *counts,
                           const uint64_t *in, uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                           const uint64_t *const *keys, void *stream);

/* Galois element of a rotation step (0 = column swap). Replaces GaloisTool::getEltFromStep
   (src/utils/galois.cpp:45-88). */
int tb_galois_elt_from_step(const tb_context *ctx, int step, uint32_t *elt);

/* ------------------------------------------------------ rescale / mod switch */

/*
 * Divides `batch` ciphertexts of `size` polynomials at level L by the last prime
 * with rounding and drops it (L limbs in, L-1 out): CKKS rescale in the NTT domain
 * (RNSTool::divideAndRoundqLastNttInplace, src/utils/rns.cpp:831), BFV modulus
 * switch (divideAndRoundqLastInplace, :805), BGV modulus switch
 * (modTAndDivideqLastInplace, :1097). Ciphertext b at in + b*in_stride, its
 * polynomials L*n words apart (out: (L-1)*n); strides 0 = packed. in and out must
 * not overlap. Replaces EvaluatorCuda::modSwitchScaleToNext (src/evaluator_cuda.cu:749-824).
 */
int tb_rescale_to_next(tb_context *ctx, int L, const uint64_t *in, uint64_t in_stride, uint64_t *out,
                       uint64_t out_stride, int size, uint64_t batch, void *stream);

/* ------------------------------------------------- keys, encryption, decryption
 *
 * PRNG: `seed8` (8 words) reproduces a Blake2xbPRNGFactory constructed with that
 * seed: every PRNG the operation creates starts that seed's stream at 0, exactly as
 * the reference (src/randomgen.h:412-427), so keys and ciphertexts are word-identical
 * to the reference's. NULL draws fresh random seeds from the host. Secret key
 * [K][N] and public key [2][K][N] are at the key level (NTT form).
 */

/* KeyGenerator::generateSk (src/keygenerator.cpp:47-74): ternary sample, NTT. */
int tb_keygen_secret(tb_context *ctx, const uint64_t *seed8, uint64_t *sk, void *stream);
/* KeyGenerator::generatePk (src/keygenerator.cpp:76-99): symmetric encryption of zero. */
int tb_keygen_public(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint64_t *pk, void *stream);
/* KeyGenerator::createRelinKeys (src/keygenerator.cpp:101-124): key for s^2, [K-1][2][K][N]. */
int tb_keygen_relin(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint64_t *key, void *stream);
/* KeyGenerator::createGaloisKeysInternal (src/keygenerator.cpp:126-170): key for one element. */
int tb_keygen_galois(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint32_t galois_elt,
                     uint64_t *key, void *stream);

/*
 * Asymmetric encryption of `batch` plaintexts at level L (Encryptor::encrypt,
 * src/encryptor_cuda.cu:92-237): BFV/BGV plaintexts are plain_count words mod t each
 * (coefficient form), CKKS plaintexts [L][n] in NTT form; plain_stride words between
 * plaintexts. plain NULL encrypts zero. Output [batch][2][L][n] (ct_stride words apart).
 */
int tb_encrypt(tb_context *ctx, const uint64_t *seed8, const uint64_t *pk, int L, const uint64_t *plain,
               uint64_t plain_stride, uint64_t plain_count, uint64_t *ct, uint64_t ct_stride, uint64_t batch,
               void *stream);
/* Symmetric encryption with the secret key (Encryptor::encryptSymmetric, src/encryptor_cuda.cuh). */
int tb_encrypt_symmetric(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, int L, const uint64_t *plain,
                         uint64_t plain_stride, uint64_t plain_count, uint64_t *ct, uint64_t ct_stride,
                         uint64_t batch, void *stream);
/*
 * Symmetric encryption in the seed-compressed form of the reference's GPU path
 * (EncryptorCuda::encryptSymmetric -> util::encryptZeroSymmetric,
 * src/utils/rlwe_cuda.cu:262-331, saved by CiphertextCuda::save as c0 plus the seed,
 * src/ciphertext_cuda.cu:8-35): the second polynomial is the cuRAND expansion of a
 * 64-bit seed (what tb_expand_seeded and the reference's loader regenerate), seeds[b]
 * (a host array of `batch` words) receives each ciphertext's seed, so only c0 and the
 * seed need to travel. BFV and CKKS; BGV is refused (the reference's loader leaves a
 * BGV c1 in the NTT domain). Waits for the seeds to reach the host.
 */
int tb_encrypt_symmetric_seeded(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, int L,
                                const uint64_t *plain, uint64_t plain_stride, uint64_t plain_count, uint64_t *ct,
                                uint64_t ct_stride, uint64_t *seeds, uint64_t batch, void *stream);
/*
 * The second polynomial ([L][n]) of a seed-compressed ciphertext, regenerated as the
 * reference's GPU loader does (CiphertextCuda::load with a context,
 * src/ciphertext_cuda.cu:157-183): one cuRAND state per coefficient g seeded with
 * g + seed, limb j = (uint64) (curand_uniform_double * q_j); inverse_ntt != 0 (BFV)
 * then takes it out of the NTT domain. seed must be non-zero.
 */
int tb_expand_seeded(tb_context *ctx, int L, uint64_t seed, int inverse_ntt, uint64_t *c1, void *stream);
/*
 * tb_expand_seeded for `count` ciphertexts in one launch: seeds is a device array of
 * count seeds (each non-zero), c1 of ciphertext b goes to c1 + b*c1_stride (0 = L*n).
 * For a server that receives a batch of seed-compressed ciphertexts (c0 and the seed
 * each, half the bytes of full ones); the reference loads them one per call.
 */
int tb_expand_seeded_batch(tb_context *ctx, int L, const uint64_t *seeds, uint64_t count, int inverse_ntt,
                           uint64_t *c1, uint64_t c1_stride, void *stream);
/*
 * Decrypts `batch` ciphertexts of `size` polynomials at level L (DecryptorCuda::decrypt,
 * src/decryptor_cuda.cu:92-328): BFV scale-and-round / BGV exact conversion (times
 * correction^-1) give n words mod t per plaintext; CKKS gives [L][n] in NTT form.
 */
int tb_decrypt(tb_context *ctx, const uint64_t *sk, int L, int size, const uint64_t *ct, uint64_t ct_stride,
               uint64_t *plain, uint64_t plain_stride, uint64_t correction, uint64_t batch, void *stream);

/* ------------------------------------------------------------ batch encoder */

/* BatchEncoderCuda::encode (src/batchencoder_cuda.cu:42-100): `count` <= n slot values
   mod t per plaintext -> n coefficients. Needs an NTT-friendly plain modulus. */
int tb_batch_encode(tb_context *ctx, const uint64_t *slots, uint64_t slot_stride, uint64_t count, uint64_t *plain,
                    uint64_t batch, void *stream);
/* BatchEncoderCuda::decode (src/batchencoder_cuda.cu:182-265): n coefficients -> n slots. */
int tb_batch_decode(tb_context *ctx, const uint64_t *plain, uint64_t *slots, uint64_t slot_stride, uint64_t batch,
                    void *stream);

/* ------------------------------------------------------------ CKKS encoder */

/*
 * CKKSEncoderCuda::encode (src/ckks_cuda.cu:314-453): `count` <= n/2 complex values
 * per plaintext (device doubles, re/im interleaved, value_stride complex numbers
 * apart) -> plaintexts [batch][L][n] in NTT form at level L with the given scale.
 */
int tb_ckks_encode(tb_context *ctx, int L, const double *values, uint64_t value_stride, uint64_t count,
                   double scale, uint64_t *plain, uint64_t batch, void *stream);
/* CKKSEncoderCuda::decode (src/ckks_cuda.cu:900-971): plaintexts [batch][L][n] (NTT form)
   -> n/2 complex values each (value_stride complex numbers apart). */
int tb_ckks_decode(tb_context *ctx, int L, const uint64_t *plain, double scale, double *values,
                   uint64_t value_stride, uint64_t batch, void *stream);

/* CKKSEncoderCuda::encodePolynomial (src/ckks_cuda.cu:455-565): `count` <= n real
   coefficients per plaintext (coeff_stride doubles apart) times scale, rounded, reduced
   and transformed -> [batch][L][n] NTT form. */
int tb_ckks_encode_polynomial(tb_context *ctx, int L, const double *coeffs, uint64_t coeff_stride, uint64_t count,
                              double scale, uint64_t *plain, uint64_t batch, void *stream);
/* CKKSEncoderCuda::decodePolynomial (src/ckks_cuda.cu:983-1040): n real coefficients
   (centred, divided by scale) per plaintext. */
int tb_ckks_decode_polynomial(tb_context *ctx, int L, const uint64_t *plain, double scale, double *coeffs,
                              uint64_t coeff_stride, uint64_t batch, void *stream);
/* CKKSEncoder::encode(double value, scale) (src/ckks.cpp:279-400): round(value*scale) in
   every slot, one plaintext [L][n] in NTT form. */
int tb_ckks_encode_double(tb_context *ctx, int L, double value, double scale, uint64_t *plain, void *stream);
/* CKKSEncoder::encode(int64_t value) (src/ckks.cpp:402-440): the integer in every slot, scale 1. */
int tb_ckks_encode_int64(tb_context *ctx, int L, int64_t value, uint64_t *plain, void *stream);

/* ------------------------------------------------------ plaintext arithmetic */

/*
 * Multiplies `batch` ciphertexts of `size` polynomials at level L by plaintexts
 * (EvaluatorCuda::multiplyPlain, src/evaluator_cuda.cu:1744-1850): BFV/BGV plaintexts
 * of plain_count words mod t (centred lift, NTT, dyadic, inverse NTT), CKKS plaintexts
 * [L][n] in NTT form. plain_stride 0 = one plaintext for every ciphertext.
 */
int tb_multiply_plain(tb_context *ctx, int L, int size, const uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                      uint64_t plain_stride, uint64_t plain_count, uint64_t *out, uint64_t out_stride,
                      uint64_t batch, void *stream);
/* c0 += plaintext (BFV scaled by Delta, BGV reduced, CKKS NTT form) (EvaluatorCuda::addPlain /
   subPlain via scalingvariant_cuda, src/utils/scalingvariant_cuda.cu:21-128). */
int tb_add_plain(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                 uint64_t plain_stride, uint64_t plain_count, uint64_t batch, void *stream);
int tb_sub_plain(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                 uint64_t plain_stride, uint64_t plain_count, uint64_t batch, void *stream);

/* Lifts `batch` BFV/BGV plaintexts (plain_count words mod t) to level L and transforms
   them -> [batch][L][n] NTT form (EvaluatorCuda::transformToNttInplace(Plaintext),
   src/evaluator_cuda.cu:1869-1935). */
int tb_plain_to_ntt(tb_context *ctx, int L, const uint64_t *plain, uint64_t plain_stride, uint64_t plain_count,
                    uint64_t *out, uint64_t batch, void *stream);
/* out = a * scalar mod q_l over `size` polynomials at level L
   (kernel_util::kMultiplyPolyScalarCoeffmod, src/kernelutils.cuh; BGV correction balancing). */
int tb_multiply_scalar(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, uint64_t scalar,
                       uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);
/* out = plain * scalar mod t over `count` words per plaintext (BGV addPlain's correction
   factor, src/evaluator_cuda.cu:1597-1604). */
int tb_plain_multiply_scalar(tb_context *ctx, const uint64_t *plain, uint64_t plain_stride, uint64_t count,
                             uint64_t scalar, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);

/*
 * Sum of plaintext products in the NTT domain, the inner loop of the reference's
 * matrix helpers (MatmulHelper::matmul: multiplyPlain then addInplace per output,
 * app/LinearHelper.cuh:323-346) done as one pass: for each of `outputs` results o,
 *   out[o] = sum_{k = term_offsets[o]} ^{term_offsets[o+1]-1} a[term_a[k]] (.) w[term_w[k]]
 * where a[i] has `size` polynomials of L limbs (a_stride words apart), w[j] one
 * polynomial of L limbs (w_stride apart), out[o] `size` polynomials (out_stride
 * apart); strides 0 = packed. term_offsets / term_a / term_w are DEVICE arrays of
 * uint32 (outputs+1, and one entry per term). Exact: canonical residues of the
 * same sums the reference computes one product at a time.
 */
int tb_dyadic_accumulate(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *w,
                         uint64_t w_stride, uint64_t *out, uint64_t out_stride, const uint32_t *term_offsets,
                         const uint32_t *term_a, const uint32_t *term_w, uint32_t outputs, void *stream);

/*
 * Weight plaintexts of the matrix helpers' coefficient encoding
 * (MatmulHelper::encodeWeightSmall, app/LinearHelper.cuh:230-247) built on the device:
 * `count` plaintexts of n words each. blocks is a DEVICE array of `count` records of
 * 8 uint32: {source word offset (low, high), in, out, input block, output block,
 * first row li, first column lj}; plaintext p takes rows li..li+block-1 and columns
 * lj..lj+block-1 of the row-major in x out matrix at weights + offset, weight (i, j) at
 * coefficient (j - lj) * input_block + input_block - 1 - (i - li), zeros elsewhere.
 */
int tb_matmul_encode_weights(tb_context *ctx, const uint64_t *weights, const uint32_t *blocks, uint64_t count,
                             uint64_t *plain, void *stream);

/* Element-wise ciphertext add / sub / negate over `size` polynomials at level L
   (kernel_util::kAddPolyCoeffmod / kSubPolyCoeffmod / kNegatePolyCoeffmod, src/kernelutils.cuh). */
int tb_add(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
           uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);
int tb_sub(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
           uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream);
int tb_negate(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, uint64_t *out,
              uint64_t out_stride, uint64_t batch, void *stream);

/* ---------------------------------------------------------------- tuning
 *
 * Speed knobs; every setting computes the same words. No counterpart in the reference
 * (its kernels have fixed launch shapes). Settings are process-wide.
 */

/* NTT launch variant for one direction and log2 block size (12..14 have variants 0 to
   5: 0, 1 and 2 the default thread count, half and a quarter of it, each thread taking
   correspondingly more radix-8 groups per pass, fewer threads letting several limbs
   share an SM; 3, 4 and 5 transform a whole limb on a cluster of two CTAs holding half
   of it each, with the thread counts of 0, 1 and 2 for the half block, and launch the
   sub-blocks of longer limbs as 0, 1 and 2). */
int tb_ntt_set_variant(int forward, int log_block, int variant);
int tb_ntt_get_variant(int forward, int log_block, int *variant);
/* On (the default): a launch of whole 2^12..2^14 limbs with at most half as many limbs
   as the device has SMs takes the two-CTA form of its variant (0 -> 3, 1 -> 4, 2 -> 5),
   so small batches (one ciphertext per call) occupy twice as many SMs; off: every launch
   takes the set variant. */
int tb_ntt_set_small_launch_pairs(int on);
/* Times every variant of the context's transform size on `polys` scratch limbs (0 =
   256) with CUDA events on `stream` and keeps the fastest per direction. */
int tb_autotune_ntt(tb_context *ctx, uint64_t polys, void *stream, int *forward_variant, int *inverse_variant);
/* The integer ceiling of the transforms on this device: butterflies per second of the
   lazy Cooley-Tukey butterfly every forward NTT pass runs (Shoup product, conditional
   subtraction, two 64-bit additions), with operands and twiddles in registers and every
   SM at full occupancy, modulo `modulus` (odd, 3 <= modulus < 2^61). One transform of a
   2^logn limb runs (2^logn / 2) * logn butterflies, so a transform kernel's achieved
   rate over this one is its fraction of the integer ceiling. No counterpart in the
   reference. */
int tb_measure_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second);
/* The same rate for the butterfly without the conditional subtraction of its first
   input, which the forward transforms with deferred reductions run at most stages for
   moduli below 2^60. No counterpart in the reference. */
int tb_measure_slack_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second);
/* The same rate for the no-subtraction form's butterfly (moduli below 2^57 in the
   one-CTA forward transforms of the mod-up, the CKKS mod-down and the rescale), whose
   Shoup quotient is estimated from three 32-bit partial products. No counterpart in the
   reference. */
int tb_measure_wide_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second);
/* The device's 64-bit integer multiply throughput in products per second: kind 0 the
   low word (mul.lo.u64), kind 1 the high word (mul.hi.u64), each in long independent
   chains at full occupancy. A Shoup product is one high and two low products, so
   1 / (1 / hi + 2 / lo) bounds the butterflies per second of any transform built on it
   (the bound the measured butterfly rates are set against). No counterpart in the
   reference. */
int tb_measure_mul64_rate(int kind, void *stream, double *products_per_second);
/* Scratch budget of one key-switch launch sequence: a batch whose intermediates exceed
   it is processed in chunks (default 2 GiB, or the TB_KS_SCRATCH_BYTES environment
   value; 0 restores the default). */
int tb_keyswitch_set_budget(uint64_t bytes);
uint64_t tb_keyswitch_get_budget(void);
/* Key switching (relinearize, rotations) of degrees 4096 .. 16384 through one persistent
   launch per step (CTAs that take the next limb from a device counter) instead of one CTA
   per limb; the same words either way. Off by default. No counterpart in the reference. */
int tb_keyswitch_set_persistent(int on);
int tb_keyswitch_get_persistent(void);

/* ----------------------------------------------------------- uneven batches */

/*
 * Batches of ciphertexts with different ring degrees and modulus chains: each shape
 * group is `count` size-2 ciphertext pairs of one context at level L (a, b:
 * [count][2][L][n] device words), multiplied, relinearized with relin_key and rotated
 * by galois_elt with galois_key into out ([count][2][L][n]). The reference drives
 * these operations one ciphertext per call (EvaluatorCuda::multiply /
 * relinearizeInplace / applyGaloisInplace, src/evaluator_cuda.cu:262-382, 703-744,
 * 2011-2163); the batch has no counterpart there. The buffers must stay valid for the
 * batch's lifetime; a captured batch replays on the same buffers.
 */
typedef struct {
    tb_context *ctx;
    int L;
    uint64_t count;
    const uint64_t *a, *b;
    const uint64_t *relin_key, *galois_key;
    uint32_t galois_elt;
    uint64_t *out;
} tb_uneven_group;

typedef struct tb_uneven tb_uneven;

/* Validates the groups (every context on one device) and allocates the products'
   scratch, one stream per group and the events of the fork/join. */
int tb_uneven_create(const tb_uneven_group *groups, int count, tb_uneven **out);
/* Every group's pipeline as batched calls on a stream of its own, forked from and
   joined back to `stream` (asynchronous). */
int tb_uneven_run(tb_uneven *batch, void *stream);
/* The same pipelines one ciphertext per call on `stream`: the reference's usage. */
int tb_uneven_run_per_op(tb_uneven *batch, void *stream);
/* Records tb_uneven_run once as a CUDA graph (after one uncaptured run, so every table
   and pool setting made on first use exists; waits for it). */
int tb_uneven_capture(tb_uneven *batch);
/* One graph launch of the whole captured batch on `stream`. */
int tb_uneven_replay(tb_uneven *batch, void *stream);
/* on != 0: after the groups' products (one stream each), the relinearizations and the
   rotations of every group run with one persistent launch per key-switch step for all
   groups (at most 8 groups, degrees 4096 .. 16384; set before capture). Same words. */
int tb_uneven_set_shapes(tb_uneven *batch, int on);
int tb_uneven_destroy(tb_uneven *batch);

/* ---------------------------------------------------------------- tracing */

/* Per-kernel device time of the library's launches (CUDA events on each launch's
   stream). The reference has no tracing (its timers are host gettimeofday,
   test/timetest.cu:16-57); this is new. */
typedef struct {
    char name[32];
    uint64_t launches;
    double total_ms;
} tb_trace_entry;

/* Starts (on != 0) or stops recording; either way drops what was recorded. */
int tb_trace_enable(int on);
/* Waits for the recorded launches and returns per-name totals; clears the record. */
int tb_trace_collect(tb_trace_entry *out, int capacity, int *count);

#ifdef __cplusplus
}
#endif
#endif

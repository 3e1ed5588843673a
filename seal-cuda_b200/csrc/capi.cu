// The extern "C" boundary (include/troy_b200.h): argument checks, device selection
// and status conversion around the internal launchers.
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <map>
#include <string>

#include "../../include/troy_b200.h"
#include "context.hpp"
#include "hostmath.hpp"

namespace tb {
extern thread_local std::string g_last_error;
int dyadic_product(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t polys, int first,
                   int limbs, cudaStream_t s);
int tensor_product(const Context &c, int first, int L, const uint64_t *a, uint64_t astride, const uint64_t *b,
                   uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s);
int multiply_sizes(const Context &c, int L, const uint64_t *a, int sa, const uint64_t *b, int sb, uint64_t *out,
                   cudaStream_t s);
int multiply(const Context &c, int L, const uint64_t *a, uint64_t astride, const uint64_t *b, uint64_t bstride,
             uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s);
int keyswitch(const Context &c, int L, const uint64_t *target, uint64_t tstride, uint64_t *ct, uint64_t cstride,
              const uint64_t *key, uint64_t B, cudaStream_t s);
int apply_galois(Context &c, int L, uint32_t elt, const uint64_t *in, uint64_t istride, uint64_t *out,
                 uint64_t ostride, const uint64_t *key, uint64_t B, cudaStream_t s);
int galois_elt_from_step(const Context &c, int step, uint32_t *elt);
int relinearize_noalloc(const Context &c, int L, uint64_t *ct3, uint64_t cstride, const uint64_t *key, uint64_t B,
                        cudaStream_t s);
int apply_galois_groups(Context &c, int L, int groups, const uint32_t *elts, const uint64_t *counts,
                        const uint64_t *in, uint64_t istride, uint64_t *out, uint64_t ostride,
                        const uint64_t *const *keys, cudaStream_t s);
void trace_enable(bool on);
int keygen_secret(Context &c, const uint64_t *seed8, uint64_t *sk, cudaStream_t s);
int keygen_public(Context &c, const uint64_t *seed8, const uint64_t *sk, uint64_t *pk, cudaStream_t s);
int keygen_relin(Context &c, const uint64_t *seed8, const uint64_t *sk, uint64_t *out, cudaStream_t s);
int keygen_galois(Context &c, const uint64_t *seed8, const uint64_t *sk, uint32_t elt, uint64_t *out, cudaStream_t s);
int encrypt(Context &c, const uint64_t *seed8, const uint64_t *pk, int L, const uint64_t *plain, uint64_t pstride,
            uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t count, cudaStream_t s);
int encrypt_symmetric(Context &c, const uint64_t *seed8, const uint64_t *sk, int L, const uint64_t *plain,
                      uint64_t pstride, uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t count,
                      cudaStream_t s, uint64_t *seeds);
int decrypt(Context &c, const uint64_t *sk, int L, int size, const uint64_t *ct, uint64_t cstride, uint64_t *out,
            uint64_t ostride, uint64_t correction, uint64_t B, cudaStream_t s);
int expand_seeded(Context &c, int L, uint64_t seed, bool inverse_ntt, uint64_t *c1, cudaStream_t s);
int expand_seeded_batch(Context &c, int L, const uint64_t *seeds, uint64_t count, bool inverse_ntt, uint64_t *c1,
                        uint64_t stride, cudaStream_t s);
int batch_encode(Context &c, const uint64_t *slots, uint64_t sstride, uint32_t count, uint64_t *out, uint64_t B,
                 cudaStream_t s);
int batch_decode(Context &c, const uint64_t *plain, uint64_t *slots, uint64_t sstride, uint64_t B, cudaStream_t s);
int multiply_plain(Context &c, int L, int size, const uint64_t *ct, uint64_t cstride, const uint64_t *plain,
                   uint64_t pstride, uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s);
int ckks_encode(Context &c, int L, const double *values, uint64_t vstride, uint32_t count, double scale, uint64_t *out,
                uint64_t B, cudaStream_t s);
int ckks_decode(Context &c, int L, const uint64_t *plain, double scale, double *values, uint64_t ostride, uint64_t B,
                cudaStream_t s);
int add_sub(const Context &c, int op, int L, int size, const uint64_t *a, uint64_t astride, const uint64_t *b,
            uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s);
int add_plain(Context &c, int L, int negate, uint64_t *ct, uint64_t cstride, const uint64_t *plain, uint64_t pstride,
              uint32_t pcount, uint64_t B, cudaStream_t s);
int trace_collect(std::map<std::string, std::pair<uint64_t, double>> &out);
int multiply_scalar(Context &c, int L, int size, const uint64_t *a, uint64_t astride, uint64_t scalar, uint64_t *out,
                    uint64_t ostride, uint64_t B, cudaStream_t s);
int plain_multiply_scalar(Context &c, const uint64_t *a, uint64_t astride, uint64_t count, uint64_t scalar,
                          uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s);
int plain_to_ntt(Context &c, int L, const uint64_t *plain, uint64_t pstride, uint32_t pcount, uint64_t *out,
                 uint64_t B, cudaStream_t s);
int ckks_encode_polynomial(Context &c, int L, const double *values, uint64_t vstride, uint32_t count, double scale,
                           uint64_t *out, uint64_t B, cudaStream_t s);
int ckks_decode_polynomial(Context &c, int L, const uint64_t *plain, double scale, double *values, uint64_t ostride,
                           uint64_t B, cudaStream_t s);
int ckks_encode_double(Context &c, int L, double value, double scale, uint64_t *out, cudaStream_t s);
int ckks_encode_int64(Context &c, int L, int64_t value, uint64_t *out, cudaStream_t s);
int autotune_ntt(Context &c, uint64_t polys, cudaStream_t s, int *chosen_fwd, int *chosen_inv);
int matmul_encode_weights(Context &c, const uint64_t *weights, const uint32_t *blocks, uint64_t count, uint64_t *out,
                          cudaStream_t s);
int dyadic_accumulate(const Context &c, int L, int size, const uint64_t *a, uint64_t astride, const uint64_t *w,
                      uint64_t wstride, uint64_t *out, uint64_t ostride, const uint32_t *off, const uint32_t *ia,
                      const uint32_t *iw, uint32_t nout, cudaStream_t s);

int rescale_to_next(Context &c, int L, const uint64_t *in, uint64_t cstride_in, uint64_t *out, uint64_t cstride_out,
                    int size, uint64_t B, cudaStream_t s);
}  // namespace tb


using tb::set_error;

namespace {
// Runs f with the context's device current; restores the caller's device.
template <class F>
int on_device(const tb_context *ctx, F &&f) {
    if (!ctx || !ctx->c) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null context");
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ctx->c->device) cudaSetDevice(ctx->c->device);
    int st = f(*ctx->c);
    if (prev != ctx->c->device && prev >= 0) cudaSetDevice(prev);
    return st;
}
inline cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// The transform kernels move coefficient pairs as 16-byte words, so coefficient
// buffers must start on 16-byte boundaries and strides (in words) must be even; a
// call that breaks this is refused here rather than faulting on the device.
int require_vec(std::initializer_list<const void *> ptrs, std::initializer_list<uint64_t> strides) {
    for (const void *p : ptrs)
        if (p && (reinterpret_cast<uintptr_t>(p) & 15u))
            return set_error(tb::TB_ERR_INVALID_ARGUMENT, "device buffers must start on 16-byte boundaries");
    for (uint64_t st : strides)
        if (st & 1) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "strides must be even numbers of words");
    return tb::TB_OK;
}
}  // namespace

extern "C" {

const char *tb_last_error(void) { return tb::g_last_error.c_str(); }

int tb_context_create(int scheme, uint64_t poly_degree, const uint64_t *coeff_moduli, int count,
                      uint64_t plain_modulus, tb_context **out) {
    if (!out) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    tb::Context *c = nullptr;
    int st = tb::context_create(scheme, poly_degree, coeff_moduli, count, plain_modulus, &c);
    if (st != TB_OK) return st;
    *out = new tb_context{c};
    return TB_OK;
}

int tb_context_destroy(tb_context *ctx) {
    if (!ctx) return TB_OK;
    delete ctx->c;
    delete ctx;
    return TB_OK;
}

int tb_coeff_modulus_create(uint64_t poly_degree, const int *bit_sizes, int count, uint64_t *out) {
    using namespace tb::host;
    if (!bit_sizes || !out || count < 1 || count > 64) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "bad bit sizes");
    if (poly_degree < 2 || poly_degree > 131072 || (poly_degree & (poly_degree - 1)))
        return set_error(tb::TB_ERR_INVALID_ARGUMENT, "poly degree must be a power of two in [2, 131072]");
    std::map<int, int> need;
    for (int i = 0; i < count; i++) {
        if (bit_sizes[i] < 2 || bit_sizes[i] > 60) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "bit sizes must be in [2, 60]");
        need[bit_sizes[i]]++;
    }
    std::map<int, std::vector<uint64_t>> lists;
    for (auto &kv : need)
        if (!get_primes(2 * poly_degree, kv.first, (size_t)kv.second, lists[kv.first]))
            return set_error(tb::TB_ERR_INVALID_ARGUMENT, "failed to find enough qualifying primes");
    for (int i = 0; i < count; i++) {
        auto &l = lists[bit_sizes[i]];
        out[i] = l.back();
        l.pop_back();
    }
    return TB_OK;
}

int tb_plain_modulus_batching(uint64_t poly_degree, int bits, uint64_t *out) {
    return tb_coeff_modulus_create(poly_degree, &bits, 1, out);
}

int tb_context_moduli(const tb_context *ctx, uint64_t *out, int capacity, int *count) {
    if (!ctx || !ctx->c || !count) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null argument");
    const auto &m = ctx->c->table_moduli;
    *count = (int)m.size();
    if (out) std::memcpy(out, m.data(), sizeof(uint64_t) * std::min<size_t>(m.size(), capacity > 0 ? capacity : 0));
    return TB_OK;
}

int tb_ntt_forward(tb_context *ctx, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, int lazy,
                   void *stream) {
    if (const int vst = require_vec({in, out}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) { return tb::ntt_forward(c, in, out, polys, first, limbs, lazy != 0, S(stream)); });
}

int tb_ntt_inverse(tb_context *ctx, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, int lazy,
                   void *stream) {
    if (const int vst = require_vec({in, out}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) { return tb::ntt_inverse(c, in, out, polys, first, limbs, lazy != 0, S(stream)); });
}

int tb_dyadic_product(tb_context *ctx, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t polys, int first,
                      int limbs, void *stream) {
    if (const int vst = require_vec({a, b, out}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) { return tb::dyadic_product(c, a, b, out, polys, first, limbs, S(stream)); });
}

int tb_tensor_product(tb_context *ctx, int first, int L, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
                      uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    if (const int vst = require_vec({a, b, out}, {a_stride, b_stride, out_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::tensor_product(c, first, L, a, a_stride, b, b_stride, out, out_stride, batch, S(stream));
    });
}

int tb_multiply(tb_context *ctx, int L, const uint64_t *a, uint64_t a_stride, const uint64_t *b, uint64_t b_stride,
                uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    if (const int vst = require_vec({a, b, out}, {a_stride, b_stride, out_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::multiply(c, L, a, a_stride, b, b_stride, out, out_stride, batch, S(stream));
    });
}

int tb_multiply_sizes(tb_context *ctx, int L, const uint64_t *a, int a_size, const uint64_t *b, int b_size,
                      uint64_t *out, void *stream) {
    if (const int vst = require_vec({a, b, out}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) { return tb::multiply_sizes(c, L, a, a_size, b, b_size, out, S(stream)); });
}

int tb_keyswitch(tb_context *ctx, int L, const uint64_t *target, uint64_t target_stride, uint64_t *ct,
                 uint64_t ct_stride, const uint64_t *key, uint64_t batch, void *stream) {
    if (const int vst = require_vec({target, ct, key}, {target_stride, ct_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::keyswitch(c, L, target, target_stride, ct, ct_stride, key, batch, S(stream));
    });
}

int tb_relinearize(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *key, uint64_t batch,
                   void *stream) {
    if (const int vst = require_vec({ct, key}, {ct_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        const uint64_t stride = ct_stride ? ct_stride : 3ull * L * c.n;
        if (!ct) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer");
        return tb::keyswitch(c, L, ct + 2ull * L * c.n, stride, ct, stride, key, batch, S(stream));
    });
}

int tb_relinearize_noalloc(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *key,
                           uint64_t batch, void *stream) {
    if (const int vst = require_vec({ct, key}, {ct_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::relinearize_noalloc(c, L, ct, ct_stride, key, batch, S(stream));
    });
}

int tb_apply_galois(tb_context *ctx, int L, uint32_t galois_elt, const uint64_t *in, uint64_t in_stride,
                    uint64_t *out, uint64_t out_stride, const uint64_t *key, uint64_t batch, void *stream) {
    if (const int vst = require_vec({in, out, key}, {in_stride, out_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::apply_galois(c, L, galois_elt, in, in_stride, out, out_stride, key, batch, S(stream));
    });
}

int tb_apply_galois_groups(tb_context *ctx, int L, int groups, const uint32_t *elts, const uint64_t *counts,
                           const uint64_t *in, uint64_t in_stride, uint64_t *out, uint64_t out_stride,
                           const uint64_t *const *keys, void *stream) {
    if (const int vst = require_vec({in, out}, {in_stride, out_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::apply_galois_groups(c, L, groups, elts, counts, in, in_stride, out, out_stride, keys, S(stream));
    });
}

int tb_galois_elt_from_step(const tb_context *ctx, int step, uint32_t *elt) {
    if (!ctx || !ctx->c || !elt) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null argument");
    return tb::galois_elt_from_step(*ctx->c, step, elt);
}

int tb_rescale_to_next(tb_context *ctx, int L, const uint64_t *in, uint64_t in_stride, uint64_t *out,
                       uint64_t out_stride, int size, uint64_t batch, void *stream) {
    if (const int vst = require_vec({in, out}, {in_stride, out_stride})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        return tb::rescale_to_next(c, L, in, in_stride, out, out_stride, size, batch, S(stream));
    });
}

int tb_keygen_secret(tb_context *ctx, const uint64_t *seed8, uint64_t *sk, void *stream) {
    if (!sk) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer");
    return on_device(ctx, [&](tb::Context &c) { return tb::keygen_secret(c, seed8, sk, S(stream)); });
}

int tb_keygen_public(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint64_t *pk, void *stream) {
    if (!sk || !pk) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer");
    return on_device(ctx, [&](tb::Context &c) { return tb::keygen_public(c, seed8, sk, pk, S(stream)); });
}

int tb_keygen_relin(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint64_t *key, void *stream) {
    if (!sk || !key) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer");
    return on_device(ctx, [&](tb::Context &c) { return tb::keygen_relin(c, seed8, sk, key, S(stream)); });
}

int tb_keygen_galois(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, uint32_t galois_elt, uint64_t *key,
                     void *stream) {
    if (!sk || !key) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer");
    return on_device(ctx, [&](tb::Context &c) { return tb::keygen_galois(c, seed8, sk, galois_elt, key, S(stream)); });
}

int tb_encrypt(tb_context *ctx, const uint64_t *seed8, const uint64_t *pk, int L, const uint64_t *plain,
               uint64_t plain_stride, uint64_t plain_count, uint64_t *ct, uint64_t ct_stride, uint64_t batch,
               void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (plain_count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
        return tb::encrypt(c, seed8, pk, L, plain, plain_stride, (uint32_t)plain_count, ct, ct_stride, batch, S(stream));
    });
}

int tb_encrypt_symmetric(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, int L, const uint64_t *plain,
                         uint64_t plain_stride, uint64_t plain_count, uint64_t *ct, uint64_t ct_stride,
                         uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (plain_count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
        return tb::encrypt_symmetric(c, seed8, sk, L, plain, plain_stride, (uint32_t)plain_count, ct, ct_stride, batch,
                                     S(stream), nullptr);
    });
}

int tb_encrypt_symmetric_seeded(tb_context *ctx, const uint64_t *seed8, const uint64_t *sk, int L,
                                const uint64_t *plain, uint64_t plain_stride, uint64_t plain_count, uint64_t *ct,
                                uint64_t ct_stride, uint64_t *seeds, uint64_t batch, void *stream) {
    if (!seeds && batch) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null seed array");
    return on_device(ctx, [&](tb::Context &c) {
        if (plain_count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
        return tb::encrypt_symmetric(c, seed8, sk, L, plain, plain_stride, (uint32_t)plain_count, ct, ct_stride, batch,
                                     S(stream), seeds);
    });
}

int tb_expand_seeded_batch(tb_context *ctx, int L, const uint64_t *seeds, uint64_t count, int inverse_ntt,
                           uint64_t *c1, uint64_t c1_stride, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::expand_seeded_batch(c, L, seeds, count, inverse_ntt != 0, c1, c1_stride, S(stream));
    });
}

int tb_expand_seeded(tb_context *ctx, int L, uint64_t seed, int inverse_ntt, uint64_t *c1, void *stream) {
    if (const int vst = require_vec({c1}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) { return tb::expand_seeded(c, L, seed, inverse_ntt != 0, c1, S(stream)); });
}

int tb_decrypt(tb_context *ctx, const uint64_t *sk, int L, int size, const uint64_t *ct, uint64_t ct_stride,
               uint64_t *plain, uint64_t plain_stride, uint64_t correction, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::decrypt(c, sk, L, size, ct, ct_stride, plain, plain_stride, correction, batch, S(stream));
    });
}

int tb_batch_encode(tb_context *ctx, const uint64_t *slots, uint64_t slot_stride, uint64_t count, uint64_t *plain,
                    uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "values_matrix size is too large");
        return tb::batch_encode(c, slots, slot_stride, (uint32_t)count, plain, batch, S(stream));
    });
}

int tb_batch_decode(tb_context *ctx, const uint64_t *plain, uint64_t *slots, uint64_t slot_stride, uint64_t batch,
                    void *stream) {
    return on_device(ctx, [&](tb::Context &c) { return tb::batch_decode(c, plain, slots, slot_stride, batch, S(stream)); });
}

int tb_ckks_encode(tb_context *ctx, int L, const double *values, uint64_t value_stride, uint64_t count,
                   double scale, uint64_t *plain, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (count > c.n / 2) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "values_size is too large");
        return tb::ckks_encode(c, L, values, value_stride, (uint32_t)count, scale, plain, batch, S(stream));
    });
}

int tb_ckks_decode(tb_context *ctx, int L, const uint64_t *plain, double scale, double *values,
                   uint64_t value_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::ckks_decode(c, L, plain, scale, values, value_stride, batch, S(stream));
    });
}

int tb_ckks_encode_polynomial(tb_context *ctx, int L, const double *coeffs, uint64_t coeff_stride, uint64_t count,
                              double scale, uint64_t *plain, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "values_size is too large");
        return tb::ckks_encode_polynomial(c, L, coeffs, coeff_stride, (uint32_t)count, scale, plain, batch, S(stream));
    });
}

int tb_ckks_decode_polynomial(tb_context *ctx, int L, const uint64_t *plain, double scale, double *coeffs,
                              uint64_t coeff_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::ckks_decode_polynomial(c, L, plain, scale, coeffs, coeff_stride, batch, S(stream));
    });
}

int tb_ckks_encode_double(tb_context *ctx, int L, double value, double scale, uint64_t *plain, void *stream) {
    return on_device(ctx, [&](tb::Context &c) { return tb::ckks_encode_double(c, L, value, scale, plain, S(stream)); });
}

int tb_ckks_encode_int64(tb_context *ctx, int L, int64_t value, uint64_t *plain, void *stream) {
    return on_device(ctx, [&](tb::Context &c) { return tb::ckks_encode_int64(c, L, value, plain, S(stream)); });
}

int tb_plain_to_ntt(tb_context *ctx, int L, const uint64_t *plain, uint64_t plain_stride, uint64_t plain_count,
                    uint64_t *out, uint64_t batch, void *stream) {
    if (const int vst = require_vec({out}, {})) return vst;
    return on_device(ctx, [&](tb::Context &c) {
        if (plain_count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
        return tb::plain_to_ntt(c, L, plain, plain_stride, (uint32_t)plain_count, out, batch, S(stream));
    });
}

int tb_multiply_scalar(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, uint64_t scalar,
                       uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::multiply_scalar(c, L, size, a, a_stride, scalar, out, out_stride, batch, S(stream));
    });
}

int tb_plain_multiply_scalar(tb_context *ctx, const uint64_t *plain, uint64_t plain_stride, uint64_t count,
                             uint64_t scalar, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::plain_multiply_scalar(c, plain, plain_stride, count, scalar, out, out_stride, batch, S(stream));
    });
}

int tb_dyadic_accumulate(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *w,
                         uint64_t w_stride, uint64_t *out, uint64_t out_stride, const uint32_t *term_offsets,
                         const uint32_t *term_a, const uint32_t *term_w, uint32_t outputs, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::dyadic_accumulate(c, L, size, a, a_stride, w, w_stride, out, out_stride, term_offsets, term_a,
                                     term_w, outputs, S(stream));
    });
}

int tb_matmul_encode_weights(tb_context *ctx, const uint64_t *weights, const uint32_t *blocks, uint64_t count,
                             uint64_t *plain, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::matmul_encode_weights(c, weights, blocks, count, plain, S(stream));
    });
}

int tb_autotune_ntt(tb_context *ctx, uint64_t polys, void *stream, int *forward_variant, int *inverse_variant) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::autotune_ntt(c, polys, S(stream), forward_variant, inverse_variant);
    });
}

int tb_multiply_plain(tb_context *ctx, int L, int size, const uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                      uint64_t plain_stride, uint64_t plain_count, uint64_t *out, uint64_t out_stride,
                      uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        if (plain_count > c.n) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
        return tb::multiply_plain(c, L, size, ct, ct_stride, plain, plain_stride, (uint32_t)plain_count, out,
                                  out_stride, batch, S(stream));
    });
}

int tb_add_plain(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                 uint64_t plain_stride, uint64_t plain_count, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::add_plain(c, L, 0, ct, ct_stride, plain, plain_stride, (uint32_t)plain_count, batch, S(stream));
    });
}

int tb_sub_plain(tb_context *ctx, int L, uint64_t *ct, uint64_t ct_stride, const uint64_t *plain,
                 uint64_t plain_stride, uint64_t plain_count, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::add_plain(c, L, 1, ct, ct_stride, plain, plain_stride, (uint32_t)plain_count, batch, S(stream));
    });
}

int tb_add(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
           uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::add_sub(c, 0, L, size, a, a_stride, b, b_stride, out, out_stride, batch, S(stream));
    });
}

int tb_sub(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, const uint64_t *b,
           uint64_t b_stride, uint64_t *out, uint64_t out_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::add_sub(c, 1, L, size, a, a_stride, b, b_stride, out, out_stride, batch, S(stream));
    });
}

int tb_negate(tb_context *ctx, int L, int size, const uint64_t *a, uint64_t a_stride, uint64_t *out,
              uint64_t out_stride, uint64_t batch, void *stream) {
    return on_device(ctx, [&](tb::Context &c) {
        return tb::add_sub(c, 2, L, size, a, a_stride, nullptr, 0, out, out_stride, batch, S(stream));
    });
}

int tb_trace_enable(int on) {
    tb::trace_enable(on != 0);
    return TB_OK;
}

int tb_trace_collect(tb_trace_entry *out, int capacity, int *count) {
    if (!count) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null count");
    std::map<std::string, std::pair<uint64_t, double>> m;
    int st = tb::trace_collect(m);
    if (st != TB_OK) return st;
    int k = 0;
    for (auto &kv : m) {
        if (out && k < capacity) {
            std::memset(out[k].name, 0, sizeof(out[k].name));
            std::strncpy(out[k].name, kv.first.c_str(), sizeof(out[k].name) - 1);
            out[k].launches = kv.second.first;
            out[k].total_ms = kv.second.second;
        }
        k++;
    }
    *count = k;
    return TB_OK;
}

}  // extern "C"

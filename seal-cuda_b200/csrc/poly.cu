// Element-wise RNS polynomial kernels (HBM-bound): dyadic products, ciphertext
// tensor products, additions, negation, scalar multiplication.
#include "context.hpp"
#include "trace.cuh"

namespace tb {

// out = a * b mod q over [polys][limbs][n], two coefficients per thread (16-byte ld/st).
__global__ void dyadic_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                              uint64_t *__restrict__ out, const Mod *__restrict__ mods, int first, int limbs,
                              int logn, uint64_t total_pairs) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total_pairs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = i * 2;
        // limb of the coefficient: a 32-bit remainder (polynomial-limb indices fit 32 bits)
        const int l = (int)((uint32_t)(e >> logn) % (uint32_t)limbs);
        const Mod m = mods[first + l];
        const ulonglong2 x = *reinterpret_cast<const ulonglong2 *>(a + e);
        const ulonglong2 y = *reinterpret_cast<const ulonglong2 *>(b + e);
        *reinterpret_cast<ulonglong2 *>(out + e) = make_ulonglong2(mul_mod(x.x, y.x, m), mul_mod(x.y, y.y, m));
    }
}

unsigned grid_for(uint64_t work, int threads) {
    uint64_t g = (work + threads - 1) / threads;
    const uint64_t cap = 148ull * 16;  // 16 resident CTAs per SM, 148 SMs
    return (unsigned)(g < cap ? (g ? g : 1) : cap);
}

int dyadic_product(const Context &c, const uint64_t *a, const uint64_t *b, uint64_t *out, uint64_t polys, int first,
                   int limbs, cudaStream_t s) {
    if (limbs < 1 || first < 0 || first + limbs > (int)c.table_moduli.size())
        return set_error(TB_ERR_INVALID_ARGUMENT, "modulus range outside the context");
    if (!a || !b || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    const uint64_t pairs = polys * limbs * (uint64_t)c.n / 2;
    if (!pairs) return TB_OK;
    TraceScope ts("dyadic", s);
    dyadic_kernel<<<grid_for(pairs, 256), 256, 0, s>>>(a, b, out, c.d_mods, first, limbs, c.logn, pairs);
    return status_from(cudaGetLastError());
}

}  // namespace tb

namespace tb {

void ensure_pool_retains(int device) {
    static bool done[64] = {false};
    if (device < 0 || device >= 64 || done[device]) return;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done[device] = true;
}

// Ciphertext tensor product of two size-2 ciphertexts in the NTT domain
// (Evaluator::ckksMultiply, src/evaluator.cpp:626-702):
// d0 = a0 b0, d1 = a0 b1 + a1 b0, d2 = a1 b1 per limb. CANON: the words are residues
// below q (a valid ciphertext's), so every product is below q^2 and d1's sum below
// 2 q^2, reduce_prod's range; otherwise (lazy transform outputs of the BFV and BGV
// multiplies, any words of tb_tensor_product) the general 128-bit reduction.
template <bool CANON>
__global__ void tensor_kernel(const uint64_t *__restrict__ a, uint64_t astride, const uint64_t *__restrict__ b,
                              uint64_t bstride, uint64_t *__restrict__ out, uint64_t ostride,
                              const Mod *__restrict__ mods, int first, int L, int logn, uint64_t B) {
    const uint64_t per = (uint64_t)L << (logn - 1);  // coefficient pairs per polynomial
    const uint64_t total = B * per;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        // ciphertext and word offset inside its polynomial: one 32-bit division by the
        // limb count (i >> (logn - 1) counts whole limbs) where the index fits 32 bits
        uint64_t cb, w;
        if (total <= 0xffffffffull) {
            const uint32_t limb_idx = (uint32_t)i >> (logn - 1);
            const uint32_t c32 = limb_idx / (uint32_t)L;
            cb = c32;
            w = ((uint64_t)(limb_idx - c32 * (uint32_t)L) << logn) + ((i & ((1ull << (logn - 1)) - 1)) << 1);
        } else {
            cb = i / per;
            w = (i - cb * per) * 2;
        }
        const int l = (int)(w >> logn);
        const Mod m = mods[first + l];
        const uint64_t pl = (uint64_t)L << logn;
        const uint64_t *pa = a + cb * astride + w, *pb = b + cb * bstride + w;
        uint64_t *po = out + cb * ostride + w;
        const ulonglong2 a0 = *reinterpret_cast<const ulonglong2 *>(pa);
        const ulonglong2 a1 = *reinterpret_cast<const ulonglong2 *>(pa + pl);
        const ulonglong2 b0 = *reinterpret_cast<const ulonglong2 *>(pb);
        const ulonglong2 b1 = *reinterpret_cast<const ulonglong2 *>(pb + pl);
        U128 s0{0, 0}, s1{0, 0};
        mac128(s0, a0.x, b1.x);
        mac128(s0, a1.x, b0.x);
        mac128(s1, a0.y, b1.y);
        mac128(s1, a1.y, b0.y);
        if constexpr (CANON) {
            *reinterpret_cast<ulonglong2 *>(po) =
                make_ulonglong2(mul_mod_canon(a0.x, b0.x, m), mul_mod_canon(a0.y, b0.y, m));
            *reinterpret_cast<ulonglong2 *>(po + pl) =
                make_ulonglong2(reduce_prod(s0.hi, s0.lo, m), reduce_prod(s1.hi, s1.lo, m));
            *reinterpret_cast<ulonglong2 *>(po + 2 * pl) =
                make_ulonglong2(mul_mod_canon(a1.x, b1.x, m), mul_mod_canon(a1.y, b1.y, m));
        } else {
            *reinterpret_cast<ulonglong2 *>(po) = make_ulonglong2(mul_mod(a0.x, b0.x, m), mul_mod(a0.y, b0.y, m));
            *reinterpret_cast<ulonglong2 *>(po + pl) =
                make_ulonglong2(reduce128(s0.hi, s0.lo, m), reduce128(s1.hi, s1.lo, m));
            *reinterpret_cast<ulonglong2 *>(po + 2 * pl) = make_ulonglong2(mul_mod(a1.x, b1.x, m), mul_mod(a1.y, b1.y, m));
        }
    }
}

// Tensor product with limb l reduced by mods[l] (chain prefix or a Bsk array); canon:
// every input word is a residue below its modulus.
int tensor_product_mods(const Context &c, const Mod *mods, int L, const uint64_t *a, uint64_t astride,
                        const uint64_t *b, uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B,
                        cudaStream_t s, bool canon) {
    TraceScope ts("tensor", s);
    const unsigned grid = grid_for(B * L * c.n / 2, 256);
    if (canon)
        tensor_kernel<true><<<grid, 256, 0, s>>>(a, astride, b, bstride, out, ostride, mods, 0, L, c.logn, B);
    else
        tensor_kernel<false><<<grid, 256, 0, s>>>(a, astride, b, bstride, out, ostride, mods, 0, L, c.logn, B);
    return status_from(cudaGetLastError());
}

int tensor_product(const Context &c, int first, int L, const uint64_t *a, uint64_t astride, const uint64_t *b,
                   uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s) {
    if (L < 1 || first < 0 || first + L > (int)c.table_moduli.size())
        return set_error(TB_ERR_INVALID_ARGUMENT, "modulus range outside the context");
    if (!a || !b || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    const uint64_t n = c.n;
    if (!astride) astride = 2ull * L * n;
    if (!bstride) bstride = 2ull * L * n;
    if (!ostride) ostride = 3ull * L * n;
    return tensor_product_mods(c, c.d_mods + first, L, a, astride, b, bstride, out, ostride, B, s, false);
}

}  // namespace tb

namespace tb {
namespace {

// out[o] = sum over terms k of output o of a[ia[k]] (.) w[iw[k]]: `size` polynomials
// of L limbs each for a and out, one polynomial of L limbs for w (NTT domain).
// Products are summed in 128 bits and reduced once per 63 terms, so any table
// modulus (< 2^61) is safe; the result is canonical.
__global__ void dyadic_accumulate_kernel(const uint64_t *__restrict__ a, uint64_t astride,
                                         const uint64_t *__restrict__ w, uint64_t wstride, uint64_t *__restrict__ out,
                                         uint64_t ostride, const uint32_t *__restrict__ off,
                                         const uint32_t *__restrict__ ia, const uint32_t *__restrict__ iw,
                                         const Mod *__restrict__ mods, int L, int logn, int size, uint32_t nout) {
    const uint64_t n = 1ull << logn;
    const uint64_t per = (uint64_t)size * L * n;
    const uint64_t total = (uint64_t)nout * per;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total; x += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t o = (uint32_t)(x / per);
        const uint64_t r = x - (uint64_t)o * per;      // (poly, limb, coefficient) inside the output
        const uint64_t lw = r % (L * n);                // (limb, coefficient) inside one polynomial
        const Mod m = mods[lw >> logn];
        U128 acc{0, 0};
        uint64_t folded = 0;
        int pending = 0;
        const uint32_t k1 = off[o + 1];
        for (uint32_t k = off[o]; k < k1; k++) {
            mac128(acc, a[(uint64_t)ia[k] * astride + r], w[(uint64_t)iw[k] * wstride + lw]);
            if (++pending == 63) {
                folded = add_mod(folded, reduce128(acc.hi, acc.lo, m), m.value);
                acc = U128{0, 0};
                pending = 0;
            }
        }
        out[(uint64_t)o * ostride + r] = add_mod(folded, reduce128(acc.hi, acc.lo, m), m.value);
    }
}

}  // namespace

int dyadic_accumulate(const Context &c, int L, int size, const uint64_t *a, uint64_t astride, const uint64_t *w,
                      uint64_t wstride, uint64_t *out, uint64_t ostride, const uint32_t *off, const uint32_t *ia,
                      const uint32_t *iw, uint32_t nout, cudaStream_t s) {
    if (L < 1 || L > (int)c.table_moduli.size() || size < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level or size");
    if (!nout) return TB_OK;
    if (!a || !w || !out || !off || !ia || !iw) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    const uint64_t pl = (uint64_t)L << c.logn;
    if (!astride) astride = size * pl;
    if (!wstride) wstride = pl;
    if (!ostride) ostride = size * pl;
    TraceScope ts("dyadic_accumulate", s);
    dyadic_accumulate_kernel<<<grid_for((uint64_t)nout * size * pl, 256), 256, 0, s>>>(
        a, astride, w, wstride, out, ostride, off, ia, iw, c.d_mods, L, c.logn, size, nout);
    return status_from(cudaGetLastError());
}

}  // namespace tb

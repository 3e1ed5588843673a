// Scheme operations around the evaluator: key generation, encryption, decryption,
// batch encoding, plaintext multiplication and element-wise arithmetic.
//
// Encryption and key generation consume the PRNG stream in the reference's order
// (src/utils/rlwe.cpp:152-357, src/keygenerator.cpp:47-329,
// src/encryptor.cpp:92-237), so with a seeded factory the ciphertext and key words
// are identical to the reference's CPU path.
#include <curand_kernel.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "context.hpp"
#include "hostmath.hpp"
#include "prng.hpp"
#include "trace.cuh"

namespace tb {

unsigned grid_for(uint64_t work, int threads);
void ensure_pool_retains(int device);
int rescale_to_next(Context &c, int L, const uint64_t *in, uint64_t cstride_in, uint64_t *out, uint64_t cstride_out,
                    int size, uint64_t B, cudaStream_t s);
int galois_ntt_table(Context &c, uint32_t elt, const uint32_t **out);

namespace {

struct DevBuf {
    void *p = nullptr;
    cudaStream_t s;
    explicit DevBuf(cudaStream_t st) : s(st) {}
    cudaError_t alloc(size_t bytes) { return cudaMallocAsync(&p, bytes, s); }
    template <class T>
    T *as() const { return (T *)p; }
    ~DevBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// ---------------------------------------------------------------- transforms

// In-place NTT / inverse NTT of P packed polynomials [P][L][N] over table moduli
// first..first+L-1, full (canonical) outputs.
template <bool FWD>
struct InplaceOp {
    uint64_t *buf;
    const Mod *mods;
    int L, logn, lazy;
    struct Ctx {
        NttLimb lm;
        uint64_t *p;
    };
    __device__ Ctx ctx(int b) const {
        Ctx c;
        c.lm = make_limb(mods[b % L], 0);
        c.p = buf + ((size_t)b << logn);
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const { return c.p[e]; }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.p + e);
        a = v.x;
        b = v.y;
    }
    __device__ uint64_t fix(const Ctx &c, uint64_t v) const {
        if (lazy) return v;
        const uint64_t q = c.lm.q;
        if (FWD) v = csub(v, 2 * q);
        return csub(v, q);
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const { c.p[e] = fix(c, v); }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b) const {
        *reinterpret_cast<ulonglong2 *>(c.p + e) = make_ulonglong2(fix(c, a), fix(c, b));
    }
};

template <bool FWD>
cudaError_t transform(const Context &c, uint64_t *buf, uint64_t polys, int first, int L, bool lazy, cudaStream_t s) {
    if (!polys) return cudaSuccess;
    if (c.logn > MAX_LOGB) {  // limbs longer than one CTA's block: the split transform
        const int st = FWD ? ntt_forward(c, buf, buf, polys, first, L, lazy, s)
                           : ntt_inverse(c, buf, buf, polys, first, L, lazy, s);
        return st == TB_OK ? cudaSuccess : cudaErrorUnknown;
    }
    InplaceOp<FWD> op{buf, c.d_mods + first, L, c.logn, lazy ? 1 : 0};
    TraceScope ts(FWD ? "ntt_forward" : "ntt_inverse", s);
    return dispatch_ntt<FWD>(c.logn, op, (unsigned)(polys * L), FWD ? 0 : c.logn, 1, s);
}

// ---------------------------------------------------------------- element-wise

// Index w of a limb-major layout split by units of d limbs of 2^logn words:
// (w / (d << logn), w mod (d << logn)), with a 32-bit division where the limb index fits.
__device__ __forceinline__ void split_limbs(uint64_t w, uint32_t d, int logn, uint64_t &q, uint64_t &r) {
    const uint64_t limb = w >> logn, low = w & ((1ull << logn) - 1);
    if (limb <= 0xffffffffull) {
        const uint32_t l32 = (uint32_t)limb, q32 = l32 / d;
        q = q32;
        r = ((uint64_t)(l32 - q32 * d) << logn) | low;
    } else {
        q = limb / d;
        r = ((limb - q * d) << logn) | low;
    }
}

// Limb of a limb-major index: (w >> logn) mod L, a 32-bit remainder where it fits.
__device__ __forceinline__ int limb_of(uint64_t w, int logn, int L) {
    const uint64_t limb = w >> logn;
    return limb <= 0xffffffffull ? (int)((uint32_t)limb % (uint32_t)L) : (int)(limb % (uint64_t)L);
}

// out[p][l] = a[p][l] (*) b[pb][l] with pb = p / bdiv (broadcast b over ciphertexts).
__global__ void dyadic_bcast_kernel(const uint64_t *__restrict__ a, const uint64_t *__restrict__ b,
                                    uint64_t *__restrict__ out, const Mod *__restrict__ mods, int L, int logn,
                                    uint64_t P, uint64_t bdiv, uint64_t bstride_poly) {
    const uint64_t per = (uint64_t)L << logn;
    const uint64_t total = P * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t p, r;
        split_limbs(w, (uint32_t)L, logn, p, r);
        const int l = (int)(r >> logn);
        const uint64_t pb = (p <= 0xffffffffull && bdiv <= 0xffffffffull) ? (uint32_t)p / (uint32_t)bdiv : p / bdiv;
        const uint64_t bi = pb * bstride_poly + r;
        out[w] = mul_mod(a[w], b[bi], mods[l]);
    }
}

// op: 0 add, 1 sub, 2 negate (b unused); polynomials of B ciphertexts with strides.
__global__ void addsub_kernel(const uint64_t *__restrict__ a, uint64_t astride, const uint64_t *__restrict__ b,
                              uint64_t bstride, uint64_t *__restrict__ out, uint64_t ostride,
                              const Mod *__restrict__ mods, int L, int logn, int size, uint64_t B, int op) {
    const uint64_t per = (uint64_t)size * L << logn;
    const uint64_t total = B * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t cb, r;
        split_limbs(w, (uint32_t)size * (uint32_t)L, logn, cb, r);
        const int l = limb_of(r, logn, L);
        const uint64_t q = mods[l].value;
        const uint64_t x = a[cb * astride + r];
        uint64_t y;
        if (op == 0) y = add_mod(x, b[cb * bstride + r], q);
        else if (op == 1) y = sub_mod(x, b[cb * bstride + r], q);
        else y = neg_mod(x, q);
        out[cb * ostride + r] = y;
    }
}

// x += e (BFV/CKKS) or x += t*e mod q (BGV), over P packed polynomials.
__global__ void add_noise_kernel(uint64_t *__restrict__ x, const uint64_t *__restrict__ e, const Mod *__restrict__ mods,
                                 int L, int logn, uint64_t total, uint64_t t_scale) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const Mod m = mods[limb_of(w, logn, L)];
        uint64_t v = e[w];
        if (t_scale) v = mul_mod(v, reduce64(t_scale, m), m);
        x[w] = add_mod(x[w], v, m.value);
    }
}

// c0 = -(sk * c1 + e) pieces of the symmetric encryption: in: prod = sk*c1 (already),
// e noise; writes c0 = -(prod + e).
__global__ void neg_sum_kernel(uint64_t *__restrict__ c0, const uint64_t *__restrict__ e, const Mod *__restrict__ mods,
                               int L, int logn, uint64_t total, uint64_t t_scale, uint64_t cstride, uint64_t per) {
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / per, r = w - b * per;
        const int l = (int)(r >> logn);
        const Mod m = mods[l];
        uint64_t v = e[w];
        if (t_scale) v = mul_mod(v, reduce64(t_scale, m), m);
        uint64_t *p = c0 + b * cstride + r;
        *p = neg_mod(add_mod(v, *p, m.value), m.value);
    }
}

// BFV: c0 += round(Q m / t) per coefficient (multiplyAddPlainWithScalingVariant,
// src/utils/scalingvariant.cpp:51-81); BGV/CKKS: c0 += m mod q_j.
__global__ void add_plain_kernel(uint64_t *__restrict__ ct, uint64_t cstride, const uint64_t *__restrict__ plain,
                                 uint64_t pstride, uint32_t pcount, const Mod *__restrict__ mods,
                                 const uint64_t *__restrict__ K, RnsOff o, int L, int logn, uint64_t t, int mode,
                                 int negate, uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B * (uint64_t)L * n;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t b, r;
        split_limbs(w, (uint32_t)L, logn, b, r);
        const int l = (int)(r >> logn);
        const uint32_t i = (uint32_t)(r & (n - 1));
        const Mod m = mods[l];
        uint64_t add;
        if (mode == 0) {  // BFV scaling variant
            if (i >= pcount) continue;
            const uint64_t pv = plain[b * pstride + i];
            const uint64_t qmt = K[o.q_mod_t];
            // fix = floor((pv * (Q mod t) + (t + 1) / 2) / t)
            unsigned __int128 num = (unsigned __int128)pv * qmt + ((t + 1) >> 1);
            const uint64_t fix = (uint64_t)(num / t);
            const uint64_t cd = K[o.cdpt + 2 * l], cdq = K[o.cdpt + 2 * l + 1];
            add = add_mod(mul_shoup(pv, cd, cdq, m.value), reduce64(fix, m), m.value);
        } else if (mode == 1) {  // BGV: plain mod q
            if (i >= pcount) continue;
            add = reduce64(plain[b * pstride + i], m);
        } else {  // CKKS: plain [L][N] in NTT form
            add = plain[b * pstride + r];
        }
        uint64_t *p = ct + b * cstride + r;
        *p = negate ? sub_mod(*p, add, m.value) : add_mod(*p, add, m.value);
    }
}

// BFV decryptScaleAndRound (src/utils/rns.cpp:1039-1095), one coefficient per thread.
__global__ void decrypt_scale_round_kernel(const uint64_t *__restrict__ phase, uint64_t *__restrict__ out,
                                           uint64_t ostride, const Mod *__restrict__ mods,
                                           const uint64_t *__restrict__ K, RnsOff o, Mod tm, Mod gm, int L, int logn,
                                           uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        const uint32_t i = (uint32_t)(w & (n - 1));
        const uint64_t *ph = phase + ((b * L) << logn) + i;
        U128 at{0, 0}, ag{0, 0};
        for (int l = 0; l < L; l++) {
            const uint64_t q = mods[l].value;
            uint64_t x = mul_shoup(ph[(size_t)l << logn], K[o.tg_q + 2 * l], K[o.tg_q + 2 * l + 1], q);
            x = mul_shoup(x, K[o.q_ip + 2 * l], K[o.q_ip + 2 * l + 1], q);
            mac128(at, x, K[o.M_qtg + l]);
            mac128(ag, x, K[o.M_qtg + L + l]);
        }
        uint64_t vt = reduce128(at.hi, at.lo, tm), vg = reduce128(ag.hi, ag.lo, gm);
        vt = mul_mod(vt, K[o.neg_inv_q_tg], tm);
        vg = mul_mod(vg, K[o.neg_inv_q_tg + 1], gm);
        const uint64_t t = tm.value, g = gm.value;
        uint64_t d;
        if (vg > (g >> 1)) d = add_mod(vt, reduce64(g - vg, tm), t);
        else d = sub_mod(vt, reduce64(vg, tm), t);
        if (d) d = mul_mod(d, K[o.inv_gamma_t], tm);
        out[b * ostride + i] = d;
    }
}

// BGV decryptModt: exact q -> t conversion with the FP64 rounding sum accumulated in
// the reference's order (BaseConverter::exactConvertArray, src/utils/rns.cpp:461-548),
// then times the inverse correction factor.
__global__ void decrypt_mod_t_kernel(const uint64_t *__restrict__ phase, uint64_t *__restrict__ out, uint64_t ostride,
                                     const Mod *__restrict__ mods, const uint64_t *__restrict__ K, RnsOff o, Mod tm,
                                     int L, int logn, uint64_t inv_corr, uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        const uint32_t i = (uint32_t)(w & (n - 1));
        const uint64_t *ph = phase + ((b * L) << logn) + i;
        double agg = 0.0;
        U128 acc{0, 0};
        for (int l = 0; l < L; l++) {
            const uint64_t q = mods[l].value;
            const uint64_t ip = K[o.q_ip + 2 * l];
            const uint64_t x = ip == 1 ? reduce64(ph[(size_t)l << logn], mods[l])
                                       : mul_shoup(ph[(size_t)l << logn], ip, K[o.q_ip + 2 * l + 1], q);
            agg = __dadd_rn(agg, __ddiv_rn((double)x, (double)q));
            mac128(acc, x, K[o.M_qt + l]);
        }
        agg = __dadd_rn(agg, 0.5);
        const uint64_t v = (uint64_t)agg;
        const uint64_t s = reduce128(acc.hi, acc.lo, tm);
        uint64_t d = sub_mod(s, mul_mod(reduce64(v, tm), K[o.q_mod_t], tm), tm.value);
        if (inv_corr != 1) d = mul_mod(d, inv_corr, tm);
        out[b * ostride + i] = d;
    }
}

// Plain lift of a BFV/BGV plaintext (mod t) into every q_j, centred: values at or
// above (t + 1) / 2 get (Q - t) added (Evaluator::multiplyPlainNormal,
// src/evaluator.cpp:1791-1930); out [B][L][N].
__global__ void plain_lift_kernel(const uint64_t *__restrict__ plain, uint64_t pstride, uint32_t pcount,
                                  uint64_t *__restrict__ out, const Mod *__restrict__ mods,
                                  const uint64_t *__restrict__ K, RnsOff o, uint64_t t, int L, int logn, uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B * ((uint64_t)L << logn);
    const uint64_t thr = (t + 1) >> 1;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / ((uint64_t)L << logn), r = w - b * ((uint64_t)L << logn);
        const int l = (int)(r >> logn);
        const uint32_t i = (uint32_t)(r & (n - 1));
        uint64_t v = 0;
        if (i < pcount) {
            const uint64_t p = plain[b * pstride + i];
            const Mod m = mods[l];
            v = p >= thr ? add_mod(reduce64(p, m), K[o.plain_incr + l], m.value) : reduce64(p, m);
        }
        out[w] = v;
    }
}

// Slot <-> coefficient permutation of the batch encoder (src/batchencoder.cpp:64-82).
__global__ void slot_scatter_kernel(const uint64_t *__restrict__ slots, uint64_t sstride, uint32_t count,
                                    uint64_t *__restrict__ out, const uint32_t *__restrict__ map, uint32_t n,
                                    uint64_t t, uint64_t B) {
    const uint64_t total = B * n;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / n;
        const uint32_t i = (uint32_t)(w - b * n);
        out[b * n + map[i]] = i < count ? slots[b * sstride + i] : 0;
    }
}

__global__ void slot_gather_kernel(const uint64_t *__restrict__ coeffs, uint64_t *__restrict__ slots, uint64_t sstride,
                                   const uint32_t *__restrict__ map, uint32_t n, uint64_t B) {
    const uint64_t total = B * n;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / n;
        const uint32_t i = (uint32_t)(w - b * n);
        slots[b * sstride + i] = coeffs[b * n + map[i]];
    }
}

__global__ void galois_ntt_poly_kernel(const uint64_t *__restrict__ in, uint64_t *__restrict__ out,
                                       const uint32_t *__restrict__ perm, int logn, uint64_t P) {
    const uint64_t total = P << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = w >> logn;
        out[w] = in[(p << logn) + perm[w & ((1u << logn) - 1)]];
    }
}

// key digit i, limb i += new_key_i * (q_special mod q_i)  (generateOneKswitchKey).
__global__ void add_key_term_kernel(uint64_t *__restrict__ keys, const uint64_t *__restrict__ new_key,
                                    const Mod *__restrict__ mods, int K, int logn) {
    const uint32_t n = 1u << logn;
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (e >= n) return;
    const Mod m = mods[i];
    const uint64_t f = reduce64(mods[K - 1].value, m);
    uint64_t *p = keys + ((((size_t)i * 2) * K + i) << logn) + e;
    *p = add_mod(*p, mul_mod(new_key[((size_t)i << logn) + e], f, m), m.value);
}

}  // namespace

// ------------------------------------------------------------ batch encoder map

int slot_map(Context &c, const uint32_t **out) {
    std::lock_guard<std::mutex> g(c.galois_mu);
    static_assert(sizeof(uint32_t) == 4, "");
    if (!c.d_slot_map) {
        const uint32_t n = c.n;
        std::vector<uint32_t> map(n);
        const uint64_t m = 2ull * n;
        uint64_t pos = 1;
        for (uint32_t i = 0; i < n / 2; i++) {
            map[i] = host::bitrev((uint32_t)((pos - 1) >> 1), c.logn);
            map[n / 2 + i] = host::bitrev((uint32_t)((m - pos - 1) >> 1), c.logn);
            pos = (pos * 3) & (m - 1);
        }
        cudaError_t e = cudaMalloc(&c.d_slot_map, n * 4);
        if (e == cudaSuccess) e = cudaMemcpy(c.d_slot_map, map.data(), n * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return status_from(e);
    }
    *out = c.d_slot_map;
    return TB_OK;
}

// ------------------------------------------------------------------ key generation

// sk = NTT(ternary) over the key level (KeyGenerator::generateSk).
int keygen_secret(Context &c, const uint64_t *seed8, uint64_t *sk, cudaStream_t s) {
    const int K = (int)c.chain.size();
    DevBuf st(s);
    cudaError_t e = st.alloc(sizeof(PrngState));
    if (e != cudaSuccess) return status_from(e);
    int r = prng_init(st.as<PrngState>(), 1, seed8, s);
    if (r != TB_OK) return r;
    r = sample_poly(c, SAMPLE_TERNARY, st.as<PrngState>(), 1, 0, K, sk, 0, s);
    if (r != TB_OK) return r;
    return status_from(transform<true>(c, sk, 1, 0, K, false, s));
}

__global__ void seeded_uniform_kernel(uint64_t *c1, const Mod *__restrict__ mods, int L, uint32_t n, uint64_t seed);

// `count` symmetric encryptions of zero at level L in NTT (ntt=1) or coefficient form
// into out[b] ([2][L][N] at out + b*ostride). Every encryption creates its PRNGs from
// the factory (encryptZeroSymmetric, src/utils/rlwe.cpp:232-357).
//
// seeds != nullptr (host array of `count` words): the seed-compressed form of the
// reference's GPU path (util::encryptZeroSymmetric, src/utils/rlwe_cuda.cu:262-331).
// The PRNG keyed by the public seed gives the 64-bit seed (first 32-bit word << 32) +
// second word (the next pair if that is zero), c1 is the cuRAND expansion of it that
// the reference's loader regenerates, and seeds[b] returns it; the call waits for the
// seeds to reach the host.
int encrypt_zero_symmetric(Context &c, const uint64_t *seed8, const uint64_t *sk, int L, bool ntt, uint64_t *out,
                           uint64_t ostride, int count, cudaStream_t s, uint64_t *seeds = nullptr) {
    const uint64_t n = c.n;
    if (!ostride) ostride = 2ull * L * n;
    DevBuf st(s), pub(s), noise(s), sw(s);
    cudaError_t e = st.alloc(sizeof(PrngState) * count);
    if (e == cudaSuccess) e = pub.alloc(sizeof(PrngState) * count);
    if (e == cudaSuccess) e = noise.alloc(8ull * count * L * n);
    if (e == cudaSuccess && seeds) e = sw.alloc(16ull * count);
    if (e != cudaSuccess) return status_from(e);
    PrngState *bs = st.as<PrngState>(), *ps = pub.as<PrngState>();
    int r = prng_init(bs, count, seed8, s);
    if (r != TB_OK) return r;
    // public seed = first 64 bytes of the bootstrap stream; c1 = uniform from it
    e = cudaMemsetAsync(ps, 0, sizeof(PrngState) * count, s);
    if (e != cudaSuccess) return status_from(e);
    for (int b = 0; b < count; b++) {
        r = prng_bytes(bs + b, 64, reinterpret_cast<uint8_t *>(ps + b), s);   // seed is the first member
        if (r != TB_OK) return r;
    }
    if (seeds) {
        uint8_t *words = sw.as<uint8_t>();
        for (int b = 0; b < count; b++) {
            r = prng_bytes(ps + b, 16, words + 16 * b, s);
            if (r != TB_OK) return r;
        }
        std::vector<uint32_t> host(4ull * count);
        e = cudaMemcpyAsync(host.data(), words, 16ull * count, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return status_from(e);
        for (int b = 0; b < count; b++) {
            const uint32_t *w = &host[4ull * b];
            uint64_t sd = ((uint64_t)w[0] << 32) + w[1];
            if (!sd) sd = ((uint64_t)w[2] << 32) + w[3];
            if (!sd) return set_error(TB_ERR_INVALID_ARGUMENT, "ciphertext PRNG gave a zero seed twice");
            seeds[b] = sd;
            seeded_uniform_kernel<<<grid_for(n, 256), 256, 0, s>>>(out + b * ostride + (uint64_t)L * n, c.d_mods, L,
                                                                   (uint32_t)n, sd);
        }
        e = cudaGetLastError();
        if (e != cudaSuccess) return status_from(e);
    } else {
        for (int b = 0; b < count; b++) {
            r = sample_poly(c, SAMPLE_UNIFORM, ps + b, 1, 0, L, out + b * ostride + (uint64_t)L * n, 0, s);
            if (r != TB_OK) return r;
        }
    }
    r = sample_poly(c, SAMPLE_CBD, bs, count, 0, L, noise.as<uint64_t>(), 0, s);
    if (r != TB_OK) return r;
    // c0 = sk * c1 (NTT domain)
    for (int b = 0; b < count; b++) {
        dyadic_bcast_kernel<<<grid_for((uint64_t)L * n, 256), 256, 0, s>>>(out + b * ostride + (uint64_t)L * n, sk,
                                                                         out + b * ostride, c.d_mods, L, c.logn, 1,
                                                                         1, 0);
    }
    if (ntt) {
        e = transform<true>(c, noise.as<uint64_t>(), count, 0, L, false, s);
    } else {
        for (int b = 0; b < count && e == cudaSuccess; b++) e = transform<false>(c, out + b * ostride, 1, 0, L, false, s);
    }
    if (e != cudaSuccess) return status_from(e);
    const uint64_t tsc = c.scheme == SCHEME_BGV ? c.t : 0;
    neg_sum_kernel<<<grid_for((uint64_t)count * L * n, 256), 256, 0, s>>>(out, noise.as<uint64_t>(), c.d_mods, L,
                                                                         c.logn, (uint64_t)count * L * n, tsc,
                                                                         ostride, (uint64_t)L * n);
    if (!ntt)
        for (int b = 0; b < count && e == cudaSuccess; b++)
            e = transform<false>(c, out + b * ostride + (uint64_t)L * n, 1, 0, L, false, s);
    if (e == cudaSuccess) e = cudaGetLastError();
    return status_from(e);
}

int keygen_public(Context &c, const uint64_t *seed8, const uint64_t *sk, uint64_t *pk, cudaStream_t s) {
    return encrypt_zero_symmetric(c, seed8, sk, (int)c.chain.size(), true, pk, 0, 1, s);
}

// Key-switching key for new_key [K][N] (NTT): [K-1][2][K][N] (generateOneKswitchKey).
int keygen_kswitch(Context &c, const uint64_t *seed8, const uint64_t *sk, const uint64_t *new_key, uint64_t *out,
                   cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (K < 2) return set_error(TB_ERR_UNSUPPORTED, "key switching needs a special prime");
    int r = encrypt_zero_symmetric(c, seed8, sk, K, true, out, 0, K - 1, s);
    if (r != TB_OK) return r;
    dim3 g((c.n + 255) / 256, K - 1);
    add_key_term_kernel<<<g, 256, 0, s>>>(out, new_key, c.d_mods, K, c.logn);
    return status_from(cudaGetLastError());
}

int keygen_relin(Context &c, const uint64_t *seed8, const uint64_t *sk, uint64_t *out, cudaStream_t s) {
    const int K = (int)c.chain.size();
    DevBuf s2(s);
    cudaError_t e = s2.alloc(8ull * K * c.n);
    if (e != cudaSuccess) return status_from(e);
    dyadic_bcast_kernel<<<grid_for((uint64_t)K * c.n, 256), 256, 0, s>>>(sk, sk, s2.as<uint64_t>(), c.d_mods, K,
                                                                        c.logn, 1, 1, 0);
    return keygen_kswitch(c, seed8, sk, s2.as<uint64_t>(), out, s);
}

int keygen_galois(Context &c, const uint64_t *seed8, const uint64_t *sk, uint32_t elt, uint64_t *out, cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (!(elt & 1) || elt >= 2 * c.n) return set_error(TB_ERR_INVALID_ARGUMENT, "Galois element is not valid");
    const uint32_t *perm = nullptr;
    int r = galois_ntt_table(c, elt, &perm);
    if (r != TB_OK) return r;
    DevBuf rot(s);
    cudaError_t e = rot.alloc(8ull * K * c.n);
    if (e != cudaSuccess) return status_from(e);
    galois_ntt_poly_kernel<<<grid_for((uint64_t)K * c.n, 256), 256, 0, s>>>(sk, rot.as<uint64_t>(), perm, c.logn, K);
    return keygen_kswitch(c, seed8, sk, rot.as<uint64_t>(), out, s);
}

// ------------------------------------------------------------------ encryption

// Asymmetric encryption of `count` plaintexts at level L (data limbs). BFV/BGV plain:
// [pcount] words mod t per plaintext; CKKS plain: [L][N] NTT form. plain may be null
// (encryption of zero). Encryptor::encryptInternal / encryptZeroInternal.
int encrypt(Context &c, const uint64_t *seed8, const uint64_t *pk, int L, const uint64_t *plain, uint64_t pstride,
            uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t count, cudaStream_t s) {
    const int K = (int)c.chain.size();
    const uint64_t n = c.n;
    if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "encryption needs a scheme context");
    if (L < 1 || L > K) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!pk || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!count) return TB_OK;
    if (!ostride) ostride = 2ull * L * n;
    const bool ckks = c.scheme == SCHEME_CKKS;
    const int Lp = L < K ? L + 1 : L;   // encrypt one level up, then drop its last prime
    ensure_pool_retains(c.device);
    DevBuf st(s), u(s), tmp(s), en(s);
    cudaError_t e = st.alloc(sizeof(PrngState) * count);
    if (e == cudaSuccess) e = u.alloc(8ull * count * Lp * n);
    if (e == cudaSuccess) e = tmp.alloc(8ull * count * 2 * Lp * n);
    if (e == cudaSuccess) e = en.alloc(8ull * count * Lp * n);
    if (e != cudaSuccess) return status_from(e);
    PrngState *ps = st.as<PrngState>();
    int r = prng_init(ps, (int)count, seed8, s);
    if (r != TB_OK) return r;
    TraceScope ts("encrypt", s);
    uint64_t *U = u.as<uint64_t>(), *T = tmp.as<uint64_t>(), *E = en.as<uint64_t>();
    r = sample_poly(c, SAMPLE_TERNARY, ps, (int)count, 0, Lp, U, 0, s);
    if (r != TB_OK) return r;
    e = transform<true>(c, U, count, 0, Lp, false, s);
    if (e != cudaSuccess) return status_from(e);
    // T[b][j] = u * pk_j (pk limbs 0..Lp-1 of the key-level public key)
    for (int j = 0; j < 2; j++) {
        for (uint64_t b = 0; b < count; b++) {
            dyadic_bcast_kernel<<<grid_for((uint64_t)Lp * n, 256), 256, 0, s>>>(
                U + b * Lp * n, pk + (uint64_t)j * K * n, T + (b * 2 + j) * Lp * n, c.d_mods, Lp, c.logn, 1, 1, 0);
        }
    }
    if (!ckks) {
        e = transform<false>(c, T, count * 2, 0, Lp, false, s);
        if (e != cudaSuccess) return status_from(e);
    }
    for (int j = 0; j < 2; j++) {
        r = sample_poly(c, SAMPLE_CBD, ps, (int)count, 0, Lp, E, 0, s);
        if (r != TB_OK) return r;
        if (ckks) e = transform<true>(c, E, count, 0, Lp, false, s);
        if (e != cudaSuccess) return status_from(e);
        const uint64_t tsc = c.scheme == SCHEME_BGV ? c.t : 0;
        for (uint64_t b = 0; b < count; b++)
            add_noise_kernel<<<grid_for((uint64_t)Lp * n, 256), 256, 0, s>>>(T + (b * 2 + j) * Lp * n, E + b * Lp * n,
                                                                           c.d_mods, Lp, c.logn, (uint64_t)Lp * n, tsc);
    }
    if (Lp != L) {
        r = rescale_to_next(c, Lp, T, 2ull * Lp * n, out, ostride, 2, count, s);
        if (r != TB_OK) return r;
    } else {
        e = cudaMemcpy2DAsync(out, ostride * 8, T, 2ull * Lp * n * 8, 2ull * Lp * n * 8, count,
                              cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return status_from(e);
    }
    if (plain) {
        const RnsLevel &lv = c.levels[L];
        const int mode = c.scheme == SCHEME_BFV ? 0 : (c.scheme == SCHEME_BGV ? 1 : 2);
        if (mode == 0 && !lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
        add_plain_kernel<<<grid_for(count * L * n, 256), 256, 0, s>>>(out, ostride, plain, pstride, pcount, c.d_mods,
                                                                      lv.d_consts, lv.off, L, c.logn, c.t, mode, 0,
                                                                      count);
    }
    return status_from(cudaGetLastError());
}

// Symmetric encryption with the secret key at level L (Encryptor::encryptSymmetric).
int encrypt_symmetric(Context &c, const uint64_t *seed8, const uint64_t *sk, int L, const uint64_t *plain,
                      uint64_t pstride, uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t count,
                      cudaStream_t s, uint64_t *seeds) {
    const uint64_t n = c.n;
    if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "encryption needs a scheme context");
    if (seeds && c.scheme == SCHEME_BGV)
        return set_error(TB_ERR_UNSUPPORTED,
                         "seed-compressed BGV ciphertexts are not written: the reference's loader keeps their "
                         "second polynomial in the NTT domain");
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!sk || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!count) return TB_OK;
    if (count > 0x7fffffffull) return set_error(TB_ERR_INVALID_ARGUMENT, "too many ciphertexts in one call");
    if (!ostride) ostride = 2ull * L * n;
    int r = encrypt_zero_symmetric(c, seed8, sk, L, c.scheme == SCHEME_CKKS, out, ostride, (int)count, s, seeds);
    if (r != TB_OK) return r;
    if (plain) {
        const RnsLevel &lv = c.levels[L];
        const int mode = c.scheme == SCHEME_BFV ? 0 : (c.scheme == SCHEME_BGV ? 1 : 2);
        if (mode == 0 && !lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
        add_plain_kernel<<<grid_for(count * L * n, 256), 256, 0, s>>>(out, ostride, plain, pstride, pcount, c.d_mods,
                                                                      lv.d_consts, lv.off, L, c.logn, c.t, mode, 0,
                                                                      count);
    }
    return status_from(cudaGetLastError());
}

// ------------------------------------------------------------------ seeded ciphertexts

// The second polynomial of a seed-compressed ciphertext as the reference's GPU loader
// regenerates it (CiphertextCuda::load, src/ciphertext_cuda.cu:157-183, with
// sampler::setupCurandStates / kSamplePolyUniform, src/utils/rlwe_cuda.cu:25-28,
// 136-151): coefficient g takes a cuRAND XORWOW state initialised with seed g + seed,
// subsequence 0, offset 0, and limb j takes (uint64) (uniform double * q_j). The
// values come from cuRAND itself, called here exactly as there.
__global__ void seeded_uniform_kernel(uint64_t *c1, const Mod *__restrict__ mods, int L, uint32_t n, uint64_t seed) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    curandState st;
    curand_init((unsigned long long)g + seed, 0ull, 0ull, &st);
    for (int j = 0; j < L; j++) c1[g + (size_t)j * n] = (uint64_t)(curand_uniform_double(&st) * (double)mods[j].value);
}

// The second polynomials of `count` seed-compressed ciphertexts at once: ciphertext b's
// seed is seeds[b] (device memory), its c1 goes to c1 + b*stride; the same values as
// expand_seeded per ciphertext.
__global__ void seeded_uniform_batch_kernel(uint64_t *c1, uint64_t stride, const uint64_t *__restrict__ seeds,
                                            const Mod *__restrict__ mods, int L, uint32_t n) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint64_t seed = seeds[blockIdx.y];
    curandState st;
    curand_init((unsigned long long)g + seed, 0ull, 0ull, &st);
    uint64_t *out = c1 + (size_t)blockIdx.y * stride + g;
    for (int j = 0; j < L; j++) out[(size_t)j * n] = (uint64_t)(curand_uniform_double(&st) * (double)mods[j].value);
}

int expand_seeded_batch(Context &c, int L, const uint64_t *seeds, uint64_t count, bool inverse_ntt, uint64_t *c1,
                        uint64_t stride, cudaStream_t s) {
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!count) return TB_OK;
    if (!c1 || !seeds) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (count > 65535) return set_error(TB_ERR_INVALID_ARGUMENT, "at most 65535 ciphertexts per call");
    if (!stride) stride = (uint64_t)L * c.n;
    dim3 grid((unsigned)((c.n + 255) / 256), (unsigned)count);
    seeded_uniform_batch_kernel<<<grid, 256, 0, s>>>(c1, stride, seeds, c.d_mods, L, (uint32_t)c.n);
    cudaError_t e = cudaGetLastError();
    for (uint64_t b = 0; e == cudaSuccess && inverse_ntt && b < count; b++)
        e = transform<false>(c, c1 + b * stride, 1, 0, L, false, s);
    return status_from(e);
}

int expand_seeded(Context &c, int L, uint64_t seed, bool inverse_ntt, uint64_t *c1, cudaStream_t s) {
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!c1) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!seed) return set_error(TB_ERR_INVALID_ARGUMENT, "seed is zero");
    seeded_uniform_kernel<<<grid_for(c.n, 256), 256, 0, s>>>(c1, c.d_mods, L, (uint32_t)c.n, seed);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && inverse_ntt) e = transform<false>(c, c1, 1, 0, L, false, s);
    return status_from(e);
}

// ------------------------------------------------------------------ decryption

// phase = sum_k c_k s^k (NTT domain for CKKS; coefficient form for BFV/BGV)
// (Decryptor::dotProductCtSkArray). out [B][L][N].
static int phase(Context &c, const uint64_t *sk, int L, int size, const uint64_t *ct, uint64_t cstride, uint64_t *out,
                 uint64_t B, cudaStream_t s) {
    const uint64_t n = c.n;
    const bool ckks = c.scheme == SCHEME_CKKS;
    const uint64_t pl = (uint64_t)L * n;
    DevBuf pw(s), tmp(s);
    cudaError_t e = pw.alloc(8ull * pl * 2);   // s^k and scratch
    if (e == cudaSuccess) e = tmp.alloc(8ull * B * size * pl);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *T = tmp.as<uint64_t>();
    e = cudaMemcpy2DAsync(T, size * pl * 8, ct, cstride * 8, size * pl * 8, B, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return status_from(e);
    if (!ckks) {
        e = transform<true>(c, T, B * size, 0, L, false, s);
        if (e != cudaSuccess) return status_from(e);
    }
    // acc = c0; acc += c_k * s^k
    uint64_t *S = pw.as<uint64_t>(), *S2 = S + pl;
    e = cudaMemcpy2DAsync(S, pl * 8, sk, pl * 8, pl * 8, 1, cudaMemcpyDeviceToDevice, s);   // s (first L limbs)
    if (e != cudaSuccess) return status_from(e);
    e = cudaMemcpy2DAsync(out, pl * 8, T, size * pl * 8, pl * 8, B, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return status_from(e);
    for (int k = 1; k < size; k++) {
        for (uint64_t b = 0; b < B; b++) {
            uint64_t *ck = T + (b * size + k) * pl;
            dyadic_bcast_kernel<<<grid_for(pl, 256), 256, 0, s>>>(ck, S, ck, c.d_mods, L, c.logn, 1, 1, 0);
            addsub_kernel<<<grid_for(pl, 256), 256, 0, s>>>(out + b * pl, 0, ck, 0, out + b * pl, 0, c.d_mods, L,
                                                            c.logn, 1, 1, 0);
        }
        if (k + 1 < size) {
            dyadic_bcast_kernel<<<grid_for(pl, 256), 256, 0, s>>>(S, sk, S2, c.d_mods, L, c.logn, 1, 1, 0);
            std::swap(S, S2);
        }
    }
    if (!ckks) {
        e = transform<false>(c, out, B, 0, L, false, s);
        if (e != cudaSuccess) return status_from(e);
    }
    return status_from(cudaGetLastError());
}

// BFV/BGV: plaintext words mod t [B][N] (ostride words apart); CKKS: [B][L][N] NTT form.
int decrypt(Context &c, const uint64_t *sk, int L, int size, const uint64_t *ct, uint64_t cstride, uint64_t *out,
            uint64_t ostride, uint64_t correction, uint64_t B, cudaStream_t s) {
    const uint64_t n = c.n;
    if (c.scheme == SCHEME_RAW) return set_error(TB_ERR_UNSUPPORTED, "decryption needs a scheme context");
    if (L < 1 || L > (int)c.chain.size() || size < 2) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level or size");
    if (!sk || !ct || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!cstride) cstride = (uint64_t)size * L * n;
    ensure_pool_retains(c.device);
    TraceScope ts("decrypt", s);
    if (c.scheme == SCHEME_CKKS) {
        if (!ostride || ostride == (uint64_t)L * n) return phase(c, sk, L, size, ct, cstride, out, B, s);
        DevBuf ph(s);
        cudaError_t e = ph.alloc(8ull * B * L * n);
        if (e != cudaSuccess) return status_from(e);
        int r = phase(c, sk, L, size, ct, cstride, ph.as<uint64_t>(), B, s);
        if (r != TB_OK) return r;
        return status_from(cudaMemcpy2DAsync(out, ostride * 8, ph.p, L * n * 8, L * n * 8, B, cudaMemcpyDeviceToDevice, s));
    }
    if (!ostride) ostride = n;
    const RnsLevel &lv = c.levels[L];
    if (!lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
    DevBuf ph(s);
    cudaError_t e = ph.alloc(8ull * B * L * n);
    if (e != cudaSuccess) return status_from(e);
    int r = phase(c, sk, L, size, ct, cstride, ph.as<uint64_t>(), B, s);
    if (r != TB_OK) return r;
    if (c.scheme == SCHEME_BFV) {
        decrypt_scale_round_kernel<<<grid_for(B * n, 256), 256, 0, s>>>(ph.as<uint64_t>(), out, ostride, c.d_mods,
                                                                       lv.d_consts, lv.off, c.t_mod, lv.gamma_mod, L,
                                                                       c.logn, B);
    } else {
        uint64_t inv = 1;
        if (correction != 1) {
            inv = host::invmod(correction % c.t, c.t);
            if (!inv) return set_error(TB_ERR_INVALID_ARGUMENT, "invalid correction factor");
        }
        decrypt_mod_t_kernel<<<grid_for(B * n, 256), 256, 0, s>>>(ph.as<uint64_t>(), out, ostride, c.d_mods,
                                                                 lv.d_consts, lv.off, c.t_mod, L, c.logn, inv, B);
    }
    return status_from(cudaGetLastError());
}

// ------------------------------------------------------------------ batch encoder

// slots [B][count] (values mod t) -> plaintexts [B][N] (BatchEncoder::encode).
int batch_encode(Context &c, const uint64_t *slots, uint64_t sstride, uint32_t count, uint64_t *out, uint64_t B,
                 cudaStream_t s) {
    if (c.plain_index < 0) return set_error(TB_ERR_UNSUPPORTED, "plain modulus does not support batching");
    if (count > c.n) return set_error(TB_ERR_INVALID_ARGUMENT, "values_matrix size is too large");
    if (!slots || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!sstride) sstride = count;
    const uint32_t *map = nullptr;
    int r = slot_map(c, &map);
    if (r != TB_OK) return r;
    TraceScope ts("batch_encode", s);
    slot_scatter_kernel<<<grid_for(B * c.n, 256), 256, 0, s>>>(slots, sstride, count, out, map, c.n, c.t, B);
    return status_from(transform<false>(c, out, B, c.plain_index, 1, false, s));
}

// plaintexts [B][N] -> slots [B][N] (BatchEncoder::decode).
int batch_decode(Context &c, const uint64_t *plain, uint64_t *slots, uint64_t sstride, uint64_t B, cudaStream_t s) {
    if (c.plain_index < 0) return set_error(TB_ERR_UNSUPPORTED, "plain modulus does not support batching");
    if (!plain || !slots) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!sstride) sstride = c.n;
    const uint32_t *map = nullptr;
    int r = slot_map(c, &map);
    if (r != TB_OK) return r;
    DevBuf tmp(s);
    cudaError_t e = tmp.alloc(8ull * B * c.n);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp.p, plain, 8ull * B * c.n, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = transform<true>(c, tmp.as<uint64_t>(), B, c.plain_index, 1, false, s);
    if (e != cudaSuccess) return status_from(e);
    TraceScope ts("batch_decode", s);
    slot_gather_kernel<<<grid_for(B * c.n, 256), 256, 0, s>>>(tmp.as<uint64_t>(), slots, sstride, map, c.n, B);
    return status_from(cudaGetLastError());
}

// ------------------------------------------------------------------ plain multiply

// ct (size polys, L limbs) times a plaintext: BFV/BGV plaintext [pcount] words mod t
// (lifted, transformed, multiplied, transformed back); CKKS plaintext [L][N] NTT form
// (dyadic). One plaintext per ciphertext (pstride words apart, 0 = shared).
int multiply_plain(Context &c, int L, int size, const uint64_t *ct, uint64_t cstride, const uint64_t *plain,
                   uint64_t pstride, uint32_t pcount, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s) {
    const uint64_t n = c.n;
    if (L < 1 || L > (int)c.chain.size() || size < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level or size");
    if (!ct || !plain || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    const uint64_t pl = (uint64_t)L * n;
    if (!cstride) cstride = size * pl;
    if (!ostride) ostride = size * pl;
    ensure_pool_retains(c.device);
    TraceScope ts("multiply_plain", s);
    const uint64_t nplain = pstride ? B : 1;
    DevBuf pn(s), tmp(s);
    cudaError_t e = tmp.alloc(8ull * B * size * pl);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *T = tmp.as<uint64_t>();
    e = cudaMemcpy2DAsync(T, size * pl * 8, ct, cstride * 8, size * pl * 8, B, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return status_from(e);
    const uint64_t *P = plain;
    if (c.scheme != SCHEME_CKKS) {
        const RnsLevel &lv = c.levels[L];
        if (!lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
        e = pn.alloc(8ull * nplain * pl);
        if (e != cudaSuccess) return status_from(e);
        plain_lift_kernel<<<grid_for(nplain * pl, 256), 256, 0, s>>>(plain, pstride, pcount, pn.as<uint64_t>(),
                                                                    c.d_mods, lv.d_consts, lv.off, c.t, L, c.logn,
                                                                    nplain);
        e = transform<true>(c, pn.as<uint64_t>(), nplain, 0, L, false, s);
        if (e == cudaSuccess) e = transform<true>(c, T, B * size, 0, L, true, s);
        if (e != cudaSuccess) return status_from(e);
        P = pn.as<uint64_t>();
    }
    const uint64_t pstep = pstride ? (c.scheme == SCHEME_CKKS ? pstride : pl) : 0;
    dyadic_bcast_kernel<<<grid_for(B * size * pl, 256), 256, 0, s>>>(T, P, T, c.d_mods, L, c.logn, B * size,
                                                                     pstride ? size : B * size, pstep);
    if (c.scheme != SCHEME_CKKS) {
        e = transform<false>(c, T, B * size, 0, L, false, s);
        if (e != cudaSuccess) return status_from(e);
    }
    e = cudaMemcpy2DAsync(out, ostride * 8, T, size * pl * 8, size * pl * 8, B, cudaMemcpyDeviceToDevice, s);
    return status_from(e);
}

// ------------------------------------------------------------------ add / sub / negate

int add_sub(const Context &c, int op, int L, int size, const uint64_t *a, uint64_t astride, const uint64_t *b,
            uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s) {
    const uint64_t n = c.n;
    if (L < 1 || L > (int)c.table_moduli.size() || size < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level or size");
    if (!a || !out || (op != 2 && !b)) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    const uint64_t per = (uint64_t)size * L * n;
    if (!astride) astride = per;
    if (!bstride) bstride = per;
    if (!ostride) ostride = per;
    TraceScope ts("add_sub", s);
    addsub_kernel<<<grid_for(B * per, 256), 256, 0, s>>>(a, astride, b, bstride, out, ostride, c.d_mods, L, c.logn,
                                                         size, B, op);
    return status_from(cudaGetLastError());
}

// c0 +/- plain for BFV (scaled), BGV (mod q) and CKKS (NTT form) (Evaluator::addPlain/subPlain).
int add_plain(Context &c, int L, int negate, uint64_t *ct, uint64_t cstride, const uint64_t *plain, uint64_t pstride,
              uint32_t pcount, uint64_t B, cudaStream_t s) {
    const uint64_t n = c.n;
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level");
    if (!ct || !plain) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!cstride) cstride = 2ull * L * n;
    const RnsLevel &lv = c.levels[L];
    const int mode = c.scheme == SCHEME_BFV ? 0 : (c.scheme == SCHEME_BGV ? 1 : 2);
    if (mode == 0 && !lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
    add_plain_kernel<<<grid_for(B * L * n, 256), 256, 0, s>>>(ct, cstride, plain, pstride, pcount, c.d_mods,
                                                              lv.d_consts, lv.off, L, c.logn, c.t, mode, negate, B);
    return status_from(cudaGetLastError());
}

}  // namespace tb

namespace tb {

// ------------------------------------------------------------------ scalars, constants

namespace {

// out = a * scalar mod q_l over `size` polys of L limbs (kMultiplyPolyScalarCoeffmod).
__global__ void scalar_mul_kernel(const uint64_t *__restrict__ a, uint64_t astride, uint64_t *__restrict__ out,
                                  uint64_t ostride, uint64_t scalar, const Mod *__restrict__ mods, int L, int logn,
                                  int size, uint64_t B) {
    const uint64_t per = ((uint64_t)size * L) << logn;
    const uint64_t total = B * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / per, r = w - b * per;
        const Mod m = mods[(r >> logn) % L];
        out[b * ostride + r] = mul_mod(reduce64(a[b * astride + r], m), reduce64(scalar, m), m);
    }
}

// words mod t times scalar mod t.
__global__ void scalar_mul_t_kernel(const uint64_t *__restrict__ a, uint64_t astride, uint64_t *__restrict__ out,
                                    uint64_t ostride, uint64_t count, uint64_t scalar, Mod t, uint64_t B) {
    const uint64_t total = B * count;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / count, i = w - b * count;
        out[b * ostride + i] = mul_mod(reduce64(a[b * astride + i], t), reduce64(scalar, t), t);
    }
}

constexpr int MAX_FILL_LIMBS = 64;
struct LimbValues {
    uint64_t v[MAX_FILL_LIMBS];
};

__global__ void fill_limbs_kernel(uint64_t *__restrict__ out, LimbValues vals, int L, int logn, uint64_t B) {
    const uint64_t total = (B * L) << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x)
        out[w] = vals.v[(w >> logn) % L];
}

}  // namespace

int multiply_scalar(Context &c, int L, int size, const uint64_t *a, uint64_t astride, uint64_t scalar, uint64_t *out,
                    uint64_t ostride, uint64_t B, cudaStream_t s) {
    if (L < 1 || L > (int)c.table_moduli.size() || size < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level or size");
    if (!a || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    const uint64_t per = ((uint64_t)size * L) << c.logn;
    if (!astride) astride = per;
    if (!ostride) ostride = per;
    TraceScope ts("multiply_scalar", s);
    scalar_mul_kernel<<<grid_for(B * per, 256), 256, 0, s>>>(a, astride, out, ostride, scalar, c.d_mods, L, c.logn,
                                                             size, B);
    return status_from(cudaGetLastError());
}

int plain_multiply_scalar(Context &c, const uint64_t *a, uint64_t astride, uint64_t count, uint64_t scalar,
                          uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s) {
    if (c.scheme != SCHEME_BFV && c.scheme != SCHEME_BGV) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (!a || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B || !count) return TB_OK;
    if (!astride) astride = count;
    if (!ostride) ostride = count;
    TraceScope ts("multiply_scalar", s);
    scalar_mul_t_kernel<<<grid_for(B * count, 256), 256, 0, s>>>(a, astride, out, ostride, count, scalar, c.t_mod, B);
    return status_from(cudaGetLastError());
}

// Lift `B` plaintexts mod t to level L (centred: values >= (t+1)/2 become value - t
// mod q_l) and transform them: EvaluatorCuda::transformToNttInplace(Plaintext)
// (src/evaluator_cuda.cu:1869-1935). Output [B][L][N], NTT form.
int plain_to_ntt(Context &c, int L, const uint64_t *plain, uint64_t pstride, uint32_t pcount, uint64_t *out,
                 uint64_t B, cudaStream_t s) {
    if (c.scheme != SCHEME_BFV && c.scheme != SCHEME_BGV) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level");
    if (pcount > c.n) return set_error(TB_ERR_INVALID_ARGUMENT, "plaintext longer than the ring degree");
    if (!plain || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!pstride) pstride = pcount;
    const RnsLevel &lv = c.levels[L];
    if (!lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to q");
    const uint64_t pl = (uint64_t)L * c.n;
    TraceScope ts("plain_to_ntt", s);
    plain_lift_kernel<<<grid_for(B * pl, 256), 256, 0, s>>>(plain, pstride, pcount, out, c.d_mods, lv.d_consts,
                                                            lv.off, c.t, L, c.logn, B);
    return status_from(transform<true>(c, out, B, 0, L, false, s));
}

// Every coefficient of limb l of each of B plaintexts [L][N] set to vals[l].
int fill_limbs(Context &c, int L, const uint64_t *vals, uint64_t *out, uint64_t B, cudaStream_t s) {
    if (L < 1 || L > (int)c.chain.size() || L > MAX_FILL_LIMBS) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level");
    if (!out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    LimbValues lv{};
    for (int l = 0; l < L; l++) lv.v[l] = vals[l];
    fill_limbs_kernel<<<grid_for((B * L) << c.logn, 256), 256, 0, s>>>(out, lv, L, c.logn, B);
    return status_from(cudaGetLastError());
}

}  // namespace tb

namespace tb {
namespace {

// One weight plaintext of the matrix helpers' coefficient encoding
// (MatmulHelper::encodeWeightSmall, app/LinearHelper.cuh:230-247): rows li.., columns
// lj.. of a row-major in x out matrix at word offset src; coefficient
// (j - lj) * ib + ib - 1 - (i - li) holds weight (i, j), all others are zero.
struct WeightBlock {
    uint64_t src;
    uint32_t in, out, ib, ob, li, lj;
};

__global__ void weight_scatter_kernel(const uint64_t *__restrict__ weights, const WeightBlock *__restrict__ blocks,
                                      uint64_t *__restrict__ out, int logn, uint64_t count) {
    const uint32_t n = 1u << logn;
    const uint64_t total = count << logn;
    for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < total; x += (uint64_t)gridDim.x * blockDim.x) {
        const WeightBlock b = blocks[x >> logn];
        const uint32_t r = (uint32_t)(x & (n - 1));
        uint64_t v = 0;
        const uint32_t jj = r / b.ib, ii = b.ib - 1 - (r - jj * b.ib);
        const uint32_t i = b.li + ii, j = b.lj + jj;
        if (jj < b.ob && i < b.in && j < b.out && i < b.li + b.ib) v = weights[b.src + (uint64_t)i * b.out + j];
        out[x] = v;
    }
}

}  // namespace

int matmul_encode_weights(Context &c, const uint64_t *weights, const uint32_t *blocks, uint64_t count, uint64_t *out,
                          cudaStream_t s) {
    if (!count) return TB_OK;
    if (!weights || !blocks || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    TraceScope ts("matmul_encode_weights", s);
    weight_scatter_kernel<<<grid_for(count << c.logn, 256), 256, 0, s>>>(
        weights, reinterpret_cast<const WeightBlock *>(blocks), out, c.logn, count);
    return status_from(cudaGetLastError());
}

}  // namespace tb

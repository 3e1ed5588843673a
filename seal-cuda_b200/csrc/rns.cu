// RNS tool kernels: BEHZ base conversions for BFV multiplication, rescale and
// modulus switching, and decryption scale-and-round.
#include "context.hpp"
#include "hostmath.hpp"
#include "trace.cuh"

namespace tb {

int build_level_consts(Context &c, int L);  // multiply.cu

int build_rns_levels(Context &c) {
    using namespace host;
    const int K = (int)c.chain.size();
    c.levels.resize(K + 1);
    for (int L = 1; L <= K; L++) {
        c.levels[L].L = L;
        int st = build_level_consts(c, L);
        if (st != TB_OK) return st;
    }
    // drop-last-prime constants
    std::vector<DropC> drop((size_t)(K + 1) * K);
    for (int Lf = 2; Lf <= K; Lf++) {
        const uint64_t last = c.chain[Lf - 1];
        for (int j = 0; j < Lf - 1; j++) {
            const uint64_t q = c.chain[j];
            DropC d{};
            d.inv = invmod(last % q, q);
            d.inv_quo = shoup(d.inv, q);
            d.half_mod = (last >> 1) % q;
            d.fix = q - d.half_mod;
            d.lastmod = last % q;
            d.lastmod_quo = shoup(d.lastmod, q);
            drop[(size_t)Lf * K + j] = d;
        }
    }
    cudaError_t e = cudaMalloc(&c.d_drop, drop.size() * sizeof(DropC));
    if (e == cudaSuccess) e = cudaMemcpy(c.d_drop, drop.data(), drop.size() * sizeof(DropC), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return status_from(e);
    if (c.t) {
        c.t_mod.value = c.t;
        barrett_ratio(c.t, c.t_mod.ratio_lo, c.t_mod.ratio_hi);
        c.inv_qlast_t.assign(K + 1, 0);
        for (int Lf = 1; Lf <= K; Lf++) c.inv_qlast_t[Lf] = invmod(c.chain[Lf - 1] % c.t, c.t);
    }
    return TB_OK;
}

}  // namespace tb

// ------------------------------------------------------ rescale / mod switch

namespace tb {

unsigned grid_for(uint64_t work, int threads);

namespace {

// Inverse NTT of the last limb of each polynomial, plus (q_last - 1)/2
// (RNSTool::divideAndRoundqLastNttInplace, src/utils/rns.cpp:831-850).
struct LastInttOp {
    const uint64_t *in;
    uint64_t istride;   // words between ciphertexts; polynomials L*N apart
    uint64_t *r;        // [P][N]
    const Mod *mods;
    int L, logn, size;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
        int islack;   // the wide inverse form: outputs below 4q, reduced at the store
    };
    __device__ Ctx ctx(int b) const {
        Ctx c;
        c.lm = make_limb(mods[L - 1], 0);
        c.in = in + (size_t)(b / size) * istride + ((size_t)((b % size) * L + L - 1) << logn);
        c.out = r + ((size_t)b << logn);
        c.islack = 1;
        return c;
    }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const {
        const uint64_t q = c.lm.q;
        v = csub(csub(v, 2 * q), q);      // canonical inverse transform (from below 4q)
        uint64_t x = v + (q >> 1);
        c.out[e] = x >= q ? x - q : x;
    }
};

// out_j = (in_j + 4 q_j - NTT_j((r mod q_j) + fix_j)) * q_last^-1 mod q_j
// (src/utils/rns.cpp:851-875).
struct RescaleNttOp {
    const uint64_t *in;
    uint64_t istride;
    uint64_t *out;
    uint64_t ostride;
    const uint64_t *r;
    const Mod *mods;
    const DropC *drop;
    int L, K, logn, size;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in, *r;
        uint64_t *out;
        uint64_t ratio_hi;
        DropC d;
        int reduce;
        int slack;   // forward transform with deferred reductions
        uint64_t wide_off;   // (floor(2^64 / q_j) - 1) q_j: the epilogue's offset after the wide form
    };
    static constexpr bool wide_slack = true;
    __device__ Ctx ctx(int b) const {
        const int j = b % (L - 1), p = b / (L - 1);
        const Mod &m = mods[j];
        Ctx c;
        c.lm = make_limb(m, 0);
        c.ratio_hi = m.ratio_hi;
        c.d = drop[(size_t)L * K + j];
        c.reduce = mods[L - 1].value > m.value;
        c.slack = (logn <= MAX_LOGB && m.value < (1ull << 57)) ? SLACK_WIDE : m.value < (1ull << 60) ? SLACK_M : 0;
        c.wide_off = (m.ratio_hi - 1) * m.value;
        const size_t cb = p / size, k = p % size;
        c.in = in + cb * istride + ((k * L + j) << logn);
        c.out = out + cb * ostride + ((k * (L - 1) + j) << logn);
        c.r = r + ((size_t)p << logn);
        return c;
    }
    // the transform takes any input below 4 q_j: the Barrett remainder (< 2 q_j) plus fix
    // (at most q_j); the no-subtraction form (q_j < 2^57, one CTA per limb) takes r itself
    // (below 2^61) plus fix
    __device__ uint64_t load(const Ctx &c, int e) const {
        uint64_t x = c.r[e];
        if (c.reduce && c.slack != SLACK_WIDE) x = x - mulhi(x, c.ratio_hi) * c.lm.q;
        return x + c.d.fix;
    }
    // epilogue reads of a coefficient pair: the limb being rescaled
    struct Epi {
        ulonglong2 in;
    };
    __device__ Epi epi2(const Ctx &c, int e) const { return {*reinterpret_cast<const ulonglong2 *>(c.in + e)}; }
    __device__ uint64_t fin(const Ctx &c, uint64_t in, uint64_t v) const {
        const uint64_t q = c.lm.q;
        // after deferred reductions v is below 16 q: one subtraction of 8 q keeps
        // in + 8 q - v below 9 q < 2^64 (in + 16 q - v would pass 2^64 for a 60-bit q);
        // after the no-subtraction form v is below 2^61 + 57 q < 2^63.2 < wide_off, and
        // in + wide_off - v stays below 2^64
        const uint64_t x = c.slack == SLACK_WIDE ? in + c.wide_off - v
                           : c.slack ? in + (q << 3) - csub(v, q << 3) : in + (q << 2) - v;
        return mul_shoup(x, c.d.inv, c.d.inv_quo, q);
    }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b, const Epi &p) const {
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(fin(c, p.in.x, a), fin(c, p.in.y, b));
    }
};

// BFV divideAndRoundqLastInplace (src/utils/rns.cpp:805-829) and BGV
// modTAndDivideqLastInplace (src/utils/rns.cpp:1097-1140), coefficient domain.
__global__ void mod_switch_coeff_kernel(const uint64_t *__restrict__ in, uint64_t istride, uint64_t *__restrict__ out,
                                        uint64_t ostride, const Mod *__restrict__ mods,
                                        const DropC *__restrict__ drop, Mod tm, uint64_t inv_qlast_t, int L, int K,
                                        int logn, int bgv, uint64_t P, int size) {
    const uint32_t n = 1u << logn;
    const uint64_t total = P * n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = i >> logn;
        const uint32_t e = (uint32_t)(i & (n - 1));
        // ciphertext and polynomial of p: a 32-bit division where the count fits 32 bits
        uint64_t pc, pk;
        if (P <= 0xffffffffull) {
            const uint32_t c32 = (uint32_t)p / (uint32_t)size;
            pc = c32;
            pk = (uint32_t)p - c32 * (uint32_t)size;
        } else {
            pc = p / size;
            pk = p % size;
        }
        const uint64_t *src = in + pc * istride + ((pk * L) << logn);
        uint64_t *dst = out + pc * ostride + ((pk * (L - 1)) << logn);
        const Mod ml = mods[L - 1];
        const uint64_t ql = ml.value;
        const uint64_t last = src[((size_t)(L - 1) << logn) + e];
        if (!bgv) {
            const uint64_t l2 = add_mod(last, ql >> 1, ql);
            for (int j = 0; j < L - 1; j++) {
                const Mod m = mods[j];
                const DropC d = drop[(size_t)L * K + j];
                const uint64_t t = sub_mod(reduce64(l2, m), d.half_mod, m.value);
                const uint64_t x = sub_mod(src[((size_t)j << logn) + e], t, m.value);
                dst[((size_t)j << logn) + e] = mul_shoup(x, d.inv, d.inv_quo, m.value);
            }
        } else {
            uint64_t k = neg_mod(reduce64(last, tm), tm.value);
            if (inv_qlast_t != 1) k = mul_mod(k, inv_qlast_t, tm);
            for (int j = 0; j < L - 1; j++) {
                const Mod m = mods[j];
                const DropC d = drop[(size_t)L * K + j];
                const uint64_t q = m.value;
                const uint64_t delta = mul_shoup(reduce64(k, m), d.lastmod, d.lastmod_quo, q);
                const uint64_t x = src[((size_t)j << logn) + e] + 2 * q - reduce64(last, m) - delta;
                dst[((size_t)j << logn) + e] = mul_shoup(x, d.inv, d.inv_quo, q);
            }
        }
    }
}

}  // namespace

void ensure_pool_retains(int device);

// Drops the last prime of `size` polynomials of B ciphertexts at level L (L limbs in,
// L-1 limbs out); ciphertext b at in + b*cstride_in, its polynomials L*n apart.
int rescale_to_next(Context &c, int L, const uint64_t *in, uint64_t cstride_in, uint64_t *out, uint64_t cstride_out,
                    int size, uint64_t B, cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (L < 2 || L > K) return set_error(TB_ERR_INVALID_ARGUMENT, "nothing to drop at this level");
    if (!in || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (size < 1) return set_error(TB_ERR_INVALID_ARGUMENT, "ciphertext size must be positive");
    if (B == 0) return TB_OK;
    const uint64_t n = c.n;
    if (!cstride_in) cstride_in = (uint64_t)size * L * n;
    if (!cstride_out) cstride_out = (uint64_t)size * (L - 1) * n;
    const uint64_t P = B * size;
    cudaError_t e;
    if (c.scheme == SCHEME_CKKS) {
        if (c.logn > MAX_FUSED_LOGN) return set_error(TB_ERR_UNSUPPORTED, "fused rescale supports N <= 131072");
        ensure_pool_retains(c.device);
        uint64_t *r = nullptr;
        e = cudaMallocAsync(&r, P * n * 8, s);
        if (e != cudaSuccess) return status_from(e);
        LastInttOp a{in, cstride_in, r, c.d_mods, L, c.logn, size};
        {
            TraceScope ts("rescale_last_intt", s);
            e = dispatch_ntt<false>(c.logn, a, (unsigned)P, c.logn, 1, s);
        }
        if (e == cudaSuccess) {
            TraceScope ts("rescale_ntt", s);
            RescaleNttOp b{in, cstride_in, out, cstride_out, r, c.d_mods, c.d_drop, L, K, c.logn, size};
            e = dispatch_ntt<true>(c.logn, b, (unsigned)(P * (L - 1)), 0, 0, s);
        }
        cudaFreeAsync(r, s);
        return e == cudaSuccess ? TB_OK : status_from(e);
    }
    if (c.scheme != SCHEME_BFV && c.scheme != SCHEME_BGV) return set_error(TB_ERR_UNSUPPORTED, "scheme has no mod switch");
    const int bgv = c.scheme == SCHEME_BGV;
    TraceScope ts("mod_switch", s);
    mod_switch_coeff_kernel<<<grid_for(P * n, 256), 256, 0, s>>>(in, cstride_in, out, cstride_out, c.d_mods,
                                                                  c.d_drop, c.t_mod, bgv ? c.inv_qlast_t[L] : 0, L,
                                                                  K, c.logn, bgv, P, size);
    return status_from(cudaGetLastError());
}

}  // namespace tb

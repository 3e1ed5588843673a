// Ciphertext multiplication for the three schemes.
//
// BFV follows the BEHZ steps of Evaluator::bfvMultiply (src/evaluator.cpp:385-624):
// (1) lift q -> Bsk U {m~} and (2) Montgomery-reduce to Bsk, fused into one kernel
// per coefficient (RNSTool::fastbconvmTilde + smMrq, src/utils/rns.cpp:934-1037);
// (3) NTT in q and Bsk; (4) tensor; (5) inverse NTT; (6)-(8) multiply by t, fast
// floor into Bsk and Shenoy-Kumaresan back to q, fused into one kernel per
// coefficient (RNSTool::fastFloor + fastbconvSk, src/utils/rns.cpp:878-1008).
// BGV: NTT, tensor, inverse NTT (src/evaluator.cpp:704-794). CKKS: tensor only.
#include <algorithm>

#include "context.hpp"
#include "hostmath.hpp"
#include "trace.cuh"

namespace tb {

unsigned grid_for(uint64_t work, int threads);
void ensure_pool_retains(int device);
int tensor_product_mods(const Context &c, const Mod *mods, int L, const uint64_t *a, uint64_t astride,
                        const uint64_t *b, uint64_t bstride, uint64_t *out, uint64_t ostride, uint64_t B,
                        cudaStream_t s, bool canon = false);

// ---------------------------------------------------------- level constants

int build_level_consts(Context &c, int L) {
    using namespace host;
    RnsLevel &lv = c.levels[L];
    const uint64_t t = c.t;
    if (!t) return TB_OK;
    const uint64_t *q = c.chain.data();
    const auto Q = product(q, L);
    const int total_bits = bit_count(Q);
    int bB = L;
    if (32 + bit_count(t) + total_bits >= 61 * L + 61) bB++;
    const int bsk = bB + 1;
    const int ext = (int)c.chain.size() + (c.plain_index >= 0 ? 1 : 0);
    // table_moduli[ext + i] = getPrimes(2N, 61, .)[i] = [m_sk, gamma, B_0, ...]
    if (ext + 2 + bB > (int)c.table_moduli.size()) return set_error(TB_ERR_UNSUPPORTED, "Bsk base too large");
    lv.bB = bB;
    lv.bsk = bsk;
    lv.m_sk = c.table_moduli[ext];
    lv.gamma = c.table_moduli[ext + 1];
    std::vector<uint64_t> Bv(bB), bskv(bsk);
    std::vector<int> bidx(bsk);
    for (int k = 0; k < bB; k++) {
        Bv[k] = c.table_moduli[ext + 2 + k];
        bidx[k] = ext + 2 + k;
    }
    bidx[bB] = ext;
    for (int k = 0; k < bsk; k++) bskv[k] = c.table_moduli[bidx[k]];
    const uint64_t mt = uint64_t(1) << 32, msk = lv.m_sk, gam = lv.gamma;
    barrett_ratio(gam, lv.gamma_mod.ratio_lo, lv.gamma_mod.ratio_hi);
    lv.gamma_mod.value = gam;

    RnsOff &o = lv.off;
    int pos = 0;
    auto take = [&](int words) { int p = pos; pos += words; return p; };
    o.q_mtip = take(2 * L);
    o.q_ip = take(2 * L);
    o.M_qB = take((bsk + 1) * L);
    o.M_qB_fl = take(bsk * L);
    o.Qmt_b = take(2 * bsk);
    o.tc_b = take(2 * bsk);
    o.neg_inv_q_mt = take(1);
    o.Qmod_b = take(2 * bsk);
    o.inv_mt_b = take(2 * bsk);
    o.t_q = take(2 * L);
    o.t_b = take(2 * bsk);
    o.inv_q_b = take(2 * bsk);
    o.B_ip = take(2 * bB);
    o.tq_ip = take(2 * L);
    o.iqb_Bip = take(2 * bB);
    o.M_Bq = take(L * bB);
    o.M_Bmsk = take(bB);
    o.inv_pb_msk = take(2);
    o.pb_q = take(2 * L);
    o.negpb_q = take(2 * L);
    o.tg_q = take(2 * L);
    o.M_qtg = take(2 * L);
    o.neg_inv_q_tg = take(2);
    o.inv_gamma_t = take(1);
    o.M_qt = take(L);
    o.q_mod_t = take(1);
    o.cdpt = take(2 * L);
    o.plain_incr = take(L);
    o.total = pos;
    std::vector<uint64_t> h(pos, 0);
    auto pair = [&](int off, int i, uint64_t v, uint64_t m) {
        h[off + 2 * i] = v;
        h[off + 2 * i + 1] = shoup(v, m);
    };
    bool ok = true;
    for (int i = 0; i < L; i++) {
        const uint64_t ip = invmod(punctured_mod(q, L, i, q[i]), q[i]);
        ok &= ip != 0;
        pair(o.q_ip, i, ip, q[i]);
        pair(o.q_mtip, i, mulmod(mt % q[i], ip, q[i]), q[i]);
        pair(o.t_q, i, t % q[i], q[i]);
        pair(o.tq_ip, i, mulmod(t % q[i], ip, q[i]), q[i]);
        h[o.M_qB + bsk * L + i] = punctured_mod(q, L, i, mt);
        const uint64_t pbq = prod_mod(Bv.data(), bB, q[i]);
        pair(o.pb_q, i, pbq, q[i]);
        pair(o.negpb_q, i, q[i] - pbq, q[i]);
        pair(o.tg_q, i, mulmod(t, gam, q[i]), q[i]);
        h[o.M_qtg + i] = punctured_mod(q, L, i, t);
        h[o.M_qtg + L + i] = punctured_mod(q, L, i, gam);
        h[o.M_qt + i] = punctured_mod(q, L, i, t);
        for (int k = 0; k < bB; k++) h[o.M_Bq + i * bB + k] = punctured_mod(Bv.data(), bB, k, q[i]);
    }
    const uint64_t inv_q_mt = invmod(mod_words(Q, mt), mt);
    ok &= inv_q_mt != 0;
    h[o.neg_inv_q_mt] = (mt - inv_q_mt) & (mt - 1);
    for (int k = 0; k < bsk; k++) {
        const uint64_t b = bskv[k];
        const uint64_t qb = mod_words(Q, b);
        pair(o.Qmod_b, k, qb, b);
        const uint64_t imt = invmod(mt % b, b);
        pair(o.inv_mt_b, k, imt, b);
        pair(o.t_b, k, t % b, b);
        const uint64_t iqb = invmod(qb, b);
        ok &= imt != 0 && iqb != 0;
        pair(o.inv_q_b, k, iqb, b);
    }
    for (int k = 0; k < bB; k++) {
        const uint64_t ip = invmod(punctured_mod(Bv.data(), bB, k, Bv[k]), Bv[k]);
        ok &= ip != 0;
        pair(o.B_ip, k, ip, Bv[k]);
        pair(o.iqb_Bip, k, mulmod(ip, invmod(mod_words(Q, Bv[k]), Bv[k]), Bv[k]), Bv[k]);
        h[o.M_Bmsk + k] = punctured_mod(Bv.data(), bB, k, msk);
    }
    // base-conversion rows with the constant that follows each sum folded in: the lift
    // multiplies its result by m~^-1, the floor by c_k (Q^-1, and for B_k also the
    // B-base factor (P_B/B_k)^-1)
    for (int k = 0; k < bsk; k++) {
        const uint64_t b = bskv[k];
        const uint64_t imt = h[o.inv_mt_b + 2 * k];
        const uint64_t ck = k < bB ? h[o.iqb_Bip + 2 * k] : h[o.inv_q_b + 2 * k];
        for (int i = 0; i < L; i++) {
            const uint64_t mq = punctured_mod(q, L, i, b);
            h[o.M_qB + k * L + i] = mulmod(mq, imt, b);
            h[o.M_qB_fl + k * L + i] = mulmod(mq, ck, b);
        }
        pair(o.Qmt_b, k, mulmod(h[o.Qmod_b + 2 * k], imt, b), b);
        pair(o.tc_b, k, mulmod(t % b, ck, b), b);
    }
    const uint64_t ipb = invmod(prod_mod(Bv.data(), bB, msk), msk);
    ok &= ipb != 0;
    pair(o.inv_pb_msk, 0, ipb, msk);
    const uint64_t qt = mod_words(Q, t), qg = mod_words(Q, gam);
    const uint64_t iqt = invmod(qt, t), iqg = invmod(qg, gam);
    h[o.neg_inv_q_tg] = iqt ? t - iqt : 0;
    h[o.neg_inv_q_tg + 1] = iqg ? gam - iqg : 0;
    h[o.inv_gamma_t] = invmod(gam % t, t);
    h[o.q_mod_t] = qt;
    uint64_t rem = 0;
    const auto Qdt = div_words(Q, t, rem);
    for (int i = 0; i < L; i++) {
        pair(o.cdpt, i, mod_words(Qdt, q[i]), q[i]);
        h[o.plain_incr + i] = (q[i] - t % q[i]) % q[i];
    }
    if (!ok) return TB_OK;  // t shares a factor with q: BFV/BGV arithmetic unavailable at this level
    std::vector<Mod> bm(bsk);
    for (int k = 0; k < bsk; k++) bm[k] = c.h_mods[bidx[k]];
    cudaError_t e = cudaMalloc(&lv.d_consts, h.size() * 8);
    if (e == cudaSuccess) e = cudaMemcpy(lv.d_consts, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&lv.d_bsk_mods, bsk * sizeof(Mod));
    if (e == cudaSuccess) e = cudaMemcpy(lv.d_bsk_mods, bm.data(), bsk * sizeof(Mod), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&lv.d_bsk_idx, bsk * sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(lv.d_bsk_idx, bidx.data(), bsk * sizeof(int), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? TB_OK : status_from(e);
}

// ------------------------------------------------------------------ kernels

namespace {

constexpr int MAXL_RT = 32;  // data limbs of the run-time form (LT = 0)
constexpr int MAXL = 64;     // data limbs of the wide run-time form (LT = -1): every chain a context takes

__device__ __forceinline__ uint64_t pw(const uint64_t *K, int off, int i, uint64_t x, uint64_t q) {
    return mul_shoup(x, K[off + 2 * i], K[off + 2 * i + 1], q);
}

// The per-coefficient BEHZ kernels are templates over the data-limb count LT, with LT = 0
// the run-time form for any count up to MAXL_RT and LT = -1 the same form with arrays for
// MAXL limbs (its per-coefficient arrays live in local memory). With LT fixed the loops
// over the data limbs unroll and the per-coefficient residues and accumulators stay in
// registers; the loops over the B / Bsk primes stay rolled, so one iteration's constants
// are all that is live beside them.

// Steps (1)+(2): q (coefficient form) -> Bsk, one coefficient per thread, for both
// inputs of B products: polynomial p = ct*4 + slot, slots 0,1 from a and 2,3 from b;
// output [B][4][bsk][N].
template <int LT>
__global__ void __launch_bounds__(256, 3) behz_lift_kernel(const uint64_t *__restrict__ a, uint64_t astride,
                                                        const uint64_t *__restrict__ b, uint64_t bstride,
                                                        uint64_t *__restrict__ dst, const Mod *__restrict__ qm,
                                                        const Mod *__restrict__ bm, const uint64_t *__restrict__ K,
                                                        RnsOff o, int L_, int bsk, int logn, uint64_t P) {
    constexpr int NL = LT > 0 ? LT : (LT == 0 ? MAXL_RT : MAXL), UNROLL = LT > 0 ? LT : 1;
    const int L = LT > 0 ? LT : L_;
    const uint32_t n = 1u << logn;
    const uint64_t total = P << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = w >> logn;
        const uint32_t e = (uint32_t)(w & (n - 1));
        const uint64_t ct = p >> 2, slot = p & 3;
        const uint64_t *in = (slot < 2 ? a + ct * astride + ((slot * L) << logn)
                                       : b + ct * bstride + (((slot - 2) * L) << logn)) + e;
        uint64_t tmp[NL];
        uint64_t mt = 0;
#pragma unroll UNROLL
        for (int i = 0; i < NL; i++) {
            if (i >= L) break;
            tmp[i] = pw(K, o.q_mtip, i, in[(size_t)i << logn], qm[i].value);
            mt += tmp[i] * K[o.M_qB + bsk * L + i];
        }
        const uint64_t r = ((mt & 0xffffffffull) * K[o.neg_inv_q_mt]) & 0xffffffffull;
        uint64_t *out = dst + ((p * bsk) << logn) + e;
#pragma unroll 1
        for (int k = 0; k < bsk; k++) {
            const Mod &m = bm[k];
            U128 acc{0, 0};
#pragma unroll UNROLL
            for (int i = 0; i < NL; i++) {
                if (i >= L) break;
                mac128(acc, tmp[i], K[o.M_qB + k * L + i]);
            }
            const uint64_t v = reduce128(acc.hi, acc.lo, m);   // already times m~^-1
            const uint64_t rr = r >= (1ull << 31) ? r + m.value - (1ull << 32) : r;
            out[(size_t)k << logn] = add_mod(pw(K, o.Qmt_b, k, rr, m.value), v, m.value);
        }
    }
}

// Steps (6)-(8): (q U Bsk, inverse-NTT outputs) -> q, one coefficient per thread. The
// floor residue of each B prime feeds the Shenoy-Kumaresan sums (into every q_i and into
// m_sk) as soon as it is made, so no per-prime array is kept.
template <int LT>
__global__ void __launch_bounds__(256, 2) behz_floor_sk_kernel(const uint64_t *__restrict__ tq,
                                                            const uint64_t *__restrict__ tbk,
                                                            uint64_t *__restrict__ out, uint64_t ostride,
                                                            const Mod *__restrict__ qm, const Mod *__restrict__ bm,
                                                            const uint64_t *__restrict__ K, RnsOff o, int L_, int bB,
                                                            int logn, uint64_t P) {
    constexpr int NL = LT > 0 ? LT : (LT == 0 ? MAXL_RT : MAXL), UNROLL = LT > 0 ? LT : 1;
    const int L = LT > 0 ? LT : L_;
    const int bsk = bB + 1;
    const uint32_t n = 1u << logn;
    const uint64_t total = P << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t p = w >> logn;   // p = ct * 3 + poly
        const uint32_t e = (uint32_t)(w & (n - 1));
        const uint64_t *iq = tq + ((p * L) << logn) + e;
        const uint64_t *ib = tbk + ((p * bsk) << logn) + e;
        uint64_t tmp[NL];
#pragma unroll UNROLL
        for (int i = 0; i < NL; i++) {
            if (i >= L) break;
            // t ct_i (Q/q_i)^-1 mod q_i, the two constants folded into one
            tmp[i] = pw(K, o.tq_ip, i, iq[(size_t)i << logn], qm[i].value);
        }
        // floor residue of Bsk prime k, (t * ct_k - conv_k(t * ct_q)) / q mod m_k, with
        // the B-base factor (P_B/B_k)^-1 folded in for k < bB: c_k (t ct_k - conv_k)
        auto floor_residue = [&](int k) {
            const Mod &m = bm[k];
            U128 acc{0, 0};
#pragma unroll UNROLL
            for (int i = 0; i < NL; i++) {
                if (i >= L) break;
                mac128(acc, tmp[i], K[o.M_qB_fl + k * L + i]);
            }
            const uint64_t conv = reduce128(acc.hi, acc.lo, m);   // c_k conv_k(t ct_q)
            return sub_mod(pw(K, o.tc_b, k, ib[(size_t)k << logn], m.value), conv, m.value);
        };
        // Shenoy-Kumaresan: B -> q with the m_sk correction
        U128 acc_q[NL];
#pragma unroll UNROLL
        for (int i = 0; i < NL; i++) acc_q[i] = U128{0, 0};
        U128 acc_sk{0, 0};
#pragma unroll 1
        for (int k = 0; k < bB; k++) {
            const uint64_t f = floor_residue(k);   // times (P_B/B_k)^-1
            mac128(acc_sk, f, K[o.M_Bmsk + k]);
#pragma unroll UNROLL
            for (int i = 0; i < NL; i++) {
                if (i >= L) break;
                mac128(acc_q[i], f, K[o.M_Bq + i * bB + k]);
            }
        }
        const Mod &ms = bm[bB];
        const uint64_t fsk = floor_residue(bB);
        const uint64_t tmsk = reduce128(acc_sk.hi, acc_sk.lo, ms);
        const uint64_t alpha = mul_shoup(tmsk + (ms.value - fsk), K[o.inv_pb_msk], K[o.inv_pb_msk + 1], ms.value);
        const bool neg = alpha > (ms.value >> 1);
        uint64_t *dst = out + (p / 3) * ostride + (((p % 3) * L) << logn) + e;
#pragma unroll UNROLL
        for (int i = 0; i < NL; i++) {
            if (i >= L) break;
            const Mod &m = qm[i];
            const uint64_t d = reduce128(acc_q[i].hi, acc_q[i].lo, m);
            const uint64_t corr = neg ? pw(K, o.pb_q, i, ms.value - alpha, m.value) : pw(K, o.negpb_q, i, alpha, m.value);
            dst[(size_t)i << logn] = add_mod(corr, d, m.value);
        }
    }
}

template <int LT>
struct LiftLaunch {
    template <class... A>
    static cudaError_t run(uint64_t threads, cudaStream_t s, A... args) {
        behz_lift_kernel<LT><<<grid_for(threads, 256), 256, 0, s>>>(args...);
        return cudaGetLastError();
    }
};

template <int LT>
struct FloorLaunch {
    template <class... A>
    static cudaError_t run(uint64_t threads, cudaStream_t s, A... args) {
        behz_floor_sk_kernel<LT><<<grid_for(threads, 256), 256, 0, s>>>(args...);
        return cudaGetLastError();
    }
};

// Launches a BEHZ kernel with the data-limb count fixed for L <= 16, the run-time form
// up to 32 limbs and its wide form above.
#define TB_BEHZ_CASE(LV) \
    case LV:             \
        return Launch<LV>::run(threads, s, args...);
template <template <int> class Launch, class... A>
cudaError_t behz_dispatch(int L, uint64_t threads, cudaStream_t s, A... args) {
    switch (L) {
        TB_BEHZ_CASE(1) TB_BEHZ_CASE(2) TB_BEHZ_CASE(3) TB_BEHZ_CASE(4) TB_BEHZ_CASE(5) TB_BEHZ_CASE(6)
        TB_BEHZ_CASE(7) TB_BEHZ_CASE(8) TB_BEHZ_CASE(9) TB_BEHZ_CASE(10) TB_BEHZ_CASE(11) TB_BEHZ_CASE(12)
        TB_BEHZ_CASE(13) TB_BEHZ_CASE(14) TB_BEHZ_CASE(15) TB_BEHZ_CASE(16)
    default:
        if (L <= MAXL_RT) return Launch<0>::run(threads, s, args...);
        return Launch<-1>::run(threads, s, args...);
    }
}
#undef TB_BEHZ_CASE

// NTT over a packed [P][limbs][N] buffer; limb l uses mods[l] (chain or Bsk array).
template <bool FWD>
struct PackedNttOp {
    const uint64_t *in;
    uint64_t *out;
    const Mod *mods;
    int limbs, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
    };
    __device__ Ctx ctx(int b) const {
        Ctx c;
        c.lm = make_limb(mods[b % limbs], 0);
        c.in = in + ((size_t)b << logn);
        c.out = out + ((size_t)b << logn);
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const { return c.in[e]; }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const { c.out[e] = v; }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b) const {
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(a, b);
    }
};

// Forward NTT (lazy) of both operands of B products into a packed [B][4][L][N]
// buffer: slots 0,1 from a, 2,3 from b.
struct PairNttOp {
    const uint64_t *a, *b;
    uint64_t astride, bstride;
    uint64_t *out;
    const Mod *mods;
    int L, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
    };
    __device__ Ctx ctx(int blk) const {
        const int l = blk % L;
        const int p = blk / L;
        const int ct = p >> 2, slot = p & 3;
        Ctx c;
        c.lm = make_limb(mods[l], 0);
        c.in = (slot < 2 ? a + (size_t)ct * astride + (((size_t)slot * L + l) << logn)
                         : b + (size_t)ct * bstride + (((size_t)(slot - 2) * L + l) << logn));
        c.out = out + ((size_t)blk << logn);
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const { return c.in[e]; }
    __device__ void store2(const Ctx &c, int e, uint64_t x, uint64_t y) const {
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(x, y);
    }
};

// Inverse NTT from a packed [P][L][N] buffer into a strided destination with canonical
// outputs (BGV multiply's last step).
struct CtInttOutOp {
    const uint64_t *in;
    uint64_t *out;
    uint64_t ostride;
    const Mod *mods;
    int per, L, logn;
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
    };
    __device__ Ctx ctx(int b) const {
        const int l = b % L;
        const int p = b / L;
        Ctx c;
        c.lm = make_limb(mods[l], 0);
        c.in = in + ((size_t)b << logn);
        c.out = out + (size_t)(p / per) * ostride + (((size_t)(p % per) * L + l) << logn);
        return c;
    }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const { c.out[e] = csub(v, c.lm.q); }
};

}  // namespace

struct ScratchBuf {
    void *p = nullptr;
    cudaStream_t s;
    explicit ScratchBuf(cudaStream_t st) : s(st) {}
    ~ScratchBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// Multiplies B pairs of size-2 ciphertexts at level L into size-3 outputs.
int multiply(const Context &c, int L, const uint64_t *a, uint64_t astride, const uint64_t *b, uint64_t bstride,
             uint64_t *out, uint64_t ostride, uint64_t B, cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (L < 1 || L > K) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!a || !b || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    const uint64_t n = c.n;
    if (!astride) astride = 2ull * L * n;
    if (!bstride) bstride = 2ull * L * n;
    if (!ostride) ostride = 3ull * L * n;
    // CKKS: the NTT-domain tensor of two ciphertexts, whose words are residues below q
    if (c.scheme == SCHEME_CKKS)
        return tensor_product_mods(c, c.d_mods, L, a, astride, b, bstride, out, ostride, B, s, true);
    if (c.scheme != SCHEME_BFV && c.scheme != SCHEME_BGV) return set_error(TB_ERR_UNSUPPORTED, "scheme has no multiply");
    if (c.logn > MAX_FUSED_LOGN) return set_error(TB_ERR_UNSUPPORTED, "multiply supports N <= 131072");
    ensure_pool_retains(c.device);
    const int logn = c.logn;
    cudaError_t e;
    if (c.scheme == SCHEME_BGV) {
        ScratchBuf buf(s);
        e = cudaMallocAsync(&buf.p, B * 7ull * L * n * 8, s);
        if (e != cudaSuccess) return status_from(e);
        uint64_t *x = (uint64_t *)buf.p, *tn = x + B * 4ull * L * n;
        {
            TraceScope ts("mul_ntt", s);
            PairNttOp op{a, b, astride, bstride, x, c.d_mods, L, logn};
            e = dispatch_ntt<true>(logn, op, (unsigned)(B * 4 * L), 0, 0, s);
        }
        if (e != cudaSuccess) return status_from(e);
        const uint64_t pq = (uint64_t)L * n;
        int st = tensor_product_mods(c, c.d_mods, L, x, 4 * pq, x + 2 * pq, 4 * pq, tn, 3 * pq, B, s);
        if (st != TB_OK) return st;
        TraceScope ts("mul_intt", s);
        CtInttOutOp oi{tn, out, ostride, c.d_mods, 3, L, logn};
        e = dispatch_ntt<false>(logn, oi, (unsigned)(B * 3 * L), logn, 1, s);
        return e == cudaSuccess ? TB_OK : status_from(e);
    }
    // BFV
    const RnsLevel &lv = c.levels[L];
    if (!lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to the coefficient moduli");
    if (L > MAXL) return set_error(TB_ERR_UNSUPPORTED, "BFV multiply supports at most 64 data limbs");
    const int bsk = lv.bsk;
    const uint64_t pq = (uint64_t)L * n, pb = (uint64_t)bsk * n;
    ScratchBuf buf(s);
    e = cudaMallocAsync(&buf.p, B * (4 * pq + 4 * pb + 3 * pq + 3 * pb) * 8, s);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *xq = (uint64_t *)buf.p;          // [B][4][L][N]: a0 a1 b0 b1 (NTT, lazy)
    uint64_t *xb = xq + B * 4 * pq;            // [B][4][bsk][N]
    uint64_t *tq = xb + B * 4 * pb;            // [B][3][L][N]
    uint64_t *tbk = tq + B * 3 * pq;           // [B][3][bsk][N]
    {
        TraceScope ts("bfv_ntt_q", s);
        PairNttOp op{a, b, astride, bstride, xq, c.d_mods, L, logn};
        e = dispatch_ntt<true>(logn, op, (unsigned)(B * 4 * L), 0, 0, s);
        if (e != cudaSuccess) return status_from(e);
    }
    {
        TraceScope ts("bfv_lift", s);
        e = behz_dispatch<LiftLaunch>(L, 4 * B * n, s, a, astride, b, bstride, xb, (const Mod *)c.d_mods,
                                      (const Mod *)lv.d_bsk_mods, (const uint64_t *)lv.d_consts, lv.off, L, bsk, logn,
                                      (uint64_t)(4 * B));
        if (e != cudaSuccess) return status_from(e);
    }
    {
        TraceScope ts("bfv_ntt_bsk", s);
        PackedNttOp<true> op{xb, xb, lv.d_bsk_mods, bsk, logn};
        e = dispatch_ntt<true>(logn, op, (unsigned)(B * 4 * bsk), 0, 0, s);
        if (e != cudaSuccess) return status_from(e);
    }
    int st = tensor_product_mods(c, c.d_mods, L, xq, 4 * pq, xq + 2 * pq, 4 * pq, tq, 3 * pq, B, s);
    if (st != TB_OK) return st;
    st = tensor_product_mods(c, lv.d_bsk_mods, bsk, xb, 4 * pb, xb + 2 * pb, 4 * pb, tbk, 3 * pb, B, s);
    if (st != TB_OK) return st;
    {
        TraceScope ts("bfv_intt", s);
        PackedNttOp<false> oq{tq, tq, c.d_mods, L, logn};
        e = dispatch_ntt<false>(logn, oq, (unsigned)(B * 3 * L), logn, 1, s);
        if (e != cudaSuccess) return status_from(e);
        PackedNttOp<false> ob{tbk, tbk, lv.d_bsk_mods, bsk, logn};
        e = dispatch_ntt<false>(logn, ob, (unsigned)(B * 3 * bsk), logn, 1, s);
        if (e != cudaSuccess) return status_from(e);
    }
    {
        TraceScope ts("bfv_floor_sk", s);
        e = behz_dispatch<FloorLaunch>(L, 3 * B * n, s, (const uint64_t *)tq, (const uint64_t *)tbk, out, ostride,
                                       (const Mod *)c.d_mods, (const Mod *)lv.d_bsk_mods, (const uint64_t *)lv.d_consts,
                                       lv.off, L, lv.bB, logn, (uint64_t)(3 * B));
    }
    return e == cudaSuccess ? TB_OK : status_from(e);
}

// ---------------------------------------------------------- any operand sizes

// out[k] = sum_{i+j=k} x[i] (.) y[j] over `limbs` limbs (mods[l]) for sa x sb polynomials
// (packed [sa][limbs][N] and [sb][limbs][N]); canonical outputs, the exact residues of
// the reference's dyadic products and additions (any input below 2^64).
__global__ void tensor_sizes_kernel(const uint64_t *__restrict__ x, int sa, const uint64_t *__restrict__ y, int sb,
                                    uint64_t *__restrict__ out, const Mod *__restrict__ mods, int limbs, int logn) {
    const uint64_t per = (uint64_t)limbs << logn;
    const uint64_t total = (uint64_t)(sa + sb - 1) * per;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const int k = (int)(w / per);
        const uint64_t r = w - (uint64_t)k * per;
        const Mod m = mods[r >> logn];
        uint64_t acc = 0;
        for (int i = k < sb ? 0 : k - sb + 1; i <= k && i < sa; i++)
            acc = add_mod(acc, mul_mod(x[(uint64_t)i * per + r], y[(uint64_t)(k - i) * per + r], m), m.value);
        out[w] = acc;
    }
}

// One product of a size-sa and a size-sb ciphertext at level L into sa + sb - 1
// polynomials (bfvMultiply / bgvMultiply / ckksMultiply for any sizes,
// src/evaluator_cuda.cu:283-501): the same steps as the batched size-2 path, on
// packed copies of the operands, with the general tensor.
int multiply_sizes(const Context &c, int L, const uint64_t *a, int sa, const uint64_t *b, int sb, uint64_t *out,
                   cudaStream_t s) {
    const int K = (int)c.chain.size();
    if (L < 1 || L > K) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (!a || !b || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (sa < 2 || sb < 2 || sa > 64 || sb > 64) return set_error(TB_ERR_INVALID_ARGUMENT, "ciphertext sizes must be 2 .. 64");
    if (c.scheme != SCHEME_BFV && c.scheme != SCHEME_BGV && c.scheme != SCHEME_CKKS)
        return set_error(TB_ERR_UNSUPPORTED, "scheme has no multiply");
    if (c.logn > MAX_FUSED_LOGN) return set_error(TB_ERR_UNSUPPORTED, "multiply supports N <= 131072");
    const int logn = c.logn;
    const uint64_t n = c.n, pq = (uint64_t)L * n;
    const int P = sa + sb, D = sa + sb - 1;
    if (c.scheme == SCHEME_CKKS) {
        TraceScope ts("tensor", s);
        tensor_sizes_kernel<<<grid_for((uint64_t)D * pq, 256), 256, 0, s>>>(a, sa, b, sb, out, c.d_mods, L, logn);
        return status_from(cudaGetLastError());
    }
    ensure_pool_retains(c.device);
    ScratchBuf buf(s);
    cudaError_t e;
    if (c.scheme == SCHEME_BGV) {
        e = cudaMallocAsync(&buf.p, (uint64_t)(P + D) * pq * 8, s);
        if (e != cudaSuccess) return status_from(e);
        uint64_t *x = (uint64_t *)buf.p, *t = x + (uint64_t)P * pq;
        e = cudaMemcpyAsync(x, a, sa * pq * 8, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess) e = cudaMemcpyAsync(x + sa * pq, b, sb * pq * 8, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return status_from(e);
        PackedNttOp<true> f{x, x, c.d_mods, L, logn};
        e = dispatch_ntt<true>(logn, f, (unsigned)(P * L), 0, 0, s);
        if (e != cudaSuccess) return status_from(e);
        tensor_sizes_kernel<<<grid_for((uint64_t)D * pq, 256), 256, 0, s>>>(x, sa, x + sa * pq, sb, t, c.d_mods, L,
                                                                           logn);
        e = cudaGetLastError();
        if (e != cudaSuccess) return status_from(e);
        CtInttOutOp oi{t, out, (uint64_t)D * pq, c.d_mods, D, L, logn};
        e = dispatch_ntt<false>(logn, oi, (unsigned)(D * L), logn, 1, s);
        return status_from(e);
    }
    // BFV
    const RnsLevel &lv = c.levels[L];
    if (!lv.d_consts) return set_error(TB_ERR_UNSUPPORTED, "plain modulus not coprime to the coefficient moduli");
    if (L > MAXL) return set_error(TB_ERR_UNSUPPORTED, "BFV multiply supports at most 64 data limbs");
    const int bsk = lv.bsk;
    const uint64_t pb = (uint64_t)bsk * n;
    e = cudaMallocAsync(&buf.p, ((uint64_t)P * (2 * pq + pb) + (uint64_t)D * (pq + pb)) * 8, s);
    if (e != cudaSuccess) return status_from(e);
    uint64_t *x0 = (uint64_t *)buf.p;          // [P][L][N] operands, coefficient form
    uint64_t *xq = x0 + (uint64_t)P * pq;      // [P][L][N] NTT in q
    uint64_t *xb = xq + (uint64_t)P * pq;      // [P][bsk][N] lifted to Bsk, NTT
    uint64_t *tq = xb + (uint64_t)P * pb;      // [D][L][N]
    uint64_t *tbk = tq + (uint64_t)D * pq;     // [D][bsk][N]
    e = cudaMemcpyAsync(x0, a, sa * pq * 8, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(x0 + sa * pq, b, sb * pq * 8, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess) return status_from(e);
    PackedNttOp<true> fq{x0, xq, c.d_mods, L, logn};
    e = dispatch_ntt<true>(logn, fq, (unsigned)(P * L), 0, 0, s);
    if (e != cudaSuccess) return status_from(e);
    // the lift reads polynomial p of four-polynomial groups: with both strides 4 L N
    // and b starting two polynomials in, polynomial p of x0 for every p
    e = behz_dispatch<LiftLaunch>(L, (uint64_t)P * n, s, (const uint64_t *)x0, 4 * pq,
                                  (const uint64_t *)(x0 + 2 * pq), 4 * pq, xb, (const Mod *)c.d_mods,
                                  (const Mod *)lv.d_bsk_mods, (const uint64_t *)lv.d_consts, lv.off, L, bsk, logn,
                                  (uint64_t)P);
    if (e != cudaSuccess) return status_from(e);
    PackedNttOp<true> fb{xb, xb, lv.d_bsk_mods, bsk, logn};
    e = dispatch_ntt<true>(logn, fb, (unsigned)(P * bsk), 0, 0, s);
    if (e != cudaSuccess) return status_from(e);
    tensor_sizes_kernel<<<grid_for((uint64_t)D * pq, 256), 256, 0, s>>>(xq, sa, xq + sa * pq, sb, tq, c.d_mods, L, logn);
    tensor_sizes_kernel<<<grid_for((uint64_t)D * pb, 256), 256, 0, s>>>(xb, sa, xb + sa * pb, sb, tbk, lv.d_bsk_mods,
                                                                       bsk, logn);
    e = cudaGetLastError();
    if (e != cudaSuccess) return status_from(e);
    PackedNttOp<false> iq{tq, tq, c.d_mods, L, logn};
    e = dispatch_ntt<false>(logn, iq, (unsigned)(D * L), logn, 1, s);
    if (e != cudaSuccess) return status_from(e);
    PackedNttOp<false> ib{tbk, tbk, lv.d_bsk_mods, bsk, logn};
    e = dispatch_ntt<false>(logn, ib, (unsigned)(D * bsk), logn, 1, s);
    if (e != cudaSuccess) return status_from(e);
    // the floor reads polynomial p = ct * 3 + poly: ostride 3 L N maps it to out + p L N
    e = behz_dispatch<FloorLaunch>(L, (uint64_t)D * n, s, (const uint64_t *)tq, (const uint64_t *)tbk, out,
                                   3 * pq, (const Mod *)c.d_mods, (const Mod *)lv.d_bsk_mods,
                                   (const uint64_t *)lv.d_consts, lv.off, L, lv.bB, logn, (uint64_t)D);
    return status_from(e);
}

}  // namespace tb

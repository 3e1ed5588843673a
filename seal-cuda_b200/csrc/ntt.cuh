// Negacyclic NTT / inverse NTT kernels for sm_100a.
//
// One CTA transforms one polynomial limb (or one 2^LOGB sub-block of a larger one)
// entirely inside shared memory. Stages are grouped into radix-8 register passes
// (remainder stages in the first forward / last inverse pass): a thread loads 8
// coefficients, runs three Cooley-Tukey (forward) or Gentleman-Sande (inverse)
// stages in registers with Shoup twiddles, and writes them back; the shared-memory
// slot of coefficient e is swz(e), which keeps every pass bank-conflict free.
//
// Transforms with lazy outputs run the butterflies and lazy ranges of the reference's
// DWTHandler (src/utils/dwthandler.h:88-372, src/utils/ntt.h:17-60), so their outputs
// are bit-identical to nttNegacyclicHarveyLazy / inverseNttNegacyclicHarveyLazy
// (src/utils/ntt.cpp:158-213); the N^-1 scaling is folded into the last inverse stage
// exactly as there. Transforms whose outputs are reduced afterwards (full outputs, the
// fused key-switch, rescale and multiply steps) may defer their reductions (the wide
// forms below): the residues, and so the reduced outputs, are the same.
//
// Each kernel is parameterised by an operation `Op` that maps a CTA to its limb
// (pointers + modulus) and supplies the global-memory load of the first pass and
// the store of the last, so base conversions, key-switch mod-up/mod-down and
// rescaling steps fuse into the transform instead of running as extra passes.
#pragma once

#include <cooperative_groups.h>

#include <algorithm>
#include <type_traits>

#include "common.cuh"

namespace tb {

// Per-CTA transform parameters every Op context carries.
struct NttLimb {
    uint64_t q;
    const ulonglong2 *roots;
    const ulonglong2 *iroots;
    uint64_t inv_n, inv_n_quo;   // N^-1 (Shoup)
    uint64_t sroot, sroot_quo;   // last inverse root times N^-1 (Shoup)
    uint32_t sb;                 // sub-block index when the CTA owns 2^LOGB of a longer limb
};

// Threads per CTA: variant 0 gives each thread one radix-8 group per pass at a time (at
// most 1024 threads); variant V >= 1 divides the thread count by 2^V, each thread then
// running more groups of a pass one after another. Fewer threads need fewer registers
// per CTA, so several CTAs (limbs) share an SM and one CTA's barriers and memory
// phases overlap another's arithmetic. Variants 3 .. 5 transform a whole limb on a
// cluster of two CTAs of half the block each (thread counts as variants 0 .. 2 of the
// half block): half the shared memory per CTA, so up to twice as many limbs resident
// per SM, for one exchange stage through distributed shared memory. Launches of a
// sub-block of a longer limb take variant v - 3 instead. The variant per block size is
// a tuning choice (tb_ntt_*).
constexpr int NTT_VARIANTS = 6;

template <int LOGB, int V = 0>
struct NttCfg {
    static constexpr int NB = 1 << LOGB;
    static constexpr int BASE = NB >= 8192 ? 1024 : (NB / 8 >= 64 ? NB / 8 : 64);
    static constexpr int THREADS = (BASE >> V) >= 32 ? (BASE >> V) : 32;
    static constexpr int REM = LOGB % 3;
};

// Shared-memory slot of coefficient base | (k << logsub) when the bits of k << logsub
// are clear in base: swz(base) ^ swz_delta(k << logsub), a compile-time constant per k.
__host__ __device__ constexpr int swz_delta(int kk) { return kk ^ ((kk >> 4) & 15); }

__device__ __forceinline__ void ct_butterfly(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    uint64_t u = csub(x, q2);
    uint64_t v = mul_shoup_lazy(y, w.x, w.y, q);
    x = u + v;
    y = u + q2 - v;
}

// The Cooley-Tukey butterfly without the conditional subtraction of x, and the one that
// subtracts a given multiple qs of q instead of 2q. Without the subtraction x grows by at
// most 2q a stage (y stays below x's bound + 2q; the Shoup product is in [0, 2q) for any
// 64-bit input).
__device__ __forceinline__ void ct_butterfly_slack(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    const uint64_t v = mul_shoup_lazy(y, w.x, w.y, q);
    y = x + q2 - v;
    x = x + v;
}

__device__ __forceinline__ void ct_butterfly_sub(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2,
                                                 uint64_t qs) {
    const uint64_t u = csub(x, qs);
    const uint64_t v = mul_shoup_lazy(y, w.x, w.y, q);
    x = u + v;
    y = u + q2 - v;
}

// The no-subtraction form's butterfly (q < 2^57): the Shoup quotient floor(y wq / 2^64)
// estimated from three 32-bit partial products, y1 w1 + hi(y1 w0) + hi(y0 w1), which
// drops y0 w0 and two carries: at most 2 below the exact quotient for any 64-bit y, so
// the product lies in [0, 4q) and x grows by at most 4q a stage (y stays below x's
// bound + 4q).
__device__ __forceinline__ uint64_t mul_shoup_lazy4(uint64_t y, uint64_t w, uint64_t wq, uint64_t q) {
    const uint32_t y0 = (uint32_t)y, y1 = (uint32_t)(y >> 32), w0 = (uint32_t)wq, w1 = (uint32_t)(wq >> 32);
    const uint64_t qt = (uint64_t)y1 * w1 + __umulhi(y1, w0) + __umulhi(y0, w1);
    return w * y - qt * q;
}

__device__ __forceinline__ void ct_butterfly_wide(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q4) {
    const uint64_t v = mul_shoup_lazy4(y, w.x, w.y, q);
    y = x + q4 - v;
    x = x + v;
}

// Forward stages with deferred reductions, bound M (in multiples of q). Values entering
// local stage k of a transform from inputs below 4q stay below fwd_bound(M, k) q: a stage
// skips the subtraction (bound + 2q) unless that would pass M q; then it first subtracts
// (M/2) q from x (x below (M/2) q, outputs below (M/2 + 2) q). M = 4 is the Harvey
// butterfly of every stage (subtract 2q; outputs below 4q, the reference's lazy
// outputs). M = 16, for q < 2^60 (16 q < 2^64), subtracts at two of the 14 stages of a
// 16384-coefficient transform; its outputs stay below 16 q.
__host__ __device__ constexpr int fwd_bound(int M, int k) {
    int b = 4;
    for (int i = 0; i < k; i++) b = b + 2 <= M ? b + 2 : M / 2 + 2;
    return b;
}
__host__ __device__ constexpr bool fwd_subtracts(int M, int k) { return fwd_bound(M, k) + 2 > M; }
static_assert(fwd_bound(4, 14) == 4 && fwd_subtracts(4, 0) && fwd_subtracts(4, 13), "Harvey stages");
static_assert(fwd_bound(16, 17) <= 16 && !fwd_subtracts(16, 5) && fwd_subtracts(16, 6) && fwd_subtracts(16, 10),
              "deferred stages");
static_assert(!fwd_subtracts(64, 16), "no subtraction in the wide form");

// An Op context with an int member `slack` selects per CTA the bound M of its forward
// transform: 0 for the Harvey stages, SLACK_M (q < 2^60: outputs below 16 q) or, for an
// Op that declares `static constexpr bool wide_slack = true`, SLACK_WIDE (q < 2^57, one
// CTA per limb: no subtraction at all and the estimated quotient, ct_butterfly_wide;
// from inputs below B the outputs stay below B + 4 q log2 N, below 2^61 + 56 q < 2^63.2
// for inputs below 2^61 at N <= 16384). The Op takes those outputs at its store. The
// CTA-pair and cluster forms always run the Harvey stages (outputs below 4q).
constexpr int SLACK_M = 16;
constexpr int SLACK_WIDE = 64;
template <class Ctx, class = void>
struct HasSlack : std::false_type {};
template <class Ctx>
struct HasSlack<Ctx, std::void_t<decltype(std::declval<Ctx>().slack)>> : std::true_type {};
template <class Op, class = void>
struct WideSlack : std::false_type {};
template <class Op>
struct WideSlack<Op, std::void_t<decltype(Op::wide_slack)>> : std::bool_constant<Op::wide_slack> {};

// The inverse transform's wide form, for an Op whose context has an int member `islack`
// set (its store reduces the outputs itself): values below 4q between stages instead of
// 2q, the sum reduced by 4q, the difference's Shoup product with the estimated quotient
// (mul_shoup_lazy4, [0, 4q)); the last, N^-1-scaled stage multiplies both outputs without
// reducing the sum first. Outputs below 4q. Only whole-limb single-CTA launches run it.
__device__ __forceinline__ void gs_butterfly_wide(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q4) {
    const uint64_t u = x, v = y;
    x = csub(u + v, q4);
    y = mul_shoup_lazy4(u + q4 - v, w.x, w.y, q);
}

template <class Ctx, class = void>
struct HasInvSlack : std::false_type {};
template <class Ctx>
struct HasInvSlack<Ctx, std::void_t<decltype(std::declval<Ctx>().islack)>> : std::true_type {};

__device__ __forceinline__ void gs_butterfly(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    uint64_t u = x, v = y;
    uint64_t s = u + v;
    x = csub(s, q2);
    y = mul_shoup_lazy(u + q2 - v, w.x, w.y, q);
}

// Group handled by this thread in iteration i of a pass with IT groups per thread:
// thread-major (i * T + thread) for a pass that loads from global memory (consecutive
// threads take consecutive groups: coalesced), warp-major otherwise (warp w owns the
// 32 IT consecutive groups from 32 IT w): a warp's groups then cover whole blocks of as
// many stages as possible, so more of the barriers between passes can be warp barriers.
// Within a warp the lanes still take consecutive groups, so shared-memory banks are hit
// exactly as in the thread-major order.
template <bool WARP_MAJOR, int T, int IT>
__device__ __forceinline__ int pass_group(int i) {
    if constexpr (WARP_MAJOR && IT > 1 && T % 32 == 0)
        return (int)(threadIdx.x >> 5) * (32 * IT) + i * 32 + (int)(threadIdx.x & 31);
    else
        return (int)threadIdx.x + i * T;
}

template <int N>
constexpr int ilog2c() {
    return N <= 1 ? 0 : 1 + ilog2c<N / 2>();
}

// Coefficient pairs moved between global and shared memory (forward copy-out, inverse
// copy-in) in warp-major order when every thread has whole radix-8 groups (NB >= 8 T):
// warp w moves coefficients w E .. (w+1) E - 1, E = 32 NB / T, 64 consecutive per
// instruction (coalesced), exactly the coefficients its groups hold in the last forward
// / first inverse radix-8 pass, so only a warp barrier separates the two.
template <int NB, int T>
struct WarpIO {
    static constexpr bool value = T % 32 == 0 && NB % (8 * T) == 0;
};

template <int NB, int T>
__device__ __forceinline__ int io_pair(int i) {
    if constexpr (WarpIO<NB, T>::value)
        return (int)(threadIdx.x >> 5) * (NB * 32 / T) + i * 64 + 2 * (int)(threadIdx.x & 31);
    else
        return (int)threadIdx.x * 2 + i * 2 * T;
}

// ---------------------------------------------------------------- forward
// Pass of R_LOG Cooley-Tukey stages starting at local stage s. rbase = 2^s0 + sb
// where s0 is the global stage of local stage 0 (0 when the CTA owns the limb).
// SIDE: the thread's groups are processed side by side (all loaded, then all
// butterflies, then all stored: more independent work, more registers) rather than
// one after another.
template <int R_LOG, bool FROM_GLOBAL, int LOGB, int T, int s, bool SIDE, int M = 4, class Op, class Ctx>
__device__ __forceinline__ void fwd_pass(const Op &op, const Ctx &c, uint64_t *sm, uint32_t rbase) {
    constexpr int R = 1 << R_LOG;
    constexpr int NB = 1 << LOGB;
    constexpr int G = NB >> R_LOG;
    constexpr int IT = G > 0 ? (G + T - 1) / T : 1;  // groups per thread
    constexpr int GR = SIDE ? IT : 1;                // groups in flight at once
    constexpr bool FULL = G > 0 && G % T == 0;
    constexpr int logsub = LOGB - s - R_LOG;
    const uint64_t q = c.lm.q, q2 = q << 1, qs = q * (uint64_t)(M / 2), q4 = q << 2;
#pragma unroll
    for (int i0 = 0; i0 < IT; i0 += GR) {
        uint64_t v[GR][R];
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<!FROM_GLOBAL, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const int base = ((g >> logsub) << (LOGB - s)) + (g & ((1 << logsub) - 1));
            const int sb = swz(base);
#pragma unroll
            for (int k = 0; k < R; k++) {
                if constexpr (FROM_GLOBAL) v[it][k] = op.load(c, base + (k << logsub));
                else v[it][k] = sm[sb ^ swz_delta(k << logsub)];
            }
        }
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<!FROM_GLOBAL, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const uint32_t X = (rbase << s) + (uint32_t)(g >> logsub);
#pragma unroll
            for (int t = 0; t < R_LOG; t++) {
                const int half = R >> (t + 1);
                const ulonglong2 *row = c.lm.roots + (X << t);   // this stage's twiddles
#pragma unroll
                for (int k = 0; k < R; k++) {
                    if (k & half) continue;
                    if constexpr (M == SLACK_WIDE)
                        ct_butterfly_wide(v[it][k], v[it][k + half], __ldg(row + (k >> (R_LOG - t))), q, q4);
                    else if (fwd_subtracts(M, s + t))
                        ct_butterfly_sub(v[it][k], v[it][k + half], __ldg(row + (k >> (R_LOG - t))), q, q2, qs);
                    else
                        ct_butterfly_slack(v[it][k], v[it][k + half], __ldg(row + (k >> (R_LOG - t))), q, q2);
                }
            }
        }
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<!FROM_GLOBAL, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const int sb = swz(((g >> logsub) << (LOGB - s)) + (g & ((1 << logsub) - 1)));
#pragma unroll
            for (int k = 0; k < R; k++) sm[sb ^ swz_delta(k << logsub)] = v[it][k];
        }
    }
    // A shared-memory radix-8 pass with 2^ls groups per block of 2^(LOGB-s) coefficients,
    // 8 <= 2^ls <= 32 IT, leaves each warp's 32 IT groups on 256 IT consecutive
    // coefficients, exactly the ones the same warp's groups of the next radix-8 pass
    // (s + 3) read: only the warp needs to wait there, so the warps of the CTA drift apart
    // instead of meeting at a barrier.
    // The last pass (ls = 0) hands each warp's coefficients to the same warp's copy-out.
    constexpr int ls = LOGB - s - R_LOG;
    constexpr int LIT = (IT > 1 && T % 32 == 0) ? ilog2c<IT>() : 0;
    if constexpr (!FROM_GLOBAL && R_LOG == 3 && ls >= 3 && ls <= 5 + LIT && T % 32 == 0) __syncwarp();
    else if constexpr (!FROM_GLOBAL && R_LOG == 3 && ls == 0 && WarpIO<NB, T>::value) __syncwarp();
    else __syncthreads();
}

// The radix-8 shared-memory passes from local stage S on, unrolled at compile time so
// every index offset is a constant.
template <int S, int LOGB, int T, bool SIDE, int M = 4, class Op, class Ctx>
__device__ __forceinline__ void fwd_passes(const Op &op, const Ctx &c, uint64_t *sm, uint32_t rbase) {
    if constexpr (S < LOGB) {
        fwd_pass<3, false, LOGB, T, S, SIDE, M>(op, c, sm, rbase);
        fwd_passes<S + 3, LOGB, T, SIDE, M>(op, c, sm, rbase);
    }
}

// Copy-out of a forward transform: coefficient pairs (e, e+1) from shared memory to
// op.store2. An Op whose epilogue reads global memory declares `Epi` with
// epi2(ctx, e) (the reads for a pair) and store2(ctx, e, a, b, epi): the reads of
// four pairs are then issued before any of their stores, so the epilogue keeps
// several loads in flight instead of one pair's at a time.
template <class Op, class = void>
struct HasEpi : std::false_type {};
template <class Op>
struct HasEpi<Op, std::void_t<typename Op::Epi>> : std::true_type {};

template <int NB, int T, class Op, class Ctx>
__device__ __forceinline__ void fwd_copy_out(const Op &op, const Ctx &c, const uint64_t *sm, int off) {
    constexpr int ITER = NB / (2 * T);
    if constexpr (WarpIO<NB, T>::value && !HasEpi<Op>::value) {
#pragma unroll
        for (int i = 0; i < ITER; i++) {
            const int e = io_pair<NB, T>(i);
            const int p = swz(e);
            const ulonglong2 w = *reinterpret_cast<const ulonglong2 *>(&sm[p & ~1]);
            // a select, not a branch: the slot parity changes every 8 lanes, and a branch
            // would run both copies of the store (and its reductions) one after the other
            const uint64_t a = (p & 1) ? w.y : w.x, b = (p & 1) ? w.x : w.y;
            op.store2(c, e + off, a, b);
        }
    } else if constexpr (HasEpi<Op>::value && ITER >= 1 && NB % (2 * T) == 0) {
        constexpr int BATCH = ITER >= 4 ? 4 : ITER;
        static_assert(ITER % BATCH == 0, "copy-out batches");
#pragma unroll
        for (int i0 = 0; i0 < ITER; i0 += BATCH) {
            typename Op::Epi pre[BATCH];
#pragma unroll
            for (int i = 0; i < BATCH; i++) pre[i] = op.epi2(c, io_pair<NB, T>(i0 + i) + off);
#pragma unroll
            for (int i = 0; i < BATCH; i++) {
                const int e = io_pair<NB, T>(i0 + i);
                const int p = swz(e);
                const ulonglong2 w = *reinterpret_cast<const ulonglong2 *>(&sm[p & ~1]);
                const uint64_t a = (p & 1) ? w.y : w.x, b = (p & 1) ? w.x : w.y;
                op.store2(c, e + off, a, b, pre[i]);
            }
        }
    } else {
        for (int e = threadIdx.x * 2; e < NB; e += T * 2) {
            const int p = swz(e);
            const ulonglong2 w = *reinterpret_cast<const ulonglong2 *>(&sm[p & ~1]);
            const uint64_t a = (p & 1) ? w.y : w.x, b = (p & 1) ? w.x : w.y;
            if constexpr (HasEpi<Op>::value) op.store2(c, e + off, a, b, op.epi2(c, e + off));
            else op.store2(c, e + off, a, b);
        }
    }
}

// One limb (or sub-block) b of Op by a CTA of T threads, starting at global stage s0.
template <int M, int LOGB, int T, class Op, class Ctx>
__device__ __forceinline__ void ntt_fwd_block(const Op &op, const Ctx &c, uint64_t *sm, uint32_t rbase) {
    constexpr int REM = LOGB % 3;
    constexpr int FIRST = REM != 0 ? REM : 3;
    fwd_pass<FIRST, true, LOGB, T, 0, false, M>(op, c, sm, rbase);
    fwd_passes<FIRST, LOGB, T, false, M>(op, c, sm, rbase);
    fwd_copy_out<1 << LOGB, T>(op, c, sm, 0);   // coalesced, two coefficients per thread
}

template <int LOGB, int T, class Op>
__device__ __forceinline__ void ntt_fwd_limb(const Op &op, int limb, int s0, uint64_t *sm) {
    const auto c = op.ctx(limb);
    const uint32_t rbase = (1u << s0) + c.lm.sb;
    if constexpr (HasSlack<decltype(c)>::value) {
        if constexpr (WideSlack<Op>::value) {
            if (c.slack == SLACK_WIDE) {
                ntt_fwd_block<SLACK_WIDE, LOGB, T>(op, c, sm, rbase);
                return;
            }
        }
        if (c.slack) {
            ntt_fwd_block<SLACK_M, LOGB, T>(op, c, sm, rbase);
            return;
        }
    }
    ntt_fwd_block<4, LOGB, T>(op, c, sm, rbase);
}

template <int LOGB, int V, class Op>
__global__ void __launch_bounds__(NttCfg<LOGB, V>::THREADS) ntt_fwd_kernel(Op op, int s0) {
    extern __shared__ uint64_t sm[];
    ntt_fwd_limb<LOGB, NttCfg<LOGB, V>::THREADS>(op, blockIdx.x, s0, sm);
}

// ---------------------------------------------------------------- inverse
// Pass of R_LOG Gentleman-Sande stages starting at local stage s; global stage =
// local stage (an inverse CTA always owns the low stages). logn is log2 of the full
// limb length; SCALE folds N^-1 into the pass's last stage.
template <int R_LOG, bool TO_GLOBAL, bool SCALE, int LOGB, int T, int s, bool SIDE, bool W = false, class Op,
          class Ctx>
__device__ __forceinline__ void inv_pass(const Op &op, const Ctx &c, uint64_t *sm, int logn) {
    constexpr int R = 1 << R_LOG;
    constexpr int NB = 1 << LOGB;
    constexpr int G = NB >> R_LOG;
    constexpr int IT = G > 0 ? (G + T - 1) / T : 1;  // groups per thread
    constexpr int GR = SIDE ? IT : 1;                // groups in flight at once
    constexpr bool FULL = G > 0 && G % T == 0;
    const uint64_t q = c.lm.q, q2 = q << 1, q4 = q << 2;
    const uint32_t n = 1u << logn;
#pragma unroll
    for (int i0 = 0; i0 < IT; i0 += GR) {
        uint64_t v[GR][R];
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<true, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const int sb = swz(((g >> s) << (s + R_LOG)) + (g & ((1 << s) - 1)));
#pragma unroll
            for (int k = 0; k < R; k++) v[it][k] = sm[sb ^ swz_delta(k << s)];
        }
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<true, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const int blk = g >> s;
#pragma unroll
            for (int t = 0; t < R_LOG; t++) {
                const int h = 1 << t;
                const int sg = s + t;
                const uint32_t rb =
                    n + 1 - (n >> sg) + (c.lm.sb << (LOGB - sg - 1)) + ((uint32_t)blk << (R_LOG - t - 1));
#pragma unroll
                for (int k = 0; k < R; k++) {
                    if (k & h) continue;
                    if (W && SCALE && t == R_LOG - 1) {
                        const uint64_t u = v[it][k], y = v[it][k + h];
                        v[it][k] = mul_shoup_lazy4(u + y, c.lm.inv_n, c.lm.inv_n_quo, q);
                        v[it][k + h] = mul_shoup_lazy4(u + q4 - y, c.lm.sroot, c.lm.sroot_quo, q);
                    } else if (W) {
                        gs_butterfly_wide(v[it][k], v[it][k + h], __ldg(c.lm.iroots + rb + (k >> (t + 1))), q, q4);
                    } else if (SCALE && t == R_LOG - 1) {
                        uint64_t u = csub(v[it][k], q2);
                        uint64_t y = v[it][k + h];
                        uint64_t sum = u + y;
                        sum = csub(sum, q2);
                        v[it][k] = mul_shoup_lazy(sum, c.lm.inv_n, c.lm.inv_n_quo, q);
                        v[it][k + h] = mul_shoup_lazy(u + q2 - y, c.lm.sroot, c.lm.sroot_quo, q);
                    } else {
                        gs_butterfly(v[it][k], v[it][k + h], __ldg(c.lm.iroots + rb + (k >> (t + 1))), q, q2);
                    }
                }
            }
        }
#pragma unroll
        for (int it = 0; it < GR; it++) {
            const int g = pass_group<true, T, IT>(i0 + it);
            if (!FULL && g >= G) continue;
            const int base = ((g >> s) << (s + R_LOG)) + (g & ((1 << s) - 1));
            const int sb = swz(base);
#pragma unroll
            for (int k = 0; k < R; k++) {
                if constexpr (TO_GLOBAL) op.store(c, base + (k << s), v[it][k]);
                else sm[sb ^ swz_delta(k << s)] = v[it][k];
            }
        }
    }
    // A radix-8 pass at stage s with 2^(s+3) <= 32 IT leaves each warp's 32 IT groups on
    // 256 IT consecutive coefficients, the ones the same warp's groups of the next
    // radix-8 pass (s + 3) read: a warp barrier is enough between the two.
    if constexpr (!TO_GLOBAL) {
        constexpr int LIT = (IT > 1 && T % 32 == 0) ? ilog2c<IT>() : 0;
        constexpr int PASSES_8 = (LOGB % 3) ? LOGB / 3 : LOGB / 3 - 1;   // radix-8 passes before the last
        constexpr bool next_radix8 = s + 3 < 3 * PASSES_8;
        if constexpr (R_LOG == 3 && next_radix8 && s + 3 <= 5 + LIT && T % 32 == 0) __syncwarp();
        else __syncthreads();
    }
}

// Radix-8 passes P .. PASSES-1 (local stages 3P ..), unrolled at compile time.
template <int P, int PASSES, int LOGB, int T, bool SIDE, bool W = false, class Op, class Ctx>
__device__ __forceinline__ void inv_passes(const Op &op, const Ctx &c, uint64_t *sm, int logn) {
    if constexpr (P < PASSES) {
        inv_pass<3, false, false, LOGB, T, 3 * P, SIDE, W>(op, c, sm, logn);
        inv_passes<P + 1, PASSES, LOGB, T, SIDE, W>(op, c, sm, logn);
    }
}

// Copy-in of an inverse transform: coefficient pairs from op.load2 (coefficient e + off)
// into shared memory, then the barrier before the first pass: a warp barrier when the
// copy-in is warp-major and the first pass is a radix-8 pass (each warp then reads
// exactly what it wrote), a CTA barrier otherwise.
template <int LOGB, int T, class Op, class Ctx>
__device__ __forceinline__ void inv_copy_in(const Op &op, const Ctx &c, uint64_t *sm, int off) {
    constexpr int NB = 1 << LOGB;
    constexpr int PASSES_8 = (LOGB % 3) ? LOGB / 3 : LOGB / 3 - 1;
    if constexpr (WarpIO<NB, T>::value) {
#pragma unroll 4
        for (int i = 0; i < NB / (2 * T); i++) {
            const int e = io_pair<NB, T>(i);
            uint64_t a, b;
            op.load2(c, e + off, a, b);
            const int p = swz(e);
            *reinterpret_cast<ulonglong2 *>(&sm[p & ~1]) = (p & 1) ? make_ulonglong2(b, a) : make_ulonglong2(a, b);
        }
        if constexpr (PASSES_8 >= 1) __syncwarp();
        else __syncthreads();
    } else {
        for (int e = threadIdx.x * 2; e < NB; e += T * 2) {
            uint64_t a, b;
            op.load2(c, e + off, a, b);
            const int p = swz(e);
            *reinterpret_cast<ulonglong2 *>(&sm[p & ~1]) = (p & 1) ? make_ulonglong2(b, a) : make_ulonglong2(a, b);
        }
        __syncthreads();
    }
}

// One limb (or sub-block) b of Op by a CTA of T threads; scale_last: this CTA's last
// stage is the transform's last stage (whole limb).
template <int LOGB, int T, class Op>
__device__ __forceinline__ void ntt_inv_limb(const Op &op, int limb, int logn, int scale_last, uint64_t *sm) {
    constexpr int NB = 1 << LOGB;
    constexpr int REM = LOGB % 3;
    const auto c = op.ctx(limb);
    inv_copy_in<LOGB, T>(op, c, sm, 0);
    constexpr int LAST = REM ? REM : 3;
    constexpr int PASSES = REM ? LOGB / 3 : LOGB / 3 - 1;  // radix-8 passes before the last one
    if constexpr (HasInvSlack<decltype(c)>::value) {
        if (c.islack && scale_last) {
            inv_passes<0, PASSES, LOGB, T, false, true>(op, c, sm, logn);
            inv_pass<LAST, true, true, LOGB, T, 3 * PASSES, false, true>(op, c, sm, logn);
            return;
        }
    }
    inv_passes<0, PASSES, LOGB, T, false>(op, c, sm, logn);
    if (scale_last) inv_pass<LAST, true, true, LOGB, T, 3 * PASSES, false>(op, c, sm, logn);
    else inv_pass<LAST, true, false, LOGB, T, 3 * PASSES, false>(op, c, sm, logn);
}

template <int LOGB, int V, class Op>
__global__ void __launch_bounds__(NttCfg<LOGB, V>::THREADS) ntt_inv_kernel(Op op, int logn, int scale_last) {
    extern __shared__ uint64_t sm[];
    ntt_inv_limb<LOGB, NttCfg<LOGB, V>::THREADS>(op, blockIdx.x, logn, scale_last, sm);
}

// ---------------------------------------------------------------- two-CTA limbs
// A limb of 2^(LOGB+1) coefficients transformed by a cluster of two CTAs, each holding
// one half in shared memory. Forward: the first stage (twiddle index 1) joins
// coefficient j with j + 2^LOGB; each CTA loads both operands of its butterflies and
// keeps the output in its own half (the first stage runs twice, once per CTA); one
// cluster barrier before the stores keeps an in-place transform from overwriting a half
// the partner CTA still reads. Inverse: the last stage (the N^-1-scaled pair) reads and writes the
// partner CTA's half through distributed shared memory between two cluster barriers.
// Every other stage runs inside one half exactly as the sub-block passes of the split
// transform (sub-block = half). One launch, the same arithmetic and order as the split
// transform, and the Op's load / store see whole-limb coefficient indices, so every
// fused operation works at this length unchanged.
template <int LOGB, int V, class Op>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NttCfg<LOGB, V>::THREADS)
    ntt_fwd_pair_kernel(Op op) {
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB;
    constexpr int T = NttCfg<LOGB, V>::THREADS;
    constexpr int REM = NttCfg<LOGB, V>::REM;
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    const unsigned half = cl.block_rank();
    auto c = op.ctx((int)(blockIdx.x >> 1));
    c.lm.sb = half;
    {
        const uint64_t q = c.lm.q, q2 = q << 1;
        const ulonglong2 w = __ldg(c.lm.roots + 1);
        for (int j = threadIdx.x; j < NB; j += T) {
            uint64_t x = op.load(c, j), y = op.load(c, j + NB);
            ct_butterfly(x, y, w, q, q2);
            sm[swz(j)] = half ? y : x;
        }
    }
    __syncthreads();
    const uint32_t rbase = 2u + half;   // global stage 1 onwards, sub-block = half
    constexpr int FIRST = REM != 0 ? REM : 3;
    fwd_pass<FIRST, false, LOGB, T, 0, false>(op, c, sm, rbase);
    fwd_passes<FIRST, LOGB, T, false>(op, c, sm, rbase);
    cl.sync();   // both CTAs have read every input coefficient
    fwd_copy_out<NB, T>(op, c, sm, (int)half << LOGB);
}

template <int LOGB, int V, class Op>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(NttCfg<LOGB, V>::THREADS)
    ntt_inv_pair_kernel(Op op) {
    namespace cg = cooperative_groups;
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB;
    constexpr int T = NttCfg<LOGB, V>::THREADS;
    constexpr int REM = NttCfg<LOGB, V>::REM;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned half = cl.block_rank();
    auto c = op.ctx((int)(blockIdx.x >> 1));
    c.lm.sb = half;
    const int off = (int)half << LOGB;
    inv_copy_in<LOGB, T>(op, c, sm, off);
    constexpr int LAST = REM ? REM : 3;
    constexpr int PASSES = REM ? LOGB / 3 : LOGB / 3 - 1;
    inv_passes<0, PASSES, LOGB, T, false>(op, c, sm, LOGB + 1);
    inv_pass<LAST, false, false, LOGB, T, 3 * PASSES, false>(op, c, sm, LOGB + 1);
    cl.sync();
    {
        uint64_t *lo = cl.map_shared_rank(sm, 0u), *hi = cl.map_shared_rank(sm, 1u);
        const uint64_t q = c.lm.q, q2 = q << 1;
        for (int j = (int)half * (NB / 2) + threadIdx.x; j < (int)(half + 1) * (NB / 2); j += T) {
            const int p = swz(j);
            const uint64_t x = lo[p], y = hi[p];
            const uint64_t u = csub(x, q2);
            uint64_t sum = u + y;
            sum = csub(sum, q2);
            lo[p] = mul_shoup_lazy(sum, c.lm.inv_n, c.lm.inv_n_quo, q);
            hi[p] = mul_shoup_lazy(u + q2 - y, c.lm.sroot, c.lm.sroot_quo, q);
        }
    }
    cl.sync();
    for (int e = threadIdx.x; e < NB; e += T) op.store(c, e + off, sm[swz(e)]);
}

// ---------------------------------------------------------------- clusters of 4 and 8 CTAs
// A limb of 2^(LOGB+CLOG) coefficients (CLOG = 2, 3: N = 65536, 131072 at LOGB = 14)
// transformed by a cluster of 2^CLOG CTAs, CTA r holding block r (coefficients
// r 2^LOGB .. (r+1) 2^LOGB - 1) in its shared memory. The stages whose butterflies join
// two blocks (forward: the first CLOG; inverse: the last CLOG, the N^-1-scaled one last)
// run between cluster barriers: the two CTAs of a pair of partner blocks each compute
// half of the pair's butterflies, reading and writing both blocks through distributed
// shared memory. Every other stage runs inside a block exactly as the sub-block passes
// of the split transform. The butterflies and their order are those of the split
// transform, so outputs (lazy values included) are the same, and the Op's loads and
// stores see whole-limb coefficient indices as in every other form.

// One cross-block stage over partner blocks xs (lower) and ys (upper): this CTA takes
// butterflies j0 .. j0 + NB/2 - 1 of the pair (the same slot in both blocks).
template <bool FWD, bool SCALE, int NB, int T>
__device__ __forceinline__ void cross_stage(uint64_t *xs, uint64_t *ys, int j0, ulonglong2 w, const NttLimb &lm) {
    constexpr int IT = NB / 2 / T;
    constexpr int U = IT >= 4 ? 4 : IT;
    static_assert(IT * T == NB / 2 && IT % U == 0, "cross stage split");
    const uint64_t q = lm.q, q2 = q << 1;
#pragma unroll 1
    for (int i0 = 0; i0 < IT; i0 += U) {
        uint64_t x[U], y[U];
        int p[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            p[u] = swz(j0 + threadIdx.x + (i0 + u) * T);
            x[u] = xs[p[u]];
            y[u] = ys[p[u]];
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if constexpr (FWD) {
                ct_butterfly(x[u], y[u], w, q, q2);
            } else if constexpr (SCALE) {
                const uint64_t a = csub(x[u], q2);
                uint64_t sum = a + y[u];
                sum = csub(sum, q2);
                const uint64_t dif = a + q2 - y[u];
                x[u] = mul_shoup_lazy(sum, lm.inv_n, lm.inv_n_quo, q);
                y[u] = mul_shoup_lazy(dif, lm.sroot, lm.sroot_quo, q);
            } else {
                gs_butterfly(x[u], y[u], w, q, q2);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            xs[p[u]] = x[u];
            ys[p[u]] = y[u];
        }
    }
}

template <int LOGB, int CLOG, class Op>
__global__ void __cluster_dims__(1 << CLOG, 1, 1) __launch_bounds__(NttCfg<LOGB, 0>::THREADS)
    ntt_fwd_cluster_kernel(Op op) {
    namespace cg = cooperative_groups;
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB, C = 1 << CLOG;
    constexpr int T = NttCfg<LOGB, 0>::THREADS;
    constexpr int REM = NttCfg<LOGB, 0>::REM;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned r = cl.block_rank();
    auto c = op.ctx((int)(blockIdx.x >> CLOG));
    c.lm.sb = r;
    const int off = (int)r << LOGB;
    for (int j = threadIdx.x; j < NB; j += T) sm[swz(j)] = op.load(c, j + off);
    cl.sync();   // every block loaded (and every input read: in-place stores are safe later)
#pragma unroll
    for (int s = 0; s < CLOG; s++) {
        const unsigned G = (unsigned)C >> (s + 1);   // partner distance in blocks
        const unsigned lo = r & ~G;
        const ulonglong2 w = __ldg(c.lm.roots + (1u << s) + (lo >> (CLOG - s)));
        cross_stage<true, false, NB, T>(cl.map_shared_rank(sm, lo), cl.map_shared_rank(sm, lo | G),
                                        (r & G) ? NB / 2 : 0, w, c.lm);
        cl.sync();
    }
    const uint32_t rbase = (1u << CLOG) + r;   // global stage CLOG onwards, sub-block = r
    constexpr int FIRST = REM != 0 ? REM : 3;
    fwd_pass<FIRST, false, LOGB, T, 0, false>(op, c, sm, rbase);
    fwd_passes<FIRST, LOGB, T, false>(op, c, sm, rbase);
    fwd_copy_out<NB, T>(op, c, sm, off);
}

template <int LOGB, int CLOG, class Op>
__global__ void __cluster_dims__(1 << CLOG, 1, 1) __launch_bounds__(NttCfg<LOGB, 0>::THREADS)
    ntt_inv_cluster_kernel(Op op) {
    namespace cg = cooperative_groups;
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB;
    constexpr int LOGN = LOGB + CLOG;
    constexpr uint32_t N = 1u << LOGN;
    constexpr int T = NttCfg<LOGB, 0>::THREADS;
    constexpr int REM = NttCfg<LOGB, 0>::REM;
    cg::cluster_group cl = cg::this_cluster();
    const unsigned r = cl.block_rank();
    auto c = op.ctx((int)(blockIdx.x >> CLOG));
    c.lm.sb = r;
    const int off = (int)r << LOGB;
    inv_copy_in<LOGB, T>(op, c, sm, off);
    constexpr int LAST = REM ? REM : 3;
    constexpr int PASSES = REM ? LOGB / 3 : LOGB / 3 - 1;
    inv_passes<0, PASSES, LOGB, T, false>(op, c, sm, LOGN);
    inv_pass<LAST, false, false, LOGB, T, 3 * PASSES, false>(op, c, sm, LOGN);
    cl.sync();
#pragma unroll
    for (int s = 0; s < CLOG; s++) {
        const unsigned G = 1u << s;   // global stage LOGB + s joins blocks G apart
        const unsigned lo = r & ~G;
        uint64_t *xs = cl.map_shared_rank(sm, lo), *ys = cl.map_shared_rank(sm, lo | G);
        const int j0 = (r & G) ? NB / 2 : 0;
        if (s + 1 < CLOG) {
            const int sg = LOGB + s;
            const ulonglong2 w = __ldg(c.lm.iroots + (N + 1 - (N >> sg) + (lo >> (s + 1))));
            cross_stage<false, false, NB, T>(xs, ys, j0, w, c.lm);
        } else {
            cross_stage<false, true, NB, T>(xs, ys, j0, make_ulonglong2(0, 0), c.lm);
        }
        cl.sync();
    }
    for (int e = threadIdx.x; e < NB; e += T) op.store(c, e + off, sm[swz(e)]);
}

template <int LOGB>
inline size_t ntt_smem_bytes() {
    return sizeof(uint64_t) * (size_t)(1 << LOGB);
}

__device__ __forceinline__ NttLimb make_limb(const Mod &m, uint32_t sb) {
    NttLimb l;
    l.q = m.value;
    l.roots = m.roots;
    l.iroots = m.inv_roots;
    l.inv_n = m.inv_n;
    l.inv_n_quo = m.inv_n_quo;
    l.sroot = m.sroot;
    l.sroot_quo = m.sroot_quo;
    l.sb = sb;
    return l;
}

constexpr int MAX_LOGB = 14;  // 16384 coefficients = 128 KB of shared memory per CTA
constexpr int PAIR_LOGN = MAX_LOGB + 1;   // whole limbs on a CTA pair
constexpr int MAX_CLUSTER_LOG = 3;        // clusters of up to 8 CTAs (the portable size)
constexpr int MAX_FUSED_LOGN = MAX_LOGB + MAX_CLUSTER_LOG;  // longest limb of the fused operations

template <int LOGB, int V, class Op>
inline cudaError_t launch_fwd(const Op &op, unsigned blocks, int s0, cudaStream_t s) {
    const size_t smem = ntt_smem_bytes<LOGB>();
    auto k = ntt_fwd_kernel<LOGB, V, Op>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k<<<blocks, NttCfg<LOGB, V>::THREADS, smem, s>>>(op, s0);
    return cudaGetLastError();
}

template <int LOGB, int V, class Op>
inline cudaError_t launch_inv(const Op &op, unsigned blocks, int logn, int scale_last, cudaStream_t s) {
    const size_t smem = ntt_smem_bytes<LOGB>();
    auto k = ntt_inv_kernel<LOGB, V, Op>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k<<<blocks, NttCfg<LOGB, V>::THREADS, smem, s>>>(op, logn, scale_last);
    return cudaGetLastError();
}

// Tuned thread-count variant per (direction, log2 block size); 0 = default. Written by
// the tuner (tune.cu), read at every launch.
int ntt_variant(bool fwd, int logb);
// Streaming multiprocessors of the current device (cached per device).
int sm_count();
// Whether launches of fewer limbs than SMs take the two-CTA form (tb_ntt_set_small_launch_pairs).
bool small_launch_pairs();

// Whole limbs of 2^(LOGB+1) coefficients, one CTA pair each (forward from stage 0,
// inverse with the N^-1 scaling).
template <bool FWD, int LOGB, int V, class Op>
inline cudaError_t launch_pair(const Op &op, unsigned blocks, cudaStream_t s) {
    if (blocks > 0x3fffffffu) return cudaErrorInvalidValue;
    const size_t smem = ntt_smem_bytes<LOGB>();
    auto k = [] {
        if constexpr (FWD) return ntt_fwd_pair_kernel<LOGB, V, Op>;
        else return ntt_inv_pair_kernel<LOGB, V, Op>;
    }();
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k<<<2 * blocks, NttCfg<LOGB, V>::THREADS, smem, s>>>(op);
    return cudaGetLastError();
}

// Whole limbs of 2^(LOGB+CLOG) coefficients, one cluster of 2^CLOG CTAs each (forward
// from stage 0, inverse with the N^-1 scaling). A device that cannot hold one such
// cluster at once is refused before the launch.
template <bool FWD, int LOGB, int CLOG, class Op>
inline cudaError_t launch_cluster(const Op &op, unsigned blocks, cudaStream_t s) {
    if (blocks > (0x7fffffffu >> CLOG)) return cudaErrorInvalidValue;
    const size_t smem = ntt_smem_bytes<LOGB>();
    constexpr int T = NttCfg<LOGB, 0>::THREADS;
    auto k = [] {
        if constexpr (FWD) return ntt_fwd_cluster_kernel<LOGB, CLOG, Op>;
        else return ntt_inv_cluster_kernel<LOGB, CLOG, Op>;
    }();
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    static int fits = -1;   // per instantiation: clusters that can be resident at once
    if (fits < 0) {
        cudaLaunchConfig_t cfg = {};
        cudaLaunchAttribute attr;
        attr.id = cudaLaunchAttributeClusterDimension;
        attr.val.clusterDim.x = 1u << CLOG;
        attr.val.clusterDim.y = 1;
        attr.val.clusterDim.z = 1;
        cfg.gridDim = dim3(1u << CLOG);
        cfg.blockDim = dim3(T);
        cfg.dynamicSmemBytes = smem;
        cfg.attrs = &attr;
        cfg.numAttrs = 1;
        int n = 0;
        e = cudaOccupancyMaxActiveClusters(&n, k, &cfg);
        if (e != cudaSuccess) return e;
        fits = n;
    }
    if (fits < 1) return cudaErrorInvalidClusterSize;
    k<<<blocks << CLOG, T, smem, s>>>(op);
    return cudaGetLastError();
}

template <bool FWD, int LOGB, int V, class Op>
inline cudaError_t launch_ntt(const Op &op, unsigned blocks, int s0_or_logn, int scale_last, cudaStream_t s) {
    if constexpr (V >= 3) {
        const bool whole = FWD ? s0_or_logn == 0 : (s0_or_logn == LOGB && scale_last);
        if (whole) return launch_pair<FWD, LOGB - 1, V - 3>(op, blocks, s);
        return launch_ntt<FWD, LOGB, V - 3>(op, blocks, s0_or_logn, scale_last, s);
    } else if constexpr (FWD) {
        return launch_fwd<LOGB, V>(op, blocks, s0_or_logn, s);
    } else {
        return launch_inv<LOGB, V>(op, blocks, s0_or_logn, scale_last, s);
    }
}

// ---------------------------------------------------------------- several shapes, one launch
// Whole limbs of up to MAX_SHAPES groups of ring degrees 2^12 .. 2^14, each group with
// its own Op (context tables, buffers, level), transformed by one persistent launch: as
// many CTAs of 1024 threads as the SMs hold at once, each taking the next limb from a
// device counter until every limb of every group is done (no CTA waits on another).
// Groups come largest degree first, so the cheap limbs of the small rings fill the last
// round of the large ones. A limb runs exactly as in the one-CTA kernels (same passes,
// same butterflies), only with 1024 threads at every degree.
constexpr int MAX_SHAPES = 8;
constexpr int SHAPE_THREADS = 1024;

template <class Op>
struct ShapeTable {
    int count = 0;
    Op op[MAX_SHAPES];
    int logn[MAX_SHAPES];
    unsigned first[MAX_SHAPES + 1];   // limbs of group g: items first[g] .. first[g+1]-1
};

template <bool FWD, class Op>
__global__ void __launch_bounds__(SHAPE_THREADS) ntt_shapes_kernel(ShapeTable<Op> t, unsigned *counter) {
    extern __shared__ uint64_t sm[];
    __shared__ unsigned next;
    const unsigned total = t.first[t.count];
    for (;;) {
        if (threadIdx.x == 0) next = atomicAdd(counter, 1u);
        __syncthreads();
        const unsigned item = next;
        __syncthreads();   // every thread has the item before thread 0 takes the next one
        if (item >= total) return;
        int g = 0;
        while (g + 1 < t.count && item >= t.first[g + 1]) g++;
        const Op op = t.op[g];
        const int limb = (int)(item - t.first[g]);
        if constexpr (FWD) {
            if (t.logn[g] == 14) ntt_fwd_limb<14, SHAPE_THREADS>(op, limb, 0, sm);
            else if (t.logn[g] == 13) ntt_fwd_limb<13, SHAPE_THREADS>(op, limb, 0, sm);
            else ntt_fwd_limb<12, SHAPE_THREADS>(op, limb, 0, sm);
        } else {
            if (t.logn[g] == 14) ntt_inv_limb<14, SHAPE_THREADS>(op, limb, 14, 1, sm);
            else if (t.logn[g] == 13) ntt_inv_limb<13, SHAPE_THREADS>(op, limb, 13, 1, sm);
            else ntt_inv_limb<12, SHAPE_THREADS>(op, limb, 12, 1, sm);
        }
        __syncthreads();   // shared memory free for the next limb
    }
}

// counter: one device word, zeroed here before the launch (stream-ordered).
template <bool FWD, class Op>
inline cudaError_t launch_shapes(const ShapeTable<Op> &t, unsigned *counter, cudaStream_t s) {
    if (t.count < 1 || t.count > MAX_SHAPES || !counter) return cudaErrorInvalidValue;
    int maxlog = 0;
    for (int g = 0; g < t.count; g++) {
        if (t.logn[g] < 12 || t.logn[g] > MAX_LOGB) return cudaErrorInvalidValue;
        maxlog = t.logn[g] > maxlog ? t.logn[g] : maxlog;
    }
    const unsigned total = t.first[t.count];
    if (!total) return cudaSuccess;
    const size_t smem = sizeof(uint64_t) << maxlog;
    auto k = ntt_shapes_kernel<FWD, Op>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(8 << MAX_LOGB));
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, SHAPE_THREADS, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const unsigned grid = std::min<unsigned>(total, (unsigned)(sm_count() * per_sm));
    e = cudaMemsetAsync(counter, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    k<<<grid, SHAPE_THREADS, smem, s>>>(t, counter);
    return cudaGetLastError();
}

// A launch of at most half as many limbs as the device has SMs leaves most SMs idle with
// one CTA per limb: it takes the two-CTA form of the same thread count, which puts twice
// as many CTAs to work (one pair per call chain, as the reference drives the evaluator:
// +43% ops/s at N = 16384). Larger launches keep the tuned variant (nearer a full wave
// the one-CTA form is faster: the pair form exchanges a stage through distributed
// shared memory or loads its limb twice).
inline int small_launch_variant(int v, unsigned blocks) {
    return (v < 3 && small_launch_pairs() && 2 * blocks <= (unsigned)sm_count()) ? v + 3 : v;
}

// Dispatch on log2 of the CTA block (1 .. 14); block sizes 2^12 .. 2^14 carry variants
// with half and a quarter of the threads and their CTA-pair forms. 15, 16, 17: whole
// limbs of 2^15, 2^16, 2^17 coefficients on CTA pairs and clusters of 4 and 8 CTAs
// (forward from stage 0 only, inverse with the scaling only).
template <bool FWD, class Op>
cudaError_t dispatch_ntt(int logb, const Op &op, unsigned blocks, int s0_or_logn, int scale_last, cudaStream_t s) {
#define TB_CASE(B) \
    case B:        \
        return launch_ntt<FWD, B, 0>(op, blocks, s0_or_logn, scale_last, s);
#define TB_CASE2(B)                                                                  \
    case B:                                                                          \
        switch (small_launch_variant(ntt_variant(FWD, B), blocks)) {                 \
        case 1:                                                                      \
            return launch_ntt<FWD, B, 1>(op, blocks, s0_or_logn, scale_last, s);     \
        case 2:                                                                      \
            return launch_ntt<FWD, B, 2>(op, blocks, s0_or_logn, scale_last, s);     \
        case 3:                                                                      \
            return launch_ntt<FWD, B, 3>(op, blocks, s0_or_logn, scale_last, s);     \
        case 4:                                                                      \
            return launch_ntt<FWD, B, 4>(op, blocks, s0_or_logn, scale_last, s);     \
        case 5:                                                                      \
            return launch_ntt<FWD, B, 5>(op, blocks, s0_or_logn, scale_last, s);     \
        default:                                                                     \
            return launch_ntt<FWD, B, 0>(op, blocks, s0_or_logn, scale_last, s);     \
        }
    switch (logb) {
        TB_CASE(1) TB_CASE(2) TB_CASE(3) TB_CASE(4) TB_CASE(5) TB_CASE(6) TB_CASE(7)
        TB_CASE(8) TB_CASE(9) TB_CASE(10) TB_CASE(11) TB_CASE2(12) TB_CASE2(13) TB_CASE2(14)
    case PAIR_LOGN:
        if (FWD ? s0_or_logn != 0 : (s0_or_logn != PAIR_LOGN || !scale_last)) return cudaErrorInvalidValue;
        return launch_pair<FWD, MAX_LOGB, 0>(op, blocks, s);
    case MAX_LOGB + 2:
        if (FWD ? s0_or_logn != 0 : (s0_or_logn != MAX_LOGB + 2 || !scale_last)) return cudaErrorInvalidValue;
        return launch_cluster<FWD, MAX_LOGB, 2>(op, blocks, s);
    case MAX_LOGB + 3:
        if (FWD ? s0_or_logn != 0 : (s0_or_logn != MAX_LOGB + 3 || !scale_last)) return cudaErrorInvalidValue;
        return launch_cluster<FWD, MAX_LOGB, 3>(op, blocks, s);
    default:
        return cudaErrorInvalidValue;
    }
#undef TB_CASE
#undef TB_CASE2
}

}  // namespace tb

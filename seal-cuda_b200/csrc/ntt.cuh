// Negacyclic NTT / inverse NTT kernels for sm_100a.
//
// One CTA transforms one polynomial limb (or one 2^LOGB sub-block of a larger one)
// entirely inside shared memory. Stages are grouped into radix-8 register passes
// (remainder stages in the first forward / last inverse pass): a thread loads 8
// coefficients, runs three Cooley-Tukey (forward) or Gentleman-Sande (inverse)
// stages in registers with Shoup twiddles, and writes them back; the shared-memory
// slot of coefficient e is swz(e), which keeps every pass bank-conflict free.
//
// The butterflies and lazy ranges are those of the reference's DWTHandler
// (src/utils/dwthandler.h:88-372, src/utils/ntt.h:17-60), so full and lazy
// outputs are bit-identical to nttNegacyclicHarvey[Lazy] /
// inverseNttNegacyclicHarvey[Lazy] (src/utils/ntt.cpp:158-213); the N^-1 scaling is
// folded into the last inverse stage exactly as there.
//
// Each kernel is parameterised by an operation `Op` that maps a CTA to its limb
// (pointers + modulus) and supplies the global-memory load of the first pass and
// the store of the last, so base conversions, key-switch mod-up/mod-down and
// rescaling steps fuse into the transform instead of running as extra passes.
#pragma once

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

template <int LOGB>
struct NttCfg {
    static constexpr int NB = 1 << LOGB;
    static constexpr int THREADS = NB >= 8192 ? 1024 : (NB / 8 >= 64 ? NB / 8 : 64);
    static constexpr int REM = LOGB % 3;
};

__device__ __forceinline__ void ct_butterfly(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    uint64_t u = x >= q2 ? x - q2 : x;
    uint64_t v = mul_shoup_lazy(y, w.x, w.y, q);
    x = u + v;
    y = u + q2 - v;
}

__device__ __forceinline__ void gs_butterfly(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    uint64_t u = x, v = y;
    uint64_t s = u + v;
    x = s >= q2 ? s - q2 : s;
    y = mul_shoup_lazy(u + q2 - v, w.x, w.y, q);
}

// ---------------------------------------------------------------- forward
// Pass of R_LOG Cooley-Tukey stages starting at local stage s. rbase = 2^s0 + sb
// where s0 is the global stage of local stage 0 (0 when the CTA owns the limb).
template <int R_LOG, bool FROM_GLOBAL, int LOGB, class Op, class Ctx>
__device__ __forceinline__ void fwd_pass(const Op &op, const Ctx &c, uint64_t *sm, int s, uint32_t rbase) {
    constexpr int R = 1 << R_LOG;
    constexpr int NB = 1 << LOGB;
    constexpr int G = NB >> R_LOG;
    constexpr int T = NttCfg<LOGB>::THREADS;
    const uint64_t q = c.lm.q, q2 = q << 1;
    const int logsub = LOGB - s - R_LOG;
    for (int g = threadIdx.x; g < G; g += T) {
        const int j = g & ((1 << logsub) - 1);
        const int bi = g >> logsub;
        const int base = (bi << (LOGB - s)) + j;
        uint64_t v[R];
#pragma unroll
        for (int k = 0; k < R; k++) {
            const int e = base + (k << logsub);
            if constexpr (FROM_GLOBAL) v[k] = op.load(c, e);
            else v[k] = sm[swz(e)];
        }
        const uint32_t X = (rbase << s) + (uint32_t)bi;
#pragma unroll
        for (int t = 0; t < R_LOG; t++) {
            const int half = R >> (t + 1);
#pragma unroll
            for (int k = 0; k < R; k++) {
                if (k & half) continue;
                const uint32_t ri = (X << t) + (uint32_t)(k >> (R_LOG - t));
                ct_butterfly(v[k], v[k + half], __ldg(&c.lm.roots[ri]), q, q2);
            }
        }
#pragma unroll
        for (int k = 0; k < R; k++) sm[swz(base + (k << logsub))] = v[k];
    }
    __syncthreads();
}

template <int LOGB, class Op>
__global__ void __launch_bounds__(NttCfg<LOGB>::THREADS) ntt_fwd_kernel(Op op, int s0) {
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB;
    constexpr int T = NttCfg<LOGB>::THREADS;
    constexpr int REM = NttCfg<LOGB>::REM;
    const auto c = op.ctx(blockIdx.x);
    const uint32_t rbase = (1u << s0) + c.lm.sb;
    int s;
    if constexpr (REM != 0) {
        fwd_pass<REM, true, LOGB>(op, c, sm, 0, rbase);
        s = REM;
    } else {
        fwd_pass<3, true, LOGB>(op, c, sm, 0, rbase);
        s = 3;
    }
    for (; s < LOGB; s += 3) fwd_pass<3, false, LOGB>(op, c, sm, s, rbase);
    // coalesced copy-out, two coefficients per thread
    for (int e = threadIdx.x * 2; e < NB; e += T * 2) {
        const int p = swz(e);
        const ulonglong2 w = *reinterpret_cast<const ulonglong2 *>(&sm[p & ~1]);
        if (p & 1) op.store2(c, e, w.y, w.x);
        else op.store2(c, e, w.x, w.y);
    }
}

// ---------------------------------------------------------------- inverse
// Pass of R_LOG Gentleman-Sande stages starting at local stage s; global stage =
// local stage (an inverse CTA always owns the low stages). logn is log2 of the full
// limb length; SCALE folds N^-1 into the pass's last stage.
template <int R_LOG, bool TO_GLOBAL, bool SCALE, int LOGB, class Op, class Ctx>
__device__ __forceinline__ void inv_pass(const Op &op, const Ctx &c, uint64_t *sm, int s, int logn) {
    constexpr int R = 1 << R_LOG;
    constexpr int NB = 1 << LOGB;
    constexpr int G = NB >> R_LOG;
    constexpr int T = NttCfg<LOGB>::THREADS;
    const uint64_t q = c.lm.q, q2 = q << 1;
    const uint32_t n = 1u << logn;
    for (int g = threadIdx.x; g < G; g += T) {
        const int j = g & ((1 << s) - 1);
        const int blk = g >> s;
        const int base = (blk << (s + R_LOG)) + j;
        uint64_t v[R];
#pragma unroll
        for (int k = 0; k < R; k++) v[k] = sm[swz(base + (k << s))];
#pragma unroll
        for (int t = 0; t < R_LOG; t++) {
            const int h = 1 << t;
            const int sg = s + t;
            const uint32_t rb = n + 1 - (n >> sg) + (c.lm.sb << (LOGB - sg - 1)) + ((uint32_t)blk << (R_LOG - t - 1));
#pragma unroll
            for (int k = 0; k < R; k++) {
                if (k & h) continue;
                if (SCALE && t == R_LOG - 1) {
                    uint64_t u = v[k] >= q2 ? v[k] - q2 : v[k];
                    uint64_t y = v[k + h];
                    uint64_t sum = u + y;
                    sum = sum >= q2 ? sum - q2 : sum;
                    v[k] = mul_shoup_lazy(sum, c.lm.inv_n, c.lm.inv_n_quo, q);
                    v[k + h] = mul_shoup_lazy(u + q2 - y, c.lm.sroot, c.lm.sroot_quo, q);
                } else {
                    const uint32_t ri = rb + (uint32_t)(k >> (t + 1));
                    gs_butterfly(v[k], v[k + h], __ldg(&c.lm.iroots[ri]), q, q2);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < R; k++) {
            const int e = base + (k << s);
            if constexpr (TO_GLOBAL) op.store(c, e, v[k]);
            else sm[swz(e)] = v[k];
        }
    }
    if constexpr (!TO_GLOBAL) __syncthreads();
}

// scale_last: this CTA's last stage is the transform's last stage (whole limb).
template <int LOGB, class Op>
__global__ void __launch_bounds__(NttCfg<LOGB>::THREADS) ntt_inv_kernel(Op op, int logn, int scale_last) {
    extern __shared__ uint64_t sm[];
    constexpr int NB = 1 << LOGB;
    constexpr int T = NttCfg<LOGB>::THREADS;
    constexpr int REM = NttCfg<LOGB>::REM;
    const auto c = op.ctx(blockIdx.x);
    for (int e = threadIdx.x * 2; e < NB; e += T * 2) {
        uint64_t a, b;
        op.load2(c, e, a, b);
        const int p = swz(e);
        ulonglong2 w;
        if (p & 1) w = make_ulonglong2(b, a);
        else w = make_ulonglong2(a, b);
        *reinterpret_cast<ulonglong2 *>(&sm[p & ~1]) = w;
    }
    __syncthreads();
    constexpr int LAST = REM ? REM : 3;
    constexpr int FULL = REM ? LOGB / 3 : LOGB / 3 - 1;  // radix-8 passes before the last one
    int s = 0;
    for (int p = 0; p < FULL; p++, s += 3) inv_pass<3, false, false, LOGB>(op, c, sm, s, logn);
    if (scale_last) inv_pass<LAST, true, true, LOGB>(op, c, sm, s, logn);
    else inv_pass<LAST, true, false, LOGB>(op, c, sm, s, logn);
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

template <int LOGB, class Op>
inline cudaError_t launch_fwd(const Op &op, unsigned blocks, int s0, cudaStream_t s) {
    const size_t smem = ntt_smem_bytes<LOGB>();
    auto k = ntt_fwd_kernel<LOGB, Op>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k<<<blocks, NttCfg<LOGB>::THREADS, smem, s>>>(op, s0);
    return cudaGetLastError();
}

template <int LOGB, class Op>
inline cudaError_t launch_inv(const Op &op, unsigned blocks, int logn, int scale_last, cudaStream_t s) {
    const size_t smem = ntt_smem_bytes<LOGB>();
    auto k = ntt_inv_kernel<LOGB, Op>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    k<<<blocks, NttCfg<LOGB>::THREADS, smem, s>>>(op, logn, scale_last);
    return cudaGetLastError();
}

// Dispatch on log2 of the CTA block (1 .. 14).
template <bool FWD, class Op>
cudaError_t dispatch_ntt(int logb, const Op &op, unsigned blocks, int s0_or_logn, int scale_last, cudaStream_t s) {
#define TB_CASE(B)                                                          \
    case B:                                                                 \
        if constexpr (FWD) return launch_fwd<B>(op, blocks, s0_or_logn, s); \
        else return launch_inv<B>(op, blocks, s0_or_logn, scale_last, s);
    switch (logb) {
        TB_CASE(1) TB_CASE(2) TB_CASE(3) TB_CASE(4) TB_CASE(5) TB_CASE(6) TB_CASE(7)
        TB_CASE(8) TB_CASE(9) TB_CASE(10) TB_CASE(11) TB_CASE(12) TB_CASE(13) TB_CASE(14)
    default:
        return cudaErrorInvalidValue;
    }
#undef TB_CASE
}


}  // namespace tb

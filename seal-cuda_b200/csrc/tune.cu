// Tuning knobs and the autotuner.
//
// Knobs: the NTT thread-count variant per (direction, log2 block size) and the key-
// switch scratch budget (how many ciphertexts one key-switch launch sequence takes).
// The autotuner times the candidates of a knob on the caller's device with CUDA
// events on scratch data and keeps the fastest; results are process-wide. All
// variants compute identical words, so tuning changes speed only.
#include <algorithm>
#include <atomic>
#include <cstdlib>
#include <vector>

#include "../../include/troy_b200.h"
#include "context.hpp"
#include "ntt.cuh"

namespace tb {

namespace {
std::atomic<int> g_variant[2][MAX_LOGB + 1];
std::atomic<unsigned long long> g_ks_budget{0};
std::atomic<int> g_small_pairs{1};
}  // namespace

bool small_launch_pairs() { return g_small_pairs.load(std::memory_order_relaxed) != 0; }

int sm_count() {
    static std::atomic<int> cached[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    int v = cached[dev].load(std::memory_order_relaxed);
    if (v > 0) return v;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) return 148;
    cached[dev].store(v, std::memory_order_relaxed);
    return v;
}

int ntt_variant(bool fwd, int logb) {
    if (logb < 0 || logb > MAX_LOGB) return 0;
    return g_variant[fwd ? 1 : 0][logb].load(std::memory_order_relaxed);
}

// Key switching of one context through the persistent one-launch-per-step form
// (keyswitch_shapes) instead of one CTA per limb (tb_keyswitch_set_persistent).
std::atomic<int> g_ks_persistent{0};
bool ks_persistent() { return g_ks_persistent.load(std::memory_order_relaxed) != 0; }

size_t ks_scratch_budget() {
    unsigned long long v = g_ks_budget.load(std::memory_order_relaxed);
    if (v) return (size_t)v;
    const char *e = getenv("TB_KS_SCRATCH_BYTES");
    return e ? (size_t)strtoull(e, nullptr, 10) : (size_t)(2ull << 30);
}

int ntt_forward(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s);
int ntt_inverse(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s);

// Median device time of `reps` calls of f after one warm-up call.
template <class F>
static float time_call(F &&f, cudaStream_t s, int reps, int &status) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    std::vector<float> ms;
    status = f();
    for (int r = 0; r < reps && status == TB_OK; r++) {
        cudaEventRecord(a, s);
        status = f();
        cudaEventRecord(b, s);
        cudaEventSynchronize(b);
        float t = 0;
        cudaEventElapsedTime(&t, a, b);
        ms.push_back(t);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms.empty()) return 0;
    std::sort(ms.begin(), ms.end());
    return ms[ms.size() / 2];
}

// Times every variant of the forward and inverse transform of the context's degree
// on `polys` limbs of scratch and keeps the fastest of each.
int autotune_ntt(Context &c, uint64_t polys, cudaStream_t s, int *chosen_fwd, int *chosen_inv) {
    const int logb = c.logn;
    if (logb < 12 || logb > MAX_LOGB) {
        if (chosen_fwd) *chosen_fwd = 0;
        if (chosen_inv) *chosen_inv = 0;
        return TB_OK;  // one variant only
    }
    if (!polys) polys = 256;
    const int limbs = (int)std::min<size_t>(c.chain.size(), polys);
    const uint64_t P = (polys + limbs - 1) / limbs;
    uint64_t *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, 8ull * P * limbs * c.n, s);
    if (e != cudaSuccess) return status_from(e);
    e = cudaMemsetAsync(buf, 0, 8ull * P * limbs * c.n, s);
    int st = e == cudaSuccess ? TB_OK : status_from(e);
    for (int dir = 1; dir >= 0 && st == TB_OK; dir--) {
        float best = 0;
        int best_v = 0;
        for (int v = 0; v < NTT_VARIANTS && st == TB_OK; v++) {
            g_variant[dir][logb].store(v);
            const float t = time_call(
                [&] {
                    return dir ? ntt_forward(c, buf, buf, P, 0, limbs, false, s)
                               : ntt_inverse(c, buf, buf, P, 0, limbs, false, s);
                },
                s, 5, st);
            if (st == TB_OK && (v == 0 || t < best)) {
                best = t;
                best_v = v;
            }
        }
        g_variant[dir][logb].store(best_v);
        if (dir && chosen_fwd) *chosen_fwd = best_v;
        if (!dir && chosen_inv) *chosen_inv = best_v;
    }
    cudaFreeAsync(buf, s);
    return st;
}

// The integer ceiling of the transforms: the rate of the lazy Cooley-Tukey butterfly
// (ct_butterfly, the one every forward NTT pass runs) with its operands and twiddles in
// registers, so that nothing but the 64-bit modular arithmetic is timed. Each thread
// runs the three stages of a radix-8 group (12 butterflies, 7 twiddles) `rounds` times
// over values kept in [0, 4q); the grid fills every SM at full occupancy. KIND 1 times
// ct_butterfly_slack (the deferred-reduction stages of moduli below 2^60) and KIND 2
// ct_butterfly_wide (the no-subtraction form with estimated quotients, moduli below
// 2^57) instead; their values wrap modulo 2^64 over the rounds, which changes no
// instruction and so not the rate.
struct Twiddles7 {
    ulonglong2 w[7];
};

// KIND 0: ct_butterfly (Harvey); 1: ct_butterfly_slack; 2: ct_butterfly_wide
template <int KIND>
__device__ __forceinline__ void rate_butterfly(uint64_t &x, uint64_t &y, ulonglong2 w, uint64_t q, uint64_t q2) {
    if constexpr (KIND == 2) ct_butterfly_wide(x, y, w, q, q2 << 1);
    else if constexpr (KIND == 1) ct_butterfly_slack(x, y, w, q, q2);
    else ct_butterfly(x, y, w, q, q2);
}

template <int KIND>
__global__ void __launch_bounds__(256) butterfly_rate_kernel(uint64_t *sink, Twiddles7 tw, uint64_t q, int rounds) {
    const uint64_t q2 = q << 1;
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) v[k] = (tid * 8u + (uint32_t)k) % q;
    for (int r = 0; r < rounds; r++) {
#pragma unroll
        for (int k = 0; k < 4; k++) rate_butterfly<KIND>(v[k], v[k + 4], tw.w[0], q, q2);
#pragma unroll
        for (int k = 0; k < 8; k++)
            if (!(k & 2)) rate_butterfly<KIND>(v[k], v[k + 2], tw.w[1 + (k >> 2)], q, q2);
#pragma unroll
        for (int k = 0; k < 8; k += 2) rate_butterfly<KIND>(v[k], v[k + 1], tw.w[3 + (k >> 1)], q, q2);
    }
    uint64_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) x ^= v[k];
    sink[tid] = x;
}

int measure_butterfly_rate(uint64_t q, int kind, cudaStream_t s, double *rate) {
    if (!rate || q < 3 || !(q & 1) || q >= (1ull << 61))
        return set_error(TB_ERR_INVALID_ARGUMENT, "modulus must be odd, at least 3 and below 2^61");
    Twiddles7 tw;
    uint64_t z = 0x9e3779b97f4a7c15ull ^ q;
    for (int i = 0; i < 7; i++) {
        z = z * 6364136223846793005ull + 1442695040888963407ull;
        const uint64_t w = (z >> 3) % q;
        tw.w[i] = make_ulonglong2(w, (uint64_t)(((unsigned __int128)w << 64) / q));
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const auto kernel = kind == 2 ? butterfly_rate_kernel<2> : kind == 1 ? butterfly_rate_kernel<1> : butterfly_rate_kernel<0>;
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return status_from(e);
    const unsigned blocks = (unsigned)(sms * std::max(per_sm, 1));
    const int rounds = 2048;
    uint64_t *sink = nullptr;
    e = cudaMallocAsync(&sink, 8ull * blocks * 256, s);
    if (e != cudaSuccess) return status_from(e);
    int st = TB_OK;
    const float ms = time_call(
        [&] {
            kernel<<<blocks, 256, 0, s>>>(sink, tw, q, rounds);
            const cudaError_t le = cudaGetLastError();
            return le == cudaSuccess ? TB_OK : status_from(le);
        },
        s, 3, st);
    cudaFreeAsync(sink, s);
    if (st != TB_OK) return st;
    if (!(ms > 0)) return set_error(TB_ERR_CUDA, "no timing");
    *rate = (double)blocks * 256.0 * rounds * 12.0 / (ms * 1e-3);
    return TB_OK;
}

// The machine's 64-bit integer multiply throughput, the arithmetic a butterfly is made
// of (one high and two low 64 x 64-bit products per Shoup multiplication): 8 chains per
// thread, every SM at full occupancy, of mul.lo.u64 (kind 0) or mul.hi.u64 (kind 1),
// products per second. Each round multiplies every chain by its neighbour's previous
// value, so no product can be folded into another (a chain x = x * b would be
// reassociated by the compiler) and the 8 products of a round are independent.
template <int KIND>
__global__ void __launch_bounds__(256) mul64_rate_kernel(uint64_t *sink, uint64_t b, int rounds) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    uint64_t x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = b * (tid * 8u + (uint32_t)k + 1) | 1;
    for (int r = 0; r < rounds; r++) {
        uint64_t y[8];
#pragma unroll
        for (int k = 0; k < 8; k++) y[k] = x[k];
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if constexpr (KIND == 0) x[k] = y[k] * y[(k + 1) & 7];
            else x[k] = __umul64hi(y[k], y[(k + 1) & 7]) ^ y[k];
        }
    }
    uint64_t v = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) v ^= x[k];
    sink[tid] = v;
}

int measure_mul64_rate(int kind, cudaStream_t s, double *rate) {
    if (!rate || kind < 0 || kind > 1) return set_error(TB_ERR_INVALID_ARGUMENT, "kind is 0 (mul.lo.u64) or 1 (mul.hi.u64)");
    const auto kernel = kind ? mul64_rate_kernel<1> : mul64_rate_kernel<0>;
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return status_from(e);
    const unsigned blocks = (unsigned)(sms * std::max(per_sm, 1));
    const int rounds = 4096;
    uint64_t *sink = nullptr;
    e = cudaMallocAsync(&sink, 8ull * blocks * 256, s);
    if (e != cudaSuccess) return status_from(e);
    int st = TB_OK;
    const float ms = time_call(
        [&] {
            kernel<<<blocks, 256, 0, s>>>(sink, 0xd1b54a32d192ed03ull, rounds);
            const cudaError_t le = cudaGetLastError();
            return le == cudaSuccess ? TB_OK : status_from(le);
        },
        s, 3, st);
    cudaFreeAsync(sink, s);
    if (st != TB_OK) return st;
    if (!(ms > 0)) return set_error(TB_ERR_CUDA, "no timing");
    *rate = (double)blocks * 256.0 * rounds * 8.0 / (ms * 1e-3);
    return TB_OK;
}

}  // namespace tb

extern "C" {

int tb_measure_mul64_rate(int kind, void *stream, double *products_per_second) {
    return tb::measure_mul64_rate(kind, (cudaStream_t)stream, products_per_second);
}


int tb_measure_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second) {
    return tb::measure_butterfly_rate(modulus, 0, (cudaStream_t)stream, butterflies_per_second);
}

int tb_measure_slack_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second) {
    return tb::measure_butterfly_rate(modulus, 1, (cudaStream_t)stream, butterflies_per_second);
}

int tb_measure_wide_butterfly_rate(uint64_t modulus, void *stream, double *butterflies_per_second) {
    return tb::measure_butterfly_rate(modulus, 2, (cudaStream_t)stream, butterflies_per_second);
}

int tb_ntt_set_variant(int forward, int log_block, int variant) {
    if (log_block < 1 || log_block > tb::MAX_LOGB || variant < 0 || variant >= tb::NTT_VARIANTS ||
        (variant && log_block < 12))
        return tb::set_error(TB_ERR_INVALID_ARGUMENT, "no such NTT variant");
    tb::g_variant[forward ? 1 : 0][log_block].store(variant);
    return TB_OK;
}

int tb_ntt_get_variant(int forward, int log_block, int *variant) {
    if (!variant || log_block < 1 || log_block > tb::MAX_LOGB) return tb::set_error(TB_ERR_INVALID_ARGUMENT, "bad block");
    *variant = tb::ntt_variant(forward != 0, log_block);
    return TB_OK;
}

int tb_ntt_set_small_launch_pairs(int on) {
    tb::g_small_pairs.store(on != 0);
    return TB_OK;
}

int tb_keyswitch_set_budget(uint64_t bytes) {
    tb::g_ks_budget.store(bytes);
    return TB_OK;
}

uint64_t tb_keyswitch_get_budget(void) { return tb::ks_scratch_budget(); }

int tb_keyswitch_set_persistent(int on) {
    tb::g_ks_persistent.store(on ? 1 : 0);
    return TB_OK;
}

int tb_keyswitch_get_persistent(void) { return tb::ks_persistent() ? 1 : 0; }

}  // extern "C"

// Parameter context creation (host precompute uploaded once) and the plain
// batched NTT launchers.
#include <cstring>
#include <string>

#include "context.hpp"
#include "hostmath.hpp"
#include "trace.cuh"

namespace tb {

thread_local std::string g_last_error;

int set_error(int status, const std::string &msg) {
    g_last_error = msg;
    return status;
}

int status_from(cudaError_t e) {
    if (e == cudaSuccess) return TB_OK;
    if (e == cudaErrorMemoryAllocation) return set_error(TB_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
    return set_error(TB_ERR_CUDA, cudaGetErrorString(e));
}

Context::~Context() {
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    for (auto &kv : galois_ntt) cudaFree(kv.second);
    if (d_slot_map) cudaFree(d_slot_map);
    if (d_fft_roots) cudaFree(d_fft_roots);
    for (auto &lv : levels) {
        if (lv.d_consts) cudaFree(lv.d_consts);
        if (lv.d_bsk_mods) cudaFree(lv.d_bsk_mods);
        if (lv.d_bsk_idx) cudaFree(lv.d_bsk_idx);
    }
    if (d_drop) cudaFree(d_drop);
    if (d_mods) cudaFree(d_mods);
    if (d_tables) cudaFree(d_tables);
    cudaSetDevice(prev);
}

// NTT tables of one prime: forward roots psi^bitrev(i) and the scrambled inverse
// roots of NTTTables::initialize (src/utils/ntt.cpp:17-66).
static bool build_ntt_tables(uint64_t q, int logn, std::vector<ulonglong2> &fwd, std::vector<ulonglong2> &inv,
                             Mod &m) {
    using namespace host;
    const uint32_t n = 1u << logn;
    uint64_t root = minimal_root(2 * (uint64_t)n, q);
    if (!root) return false;
    uint64_t iroot = invmod(root, q);
    fwd.assign(n, make_ulonglong2(0, 0));
    inv.assign(n, make_ulonglong2(0, 0));
    uint64_t p = root;
    fwd[0] = make_ulonglong2(1, shoup(1, q));
    for (uint32_t i = 1; i < n; i++) {
        fwd[bitrev(i, logn)] = make_ulonglong2(p, shoup(p, q));
        p = mulmod(p, root, q);
    }
    p = iroot;
    inv[0] = make_ulonglong2(1, shoup(1, q));
    for (uint32_t i = 1; i < n; i++) {
        inv[bitrev(i - 1, logn) + 1] = make_ulonglong2(p, shoup(p, q));
        p = mulmod(p, iroot, q);
    }
    m.value = q;
    barrett_ratio(q, m.ratio_lo, m.ratio_hi);
    m.inv_n = invmod(n % q, q);
    m.inv_n_quo = shoup(m.inv_n, q);
    uint64_t last = inv[n - 1].x;
    m.sroot = mulmod(last, m.inv_n, q);
    m.sroot_quo = shoup(m.sroot, q);
    return true;
}

int build_rns_levels(Context &c);  // rns.cu
int noalloc_scratch_address(uint64_t **out);  // keyswitch.cu

int context_create(int scheme, uint64_t n, const uint64_t *moduli, int count, uint64_t t, Context **out) {
    using namespace host;
    *out = nullptr;
    if (scheme < SCHEME_RAW || scheme > SCHEME_BGV) return set_error(TB_ERR_INVALID_ARGUMENT, "unknown scheme");
    if (n < 2 || n > 131072 || (n & (n - 1))) return set_error(TB_ERR_INVALID_ARGUMENT, "poly degree must be a power of two in [2, 131072]");
    if (count < 1 || count > 64 || !moduli) return set_error(TB_ERR_INVALID_ARGUMENT, "between 1 and 64 coefficient moduli");
    for (int i = 0; i < count; i++) {
        uint64_t q = moduli[i];
        if (q < 3 || bit_count(q) > 61 || !is_prime(q))
            return set_error(TB_ERR_INVALID_ARGUMENT, "coefficient moduli must be primes of at most 61 bits");
        if ((q - 1) % (2 * n)) return set_error(TB_ERR_INVALID_ARGUMENT, "coefficient moduli must be 1 mod 2N");
    }
    if ((scheme == SCHEME_BFV || scheme == SCHEME_BGV) && (t < 2 || bit_count(t) > 60))
        return set_error(TB_ERR_INVALID_ARGUMENT, "plain modulus must have 2 to 60 bits");
    auto *c = new Context();
    cudaGetDevice(&c->device);
    c->scheme = scheme;
    c->n = (uint32_t)n;
    while ((1u << c->logn) < n) c->logn++;
    c->chain.assign(moduli, moduli + count);
    c->t = (scheme == SCHEME_BFV || scheme == SCHEME_BGV) ? t : 0;
    c->table_moduli = c->chain;
    if (c->t && is_prime(c->t) && (c->t - 1) % (2 * n) == 0) {
        c->plain_index = (int)c->table_moduli.size();
        c->table_moduli.push_back(c->t);
    }
    if (scheme == SCHEME_BFV || scheme == SCHEME_BGV) {
        // Bsk primes of every level's RNS tool are prefixes of one list
        // getPrimes(2N, 61, .) = [m_sk, gamma, B_0, B_1, ...] (src/utils/rns.cpp:627-635).
        std::vector<uint64_t> extra;
        if (!get_primes(2 * n, 61, (size_t)count + 3, extra)) {
            delete c;
            return set_error(TB_ERR_UNSUPPORTED, "not enough 61-bit NTT primes for the Bsk base");
        }
        for (auto p : extra) c->table_moduli.push_back(p);
    }
    const size_t nm = c->table_moduli.size();
    std::vector<ulonglong2> all(2 * nm * n);
    c->h_mods.resize(nm);
    for (size_t i = 0; i < nm; i++) {
        std::vector<ulonglong2> f, v;
        if (!build_ntt_tables(c->table_moduli[i], c->logn, f, v, c->h_mods[i])) {
            delete c;
            return set_error(TB_ERR_INVALID_ARGUMENT, "modulus has no primitive 2N-th root of unity");
        }
        std::memcpy(&all[(2 * i) * n], f.data(), n * sizeof(ulonglong2));
        std::memcpy(&all[(2 * i + 1) * n], v.data(), n * sizeof(ulonglong2));
    }
    cudaError_t e = cudaMalloc(&c->d_tables, all.size() * sizeof(ulonglong2));
    if (e == cudaSuccess) e = cudaMemcpy(c->d_tables, all.data(), all.size() * sizeof(ulonglong2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete c;
        return status_from(e);
    }
    for (size_t i = 0; i < nm; i++) {
        c->h_mods[i].roots = c->d_tables + (2 * i) * n;
        c->h_mods[i].inv_roots = c->d_tables + (2 * i + 1) * n;
    }
    e = cudaMalloc(&c->d_mods, nm * sizeof(Mod));
    if (e == cudaSuccess) e = cudaMemcpy(c->d_mods, c->h_mods.data(), nm * sizeof(Mod), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        delete c;
        return status_from(e);
    }
    int st = build_rns_levels(*c);
    if (st == TB_OK) st = noalloc_scratch_address(&c->noalloc_scratch);
    if (st != TB_OK) {
        delete c;
        return st;
    }
    *out = c;
    return TB_OK;
}

// ------------------------------------------------------------ plain NTT

// [polys][limbs][n] in -> out; a CTA owns one limb, or one 2^LOGB sub-block of it.
template <bool FWD>
struct PlainNttOp {
    const uint64_t *in;
    uint64_t *out;
    const Mod *mods;
    int first, limbs, lazy;
    int log_nsub;   // log2(sub-blocks per limb)
    int logb;       // log2(sub-block length)
    struct Ctx {
        NttLimb lm;
        const uint64_t *in;
        uint64_t *out;
        int slack;    // full forward outputs: deferred reductions, outputs below 16 q
        int islack;   // full inverse outputs: the wide inverse form, outputs below 4q
    };
    __device__ Ctx ctx(int b) const {
        const int limb_block = b >> log_nsub;
        const uint32_t sb = (uint32_t)(b & ((1 << log_nsub) - 1));
        const int l = limb_block % limbs;
        Ctx c;
        c.lm = make_limb(mods[first + l], sb);
        c.slack = (FWD && !lazy && c.lm.q < (1ull << 60)) ? SLACK_M : 0;
        c.islack = !FWD && !lazy;
        const size_t off = ((size_t)limb_block << (logb + log_nsub)) + ((size_t)sb << logb);
        c.in = in + off;
        c.out = out + off;
        return c;
    }
    __device__ uint64_t load(const Ctx &c, int e) const { return c.in[e]; }
    __device__ void load2(const Ctx &c, int e, uint64_t &a, uint64_t &b) const {
        const ulonglong2 v = *reinterpret_cast<const ulonglong2 *>(c.in + e);
        a = v.x;
        b = v.y;
    }
    __device__ uint64_t fix(const Ctx &c, uint64_t v) const {
        if (lazy) return v;
        const uint64_t q = c.lm.q;
        if (FWD && c.slack) v = csub(csub(v, 8 * q), 4 * q);
        return csub(csub(v, 2 * q), q);
    }
    __device__ void store(const Ctx &c, int e, uint64_t v) const { c.out[e] = fix(c, v); }
    __device__ void store2(const Ctx &c, int e, uint64_t a, uint64_t b) const {
        *reinterpret_cast<ulonglong2 *>(c.out + e) = make_ulonglong2(fix(c, a), fix(c, b));
    }
};

// Top stages of a limb longer than one CTA's block, in place over global memory.
// Forward: the first H_LOG Cooley-Tukey stages; inverse: the last H_LOG
// Gentleman-Sande stages including the N^-1 scaling.
template <int H_LOG, bool FWD>
__global__ void ntt_top_kernel(uint64_t *data, const Mod *mods, int first, int limbs, int logn, int lazy_out) {
    constexpr int H = 1 << H_LOG;
    const uint32_t n = 1u << logn;
    const uint32_t sub = n >> H_LOG;
    const size_t limb = blockIdx.y;
    const Mod m = mods[first + (int)(limb % limbs)];
    const uint64_t q = m.value, q2 = q << 1;
    uint64_t *p = data + limb * n;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < sub; j += gridDim.x * blockDim.x) {
        uint64_t v[H];
#pragma unroll
        for (int k = 0; k < H; k++) v[k] = p[j + k * sub];
        if (FWD) {
#pragma unroll
            for (int t = 0; t < H_LOG; t++) {
                const int half = H >> (t + 1);
#pragma unroll
                for (int k = 0; k < H; k++) {
                    if (k & half) continue;
                    const uint32_t ri = (1u << t) + (uint32_t)(k >> (H_LOG - t));
                    ct_butterfly(v[k], v[k + half], __ldg(&m.roots[ri]), q, q2);
                }
            }
        } else {
            // global stages logn-H_LOG .. logn-1; gap = sub << t
#pragma unroll
            for (int t = 0; t < H_LOG; t++) {
                const int h = 1 << t;
                const int sg = logn - H_LOG + t;
#pragma unroll
                for (int k = 0; k < H; k++) {
                    if (k & h) continue;
                    if (t == H_LOG - 1) {
                        uint64_t u = v[k] >= q2 ? v[k] - q2 : v[k];
                        uint64_t y = v[k + h];
                        uint64_t s = u + y;
                        s = s >= q2 ? s - q2 : s;
                        v[k] = mul_shoup_lazy(s, m.inv_n, m.inv_n_quo, q);
                        v[k + h] = mul_shoup_lazy(u + q2 - y, m.sroot, m.sroot_quo, q);
                    } else {
                        const uint32_t ri = n + 1 - (n >> sg) + (uint32_t)(k >> (t + 1));
                        gs_butterfly(v[k], v[k + h], __ldg(&m.inv_roots[ri]), q, q2);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < H; k++) {
            uint64_t x = v[k];
            if (!lazy_out) {
                if (FWD) x = x >= q2 ? x - q2 : x;
                x = x >= q ? x - q : x;
            }
            p[j + k * sub] = x;
        }
    }
}

template <bool FWD>
static int ntt_plain(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs,
                     bool lazy, cudaStream_t s) {
    if (limbs < 1 || first < 0 || first + limbs > (int)c.table_moduli.size())
        return set_error(TB_ERR_INVALID_ARGUMENT, "modulus range outside the context");
    if (!in || !out) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (polys == 0) return TB_OK;
    const uint64_t total = polys * (uint64_t)limbs;
    const int logn = c.logn;
    // limbs up to 2^14 in one launch, and 2^15 inverse transforms on two-CTA clusters;
    // longer limbs (and 2^15 forward transforms, measured faster so) split into global
    // top stages and 2^14 sub-blocks
    const int logb = (logn <= MAX_LOGB || (!FWD && logn == PAIR_LOGN)) ? logn : MAX_LOGB;
    const int h = logn - logb;
    if ((total << h) > 0x7fffffffULL || (h > 0 && total > 65535))
        return set_error(TB_ERR_INVALID_ARGUMENT, "too many limbs in one launch");
    PlainNttOp<FWD> op;
    op.mods = c.d_mods;
    op.first = first;
    op.limbs = limbs;
    op.log_nsub = h;
    op.logb = logb;
    cudaError_t e = cudaSuccess;
    if (FWD) {
        op.in = in;
        op.out = out;
        op.lazy = lazy;
        if (h > 0) {
            if (in != out) {
                e = cudaMemcpyAsync(out, in, total * c.n * 8, cudaMemcpyDeviceToDevice, s);
                if (e != cudaSuccess) return status_from(e);
            }
            dim3 grid(std::max(1u, (c.n >> h) / 256), (unsigned)total);
            if (h == 1) ntt_top_kernel<1, true><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, 1);
            else if (h == 2) ntt_top_kernel<2, true><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, 1);
            else ntt_top_kernel<3, true><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, 1);
            op.in = out;
        }
        TraceScope ts("ntt_forward", s);
        e = dispatch_ntt<true>(logb, op, (unsigned)(total << h), h, 0, s);
    } else {
        TraceScope ts("ntt_inverse", s);
        op.in = in;
        op.out = out;
        op.lazy = h > 0 ? 1 : lazy;
        e = dispatch_ntt<false>(logb, op, (unsigned)(total << h), logn, h == 0, s);
        if (e == cudaSuccess && h > 0) {
            dim3 grid(std::max(1u, (c.n >> h) / 256), (unsigned)total);
            if (h == 1) ntt_top_kernel<1, false><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, lazy);
            else if (h == 2) ntt_top_kernel<2, false><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, lazy);
            else ntt_top_kernel<3, false><<<grid, 256, 0, s>>>(out, c.d_mods, first, limbs, logn, lazy);
            e = cudaGetLastError();
        }
    }
    return e == cudaSuccess ? TB_OK : status_from(e);
}

int ntt_forward(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s) {
    return ntt_plain<true>(c, in, out, polys, first, limbs, lazy, s);
}

int ntt_inverse(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s) {
    return ntt_plain<false>(c, in, out, polys, first, limbs, lazy, s);
}

}  // namespace tb

// ------------------------------------------------------------------ tracing

#include <map>
#include <mutex>
#include <tuple>

#include "trace.cuh"

namespace tb {

std::atomic<bool> g_trace_on{false};
static std::mutex g_trace_mu;
static std::vector<std::tuple<const char *, cudaEvent_t, cudaEvent_t>> g_trace;

void trace_record(const char *name, cudaEvent_t a, cudaEvent_t b) {
    std::lock_guard<std::mutex> g(g_trace_mu);
    g_trace.emplace_back(name, a, b);
}

static void trace_clear_locked() {
    for (auto &r : g_trace) {
        cudaEventDestroy(std::get<1>(r));
        cudaEventDestroy(std::get<2>(r));
    }
    g_trace.clear();
}

void trace_enable(bool on) {
    std::lock_guard<std::mutex> g(g_trace_mu);
    trace_clear_locked();
    g_trace_on.store(on);
}

// name -> (launches, total ms); waits for the recorded events.
int trace_collect(std::map<std::string, std::pair<uint64_t, double>> &out) {
    std::lock_guard<std::mutex> g(g_trace_mu);
    for (auto &r : g_trace) {
        cudaError_t e = cudaEventSynchronize(std::get<2>(r));
        if (e != cudaSuccess) return status_from(e);
        float ms = 0;
        cudaEventElapsedTime(&ms, std::get<1>(r), std::get<2>(r));
        auto &v = out[std::get<0>(r)];
        v.first++;
        v.second += ms;
    }
    trace_clear_locked();
    return TB_OK;
}

}  // namespace tb

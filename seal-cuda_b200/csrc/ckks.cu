// CKKS encoding and decoding (CKKSEncoder, src/ckks.cpp:32-579) on the device.
//
// Encode: slots -> conjugate-symmetric vector in bit-reversed index order ->
// inverse special FFT (Gentleman-Sande, scaled by scale/N in its last stage) ->
// round the real parts -> reduce into every prime -> NTT. Decode: inverse NTT ->
// CRT compose -> centre and scale to doubles -> forward special FFT -> slots.
// FP64 is used only here. The FFT butterflies follow the reference's DWTHandler
// order with complex products computed as (ac - bd, ad + bc) from individually
// rounded IEEE operations (no fused multiply-add), and the root tables are
// built on the host exactly like ComplexRoots (src/utils/croots.cpp:10-59).
#include <cmath>
#include <complex>
#include <functional>
#include <mutex>
#include <vector>

#include "context.hpp"
#include "hostmath.hpp"
#include "trace.cuh"

namespace tb {

unsigned grid_for(uint64_t work, int threads);
void ensure_pool_retains(int device);
int slot_map(Context &c, const uint32_t **out);
int ntt_forward(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s);
int ntt_inverse(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs, bool lazy,
                cudaStream_t s);

namespace {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(__dadd_rn(a.x, b.x), __dadd_rn(a.y, b.y)); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(__dsub_rn(a.x, b.x), __dsub_rn(a.y, b.y)); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(__dsub_rn(__dmul_rn(a.x, b.x), __dmul_rn(a.y, b.y)),
                        __dadd_rn(__dmul_rn(a.x, b.y), __dmul_rn(a.y, b.x)));
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(__dmul_rn(a.x, s), __dmul_rn(a.y, s)); }

// One Gentleman-Sande stage (gap = 2^s) of transformFromRev over B vectors; the
// last stage (m == 1) multiplies by `scalar`.
__global__ void fft_inv_stage(double2 *__restrict__ a, const double2 *__restrict__ iroots, int logn, int s,
                              double scalar, uint64_t B) {
    const uint32_t n = 1u << logn, half = n >> 1;
    const uint64_t total = B * half;
    const uint32_t gap = 1u << s;
    const uint32_t m = n >> (s + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / half;
        const uint32_t k = (uint32_t)(w - b * half);
        const uint32_t i = k >> s, j = k & (gap - 1);
        double2 *x = a + b * n + 2 * i * gap + j, *y = x + gap;
        const uint32_t ri = n - 2 * m + 1 + i;
        const double2 r = iroots[ri];
        const double2 u = *x, v = *y;
        if (m > 1) {
            *x = cadd(u, v);
            *y = cmul(csub(u, v), r);
        } else {
            const double2 sr = cscale(r, scalar);
            *x = cscale(cadd(u, v), scalar);
            *y = cmul(csub(u, v), sr);
        }
    }
}

// One Cooley-Tukey stage (m = 2^s groups) of transformToRev.
__global__ void fft_fwd_stage(double2 *__restrict__ a, const double2 *__restrict__ roots, int logn, int s, uint64_t B) {
    const uint32_t n = 1u << logn, half = n >> 1;
    const uint64_t total = B * half;
    const uint32_t m = 1u << s, gap = n >> (s + 1);
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / half;
        const uint32_t k = (uint32_t)(w - b * half);
        const uint32_t i = k / gap, j = k - i * gap;
        double2 *x = a + b * n + 2 * i * gap + j, *y = x + gap;
        const double2 r = roots[m + i];
        const double2 u = *x, v = cmul(*y, r);
        *x = cadd(u, v);
        *y = csub(u, v);
    }
}

// conj[map[i]] = v_i, conj[map[i + n/2]] = conj(v_i) for i < count; zero elsewhere.
__global__ void ckks_scatter(const double2 *__restrict__ vals, uint64_t vstride, uint32_t count,
                             double2 *__restrict__ out, const uint32_t *__restrict__ map, int logn, uint64_t B) {
    const uint32_t n = 1u << logn, slots = n >> 1;
    const uint64_t total = B * slots;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / slots;
        const uint32_t i = (uint32_t)(w - b * slots);
        double2 v = make_double2(0.0, 0.0);
        if (i < count) v = vals[b * vstride + i];
        out[b * n + map[i]] = v;
        out[b * n + map[i + slots]] = make_double2(v.x, -v.y);
    }
}

// Round the real parts and reduce into primes 0..L-1 (src/ckks.cpp:158-230); flags
// coefficients of 128 bits or more.
__global__ void ckks_round_reduce(const double2 *__restrict__ a, uint64_t *__restrict__ out,
                                  const Mod *__restrict__ mods, int L, int logn, uint64_t B, int *__restrict__ err,
                                  int total_bits) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    const double two64 = 18446744073709551616.0;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        const uint32_t i = (uint32_t)(w & (n - 1));
        const double mag = fabs(a[w].x);
        // max_coeff_bit_count = ceil(log2(max(|x|, 1))) + 1 must stay below the modulus bits
        if ((mag > 1.0 ? (int)ceil(log2(mag)) : 0) + 1 >= total_bits) atomicOr(err, 1);
        double c = round(a[w].x);
        const bool neg = signbit(c);
        c = fabs(c);
        if (!(c < 170141183460469231731687303715884105728.0)) {  // 2^127
            atomicOr(err, 1);
            c = 0.0;
        }
        const uint64_t lo = (uint64_t)fmod(c, two64), hi = (uint64_t)(c / two64);
        for (int l = 0; l < L; l++) {
            const Mod m = mods[l];
            uint64_t r = reduce128(hi, lo, m);
            if (neg) r = neg_mod(r, m.value);
            out[((b * L + l) << logn) + i] = r;
        }
    }
}

// CRT compose, centre and scale (src/ckks.cpp:520-563): per coefficient the
// multi-word x = sum_j [c_j (Q/q_j)^-1]_{q_j} (Q/q_j) mod Q, then the word-wise
// signed sum scaled by inv_scale * 2^(64 j).
constexpr int MAXW = 34;
__global__ void ckks_compose(const uint64_t *__restrict__ coeff, double2 *__restrict__ out,
                             const Mod *__restrict__ mods, const uint64_t *__restrict__ ip,
                             const uint64_t *__restrict__ punct, const uint64_t *__restrict__ Qw,
                             const uint64_t *__restrict__ thr, int L, int logn, double inv_scale, uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        const uint32_t i = (uint32_t)(w & (n - 1));
        uint64_t x[MAXW];
        for (int k = 0; k <= L; k++) x[k] = 0;
        for (int j = 0; j < L; j++) {
            const uint64_t q = mods[j].value;
            const uint64_t t = mul_shoup(coeff[((b * L + j) << logn) + i], ip[2 * j], ip[2 * j + 1], q);
            // x += t * punct_j (L words)
            uint64_t carry = 0;
            for (int k = 0; k < L; k++) {
                const uint64_t pk = punct[j * L + k];
                const uint64_t lo = t * pk, hi = mulhi(t, pk);
                uint64_t s = x[k] + lo;
                uint64_t c1 = s < lo;
                s += carry;
                c1 += s < carry;
                x[k] = s;
                carry = hi + c1;
            }
            x[L] += carry;
        }
        // reduce mod Q: x < L Q, subtract Q while x >= Q
        for (int rep = 0; rep < L + 1; rep++) {
            bool ge = x[L] != 0;
            if (!ge) {
                ge = true;
                for (int k = L - 1; k >= 0; k--) {
                    if (x[k] != Qw[k]) {
                        ge = x[k] > Qw[k];
                        break;
                    }
                }
            }
            if (!ge) break;
            uint64_t borrow = 0;
            for (int k = 0; k < L; k++) {
                const uint64_t d = x[k] - Qw[k] - borrow;
                borrow = (x[k] < Qw[k]) || (x[k] - Qw[k] < borrow);
                x[k] = d;
            }
            x[L] -= borrow;
        }
        // compare with the upper-half threshold (Q + 1) / 2
        bool upper = true;
        for (int k = L - 1; k >= 0; k--) {
            if (x[k] != thr[k]) {
                upper = x[k] > thr[k];
                break;
            }
        }
        double res = 0.0, sc = inv_scale;
        const double two64 = 18446744073709551616.0;
        for (int k = 0; k < L; k++) {
            if (upper) {
                if (x[k] > Qw[k]) {
                    const uint64_t d = x[k] - Qw[k];
                    res = __dadd_rn(res, d ? __dmul_rn((double)d, sc) : 0.0);
                } else {
                    const uint64_t d = Qw[k] - x[k];
                    res = __dsub_rn(res, d ? __dmul_rn((double)d, sc) : 0.0);
                }
            } else {
                res = __dadd_rn(res, x[k] ? __dmul_rn((double)x[k], sc) : 0.0);
            }
            sc = __dmul_rn(sc, two64);
        }
        out[w] = make_double2(res, 0.0);
    }
}

__global__ void ckks_gather(const double2 *__restrict__ a, double2 *__restrict__ out, uint64_t ostride,
                            const uint32_t *__restrict__ map, int logn, uint64_t B) {
    const uint32_t n = 1u << logn, slots = n >> 1;
    const uint64_t total = B * slots;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w / slots;
        const uint32_t i = (uint32_t)(w - b * slots);
        out[b * ostride + i] = a[b * n + map[i]];
    }
}

// a[b][i] = (v[b][i] * scale, 0) for i < count, 0 elsewhere (coefficient encode).
__global__ void ckks_load_real(const double *__restrict__ vals, uint64_t vstride, uint32_t count, double scale,
                               double2 *__restrict__ out, int logn, uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        const uint32_t i = (uint32_t)(w & (n - 1));
        out[w] = make_double2(i < count ? __dmul_rn(vals[b * vstride + i], scale) : 0.0, 0.0);
    }
}

__global__ void ckks_store_real(const double2 *__restrict__ a, double *__restrict__ out, uint64_t ostride, int logn,
                                uint64_t B) {
    const uint32_t n = 1u << logn;
    const uint64_t total = B << logn;
    for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < total; w += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = w >> logn;
        out[b * ostride + (w & (n - 1))] = a[w].x;
    }
}

}  // namespace

// Complex root tables of the special FFT (CKKSEncoder constructor, src/ckks.cpp:62-77).
static std::mutex g_ckks_mu;

static int ckks_tables(Context &c, double2 **roots, double2 **iroots) {
    std::lock_guard<std::mutex> g(g_ckks_mu);
    if (!c.d_fft_roots) {
        const uint32_t n = c.n;
        const uint64_t m = 2ull * n;
        const double PI = 3.1415926535897932384626433832795028842;
        std::vector<std::complex<double>> base(m / 8 + 1);
        for (size_t i = 0; i <= m / 8; i++) base[i] = std::polar<double>(1.0, 2 * PI * (double)i / (double)m);
        std::function<std::complex<double>(uint64_t)> get = [&](uint64_t idx) -> std::complex<double> {
            idx &= m - 1;
            if (idx <= m / 8) return base[idx];
            if (idx <= m / 4) {
                auto a = base[m / 4 - idx];
                return {a.imag(), a.real()};
            }
            if (idx <= m / 2) return -std::conj(get(m / 2 - idx));
            if (idx <= 3 * m / 4) return -get(idx - m / 2);
            return std::conj(get(m - idx));
        };
        std::vector<double2> r(n, make_double2(0, 0)), ir(n, make_double2(0, 0));
        if (m >= 8) {
            for (uint32_t i = 1; i < n; i++) {
                auto a = get(host::bitrev(i, c.logn));
                auto b = std::conj(get(host::bitrev(i - 1, c.logn) + 1));
                r[i] = make_double2(a.real(), a.imag());
                ir[i] = make_double2(b.real(), b.imag());
            }
        } else if (m == 4) {
            r[1] = make_double2(0, 1);
            ir[1] = make_double2(0, -1);
        }
        double2 *d = nullptr;
        cudaError_t e = cudaMalloc(&d, 2ull * n * sizeof(double2));
        if (e == cudaSuccess) e = cudaMemcpy(d, r.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(d + n, ir.data(), n * sizeof(double2), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) return status_from(e);
        c.d_fft_roots = d;
    }
    *roots = (double2 *)c.d_fft_roots;
    *iroots = (double2 *)c.d_fft_roots + c.n;
    return TB_OK;
}

static int total_bits(const Context &c, int L) {
    return host::bit_count(host::product(c.chain.data(), L));
}

// Rounds the real parts of buf [B][N] into plaintexts [B][L][N] and transforms them;
// fails with "encoded values are too large" when a coefficient reaches the modulus.
static int round_reduce_ntt(Context &c, int L, double2 *buf, uint64_t *out, uint64_t B, cudaStream_t s) {
    int *err = nullptr;
    cudaError_t e = cudaMallocAsync(&err, sizeof(int), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return status_from(e);
    ckks_round_reduce<<<grid_for(B * c.n, 256), 256, 0, s>>>(buf, out, c.d_mods, L, c.logn, B, err, total_bits(c, L));
    int herr = 0;
    e = cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s);
    cudaFreeAsync(err, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return status_from(e);
    if (herr) return set_error(TB_ERR_INVALID_ARGUMENT, "encoded values are too large");
    return ntt_forward(c, out, out, B, 0, L, false, s);
}

// values [B][vstride] complex (count used) -> plaintexts [B][L][N], NTT form.
int ckks_encode(Context &c, int L, const double *values, uint64_t vstride, uint32_t count, double scale, uint64_t *out,
                uint64_t B, cudaStream_t s) {
    if (c.scheme != SCHEME_CKKS) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    const uint32_t n = c.n;
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (count > n / 2) return set_error(TB_ERR_INVALID_ARGUMENT, "values_size is too large");
    if (!(scale > 0) || (int)std::log2(scale) + 1 >= total_bits(c, L))
        return set_error(TB_ERR_INVALID_ARGUMENT, "scale out of bounds");
    if (!out || (count && !values)) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!vstride) vstride = count;
    const uint32_t *map = nullptr;
    double2 *roots, *iroots;
    int r = slot_map(c, &map);
    if (r == TB_OK) r = ckks_tables(c, &roots, &iroots);
    if (r != TB_OK) return r;
    ensure_pool_retains(c.device);
    double2 *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, B * n * sizeof(double2), s);
    if (e != cudaSuccess) return status_from(e);
    {
        TraceScope ts("ckks_encode", s);
        ckks_scatter<<<grid_for(B * n / 2, 256), 256, 0, s>>>((const double2 *)values, vstride, count, buf, map,
                                                              c.logn, B);
        for (int st = 0; st < c.logn; st++)
            fft_inv_stage<<<grid_for(B * n / 2, 256), 256, 0, s>>>(buf, iroots, c.logn, st, scale / (double)n, B);
    }
    r = round_reduce_ntt(c, L, buf, out, B, s);
    cudaFreeAsync(buf, s);
    return r;
}

// Real coefficients [B][vstride] (count <= N used) times scale, rounded, reduced and
// transformed: CKKSEncoderCuda::encodePolynomialInternal (src/ckks_cuda.cu:455-565).
int ckks_encode_polynomial(Context &c, int L, const double *values, uint64_t vstride, uint32_t count, double scale,
                           uint64_t *out, uint64_t B, cudaStream_t s) {
    if (c.scheme != SCHEME_CKKS) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    if (count > c.n) return set_error(TB_ERR_INVALID_ARGUMENT, "values_size is too large");
    if (!out || (count && !values)) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    if (!B) return TB_OK;
    if (!vstride) vstride = count;
    ensure_pool_retains(c.device);
    double2 *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, B * c.n * sizeof(double2), s);
    if (e != cudaSuccess) return status_from(e);
    {
        TraceScope ts("ckks_encode", s);
        ckks_load_real<<<grid_for(B * c.n, 256), 256, 0, s>>>(values, vstride, count, scale, buf, c.logn, B);
    }
    const int r = round_reduce_ntt(c, L, buf, out, B, s);
    cudaFreeAsync(buf, s);
    return r;
}

int fill_limbs(Context &c, int L, const uint64_t *vals, uint64_t *out, uint64_t B, cudaStream_t s);

// |x| mod q for a non-negative integral double x, through its base-2^64 digits.
static uint64_t double_mod(double x, uint64_t q) {
    const double two64 = 18446744073709551616.0;
    std::vector<uint64_t> words;
    while (x >= 1) {
        words.push_back((uint64_t)std::fmod(x, two64));
        x /= two64;
    }
    unsigned __int128 r = 0;
    for (size_t k = words.size(); k-- > 0;) r = ((r << 64) | words[k]) % q;
    return (uint64_t)r;
}

// The constant round(value * scale) in every slot: every NTT coefficient of limb l
// equals the constant mod q_l (CKKSEncoder::encodeInternal(double), src/ckks.cpp:279-400).
int ckks_encode_double(Context &c, int L, double value, double scale, uint64_t *out, cudaStream_t s) {
    if (c.scheme != SCHEME_CKKS) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    const int bits = total_bits(c, L);
    if (!(scale > 0) || (int)std::log2(scale) >= bits) return set_error(TB_ERR_INVALID_ARGUMENT, "scale out of bounds");
    value *= scale;
    if (value != 0.0 && (int)std::log2(std::fabs(value)) + 2 >= bits)
        return set_error(TB_ERR_INVALID_ARGUMENT, "encoded value is too large");
    double cd = std::round(value);
    const bool neg = std::signbit(cd);
    cd = std::fabs(cd);
    std::vector<uint64_t> vals(L);
    for (int l = 0; l < L; l++) {
        const uint64_t q = c.chain[l];
        const uint64_t r = double_mod(cd, q);
        vals[l] = (neg && r) ? q - r : r;
    }
    TraceScope ts("ckks_encode", s);
    return fill_limbs(c, L, vals.data(), out, 1, s);
}

// The integer `value` in every slot, scale 1 (CKKSEncoder::encodeInternal(int64_t),
// src/ckks.cpp:402-440): residue ((uint64)value + q) mod q for negative values.
int ckks_encode_int64(Context &c, int L, int64_t value, uint64_t *out, cudaStream_t s) {
    if (c.scheme != SCHEME_CKKS) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (L < 1 || L > (int)c.chain.size()) return set_error(TB_ERR_INVALID_ARGUMENT, "level outside the chain");
    const uint64_t mag = value < 0 ? 0 - (uint64_t)value : (uint64_t)value;
    if (host::bit_count(mag) + 2 >= total_bits(c, L))
        return set_error(TB_ERR_INVALID_ARGUMENT, "encoded value is too large");
    std::vector<uint64_t> vals(L);
    for (int l = 0; l < L; l++) {
        const uint64_t q = c.chain[l];
        const uint64_t fill = value < 0 ? (uint64_t)value + q : (uint64_t)value;
        vals[l] = fill % q;
    }
    TraceScope ts("ckks_encode", s);
    return fill_limbs(c, L, vals.data(), out, 1, s);
}

// Inverse NTT, CRT compose, centre and scale by 1/scale: buf [B][N] (real parts).
static int compose_level(Context &c, int L, const uint64_t *plain, double scale, double2 *buf, uint64_t B,
                         cudaStream_t s) {
    using namespace host;
    const uint32_t n = c.n;
    const uint64_t *q = c.chain.data();
    auto Q = product(q, L);
    Q.resize(L, 0);
    std::vector<uint64_t> hc(2 * L + L * L + L + L);
    for (int j = 0; j < L; j++) {
        const uint64_t ipj = invmod(punctured_mod(q, L, j, q[j]), q[j]);
        hc[2 * j] = ipj;
        hc[2 * j + 1] = shoup(ipj, q[j]);
        uint64_t rem = 0;
        auto pj = div_words(Q, q[j], rem);
        pj.resize(L, 0);
        for (int k = 0; k < L; k++) hc[2 * L + j * L + k] = pj[k];
    }
    for (int k = 0; k < L; k++) hc[2 * L + L * L + k] = Q[k];
    // threshold (Q + 1) / 2
    {
        std::vector<uint64_t> t(Q);
        int k = 0;
        while (k < L && ++t[k] == 0) k++;
        uint64_t carry = 0;
        for (int i = L - 1; i >= 0; i--) {
            const uint64_t v = t[i];
            t[i] = (v >> 1) | (carry << 63);
            carry = v & 1;
        }
        for (int i = 0; i < L; i++) hc[2 * L + L * L + L + i] = t[i];
    }
    ensure_pool_retains(c.device);
    uint64_t *tmp = nullptr, *dc = nullptr;
    cudaError_t e = cudaMallocAsync(&tmp, 8ull * B * L * n, s);
    if (e == cudaSuccess) e = cudaMallocAsync(&dc, hc.size() * 8, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dc, hc.data(), hc.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(tmp, plain, 8ull * B * L * n, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // hc is a host vector
    if (e != cudaSuccess) return status_from(e);
    int r = ntt_inverse(c, tmp, tmp, B, 0, L, false, s);
    if (r == TB_OK) {
        TraceScope ts("ckks_decode", s);
        ckks_compose<<<grid_for(B * n, 128), 128, 0, s>>>(tmp, buf, c.d_mods, dc, dc + 2 * L, dc + 2 * L + L * L,
                                                          dc + 2 * L + L * L + L, L, c.logn, 1.0 / scale, B);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = status_from(e);
    }
    cudaFreeAsync(tmp, s);
    cudaFreeAsync(dc, s);
    return r;
}

static int decode_checks(const Context &c, int L, const uint64_t *plain, double scale, const double *values) {
    if (c.scheme != SCHEME_CKKS) return set_error(TB_ERR_UNSUPPORTED, "unsupported scheme");
    if (L < 1 || L > (int)c.chain.size() || L + 1 > MAXW) return set_error(TB_ERR_INVALID_ARGUMENT, "bad level");
    if (!(scale > 0) || (int)std::log2(scale) >= total_bits(c, L))
        return set_error(TB_ERR_INVALID_ARGUMENT, "scale out of bounds");
    if (!plain || !values) return set_error(TB_ERR_INVALID_ARGUMENT, "null buffer");
    return TB_OK;
}

// plaintexts [B][L][N] (NTT form) -> slot values [B][ostride] complex (N/2 used).
int ckks_decode(Context &c, int L, const uint64_t *plain, double scale, double *values, uint64_t ostride, uint64_t B,
                cudaStream_t s) {
    int r = decode_checks(c, L, plain, scale, values);
    if (r != TB_OK || !B) return r;
    const uint32_t n = c.n;
    if (!ostride) ostride = n / 2;
    const uint32_t *map = nullptr;
    double2 *roots, *iroots;
    r = slot_map(c, &map);
    if (r == TB_OK) r = ckks_tables(c, &roots, &iroots);
    if (r != TB_OK) return r;
    ensure_pool_retains(c.device);
    double2 *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, B * n * sizeof(double2), s);
    if (e != cudaSuccess) return status_from(e);
    r = compose_level(c, L, plain, scale, buf, B, s);
    if (r == TB_OK) {
        TraceScope ts("ckks_decode", s);
        for (int st = 0; st < c.logn; st++)
            fft_fwd_stage<<<grid_for(B * n / 2, 256), 256, 0, s>>>(buf, roots, c.logn, st, B);
        ckks_gather<<<grid_for(B * n / 2, 256), 256, 0, s>>>(buf, (double2 *)values, ostride, map, c.logn, B);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = status_from(e);
    }
    cudaFreeAsync(buf, s);
    return r;
}

// plaintexts [B][L][N] (NTT form) -> N real coefficients each, divided by scale
// (CKKSEncoderCuda::decodePolynomialInternal, src/ckks_cuda.cu:983-1040).
int ckks_decode_polynomial(Context &c, int L, const uint64_t *plain, double scale, double *values, uint64_t ostride,
                           uint64_t B, cudaStream_t s) {
    int r = decode_checks(c, L, plain, scale, values);
    if (r != TB_OK || !B) return r;
    const uint32_t n = c.n;
    if (!ostride) ostride = n;
    ensure_pool_retains(c.device);
    double2 *buf = nullptr;
    cudaError_t e = cudaMallocAsync(&buf, B * n * sizeof(double2), s);
    if (e != cudaSuccess) return status_from(e);
    r = compose_level(c, L, plain, scale, buf, B, s);
    if (r == TB_OK) {
        ckks_store_real<<<grid_for(B * n, 256), 256, 0, s>>>(buf, values, ostride, c.logn, B);
        e = cudaGetLastError();
        if (e != cudaSuccess) r = status_from(e);
    }
    cudaFreeAsync(buf, s);
    return r;
}

}  // namespace tb

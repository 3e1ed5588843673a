// troyn:: classes over the C ABI. Every operation is one or a few tb_* calls on
// the legacy default stream (the reference's stream); objects own device memory
// from the stream-ordered pool. Validation and exceptions follow the reference's
// EvaluatorCuda / EncryptorCuda / DecryptorCuda / KeyGeneratorCuda (file:line cited
// per method); the arithmetic is the CUDA library's.
#include "troy_b200.hpp"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstring>
#include <numeric>
#include <sstream>

#include "hash.hpp"
#include "hostmath.hpp"

namespace troyn {

const ParmsID parmsIDZero = {0, 0, 0, 0};

namespace {

constexpr int POLY_DEGREE_MIN = 2, POLY_DEGREE_MAX = 131072;
constexpr int COEFF_COUNT_MAX = 64, MOD_BITS_MIN = 2, MOD_BITS_MAX = 60;
constexpr int PLAIN_BITS_MIN = 2, PLAIN_BITS_MAX = 60;

void cuda_check(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// Status -> the exception type the reference throws for the same condition.
void check(int st) {
    if (st == TB_OK) return;
    const std::string msg = tb_last_error();
    switch (st) {
    case TB_ERR_INVALID_ARGUMENT:
    case TB_ERR_NO_KEY:
        throw std::invalid_argument(msg);
    case TB_ERR_UNSUPPORTED:
        throw std::logic_error(msg);
    default:
        throw std::runtime_error(msg);
    }
}

int bits_of(uint64_t v) { return v ? 64 - __builtin_clzll(v) : 0; }

uint64_t gcd64(uint64_t a, uint64_t b) {
    while (b) {
        uint64_t t = a % b;
        a = b;
        b = t;
    }
    return a;
}

// Non-adjacent form of value as signed powers of two, lowest first (util::naf).
std::vector<int> naf(int value) {
    std::vector<int> out;
    const bool neg = value < 0;
    long long v = value < 0 ? -(long long)value : value;
    for (int i = 0; v; i++) {
        const long long z = (v & 1) ? 2 - (v & 3) : 0;
        v = (v - z) >> 1;
        if (z) out.push_back((int)((neg ? -z : z) * (1LL << i)));
    }
    return out;
}

}  // namespace

// ------------------------------------------------------------------ DeviceBuffer

DeviceBuffer::DeviceBuffer(std::size_t words) { resize(words); }

DeviceBuffer::DeviceBuffer(const DeviceBuffer &o) { *this = o; }

DeviceBuffer::DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_) {
    o.p_ = nullptr;
    o.n_ = 0;
}

DeviceBuffer &DeviceBuffer::operator=(const DeviceBuffer &o) {
    if (this == &o) return *this;
    if (n_ != o.n_) {
        DeviceBuffer fresh(o.n_);
        *this = std::move(fresh);
    }
    if (n_) cuda_check(cudaMemcpyAsync(p_, o.p_, n_ * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
    return *this;
}

DeviceBuffer &DeviceBuffer::operator=(DeviceBuffer &&o) noexcept {
    if (this != &o) {
        if (p_) cudaFreeAsync(p_, 0);
        p_ = o.p_;
        n_ = o.n_;
        o.p_ = nullptr;
        o.n_ = 0;
    }
    return *this;
}

DeviceBuffer::~DeviceBuffer() {
    if (p_) cudaFreeAsync(p_, 0);
}

// Keeps the common prefix; new words are zero (Plaintext/Ciphertext::resize semantics).
void DeviceBuffer::resize(std::size_t words) {
    if (words == n_) return;
    uint64_t *np = nullptr;
    if (words) {
        cuda_check(cudaMallocAsync(reinterpret_cast<void **>(&np), words * 8, 0), "device allocation");
        const std::size_t keep = std::min(words, n_);
        if (keep) cuda_check(cudaMemcpyAsync(np, p_, keep * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
        if (words > keep) cuda_check(cudaMemsetAsync(np + keep, 0, (words - keep) * 8, 0), "device memset");
    }
    if (p_) cudaFreeAsync(p_, 0);
    p_ = np;
    n_ = words;
}

void DeviceBuffer::zero() {
    if (n_) cuda_check(cudaMemsetAsync(p_, 0, n_ * 8, 0), "device memset");
}

std::vector<uint64_t> DeviceBuffer::toHost() const {
    std::vector<uint64_t> h(n_);
    if (n_) cuda_check(cudaMemcpy(h.data(), p_, n_ * 8, cudaMemcpyDeviceToHost), "copy to host");
    return h;
}

void DeviceBuffer::fromHost(const uint64_t *data, std::size_t words) {
    resize(words);
    if (words) cuda_check(cudaMemcpy(p_, data, words * 8, cudaMemcpyHostToDevice), "copy to device");
}

// ------------------------------------------------------------------ moduli

bool Modulus::isPrime() const { return tb::host::is_prime(v_); }
int Modulus::bitCount() const { return bits_of(v_); }

static std::vector<Modulus> create_primes(std::size_t n, uint64_t factor, const std::vector<int> &bit_sizes) {
    if (n > (std::size_t)POLY_DEGREE_MAX || n < (std::size_t)POLY_DEGREE_MIN || (n & (n - 1)))
        throw std::invalid_argument("poly_modulus_degree is invalid");
    if (bit_sizes.size() > (std::size_t)COEFF_COUNT_MAX) throw std::invalid_argument("bit_sizes is invalid");
    for (int b : bit_sizes)
        if (b < MOD_BITS_MIN || b > MOD_BITS_MAX) throw std::invalid_argument("bit_sizes is invalid");
    std::map<int, std::vector<uint64_t>> table;
    std::map<int, std::size_t> count;
    for (int b : bit_sizes) count[b]++;
    for (auto &kv : count) {
        std::vector<uint64_t> primes;
        if (!tb::host::get_primes(factor, kv.first, kv.second, primes))
            throw std::logic_error("failed to find enough qualifying primes");
        table[kv.first] = primes;
    }
    std::vector<Modulus> out;
    for (int b : bit_sizes) {  // each size's list is largest first; hand out from its end
        out.emplace_back(table[b].back());
        table[b].pop_back();
    }
    return out;
}

std::vector<Modulus> CoeffModulus::Create(std::size_t n, std::vector<int> bit_sizes) {
    return create_primes(n, 2 * (uint64_t)n, bit_sizes);
}

std::vector<Modulus> CoeffModulus::Create(std::size_t n, const Modulus &plain, std::vector<int> bit_sizes) {
    uint64_t factor = 2 * (uint64_t)n;
    factor *= plain.value() / gcd64(plain.value(), factor);
    return create_primes(n, factor, bit_sizes);
}

// Largest total coefficient-modulus bit counts of the HomomorphicEncryption.org
// security standard (ternary secrets) at 128/192/256-bit security.
int CoeffModulus::MaxBitCount(std::size_t n, SecurityLevel sec) {
    static const std::map<std::size_t, std::array<int, 3>> table = {
        {1024, {27, 19, 14}},   {2048, {54, 37, 29}},    {4096, {109, 75, 58}},
        {8192, {218, 152, 118}}, {16384, {438, 305, 237}}, {32768, {881, 611, 476}}};
    if (sec == SecurityLevel::none) return std::numeric_limits<int>::max();
    auto it = table.find(n);
    if (it == table.end()) return 0;
    return it->second[sec == SecurityLevel::tc128 ? 0 : (sec == SecurityLevel::tc192 ? 1 : 2)];
}

// The default primes (the reference's util/globals.cpp tables): per degree and level,
// groups of equal bit size, each the largest primes = 1 mod 2N of that size in
// descending order; five single-prime entries are other primes of their size, listed.
std::vector<Modulus> CoeffModulus::BFVDefault(std::size_t n, SecurityLevel sec) {
    if (!MaxBitCount(n, sec)) throw std::invalid_argument("non-standard poly_modulus_degree");
    if (sec == SecurityLevel::none) throw std::invalid_argument("invalid security level");
    struct Group {
        int bits, count;
    };
    static const std::map<std::pair<std::size_t, int>, std::vector<Group>> groups = {
        {{1024, 128}, {{27, 1}}},   {{2048, 128}, {{54, 1}}},  {{4096, 128}, {{36, 2}, {37, 1}}},
        {{8192, 128}, {{43, 2}, {44, 3}}}, {{16384, 128}, {{48, 3}, {49, 6}}}, {{32768, 128}, {{55, 15}, {56, 1}}},
        {{1024, 192}, {{19, 1}}},   {{2048, 192}, {{37, 1}}},  {{4096, 192}, {{25, 3}}},
        {{8192, 192}, {{38, 4}}},   {{16384, 192}, {{50, 6}}}, {{32768, 192}, {{54, 5}, {55, 6}}},
        {{1024, 256}, {{14, 1}}},   {{2048, 256}, {{29, 1}}},  {{4096, 256}, {{58, 1}}},
        {{8192, 256}, {{39, 2}, {40, 1}}}, {{16384, 256}, {{47, 3}, {48, 2}}}, {{32768, 256}, {{52, 1}, {53, 8}}}};
    static const std::map<std::pair<std::size_t, int>, uint64_t> single = {
        {{1024, 128}, 0x7e00001ull},           {{2048, 128}, 0x3fffffff000001ull}, {{2048, 192}, 0x1ffffc0001ull},
        {{2048, 256}, 0x1ffc0001ull},          {{4096, 256}, 0x3ffffffff040001ull}};
    const std::pair<std::size_t, int> key{n, (int)sec};
    auto it = single.find(key);
    if (it != single.end()) return {Modulus(it->second)};
    std::vector<Modulus> out;
    for (const Group &g : groups.at(key)) {
        std::vector<uint64_t> primes;
        if (!tb::host::get_primes(2 * (uint64_t)n, g.bits, (std::size_t)g.count, primes))
            throw std::logic_error("failed to find enough qualifying primes");
        for (uint64_t p : primes) out.emplace_back(p);   // largest first
    }
    return out;
}

Modulus PlainModulus::Batching(std::size_t n, int bit_size) { return CoeffModulus::Create(n, {bit_size})[0]; }
std::vector<Modulus> PlainModulus::Batching(std::size_t n, std::vector<int> bit_sizes) {
    return CoeffModulus::Create(n, bit_sizes);
}

// ------------------------------------------------------------------ parameters

// BLAKE2b-256 of [scheme, n, q_0 .. q_{k-1}, t] (EncryptionParameters::computeParmsID,
// src/encryptionparams.cpp:118-152).
ParmsID EncryptionParameters::parmsID() const {
    std::vector<uint64_t> words;
    words.push_back((uint64_t)scheme_);
    words.push_back((uint64_t)n_);
    for (auto &m : coeff_) words.push_back(m.value());
    words.push_back(t_.value());
    ParmsID id;
    blake2b(words.data(), words.size() * 8, id.data(), 32);
    if (id == parmsIDZero) throw std::logic_error("parms_id cannot be zero");
    return id;
}

// Checks of SEALContext::validate (src/context.cpp:138-380) that decide whether a
// parameter set is usable; returns the reference's error name.
static std::string validate(const EncryptionParameters &p, SecurityLevel sec, int &total_bits, bool &batching) {
    total_bits = 0;
    batching = false;
    if (p.scheme() == SchemeType::none) return "invalid_scheme";
    const auto &q = p.coeffModulus();
    if (q.empty() || q.size() > (std::size_t)COEFF_COUNT_MAX) return "invalid_coeff_modulus_size";
    for (auto &m : q)
        if (m.value() >> MOD_BITS_MAX || !(m.value() >> (MOD_BITS_MIN - 1))) return "invalid_coeff_modulus_bit_count";
    std::vector<uint64_t> qv;
    for (auto &m : q) qv.push_back(m.value());
    const auto Q = tb::host::product(qv.data(), qv.size());
    total_bits = tb::host::bit_count(Q);
    const std::size_t n = p.polyModulusDegree();
    if (n < (std::size_t)POLY_DEGREE_MIN || n > (std::size_t)POLY_DEGREE_MAX) return "invalid_poly_modulus_degree";
    if (n & (n - 1)) return "invalid_poly_modulus_degree_non_power_of_two";
    if (total_bits > CoeffModulus::MaxBitCount(n, sec) && sec != SecurityLevel::none) return "invalid_parameters_insecure";
    for (std::size_t i = 0; i < qv.size(); i++)
        for (std::size_t j = i + 1; j < qv.size(); j++)
            if (gcd64(qv[i], qv[j]) != 1) return "failed_creating_rns_base";
    for (uint64_t v : qv)
        if (!tb::host::is_prime(v) || v % (2 * n) != 1) return "invalid_coeff_modulus_no_ntt";
    const uint64_t t = p.plainModulus().value();
    if (p.scheme() == SchemeType::bfv || p.scheme() == SchemeType::bgv) {
        if (t >> PLAIN_BITS_MAX || !(t >> (PLAIN_BITS_MIN - 1))) return "invalid_plain_modulus_bit_count";
        for (uint64_t v : qv)
            if (gcd64(v, t) != 1) return "invalid_plain_modulus_coprimality";
        bool less = false;  // t < Q
        for (std::size_t k = 1; k < Q.size() && !less; k++) less = Q[k] != 0;
        if (!less && !(t < Q[0])) return "invalid_plain_modulus_too_large";
        batching = tb::host::is_prime(t) && t % (2 * n) == 1;
    } else if (p.scheme() == SchemeType::ckks) {
        if (t != 0) return "invalid_plain_modulus_nonzero";
        batching = true;
    }
    return "success";
}

namespace {

using ErrorType = EncryptionParameterQualifiers::ErrorType;

struct ErrorInfo {
    ErrorType type;
    const char *name, *message;
};

// The reference's error names (EncryptionParameterQualifiers::parameterErrorName,
// src/context.cpp:24-79) with a description of each.
const ErrorInfo kErrors[] = {
    {ErrorType::none, "none", "the parameters have not been validated"},
    {ErrorType::success, "success", "the parameters are valid"},
    {ErrorType::invalid_scheme, "invalid_scheme", "the scheme is not BFV, CKKS or BGV"},
    {ErrorType::invalid_coeff_modulus_size, "invalid_coeff_modulus_size", "the number of coefficient moduli is out of range"},
    {ErrorType::invalid_coeff_modulus_bit_count, "invalid_coeff_modulus_bit_count",
     "a coefficient modulus has a bit count out of range"},
    {ErrorType::invalid_coeff_modulus_no_ntt, "invalid_coeff_modulus_no_ntt",
     "a coefficient modulus is not a prime congruent to 1 modulo 2 * poly_modulus_degree"},
    {ErrorType::invalid_poly_modulus_degree, "invalid_poly_modulus_degree", "poly_modulus_degree is out of range"},
    {ErrorType::invalid_poly_modulus_degree_non_power_of_two, "invalid_poly_modulus_degree_non_power_of_two",
     "poly_modulus_degree is not a power of two"},
    {ErrorType::invalid_parameters_too_large, "invalid_parameters_too_large", "the parameters are too large"},
    {ErrorType::invalid_parameters_insecure, "invalid_parameters_insecure",
     "the coefficient modulus is too large for the security level"},
    {ErrorType::failed_creating_rns_base, "failed_creating_rns_base", "the coefficient moduli are not pairwise coprime"},
    {ErrorType::invalid_plain_modulus_bit_count, "invalid_plain_modulus_bit_count",
     "the plain modulus has a bit count out of range"},
    {ErrorType::invalid_plain_modulus_coprimality, "invalid_plain_modulus_coprimality",
     "the plain modulus is not coprime to the coefficient moduli"},
    {ErrorType::invalid_plain_modulus_too_large, "invalid_plain_modulus_too_large",
     "the plain modulus is not smaller than the coefficient modulus"},
    {ErrorType::invalid_plain_modulus_nonzero, "invalid_plain_modulus_nonzero", "CKKS needs a plain modulus of zero"},
    {ErrorType::failed_creating_rns_tool, "failed_creating_rns_tool", "the RNS tool could not be created"},
};

const ErrorInfo &error_info(ErrorType t) {
    for (const auto &e : kErrors)
        if (e.type == t) return e;
    return kErrors[0];
}

ErrorType error_of(const std::string &name) {
    for (const auto &e : kErrors)
        if (name == e.name) return e.type;
    return ErrorType::none;
}

}  // namespace

const char *EncryptionParameterQualifiers::parameterErrorName() const { return error_info(parameter_error).name; }
const char *EncryptionParameterQualifiers::parameterErrorMessage() const { return error_info(parameter_error).message; }

// SEALContext::SEALContext (src/context.cpp:458-523): key level, first level (key
// level minus the special prime), then the chain down while levels stay valid.
SEALContext::SEALContext(EncryptionParameters parms, bool expand_mod_chain, SecurityLevel sec_level) {
    if (!parms.randomGenerator()) parms.setRandomGenerator(std::make_shared<Blake2xbPRNGFactory>());
    scheme_ = parms.scheme();
    n_ = parms.polyModulusDegree();
    key_parms_ = parms;
    // validation and the per-level constants (SEALContext::validate, src/context.cpp:138-425)
    auto make = [&](const EncryptionParameters &p, std::string &err) {
        auto d = std::make_shared<ContextData>();
        d->parms_ = p;
        d->id_ = p.parmsID();
        bool batching = false;
        err = validate(p, sec_level, d->total_bits_, batching);
        auto &q = d->q_;
        q.parameter_error = error_of(err);
        const ErrorType e = q.parameter_error;
        const bool shape_ok = e != ErrorType::invalid_scheme && e != ErrorType::invalid_coeff_modulus_size &&
                              e != ErrorType::invalid_coeff_modulus_bit_count &&
                              e != ErrorType::invalid_poly_modulus_degree &&
                              e != ErrorType::invalid_poly_modulus_degree_non_power_of_two;
        q.using_fft = shape_ok;
        if (shape_ok)
            q.sec_level = d->total_bits_ > CoeffModulus::MaxBitCount(p.polyModulusDegree(), sec_level) ? SecurityLevel::none
                                                                                                     : sec_level;
        q.using_ntt = shape_ok && e != ErrorType::invalid_parameters_insecure &&
                      e != ErrorType::failed_creating_rns_base && e != ErrorType::invalid_coeff_modulus_no_ntt;
        q.using_batching = batching;
        if (e != ErrorType::success) return d;
        std::vector<uint64_t> qv;
        for (auto &m : p.coeffModulus()) qv.push_back(m.value());
        const std::size_t L = qv.size();
        d->total_ = tb::host::product(qv.data(), L);
        d->total_.resize(L, 0);
        q.using_descending_modulus_chain = true;
        for (std::size_t i = 0; i + 1 < L; i++) q.using_descending_modulus_chain &= qv[i] > qv[i + 1];
        if (p.scheme() == SchemeType::ckks) {
            d->plain_thr_ = uint64_t(1) << 63;
            for (uint64_t qi : qv) d->plain_inc_.push_back(tb::host::mulmod((uint64_t(1) << 63) % qi, qi - 2, qi));
            d->upper_thr_ = d->total_;   // (Q + 1) / 2
            for (std::size_t i = 0; i < L && ++d->upper_thr_[i] == 0; i++) {
            }
            for (std::size_t i = 0; i < L; i++)
                d->upper_thr_[i] = (d->upper_thr_[i] >> 1) | (i + 1 < L ? d->upper_thr_[i + 1] << 63 : 0);
            return d;
        }
        const uint64_t t = p.plainModulus().value();
        q.using_fast_plain_lift = true;
        for (uint64_t qi : qv) q.using_fast_plain_lift &= qi > t;
        uint64_t rem = 0;
        const auto delta = tb::host::div_words(d->total_, t, rem);
        d->q_mod_t_ = rem;
        for (uint64_t qi : qv) {
            const uint64_t v = tb::host::mod_words(delta, qi);
            d->delta_.push_back({v, tb::host::shoup(v, qi)});
            d->upper_inc_.push_back(rem % qi);
        }
        d->plain_thr_ = (t + 1) >> 1;
        if (q.using_fast_plain_lift) {
            for (uint64_t qi : qv) d->plain_inc_.push_back(qi - t);
        } else {   // Q - t as words
            d->plain_inc_ = d->total_;
            uint64_t borrow = t;
            for (std::size_t i = 0; i < L && borrow; i++) {
                const uint64_t w = d->plain_inc_[i];
                d->plain_inc_[i] = w - borrow;
                borrow = w < borrow ? 1 : 0;
            }
        }
        return d;
    };
    auto next_of = [](const EncryptionParameters &p) {
        EncryptionParameters next = p;
        auto q = p.coeffModulus();
        q.pop_back();
        next.setCoeffModulus(q);
        return next;
    };
    std::string err;
    auto key = make(parms, err);
    key_ = key->id_;
    data_[key_] = key;
    error_ = err;
    first_ = key_;
    if (err == "success" && parms.coeffModulus().size() > 1) {
        std::string e2;
        auto d = make(next_of(parms), e2);
        if (e2 == "success") {
            data_[d->id_] = d;
            key->next_ = d;
            d->prev_ = key;
            first_ = d->id_;
        }
    }
    last_ = first_;
    if (expand_mod_chain && err == "success") {
        auto prev = data_[first_];
        while (prev->parms_.coeffModulus().size() > 1) {
            std::string e2;
            auto d = make(next_of(prev->parms_), e2);
            if (e2 != "success") break;
            data_[d->id_] = d;
            prev->next_ = d;
            d->prev_ = prev;
            prev = d;
            last_ = d->id_;
        }
    }
    std::size_t count = data_.size();
    for (auto d = data_[key_]; d; d = std::const_pointer_cast<ContextData>(d->next_)) d->chain_index_ = --count;
    if (err != "success") return;
    std::vector<uint64_t> qv;
    for (auto &m : parms.coeffModulus()) qv.push_back(m.value());
    K_ = (int)qv.size();
    tb_context *h = nullptr;
    const int sch = scheme_ == SchemeType::bfv ? TB_SCHEME_BFV : (scheme_ == SchemeType::bgv ? TB_SCHEME_BGV : TB_SCHEME_CKKS);
    check(tb_context_create(sch, n_, qv.data(), K_, parms.plainModulus().value(), &h));
    handle_ = std::shared_ptr<tb_context>(h, [](tb_context *p) { tb_context_destroy(p); });
    // containers allocate from the device's stream-ordered pool: keep freed blocks for
    // reuse instead of returning them to the driver at every synchronisation
    int dev = 0;
    cudaMemPool_t pool;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
}

void SEALContext::requireSet() const {
    if (!parametersSet()) throw std::invalid_argument("encryption parameters are not set correctly");
}

std::shared_ptr<const SEALContext::ContextData> SEALContext::getContextData(const ParmsID &id) const {
    auto it = data_.find(id);
    return it == data_.end() ? nullptr : it->second;
}

// ------------------------------------------------------------------ containers

void Plaintext::resize(std::size_t coeff_count) {
    data_.resize(coeff_count);
    count_ = coeff_count;
}

void Plaintext::fromHost(const std::vector<uint64_t> &v) {
    data_.fromHost(v.data(), v.size());
    count_ = v.size();
}

Ciphertext::Ciphertext(const SEALContext &context) { resize(context, context.firstParmsID(), 2); }

void Ciphertext::resize(const SEALContext &context, const ParmsID &parms_id, std::size_t size) {
    auto d = context.getContextData(parms_id);
    if (!d) throw std::invalid_argument("parms_id is not valid for encryption parameters");
    if (size < 2 && size != 0) throw std::invalid_argument("invalid size");
    limbs_ = d->parms().coeffModulus().size();
    n_ = d->parms().polyModulusDegree();
    size_ = size;
    parms_id_ = parms_id;
    data_.resize(size * limbs_ * n_);
}

namespace {

// hexadecimal digits at p, and the degree of an "x^<decimal>" after them (0 when
// absent; -1 when malformed)
int hex_digits(const std::string &s, std::size_t p) {
    std::size_t k = p;
    while (k < s.size() && std::isxdigit((unsigned char)s[k])) k++;
    return (int)(k - p);
}

long long term_power(const std::string &s, std::size_t p, std::size_t &len) {
    len = 0;
    if (p >= s.size() || s[p] != 'x') return 0;
    if (p + 1 >= s.size() || s[p + 1] != '^') return -1;
    std::size_t k = p + 2;
    long long v = 0;
    while (k < s.size() && std::isdigit((unsigned char)s[k])) {
        v = v * 10 + (s[k] - '0');
        if (v > (1ll << 31)) return -1;
        k++;
    }
    if (k == p + 2) return -1;
    len = k - p;
    return v;
}

}  // namespace

Plaintext &Plaintext::operator=(const std::string &hex) {
    if (isNttForm()) throw std::logic_error("cannot set an NTT transformed Plaintext");
    struct Term {
        long long power;
        uint64_t value;
    };
    std::vector<Term> terms;
    long long last = 1ll << 31;
    std::size_t pos = 0;
    while (pos < hex.size()) {
        const int digits = hex_digits(hex, pos);
        if (digits == 0) throw std::invalid_argument("unable to parse hex_poly");
        std::size_t first = pos;
        while (first < pos + digits - 1 && hex[first] == '0') first++;   // leading zeros
        if (pos + digits - first > 16) throw std::invalid_argument("hex_poly has too large coefficients");
        const uint64_t value = std::stoull(hex.substr(first, pos + digits - first), nullptr, 16);
        pos += digits;
        std::size_t len = 0;
        const long long power = term_power(hex, pos, len);
        if (power < 0 || power >= last) throw std::invalid_argument("unable to parse hex_poly");
        pos += len;
        last = power;
        terms.push_back({power, value});
        if (pos < hex.size()) {   // " + " between terms (also accepted at the very end)
            if (hex.compare(pos, 3, " + ") != 0) throw std::invalid_argument("unable to parse hex_poly");
            pos += 3;
        }
    }
    bool any = false;
    for (auto &t : terms) any |= t.value != 0;
    if (terms.empty() || !any) {
        setZero();
        return *this;
    }
    std::vector<uint64_t> v((std::size_t)terms.front().power + 1, 0);
    for (auto &t : terms) v[(std::size_t)t.power] = t.value;
    fromHost(v);
    return *this;
}

std::string Plaintext::to_string() const {
    if (isNttForm()) throw std::invalid_argument("cannot convert NTT transformed plaintext to string");
    const auto v = toHost();
    std::ostringstream out;
    bool empty = true;
    for (std::size_t i = count_; i-- > 0;) {
        if (!v[i]) continue;
        if (!empty) out << " + ";
        out << std::uppercase << std::hex << v[i] << std::dec;
        if (i) out << "x^" << i;
        empty = false;
    }
    return empty ? "0" : out.str();
}

bool Plaintext::isZero() const {
    for (uint64_t w : toHost())
        if (w) return false;
    return true;
}

uint64_t Plaintext::operator[](std::size_t i) const {
    if (i >= count_) throw std::out_of_range("coeff_index must be within [0, coeff_count)");
    uint64_t v = 0;
    cuda_check(cudaMemcpy(&v, data_.get() + i, 8, cudaMemcpyDeviceToHost), "copy to host");
    return v;
}

bool Plaintext::operator==(const Plaintext &o) const {
    if (parms_id_ != o.parms_id_ || (isNttForm() && scale_ != o.scale_)) return false;
    auto a = toHost(), b = o.toHost();
    a.resize(std::max(a.size(), b.size()), 0);
    b.resize(a.size(), 0);
    return a == b;
}

bool Ciphertext::isTransparent() const {
    if (!data_.size() || size_ < 2) return true;
    const auto v = toHost();
    for (std::size_t i = n_ * limbs_; i < v.size(); i++)
        if (v[i]) return false;
    return true;
}

void Ciphertext::fromHost(const std::vector<uint64_t> &v) {
    if (v.size() != size_ * limbs_ * n_) throw std::invalid_argument("data size mismatch");
    data_.fromHost(v.data(), v.size());
    seed_ = 0;
}

const uint64_t *KSwitchKeys::key(std::size_t index) const {
    auto it = keys_.find(index);
    if (it == keys_.end()) throw std::invalid_argument("key not present");
    return it->second.get();
}

void KernelProvider::initialize(int device) { cuda_check(cudaSetDevice(device), "cudaSetDevice"); }

// ------------------------------------------------------------------ uneven batches

tb_uneven_group UnevenBatch::group(const SEALContext &context, int level_limbs, std::uint64_t count,
                                   const std::uint64_t *a, const std::uint64_t *b, const std::uint64_t *relin_key,
                                   const std::uint64_t *galois_key, std::uint32_t galois_elt, std::uint64_t *out) {
    context.requireSet();
    tb_uneven_group g{};
    g.ctx = context.handle();
    g.L = level_limbs;
    g.count = count;
    g.a = a;
    g.b = b;
    g.relin_key = relin_key;
    g.galois_key = galois_key;
    g.galois_elt = galois_elt;
    g.out = out;
    return g;
}

UnevenBatch::UnevenBatch(const std::vector<tb_uneven_group> &groups) {
    check(tb_uneven_create(groups.data(), (int)groups.size(), &h_));
}

UnevenBatch::~UnevenBatch() { tb_uneven_destroy(h_); }

void UnevenBatch::run(void *stream) { check(tb_uneven_run(h_, stream)); }
void UnevenBatch::runPerOp(void *stream) { check(tb_uneven_run_per_op(h_, stream)); }
void UnevenBatch::capture() { check(tb_uneven_capture(h_)); }
void UnevenBatch::replay(void *stream) { check(tb_uneven_replay(h_, stream)); }

// ------------------------------------------------------------------ keys

// KeyGeneratorCuda (src/keygenerator_cuda.cuh:36-312): secret key from the context's
// PRNG factory; the library generates every key on the device.
KeyGenerator::KeyGenerator(const SEALContext &context) : context_(context) {
    context.requireSet();
    const std::size_t n = context.polyModulusDegree();
    sk_.data().resize((std::size_t)context.keyLimbs() * n);
    check(tb_keygen_secret(context.handle(), context.keyParms().randomGenerator()->seedPtr(), sk_.data().get(),
                           nullptr));
    sk_.parmsID() = context.keyParmsID();
}

KeyGenerator::KeyGenerator(const SEALContext &context, const SecretKey &secret_key) : context_(context) {
    context.requireSet();
    if (secret_key.parmsID() != context.keyParmsID())
        throw std::invalid_argument("secret key is not valid for encryption parameters");
    sk_ = secret_key;
}

void KeyGenerator::createPublicKey(PublicKey &pk) const {
    pk.data().resize(2ull * context_.keyLimbs() * context_.polyModulusDegree());
    check(tb_keygen_public(context_.handle(), context_.keyParms().randomGenerator()->seedPtr(), sk_.data().get(),
                           pk.data().get(), nullptr));
    pk.parmsID() = context_.keyParmsID();
    pk.polyModulusDegree() = context_.polyModulusDegree();
    pk.limbs() = context_.keyLimbs();
}

static std::size_t kswitch_words(const SEALContext &c) {
    return (std::size_t)(c.keyLimbs() - 1) * 2 * c.keyLimbs() * c.polyModulusDegree();
}

void KeyGenerator::createRelinKeys(RelinKeys &dest) const {
    if (!context_.using_keyswitching()) throw std::logic_error("keyswitching is not supported by the context");
    dest.data().clear();
    DeviceBuffer k(kswitch_words(context_));
    check(tb_keygen_relin(context_.handle(), context_.keyParms().randomGenerator()->seedPtr(), sk_.data().get(),
                          k.get(), nullptr));
    dest.data()[RelinKeys::getIndex(2)] = std::move(k);
    dest.slotCount() = 1;
    dest.polyModulusDegree() = context_.polyModulusDegree();
    dest.limbs() = context_.keyLimbs();
    dest.parmsID() = context_.keyParmsID();
}

void KeyGenerator::createGaloisKeys(const std::vector<uint32_t> &elts, GaloisKeys &dest) const {
    if (!context_.using_keyswitching()) throw std::logic_error("keyswitching is not supported by the context");
    const uint64_t m = 2 * (uint64_t)context_.polyModulusDegree();
    dest.data().clear();
    for (uint32_t e : elts) {
        if (!(e & 1) || e >= m) throw std::invalid_argument("Galois element is not valid");
        if (dest.hasKeyElt(e)) continue;
        DeviceBuffer k(kswitch_words(context_));
        check(tb_keygen_galois(context_.handle(), context_.keyParms().randomGenerator()->seedPtr(), sk_.data().get(),
                               e, k.get(), nullptr));
        dest.data()[GaloisKeys::getIndex(e)] = std::move(k);
    }
    dest.slotCount() = context_.polyModulusDegree();
    dest.polyModulusDegree() = context_.polyModulusDegree();
    dest.limbs() = context_.keyLimbs();
    dest.parmsID() = context_.keyParmsID();
}

uint32_t KeyGenerator::galoisEltFromStep(int step) const {
    uint32_t e = 0;
    check(tb_galois_elt_from_step(context_.handle(), step, &e));
    return e;
}

void KeyGenerator::createGaloisKeys(const std::vector<int> &steps, GaloisKeys &dest) const {
    if (!context_.keyContextData()->usingBatching())
        throw std::logic_error("encryption parameters do not support batching");
    std::vector<uint32_t> elts;
    for (int s : steps) elts.push_back(galoisEltFromStep(s));
    createGaloisKeys(elts, dest);
}

// GaloisTool::getEltsAll (src/utils/galois.cpp:101-129): m - 1, then 3^(2^i) and
// 3^(-2^i) for i < log2(n) - 1.
std::vector<uint32_t> KeyGenerator::galoisEltsAll() const {
    const uint64_t m = 2 * (uint64_t)context_.polyModulusDegree();
    const int logn = bits_of(context_.polyModulusDegree()) - 1;
    std::vector<uint32_t> out{(uint32_t)(m - 1)};
    uint64_t pos = 3, neg = tb::host::invmod(3, m);
    for (int i = 0; i < logn - 1; i++) {
        out.push_back((uint32_t)pos);
        pos = (pos * pos) & (m - 1);
        out.push_back((uint32_t)neg);
        neg = (neg * neg) & (m - 1);
    }
    return out;
}

void KeyGenerator::createGaloisKeys(GaloisKeys &dest) const { createGaloisKeys(galoisEltsAll(), dest); }

// ------------------------------------------------------------------ encryption

static int limbs_of(const SEALContext &c, const ParmsID &id, const char *what) {
    auto d = c.getContextData(id);
    if (!d) throw std::invalid_argument(std::string(what) + " is not valid for encryption parameters");
    return d->levelLimbs();
}

// EncryptorCuda::encryptInternal (src/encryptor_cuda.cu:92-237).
void Encryptor::run(const Plaintext *plain, const ParmsID &id, bool asym, Ciphertext &dest, bool seeded) const {
    context_.requireSet();
    if (asym && !has_pk_) throw std::logic_error("public key is not set");
    if (!asym && !has_sk_) throw std::logic_error("secret key is not set");
    const bool ckks = context_.scheme() == SchemeType::ckks;
    ParmsID level = id;
    if (plain) {
        if (ckks) {
            if (!plain->isNttForm()) throw std::invalid_argument("plain must be in NTT form");
            level = plain->parmsID();
        } else {
            if (plain->isNttForm()) throw std::invalid_argument("plain cannot be in NTT form");
            if (plain->coeffCount() > context_.polyModulusDegree())
                throw std::invalid_argument("plain is not valid for encryption parameters");
            level = context_.firstParmsID();
        }
    }
    const int L = limbs_of(context_, level, "parms_id");
    Ciphertext out;
    out.resize(context_, level, 2);
    const uint64_t *seed = context_.keyParms().randomGenerator()->seedPtr();
    const uint64_t *p = plain ? plain->data() : nullptr;
    const uint64_t count = plain ? (ckks ? 0 : plain->coeffCount()) : 0;
    std::uint64_t ct_seed = 0;
    if (asym)
        check(tb_encrypt(context_.handle(), seed, pk_.data().get(), L, p, 0, count, out.data(), 0, 1, nullptr));
    else if (seeded)
        check(tb_encrypt_symmetric_seeded(context_.handle(), seed, sk_.data().get(), L, p, 0, count, out.data(), 0,
                                          &ct_seed, 1, nullptr));
    else
        check(tb_encrypt_symmetric(context_.handle(), seed, sk_.data().get(), L, p, 0, count, out.data(), 0, 1,
                                   nullptr));
    out.isNttForm() = ckks;
    out.scale() = (plain && ckks) ? plain->scale() : 1.0;
    out.correctionFactor() = 1;
    out.seed() = ct_seed;
    dest = std::move(out);
}

void Encryptor::encrypt(const Plaintext &plain, Ciphertext &dest) const { run(&plain, parmsIDZero, true, dest); }
void Encryptor::encryptZero(const ParmsID &id, Ciphertext &dest) const { run(nullptr, id, true, dest); }
void Encryptor::encryptSymmetric(const Plaintext &plain, Ciphertext &dest) const {
    run(&plain, parmsIDZero, false, dest);
}
void Encryptor::encryptZeroSymmetric(const ParmsID &id, Ciphertext &dest) const { run(nullptr, id, false, dest); }
void Encryptor::encryptSymmetricSeeded(const Plaintext &plain, Ciphertext &dest) const {
    run(&plain, parmsIDZero, false, dest, true);
}
void Encryptor::encryptZeroSymmetricSeeded(const ParmsID &id, Ciphertext &dest) const {
    run(nullptr, id, false, dest, true);
}

// DecryptorCuda::decrypt (src/decryptor_cuda.cu:92-328).
void Decryptor::decrypt(const Ciphertext &ct, Plaintext &dest) {
    context_.requireSet();
    const int L = limbs_of(context_, ct.parmsID(), "encrypted");
    if (ct.size() < 2) throw std::invalid_argument("encrypted is empty");
    const std::size_t n = context_.polyModulusDegree();
    switch (context_.scheme()) {
    case SchemeType::bfv:
    case SchemeType::bgv: {
        if (ct.isNttForm()) throw std::invalid_argument("encrypted cannot be in NTT form");
        Plaintext p(n);
        check(tb_decrypt(context_.handle(), sk_.data().get(), L, (int)ct.size(), ct.data(), 0, p.data(), 0,
                         ct.correctionFactor(), 1, nullptr));
        dest = std::move(p);
        break;
    }
    case SchemeType::ckks: {
        if (!ct.isNttForm()) throw std::invalid_argument("encrypted must be in NTT form");
        Plaintext p((std::size_t)L * n);
        check(tb_decrypt(context_.handle(), sk_.data().get(), L, (int)ct.size(), ct.data(), 0, p.data(), 0, 1, 1,
                         nullptr));
        p.parmsID() = ct.parmsID();
        p.scale() = ct.scale();
        dest = std::move(p);
        break;
    }
    default:
        throw std::invalid_argument("unsupported scheme");
    }
}

// ------------------------------------------------------------------ evaluator helpers

// isScaleWithinBounds (src/evaluator_cuda.cu): log2(scale) below the plain modulus
// bits (BFV/BGV) or the level's total modulus bits (CKKS).
bool isScaleWithinBounds(double scale, const SEALContext::ContextData &d) {
    int bound = 0;
    switch (d.parms().scheme()) {
    case SchemeType::bfv:
    case SchemeType::bgv:
        bound = d.parms().plainModulus().bitCount();
        break;
    case SchemeType::ckks:
        bound = d.totalCoeffModulusBitCount();
        break;
    default:
        return false;
    }
    return !(scale <= 0 || (int)std::log2(scale) >= bound);
}

namespace {

bool scale_ok(double scale, const SEALContext::ContextData &d) { return isScaleWithinBounds(scale, d); }

// Relative closeness of two scales (areClose, src/utils/common.h).
bool same_scale(double a, double b) {
    const double scale = std::max(std::fabs(a), std::fabs(b));
    return std::fabs(a - b) < std::max(scale * std::numeric_limits<double>::epsilon() * 4096.0,
                                       std::numeric_limits<double>::min());
}

uint64_t mulmod(uint64_t a, uint64_t b, uint64_t t) { return tb::host::mulmod(a, b, t); }

// BGV correction-factor balancing (balanceCorrectionFactors,
// src/evaluator_cuda.cu:53-114): the pair (e1, e2) with e1 f1 = e2 f2 mod t of
// smallest centred magnitude, found along the extended Euclidean sequence of
// (t, f2/f1). Returns (e1 f1, e1, e2).
std::array<uint64_t, 3> balance(uint64_t f1, uint64_t f2, uint64_t t) {
    const uint64_t half = t / 2;
    auto centred = [&](uint64_t x) { return (long long)(x > half ? x - t : x); };
    auto cost = [&](uint64_t x, uint64_t y) { return std::llabs(centred(x)) + std::llabs(centred(y)); };
    const uint64_t inv = tb::host::invmod(f1 % t, t);
    if (!inv) throw std::logic_error("invalid correction factor1");
    const uint64_t ratio = mulmod(inv, f2, t);
    uint64_t e1 = ratio, e2 = 1;
    long long best = cost(e1, e2);
    long long pa = (long long)t, pb = 0, a = (long long)ratio, b = 1;
    auto red = [&](long long v) {
        const uint64_t r = (uint64_t)std::llabs(v) % t;
        return (v < 0 && r) ? t - r : r;
    };
    while (a != 0) {
        const long long q = pa / a;
        long long tmp = pa % a;
        pa = a;
        a = tmp;
        tmp = pb - b * q;
        pb = b;
        b = tmp;
        const uint64_t am = red(a), bm = red(b);
        if (am != 0 && gcd64(am, t) == 1) {
            const long long c = cost(am, bm);
            if (c < best) {
                best = c;
                e1 = am;
                e2 = bm;
            }
        }
    }
    return {mulmod(e1, f1, t), e1, e2};
}

}  // namespace

static const SEALContext::ContextData &data_of(const SEALContext &c, const Ciphertext &ct) {
    auto d = c.getContextData(ct.parmsID());
    if (!d) throw std::invalid_argument("encrypted is not valid for encryption parameters");
    return *d;
}

static void check_form(const SEALContext &c, const Ciphertext &ct) {
    const SchemeType s = c.scheme();
    if (s == SchemeType::bfv && ct.isNttForm()) throw std::invalid_argument("BFV encrypted cannot be in NTT form");
    if (s == SchemeType::ckks && !ct.isNttForm()) throw std::invalid_argument("CKKS encrypted must be in NTT form");
    if (s == SchemeType::bgv && ct.isNttForm()) throw std::invalid_argument("BGV encrypted cannot be in NTT form");
}

// ------------------------------------------------------------------ evaluator

void Evaluator::negateInplace(Ciphertext &ct) const {
    const int L = data_of(context_, ct).levelLimbs();
    check(tb_negate(context_.handle(), L, (int)ct.size(), ct.data(), 0, ct.data(), 0, 1, nullptr));
}
void Evaluator::negate(const Ciphertext &a, Ciphertext &d) const {
    d = a;
    negateInplace(d);
}

// EvaluatorCuda::addInplace / subInplace (src/evaluator_cuda.cu:156-260).
static void add_sub(const SEALContext &context, Ciphertext &a, const Ciphertext &b, bool sub) {
    const auto &d = data_of(context, a);
    if (a.parmsID() != b.parmsID()) throw std::invalid_argument("encrypted1 and encrypted2 parameter mismatch");
    if (a.isNttForm() != b.isNttForm()) throw std::invalid_argument("NTT form mismatch");
    if (!same_scale(a.scale(), b.scale())) throw std::invalid_argument("scale mismatch");
    const int L = d.levelLimbs();
    if (a.correctionFactor() != b.correctionFactor()) {
        const uint64_t t = d.parms().plainModulus().value();
        auto f = balance(a.correctionFactor(), b.correctionFactor(), t);
        check(tb_multiply_scalar(context.handle(), L, (int)a.size(), a.data(), 0, f[1], a.data(), 0, 1, nullptr));
        Ciphertext bc = b;
        check(tb_multiply_scalar(context.handle(), L, (int)b.size(), b.data(), 0, f[2], bc.data(), 0, 1, nullptr));
        a.correctionFactor() = f[0];
        bc.correctionFactor() = f[0];
        add_sub(context, a, bc, sub);
        return;
    }
    const std::size_t sa = a.size(), sb = b.size(), mn = std::min(sa, sb);
    if (sa < sb) a.resize(context, a.parmsID(), sb);
    auto fn = sub ? tb_sub : tb_add;
    check(fn(context.handle(), L, (int)mn, a.data(), 0, b.data(), 0, a.data(), 0, 1, nullptr));
    if (sa < sb) {
        const std::size_t extra = sb - sa;
        if (sub)
            check(tb_negate(context.handle(), L, (int)extra, b.data(mn), 0, a.data(mn), 0, 1, nullptr));
        else
            cuda_check(cudaMemcpyAsync(a.data(mn), b.data(mn), extra * L * a.polyModulusDegree() * 8,
                                       cudaMemcpyDeviceToDevice, 0),
                       "device copy");
    }
}

void Evaluator::addInplace(Ciphertext &a, const Ciphertext &b) const { add_sub(context_, a, b, false); }
void Evaluator::add(const Ciphertext &a, const Ciphertext &b, Ciphertext &d) const {
    Ciphertext t = a;
    addInplace(t, b);
    d = std::move(t);
}
void Evaluator::subInplace(Ciphertext &a, const Ciphertext &b) const { add_sub(context_, a, b, true); }
void Evaluator::sub(const Ciphertext &a, const Ciphertext &b, Ciphertext &d) const {
    Ciphertext t = a;
    subInplace(t, b);
    d = std::move(t);
}

void Evaluator::addMany(const std::vector<Ciphertext> &cts, Ciphertext &d) const {
    if (cts.empty()) throw std::invalid_argument("encrypteds cannot be empty");
    for (auto &c : cts)
        if (&c == &d) throw std::invalid_argument("encrypteds must be different from destination");
    d = cts[0];
    for (std::size_t i = 1; i < cts.size(); i++) addInplace(d, cts[i]);
}

// EvaluatorCuda::multiplyInplace -> bfvMultiply / ckksMultiply / bgvMultiply
// (src/evaluator_cuda.cu:262-501): size-2 operands take the fused batched product,
// larger ones the general-size product (size a + size b - 1 polynomials).
void Evaluator::multiplyInplace(Ciphertext &a, const Ciphertext &b) const {
    const auto &d = data_of(context_, a);
    if (a.parmsID() != b.parmsID()) throw std::invalid_argument("encrypted1 and encrypted2 parameter mismatch");
    check_form(context_, a);
    check_form(context_, b);
    if (a.size() < 2 || b.size() < 2) throw std::invalid_argument("encrypted is empty");
    const int L = d.levelLimbs();
    Ciphertext out;
    out.resize(context_, a.parmsID(), a.size() + b.size() - 1);
    if (a.size() == 2 && b.size() == 2)
        check(tb_multiply(context_.handle(), L, a.data(), 0, b.data(), 0, out.data(), 0, 1, nullptr));
    else
        check(tb_multiply_sizes(context_.handle(), L, a.data(), (int)a.size(), b.data(), (int)b.size(), out.data(),
                                nullptr));
    out.isNttForm() = a.isNttForm();
    out.scale() = a.scale();
    out.correctionFactor() = a.correctionFactor();
    if (context_.scheme() == SchemeType::ckks) {
        out.scale() = a.scale() * b.scale();
        if (!scale_ok(out.scale(), d)) throw std::invalid_argument("scale out of bounds");
    } else if (context_.scheme() == SchemeType::bgv) {
        out.correctionFactor() = mulmod(a.correctionFactor(), b.correctionFactor(), d.parms().plainModulus().value());
    }
    a = std::move(out);
}

void Evaluator::multiply(const Ciphertext &a, const Ciphertext &b, Ciphertext &d) const {
    Ciphertext t = a;
    multiplyInplace(t, b);
    d = std::move(t);
}

// EvaluatorCuda::relinearizeInternal (src/evaluator_cuda.cu:703-744): the last
// polynomial is switched with key s^(size-1) until two remain.
void Evaluator::relinearizeInplace(Ciphertext &ct, const RelinKeys &keys) const {
    const auto &d = data_of(context_, ct);
    if (keys.parmsID() != context_.keyParmsID())
        throw std::invalid_argument("relin_keys is not valid for encryption parameters");
    if (ct.size() < 2)
        throw std::invalid_argument("destination_size must be at least 2 and less than or equal to current count");
    if (keys.size() < ct.size() - 2) throw std::invalid_argument("not enough relinearization keys");
    const int L = d.levelLimbs();
    std::size_t size = ct.size();
    while (size > 2) {
        const uint64_t *k = keys.key(RelinKeys::getIndex(size - 1));
        if (size == 3)
            check(tb_relinearize(context_.handle(), L, ct.data(), 0, k, 1, nullptr));
        else
            check(tb_keyswitch(context_.handle(), L, ct.data(size - 1), 0, ct.data(), 0, k, 1, nullptr));
        size--;
    }
    if (size != ct.size()) ct.resize(context_, ct.parmsID(), size);
}

void Evaluator::relinearize(const Ciphertext &ct, const RelinKeys &keys, Ciphertext &d) const {
    Ciphertext t = ct;
    relinearizeInplace(t, keys);
    d = std::move(t);
}

// modSwitchScaleToNext (src/evaluator_cuda.cu:749-824): BFV/BGV divide-and-round by the
// last prime in the coefficient domain, CKKS rescale in the NTT domain.
void Evaluator::modSwitchScaleToNext(const Ciphertext &ct, Ciphertext &dest) const {
    const auto &d = data_of(context_, ct);
    check_form(context_, ct);
    auto next = d.nextContextData();
    if (!next) throw std::invalid_argument("end of modulus switching chain reached");
    const int L = d.levelLimbs();
    Ciphertext out;
    out.resize(context_, next->parmsID(), ct.size());
    check(tb_rescale_to_next(context_.handle(), L, ct.data(), 0, out.data(), 0, (int)ct.size(), 1, nullptr));
    out.isNttForm() = ct.isNttForm();
    out.scale() = ct.scale();
    out.correctionFactor() = ct.correctionFactor();
    if (context_.scheme() == SchemeType::ckks) {
        out.scale() = ct.scale() / (double)d.parms().coeffModulus().back().value();
    } else if (context_.scheme() == SchemeType::bgv) {
        const uint64_t t = d.parms().plainModulus().value();
        const uint64_t qlast = d.parms().coeffModulus().back().value();
        out.correctionFactor() = mulmod(ct.correctionFactor(), tb::host::invmod(qlast % t, t), t);
    }
    dest = std::move(out);
}

// modSwitchDropToNext (src/evaluator_cuda.cu:826-889): keep the first L-1 limbs.
void Evaluator::modSwitchDropToNext(const Ciphertext &ct, Ciphertext &dest) const {
    const auto &d = data_of(context_, ct);
    if (context_.scheme() == SchemeType::ckks && !ct.isNttForm())
        throw std::invalid_argument("CKKS encrypted must be in NTT form");
    auto next = d.nextContextData();
    if (!next) throw std::invalid_argument("end of modulus switching chain reached");
    if (!scale_ok(ct.scale(), *next)) throw std::invalid_argument("scale out of bounds");
    const std::size_t L = d.levelLimbs(), n = ct.polyModulusDegree();
    Ciphertext out;
    out.resize(context_, next->parmsID(), ct.size());
    if (ct.size())
        cuda_check(cudaMemcpy2DAsync(out.data(), (L - 1) * n * 8, ct.data(), L * n * 8, (L - 1) * n * 8, ct.size(),
                                     cudaMemcpyDeviceToDevice, 0),
                   "device copy");
    out.isNttForm() = ct.isNttForm();
    out.scale() = ct.scale();
    out.correctionFactor() = ct.correctionFactor();
    dest = std::move(out);
}

// modSwitchToNext (src/evaluator_cuda.cu:926-956).
void Evaluator::modSwitchToNext(const Ciphertext &ct, Ciphertext &dest) const {
    data_of(context_, ct);
    if (context_.lastParmsID() == ct.parmsID()) throw std::invalid_argument("end of modulus switching chain reached");
    if (context_.scheme() == SchemeType::ckks)
        modSwitchDropToNext(ct, dest);
    else
        modSwitchScaleToNext(ct, dest);
}
void Evaluator::modSwitchToNextInplace(Ciphertext &ct) const { modSwitchToNext(ct, ct); }

// modSwitchDropToNext(Plaintext) (src/evaluator_cuda.cu:891-924).
void Evaluator::modSwitchToNextInplace(Plaintext &plain) const {
    if (!plain.isNttForm()) throw std::invalid_argument("plain is not in NTT form");
    auto d = context_.getContextData(plain.parmsID());
    if (!d) throw std::invalid_argument("plain is not valid for encryption parameters");
    auto next = d->nextContextData();
    if (!next) throw std::invalid_argument("end of modulus switching chain reached");
    if (!scale_ok(plain.scale(), *next)) throw std::invalid_argument("scale out of bounds");
    plain.resize((std::size_t)next->levelLimbs() * context_.polyModulusDegree());
    plain.parmsID() = next->parmsID();
}
void Evaluator::modSwitchToNext(const Plaintext &plain, Plaintext &dest) const {
    Plaintext t = plain;
    modSwitchToNextInplace(t);
    dest = std::move(t);
}

// modSwitchToInplace (src/evaluator_cuda.cu:958-1010).
void Evaluator::modSwitchToInplace(Ciphertext &ct, const ParmsID &id) const {
    auto d = context_.getContextData(ct.parmsID());
    auto target = context_.getContextData(id);
    if (!d) throw std::invalid_argument("encrypted is not valid for encryption parameters");
    if (!target) throw std::invalid_argument("parms_id is not valid for encryption parameters");
    if (d->chainIndex() < target->chainIndex()) throw std::invalid_argument("cannot switch to higher level modulus");
    while (ct.parmsID() != id) modSwitchToNextInplace(ct);
}
void Evaluator::modSwitchTo(const Ciphertext &ct, const ParmsID &id, Ciphertext &dest) const {
    Ciphertext t = ct;
    modSwitchToInplace(t, id);
    dest = std::move(t);
}
void Evaluator::modSwitchToInplace(Plaintext &plain, const ParmsID &id) const {
    auto d = context_.getContextData(plain.parmsID());
    auto target = context_.getContextData(id);
    if (!d) throw std::invalid_argument("plain is not valid for encryption parameters");
    if (!target) throw std::invalid_argument("parms_id is not valid for encryption parameters");
    if (!plain.isNttForm()) throw std::invalid_argument("plain is not in NTT form");
    if (d->chainIndex() < target->chainIndex()) throw std::invalid_argument("cannot switch to higher level modulus");
    while (plain.parmsID() != id) modSwitchToNextInplace(plain);
}
void Evaluator::modSwitchTo(const Plaintext &plain, const ParmsID &id, Plaintext &dest) const {
    Plaintext t = plain;
    modSwitchToInplace(t, id);
    dest = std::move(t);
}

// rescaleToNext / rescaleToInplace (src/evaluator_cuda.cu:1367-1432): CKKS only.
void Evaluator::rescaleToNext(const Ciphertext &ct, Ciphertext &dest) const {
    if (context_.lastParmsID() == ct.parmsID()) throw std::invalid_argument("end of modulus switching chain reached");
    if (context_.scheme() != SchemeType::ckks) throw std::invalid_argument("unsupported operation for scheme type");
    modSwitchScaleToNext(ct, dest);
}
void Evaluator::rescaleToNextInplace(Ciphertext &ct) const { rescaleToNext(ct, ct); }
void Evaluator::rescaleToInplace(Ciphertext &ct, const ParmsID &id) const {
    auto d = context_.getContextData(ct.parmsID());
    auto target = context_.getContextData(id);
    if (!d) throw std::invalid_argument("encrypted is not valid for encryption parameters");
    if (!target) throw std::invalid_argument("parms_id is not valid for encryption parameters");
    if (d->chainIndex() < target->chainIndex()) throw std::invalid_argument("cannot switch to higher level modulus");
    if (context_.scheme() != SchemeType::ckks) throw std::invalid_argument("unsupported operation for scheme type");
    while (ct.parmsID() != id) modSwitchScaleToNext(ct, ct);
}
void Evaluator::rescaleTo(const Ciphertext &ct, const ParmsID &id, Ciphertext &dest) const {
    Ciphertext t = ct;
    rescaleToInplace(t, id);
    dest = std::move(t);
}

// multiplyMany (src/evaluator_cuda.cu:1434-1510): pairwise product tree with
// relinearization, pairs taken in the reference's order.
void Evaluator::multiplyMany(const std::vector<Ciphertext> &cts, const RelinKeys &keys, Ciphertext &dest) const {
    if (cts.empty()) throw std::invalid_argument("encrypteds vector must not be empty");
    for (auto &c : cts)
        if (&c == &dest) throw std::invalid_argument("encrypteds must be different from destination");
    data_of(context_, cts[0]);
    if (context_.scheme() != SchemeType::bfv && context_.scheme() != SchemeType::bgv)
        throw std::logic_error("unsupported scheme");
    if (cts.size() == 1) {
        dest = cts[0];
        return;
    }
    std::vector<Ciphertext> prod;
    for (std::size_t i = 0; i + 1 < cts.size(); i += 2) {
        Ciphertext t;
        multiply(cts[i], cts[i + 1], t);
        relinearizeInplace(t, keys);
        prod.push_back(std::move(t));
    }
    if (cts.size() & 1) prod.push_back(cts.back());
    for (std::size_t i = 0; i + 1 < prod.size(); i += 2) {
        Ciphertext t;
        multiply(prod[i], prod[i + 1], t);
        relinearizeInplace(t, keys);
        prod.push_back(std::move(t));
    }
    dest = prod.back();
}

// exponentiateInplace (src/evaluator_cuda.cu:1512-1542).
void Evaluator::exponentiateInplace(Ciphertext &ct, uint64_t exponent, const RelinKeys &keys) const {
    data_of(context_, ct);
    if (!context_.getContextData(keys.parmsID()))
        throw std::invalid_argument("relin_keys is not valid for encryption parameters");
    if (exponent == 0) throw std::invalid_argument("exponent cannot be 0");
    if (exponent == 1) return;
    std::vector<Ciphertext> v((std::size_t)exponent, ct);
    multiplyMany(v, keys, ct);
}
void Evaluator::exponentiate(const Ciphertext &ct, uint64_t exponent, const RelinKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    exponentiateInplace(t, exponent, keys);
    dest = std::move(t);
}

// addPlainInplace / subPlainInplace (src/evaluator_cuda.cu:1544-1689).
static void add_plain(const SEALContext &context, Ciphertext &ct, const Plaintext &plain, bool sub) {
    const auto &d = data_of(context, ct);
    check_form(context, ct);
    if (plain.isNttForm() != ct.isNttForm()) throw std::invalid_argument("NTT form mismatch");
    if (ct.isNttForm() && ct.parmsID() != plain.parmsID())
        throw std::invalid_argument("encrypted and plain parameter mismatch");
    if (!same_scale(ct.scale(), plain.scale())) throw std::invalid_argument("scale mismatch");
    const int L = d.levelLimbs();
    const std::size_t n = context.polyModulusDegree();
    if (!ct.isNttForm() && plain.coeffCount() > n)
        throw std::invalid_argument("plain is not valid for encryption parameters");
    const uint64_t count = ct.isNttForm() ? 0 : plain.coeffCount();
    const uint64_t *p = plain.data();
    Plaintext scaled;
    if (context.scheme() == SchemeType::bgv && ct.correctionFactor() != 1 && count) {
        scaled.resize(count);
        check(tb_plain_multiply_scalar(context.handle(), plain.data(), 0, count, ct.correctionFactor(), scaled.data(),
                                       0, 1, nullptr));
        p = scaled.data();
    }
    auto fn = sub ? tb_sub_plain : tb_add_plain;
    check(fn(context.handle(), L, ct.data(), 0, p, 0, count, 1, nullptr));
}

void Evaluator::addPlainInplace(Ciphertext &ct, const Plaintext &plain) const { add_plain(context_, ct, plain, false); }
void Evaluator::addPlain(const Ciphertext &ct, const Plaintext &plain, Ciphertext &dest) const {
    Ciphertext t = ct;
    addPlainInplace(t, plain);
    dest = std::move(t);
}
void Evaluator::subPlainInplace(Ciphertext &ct, const Plaintext &plain) const { add_plain(context_, ct, plain, true); }
void Evaluator::subPlain(const Ciphertext &ct, const Plaintext &plain, Ciphertext &dest) const {
    Ciphertext t = ct;
    subPlainInplace(t, plain);
    dest = std::move(t);
}

// multiplyPlainInplace -> multiplyPlainNormal / multiplyPlainNtt
// (src/evaluator_cuda.cu:1691-1867).
void Evaluator::multiplyPlainInplace(Ciphertext &ct, const Plaintext &plain) const {
    const auto &d = data_of(context_, ct);
    if (ct.isNttForm() != plain.isNttForm()) throw std::invalid_argument("NTT form mismatch");
    const int L = d.levelLimbs();
    if (ct.isNttForm()) {
        if (ct.parmsID() != plain.parmsID())
            throw std::invalid_argument("encrypted_ntt and plain_ntt parameter mismatch");
        for (std::size_t i = 0; i < ct.size(); i++)
            check(tb_dyadic_product(context_.handle(), ct.data(i), plain.data(), ct.data(i), 1, 0, L, nullptr));
        const double scale = ct.scale() * plain.scale();
        if (!scale_ok(scale, d)) throw std::invalid_argument("scale out of bounds");
        ct.scale() = scale;
    } else {
        if (plain.coeffCount() > context_.polyModulusDegree())
            throw std::invalid_argument("plain is not valid for encryption parameters");
        check(tb_multiply_plain(context_.handle(), L, (int)ct.size(), ct.data(), 0, plain.data(), 0,
                                plain.coeffCount(), ct.data(), 0, 1, nullptr));
    }
}
void Evaluator::multiplyPlain(const Ciphertext &ct, const Plaintext &plain, Ciphertext &dest) const {
    Ciphertext t = ct;
    multiplyPlainInplace(t, plain);
    dest = std::move(t);
}

// transformToNttInplace(Plaintext, parms_id) (src/evaluator_cuda.cu:1869-1935).
void Evaluator::transformToNttInplace(Plaintext &plain, const ParmsID &id) const {
    auto d = context_.getContextData(id);
    if (!d) throw std::invalid_argument("parms_id is not valid for the current context");
    if (plain.isNttForm()) throw std::invalid_argument("plain is already in NTT form");
    if (context_.scheme() == SchemeType::ckks) throw std::logic_error("unsupported scheme");
    const int L = d->levelLimbs();
    Plaintext out((std::size_t)L * context_.polyModulusDegree());
    check(tb_plain_to_ntt(context_.handle(), L, plain.data(), 0, plain.coeffCount(), out.data(), 1, nullptr));
    out.parmsID() = id;
    out.scale() = plain.scale();
    plain = std::move(out);
}
void Evaluator::transformToNtt(const Plaintext &plain, const ParmsID &id, Plaintext &dest) const {
    Plaintext t = plain;
    transformToNttInplace(t, id);
    dest = std::move(t);
}

// transformToNttInplace / transformFromNttInplace(Ciphertext) (src/evaluator_cuda.cu:1937-2009).
void Evaluator::transformToNttInplace(Ciphertext &ct) const {
    const auto &d = data_of(context_, ct);
    if (ct.isNttForm()) throw std::invalid_argument("encrypted is already in NTT form");
    check(tb_ntt_forward(context_.handle(), ct.data(), ct.data(), ct.size(), 0, d.levelLimbs(), 0, nullptr));
    ct.isNttForm() = true;
}
void Evaluator::transformToNtt(const Ciphertext &ct, Ciphertext &dest) const {
    Ciphertext t = ct;
    transformToNttInplace(t);
    dest = std::move(t);
}
void Evaluator::transformFromNttInplace(Ciphertext &ct) const {
    const auto &d = data_of(context_, ct);
    if (!ct.isNttForm()) throw std::invalid_argument("encrypted is not in NTT form");
    check(tb_ntt_inverse(context_.handle(), ct.data(), ct.data(), ct.size(), 0, d.levelLimbs(), 0, nullptr));
    ct.isNttForm() = false;
}
void Evaluator::transformFromNtt(const Ciphertext &ct, Ciphertext &dest) const {
    Ciphertext t = ct;
    transformFromNttInplace(t);
    dest = std::move(t);
}

// applyGaloisInplace (src/evaluator_cuda.cu:2011-2104).
void Evaluator::applyGaloisInplace(Ciphertext &ct, uint32_t elt, const GaloisKeys &keys) const {
    if (keys.parmsID() != context_.keyParmsID())
        throw std::invalid_argument("galois_keys is not valid for encryption parameters");
    const auto &d = data_of(context_, ct);
    check_form(context_, ct);
    if (!keys.hasKeyElt(elt)) throw std::invalid_argument("Galois key not present");
    const uint64_t m = 2 * (uint64_t)context_.polyModulusDegree();
    if (!(elt & 1) || elt >= m) throw std::invalid_argument("Galois element is not valid");
    if (ct.size() > 2) throw std::invalid_argument("encrypted size must be 2");
    check(tb_apply_galois(context_.handle(), d.levelLimbs(), elt, ct.data(), 0, ct.data(), 0,
                          keys.key(GaloisKeys::getIndex(elt)), 1, nullptr));
}
void Evaluator::applyGalois(const Ciphertext &ct, uint32_t elt, const GaloisKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    applyGaloisInplace(t, elt, keys);
    dest = std::move(t);
}

// rotateInternal (src/evaluator_cuda.cu:2106-2163): one key, or the NAF of the step.
void Evaluator::rotateInternal(Ciphertext &ct, int steps, const GaloisKeys &keys) const {
    const auto &d = data_of(context_, ct);
    if (!d.usingBatching()) throw std::logic_error("encryption parameters do not support batching");
    if (keys.parmsID() != context_.keyParmsID())
        throw std::invalid_argument("galois_keys is not valid for encryption parameters");
    if (steps == 0) return;
    uint32_t elt = 0;
    check(tb_galois_elt_from_step(context_.handle(), steps, &elt));
    if (keys.hasKeyElt(elt)) {
        applyGaloisInplace(ct, elt, keys);
        return;
    }
    const std::vector<int> parts = naf(steps);
    if (parts.size() == 1) throw std::invalid_argument("Galois key not present");
    const int half = (int)(context_.polyModulusDegree() >> 1);
    for (int s : parts)
        if (std::abs(s) != half) rotateInternal(ct, s, keys);
}

void Evaluator::rotateRowsInplace(Ciphertext &ct, int steps, const GaloisKeys &keys) const {
    if (context_.scheme() != SchemeType::bfv && context_.scheme() != SchemeType::bgv)
        throw std::logic_error("unsupported scheme");
    rotateInternal(ct, steps, keys);
}
void Evaluator::rotateRows(const Ciphertext &ct, int steps, const GaloisKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    rotateRowsInplace(t, steps, keys);
    dest = std::move(t);
}
void Evaluator::rotateColumnsInplace(Ciphertext &ct, const GaloisKeys &keys) const {
    if (context_.scheme() != SchemeType::bfv && context_.scheme() != SchemeType::bgv)
        throw std::logic_error("unsupported scheme");
    uint32_t elt = 0;
    check(tb_galois_elt_from_step(context_.handle(), 0, &elt));
    applyGaloisInplace(ct, elt, keys);
}
void Evaluator::rotateColumns(const Ciphertext &ct, const GaloisKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    rotateColumnsInplace(t, keys);
    dest = std::move(t);
}
void Evaluator::rotateVectorInplace(Ciphertext &ct, int steps, const GaloisKeys &keys) const {
    if (context_.scheme() != SchemeType::ckks) throw std::logic_error("unsupported scheme");
    rotateInternal(ct, steps, keys);
}
void Evaluator::rotateVector(const Ciphertext &ct, int steps, const GaloisKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    rotateVectorInplace(t, steps, keys);
    dest = std::move(t);
}
void Evaluator::complexConjugateInplace(Ciphertext &ct, const GaloisKeys &keys) const {
    if (context_.scheme() != SchemeType::ckks) throw std::logic_error("unsupported scheme");
    uint32_t elt = 0;
    check(tb_galois_elt_from_step(context_.handle(), 0, &elt));
    applyGaloisInplace(ct, elt, keys);
}
void Evaluator::complexConjugate(const Ciphertext &ct, const GaloisKeys &keys, Ciphertext &dest) const {
    Ciphertext t = ct;
    complexConjugateInplace(t, keys);
    dest = std::move(t);
}

// ------------------------------------------------------------------ encoders

BatchEncoder::BatchEncoder(const SEALContext &context) : context_(context), slots_(context.polyModulusDegree()) {
    context.requireSet();
    if (context.scheme() == SchemeType::ckks) throw std::invalid_argument("unsupported scheme");
    if (!context.firstContextData()->usingBatching())
        throw std::invalid_argument("encryption parameters are not valid for batching");
}

// BatchEncoderCuda::encode (src/batchencoder_cuda.cu:42-100).
void BatchEncoder::encode(const std::vector<uint64_t> &values, Plaintext &dest) const {
    if (values.size() > slots_) throw std::invalid_argument("values_matrix size is too large");
    const uint64_t t = context_.firstContextData()->parms().plainModulus().value();
    for (uint64_t v : values)
        if (v >= t) throw std::invalid_argument("input value is larger than plain_modulus");
    DeviceBuffer slots;
    slots.fromHost(values.data(), values.size());
    Plaintext out(slots_);
    check(tb_batch_encode(context_.handle(), slots.get(), 0, values.size(), out.data(), 1, nullptr));
    dest = std::move(out);
}

void BatchEncoder::encode(const std::vector<int64_t> &values, Plaintext &dest) const {
    const uint64_t t = context_.firstContextData()->parms().plainModulus().value();
    const int64_t half = (int64_t)(t >> 1);
    std::vector<uint64_t> u(values.size());
    for (std::size_t i = 0; i < values.size(); i++) {
        const int64_t v = values[i];
        if (v > half || v < -half) throw std::invalid_argument("input value is larger than plain_modulus");
        u[i] = v < 0 ? t - (uint64_t)(-v) : (uint64_t)v;
    }
    encode(u, dest);
}

// BatchEncoderCuda::decode (src/batchencoder_cuda.cu:182-265).
void BatchEncoder::decode(const Plaintext &plain, std::vector<uint64_t> &dest) const {
    if (plain.isNttForm()) throw std::invalid_argument("plain cannot be in NTT form");
    const std::size_t n = context_.polyModulusDegree();
    if (plain.coeffCount() > n) throw std::invalid_argument("plain is not valid for encryption parameters");
    Plaintext full = plain;
    full.resize(n);
    DeviceBuffer out(n);
    check(tb_batch_decode(context_.handle(), full.data(), out.get(), 0, 1, nullptr));
    dest = out.toHost();
}

void BatchEncoder::decode(const Plaintext &plain, std::vector<int64_t> &dest) const {
    std::vector<uint64_t> u;
    decode(plain, u);
    const uint64_t t = context_.firstContextData()->parms().plainModulus().value();
    dest.resize(u.size());
    for (std::size_t i = 0; i < u.size(); i++)
        dest[i] = u[i] > (t >> 1) ? (int64_t)u[i] - (int64_t)t : (int64_t)u[i];
}

// BatchEncoderCuda::encodePolynomial (src/batchencoder_cuda.cu:124-144): the values,
// each reduced mod t, as coefficients.
void BatchEncoder::encodePolynomial(const std::vector<uint64_t> &values, Plaintext &dest) const {
    if (values.size() > slots_) throw std::invalid_argument("values_matrix size is too large");
    const uint64_t t = context_.firstContextData()->parms().plainModulus().value();
    std::vector<uint64_t> v(values.size());
    for (std::size_t i = 0; i < v.size(); i++) v[i] = values[i] % t;
    Plaintext p;
    p.fromHost(v);
    dest = std::move(p);
}

// BatchEncoderCuda::decodePolynomial (src/batchencoder_cuda.cu:267-270): N coefficients.
void BatchEncoder::decodePolynomial(const Plaintext &plain, std::vector<uint64_t> &dest) const {
    if (plain.isNttForm()) throw std::invalid_argument("plain cannot be in NTT form");
    dest = plain.toHost();
    dest.resize(slots_, 0);
}

CKKSEncoder::CKKSEncoder(const SEALContext &context) : context_(context), slots_(context.polyModulusDegree() / 2) {
    context.requireSet();
    if (context.scheme() != SchemeType::ckks) throw std::invalid_argument("unsupported scheme");
}

static int level_of(const SEALContext &c, const ParmsID &id) {
    auto d = c.getContextData(id);
    if (!d) throw std::invalid_argument("parms_id is not valid for encryption parameters");
    return d->levelLimbs();
}

// CKKSEncoderCuda::encodeInternal (src/ckks_cuda.cu:314-453).
void CKKSEncoder::encode(const std::vector<std::complex<double>> &values, const ParmsID &id, double scale,
                         Plaintext &dest) const {
    const int L = level_of(context_, id);
    if (values.size() > slots_) throw std::invalid_argument("values_size is too large");
    DeviceBuffer v;
    v.fromHost(reinterpret_cast<const uint64_t *>(values.data()), values.size() * 2);
    Plaintext out((std::size_t)L * context_.polyModulusDegree());
    check(tb_ckks_encode(context_.handle(), L, reinterpret_cast<const double *>(v.get()), 0, values.size(), scale,
                         out.data(), 1, nullptr));
    out.parmsID() = id;
    out.scale() = scale;
    dest = std::move(out);
}

void CKKSEncoder::encode(const std::vector<double> &values, double scale, Plaintext &dest) const {
    std::vector<std::complex<double>> c(values.begin(), values.end());
    encode(c, context_.firstParmsID(), scale, dest);
}

void CKKSEncoder::encode(double value, const ParmsID &id, double scale, Plaintext &dest) const {
    const int L = level_of(context_, id);
    Plaintext out((std::size_t)L * context_.polyModulusDegree());
    check(tb_ckks_encode_double(context_.handle(), L, value, scale, out.data(), nullptr));
    out.parmsID() = id;
    out.scale() = scale;
    dest = std::move(out);
}

void CKKSEncoder::encode(int64_t value, const ParmsID &id, Plaintext &dest) const {
    const int L = level_of(context_, id);
    Plaintext out((std::size_t)L * context_.polyModulusDegree());
    check(tb_ckks_encode_int64(context_.handle(), L, value, out.data(), nullptr));
    out.parmsID() = id;
    out.scale() = 1.0;
    dest = std::move(out);
}

void CKKSEncoder::encode(std::complex<double> value, const ParmsID &id, double scale, Plaintext &dest) const {
    encode(std::vector<std::complex<double>>(slots_, value), id, scale, dest);
}

void CKKSEncoder::encodePolynomial(const std::vector<double> &coeffs, const ParmsID &id, double scale,
                                   Plaintext &dest) const {
    const int L = level_of(context_, id);
    if (coeffs.size() > 2 * slots_) throw std::invalid_argument("values_size is too large");
    DeviceBuffer v;
    v.fromHost(reinterpret_cast<const uint64_t *>(coeffs.data()), coeffs.size());
    Plaintext out((std::size_t)L * context_.polyModulusDegree());
    check(tb_ckks_encode_polynomial(context_.handle(), L, reinterpret_cast<const double *>(v.get()), 0,
                                    coeffs.size(), scale, out.data(), 1, nullptr));
    out.parmsID() = id;
    out.scale() = scale;
    dest = std::move(out);
}

// CKKSEncoderCuda::decodeInternal (src/ckks_cuda.cu:900-971).
void CKKSEncoder::decode(const Plaintext &plain, std::vector<std::complex<double>> &dest) const {
    if (!plain.isNttForm()) throw std::invalid_argument("plain is not in NTT form");
    const int L = level_of(context_, plain.parmsID());
    DeviceBuffer out(2 * slots_);
    check(tb_ckks_decode(context_.handle(), L, plain.data(), plain.scale(), reinterpret_cast<double *>(out.get()), 0,
                         1, nullptr));
    auto h = out.toHost();
    dest.resize(slots_);
    std::memcpy(dest.data(), h.data(), slots_ * 16);
}

void CKKSEncoder::decodePolynomial(const Plaintext &plain, std::vector<double> &dest) const {
    if (!plain.isNttForm()) throw std::invalid_argument("plain is not in NTT form");
    const int L = level_of(context_, plain.parmsID());
    DeviceBuffer out(2 * slots_);
    check(tb_ckks_decode_polynomial(context_.handle(), L, plain.data(), plain.scale(),
                                    reinterpret_cast<double *>(out.get()), 0, 1, nullptr));
    auto h = out.toHost();
    dest.resize(2 * slots_);
    std::memcpy(dest.data(), h.data(), 2 * slots_ * 8);
}

}  // namespace troyn

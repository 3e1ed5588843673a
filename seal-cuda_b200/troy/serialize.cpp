// Byte-level save/load of the troyn:: containers in the reference's wire format:
// host-endian raw fields written one after another (savet/loadt,
// src/serialize.h:3-11), so bytes written by either library load in the other.
#include <cuda_runtime_api.h>

#include <algorithm>
#include <istream>
#include <ostream>

#include "device_util.hpp"
#include "troy_b200.hpp"

namespace troyn {
namespace {

template <class T>
void put(std::ostream &s, const T &v) {
    s.write(reinterpret_cast<const char *>(&v), sizeof(T));
}

template <class T>
T get(std::istream &s) {
    T v{};
    s.read(reinterpret_cast<char *>(&v), sizeof(T));
    if (!s) throw std::invalid_argument("unexpected end of stream");
    return v;
}

void put_words(std::ostream &s, const std::vector<uint64_t> &w) {
    put<std::size_t>(s, w.size());
    s.write(reinterpret_cast<const char *>(w.data()), (std::streamsize)(w.size() * 8));
}

std::vector<uint64_t> get_words(std::istream &s, std::size_t count) {
    std::vector<uint64_t> w(count);
    s.read(reinterpret_cast<char *>(w.data()), (std::streamsize)(count * 8));
    if (!s) throw std::invalid_argument("unexpected end of stream");
    return w;
}

// Largest degree and limb count a context describes: no valid object holds more words
// per polynomial than their product, so a corrupt length is refused before allocating.
constexpr std::size_t MAX_DEGREE = std::size_t(1) << 17;
constexpr std::size_t MAX_LIMBS = 64;
// Payload limit of a plaintext: one NTT-form polynomial over every limb at the largest degree.
constexpr std::size_t MAX_WORDS = MAX_DEGREE * MAX_LIMBS;

// A size-2 NTT-form ciphertext header and payload (scale 1, correction 1, no seed):
// how public keys and every digit of a key-switching key travel.
void save_pk_words(std::ostream &s, const ParmsID &id, std::size_t n, std::size_t limbs, const uint64_t *w) {
    put(s, id);
    put<bool>(s, true);
    put<std::size_t>(s, 2);
    put<std::size_t>(s, n);
    put<std::size_t>(s, limbs);
    put<double>(s, 1.0);
    put<std::uint64_t>(s, 1);
    put<std::uint64_t>(s, 0);
    put<bool>(s, false);
    put<std::size_t>(s, 2 * n * limbs);
    s.write(reinterpret_cast<const char *>(w), (std::streamsize)(2 * n * limbs * 8));
}

}  // namespace

void Plaintext::save(std::ostream &s) const {
    put(s, parms_id_);
    put<std::size_t>(s, count_);
    put(s, scale_);
    put_words(s, data_.toHost());
}

void Plaintext::load(std::istream &s) {
    const auto id = get<ParmsID>(s);
    const auto count = get<std::size_t>(s);
    const auto scale = get<double>(s);
    const auto words = get<std::size_t>(s);
    if (words > MAX_WORDS) throw std::invalid_argument("plaintext too large");
    auto w = get_words(s, words);
    data_.fromHost(w.data(), w.size());
    parms_id_ = id;
    count_ = count;
    scale_ = scale;
}

void Ciphertext::save(std::ostream &s) const {
    if (seed_ != 0 && size_ > 2) throw std::invalid_argument("Seed exists but size is not 2.");
    put(s, parms_id_);
    put<bool>(s, ntt_);
    put<std::size_t>(s, size_);
    put<std::size_t>(s, n_);
    put<std::size_t>(s, limbs_);
    put(s, scale_);
    put<std::uint64_t>(s, corr_);
    put<std::uint64_t>(s, seed_);
    put<bool>(s, false);       // not a termed ciphertext
    auto w = data_.toHost();
    if (seed_ != 0) w.resize(n_ * limbs_);   // c0 only: c1 is the expansion of the seed
    put_words(s, w);
}

void Ciphertext::loadHeader(std::istream &s, bool &terms, std::uint64_t &seed) {
    seed_ = 0;   // a loaded ciphertext holds both polynomials (CiphertextCuda::load)
    parms_id_ = get<ParmsID>(s);
    ntt_ = get<bool>(s);
    size_ = get<std::size_t>(s);
    n_ = get<std::size_t>(s);
    limbs_ = get<std::size_t>(s);
    scale_ = get<double>(s);
    corr_ = get<std::uint64_t>(s);
    seed = get<std::uint64_t>(s);
    terms = get<bool>(s);
    if (size_ > 64 || n_ > MAX_DEGREE || (n_ & (n_ - 1)) || limbs_ > MAX_LIMBS)
        throw std::invalid_argument("ciphertext header out of range");
}

void Ciphertext::load(std::istream &s) {
    bool terms;
    std::uint64_t seed;
    loadHeader(s, terms, seed);
    if (terms) throw std::invalid_argument("Trying to load a termed ciphertext, but indices is not specified");
    if (seed != 0) throw std::invalid_argument("seed is not zero.");
    const auto words = get<std::size_t>(s);
    if (words != size_ * n_ * limbs_) throw std::invalid_argument("ciphertext data size mismatch");
    auto w = get_words(s, words);
    data_.fromHost(w.data(), w.size());
}

// With a context, a seed-compressed ciphertext (seed != 0: only c0 on the wire) is
// expanded: c1 regenerated from the seed as the reference's GPU loader does
// (src/ciphertext_cuda.cu:137-184), inverse-transformed for BFV.
void Ciphertext::load(std::istream &s, const SEALContext &context) {
    bool terms;
    std::uint64_t seed;
    loadHeader(s, terms, seed);
    if (terms) throw std::invalid_argument("Trying to load a termed ciphertext, but indices is not specified");
    auto d = context.getContextData(parms_id_);
    if (!d || (std::size_t)d->levelLimbs() != limbs_ || context.polyModulusDegree() != n_)
        throw std::invalid_argument("ciphertext is not valid for encryption parameters");
    const auto words = get<std::size_t>(s);
    if (seed == 0) {
        if (words != size_ * n_ * limbs_) throw std::invalid_argument("ciphertext data size mismatch");
        auto w = get_words(s, words);
        data_.fromHost(w.data(), w.size());
        return;
    }
    if (size_ > 2) throw std::invalid_argument("Seed exists but size is not 2.");
    if (words != n_ * limbs_) throw std::invalid_argument("ciphertext data size mismatch");
    auto w = get_words(s, words);
    size_ = 2;
    data_.fromHost(w.data(), w.size());
    data_.resize(2 * n_ * limbs_);
    detail::tb_ok(tb_expand_seeded(context.handle(), (int)limbs_, seed, context.scheme() == SchemeType::bfv,
                                   data_.get() + n_ * limbs_, nullptr));
}

// Only the listed coefficients of c0 travel (in coefficient form), then the remaining
// polynomials in full.
void Ciphertext::saveTerms(std::ostream &s, const Evaluator &ev, const std::vector<std::size_t> &ids) const {
    std::vector<uint64_t> r;
    if (ntt_) {
        Ciphertext copy = *this;
        ev.transformFromNttInplace(copy);
        r = copy.toHost();
    } else {
        r = toHost();
    }
    put(s, parms_id_);
    put<bool>(s, ntt_);
    put<std::size_t>(s, size_);
    put<std::size_t>(s, n_);
    put<std::size_t>(s, limbs_);
    put(s, scale_);
    put<std::uint64_t>(s, corr_);
    put<std::uint64_t>(s, 0);
    put<bool>(s, true);
    for (std::size_t id : ids) {
        if (id >= n_) throw std::invalid_argument("term index out of range");
        for (std::size_t j = 0; j < limbs_; j++) put<uint64_t>(s, r[j * n_ + id]);
    }
    const std::size_t off = n_ * limbs_;
    put<std::size_t>(s, r.size() - off);
    s.write(reinterpret_cast<const char *>(r.data() + off), (std::streamsize)((r.size() - off) * 8));
}

void Ciphertext::loadTerms(std::istream &s, const Evaluator &ev, const std::vector<std::size_t> &ids) {
    bool terms;
    std::uint64_t seed;
    loadHeader(s, terms, seed);
    if (!terms) throw std::invalid_argument("Trying to load a normal ciphertext, but term indices is specified");
    if (seed != 0) throw std::invalid_argument("seed is not zero.");
    std::vector<uint64_t> host(limbs_ * n_ * size_, 0);
    for (std::size_t id : ids) {
        if (id >= n_) throw std::invalid_argument("term index out of range");
        for (std::size_t j = 0; j < limbs_; j++) host[j * n_ + id] = get<uint64_t>(s);
    }
    const std::size_t off = n_ * limbs_;
    const auto words = get<std::size_t>(s);
    if (words != host.size() - off) throw std::invalid_argument("ciphertext data size mismatch");
    auto rest = get_words(s, words);
    std::copy(rest.begin(), rest.end(), host.begin() + off);
    data_.fromHost(host.data(), host.size());
    if (ntt_) {
        ntt_ = false;
        ev.transformToNttInplace(*this);
    }
}

// The secret key travels as a plaintext of K*N words (NTT form, key parms_id).
void SecretKey::save(std::ostream &s) const {
    put(s, id_);
    put<std::size_t>(s, data_.size());
    put<double>(s, 1.0);
    put_words(s, data_.toHost());
}

void SecretKey::load(std::istream &s) {
    Plaintext p;
    p.load(s);
    id_ = p.parmsID();
    auto w = p.toHost();
    data_.fromHost(w.data(), w.size());
}

void PublicKey::save(std::ostream &s) const {
    if (!n_ || data_.size() != 2 * n_ * limbs_) throw std::logic_error("public key is empty");
    auto w = data_.toHost();
    save_pk_words(s, id_, n_, limbs_, w.data());
}

void PublicKey::load(std::istream &s) {
    Ciphertext c;
    c.load(s);
    if (c.size() != 2) throw std::invalid_argument("public key must have two polynomials");
    id_ = c.parmsID();
    n_ = c.polyModulusDegree();
    limbs_ = c.coeffModulusSize();
    auto w = c.toHost();
    data_.fromHost(w.data(), w.size());
}

void KSwitchKeys::save(std::ostream &s) const {
    put(s, id_);
    std::size_t slots = slots_;
    for (auto &kv : keys_) slots = std::max(slots, kv.first + 1);
    put<std::size_t>(s, slots);
    const std::size_t per = 2 * n_ * limbs_;
    for (std::size_t i = 0; i < slots; i++) {
        auto it = keys_.find(i);
        if (it == keys_.end()) {
            put<std::size_t>(s, 0);
            continue;
        }
        if (!per || it->second.size() % per) throw std::logic_error("key-switching key has an unexpected size");
        const std::size_t digits = it->second.size() / per;
        put<std::size_t>(s, digits);
        auto w = it->second.toHost();
        for (std::size_t j = 0; j < digits; j++) save_pk_words(s, id_, n_, limbs_, w.data() + j * per);
    }
}

void KSwitchKeys::load(std::istream &s) {
    id_ = get<ParmsID>(s);
    const auto slots = get<std::size_t>(s);
    if (slots > (std::size_t(1) << 20)) throw std::invalid_argument("too many key slots");
    keys_.clear();
    slots_ = slots;
    for (std::size_t i = 0; i < slots; i++) {
        const auto digits = get<std::size_t>(s);
        if (!digits) continue;
        if (digits > 64) throw std::invalid_argument("too many key digits");
        std::vector<uint64_t> all;
        for (std::size_t j = 0; j < digits; j++) {
            Ciphertext c;
            c.load(s);
            if (c.size() != 2) throw std::invalid_argument("key digit must have two polynomials");
            n_ = c.polyModulusDegree();
            limbs_ = c.coeffModulusSize();
            auto w = c.toHost();
            all.insert(all.end(), w.begin(), w.end());
        }
        DeviceBuffer b;
        b.fromHost(all.data(), all.size());
        keys_[i] = std::move(b);
    }
}

}  // namespace troyn

// C++ class surface of the B200 library: the troyn:: names of the reference's
// facade (src/troy_cuda.cuh:20-42) — EncryptionParameters, SEALContext, Plaintext,
// Ciphertext, keys, KeyGenerator, Encryptor, Decryptor, Evaluator, BatchEncoder,
// CKKSEncoder — implemented over the C ABI (include/troy_b200.h). Objects hold their
// data in device memory in the reference's layouts; errors surface as the
// exceptions the reference throws (std::invalid_argument / std::logic_error /
// std::runtime_error).
#pragma once

#include <array>
#include <complex>
#include <cstdint>
#include <iosfwd>
#include <limits>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "troy_b200.h"

namespace troyn {

enum class SchemeType : std::uint8_t { none = 0, bfv = 1, ckks = 2, bgv = 3 };
enum class SecurityLevel : int { none = 0, tc128 = 128, tc192 = 192, tc256 = 256 };

using ParmsID = std::array<std::uint64_t, 4>;
using PRNGSeed = std::array<std::uint64_t, 8>;
extern const ParmsID parmsIDZero;

class Evaluator;
class SEALContext;

// Device words with value semantics (deep copies), like DeviceDynamicArray.
class DeviceBuffer {
public:
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t words);
    DeviceBuffer(const DeviceBuffer &o);
    DeviceBuffer(DeviceBuffer &&o) noexcept;
    DeviceBuffer &operator=(const DeviceBuffer &o);
    DeviceBuffer &operator=(DeviceBuffer &&o) noexcept;
    ~DeviceBuffer();
    void resize(std::size_t words);     // keeps the common prefix, zero-fills the rest
    void zero();
    std::uint64_t *get() const { return p_; }
    std::size_t size() const { return n_; }
    std::vector<std::uint64_t> toHost() const;
    void fromHost(const std::uint64_t *data, std::size_t words);

private:
    std::uint64_t *p_ = nullptr;
    std::size_t n_ = 0;
};

class Modulus {
public:
    Modulus(std::uint64_t value = 0) : v_(value) {}
    std::uint64_t value() const { return v_; }
    bool isZero() const { return v_ == 0; }
    bool isPrime() const;
    int bitCount() const;
    bool operator==(const Modulus &o) const { return v_ == o.v_; }
    bool operator!=(const Modulus &o) const { return v_ != o.v_; }
    bool operator<(const Modulus &o) const { return v_ < o.v_; }
    bool operator<=(const Modulus &o) const { return v_ <= o.v_; }

private:
    std::uint64_t v_;
};

struct CoeffModulus {
    // CoeffModulus::Create (src/modulus.cpp:80-118)
    static std::vector<Modulus> Create(std::size_t poly_modulus_degree, std::vector<int> bit_sizes);
    // primes = 1 mod lcm(2n, t) (src/modulus.cpp:120-162)
    static std::vector<Modulus> Create(std::size_t poly_modulus_degree, const Modulus &plain_modulus,
                                       std::vector<int> bit_sizes);
    // CoeffModulus::MaxBitCount for the HE-standard security levels (src/modulus.h:427-440)
    static int MaxBitCount(std::size_t poly_modulus_degree, SecurityLevel sec_level = SecurityLevel::tc128);
    // CoeffModulus::BFVDefault (src/modulus.cpp:53-78): the default primes of a standard
    // degree at a security level
    static std::vector<Modulus> BFVDefault(std::size_t poly_modulus_degree,
                                           SecurityLevel sec_level = SecurityLevel::tc128);
};

struct PlainModulus {
    static Modulus Batching(std::size_t poly_modulus_degree, int bit_size);
    static std::vector<Modulus> Batching(std::size_t poly_modulus_degree, std::vector<int> bit_sizes);
};

// Factory semantics of the reference (src/randomgen.h:386-476): with a default seed
// every PRNG it creates starts the same stream; without one each is random.
class UniformRandomGeneratorFactory {
public:
    UniformRandomGeneratorFactory() = default;
    explicit UniformRandomGeneratorFactory(PRNGSeed seed) : seed_(seed), use_random_seed_(false) {}
    virtual ~UniformRandomGeneratorFactory() = default;
    bool use_random_seed() const { return use_random_seed_; }
    PRNGSeed default_seed() const { return seed_; }
    const std::uint64_t *seedPtr() const { return use_random_seed_ ? nullptr : seed_.data(); }

private:
    PRNGSeed seed_{};
    bool use_random_seed_ = true;
};

class Blake2xbPRNGFactory : public UniformRandomGeneratorFactory {
public:
    Blake2xbPRNGFactory() = default;
    explicit Blake2xbPRNGFactory(PRNGSeed seed) : UniformRandomGeneratorFactory(seed) {}
};

class EncryptionParameters {
public:
    explicit EncryptionParameters(SchemeType scheme = SchemeType::none) : scheme_(scheme) {}
    void setPolyModulusDegree(std::size_t n) { n_ = n; }
    void setCoeffModulus(const std::vector<Modulus> &m) { coeff_ = m; }
    void setPlainModulus(const Modulus &t) { t_ = t; }
    void setPlainModulus(std::uint64_t t) { t_ = Modulus(t); }
    void setRandomGenerator(std::shared_ptr<UniformRandomGeneratorFactory> g) { rng_ = std::move(g); }
    SchemeType scheme() const { return scheme_; }
    std::size_t polyModulusDegree() const { return n_; }
    const std::vector<Modulus> &coeffModulus() const { return coeff_; }
    const Modulus &plainModulus() const { return t_; }
    std::shared_ptr<UniformRandomGeneratorFactory> randomGenerator() const { return rng_; }
    ParmsID parmsID() const;

private:
    SchemeType scheme_;
    std::size_t n_ = 0;
    std::vector<Modulus> coeff_;
    Modulus t_;
    std::shared_ptr<UniformRandomGeneratorFactory> rng_;
};

// A constant with its Shoup quotient floor(operand 2^64 / q) (util::MultiplyUIntModOperand,
// src/utils/uintarithsmallmod.h:166-184).
struct MultiplyUIntModOperand {
    std::uint64_t operand = 0, quotient = 0;
};

// EncryptionParameterQualifiers (src/context.h:20-140): the validation outcome and
// properties of one level's parameters.
struct EncryptionParameterQualifiers {
    enum class ErrorType : int {
        none = -1,
        success = 0,
        invalid_scheme = 1,
        invalid_coeff_modulus_size = 2,
        invalid_coeff_modulus_bit_count = 3,
        invalid_coeff_modulus_no_ntt = 4,
        invalid_poly_modulus_degree = 5,
        invalid_poly_modulus_degree_non_power_of_two = 6,
        invalid_parameters_too_large = 7,
        invalid_parameters_insecure = 8,
        failed_creating_rns_base = 9,
        invalid_plain_modulus_bit_count = 10,
        invalid_plain_modulus_coprimality = 11,
        invalid_plain_modulus_too_large = 12,
        invalid_plain_modulus_nonzero = 13,
        failed_creating_rns_tool = 14
    };
    ErrorType parameter_error = ErrorType::none;
    bool using_fft = false, using_ntt = false, using_batching = false, using_fast_plain_lift = false,
         using_descending_modulus_chain = false;
    SecurityLevel sec_level = SecurityLevel::none;
    bool parametersSet() const { return parameter_error == ErrorType::success; }
    const char *parameterErrorName() const;
    const char *parameterErrorMessage() const;
};

class SEALContext {
public:
    // One level of the modulus chain with the host-side constants of
    // SEALContext::ContextData (src/context.h:270-460, src/context.cpp:138-425).
    class ContextData {
    public:
        const EncryptionParameters &parms() const { return parms_; }
        const ParmsID &parmsID() const { return id_; }
        std::size_t chainIndex() const { return chain_index_; }
        std::shared_ptr<const ContextData> prevContextData() const { return prev_.lock(); }
        std::shared_ptr<const ContextData> nextContextData() const { return next_; }
        int levelLimbs() const { return (int)parms_.coeffModulus().size(); }
        int totalCoeffModulusBitCount() const { return total_bits_; }
        bool usingBatching() const { return q_.using_batching; }
        EncryptionParameterQualifiers qualifiers() const { return q_; }
        // Q = prod q_i as levelLimbs() little-endian words
        const std::uint64_t *totalCoeffModulus() const { return total_.data(); }
        // BFV/BGV: floor(Q / t) mod q_i (Shoup pairs) and (Q mod t) mod q_i
        const MultiplyUIntModOperand *coeffDivPlainModulus() const { return delta_.data(); }
        const std::uint64_t *upperHalfIncrement() const { return upper_inc_.data(); }
        std::uint64_t coeffModulusModPlainModulus() const { return q_mod_t_; }
        // (t + 1) / 2 (BFV/BGV) or 2^63 (CKKS), and the matching per-limb (q_i - t, or
        // Q - t as words when some q_i <= t; CKKS: 2^63 (q_i - 2) mod q_i) increments
        std::uint64_t plainUpperHalfThreshold() const { return plain_thr_; }
        const std::uint64_t *plainUpperHalfIncrement() const { return plain_inc_.data(); }
        // CKKS: (Q + 1) / 2 as words
        const std::uint64_t *upperHalfThreshold() const { return upper_thr_.empty() ? nullptr : upper_thr_.data(); }

    private:
        friend class SEALContext;
        EncryptionParameters parms_;
        int total_bits_ = 0;
        EncryptionParameterQualifiers q_;
        std::vector<std::uint64_t> total_, upper_inc_, plain_inc_, upper_thr_;
        std::vector<MultiplyUIntModOperand> delta_;
        std::uint64_t q_mod_t_ = 0, plain_thr_ = 0;
        ParmsID id_{};
        std::size_t chain_index_ = 0;
        std::weak_ptr<const ContextData> prev_;
        std::shared_ptr<const ContextData> next_;
    };

    explicit SEALContext(EncryptionParameters parms, bool expand_mod_chain = true,
                         SecurityLevel sec_level = SecurityLevel::tc128);
    std::shared_ptr<const ContextData> getContextData(const ParmsID &id) const;
    std::shared_ptr<const ContextData> firstContextData() const { return getContextData(first_); }
    std::shared_ptr<const ContextData> lastContextData() const { return getContextData(last_); }
    std::shared_ptr<const ContextData> keyContextData() const { return getContextData(key_); }
    const ParmsID &firstParmsID() const { return first_; }
    const ParmsID &lastParmsID() const { return last_; }
    const ParmsID &keyParmsID() const { return key_; }
    bool using_keyswitching() const { return first_ != key_; }
    bool parametersSet() const { return handle_ != nullptr; }
    // Name of the first failed parameter check ("success" when valid), as
    // EncryptionParameterQualifiers::parameterErrorName (src/context.cpp:24-79).
    const std::string &parameterErrorName() const { return error_; }
    // Throws std::invalid_argument unless the parameters are set.
    void requireSet() const;
    tb_context *handle() const { return handle_.get(); }
    std::size_t polyModulusDegree() const { return n_; }
    SchemeType scheme() const { return scheme_; }
    int keyLimbs() const { return K_; }
    const EncryptionParameters &keyParms() const { return key_parms_; }

private:
    std::shared_ptr<tb_context> handle_;
    std::map<ParmsID, std::shared_ptr<ContextData>> data_;
    ParmsID key_{}, first_{}, last_{};
    std::size_t n_ = 0;
    SchemeType scheme_ = SchemeType::none;
    int K_ = 0;
    EncryptionParameters key_parms_;
    std::string error_ = "none";
};

class Plaintext {
public:
    Plaintext() = default;
    explicit Plaintext(std::size_t coeff_count) { resize(coeff_count); }
    void resize(std::size_t coeff_count);
    void setZero() { data_.zero(); }
    std::size_t coeffCount() const { return count_; }
    bool isNttForm() const { return parms_id_ != parmsIDZero; }
    ParmsID &parmsID() { return parms_id_; }
    const ParmsID &parmsID() const { return parms_id_; }
    double &scale() { return scale_; }
    double scale() const { return scale_; }
    std::uint64_t *data() { return data_.get(); }
    const std::uint64_t *data() const { return data_.get(); }
    std::vector<std::uint64_t> toHost() const { return data_.toHost(); }
    void fromHost(const std::vector<std::uint64_t> &v);
    // Wire format of PlaintextCuda::save/load (src/plaintext_cuda.cu:7-27).
    void save(std::ostream &stream) const;
    void load(std::istream &stream);
    // The hexadecimal polynomial form "7FFx^3 + 1x^1 + 3" (Plaintext::to_string and
    // operator=(string), src/plaintext.h:491-498, src/plaintext.cpp:91-215): terms in
    // strictly decreasing degree joined by " + ", a term without "x^" being degree 0.
    explicit Plaintext(const std::string &hex_poly) { *this = hex_poly; }
    Plaintext &operator=(const std::string &hex_poly);
    std::string to_string() const;
    bool isZero() const;
    std::uint64_t operator[](std::size_t i) const;
    bool operator==(const Plaintext &o) const;
    std::size_t capacity() const { return count_; }
    void reserve(std::size_t) {}
    void shrinkToFit() {}
    void release() {
        data_ = DeviceBuffer();
        count_ = 0;
        parms_id_ = {0, 0, 0, 0};
        scale_ = 1.0;
    }

private:
    DeviceBuffer data_;
    std::size_t count_ = 0;
    ParmsID parms_id_ = {0, 0, 0, 0};
    double scale_ = 1.0;
};

class Ciphertext {
public:
    Ciphertext() = default;
    explicit Ciphertext(const SEALContext &context);
    Ciphertext(const SEALContext &context, const ParmsID &parms_id, std::size_t size = 2) {
        resize(context, parms_id, size);
    }
    void resize(const SEALContext &context, const ParmsID &parms_id, std::size_t size);
    void resize(const SEALContext &context, std::size_t size) { resize(context, parms_id_, size); }
    // same degree and limb count, `size` polynomials (CiphertextCuda::resize(size_t),
    // src/ciphertext_cuda.cuh:83-88): the common prefix kept, new polynomials zero
    // true when empty or every polynomial after c0 is zero (CiphertextCuda::isTransparent)
    bool isTransparent() const;
    std::size_t sizeCapacity() const { return size_; }
    void release() {
        data_ = DeviceBuffer();
        size_ = 0;
    }
    void resize(std::size_t size) {
        if ((size < 2 && size != 0) || size > 16) throw std::invalid_argument("invalid size");
        data_.resize(size * limbs_ * n_);
        size_ = size;
        seed_ = 0;
    }
    void reserve(std::size_t) {}
    std::size_t size() const { return size_; }
    std::size_t coeffModulusSize() const { return limbs_; }
    std::size_t polyModulusDegree() const { return n_; }
    bool &isNttForm() { return ntt_; }
    bool isNttForm() const { return ntt_; }
    ParmsID &parmsID() { return parms_id_; }
    const ParmsID &parmsID() const { return parms_id_; }
    double &scale() { return scale_; }
    double scale() const { return scale_; }
    std::uint64_t &correctionFactor() { return corr_; }
    std::uint64_t correctionFactor() const { return corr_; }
    // Non-zero for a seed-compressed symmetric encryption (Encryptor::
    // encryptSymmetricSeeded): c1 is the cuRAND expansion of this seed, and save() writes
    // c0 and the seed only (CiphertextCuda::seed, src/ciphertext_cuda.cuh). Any write
    // access to the words (the non-const data() accessors, resize, fromHost) clears it,
    // as the reference's evaluator clears the seed of every ciphertext it writes.
    std::uint64_t &seed() { return seed_; }
    std::uint64_t seed() const { return seed_; }
    std::uint64_t *data() {
        seed_ = 0;
        return data_.get();
    }
    const std::uint64_t *data() const { return data_.get(); }
    std::uint64_t *data(std::size_t poly) {
        seed_ = 0;
        return data_.get() + poly * limbs_ * n_;
    }
    const std::uint64_t *data(std::size_t poly) const { return data_.get() + poly * limbs_ * n_; }
    std::vector<std::uint64_t> toHost() const { return data_.toHost(); }
    void fromHost(const std::vector<std::uint64_t> &v);
    // Wire format of CiphertextCuda::save/load/saveTerms/loadTerms
    // (src/ciphertext_cuda.cu:8-185). A ciphertext with a seed travels as c0 plus the
    // seed; loading one needs the context (the second polynomial is regenerated with
    // cuRAND as the reference's loader does).
    void save(std::ostream &stream) const;
    void load(std::istream &stream);
    void load(std::istream &stream, const SEALContext &context);
    void saveTerms(std::ostream &stream, const Evaluator &evaluator, const std::vector<std::size_t> &term_ids) const;
    void loadTerms(std::istream &stream, const Evaluator &evaluator, const std::vector<std::size_t> &term_ids);

private:
    void loadHeader(std::istream &stream, bool &terms, std::uint64_t &seed);
    DeviceBuffer data_;
    std::size_t size_ = 0, limbs_ = 0, n_ = 0;
    bool ntt_ = false;
    ParmsID parms_id_ = {0, 0, 0, 0};
    double scale_ = 1.0;
    std::uint64_t corr_ = 1;
    std::uint64_t seed_ = 0;
};

class SecretKey {
public:
    DeviceBuffer &data() { return data_; }
    const DeviceBuffer &data() const { return data_; }
    ParmsID &parmsID() { return id_; }
    const ParmsID &parmsID() const { return id_; }
    // A plaintext of K*N words on the wire (SecretKeyCuda::save, src/secretkey_cuda.cuh:292-297).
    void save(std::ostream &stream) const;
    void load(std::istream &stream);

private:
    DeviceBuffer data_;   // [K][N], NTT form
    ParmsID id_{};
};

class PublicKey {
public:
    DeviceBuffer &data() { return data_; }
    const DeviceBuffer &data() const { return data_; }
    ParmsID &parmsID() { return id_; }
    const ParmsID &parmsID() const { return id_; }
    std::size_t &polyModulusDegree() { return n_; }
    std::size_t &limbs() { return limbs_; }
    // A size-2 NTT-form ciphertext on the wire (PublicKeyCuda::save, src/publickey_cuda.cuh:252-257).
    void save(std::ostream &stream) const;
    void load(std::istream &stream);

private:
    DeviceBuffer data_;   // [2][K][N], NTT form
    std::size_t n_ = 0, limbs_ = 0;
    ParmsID id_{};
};

// One key-switching key per index, each [K-1][2][K][N] (src/kswitchkeys_cuda.cuh:43-56).
class KSwitchKeys {
public:
    std::map<std::size_t, DeviceBuffer> &data() { return keys_; }
    const std::map<std::size_t, DeviceBuffer> &data() const { return keys_; }
    ParmsID &parmsID() { return id_; }
    const ParmsID &parmsID() const { return id_; }
    std::size_t size() const { return keys_.size(); }
    bool hasKey(std::size_t index) const { return keys_.count(index) != 0; }
    const std::uint64_t *key(std::size_t index) const;
    // Number of key slots written by save (the reference's keys_ vector length:
    // 1 for relinearization keys, N for Galois keys).
    std::size_t &slotCount() { return slots_; }
    std::size_t &polyModulusDegree() { return n_; }
    std::size_t &limbs() { return limbs_; }
    // KSwitchKeysCuda::save/load (src/kswitchkeys_cuda.cuh:330-355): parms_id, slot
    // count, then per slot the number of digits and each digit as a public key.
    void save(std::ostream &stream) const;
    void load(std::istream &stream);

private:
    std::map<std::size_t, DeviceBuffer> keys_;
    std::size_t slots_ = 0, n_ = 0, limbs_ = 0;
    ParmsID id_{};
};

class RelinKeys : public KSwitchKeys {
public:
    static std::size_t getIndex(std::size_t key_power) { return key_power - 2; }
};

class GaloisKeys : public KSwitchKeys {
public:
    static std::size_t getIndex(std::uint32_t galois_elt) { return (galois_elt - 1) >> 1; }
    bool hasKeyElt(std::uint32_t galois_elt) const { return hasKey(getIndex(galois_elt)); }
};

// isScaleWithinBounds (src/evaluator_cuda.cu): log2(scale) below the plain modulus
// bits (BFV/BGV) or the level's total modulus bits (CKKS).
bool isScaleWithinBounds(double scale, const SEALContext::ContextData &context_data);

class KeyGenerator {
public:
    explicit KeyGenerator(const SEALContext &context);
    KeyGenerator(const SEALContext &context, const SecretKey &secret_key);
    const SecretKey &secretKey() const { return sk_; }
    void createPublicKey(PublicKey &destination) const;
    PublicKey createPublicKey() const {
        PublicKey pk;
        createPublicKey(pk);
        return pk;
    }
    void createRelinKeys(RelinKeys &destination) const;
    RelinKeys createRelinKeys() const {
        RelinKeys k;
        createRelinKeys(k);
        return k;
    }
    void createGaloisKeys(const std::vector<std::uint32_t> &galois_elts, GaloisKeys &destination) const;
    void createGaloisKeys(const std::vector<int> &steps, GaloisKeys &destination) const;
    void createGaloisKeys(GaloisKeys &destination) const;   // all: getEltsAll
    GaloisKeys createGaloisKeys(const std::vector<int> &steps) const {
        GaloisKeys k;
        createGaloisKeys(steps, k);
        return k;
    }
    GaloisKeys createGaloisKeys() const {
        GaloisKeys k;
        createGaloisKeys(k);
        return k;
    }
    std::uint32_t galoisEltFromStep(int step) const;
    std::vector<std::uint32_t> galoisEltsAll() const;

private:
    const SEALContext &context_;
    SecretKey sk_;
};

class Encryptor {
public:
    Encryptor(const SEALContext &context, const PublicKey &pk) : context_(context), pk_(pk), has_pk_(true) {}
    Encryptor(const SEALContext &context, const SecretKey &sk) : context_(context), sk_(sk), has_sk_(true) {}
    Encryptor(const SEALContext &context, const PublicKey &pk, const SecretKey &sk)
        : context_(context), pk_(pk), sk_(sk), has_pk_(true), has_sk_(true) {}
    void setPublicKey(const PublicKey &pk) { pk_ = pk; has_pk_ = true; }
    void setSecretKey(const SecretKey &sk) { sk_ = sk; has_sk_ = true; }
    void encrypt(const Plaintext &plain, Ciphertext &destination) const;
    void encryptZero(Ciphertext &destination) const { encryptZero(context_.firstParmsID(), destination); }
    void encryptZero(const ParmsID &parms_id, Ciphertext &destination) const;
    void encryptSymmetric(const Plaintext &plain, Ciphertext &destination) const;
    // The seed-compressed symmetric encryption of the reference's GPU path
    // (EncryptorCuda::encryptSymmetric, src/encryptor_cuda.cuh:269-371): destination.seed()
    // is set and c1 is its cuRAND expansion, so save() writes half the words. BFV and
    // CKKS (the reference's loader cannot expand a BGV one).
    void encryptSymmetricSeeded(const Plaintext &plain, Ciphertext &destination) const;
    void encryptZeroSymmetricSeeded(const ParmsID &parms_id, Ciphertext &destination) const;
    void encryptZeroSymmetric(Ciphertext &destination) const { encryptZeroSymmetric(context_.firstParmsID(), destination); }
    void encryptZeroSymmetric(const ParmsID &parms_id, Ciphertext &destination) const;

private:
    void run(const Plaintext *plain, const ParmsID &id, bool asym, Ciphertext &destination,
             bool seeded = false) const;
    const SEALContext &context_;
    PublicKey pk_;
    SecretKey sk_;
    bool has_pk_ = false, has_sk_ = false;
};

class Decryptor {
public:
    Decryptor(const SEALContext &context, const SecretKey &sk) : context_(context), sk_(sk) {}
    void decrypt(const Ciphertext &encrypted, Plaintext &destination);

private:
    const SEALContext &context_;
    SecretKey sk_;
};

class Evaluator {
public:
    explicit Evaluator(const SEALContext &context) : context_(context) {}
    void negateInplace(Ciphertext &encrypted) const;
    void negate(const Ciphertext &encrypted, Ciphertext &destination) const;
    void addInplace(Ciphertext &encrypted1, const Ciphertext &encrypted2) const;
    void add(const Ciphertext &a, const Ciphertext &b, Ciphertext &destination) const;
    void addMany(const std::vector<Ciphertext> &encrypteds, Ciphertext &destination) const;
    void subInplace(Ciphertext &encrypted1, const Ciphertext &encrypted2) const;
    void sub(const Ciphertext &a, const Ciphertext &b, Ciphertext &destination) const;
    void multiplyInplace(Ciphertext &encrypted1, const Ciphertext &encrypted2) const;
    void multiply(const Ciphertext &a, const Ciphertext &b, Ciphertext &destination) const;
    void squareInplace(Ciphertext &encrypted) const { multiplyInplace(encrypted, Ciphertext(encrypted)); }
    void square(const Ciphertext &a, Ciphertext &destination) const { multiply(a, a, destination); }
    void relinearizeInplace(Ciphertext &encrypted, const RelinKeys &relin_keys) const;
    void relinearize(const Ciphertext &encrypted, const RelinKeys &relin_keys, Ciphertext &destination) const;
    void modSwitchToNextInplace(Ciphertext &encrypted) const;
    void modSwitchToNext(const Ciphertext &encrypted, Ciphertext &destination) const;
    void modSwitchToNextInplace(Plaintext &plain) const;
    void modSwitchToNext(const Plaintext &plain, Plaintext &destination) const;
    void modSwitchToInplace(Ciphertext &encrypted, const ParmsID &parms_id) const;
    void modSwitchTo(const Ciphertext &encrypted, const ParmsID &parms_id, Ciphertext &destination) const;
    void modSwitchToInplace(Plaintext &plain, const ParmsID &parms_id) const;
    void modSwitchTo(const Plaintext &plain, const ParmsID &parms_id, Plaintext &destination) const;
    void rescaleToNextInplace(Ciphertext &encrypted) const;
    void rescaleToNext(const Ciphertext &encrypted, Ciphertext &destination) const;
    void rescaleToInplace(Ciphertext &encrypted, const ParmsID &parms_id) const;
    void rescaleTo(const Ciphertext &encrypted, const ParmsID &parms_id, Ciphertext &destination) const;
    void multiplyMany(const std::vector<Ciphertext> &encrypteds, const RelinKeys &relin_keys,
                      Ciphertext &destination) const;
    void exponentiateInplace(Ciphertext &encrypted, std::uint64_t exponent, const RelinKeys &relin_keys) const;
    void exponentiate(const Ciphertext &encrypted, std::uint64_t exponent, const RelinKeys &relin_keys,
                      Ciphertext &destination) const;
    void addPlainInplace(Ciphertext &encrypted, const Plaintext &plain) const;
    void addPlain(const Ciphertext &encrypted, const Plaintext &plain, Ciphertext &destination) const;
    void subPlainInplace(Ciphertext &encrypted, const Plaintext &plain) const;
    void subPlain(const Ciphertext &encrypted, const Plaintext &plain, Ciphertext &destination) const;
    void multiplyPlainInplace(Ciphertext &encrypted, const Plaintext &plain) const;
    void multiplyPlain(const Ciphertext &encrypted, const Plaintext &plain, Ciphertext &destination) const;
    void transformToNttInplace(Plaintext &plain, const ParmsID &parms_id) const;
    void transformToNtt(const Plaintext &plain, const ParmsID &parms_id, Plaintext &destination) const;
    void transformToNttInplace(Ciphertext &encrypted) const;
    void transformToNtt(const Ciphertext &encrypted, Ciphertext &destination) const;
    void transformFromNttInplace(Ciphertext &encrypted) const;
    void transformFromNtt(const Ciphertext &encrypted, Ciphertext &destination) const;
    void applyGaloisInplace(Ciphertext &encrypted, std::uint32_t galois_elt, const GaloisKeys &galois_keys) const;
    void applyGalois(const Ciphertext &encrypted, std::uint32_t galois_elt, const GaloisKeys &galois_keys,
                     Ciphertext &destination) const;
    void rotateRowsInplace(Ciphertext &encrypted, int steps, const GaloisKeys &galois_keys) const;
    void rotateRows(const Ciphertext &encrypted, int steps, const GaloisKeys &galois_keys,
                    Ciphertext &destination) const;
    void rotateColumnsInplace(Ciphertext &encrypted, const GaloisKeys &galois_keys) const;
    void rotateColumns(const Ciphertext &encrypted, const GaloisKeys &galois_keys, Ciphertext &destination) const;
    void rotateVectorInplace(Ciphertext &encrypted, int steps, const GaloisKeys &galois_keys) const;
    void rotateVector(const Ciphertext &encrypted, int steps, const GaloisKeys &galois_keys,
                      Ciphertext &destination) const;
    void complexConjugateInplace(Ciphertext &encrypted, const GaloisKeys &galois_keys) const;
    void complexConjugate(const Ciphertext &encrypted, const GaloisKeys &galois_keys, Ciphertext &destination) const;
    const SEALContext &context() const { return context_; }

private:
    void rotateInternal(Ciphertext &encrypted, int steps, const GaloisKeys &galois_keys) const;
    void modSwitchScaleToNext(const Ciphertext &encrypted, Ciphertext &destination) const;
    void modSwitchDropToNext(const Ciphertext &encrypted, Ciphertext &destination) const;
    const SEALContext &context_;
};

class BatchEncoder {
public:
    explicit BatchEncoder(const SEALContext &context);
    std::size_t slotCount() const { return slots_; }
    void encode(const std::vector<std::uint64_t> &values, Plaintext &destination) const;
    void encode(const std::vector<std::int64_t> &values, Plaintext &destination) const;
    void decode(const Plaintext &plain, std::vector<std::uint64_t> &destination) const;
    void decode(const Plaintext &plain, std::vector<std::int64_t> &destination) const;
    void encodePolynomial(const std::vector<std::uint64_t> &values, Plaintext &destination) const;
    void decodePolynomial(const Plaintext &plain, std::vector<std::uint64_t> &destination) const;

private:
    const SEALContext &context_;
    std::size_t slots_;
};

class CKKSEncoder {
public:
    explicit CKKSEncoder(const SEALContext &context);
    std::size_t slotCount() const { return slots_; }
    void encode(const std::vector<std::complex<double>> &values, double scale, Plaintext &destination) const {
        encode(values, context_.firstParmsID(), scale, destination);
    }
    void encode(const std::vector<std::complex<double>> &values, const ParmsID &parms_id, double scale,
                Plaintext &destination) const;
    void encode(const std::vector<double> &values, double scale, Plaintext &destination) const;
    void encode(double value, double scale, Plaintext &destination) const {
        encode(value, context_.firstParmsID(), scale, destination);
    }
    void encode(double value, const ParmsID &parms_id, double scale, Plaintext &destination) const;
    void encode(std::complex<double> value, double scale, Plaintext &destination) const {
        encode(value, context_.firstParmsID(), scale, destination);
    }
    void encode(std::complex<double> value, const ParmsID &parms_id, double scale, Plaintext &destination) const;
    void encodePolynomial(const std::vector<double> &coeffs, const ParmsID &parms_id, double scale,
                          Plaintext &destination) const;
    void encodePolynomial(const std::vector<double> &coeffs, double scale, Plaintext &destination) const {
        encodePolynomial(coeffs, context_.firstParmsID(), scale, destination);
    }
    void encode(std::int64_t value, const ParmsID &parms_id, Plaintext &destination) const;
    void encode(std::int64_t value, Plaintext &destination) const {
        encode(value, context_.firstParmsID(), destination);
    }
    void decode(const Plaintext &plain, std::vector<std::complex<double>> &destination) const;
    void decodePolynomial(const Plaintext &plain, std::vector<double> &destination) const;

private:
    const SEALContext &context_;
    std::size_t slots_;
};

// Legacy kernel-provider entry of the reference (src/kernelprovider.cuh:13-21): selects device 0.
struct KernelProvider {
    static void initialize(int device = 0);
};

// Uneven batches (no counterpart in the reference, which evaluates one ciphertext per
// call): shape groups of ciphertext pairs of different contexts through multiply ->
// relinearize -> one rotation, each group batched on a stream of its own, the whole
// fork/join replayable as one CUDA graph. An RAII owner of the C ABI's tb_uneven
// (include/troy_b200.h); group() makes a shape group from a context's handle, its
// keys and device buffers ([count][2][L][n] words each).
class UnevenBatch {
public:
    static tb_uneven_group group(const SEALContext &context, int level_limbs, std::uint64_t count,
                                 const std::uint64_t *a, const std::uint64_t *b, const std::uint64_t *relin_key,
                                 const std::uint64_t *galois_key, std::uint32_t galois_elt, std::uint64_t *out);
    explicit UnevenBatch(const std::vector<tb_uneven_group> &groups);
    ~UnevenBatch();
    UnevenBatch(const UnevenBatch &) = delete;
    UnevenBatch &operator=(const UnevenBatch &) = delete;
    void run(void *stream = nullptr);
    void runPerOp(void *stream = nullptr);
    void capture();
    void replay(void *stream = nullptr);

private:
    tb_uneven *h_ = nullptr;
};

}  // namespace troyn

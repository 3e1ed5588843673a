// C-ABI shim over the reference's own CPU implementation (troy, src/*.cpp).
//
// Test infrastructure only: compiled by oracle/Makefile against the reference
// sources where they lie, into oracle/_ref/libtroyref.so. It is used to pin the
// CPU restatement in oracle/troy_oracle.c, to generate the golden fixtures under
// tests/golden/, and as the CPU baseline that bench.py times. Nothing in the
// product links it.
//
// Every entry point drives the reference's public classes exactly as a user
// would (EncryptionParameters with a seeded Blake2xbPRNGFactory, SEALContext,
// KeyGenerator, Encryptor, Evaluator, Decryptor, BatchEncoder, CKKSEncoder), or
// one of its utility routines (NTTTables, RNSTool, GaloisTool) on caller data.

#include "troy_cpu.h"
#include "utils/ntt.h"
#include "utils/rns.h"
#include "utils/galois.h"
#include "utils/numth.h"
#include "utils/polyarithsmallmod.h"
#include "randomgen.h"
#include "utils/rlwe.h"

#include <complex>
#include <map>
#include <cstring>
#include <memory>
#include <vector>

using namespace troy;
using namespace troy::util;

namespace {

struct Session {
    std::unique_ptr<EncryptionParameters> parms;
    std::unique_ptr<SEALContext> context;
    std::unique_ptr<KeyGenerator> keygen;
    PublicKey pk;
    RelinKeys rlk;
    bool have_rlk = false;
    std::unique_ptr<Encryptor> encryptor;
    std::unique_ptr<Decryptor> decryptor;
    std::unique_ptr<Evaluator> evaluator;
    std::unique_ptr<BatchEncoder> batch;
    std::unique_ptr<CKKSEncoder> ckks;
    std::vector<Ciphertext> cts;
    std::map<uint32_t, GaloisKeys> gks;   // generated once per element
    SchemeType scheme;
};

const GaloisKeys &galois_keys_for(Session *s, uint32_t elt) {
    auto it = s->gks.find(elt);
    if (it == s->gks.end())
        it = s->gks.emplace(elt, s->keygen->createGaloisKeys(std::vector<uint32_t>{elt})).first;
    return it->second;
}

int add_ct(Session *s, Ciphertext &&c) {
    s->cts.push_back(std::move(c));
    return (int)s->cts.size() - 1;
}

}  // namespace

extern "C" {

// ---------------------------------------------------------------- primitives

int ref_ntt_tables(int logn, uint64_t q, uint64_t *root_op, uint64_t *root_quo, uint64_t *inv_op,
                   uint64_t *inv_quo, uint64_t *inv_n) {
    try {
        NTTTables t(logn, Modulus(q));
        size_t n = size_t(1) << logn;
        for (size_t i = 0; i < n; i++) {
            root_op[i] = t.getFromRootPowers()[i].operand;
            root_quo[i] = t.getFromRootPowers()[i].quotient;
            inv_op[i] = t.getFromInvRootPowers()[i].operand;
            inv_quo[i] = t.getFromInvRootPowers()[i].quotient;
        }
        inv_n[0] = t.invDegreeModulo().operand;
        inv_n[1] = t.invDegreeModulo().quotient;
        inv_n[2] = t.getRoot();
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_ntt_forward(int logn, uint64_t q, uint64_t *data, int lazy) {
    try {
        NTTTables t(logn, Modulus(q));
        if (lazy) nttNegacyclicHarveyLazy(HostPointer<uint64_t>(data), t);
        else nttNegacyclicHarvey(HostPointer<uint64_t>(data), t);
        return 0;
    } catch (...) {
        return -1;
    }
}

int ref_ntt_inverse(int logn, uint64_t q, uint64_t *data, int lazy) {
    try {
        NTTTables t(logn, Modulus(q));
        if (lazy) inverseNttNegacyclicHarveyLazy(HostPointer<uint64_t>(data), t);
        else inverseNttNegacyclicHarvey(HostPointer<uint64_t>(data), t);
        return 0;
    } catch (...) {
        return -1;
    }
}

void ref_dyadic_product(uint64_t q, const uint64_t *a, const uint64_t *b, uint64_t *out, size_t n) {
    dyadicProductCoeffmod(ConstHostPointer<uint64_t>(a), ConstHostPointer<uint64_t>(b), n, Modulus(q),
                          HostPointer<uint64_t>(out));
}

int ref_coeff_modulus_create(size_t n, const int *bits, int count, uint64_t *out) {
    try {
        std::vector<int> b(bits, bits + count);
        auto mods = CoeffModulus::Create(n, b);
        for (int i = 0; i < count; i++) out[i] = mods[i].value();
        return 0;
    } catch (...) {
        return -1;
    }
}

// EncryptionParameters::parmsID of (scheme, n, moduli, t).
int ref_parms_id(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t, uint64_t *out4) {
    try {
        EncryptionParameters p(static_cast<SchemeType>(scheme));
        p.setPolyModulusDegree(n);
        std::vector<Modulus> q;
        for (int i = 0; i < count; i++) q.emplace_back(moduli[i]);
        p.setCoeffModulus(q);
        if (t) p.setPlainModulus(t);
        const auto &id = p.parmsID();
        for (int i = 0; i < 4; i++) out4[i] = id[i];
        return 0;
    } catch (...) {
        return 1;
    }
}

// CoeffModulus::BFVDefault (src/modulus.cpp:53-78): the default primes of a degree and
// security level (1 tc128, 2 tc192, 3 tc256); returns the count, -1 on error.
int ref_bfv_default(size_t n, int sec, uint64_t *out, int cap) {
    try {
        auto v = CoeffModulus::BFVDefault(n, (SecurityLevel)sec);
        if ((int)v.size() > cap) return -1;
        for (size_t i = 0; i < v.size(); i++) out[i] = v[i].value();
        return (int)v.size();
    } catch (...) {
        return -1;
    }
}

// The first data level's qualifiers and precomputed constants
// (SEALContext::ContextData, src/context.h): out = [error, using_fft, using_ntt,
// using_batching, using_fast_plain_lift, using_descending_modulus_chain, sec_level,
// q_mod_t, plain_threshold, then L words each of: total modulus, delta operands,
// delta quotients, upper-half increment, plain upper-half increment, upper-half
// threshold]; returns L, or -1.
int ref_context_consts(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t, int sec, uint64_t *out) {
    try {
        EncryptionParameters parms((SchemeType)scheme);
        parms.setPolyModulusDegree(n);
        std::vector<Modulus> mods;
        for (int i = 0; i < count; i++) mods.emplace_back(moduli[i]);
        parms.setCoeffModulus(mods);
        if (scheme != 2) parms.setPlainModulus(Modulus(t));
        SEALContext context(parms, true, (SecurityLevel)sec);
        auto d = context.firstContextData();
        const auto q = d->qualifiers();
        const size_t L = d->parms().coeffModulus().size();
        size_t k = 0;
        out[k++] = (uint64_t)(int64_t)q.parameter_error;
        out[k++] = q.using_fft;
        out[k++] = q.using_ntt;
        out[k++] = q.using_batching;
        out[k++] = q.using_fast_plain_lift;
        out[k++] = q.using_descending_modulus_chain;
        out[k++] = (uint64_t)(int)q.sec_level;
        const bool ok = q.parametersSet();
        const bool ckks = scheme == 2;
        out[k++] = ok && !ckks ? d->coeffModulusModPlainModulus() : 0;
        out[k++] = ok ? d->plainUpperHalfThreshold() : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok ? d->totalCoeffModulus()[i] : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok && !ckks ? d->coeffDivPlainModulus()[i].operand : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok && !ckks ? d->coeffDivPlainModulus()[i].quotient : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok && !ckks ? d->upperHalfIncrement()[i] : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok ? d->plainUpperHalfIncrement()[i] : 0;
        for (size_t i = 0; i < L; i++) out[k++] = ok && ckks ? d->upperHalfThreshold()[i] : 0;
        return (int)L;
    } catch (...) {
        return -1;
    }
}

// Plaintext(hex_poly) and to_string of the reference (src/plaintext.cpp:91-215): the
// parsed coefficients (count returned; -1 when the string is rejected) and the
// string printed back.
int ref_plain_hex(const char *hex, uint64_t *coeffs, size_t cap, char *out, size_t outcap) {
    try {
        Plaintext p{std::string(hex)};
        if (p.coeffCount() > cap) return -2;
        for (size_t i = 0; i < p.coeffCount(); i++) coeffs[i] = p[i];
        const std::string s = p.to_string();
        if (s.size() + 1 > outcap) return -2;
        std::memcpy(out, s.c_str(), s.size() + 1);
        return (int)p.coeffCount();
    } catch (...) {
        return -1;
    }
}

int ref_plain_modulus_batching(size_t n, int bits, uint64_t *out) {
    try {
        *out = PlainModulus::Batching(n, bits).value();
        return 0;
    } catch (...) {
        return -1;
    }
}

// Bytes [offset, offset + count) of the Blake2xb stream a PRNG with this seed emits.
void ref_prng_bytes(const uint64_t *seed8, size_t offset, size_t count, uint8_t *out) {
    PRNGSeed seed;
    std::copy_n(seed8, 8, seed.begin());
    Blake2xbPRNGFactory factory(seed);
    auto prng = factory.create();
    std::vector<std::byte> skip(offset);
    if (offset) prng->generate(offset, skip.data());
    prng->generate(count, reinterpret_cast<std::byte *>(out));
}

// Samplers over a modulus list, from a fresh PRNG with the given seed.
// kind: 0 ternary, 1 cbd, 2 uniform. Output [count][n] like the reference.
int ref_sample(int kind, const uint64_t *seed8, size_t n, const uint64_t *moduli, int count, uint64_t *out) {
    try {
        PRNGSeed seed;
        std::copy_n(seed8, 8, seed.begin());
        EncryptionParameters parms(SchemeType::ckks);
        parms.setPolyModulusDegree(n);
        std::vector<Modulus> mods;
        for (int i = 0; i < count; i++) mods.emplace_back(moduli[i]);
        parms.setCoeffModulus(mods);
        auto factory = std::make_shared<Blake2xbPRNGFactory>(seed);
        auto prng = factory->create();
        if (kind == 0) samplePolyTernary(prng, parms, out);
        else if (kind == 1) samplePolyCbd(prng, parms, out);
        else samplePolyUniform(prng, parms, out);
        return 0;
    } catch (...) {
        return -1;
    }
}

// RNSTool routines on caller data. q has `count` moduli, t the plain modulus (0 for none).
// op: 0 fastbconvmTilde (in q -> out Bsk U {m~}), 1 smMrq (in Bsk U {m~} -> out Bsk),
//     2 fastFloor (in q U Bsk -> out Bsk), 3 fastbconvSk (in Bsk -> out q),
//     4 divideAndRoundqLastInplace (in/out q), 5 divideAndRoundqLastNttInplace (in/out q),
//     6 decryptScaleAndRound (in q -> out t), 7 modTAndDivideqLastInplace (in/out q),
//     8 decryptModt (in q -> out t)
int ref_rns_op(int op, size_t n, const uint64_t *q, int count, uint64_t t, const uint64_t *in, uint64_t *out) {
    try {
        std::vector<Modulus> mods;
        for (int i = 0; i < count; i++) mods.emplace_back(q[i]);
        RNSBase base(mods);
        RNSTool tool(n, base, Modulus(t));
        size_t L = count;
        size_t bsk = tool.baseBsk()->size();
        std::vector<uint64_t> buf;
        switch (op) {
        case 0: tool.fastbconvmTilde(in, out); break;
        case 1: tool.smMrq(in, out); break;
        case 2: tool.fastFloor(in, out); break;
        case 3: tool.fastbconvSk(in, out); break;
        case 4:
            std::memcpy(out, in, sizeof(uint64_t) * n * L);
            tool.divideAndRoundqLastInplace(out);
            break;
        case 5: {
            std::memcpy(out, in, sizeof(uint64_t) * n * L);
            auto tables = CreateNTTTables(getPowerOfTwo(n), mods);
            tool.divideAndRoundqLastNttInplace(out, tables.get());
            break;
        }
        case 6: tool.decryptScaleAndRound(in, out); break;
        case 7:
            std::memcpy(out, in, sizeof(uint64_t) * n * L);
            tool.modTAndDivideqLastInplace(out);
            break;
        case 8: tool.decryptModt(in, out); break;
        default: return -2;
        }
        (void)bsk;
        return 0;
    } catch (...) {
        return -1;
    }
}

// Bsk base of the RNS tool: writes m_sk, gamma, then the Bsk moduli; returns Bsk size.
int ref_rns_bases(size_t n, const uint64_t *q, int count, uint64_t t, uint64_t *out) {
    try {
        std::vector<Modulus> mods;
        for (int i = 0; i < count; i++) mods.emplace_back(q[i]);
        RNSBase base(mods);
        RNSTool tool(n, base, Modulus(t));
        out[0] = tool.msk().value();
        out[1] = tool.gamma().value();
        size_t bsk = tool.baseBsk()->size();
        for (size_t i = 0; i < bsk; i++) out[2 + i] = (*tool.baseBsk())[i].value();
        return (int)bsk;
    } catch (...) {
        return -1;
    }
}

uint32_t ref_galois_elt_from_step(int logn, int step) {
    GaloisTool tool(logn);
    return tool.getEltFromStep(step);
}

void ref_apply_galois(int logn, uint32_t elt, uint64_t q, const uint64_t *in, uint64_t *out) {
    GaloisTool tool(logn);
    tool.applyGalois(ConstHostPointer<uint64_t>(in), elt, Modulus(q), HostPointer<uint64_t>(out));
}

void ref_apply_galois_ntt(int logn, uint32_t elt, const uint64_t *in, uint64_t *out) {
    GaloisTool tool(logn);
    tool.applyGaloisNtt(ConstHostPointer<uint64_t>(in), elt, HostPointer<uint64_t>(out));
}

// ------------------------------------------------------------------ sessions

// scheme: 1 bfv, 2 ckks, 3 bgv. moduli: the full key-level chain (special prime last).
void *ref_session_new(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t, const uint64_t *seed8) {
    try {
        auto *s = new Session();
        s->scheme = (SchemeType)scheme;
        s->parms.reset(new EncryptionParameters((SchemeType)scheme));
        s->parms->setPolyModulusDegree(n);
        std::vector<Modulus> mods;
        for (int i = 0; i < count; i++) mods.emplace_back(moduli[i]);
        s->parms->setCoeffModulus(mods);
        if (scheme != 2) s->parms->setPlainModulus(Modulus(t));
        PRNGSeed seed;
        std::copy_n(seed8, 8, seed.begin());
        s->parms->setRandomGenerator(std::make_shared<Blake2xbPRNGFactory>(seed));
        s->context.reset(new SEALContext(*s->parms, true, SecurityLevel::none));
        s->keygen.reset(new KeyGenerator(*s->context));
        s->keygen->createPublicKey(s->pk);
        s->encryptor.reset(new Encryptor(*s->context, s->pk, s->keygen->secretKey()));
        s->decryptor.reset(new Decryptor(*s->context, s->keygen->secretKey()));
        s->evaluator.reset(new Evaluator(*s->context));
        if (scheme == 2) s->ckks.reset(new CKKSEncoder(*s->context));
        else s->batch.reset(new BatchEncoder(*s->context));
        return s;
    } catch (...) {
        return nullptr;
    }
}

void ref_session_free(void *h) { delete static_cast<Session *>(h); }

size_t ref_secret_key(void *h, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    auto &d = s->keygen->secretKey().data();
    if (out) std::memcpy(out, d.data(), d.dynArray().size() * 8);
    return d.dynArray().size();
}

size_t ref_public_key(void *h, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    auto &d = s->pk.data();
    size_t words = d.dynArray().size();
    if (out) std::memcpy(out, d.data(), words * 8);
    return words;
}

static size_t dump_kswitch(const KSwitchKeys &k, size_t index, uint64_t *out) {
    size_t words = 0;
    for (auto &pk : k.data()[index]) {
        size_t w = pk.data().dynArray().size();
        if (out) std::memcpy(out + words, pk.data().data(), w * 8);
        words += w;
    }
    return words;
}

size_t ref_relin_key(void *h, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    if (!s->have_rlk) {
        s->rlk = s->keygen->createRelinKeys();
        s->have_rlk = true;
    }
    return dump_kswitch(s->rlk, RelinKeys::getIndex(2), out);
}

size_t ref_galois_key(void *h, uint32_t elt, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    return dump_kswitch(galois_keys_for(s, elt), GaloisKeys::getIndex(elt), out);
}

// Drops a stored ciphertext's data (keeps ids stable) so long timing loops stay bounded.
void ref_ct_free(void *h, int id) {
    auto *s = static_cast<Session *>(h);
    if (id >= 0 && id < (int)s->cts.size()) s->cts[id] = Ciphertext();
}

int ref_ct_encrypt_slots(void *h, const uint64_t *slots, size_t count) {
    auto *s = static_cast<Session *>(h);
    try {
        std::vector<uint64_t> v(slots, slots + count);
        Plaintext p;
        s->batch->encode(v, p);
        Ciphertext c;
        s->encryptor->encrypt(p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_encode_slots(void *h, const uint64_t *slots, size_t count, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    std::vector<uint64_t> v(slots, slots + count);
    Plaintext p;
    s->batch->encode(v, p);
    std::memcpy(out, p.data(), p.coeffCount() * 8);
    return (int)p.coeffCount();
}

int ref_ct_encrypt_ckks(void *h, const double *re, const double *im, size_t count, double scale) {
    auto *s = static_cast<Session *>(h);
    try {
        std::vector<std::complex<double>> v(count);
        for (size_t i = 0; i < count; i++) v[i] = {re[i], im[i]};
        Plaintext p;
        s->ckks->encode(v, scale, p);
        Ciphertext c;
        s->encryptor->encrypt(p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// Encoded CKKS plaintext words (NTT form, first level); returns word count.
int ref_encode_ckks(void *h, const double *re, const double *im, size_t count, double scale, uint64_t *out) {
    auto *s = static_cast<Session *>(h);
    std::vector<std::complex<double>> v(count);
    for (size_t i = 0; i < count; i++) v[i] = {re[i], im[i]};
    Plaintext p;
    s->ckks->encode(v, scale, p);
    std::memcpy(out, p.data(), p.coeffCount() * 8);
    return (int)p.coeffCount();
}

// info: [0] size, [1] coeff_modulus_size, [2] is_ntt, [3] correction factor; scale in *scale.
size_t ref_ct_get(void *h, int id, uint64_t *out, uint64_t *info, double *scale) {
    auto *s = static_cast<Session *>(h);
    auto &c = s->cts.at(id);
    size_t words = c.size() * c.coeffModulusSize() * c.polyModulusDegree();
    if (out) std::memcpy(out, c.data(), words * 8);
    if (info) {
        info[0] = c.size();
        info[1] = c.coeffModulusSize();
        info[2] = c.isNttForm();
        info[3] = c.correctionFactor();
    }
    if (scale) *scale = c.scale();
    return words;
}

int ref_ct_multiply(void *h, int a, int b) {
    auto *s = static_cast<Session *>(h);
    try {
        Ciphertext c;
        s->evaluator->multiply(s->cts.at(a), s->cts.at(b), c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_ct_relinearize(void *h, int a) {
    auto *s = static_cast<Session *>(h);
    try {
        if (!s->have_rlk) {
            s->rlk = s->keygen->createRelinKeys();
            s->have_rlk = true;
        }
        Ciphertext c;
        s->evaluator->relinearize(s->cts.at(a), s->rlk, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// kind: 0 rotate_rows, 1 rotate_columns, 2 rotate_vector
int ref_ct_rotate(void *h, int a, int kind, int step) {
    auto *s = static_cast<Session *>(h);
    try {
        auto tool = s->context->keyContextData()->galoisTool();
        uint32_t elt = kind == 1 ? tool->getEltFromStep(0) : tool->getEltFromStep(step);
        const GaloisKeys &gk = galois_keys_for(s, elt);
        Ciphertext c;
        if (kind == 0) s->evaluator->rotateRows(s->cts.at(a), step, gk, c);
        else if (kind == 1) s->evaluator->rotateColumns(s->cts.at(a), gk, c);
        else s->evaluator->rotateVector(s->cts.at(a), step, gk, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_ct_rescale(void *h, int a) {
    auto *s = static_cast<Session *>(h);
    try {
        Ciphertext c;
        s->evaluator->rescaleToNext(s->cts.at(a), c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_ct_mod_switch(void *h, int a) {
    auto *s = static_cast<Session *>(h);
    try {
        Ciphertext c;
        s->evaluator->modSwitchToNext(s->cts.at(a), c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_ct_multiply_plain_slots(void *h, int a, const uint64_t *slots, size_t count) {
    auto *s = static_cast<Session *>(h);
    try {
        std::vector<uint64_t> v(slots, slots + count);
        Plaintext p;
        s->batch->encode(v, p);
        Ciphertext c;
        s->evaluator->multiplyPlain(s->cts.at(a), p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// The coefficient encoding of BatchEncoderCuda::encodePolynomial
// (src/batchencoder_cuda.cu:124-144): count coefficients, each reduced mod t.
static Plaintext poly_plain(Session *s, const uint64_t *coeffs, size_t count) {
    const uint64_t t = s->parms->plainModulus().value();
    Plaintext p(count);
    for (size_t i = 0; i < count; i++) p.data()[i] = coeffs[i] % t;
    return p;
}

// Encrypts BatchEncoder::encodePolynomial(coeffs) (coefficient encoding) with the
// public key, or with the secret key (encryptSymmetric) when symmetric is non-zero.
int ref_ct_encrypt_poly(void *h, const uint64_t *coeffs, size_t count, int symmetric) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p = poly_plain(s, coeffs, count);
        Ciphertext c;
        if (symmetric)
            s->encryptor->encryptSymmetric(p, c);
        else
            s->encryptor->encrypt(p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// Evaluator::multiplyPlain by encodePolynomial(coeffs).
int ref_ct_multiply_plain_poly(void *h, int a, const uint64_t *coeffs, size_t count) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p = poly_plain(s, coeffs, count);
        Ciphertext c;
        s->evaluator->multiplyPlain(s->cts.at(a), p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// A plaintext given as words at parms_id (NTT-form CKKS plaintexts carry L*N words).
static Plaintext words_plain(Session *s, const ParmsID &id, const uint64_t *words, size_t count, double scale) {
    Plaintext p;
    p.resize(count);
    std::memcpy(p.data(), words, count * 8);
    if (s->scheme == SchemeType::ckks) p.parmsID() = id;
    p.scale() = scale;
    return p;
}

// A ciphertext given as words: `size` polynomials at the level with `limbs` primes.
int ref_ct_from_words(void *h, const uint64_t *words, size_t size, size_t limbs, int is_ntt, double scale,
                      uint64_t corr) {
    auto *s = static_cast<Session *>(h);
    try {
        auto cd = s->context->firstContextData();
        while (cd && cd->parms().coeffModulus().size() != limbs) cd = cd->nextContextData();
        if (!cd) return -1;
        Ciphertext c;
        c.resize(*s->context, cd->parmsID(), size);
        std::memcpy(c.data(), words, size * limbs * s->parms->polyModulusDegree() * 8);
        c.isNttForm() = is_ntt != 0;
        c.scale() = scale;
        c.correctionFactor() = corr;
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// Encrypts a plaintext given as words at the first level.
int ref_ct_encrypt_plain_words(void *h, const uint64_t *words, size_t count, double scale, int symmetric) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p = words_plain(s, s->context->firstParmsID(), words, count, scale);
        Ciphertext c;
        if (symmetric)
            s->encryptor->encryptSymmetric(p, c);
        else
            s->encryptor->encrypt(p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// Evaluator::multiplyPlain by a plaintext given as words at the ciphertext's level.
int ref_ct_multiply_plain_words(void *h, int a, const uint64_t *words, size_t count, double scale) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p = words_plain(s, s->cts.at(a).parmsID(), words, count, scale);
        Ciphertext c;
        s->evaluator->multiplyPlain(s->cts.at(a), p, c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

int ref_ct_add(void *h, int a, int b) {
    auto *s = static_cast<Session *>(h);
    try {
        Ciphertext c;
        s->evaluator->add(s->cts.at(a), s->cts.at(b), c);
        return add_ct(s, std::move(c));
    } catch (...) {
        return -1;
    }
}

// BFV/BGV decrypt + batch decode into `count` slots.
int ref_ct_decrypt_slots(void *h, int a, uint64_t *out, size_t count) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p;
        s->decryptor->decrypt(s->cts.at(a), p);
        std::vector<uint64_t> v;
        s->batch->decode(p, v);
        std::memcpy(out, v.data(), std::min(count, v.size()) * 8);
        return 0;
    } catch (...) {
        return -1;
    }
}

// CKKS decrypt + decode into `count` complex slots.
int ref_ct_decrypt_ckks(void *h, int a, double *re, double *im, size_t count) {
    auto *s = static_cast<Session *>(h);
    try {
        Plaintext p;
        s->decryptor->decrypt(s->cts.at(a), p);
        std::vector<std::complex<double>> v;
        s->ckks->decode(p, v);
        for (size_t i = 0; i < count && i < v.size(); i++) {
            re[i] = v[i].real();
            im[i] = v[i].imag();
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

}  // extern "C"

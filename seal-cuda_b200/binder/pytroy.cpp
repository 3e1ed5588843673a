// Python module `pytroy`: the reference's binding surface (binder/binder.cu:144-700)
// over the troyn:: classes of this library. Names, overload order and argument
// conventions follow the reference so that its Python callers run unchanged,
// including two overloads whose behaviour differs from their names: the second
// transform_to_ntt(Ciphertext) lambda (it calls transformFromNtt, binder.cu:664) is
// registered after the regular one and so is never reached, and
// rotate_rows(cipher, galois_keys) rotates the columns (binder.cu:682).
#include <pybind11/complex.h>
#include <pybind11/eval.h>
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <sstream>

#include "linear_ckks.hpp"
#include "serving.hpp"
#include "troy_b200.hpp"

namespace py = pybind11;
using namespace troyn;
using std::complex;
using std::vector;

// ParmsID (std::array<uint64_t, 4>) crosses as pytroy.ParmsID, a list of the four
// words with the reference binder's vec() (binder/binder.cu:186-194; there vec()
// returns an empty list, here the words); any four-int sequence converts back.
namespace pybind11 {
namespace detail {
template <>
struct type_caster<troyn::ParmsID> {
    PYBIND11_TYPE_CASTER(troyn::ParmsID, const_name("ParmsID"));
    bool load(handle src, bool) {
        if (!isinstance<sequence>(src) || isinstance<str>(src) || isinstance<bytes>(src)) return false;
        auto seq = reinterpret_borrow<sequence>(src);
        if (seq.size() != 4) return false;
        for (size_t i = 0; i < 4; i++) {
            make_caster<std::uint64_t> c;
            if (!c.load(seq[i], true)) return false;
            value[i] = cast_op<std::uint64_t>(c);
        }
        return true;
    }
    static handle cast(const troyn::ParmsID &v, return_value_policy, handle) {
        list words;
        for (auto x : v) words.append(int_(x));
        return module_::import("pytroy").attr("ParmsID")(words).release();
    }
};
}  // namespace detail
}  // namespace pybind11

namespace {

template <class T>
vector<T> from_array(const py::array_t<T, py::array::c_style | py::array::forcecast> &a) {
    py::buffer_info b = a.request();
    const T *p = static_cast<const T *>(b.ptr);
    return vector<T>(p, p + (b.ndim ? b.shape[0] : 1));
}

template <class T>
py::array_t<T> to_array(const vector<T> &v) {
    py::array_t<T> a(v.size());
    std::copy(v.begin(), v.end(), static_cast<T *>(a.request().ptr));
    return a;
}

using U64Array = py::array_t<uint64_t, py::array::c_style | py::array::forcecast>;

// every element of an array of any shape, row-major
vector<uint64_t> flat_u64(const U64Array &a) { return vector<uint64_t>(a.data(), a.data() + a.size()); }
vector<double> flat_f64(const py::array_t<double, py::array::c_style | py::array::forcecast> &a) {
    return vector<double>(a.data(), a.data() + a.size());
}
using I64Array = py::array_t<int64_t, py::array::c_style | py::array::forcecast>;
using F64Array = py::array_t<double, py::array::c_style | py::array::forcecast>;
using C128Array = py::array_t<complex<double>, py::array::c_style | py::array::forcecast>;
using SizeArray = py::array_t<std::size_t, py::array::c_style | py::array::forcecast>;

// save() -> bytes and load(bytes), as the reference's SAVE_MACRO / LOAD_MACRO.
template <class T>
py::bytes save_bytes(const T &obj) {
    std::ostringstream s;
    obj.save(s);
    return py::bytes(s.str());
}
template <class T>
void load_bytes(T &obj, const py::bytes &b) {
    std::istringstream s{std::string(b)};
    obj.load(s);
}

}  // namespace

PYBIND11_MODULE(pytroy, m) {
    m.doc() = "B200 homomorphic-encryption library (troy-compatible Python surface)";
    m.def("initialize_kernel", []() { KernelProvider::initialize(); });

    py::enum_<SchemeType>(m, "SchemeType")
        .value("none", SchemeType::none)
        .value("bfv", SchemeType::bfv)
        .value("bgv", SchemeType::bgv)
        .value("ckks", SchemeType::ckks);
    py::enum_<SecurityLevel>(m, "SecurityLevel")
        .value("none", SecurityLevel::none)
        .value("tc128", SecurityLevel::tc128)
        .value("tc192", SecurityLevel::tc192)
        .value("tc256", SecurityLevel::tc256);

    py::class_<Modulus>(m, "Modulus")
        .def(py::init<uint64_t>())
        .def("is_prime", &Modulus::isPrime)
        .def("value", &Modulus::value);
    py::class_<CoeffModulus>(m, "CoeffModulus")
        .def_static("max_bit_count", &CoeffModulus::MaxBitCount, py::arg("poly_modulus_degree"),
                    py::arg("sec_level") = SecurityLevel::tc128)
        .def_static("bfv_default", &CoeffModulus::BFVDefault, py::arg("poly_modulus_degree"),
                    py::arg("sec_level") = SecurityLevel::tc128)
        .def_static("create", py::overload_cast<std::size_t, vector<int>>(&CoeffModulus::Create))
        .def_static("create", py::overload_cast<std::size_t, const Modulus &, vector<int>>(&CoeffModulus::Create));
    py::class_<PlainModulus>(m, "PlainModulus")
        .def_static("batching", py::overload_cast<std::size_t, int>(&PlainModulus::Batching))
        .def_static("batching", py::overload_cast<std::size_t, vector<int>>(&PlainModulus::Batching));

    // pytroy.ParmsID: the parms_id words as a list, with vec() (see the caster above).
    py::exec(R"(
class ParmsID(list):
    """A parms_id: the four 64-bit words of its BLAKE2b hash."""

    def vec(self):
        return list(self)
)",
             m.attr("__dict__"));

    py::class_<Blake2xbPRNGFactory, std::shared_ptr<Blake2xbPRNGFactory>>(m, "Blake2xbPRNGFactory")
        .def(py::init<>())
        .def(py::init([](const vector<uint64_t> &seed) {
            if (seed.size() != 8) throw std::invalid_argument("seed must have 8 words");
            PRNGSeed s;
            std::copy(seed.begin(), seed.end(), s.begin());
            return std::make_shared<Blake2xbPRNGFactory>(s);
        }));

    py::class_<EncryptionParameters>(m, "EncryptionParameters")
        .def(py::init<SchemeType>())
        .def("set_poly_modulus_degree", &EncryptionParameters::setPolyModulusDegree)
        .def("set_coeff_modulus", &EncryptionParameters::setCoeffModulus)
        .def("set_plain_modulus", py::overload_cast<std::uint64_t>(&EncryptionParameters::setPlainModulus))
        .def("set_plain_modulus", py::overload_cast<const Modulus &>(&EncryptionParameters::setPlainModulus))
        .def("set_random_generator",
             [](EncryptionParameters &self, std::shared_ptr<Blake2xbPRNGFactory> g) { self.setRandomGenerator(g); })
        .def("scheme", &EncryptionParameters::scheme)
        .def("poly_modulus_degree", &EncryptionParameters::polyModulusDegree)
        .def("coeff_modulus",
             [](const EncryptionParameters &self) {
                 vector<uint64_t> v;
                 for (auto &q : self.coeffModulus()) v.push_back(q.value());
                 return v;
             })
        .def("parms_id", &EncryptionParameters::parmsID);

    using CD = SEALContext::ContextData;
    auto cd = [](std::shared_ptr<const CD> p) { return std::const_pointer_cast<CD>(p); };
    using Q = EncryptionParameterQualifiers;
    py::enum_<Q::ErrorType>(m, "ErrorType")
        .value("none", Q::ErrorType::none)
        .value("success", Q::ErrorType::success)
        .value("invalid_scheme", Q::ErrorType::invalid_scheme)
        .value("invalid_coeff_modulus_size", Q::ErrorType::invalid_coeff_modulus_size)
        .value("invalid_coeff_modulus_bit_count", Q::ErrorType::invalid_coeff_modulus_bit_count)
        .value("invalid_coeff_modulus_no_ntt", Q::ErrorType::invalid_coeff_modulus_no_ntt)
        .value("invalid_poly_modulus_degree", Q::ErrorType::invalid_poly_modulus_degree)
        .value("invalid_poly_modulus_degree_non_power_of_two", Q::ErrorType::invalid_poly_modulus_degree_non_power_of_two)
        .value("invalid_parameters_too_large", Q::ErrorType::invalid_parameters_too_large)
        .value("invalid_parameters_insecure", Q::ErrorType::invalid_parameters_insecure)
        .value("failed_creating_rns_base", Q::ErrorType::failed_creating_rns_base)
        .value("invalid_plain_modulus_bit_count", Q::ErrorType::invalid_plain_modulus_bit_count)
        .value("invalid_plain_modulus_coprimality", Q::ErrorType::invalid_plain_modulus_coprimality)
        .value("invalid_plain_modulus_too_large", Q::ErrorType::invalid_plain_modulus_too_large)
        .value("invalid_plain_modulus_nonzero", Q::ErrorType::invalid_plain_modulus_nonzero)
        .value("failed_creating_rns_tool", Q::ErrorType::failed_creating_rns_tool);
    py::class_<Q>(m, "EncryptionParameterQualifiers")
        .def_readonly("parameter_error", &Q::parameter_error)
        .def_readonly("using_fft", &Q::using_fft)
        .def_readonly("using_ntt", &Q::using_ntt)
        .def_readonly("using_batching", &Q::using_batching)
        .def_readonly("using_fast_plain_lift", &Q::using_fast_plain_lift)
        .def_readonly("using_descending_modulus_chain", &Q::using_descending_modulus_chain)
        .def_readonly("sec_level", &Q::sec_level)
        .def("parameters_set", &Q::parametersSet)
        .def("parameter_error_name", &Q::parameterErrorName)
        .def("parameter_error_message", &Q::parameterErrorMessage);
    auto words = [](const std::uint64_t *p, std::size_t k) {
        return p ? to_array(vector<std::uint64_t>(p, p + k)) : py::array_t<std::uint64_t>(0);
    };
    py::class_<CD, std::shared_ptr<CD>>(m, "ContextData")
        .def("parms", &CD::parms)
        .def("parms_id", &CD::parmsID)
        .def("chain_index", &CD::chainIndex)
        .def("qualifiers", &CD::qualifiers)
        .def("total_coeff_modulus_bit_count", &CD::totalCoeffModulusBitCount)
        .def("total_coeff_modulus",
             [words](const CD &d) { return words(d.qualifiers().parametersSet() ? d.totalCoeffModulus() : nullptr, d.levelLimbs()); })
        .def("coeff_div_plain_modulus",
             [](const CD &d) {
                 py::list out;
                 const auto *p = d.coeffDivPlainModulus();
                 if (p && d.parms().scheme() != SchemeType::ckks && d.qualifiers().parametersSet())
                     for (int i = 0; i < d.levelLimbs(); i++) out.append(py::make_tuple(p[i].operand, p[i].quotient));
                 return out;
             })
        .def("upper_half_increment",
             [words](const CD &d) {
                 const bool ok = d.parms().scheme() != SchemeType::ckks && d.qualifiers().parametersSet();
                 return words(ok ? d.upperHalfIncrement() : nullptr, d.levelLimbs());
             })
        .def("coeff_modulus_mod_plain_modulus", &CD::coeffModulusModPlainModulus)
        .def("plain_upper_half_threshold", &CD::plainUpperHalfThreshold)
        .def("plain_upper_half_increment",
             [words](const CD &d) { return words(d.qualifiers().parametersSet() ? d.plainUpperHalfIncrement() : nullptr, d.levelLimbs()); })
        .def("upper_half_threshold", [words](const CD &d) { return words(d.upperHalfThreshold(), d.levelLimbs()); })
        .def("prev_context_data", [cd](const CD &d) { return cd(d.prevContextData()); })
        .def("next_context_data", [cd](const CD &d) { return cd(d.nextContextData()); });

    py::class_<SEALContext>(m, "SEALContext")
        .def(py::init<EncryptionParameters, bool, SecurityLevel>(), py::arg("parms"), py::arg("expand_mod_chain") = true,
             py::arg("sec_level") = SecurityLevel::tc128)
        .def("get_context_data", [cd](const SEALContext &c, const ParmsID &id) { return cd(c.getContextData(id)); })
        .def("first_context_data", [cd](const SEALContext &c) { return cd(c.firstContextData()); })
        .def("last_context_data", [cd](const SEALContext &c) { return cd(c.lastContextData()); })
        .def("key_context_data", [cd](const SEALContext &c) { return cd(c.keyContextData()); })
        .def("first_parms_id", &SEALContext::firstParmsID)
        .def("last_parms_id", &SEALContext::lastParmsID)
        .def("key_parms_id", &SEALContext::keyParmsID)
        .def("using_keyswitching", &SEALContext::using_keyswitching)
        .def("parameters_set", &SEALContext::parametersSet)
        .def("parameter_error_name", &SEALContext::parameterErrorName);

    py::class_<Plaintext>(m, "Plaintext")
        .def(py::init<>())
        .def(py::init<const std::string &>())
        .def("to_string", &Plaintext::to_string)
        .def("__str__", &Plaintext::to_string)
        .def("is_zero", &Plaintext::isZero)
        .def("__getitem__", &Plaintext::operator[])
        .def("__eq__", &Plaintext::operator==)
        .def("set_zero", &Plaintext::setZero)
        .def("coeff_count", &Plaintext::coeffCount)
        .def("is_ntt_form", &Plaintext::isNttForm)
        .def("parms_id", py::overload_cast<>(&Plaintext::parmsID, py::const_))
        .def("set_parms_id", [](Plaintext &self, const ParmsID &p) { self.parmsID() = p; })
        .def("scale", py::overload_cast<>(&Plaintext::scale, py::const_))
        .def("set_scale", [](Plaintext &self, double s) { self.scale() = s; })
        .def("copy", [](const Plaintext &p) { return Plaintext(p); })
        .def("save", [](const Plaintext &p) { return save_bytes(p); })
        .def("load", [](Plaintext &p, const py::bytes &b) { load_bytes(p, b); })
        .def("data", [](const Plaintext &p) { return to_array(p.toHost()); });

    py::class_<Ciphertext>(m, "Ciphertext")
        .def(py::init<>())
        .def(py::init<const SEALContext &>())
        .def(py::init<const SEALContext &, ParmsID>())
        .def(py::init<const SEALContext &, ParmsID, std::size_t>())
        .def("correction_factor", py::overload_cast<>(&Ciphertext::correctionFactor, py::const_))
        .def("set_correction_factor", [](Ciphertext &self, uint64_t c) { self.correctionFactor() = c; })
        .def("resize", py::overload_cast<std::size_t>(&Ciphertext::resize))
        .def("is_transparent", &Ciphertext::isTransparent)
        .def("reserve", &Ciphertext::reserve)
        .def("parms_id", py::overload_cast<>(&Ciphertext::parmsID, py::const_))
        .def("set_parms_id", [](Ciphertext &self, const ParmsID &p) { self.parmsID() = p; })
        .def("scale", py::overload_cast<>(&Ciphertext::scale, py::const_))
        .def("set_scale", [](Ciphertext &self, double s) { self.scale() = s; })
        .def("is_ntt_form", py::overload_cast<>(&Ciphertext::isNttForm, py::const_))
        .def("size", &Ciphertext::size)
        .def("coeff_modulus_size", &Ciphertext::coeffModulusSize)
        .def("poly_modulus_degree", &Ciphertext::polyModulusDegree)
        .def("copy", [](const Ciphertext &p) { return Ciphertext(p); })
        .def("save", [](const Ciphertext &c) { return save_bytes(c); })
        .def("save_terms",
             [](const Ciphertext &c, Evaluator &ev, SizeArray terms) {
                 std::ostringstream s;
                 c.saveTerms(s, ev, from_array(terms));
                 return py::bytes(s.str());
             })
        .def("load", [](Ciphertext &c, const py::bytes &b) { load_bytes(c, b); })
        .def("load",
             [](Ciphertext &c, const py::bytes &b, const SEALContext &ctx) {
                 std::istringstream s{std::string(b)};
                 c.load(s, ctx);
             })
        .def("load_terms",
             [](Ciphertext &c, const py::bytes &b, Evaluator &ev, SizeArray terms) {
                 std::istringstream s{std::string(b)};
                 c.loadTerms(s, ev, from_array(terms));
             })
        .def("seed", py::overload_cast<>(&Ciphertext::seed, py::const_))
        .def("data", [](const Ciphertext &c) { return to_array(c.toHost()); });

    py::class_<KeyGenerator>(m, "KeyGenerator")
        .def(py::init<const SEALContext &>(), py::keep_alive<1, 2>())
        .def("secret_key", &KeyGenerator::secretKey)
        .def("create_public_key", py::overload_cast<PublicKey &>(&KeyGenerator::createPublicKey, py::const_))
        .def("create_public_key", py::overload_cast<>(&KeyGenerator::createPublicKey, py::const_))
        .def("create_relin_keys", py::overload_cast<RelinKeys &>(&KeyGenerator::createRelinKeys, py::const_))
        .def("create_relin_keys", py::overload_cast<>(&KeyGenerator::createRelinKeys, py::const_))
        .def("create_galois_keys", py::overload_cast<GaloisKeys &>(&KeyGenerator::createGaloisKeys, py::const_))
        .def("create_galois_keys", py::overload_cast<>(&KeyGenerator::createGaloisKeys, py::const_))
        .def("create_galois_keys",
             py::overload_cast<const vector<int> &, GaloisKeys &>(&KeyGenerator::createGaloisKeys, py::const_))
        .def("create_galois_keys", py::overload_cast<const vector<int> &>(&KeyGenerator::createGaloisKeys, py::const_));

    py::class_<SecretKey>(m, "SecretKey")
        .def(py::init<>())
        .def("parms_id", py::overload_cast<>(&SecretKey::parmsID, py::const_))
        .def("save", [](const SecretKey &k) { return save_bytes(k); })
        .def("load", [](SecretKey &k, const py::bytes &b) { load_bytes(k, b); })
        .def("data", [](const SecretKey &k) { return to_array(k.data().toHost()); });
    py::class_<PublicKey>(m, "PublicKey")
        .def(py::init<>())
        .def("parms_id", py::overload_cast<>(&PublicKey::parmsID, py::const_))
        .def("save", [](const PublicKey &k) { return save_bytes(k); })
        .def("load", [](PublicKey &k, const py::bytes &b) { load_bytes(k, b); })
        .def("data", [](const PublicKey &k) { return to_array(k.data().toHost()); });
    py::class_<KSwitchKeys>(m, "KSwitchKeys")
        .def(py::init<>())
        .def("parms_id", py::overload_cast<>(&KSwitchKeys::parmsID, py::const_))
        .def("size", &KSwitchKeys::size)
        .def("save", [](const KSwitchKeys &k) { return save_bytes(k); })
        .def("load", [](KSwitchKeys &k, const py::bytes &b) { load_bytes(k, b); });
    py::class_<RelinKeys, KSwitchKeys>(m, "RelinKeys")
        .def(py::init<>())
        .def("data", [](const RelinKeys &k, std::size_t index) { return to_array(k.data().at(index).toHost()); });
    py::class_<GaloisKeys, KSwitchKeys>(m, "GaloisKeys")
        .def(py::init<>())
        .def("has_key", &GaloisKeys::hasKeyElt)
        .def("data", [](const GaloisKeys &k, uint32_t elt) {
            return to_array(k.data().at(GaloisKeys::getIndex(elt)).toHost());
        });

    py::class_<BatchEncoder>(m, "BatchEncoder")
        .def(py::init<const SEALContext &>(), py::keep_alive<1, 2>())
        .def("encode_int64", [](const BatchEncoder &self, I64Array t, Plaintext &p) { self.encode(from_array(t), p); })
        .def("encode", [](const BatchEncoder &self, U64Array t, Plaintext &p) { self.encode(from_array(t), p); })
        .def("encode_int64",
             [](const BatchEncoder &self, I64Array t) {
                 Plaintext p;
                 self.encode(from_array(t), p);
                 return p;
             })
        .def("encode",
             [](const BatchEncoder &self, U64Array t) {
                 Plaintext p;
                 self.encode(from_array(t), p);
                 return p;
             })
        .def("encode_polynomial",
             [](const BatchEncoder &self, U64Array t) {
                 Plaintext p;
                 self.encodePolynomial(from_array(t), p);
                 return p;
             })
        .def("decode_int64",
             [](const BatchEncoder &self, const Plaintext &plain) {
                 vector<int64_t> r;
                 self.decode(plain, r);
                 return to_array(r);
             })
        .def("decode",
             [](const BatchEncoder &self, const Plaintext &plain) {
                 vector<uint64_t> r;
                 self.decode(plain, r);
                 return to_array(r);
             })
        .def("decode_polynomial",
             [](const BatchEncoder &self, const Plaintext &plain) {
                 vector<uint64_t> r;
                 self.decodePolynomial(plain, r);
                 return to_array(r);
             })
        .def("slot_count", &BatchEncoder::slotCount);

    py::class_<CKKSEncoder>(m, "CKKSEncoder")
        .def(py::init<const SEALContext &>(), py::keep_alive<1, 2>())
        .def("encode",
             [](CKKSEncoder &self, C128Array v, double scale, Plaintext &p) { self.encode(from_array(v), scale, p); })
        .def("encode", [](CKKSEncoder &self, C128Array v, ParmsID id, double scale,
                          Plaintext &p) { self.encode(from_array(v), id, scale, p); })
        .def("encode_polynomial", [](CKKSEncoder &self, F64Array v, double scale,
                                     Plaintext &p) { self.encodePolynomial(from_array(v), scale, p); })
        .def("encode_polynomial", [](CKKSEncoder &self, F64Array v, ParmsID id, double scale,
                                     Plaintext &p) { self.encodePolynomial(from_array(v), id, scale, p); })
        .def("encode", py::overload_cast<complex<double>, double, Plaintext &>(&CKKSEncoder::encode, py::const_))
        .def("encode",
             py::overload_cast<complex<double>, const ParmsID &, double, Plaintext &>(&CKKSEncoder::encode, py::const_))
        .def("encode",
             [](CKKSEncoder &self, C128Array v, double scale) {
                 Plaintext p;
                 self.encode(from_array(v), scale, p);
                 return p;
             })
        .def("encode",
             [](CKKSEncoder &self, C128Array v, ParmsID id, double scale) {
                 Plaintext p;
                 self.encode(from_array(v), id, scale, p);
                 return p;
             })
        .def("encode_polynomial",
             [](CKKSEncoder &self, F64Array v, double scale) {
                 Plaintext p;
                 self.encodePolynomial(from_array(v), scale, p);
                 return p;
             })
        .def("encode_polynomial",
             [](CKKSEncoder &self, F64Array v, ParmsID id, double scale) {
                 Plaintext p;
                 self.encodePolynomial(from_array(v), id, scale, p);
                 return p;
             })
        .def("encode",
             [](CKKSEncoder &self, complex<double> v, double scale) {
                 Plaintext p;
                 self.encode(v, scale, p);
                 return p;
             })
        .def("encode",
             [](CKKSEncoder &self, complex<double> v, ParmsID id, double scale) {
                 Plaintext p;
                 self.encode(v, id, scale, p);
                 return p;
             })
        .def("decode",
             [](CKKSEncoder &self, const Plaintext &plain) {
                 vector<complex<double>> r;
                 self.decode(plain, r);
                 return to_array(r);
             })
        .def("decode_polynomial",
             [](CKKSEncoder &self, const Plaintext &plain) {
                 vector<double> r;
                 self.decodePolynomial(plain, r);
                 return to_array(r);
             })
        .def("slot_count", &CKKSEncoder::slotCount);

    py::class_<Encryptor>(m, "Encryptor")
        .def(py::init<const SEALContext &, const PublicKey &>(), py::keep_alive<1, 2>())
        .def(py::init<const SEALContext &, const SecretKey &>(), py::keep_alive<1, 2>())
        .def(py::init<const SEALContext &, const PublicKey &, const SecretKey &>(), py::keep_alive<1, 2>())
        .def("set_public_key", &Encryptor::setPublicKey)
        .def("set_secret_key", &Encryptor::setSecretKey)
        .def("encrypt", py::overload_cast<const Plaintext &, Ciphertext &>(&Encryptor::encrypt, py::const_))
        .def("encrypt_zero", py::overload_cast<Ciphertext &>(&Encryptor::encryptZero, py::const_))
        .def("encrypt_zero", py::overload_cast<const ParmsID &, Ciphertext &>(&Encryptor::encryptZero, py::const_))
        .def("encrypt_symmetric",
             py::overload_cast<const Plaintext &, Ciphertext &>(&Encryptor::encryptSymmetric, py::const_))
        .def("encrypt_zero_symmetric", py::overload_cast<Ciphertext &>(&Encryptor::encryptZeroSymmetric, py::const_))
        .def("encrypt_zero_symmetric",
             py::overload_cast<const ParmsID &, Ciphertext &>(&Encryptor::encryptZeroSymmetric, py::const_))
        .def("encrypt",
             [](const Encryptor &self, const Plaintext &plain) {
                 Ciphertext r;
                 self.encrypt(plain, r);
                 return r;
             })
        .def("encrypt_zero",
             [](const Encryptor &self) {
                 Ciphertext r;
                 self.encryptZero(r);
                 return r;
             })
        .def("encrypt_zero",
             [](const Encryptor &self, ParmsID id) {
                 Ciphertext r;
                 self.encryptZero(id, r);
                 return r;
             })
        .def("encrypt_symmetric",
             [](const Encryptor &self, const Plaintext &plain) {
                 Ciphertext r;
                 self.encryptSymmetric(plain, r);
                 return r;
             })
        .def("encrypt_zero_symmetric",
             [](const Encryptor &self) {
                 Ciphertext r;
                 self.encryptZeroSymmetric(r);
                 return r;
             })
        .def("encrypt_zero_symmetric",
             [](const Encryptor &self, ParmsID id) {
                 Ciphertext r;
                 self.encryptZeroSymmetric(id, r);
                 return r;
             })
        .def("encrypt_symmetric_seeded",
             [](const Encryptor &self, const Plaintext &plain) {
                 Ciphertext r;
                 self.encryptSymmetricSeeded(plain, r);
                 return r;
             })
        .def("encrypt_zero_symmetric_seeded", [](const Encryptor &self, ParmsID id) {
            Ciphertext r;
            self.encryptZeroSymmetricSeeded(id, r);
            return r;
        });

    py::class_<Decryptor>(m, "Decryptor")
        .def(py::init<const SEALContext &, const SecretKey &>(), py::keep_alive<1, 2>())
        .def("decrypt", &Decryptor::decrypt)
        .def("decrypt", [](Decryptor &self, const Ciphertext &c) {
            Plaintext p;
            self.decrypt(c, p);
            return p;
        });

    using E = Evaluator;
    using C = Ciphertext;
    using P = Plaintext;
    using GK = GaloisKeys;
    using RK = RelinKeys;
    py::class_<Evaluator>(m, "Evaluator")
        .def(py::init<const SEALContext &>(), py::keep_alive<1, 2>())
        .def("negate_inplace", &E::negateInplace)
        .def("negate", [](const E &self, const C &c) { C r; self.negate(c, r); return r; })
        .def("negate", &E::negate)
        .def("add_inplace", &E::addInplace)
        .def("add", [](const E &self, const C &a, const C &b) { C r; self.add(a, b, r); return r; })
        .def("add", &E::add)
        .def("add_many", &E::addMany)
        .def("add_many", [](const E &self, const vector<C> &v) { C r; self.addMany(v, r); return r; })
        .def("sub_inplace", &E::subInplace)
        .def("sub", [](const E &self, const C &a, const C &b) { C r; self.sub(a, b, r); return r; })
        .def("sub", &E::sub)
        .def("multiply_inplace", &E::multiplyInplace)
        .def("multiply", [](const E &self, const C &a, const C &b) { C r; self.multiply(a, b, r); return r; })
        .def("multiply", &E::multiply)
        .def("square_inplace", &E::squareInplace)
        .def("square", [](const E &self, const C &a) { C r; self.square(a, r); return r; })
        .def("square", &E::square)
        .def("relinearize_inplace", &E::relinearizeInplace)
        .def("relinearize", &E::relinearize)
        .def("relinearize", [](const E &self, const C &c, const RK &k) { C r; self.relinearize(c, k, r); return r; })
        .def("mod_switch_to_next_inplace", py::overload_cast<C &>(&E::modSwitchToNextInplace, py::const_))
        .def("mod_switch_to_next_inplace", py::overload_cast<P &>(&E::modSwitchToNextInplace, py::const_))
        .def("mod_switch_to_next", py::overload_cast<const C &, C &>(&E::modSwitchToNext, py::const_))
        .def("mod_switch_to_next", [](const E &self, const C &c) { C r; self.modSwitchToNext(c, r); return r; })
        .def("mod_switch_to_next", py::overload_cast<const P &, P &>(&E::modSwitchToNext, py::const_))
        .def("mod_switch_to_next", [](const E &self, const P &p) { P r; self.modSwitchToNext(p, r); return r; })
        .def("mod_switch_to_inplace", py::overload_cast<C &, const ParmsID &>(&E::modSwitchToInplace, py::const_))
        .def("mod_switch_to_inplace", py::overload_cast<P &, const ParmsID &>(&E::modSwitchToInplace, py::const_))
        .def("mod_switch_to", py::overload_cast<const C &, const ParmsID &, C &>(&E::modSwitchTo, py::const_))
        .def("mod_switch_to", [](const E &self, ParmsID id, const C &c) { C r; self.modSwitchTo(c, id, r); return r; })
        .def("mod_switch_to", py::overload_cast<const P &, const ParmsID &, P &>(&E::modSwitchTo, py::const_))
        .def("mod_switch_to", [](const E &self, ParmsID id, const P &p) { P r; self.modSwitchTo(p, id, r); return r; })
        .def("rescale_to_next_inplace", &E::rescaleToNextInplace)
        .def("rescale_to_next", &E::rescaleToNext)
        .def("rescale_to_next", [](const E &self, const C &c) { C r; self.rescaleToNext(c, r); return r; })
        .def("rescale_to_inplace", &E::rescaleToInplace)
        .def("rescale_to", &E::rescaleTo)
        .def("rescale_to", [](const E &self, ParmsID id, const C &c) { C r; self.rescaleTo(c, id, r); return r; })
        .def("multiply_many", &E::multiplyMany)
        .def("multiply_many",
             [](const E &self, const vector<C> &v, const RK &k) { C r; self.multiplyMany(v, k, r); return r; })
        .def("exponentiate_inplace", &E::exponentiateInplace)
        .def("exponentiate", &E::exponentiate)
        .def("exponentiate",
             [](const E &self, const C &c, uint64_t e, const RK &k) { C r; self.exponentiate(c, e, k, r); return r; })
        .def("add_plain_inplace", &E::addPlainInplace)
        .def("add_plain", [](const E &self, const C &c, const P &p) { C r; self.addPlain(c, p, r); return r; })
        .def("add_plain", &E::addPlain)
        .def("sub_plain_inplace", &E::subPlainInplace)
        .def("sub_plain", [](const E &self, const C &c, const P &p) { C r; self.subPlain(c, p, r); return r; })
        .def("sub_plain", &E::subPlain)
        .def("multiply_plain_inplace", &E::multiplyPlainInplace)
        .def("multiply_plain", [](const E &self, const C &c, const P &p) { C r; self.multiplyPlain(c, p, r); return r; })
        .def("multiply_plain_1000",
             [](const E &self, const C &c, const P &p) {
                 C r;
                 for (int i = 0; i < 1000; i++) self.multiplyPlain(c, p, r);
                 return r;
             })
        .def("multiply_batch",
             [](const E &self, const vector<C> &cs, const vector<P> &ps) {
                 if (cs.size() != ps.size()) throw std::invalid_argument("size mismatch");
                 vector<C> r(cs.size());
                 for (std::size_t i = 0; i < cs.size(); i++) self.multiplyPlain(cs[i], ps[i], r[i]);
                 return r;
             })
        .def("multiply_plain", &E::multiplyPlain)
        .def("transform_to_ntt_inplace", py::overload_cast<P &, const ParmsID &>(&E::transformToNttInplace, py::const_))
        .def("transform_to_ntt_inplace", py::overload_cast<C &>(&E::transformToNttInplace, py::const_))
        .def("transform_to_ntt", py::overload_cast<const P &, const ParmsID &, P &>(&E::transformToNtt, py::const_))
        .def("transform_to_ntt", [](const E &self, const P &p, ParmsID id) { P r; self.transformToNtt(p, id, r); return r; })
        .def("transform_to_ntt", py::overload_cast<const C &, C &>(&E::transformToNtt, py::const_))
        .def("transform_to_ntt", [](const E &self, const C &c) { C r; self.transformToNtt(c, r); return r; })
        .def("transform_from_ntt_inplace", py::overload_cast<C &>(&E::transformFromNttInplace, py::const_))
        .def("transform_from_ntt", py::overload_cast<const C &, C &>(&E::transformFromNtt, py::const_))
        .def("transform_to_ntt", [](const E &self, const C &c) { C r; self.transformFromNtt(c, r); return r; })
        .def("apply_galois_inplace", &E::applyGaloisInplace)
        .def("apply_galois", &E::applyGalois)
        .def("apply_galois",
             [](const E &self, const C &c, uint32_t elt, const GK &k) { C r; self.applyGalois(c, elt, k, r); return r; })
        .def("rotate_rows_inplace", &E::rotateRowsInplace)
        .def("rotate_rows", &E::rotateRows)
        .def("rotate_rows",
             [](const E &self, const C &c, int steps, const GK &k) { C r; self.rotateRows(c, steps, k, r); return r; })
        .def("rotate_columns_inplace", &E::rotateColumnsInplace)
        .def("rotate_columns", &E::rotateColumns)
        .def("rotate_rows", [](const E &self, const C &c, const GK &k) { C r; self.rotateColumns(c, k, r); return r; })
        .def("rotate_vector_inplace", &E::rotateVectorInplace)
        .def("rotate_vector", &E::rotateVector)
        .def("rotate_vector",
             [](const E &self, const C &c, int steps, const GK &k) { C r; self.rotateVector(c, steps, k, r); return r; })
        .def("complex_conjugate_inplace", &E::complexConjugateInplace)
        .def("complex_conjugate", &E::complexConjugate)
        .def("complex_conjugate",
             [](const E &self, const C &c, const GK &k) { C r; self.complexConjugate(c, k, r); return r; });

    // Cipher2d / Plain2d (app/LinearHelper.cuh:20-195; binder/binder.cu:700-729). Rows
    // read as lists (len / indexing) and build from lists of lists as well.
    using CRows = std::vector<std::vector<Ciphertext>>;
    using PRows = std::vector<std::vector<Plaintext>>;
    py::class_<Cipher2d>(m, "Cipher2d")
        .def(py::init<>())
        .def(py::init([](CRows rows) {
            Cipher2d c;
            c.data = std::move(rows);
            return c;
        }))
        .def("save", [](const Cipher2d &c) { return save_bytes(c); })
        .def("load", [](Cipher2d &c, const py::bytes &b) { load_bytes(c, b); })
        .def("load",
             [](Cipher2d &c, const py::bytes &b, const SEALContext &ctx) {
                 std::istringstream st{std::string(b)};
                 c.load(st, ctx);
             })
        .def("add_inplace", &Cipher2d::addInplace)
        .def("add_plain_inplace", &Cipher2d::addPlainInplace)
        .def("add_plain", &Cipher2d::addPlain)
        .def("mod_switch_to_next", &Cipher2d::modSwitchToNext)
        .def("__len__", [](const Cipher2d &c) { return c.data.size(); })
        .def("__getitem__", [](const Cipher2d &c, std::size_t i) { return c.data.at(i); });
    py::class_<Plain2d>(m, "Plain2d")
        .def(py::init<>())
        .def(py::init([](PRows rows) {
            Plain2d p;
            p.data = std::move(rows);
            return p;
        }))
        .def("encrypt", &Plain2d::encrypt)
        .def("__len__", [](const Plain2d &p) { return p.data.size(); })
        .def("__getitem__", [](const Plain2d &p, std::size_t i) { return p.data.at(i); });

    // MatmulHelper (app/LinearHelper.cuh:197-530; binder/binder.cu:813-858): coefficient-
    // encoded matrix products, the products of one call fused into one device pass.
    auto check_len = [](const U64Array &a, std::size_t want, const char *what) {
        if ((std::size_t)a.size() != want) throw std::invalid_argument(std::string(what) + " size incorrect.");
    };
    py::class_<MatmulHelper>(m, "MatmulHelper")
        .def(py::init<std::size_t, std::size_t, std::size_t, std::size_t>())
        .def_property_readonly("batch_block", [](const MatmulHelper &h) { return h.plan().batchBlock; })
        .def_property_readonly("input_block", [](const MatmulHelper &h) { return h.plan().inputBlock; })
        .def_property_readonly("output_block", [](const MatmulHelper &h) { return h.plan().outputBlock; })
        .def("encode_weights",
             [check_len](const MatmulHelper &h, const BatchEncoder &enc, U64Array w) {
                 check_len(w, h.plan().in * h.plan().out, "Weight");
                 return h.encodeWeights(enc, w.data());
             })
        .def("encode_inputs",
             [check_len](const MatmulHelper &h, const BatchEncoder &enc, U64Array x) {
                 check_len(x, h.plan().batch * h.plan().in, "Input");
                 return h.encodeInputs(enc, x.data());
             })
        .def("encrypt_inputs",
             [check_len](const MatmulHelper &h, const Encryptor &e, const BatchEncoder &enc, U64Array x) {
                 check_len(x, h.plan().batch * h.plan().in, "Input");
                 return h.encryptInputs(e, enc, x.data());
             })
        .def("matmul", &MatmulHelper::matmul)
        .def("matmul", &MatmulHelper::matmulCipher)
        .def("matmul", &MatmulHelper::matmulReverse)
        .def("encode_outputs",
             [check_len](const MatmulHelper &h, const BatchEncoder &enc, U64Array y) {
                 check_len(y, h.plan().batch * h.plan().out, "Output");
                 return h.encodeOutputs(enc, y.data());
             })
        .def("decrypt_outputs",
             [](const MatmulHelper &h, const BatchEncoder &enc, Decryptor &dec, const Cipher2d &c) {
                 return to_array(h.decryptOutputs(enc, dec, c));
             })
        .def("serialize_outputs",
             [](const MatmulHelper &h, const Evaluator &ev, const Cipher2d &x) {
                 std::ostringstream st;
                 h.serializeOutputs(ev, x, st);
                 return py::bytes(st.str());
             })
        .def("deserialize_outputs",
             [](const MatmulHelper &h, const Evaluator &ev, const py::bytes &b) {
                 std::istringstream st{std::string(b)};
                 return h.deserializeOutputs(ev, st);
             })
        .def("serialize_encoded_weights",
             [](const MatmulHelper &h, const Plain2d &w) {
                 std::ostringstream st;
                 h.serializeEncodedWeights(w, st);
                 return py::bytes(st.str());
             })
        .def("deserialize_encoded_weights", [](const MatmulHelper &h, const py::bytes &b) {
            std::istringstream st{std::string(b)};
            return h.deserializeEncodedWeights(st);
        });

    // Conv2dHelper (app/LinearHelper.cuh:531-975; binder/binder.cu:860-896).
    py::class_<Conv2dHelper>(m, "Conv2dHelper")
        .def(py::init<std::size_t, std::size_t, std::size_t, std::size_t, std::size_t, std::size_t, std::size_t,
                      std::size_t>())
        .def("total_batch_size", &Conv2dHelper::totalBatchSize)
        .def("encode_weights",
             [](const Conv2dHelper &h, const BatchEncoder &enc, U64Array w) { return h.encodeWeights(enc, flat_u64(w)); })
        .def("encode_inputs",
             [](const Conv2dHelper &h, const BatchEncoder &enc, U64Array x) { return h.encodeInputs(enc, flat_u64(x)); })
        .def("encrypt_inputs",
             [](const Conv2dHelper &h, const Encryptor &e, const BatchEncoder &enc, U64Array x) {
                 return h.encryptInputs(e, enc, flat_u64(x));
             })
        .def("conv2d", &Conv2dHelper::conv2d)
        .def("conv2d", &Conv2dHelper::conv2dCipher)
        .def("conv2d", &Conv2dHelper::conv2dReverse)
        .def("encode_outputs",
             [](const Conv2dHelper &h, const BatchEncoder &enc, U64Array y) { return h.encodeOutputs(enc, flat_u64(y)); })
        .def("add_plain_inplace", &Conv2dHelper::addPlainInplace)
        .def("add_inplace", &Conv2dHelper::addInplace)
        .def("decrypt_outputs",
             [](const Conv2dHelper &h, const BatchEncoder &enc, Decryptor &dec, const Cipher2d &c) {
                 return to_array(h.decryptOutputs(enc, dec, c));
             })
        .def("serialize_outputs",
             [](const Conv2dHelper &h, const Evaluator &ev, const Cipher2d &x) {
                 std::ostringstream st;
                 h.serializeOutputs(ev, x, st);
                 return py::bytes(st.str());
             })
        .def("deserialize_outputs", [](const Conv2dHelper &h, const Evaluator &ev, const py::bytes &b) {
            std::istringstream st{std::string(b)};
            return h.deserializeOutputs(ev, st);
        });

    // LinearHelperCKKS (app/LinearHelperCKKS.cuh), bound with the method names of the
    // reference binder's CKKS helper bindings (binder/binder.cu:731-811).
    using F64 = py::array_t<double, py::array::c_style | py::array::forcecast>;
    py::class_<LinearHelperCKKS::MatmulHelper>(m, "CkksMatmulHelper")
        .def(py::init<std::size_t, std::size_t, std::size_t, std::size_t>())
        .def_property_readonly("block_height", &LinearHelperCKKS::MatmulHelper::blockHeight)
        .def_property_readonly("block_width", &LinearHelperCKKS::MatmulHelper::blockWidth)
        .def_readwrite("encoded_weights", &LinearHelperCKKS::MatmulHelper::encodedWeights)
        .def("encode_weights",
             [](LinearHelperCKKS::MatmulHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 w, double scale) {
                 h.encodeWeights(enc, id, flat_f64(w), scale);
             })
        .def("encode_inputs",
             [](const LinearHelperCKKS::MatmulHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 x,
                double scale) { return h.encodeInputs(enc, id, flat_f64(x), scale); })
        .def("encrypt_inputs",
             [](const LinearHelperCKKS::MatmulHelper &h, const Encryptor &e, const CKKSEncoder &enc, const ParmsID &id,
                F64 x, double scale) { return h.encryptInputs(e, enc, id, flat_f64(x), scale); })
        .def("matmul", &LinearHelperCKKS::MatmulHelper::matmul)
        .def("encode_outputs",
             [](const LinearHelperCKKS::MatmulHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 y,
                double scale) { return h.encodeOutputs(enc, id, flat_f64(y), scale); })
        .def("add_plain_inplace", &LinearHelperCKKS::MatmulHelper::addPlainInplace)
        .def("decrypt_outputs",
             [](const LinearHelperCKKS::MatmulHelper &h, const CKKSEncoder &enc, Decryptor &dec, const Cipher2d &c) {
                 return to_array(h.decryptOutputs(enc, dec, c));
             })
        .def("serialize_outputs",
             [](const LinearHelperCKKS::MatmulHelper &h, const Evaluator &ev, const Cipher2d &x) {
                 std::ostringstream st;
                 h.serializeOutputs(ev, x, st);
                 return py::bytes(st.str());
             })
        .def("deserialize_outputs", [](const LinearHelperCKKS::MatmulHelper &h, const Evaluator &ev, const py::bytes &b) {
            std::istringstream st{std::string(b)};
            return h.deserializeOutputs(ev, st);
        });
    py::class_<LinearHelperCKKS::Conv2dHelper>(m, "CkksConv2dHelper")
        .def(py::init<std::size_t, std::size_t, std::size_t, std::size_t, std::size_t, std::size_t, std::size_t,
                      std::size_t>())
        .def("total_batch_size", &LinearHelperCKKS::Conv2dHelper::totalBatchSize)
        .def_readwrite("encoded_weights", &LinearHelperCKKS::Conv2dHelper::encodedWeights)
        .def("encode_weights",
             [](LinearHelperCKKS::Conv2dHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 w, double scale) {
                 h.encodeWeights(enc, id, flat_f64(w), scale);
             })
        .def("encode_inputs",
             [](const LinearHelperCKKS::Conv2dHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 x,
                double scale) { return h.encodeInputs(enc, id, flat_f64(x), scale); })
        .def("encrypt_inputs",
             [](const LinearHelperCKKS::Conv2dHelper &h, const Encryptor &e, const CKKSEncoder &enc, const ParmsID &id,
                F64 x, double scale) { return h.encryptInputs(e, enc, id, flat_f64(x), scale); })
        .def("conv2d", &LinearHelperCKKS::Conv2dHelper::conv2d)
        .def("encode_outputs",
             [](const LinearHelperCKKS::Conv2dHelper &h, const CKKSEncoder &enc, const ParmsID &id, F64 y,
                double scale) { return h.encodeOutputs(enc, id, flat_f64(y), scale); })
        .def("add_plain_inplace", &LinearHelperCKKS::Conv2dHelper::addPlainInplace)
        .def("add_inplace", &LinearHelperCKKS::Conv2dHelper::addInplace)
        .def("decrypt_outputs",
             [](const LinearHelperCKKS::Conv2dHelper &h, const CKKSEncoder &enc, Decryptor &dec, const Cipher2d &c) {
                 return to_array(h.decryptOutputs(enc, dec, c));
             })
        .def("serialize_outputs",
             [](const LinearHelperCKKS::Conv2dHelper &h, const Evaluator &ev, const Cipher2d &x) {
                 std::ostringstream st;
                 h.serializeOutputs(ev, x, st);
                 return py::bytes(st.str());
             })
        .def("deserialize_outputs", [](const LinearHelperCKKS::Conv2dHelper &h, const Evaluator &ev, const py::bytes &b) {
            std::istringstream st{std::string(b)};
            return h.deserializeOutputs(ev, st);
        });

    // The diagonal CKKS matrix-vector product (app/matmul.cuh).
    using C128 = py::array_t<complex<double>, py::array::c_style | py::array::forcecast>;
    py::class_<DiagonalMatmulHelper>(m, "DiagonalMatmulHelper")
        .def(py::init<std::size_t, std::size_t, std::size_t>())
        .def_property_readonly("pack_num", &DiagonalMatmulHelper::packNum)
        .def_property_readonly("cipher_count", &DiagonalMatmulHelper::cipherCount)
        .def("prepare_input",
             [](const DiagonalMatmulHelper &h, C128 x, const CKKSEncoder &enc, double scale) {
                 return h.prepareInput(vector<complex<double>>(x.data(), x.data() + x.size()), enc, scale);
             })
        .def("decode_result",
             [](const DiagonalMatmulHelper &h, const Plaintext &p, const CKKSEncoder &enc) {
                 return to_array(h.decodeResult(p, enc));
             })
        .def("encode",
             [](DiagonalMatmulHelper &h, C128 mat, const CKKSEncoder &enc, double scale) {
                 if (mat.ndim() != 2) throw std::invalid_argument("matrix must be 2-d");
                 const auto r = mat.unchecked<2>();
                 vector<vector<complex<double>>> rows(mat.shape(0), vector<complex<double>>(mat.shape(1)));
                 for (py::ssize_t i = 0; i < mat.shape(0); i++)
                     for (py::ssize_t j = 0; j < mat.shape(1); j++) rows[i][j] = r(i, j);
                 h.encode(rows, enc, scale);
             })
        .def("multiply", &DiagonalMatmulHelper::multiply, py::arg("repeated_vector"), py::arg("evaluator"),
             py::arg("galois_keys"), py::arg("rescale"));

    // Continuous-batching server of single-row MatmulHelper products.
    py::class_<MatmulServer>(m, "MatmulServer")
        .def(py::init([](const SEALContext &ctx, std::size_t memory_budget, int slots, std::size_t max_wave_requests,
                         std::size_t output_staging) {
                 MatmulServer::Options o;
                 o.memory_budget = memory_budget;
                 o.slots = slots;
                 o.max_wave_requests = max_wave_requests;
                 o.output_staging = output_staging;
                 return std::make_unique<MatmulServer>(ctx, o);
             }),
             py::arg("context"), py::arg("memory_budget") = std::size_t(8) << 30, py::arg("slots") = 3,
             py::arg("max_wave_requests") = 256, py::arg("output_staging") = std::size_t(256) << 20,
             py::keep_alive<1, 2>())
        .def_static("now", &MatmulServer::now)
        .def(
            "submit",
            [](MatmulServer &s, std::size_t in, std::size_t out, U64Array inputs, U64Array weights, double arrival,
               py::object outputs) {
                if ((std::size_t)weights.size() != in * out) throw std::invalid_argument("Weight size incorrect.");
                uint64_t *dst = nullptr;
                py::array out_arr;
                if (!outputs.is_none()) {  // written in place: no conversion, no copy
                    if (!py::isinstance<py::array>(outputs)) throw std::invalid_argument("outputs must be an array");
                    out_arr = outputs.cast<py::array>();
                    if (!out_arr.dtype().is(py::dtype::of<uint64_t>()) || !(out_arr.flags() & py::array::c_style) ||
                        !out_arr.writeable())
                        throw std::invalid_argument("outputs must be a writable contiguous uint64 array");
                    const MatmulPlan p = MatmulPlan::make(1, in, out, s.slotDegree());
                    if ((std::size_t)out_arr.size() != p.outputBlocks() * s.ciphertextWords())
                        throw std::invalid_argument("outputs size incorrect.");
                    dst = static_cast<uint64_t *>(out_arr.mutable_data());
                }
                // the arrays are read at admission and written at completion; holding them
                // here keeps them alive (requests are admitted and finished inside step(),
                // with the GIL held)
                auto owner = std::make_shared<std::tuple<U64Array, U64Array, py::array>>(inputs, weights, out_arr);
                return s.submitBorrowed(in, out, inputs.data(), inputs.size(), weights.data(), arrival, owner, dst);
            },
            py::arg("in_dims"), py::arg("out_dims"), py::arg("inputs"), py::arg("weights"), py::arg("arrival"),
            py::arg("outputs") = py::none())
        .def("step", &MatmulServer::step)
        .def("drain", &MatmulServer::drain)
        .def("idle", &MatmulServer::idle)
        .def("queued", &MatmulServer::queued)
        .def("result",
             [](MatmulServer &s, std::uint64_t id) -> py::object {
                 vector<uint64_t> out;
                 double arrival = 0, done = 0;
                 bool ok = false;
                 if (!s.result(id, out, arrival, done, ok)) return py::none();
                 return py::make_tuple(to_array(out), arrival, done, ok);
             })
        .def("take",
             [](MatmulServer &s, std::uint64_t id) -> py::object {
                 auto *out = new vector<uint64_t>();
                 double arrival = 0, done = 0;
                 bool ok = false;
                 if (!s.take(id, *out, arrival, done, ok)) {
                     delete out;
                     return py::none();
                 }
                 py::capsule owner(out, [](void *p) { delete static_cast<vector<uint64_t> *>(p); });
                 py::array_t<uint64_t> arr({(py::ssize_t)out->size()}, {(py::ssize_t)8}, out->data(), owner);
                 return py::make_tuple(arr, arrival, done, ok);
             })
        .def("release", &MatmulServer::release)
        .def("inject_wave_failure", &MatmulServer::injectWaveFailure)
        .def("stats", [](const MatmulServer &s) {
            const auto &st = s.stats();
            py::dict d;
            d["submitted"] = st.submitted;
            d["completed"] = st.completed;
            d["failed"] = st.failed;
            d["waves"] = st.waves;
            d["peak_bytes"] = st.peak_bytes;
            d["max_wave"] = st.max_wave;
            d["launch_host_s"] = st.launch_host_s;
            d["reap_host_s"] = st.reap_host_s;
            d["alloc_host_s"] = st.alloc_host_s;
            d["device_s"] = st.device_s;
            return d;
        });
}

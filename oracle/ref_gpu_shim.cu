// Test/benchmark infrastructure, not part of the library: times the reference's own
// CUDA evaluator (troyn:: classes of src/troy_cuda.cuh, compiled from the reference
// sources by `make -C oracle ref_gpu`) on the batched CKKS workload one ciphertext
// pair per call — multiply, relinearizeInplace, rescaleToNextInplace,
// rotateVectorInplace — the "plain per-op GPU path" the batched library is compared
// with. The decrypted result of the last op is checked against the FP64 product.
// ref_gpu_batch_chain does the same for BFV / BGV (multiply, relinearize, rotate rows).
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstring>
#include <random>
#include <sstream>
#include <vector>

#include "troy_cuda.cuh"

using namespace troyn;

extern "C" int ref_gpu_ckks_chain(size_t n, const uint64_t *moduli, int count, int scale_bits, int ops,
                                  const int *steps, int nsteps, double *ms_per_op, double *max_err) {
    try {
        KernelProvider::initialize();
        EncryptionParameters parms(SchemeType::ckks);
        parms.setPolyModulusDegree(n);
        std::vector<Modulus> q;
        for (int i = 0; i < count; i++) q.emplace_back(moduli[i]);
        parms.setCoeffModulus(q);
        SEALContext context(parms, true, SecurityLevel::none);
        CKKSEncoder encoder(context);
        KeyGenerator keygen(context);
        PublicKey pk;
        keygen.createPublicKey(pk);
        RelinKeys rlk = keygen.createRelinKeys();
        GaloisKeys gk = keygen.createGaloisKeys(std::vector<int>(steps, steps + nsteps));
        Encryptor encryptor(context, pk);
        Decryptor decryptor(context, keygen.secretKey());
        Evaluator ev(context);
        const double scale = std::ldexp(1.0, scale_bits);
        const size_t slots = n / 2;
        std::mt19937_64 gen(7);
        std::uniform_real_distribution<double> u(-1.0, 1.0);
        std::vector<std::complex<double>> v(slots), w(slots);
        for (size_t i = 0; i < slots; i++) {
            v[i] = {u(gen), u(gen)};
            w[i] = {u(gen), u(gen)};
        }
        Plaintext pv, pw;
        encoder.encode(v, scale, pv);
        encoder.encode(w, scale, pw);
        Ciphertext a, b;
        encryptor.encrypt(pv, a);
        encryptor.encrypt(pw, b);
        auto chain = [&](int step, Ciphertext &m) {
            ev.multiply(a, b, m);
            ev.relinearizeInplace(m, rlk);
            ev.rescaleToNextInplace(m);
            ev.rotateVectorInplace(m, step, gk);
        };
        Ciphertext m;
        for (int i = 0; i < 2; i++) chain(steps[i % nsteps], m);  // warm-up
        cudaDeviceSynchronize();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
        int last = 0;
        for (int i = 0; i < ops; i++) {
            last = steps[i % nsteps];
            chain(last, m);
        }
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_per_op = ms / ops;
        Plaintext p;
        decryptor.decrypt(m, p);
        std::vector<std::complex<double>> got;
        encoder.decode(p, got);
        double err = 0;
        for (size_t i = 0; i < slots; i++) {
            const size_t j = (i + (size_t)last) % slots;
            err = std::max(err, std::abs(got[i] - v[j] * w[j]));
        }
        *max_err = err;
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    } catch (...) {
        return 1;
    }
}

// The same for BFV / BGV (scheme 1 / 3) with plain modulus t: multiply,
// relinearizeInplace, rotateRowsInplace(1) one ciphertext pair per call (the uneven
// batch's chain at one of its shapes). *ok = 1 when the last op decrypts to the slot
// products rotated by one inside each row.
extern "C" int ref_gpu_batch_chain(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t, int ops,
                                   double *ms_per_op, int *ok) {
    try {
        KernelProvider::initialize();
        EncryptionParameters parms((SchemeType)scheme);
        parms.setPolyModulusDegree(n);
        std::vector<Modulus> q;
        for (int i = 0; i < count; i++) q.emplace_back(moduli[i]);
        parms.setCoeffModulus(q);
        parms.setPlainModulus(t);
        SEALContext context(parms, true, SecurityLevel::none);
        BatchEncoder encoder(context);
        KeyGenerator keygen(context);
        PublicKey pk;
        keygen.createPublicKey(pk);
        RelinKeys rlk = keygen.createRelinKeys();
        GaloisKeys gk = keygen.createGaloisKeys(std::vector<int>{1});
        Encryptor encryptor(context, pk);
        Decryptor decryptor(context, keygen.secretKey());
        Evaluator ev(context);
        std::mt19937_64 gen(11);
        std::vector<uint64_t> v(n), w(n);
        for (size_t i = 0; i < n; i++) {
            v[i] = gen() % t;
            w[i] = gen() % t;
        }
        Plaintext pv, pw;
        encoder.encode(v, pv);
        encoder.encode(w, pw);
        Ciphertext a, b;
        encryptor.encrypt(pv, a);
        encryptor.encrypt(pw, b);
        auto chain = [&](Ciphertext &m) {
            ev.multiply(a, b, m);
            ev.relinearizeInplace(m, rlk);
            ev.rotateRowsInplace(m, 1, gk);
        };
        Ciphertext m;
        for (int i = 0; i < 2; i++) chain(m);  // warm-up
        cudaDeviceSynchronize();
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, 0);
        for (int i = 0; i < ops; i++) chain(m);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        *ms_per_op = ms / ops;
        Plaintext p;
        decryptor.decrypt(m, p);
        std::vector<uint64_t> got;
        encoder.decode(p, got);
        const size_t half = n / 2;
        int good = got.size() == n;
        for (size_t i = 0; good && i < n; i++) {
            const size_t row = i / half, j = row * half + (i % half + 1) % half;
            good = got[i] == (uint64_t)((unsigned __int128)v[j] * w[j] % t);
        }
        *ok = good;
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    } catch (...) {
        return 1;
    }
}

// The reference GPU path's symmetric encryption of a batch-encoded (BFV, `values`) or
// CKKS-encoded (`reals`, at `scale`) plaintext under a seeded Blake2xb factory: its
// seed-compressed wire bytes (save) and the words its own loader (load with a
// context) expands them to. bytes: cap bytes, *len written; words: 2 * L * n.
extern "C" int ref_gpu_seeded_ct(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t,
                                 const uint64_t *seed8, const uint64_t *values, const double *reals, size_t nvalues,
                                 double scale, char *bytes, size_t cap, size_t *len, uint64_t *words, uint64_t *seed_out) {
    try {
        KernelProvider::initialize();
        troy::EncryptionParameters host((SchemeType)scheme);
        host.setPolyModulusDegree(n);
        std::vector<Modulus> q;
        for (int i = 0; i < count; i++) q.emplace_back(moduli[i]);
        host.setCoeffModulus(q);
        if ((SchemeType)scheme != SchemeType::ckks) host.setPlainModulus(Modulus(t));
        troy::PRNGSeed seed;
        std::copy_n(seed8, 8, seed.begin());
        host.setRandomGenerator(std::make_shared<troy::Blake2xbPRNGFactory>(seed));
        EncryptionParameters parms(host);
        SEALContext context(parms, true, SecurityLevel::none);
        KeyGenerator keygen(context);
        Encryptor encryptor(context, keygen.secretKey());
        Plaintext p;
        if ((SchemeType)scheme == SchemeType::ckks) {
            CKKSEncoder encoder(context);
            std::vector<std::complex<double>> v(nvalues);
            for (size_t i = 0; i < nvalues; i++) v[i] = {reals[i], 0.0};
            encoder.encode(v, scale, p);
        } else {
            BatchEncoder encoder(context);
            std::vector<uint64_t> v(values, values + nvalues);
            encoder.encode(v, p);
        }
        Ciphertext c = encryptor.encryptSymmetric(p);
        *seed_out = c.seed();
        std::ostringstream os;
        c.save(os);
        const std::string b = os.str();
        if (b.size() > cap) return 3;
        std::memcpy(bytes, b.data(), b.size());
        *len = b.size();
        Ciphertext back;
        std::istringstream is(b);
        back.load(is, context);
        const size_t w = back.size() * back.coeffModulusSize() * back.polyModulusDegree();
        cudaMemcpy(words, back.data().get(), w * 8, cudaMemcpyDeviceToHost);
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    } catch (...) {
        return 1;
    }
}

// The reverse direction: wire bytes of a ciphertext made elsewhere (here: this
// library's seed-compressed symmetric encryption) loaded by the reference GPU path's
// own loader with a context (CiphertextCuda::load, src/ciphertext_cuda.cu:137-184),
// decrypted with the secret key of the same seeded factory and decoded: BFV slots
// into values, CKKS real parts into reals (nvalues of them). words: 2 * L * n, the
// loaded ciphertext.
extern "C" int ref_gpu_load_decrypt(int scheme, size_t n, const uint64_t *moduli, int count, uint64_t t,
                                    const uint64_t *seed8, const char *bytes, size_t len, uint64_t *values,
                                    double *reals, size_t nvalues, uint64_t *words) {
    try {
        KernelProvider::initialize();
        troy::EncryptionParameters host((SchemeType)scheme);
        host.setPolyModulusDegree(n);
        std::vector<Modulus> q;
        for (int i = 0; i < count; i++) q.emplace_back(moduli[i]);
        host.setCoeffModulus(q);
        if ((SchemeType)scheme != SchemeType::ckks) host.setPlainModulus(Modulus(t));
        troy::PRNGSeed seed;
        std::copy_n(seed8, 8, seed.begin());
        host.setRandomGenerator(std::make_shared<troy::Blake2xbPRNGFactory>(seed));
        EncryptionParameters parms(host);
        SEALContext context(parms, true, SecurityLevel::none);
        KeyGenerator keygen(context);
        Ciphertext c;
        std::istringstream is(std::string(bytes, len));
        c.load(is, context);
        const size_t w = c.size() * c.coeffModulusSize() * c.polyModulusDegree();
        cudaMemcpy(words, c.data().get(), w * 8, cudaMemcpyDeviceToHost);
        Decryptor decryptor(context, keygen.secretKey());
        Plaintext p;
        decryptor.decrypt(c, p);
        if ((SchemeType)scheme == SchemeType::ckks) {
            CKKSEncoder encoder(context);
            std::vector<std::complex<double>> v;
            encoder.decode(p, v);
            for (size_t i = 0; i < nvalues && i < v.size(); i++) reals[i] = v[i].real();
        } else {
            BatchEncoder encoder(context);
            std::vector<uint64_t> v;
            encoder.decode(p, v);
            for (size_t i = 0; i < nvalues && i < v.size(); i++) values[i] = v[i];
        }
        return cudaGetLastError() == cudaSuccess ? 0 : 2;
    } catch (...) {
        return 1;
    }
}

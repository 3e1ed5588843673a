// Linear layers on encrypted data: the reference's app layer (app/LinearHelper.cuh:
// Plain2d, Cipher2d, MatmulHelper, Conv2dHelper) with its coefficient encodings and
// wire formats. Every sum of ciphertext x plaintext products of one call runs as one
// device pass (each ciphertext transformed once, each plaintext lifted and
// transformed once, all products accumulated in one kernel, one inverse transform
// per output) instead of one multiplyPlain and addInplace per pair; the sums are exact,
// so the words equal the reference's.
#pragma once

#include <cstdint>
#include <iosfwd>
#include <utility>
#include <vector>

#include "troy_b200.hpp"

namespace troyn {

class Cipher2d;

class Plain2d {
public:
    std::vector<std::vector<Plaintext>> data;
    std::vector<Plaintext> &operator[](std::size_t i) { return data[i]; }
    const std::vector<Plaintext> &operator[](std::size_t i) const { return data[i]; }
    // Symmetric encryption of every plaintext (Plain2d::encrypt, app/LinearHelper.cuh:167-180).
    Cipher2d encrypt(const Encryptor &encryptor) const;
};

class Cipher2d {
public:
    std::vector<std::vector<Ciphertext>> data;
    std::vector<Ciphertext> &operator[](std::size_t i) { return data[i]; }
    const std::vector<Ciphertext> &operator[](std::size_t i) const { return data[i]; }
    // Rows x columns header then every ciphertext (app/LinearHelper.cuh:44-90).
    void save(std::ostream &stream) const;
    void load(std::istream &stream);
    void load(std::istream &stream, const SEALContext &context);
    void modSwitchToNext(const Evaluator &evaluator);
    void addInplace(const Evaluator &evaluator, const Cipher2d &x);
    void addPlainInplace(const Evaluator &evaluator, const Plain2d &x);
    Cipher2d addPlain(const Evaluator &evaluator, const Plain2d &x) const;
};

// Sums of ciphertext x plaintext products on the device: output o is
// sum_{k in [off[o], off[o+1])} cts[ia[k]] * pts[iw[k]], the words of the reference's
// multiplyPlain of each pair followed by addInplace. The ciphertexts share level, size,
// form, scale and correction factor. Coefficient-form ciphertexts (BFV/BGV) take
// coefficient plaintexts: each ciphertext and plaintext is transformed once, one
// inverse transform per output. NTT-form ciphertexts (CKKS, or BFV/BGV after
// transformToNtt) take NTT plaintexts of the same parms_id and scale, multiplied in
// place with no transform at all.
std::vector<Ciphertext> sumOfProducts(const Evaluator &evaluator, const std::vector<const Ciphertext *> &cts,
                                      const std::vector<const Plaintext *> &pts, const std::vector<uint32_t> &off,
                                      const std::vector<uint32_t> &ia, const std::vector<uint32_t> &iw);

// Block shape of MatmulHelper::determineBlock (app/LinearHelper.cuh:206-228).
struct MatmulPlan {
    std::size_t batch = 0, in = 0, out = 0, slots = 0;
    std::size_t batchBlock = 0, inputBlock = 0, outputBlock = 0;
    static MatmulPlan make(std::size_t batch, std::size_t in, std::size_t out, std::size_t slots);
    std::size_t batchBlocks() const { return (batch + batchBlock - 1) / batchBlock; }
    std::size_t inputBlocks() const { return (in + inputBlock - 1) / inputBlock; }
    std::size_t outputBlocks() const { return (out + outputBlock - 1) / outputBlock; }
};

// MatmulHelper (app/LinearHelper.cuh:197-530): y = x W for a batch of row vectors.
class MatmulHelper {
public:
    MatmulHelper(std::size_t batch, std::size_t in, std::size_t out, std::size_t slots)
        : plan_(MatmulPlan::make(batch, in, out, slots)) {}
    const MatmulPlan &plan() const { return plan_; }
    Plain2d encodeWeights(const BatchEncoder &encoder, const std::uint64_t *weights) const;
    Plain2d encodeInputs(const BatchEncoder &encoder, const std::uint64_t *inputs) const;
    Cipher2d encryptInputs(const Encryptor &encryptor, const BatchEncoder &encoder, const std::uint64_t *inputs) const;
    Cipher2d matmul(const Evaluator &evaluator, const Cipher2d &a, const Plain2d &w) const;
    // ciphertext weights (products of ciphertexts, size-3 results, not relinearized)
    Cipher2d matmulCipher(const Evaluator &evaluator, const Cipher2d &a, const Cipher2d &w) const;
    // plaintext inputs, ciphertext weights
    Cipher2d matmulReverse(const Evaluator &evaluator, const Plain2d &a, const Cipher2d &w) const;
    Plain2d encodeOutputs(const BatchEncoder &encoder, const std::uint64_t *outputs) const;
    std::vector<std::uint64_t> decryptOutputs(const BatchEncoder &encoder, Decryptor &decryptor,
                                              const Cipher2d &outputs) const;
    // Only the coefficients holding outputs travel (saveTerms / loadTerms).
    void serializeOutputs(const Evaluator &evaluator, const Cipher2d &x, std::ostream &stream) const;
    Cipher2d deserializeOutputs(const Evaluator &evaluator, std::istream &stream) const;
    void serializeEncodedWeights(const Plain2d &w, std::ostream &stream) const;
    Plain2d deserializeEncodedWeights(std::istream &stream) const;

private:
    std::vector<std::size_t> outputTerms(std::size_t li, std::size_t lj) const;
    MatmulPlan plan_;
};

// Geometry shared by the convolution helpers (app/LinearHelper.cuh:531-975 and
// app/LinearHelperCKKS.cuh:362-716): images larger than sqrt(slots) split into blocks
// that overlap by kernel - 1; `channel_slots` input channels share one polynomial.
struct ConvGeometry {
    std::size_t batch, ih, iw, kh, kw, ic, oc, slots, bh, bw;
    bool blocked;
    ConvGeometry(std::size_t batch, std::size_t ih, std::size_t iw, std::size_t kh, std::size_t kw, std::size_t ic,
                 std::size_t oc, std::size_t slots);
    std::size_t block() const { return bh * bw; }
    std::size_t channelSlots() const { return slots / block(); }
    std::size_t splitsH() const { return (ih - kh + 1 + bh - kh) / (bh - kh + 1); }
    std::size_t splitsW() const { return (iw - kw + 1 + bw - kw) / (bw - kw + 1); }
    std::size_t totalBatchSize() const { return blocked ? batch * splitsH() * splitsW() : batch; }
    std::size_t outputCount() const { return batch * oc * (ih - kh + 1) * (iw - kw + 1); }
    // coefficient vectors: [output channel][channel group] of flipped kernels, and
    // [block][channel group] of image blocks
    template <class T>
    std::vector<std::vector<std::vector<T>>> weightVectors(const std::vector<T> &weights) const;
    template <class T>
    std::vector<std::vector<std::vector<T>>> inputVectors(const std::vector<T> &inputs) const;
    // (coefficient, output index) of every output held by block b's polynomials
    std::vector<std::pair<std::size_t, std::size_t>> outputMap(std::size_t b, std::size_t channel) const;
    // the last channel slot, which every output polynomial's outputs lie in
    std::vector<std::size_t> outputTerms() const;
};

// Conv2dHelper (app/LinearHelper.cuh:531-975): a "valid" 2-d convolution of
// batch x input-channels x height x width images with output-channels x
// input-channels x kh x kw kernels; images larger than sqrt(slots) are split into
// overlapping blocks.
class Conv2dHelper {
public:
    Conv2dHelper(std::size_t batch, std::size_t image_height, std::size_t image_width, std::size_t kernel_height,
                 std::size_t kernel_width, std::size_t input_channels, std::size_t output_channels,
                 std::size_t slots)
        : g_(batch, image_height, image_width, kernel_height, kernel_width, input_channels, output_channels, slots) {}
    std::size_t totalBatchSize() const { return g_.totalBatchSize(); }
    Plain2d encodeWeights(const BatchEncoder &encoder, const std::vector<std::uint64_t> &weights) const;
    Plain2d encodeInputs(const BatchEncoder &encoder, const std::vector<std::uint64_t> &inputs) const;
    Cipher2d encryptInputs(const Encryptor &encryptor, const BatchEncoder &encoder,
                           const std::vector<std::uint64_t> &inputs) const;
    Cipher2d conv2d(const Evaluator &evaluator, const Cipher2d &a, const Plain2d &w) const;
    Cipher2d conv2dCipher(const Evaluator &evaluator, const Cipher2d &a, const Cipher2d &w) const;
    Cipher2d conv2dReverse(const Evaluator &evaluator, const Plain2d &a, const Cipher2d &w) const;
    Plain2d encodeOutputs(const BatchEncoder &encoder, const std::vector<std::uint64_t> &outputs) const;
    void addPlainInplace(const Evaluator &evaluator, Cipher2d &y, const Plain2d &x) const { y.addPlainInplace(evaluator, x); }
    void addInplace(const Evaluator &evaluator, Cipher2d &y, const Cipher2d &x) const { y.addInplace(evaluator, x); }
    std::vector<std::uint64_t> decryptOutputs(const BatchEncoder &encoder, Decryptor &decryptor,
                                              const Cipher2d &outputs) const;
    void serializeOutputs(const Evaluator &evaluator, const Cipher2d &x, std::ostream &stream) const;
    Cipher2d deserializeOutputs(const Evaluator &evaluator, std::istream &stream) const;

private:
    ConvGeometry g_;
};

// Output (b, o) = sum over channel groups i of a[b][i] * w[o][i] (the convolution
// helpers' sums), fused.
Cipher2d convolve(const Evaluator &evaluator, const ConvGeometry &g, const Cipher2d &a, const Plain2d &w);

}  // namespace troyn

// The reference's namespace for these classes (app/LinearHelper.cuh:7).
namespace LinearHelper {
using troyn::Cipher2d;
using troyn::Conv2dHelper;
using troyn::MatmulHelper;
using troyn::Plain2d;
}  // namespace LinearHelper

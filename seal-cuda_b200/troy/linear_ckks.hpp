// CKKS linear layers on encrypted data.
//
// LinearHelperCKKS::MatmulHelper / Conv2dHelper (app/LinearHelperCKKS.cuh): the BFV
// helpers' coefficient layouts over CKKS encodePolynomial (N real coefficients), the
// encoded weights kept in the helper. Products are NTT-form dyadic products, so a
// call's whole sum of products is one accumulate kernel with no transform.
//
// troyn::DiagonalMatmulHelper (app/matmul.cuh MatmulHelper): a height x width complex
// matrix times a vector packed `packNum` times into the slots, by the diagonal method:
// sum over diagonals i of rotate(v, i) * diag_i, an optional rescale, then
// log2(next_pow2(width) / cipherCount) rotate-and-add folds. The diagonal rotations of
// one call run as one batched Galois launch and the products as one accumulate kernel.
#pragma once

#include <complex>
#include <cstdint>
#include <iosfwd>
#include <vector>

#include "linear.hpp"

namespace LinearHelperCKKS {

using Plain2d = troyn::Plain2d;
using Cipher2d = troyn::Cipher2d;

// MatmulHelper (app/LinearHelperCKKS.cuh:104-360): y = x W, one row of x at a time.
class MatmulHelper {
public:
    Plain2d encodedWeights;
    MatmulHelper(std::size_t batchSize, std::size_t inputDims, std::size_t outputDims, std::size_t slotCount);
    std::size_t blockHeight() const { return bh_; }
    std::size_t blockWidth() const { return bw_; }
    void encodeWeights(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                       const std::vector<double> &weights, double scale);
    Plain2d encodeInputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                         const std::vector<double> &inputs, double scale) const;
    Cipher2d encryptInputs(const troyn::Encryptor &encryptor, const troyn::CKKSEncoder &encoder,
                           const troyn::ParmsID &parmsID, const std::vector<double> &inputs, double scale) const;
    Cipher2d matmul(const troyn::Evaluator &evaluator, const Cipher2d &a) const;
    Plain2d encodeOutputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                          const std::vector<double> &outputs, double scale) const;
    void addPlainInplace(const troyn::Evaluator &evaluator, Cipher2d &y, const Plain2d &x) const {
        y.addPlainInplace(evaluator, x);
    }
    std::vector<double> decryptOutputs(const troyn::CKKSEncoder &encoder, troyn::Decryptor &decryptor,
                                       const Cipher2d &outputs) const;
    void serializeOutputs(const troyn::Evaluator &evaluator, const Cipher2d &x, std::ostream &stream) const;
    Cipher2d deserializeOutputs(const troyn::Evaluator &evaluator, std::istream &stream) const;

private:
    std::vector<std::size_t> outputTerms(std::size_t li) const;
    std::size_t batch_, in_, out_, slots_, bh_ = 0, bw_ = 0;
};

// Conv2dHelper (app/LinearHelperCKKS.cuh:362-716): the BFV convolution layout with
// 2 x slotCount (= N) coefficients per polynomial.
class Conv2dHelper {
public:
    Plain2d encodedWeights;
    Conv2dHelper(std::size_t batchSize, std::size_t imageHeight, std::size_t imageWidth, std::size_t kernelHeight,
                 std::size_t kernelWidth, std::size_t inputChannels, std::size_t outputChannels,
                 std::size_t slotCount)
        : g_(batchSize, imageHeight, imageWidth, kernelHeight, kernelWidth, inputChannels, outputChannels,
             slotCount * 2) {}
    std::size_t totalBatchSize() const { return g_.totalBatchSize(); }
    void encodeWeights(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                       const std::vector<double> &weights, double scale);
    Plain2d encodeInputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                         const std::vector<double> &inputs, double scale) const;
    Cipher2d encryptInputs(const troyn::Encryptor &encryptor, const troyn::CKKSEncoder &encoder,
                           const troyn::ParmsID &parmsID, const std::vector<double> &inputs, double scale) const;
    Cipher2d conv2d(const troyn::Evaluator &evaluator, const Cipher2d &a) const;
    Plain2d encodeOutputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                          const std::vector<double> &outputs, double scale) const;
    void addPlainInplace(const troyn::Evaluator &evaluator, Cipher2d &y, const Plain2d &x) const {
        y.addPlainInplace(evaluator, x);
    }
    void addInplace(const troyn::Evaluator &evaluator, Cipher2d &y, const Cipher2d &x) const {
        y.addInplace(evaluator, x);
    }
    std::vector<double> decryptOutputs(const troyn::CKKSEncoder &encoder, troyn::Decryptor &decryptor,
                                       const Cipher2d &outputs) const;
    void serializeOutputs(const troyn::Evaluator &evaluator, const Cipher2d &x, std::ostream &stream) const;
    Cipher2d deserializeOutputs(const troyn::Evaluator &evaluator, std::istream &stream) const;

private:
    troyn::ConvGeometry g_;
};

}  // namespace LinearHelperCKKS

namespace troyn {

// The diagonal-method CKKS matrix-vector product of app/matmul.cuh:5-123.
class DiagonalMatmulHelper {
public:
    DiagonalMatmulHelper(std::size_t height, std::size_t width, std::size_t slot_count);
    std::size_t packNum() const { return pack_; }
    std::size_t cipherCount() const { return count_; }
    // the input repeated packNum times, next_pow2(width) slots apart (prepareInput)
    Plaintext prepareInput(const std::vector<std::complex<double>> &input, const CKKSEncoder &encoder,
                           double scale) const;
    std::vector<std::complex<double>> decodeResult(const Plaintext &plain, const CKKSEncoder &encoder) const;
    // packs the height x width matrix and encodes its cipherCount diagonals (encode)
    void encode(const std::vector<std::vector<std::complex<double>>> &matrix, const CKKSEncoder &encoder,
                double scale);
    Ciphertext multiply(const Ciphertext &repeated_vector, const Evaluator &evaluator, const GaloisKeys &galois_keys,
                        bool rescale) const;

private:
    std::vector<Plaintext> encoded_;
    std::vector<bool> zero_;
    DeviceBuffer diagonals_;   // the encoded diagonals back to back, for the accumulate kernel
    std::size_t height_, width_, slots_, pack_, count_;
};

}  // namespace troyn

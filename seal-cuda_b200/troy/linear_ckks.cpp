// CKKS linear layers (app/LinearHelperCKKS.cuh) and the diagonal CKKS matrix-vector
// product (app/matmul.cuh) over the library's batched device operations.
#include "linear_ckks.hpp"

#include <algorithm>
#include <cmath>
#include <istream>
#include <ostream>
#include <stdexcept>

#include "device_util.hpp"

namespace LinearHelperCKKS {

using troyn::Ciphertext;
using troyn::Plaintext;

namespace {

std::size_t ceil_div(std::size_t a, std::size_t b) { return (a + b - 1) / b; }

Plaintext encode_poly(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &id, const std::vector<double> &v,
                      double scale) {
    Plaintext pt;
    encoder.encodePolynomial(v, id, scale, pt);
    return pt;
}

Plain2d encode_rows(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &id,
                    const std::vector<std::vector<std::vector<double>>> &rows, double scale) {
    Plain2d out;
    for (auto &r : rows) {
        std::vector<Plaintext> row;
        for (auto &v : r) row.push_back(encode_poly(encoder, id, v, scale));
        out.data.push_back(std::move(row));
    }
    return out;
}

}  // namespace

// ------------------------------------------------------------------ MatmulHelper

// determineBlock (app/LinearHelperCKKS.cuh:113-124): the block height i and width
// min(N / i, out) with the fewest ciphertexts ceil(in / i) + ceil(out / width).
MatmulHelper::MatmulHelper(std::size_t batchSize, std::size_t inputDims, std::size_t outputDims,
                           std::size_t slotCount)
    : batch_(batchSize), in_(inputDims), out_(outputDims), slots_(slotCount * 2) {
    if (!batchSize || !inputDims || !outputDims || !slotCount) throw std::invalid_argument("matmul dimensions must be positive");
    std::size_t best = in_ + out_ + 1;
    for (std::size_t i = 1; i < in_ + 1 && slots_ / i > 0; i++) {
        const std::size_t w = std::min(slots_ / i, out_);
        const std::size_t t = ceil_div(in_, i) + ceil_div(out_, w);
        if (t < best) {
            bh_ = i;
            bw_ = w;
            best = t;
        }
    }
    if (!bh_) throw std::invalid_argument("matmul shape does not fit the slot count");
}

// encodeWeights / encodeWeightSmall (app/LinearHelperCKKS.cuh:126-183): weight (i, j)
// of a block at coefficient (j - lj) * blockHeight + blockHeight - 1 - (i - li).
void MatmulHelper::encodeWeights(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                 const std::vector<double> &weights, double scale) {
    if (weights.size() != in_ * out_) throw std::invalid_argument("Weight size incorrect.");
    encodedWeights.data.clear();
    for (std::size_t li = 0; li < in_; li += bh_) {
        const std::size_t ui = std::min(li + bh_, in_);
        std::vector<Plaintext> row;
        for (std::size_t lj = 0; lj < out_; lj += bw_) {
            const std::size_t uj = std::min(lj + bw_, out_);
            std::vector<double> vec(slots_, 0.0);
            for (std::size_t j = lj; j < uj; j++)
                for (std::size_t i = li; i < ui; i++) vec[(j - lj) * bh_ + bh_ - (i - li) - 1] = weights[i * out_ + j];
            row.push_back(encode_poly(encoder, parmsID, vec, scale));
        }
        encodedWeights.data.push_back(std::move(row));
    }
}

// encodeInputs (app/LinearHelperCKKS.cuh:185-210): each row in blockHeight pieces.
Plain2d MatmulHelper::encodeInputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                   const std::vector<double> &inputs, double scale) const {
    if (inputs.size() != in_ * batch_) throw std::invalid_argument("Input size incorrect.");
    Plain2d out;
    for (std::size_t i = 0; i < batch_; i++) {
        std::vector<Plaintext> row;
        for (std::size_t lj = 0; lj < in_; lj += bh_) {
            const std::size_t uj = std::min(lj + bh_, in_);
            std::vector<double> vec(inputs.begin() + i * in_ + lj, inputs.begin() + i * in_ + uj);
            row.push_back(encode_poly(encoder, parmsID, vec, scale));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

Cipher2d MatmulHelper::encryptInputs(const troyn::Encryptor &encryptor, const troyn::CKKSEncoder &encoder,
                                     const troyn::ParmsID &parmsID, const std::vector<double> &inputs,
                                     double scale) const {
    return encodeInputs(encoder, parmsID, inputs, scale).encrypt(encryptor);
}

// matmul (app/LinearHelperCKKS.cuh:229-251): output (b, j) = sum_i a[b][i] * w[i][j],
// all outputs of the call in one accumulate kernel.
Cipher2d MatmulHelper::matmul(const troyn::Evaluator &ev, const Cipher2d &a) const {
    if (a.data.size() != batch_) throw std::invalid_argument("Input batchsize incorrect.");
    const std::size_t ni = encodedWeights.data.size();
    if (!ni) throw std::logic_error("Encoded weights not set.");
    const std::size_t no = encodedWeights[0].size();
    std::vector<const Ciphertext *> cts;
    std::vector<const Plaintext *> pts;
    for (auto &row : a.data) {
        if (row.size() != ni) throw std::invalid_argument("Input dimension incorrect.");
        for (auto &c : row) cts.push_back(&c);
    }
    for (auto &row : encodedWeights.data) {
        if (row.size() != no) throw std::invalid_argument("Weight output dimension incorrect.");
        for (auto &p : row) pts.push_back(&p);
    }
    std::vector<std::uint32_t> off{0}, ia, iw;
    for (std::size_t b = 0; b < batch_; b++)
        for (std::size_t j = 0; j < no; j++) {
            for (std::size_t i = 0; i < ni; i++) {
                ia.push_back((std::uint32_t)(b * ni + i));
                iw.push_back((std::uint32_t)(i * no + j));
            }
            off.push_back((std::uint32_t)ia.size());
        }
    auto flat = troyn::sumOfProducts(ev, cts, pts, off, ia, iw);
    Cipher2d out;
    out.data.resize(batch_);
    for (std::size_t b = 0; b < batch_; b++)
        for (std::size_t j = 0; j < no; j++) out.data[b].push_back(std::move(flat[b * no + j]));
    return out;
}

// encodeOutputs (app/LinearHelperCKKS.cuh:253-279): output t of a block at
// coefficient (t - li + 1) * blockHeight - 1.
Plain2d MatmulHelper::encodeOutputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                    const std::vector<double> &outputs, double scale) const {
    if (outputs.size() != batch_ * out_) throw std::invalid_argument("Output size incorrect.");
    Plain2d ret;
    for (std::size_t i = 0; i < batch_; i++) {
        std::vector<Plaintext> row;
        for (std::size_t li = 0; li < out_; li += bw_) {
            const std::size_t ui = std::min(li + bw_, out_);
            std::vector<double> vec(slots_, 0.0);
            for (std::size_t t = li; t < ui; t++) vec[(t - li) * bh_ + bh_ - 1] = outputs[i * out_ + t];
            row.push_back(encode_poly(encoder, parmsID, vec, scale));
        }
        ret.data.push_back(std::move(row));
    }
    return ret;
}

std::vector<double> MatmulHelper::decryptOutputs(const troyn::CKKSEncoder &encoder, troyn::Decryptor &decryptor,
                                                 const Cipher2d &outputs) const {
    std::vector<double> dec(batch_ * out_);
    for (std::size_t i = 0; i < batch_; i++) {
        std::size_t cid = 0;
        for (std::size_t li = 0; li < out_; li += bw_, cid++) {
            const std::size_t ui = std::min(li + bw_, out_);
            Plaintext pt;
            decryptor.decrypt(outputs.data.at(i).at(cid), pt);
            std::vector<double> buf;
            encoder.decodePolynomial(pt, buf);
            for (std::size_t j = li; j < ui; j++) dec[i * out_ + j] = buf[(j - li + 1) * bh_ - 1];
        }
    }
    return dec;
}

std::vector<std::size_t> MatmulHelper::outputTerms(std::size_t li) const {
    const std::size_t ui = std::min(li + bw_, out_);
    std::vector<std::size_t> r(ui - li);
    for (std::size_t j = li; j < ui; j++) r[j - li] = (j - li + 1) * bh_ - 1;
    return r;
}

// serializeOutputs / deserializeOutputs (app/LinearHelperCKKS.cuh:319-357).
void MatmulHelper::serializeOutputs(const troyn::Evaluator &ev, const Cipher2d &x, std::ostream &s) const {
    for (std::size_t i = 0; i < batch_; i++) {
        std::size_t cid = 0;
        for (std::size_t li = 0; li < out_; li += bw_, cid++) x.data.at(i).at(cid).saveTerms(s, ev, outputTerms(li));
    }
}

Cipher2d MatmulHelper::deserializeOutputs(const troyn::Evaluator &ev, std::istream &s) const {
    Cipher2d ret;
    for (std::size_t i = 0; i < batch_; i++) {
        std::vector<Ciphertext> row;
        for (std::size_t li = 0; li < out_; li += bw_) {
            Ciphertext c;
            c.loadTerms(s, ev, outputTerms(li));
            row.push_back(std::move(c));
        }
        ret.data.push_back(std::move(row));
    }
    return ret;
}

// ------------------------------------------------------------------ Conv2dHelper

void Conv2dHelper::encodeWeights(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                 const std::vector<double> &weights, double scale) {
    encodedWeights = encode_rows(encoder, parmsID, g_.weightVectors(weights), scale);
}

Plain2d Conv2dHelper::encodeInputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                   const std::vector<double> &inputs, double scale) const {
    return encode_rows(encoder, parmsID, g_.inputVectors(inputs), scale);
}

Cipher2d Conv2dHelper::encryptInputs(const troyn::Encryptor &encryptor, const troyn::CKKSEncoder &encoder,
                                     const troyn::ParmsID &parmsID, const std::vector<double> &inputs,
                                     double scale) const {
    return encodeInputs(encoder, parmsID, inputs, scale).encrypt(encryptor);
}

// conv2d (app/LinearHelperCKKS.cuh:572-593).
Cipher2d Conv2dHelper::conv2d(const troyn::Evaluator &ev, const Cipher2d &a) const {
    if (encodedWeights.data.empty()) throw std::logic_error("Encoded weights not set.");
    return troyn::convolve(ev, g_, a, encodedWeights);
}

// encodeOutputs (app/LinearHelperCKKS.cuh:595-634): one mask vector reused across
// outputs, as the reference.
Plain2d Conv2dHelper::encodeOutputs(const troyn::CKKSEncoder &encoder, const troyn::ParmsID &parmsID,
                                    const std::vector<double> &outputs, double scale) const {
    if (outputs.size() != g_.outputCount()) throw std::invalid_argument("Outputs shape incorrect.");
    std::vector<double> mask(g_.channelSlots() * g_.block(), 0.0);
    Plain2d out;
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++) {
        std::vector<Plaintext> group;
        for (std::size_t c = 0; c < g_.oc; c++) {
            for (auto &[mi, oi] : g_.outputMap(b, c)) mask[mi] = outputs[oi];
            group.push_back(encode_poly(encoder, parmsID, mask, scale));
        }
        out.data.push_back(std::move(group));
    }
    return out;
}

std::vector<double> Conv2dHelper::decryptOutputs(const troyn::CKKSEncoder &encoder, troyn::Decryptor &decryptor,
                                                 const Cipher2d &outputs) const {
    std::vector<double> ret(g_.outputCount());
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++)
        for (std::size_t c = 0; c < g_.oc; c++) {
            Plaintext pt;
            decryptor.decrypt(outputs.data.at(b).at(c), pt);
            std::vector<double> buf;
            encoder.decodePolynomial(pt, buf);
            for (auto &[mi, oi] : g_.outputMap(b, c)) ret[oi] = buf[mi];
        }
    return ret;
}

void Conv2dHelper::serializeOutputs(const troyn::Evaluator &ev, const Cipher2d &x, std::ostream &s) const {
    const auto required = g_.outputTerms();
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++)
        for (std::size_t oc = 0; oc < g_.oc; oc++) x.data.at(b).at(oc).saveTerms(s, ev, required);
}

Cipher2d Conv2dHelper::deserializeOutputs(const troyn::Evaluator &ev, std::istream &s) const {
    const auto required = g_.outputTerms();
    Cipher2d out;
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++) {
        std::vector<Ciphertext> row(g_.oc);
        for (auto &c : row) c.loadTerms(s, ev, required);
        out.data.push_back(std::move(row));
    }
    return out;
}

}  // namespace LinearHelperCKKS

namespace troyn {

namespace {

// nextPow2 (app/matmul.cuh:15): 2^ceil(log(v) / log(2)) in double precision.
std::size_t next_pow2(std::size_t v) {
    return (std::size_t)(int)std::pow(2.0, std::ceil(std::log((double)v) / std::log(2.0)));
}

}  // namespace

DiagonalMatmulHelper::DiagonalMatmulHelper(std::size_t height, std::size_t width, std::size_t slot_count)
    : height_(height), width_(width), slots_(slot_count) {
    if (!height || !width || !slot_count) throw std::invalid_argument("matrix dimensions must be positive");
    if (next_pow2(width) > slot_count) throw std::invalid_argument("Width exceeds the slot count.");
    pack_ = slots_ / next_pow2(width);
    count_ = (std::size_t)std::ceil((float)next_pow2(height) / (float)pack_);
    // the repacked diagonal index is below next_pow2(width): more diagonals than that
    // would lose rows
    if (count_ > next_pow2(width)) throw std::invalid_argument("Matrix too tall for the diagonal packing.");
}

// prepareInput (app/matmul.cuh:19-32).
Plaintext DiagonalMatmulHelper::prepareInput(const std::vector<std::complex<double>> &input,
                                             const CKKSEncoder &encoder, double scale) const {
    if (input.size() != width_) throw std::invalid_argument("Input size should equal Width.");
    std::vector<std::complex<double>> v(slots_);
    const std::size_t p2 = next_pow2(width_);
    for (std::size_t col = 0; col < width_; col++)
        for (std::size_t idx = 0; idx < pack_; idx++) v[col + p2 * idx] = input[col];
    Plaintext pt;
    encoder.encode(v, scale, pt);
    return pt;
}

// decodeResult (app/matmul.cuh:34-43): row i at slot (i mod cipherCount) +
// next_pow2(width) * (i / cipherCount).
std::vector<std::complex<double>> DiagonalMatmulHelper::decodeResult(const Plaintext &plain,
                                                                     const CKKSEncoder &encoder) const {
    std::vector<std::complex<double>> dec;
    encoder.decode(plain, dec);
    std::vector<std::complex<double>> ret(height_);
    const std::size_t p2 = next_pow2(width_);
    for (std::size_t i = 0; i < height_; i++) ret[i] = dec.at((i % count_) + p2 * (i / count_));
    return ret;
}

// encode (app/matmul.cuh:45-90): rows packed cipherCount at a time, then repacked
// into generalized diagonals; a diagonal with every |value|^2 <= 1e-6 is skipped by
// multiply.
void DiagonalMatmulHelper::encode(const std::vector<std::vector<std::complex<double>>> &matrix,
                                  const CKKSEncoder &encoder, double scale) {
    if (matrix.size() != height_) throw std::invalid_argument("Matrix height incorrect.");
    for (auto &r : matrix)
        if (r.size() != width_) throw std::invalid_argument("Matrix width incorrect.");
    const int cc = (int)count_, p2 = (int)next_pow2(width_);
    std::vector<std::vector<std::complex<double>>> pack(count_, std::vector<std::complex<double>>(slots_));
    for (int row = 0; row < (int)height_; row++)
        for (int col = 0; col < (int)width_; col++) pack[row % cc][col + p2 * (row / cc)] = matrix[row][col];
    const int mod_mask = cc - 1, wrap_mask = p2 - 1, slots = (int)slots_;
    std::vector<std::vector<std::complex<double>>> diag(count_, std::vector<std::complex<double>>(slots_));
    for (int ct = 0; ct < cc; ct++)
        for (int col = 0; col < slots; col++) {
            const int dl = (col - ct) & wrap_mask & mod_mask;
            const int dh = (col ^ ct) & slots & mod_mask;
            const int cl = (col - dl) & wrap_mask;
            const int ch = (p2 * (col / p2)) ^ dh;
            diag[dh + dl][ch + cl] = pack[ct][col];
        }
    encoded_.clear();
    zero_.clear();
    for (std::size_t i = 0; i < count_; i++) {
        bool zero = true;
        for (auto &p : diag[i])
            if (p.real() * p.real() + p.imag() * p.imag() > 1e-6) zero = false;
        Plaintext pt;
        encoder.encode(diag[i], scale, pt);
        encoded_.push_back(std::move(pt));
        zero_.push_back(zero);
    }
    const std::size_t w = encoded_[0].coeffCount();
    diagonals_ = DeviceBuffer(count_ * w);
    for (std::size_t i = 0; i < count_; i++)
        detail::cuda_ok(cudaMemcpyAsync(diagonals_.get() + i * w, encoded_[i].data(), w * 8, cudaMemcpyDeviceToDevice, 0),
                        "device copy");
}

// multiply (app/matmul.cuh:98-121).
Ciphertext DiagonalMatmulHelper::multiply(const Ciphertext &v, const Evaluator &ev, const GaloisKeys &gk,
                                          bool rescale) const {
    if (encoded_.empty()) throw std::logic_error("Encoded matrix not set.");
    const SEALContext &ctx = ev.context();
    if (ctx.scheme() != SchemeType::ckks) throw std::logic_error("unsupported scheme");
    // the reference accumulates into the diagonal-0 product and fails when it is skipped
    if (zero_[0]) throw std::invalid_argument("the matrix's first diagonal is zero");
    if (gk.parmsID() != ctx.keyParmsID()) throw std::invalid_argument("galois_keys is not valid for encryption parameters");
    if (!v.isNttForm() || v.size() != 2) throw std::invalid_argument("encrypted must be a size-2 NTT-form ciphertext");
    if (v.parmsID() != encoded_[0].parmsID())
        throw std::invalid_argument("encrypted_ntt and plain_ntt parameter mismatch");
    auto d = ctx.getContextData(v.parmsID());
    const int L = d->levelLimbs();
    const std::size_t n = ctx.polyModulusDegree(), ctw = 2 * (std::size_t)L * n;
    const double scale = v.scale() * encoded_[0].scale();
    if (!isScaleWithinBounds(scale, *d)) throw std::invalid_argument("scale out of bounds");
    tb_context *h = ctx.handle();

    // rotated copies: slot 0 the input; then the steps whose keys are present, rotated
    // by one grouped launch; then any step that needs a NAF chain of rotations
    std::vector<int> direct, chained;
    std::vector<std::uint32_t> elts;
    std::vector<const std::uint64_t *> keys;
    for (std::size_t i = 1; i < count_; i++) {
        if (zero_[i]) continue;
        std::uint32_t elt = 0;
        detail::tb_ok(tb_galois_elt_from_step(h, (int)i, &elt));
        if (gk.hasKeyElt(elt)) {
            direct.push_back((int)i);
            elts.push_back(elt);
            keys.push_back(gk.key(GaloisKeys::getIndex(elt)));
        } else {
            chained.push_back((int)i);
        }
    }
    const std::size_t slots = 1 + direct.size() + chained.size();
    DeviceBuffer R(slots * ctw);
    detail::cuda_ok(cudaMemcpyAsync(R.get(), v.data(), ctw * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
    if (!direct.empty()) {
        DeviceBuffer in(direct.size() * ctw);
        for (std::size_t k = 0; k < direct.size(); k++)
            detail::cuda_ok(cudaMemcpyAsync(in.get() + k * ctw, v.data(), ctw * 8, cudaMemcpyDeviceToDevice, 0),
                            "device copy");
        std::vector<std::uint64_t> counts(direct.size(), 1);
        detail::tb_ok(tb_apply_galois_groups(h, L, (int)direct.size(), elts.data(), counts.data(), in.get(), 0,
                                             R.get() + ctw, 0, keys.data(), nullptr));
    }
    for (std::size_t k = 0; k < chained.size(); k++) {
        Ciphertext t;
        ev.rotateVector(v, chained[k], gk, t);
        detail::cuda_ok(cudaMemcpyAsync(R.get() + (1 + direct.size() + k) * ctw, t.data(), ctw * 8,
                                        cudaMemcpyDeviceToDevice, 0),
                        "device copy");
    }
    // one output: sum over slots s of R[s] * diagonal(step of s)
    std::vector<std::uint32_t> off{0, (std::uint32_t)slots}, ia, iw;
    ia.push_back(0);
    iw.push_back(0);
    for (std::size_t k = 0; k < direct.size(); k++) {
        ia.push_back((std::uint32_t)(1 + k));
        iw.push_back((std::uint32_t)direct[k]);
    }
    for (std::size_t k = 0; k < chained.size(); k++) {
        ia.push_back((std::uint32_t)(1 + direct.size() + k));
        iw.push_back((std::uint32_t)chained[k]);
    }
    DeviceBuffer doff = detail::upload_u32(off), dia = detail::upload_u32(ia), diw = detail::upload_u32(iw);
    Ciphertext result(ctx, v.parmsID(), 2);
    detail::tb_ok(tb_dyadic_accumulate(h, L, 2, R.get(), 0, diagonals_.get(), 0, result.data(), 0,
                                       (const std::uint32_t *)doff.get(), (const std::uint32_t *)dia.get(),
                                       (const std::uint32_t *)diw.get(), 1, nullptr));
    result.isNttForm() = true;
    result.scale() = scale;
    if (rescale) ev.rescaleToNextInplace(result);
    const std::size_t p2 = next_pow2(width_);
    for (std::size_t rot = count_; rot < p2; rot *= 2) {
        Ciphertext t;
        ev.rotateVector(result, (int)rot, gk, t);
        ev.addInplace(result, t);
    }
    return result;
}

}  // namespace troyn

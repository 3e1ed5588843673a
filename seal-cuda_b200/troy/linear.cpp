// Plain2d, Cipher2d, MatmulHelper and Conv2dHelper (app/LinearHelper.cuh) over the
// library's fused device sum of products.
#include "linear.hpp"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <istream>
#include <ostream>
#include <stdexcept>
#include <string>

namespace troyn {

namespace {

std::size_t ceil_div(std::size_t a, std::size_t b) { return (a + b - 1) / b; }

void cuda_ok(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

void tb_ok(int st) {
    if (st == TB_OK) return;
    if (st == TB_ERR_INVALID_ARGUMENT) throw std::invalid_argument(tb_last_error());
    if (st == TB_ERR_UNSUPPORTED) throw std::logic_error(tb_last_error());
    throw std::runtime_error(tb_last_error());
}

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

// uint32 arrays travel packed two per device word.
DeviceBuffer upload_u32(const std::vector<uint32_t> &v) {
    std::vector<uint64_t> w((v.size() + 1) / 2, 0);
    if (!v.empty()) std::memcpy(w.data(), v.data(), v.size() * 4);
    DeviceBuffer b;
    b.fromHost(w.data(), w.size());
    return b;
}

void check_rect(std::size_t a, std::size_t b) {
    if (a != b) throw std::invalid_argument("Size incorrect.");
}

}  // namespace

// ------------------------------------------------------------------ Plain2d / Cipher2d

Cipher2d Plain2d::encrypt(const Encryptor &encryptor) const {
    Cipher2d out;
    for (auto &row : data) {
        std::vector<Ciphertext> r;
        for (auto &pt : row) {
            Ciphertext c;
            encryptor.encryptSymmetric(pt, c);
            r.push_back(std::move(c));
        }
        out.data.push_back(std::move(r));
    }
    return out;
}

void Cipher2d::save(std::ostream &s) const {
    const std::size_t n = data.size();
    if (!n) return;
    const std::size_t m = data[0].size();
    for (auto &row : data)
        if (row.size() != m) throw std::invalid_argument("Not a rectangle Conv2d.");
    put(s, n);
    put(s, m);
    for (auto &row : data)
        for (auto &c : row) c.save(s);
}

void Cipher2d::load(std::istream &s) {
    const auto n = get<std::size_t>(s), m = get<std::size_t>(s);
    if (n > (1u << 24) || m > (1u << 24)) throw std::invalid_argument("Cipher2d too large");
    data.assign(n, std::vector<Ciphertext>(m));
    for (auto &row : data)
        for (auto &c : row) c.load(s);
}

void Cipher2d::load(std::istream &s, const SEALContext &context) {
    const auto n = get<std::size_t>(s), m = get<std::size_t>(s);
    if (n > (1u << 24) || m > (1u << 24)) throw std::invalid_argument("Cipher2d too large");
    data.assign(n, std::vector<Ciphertext>(m));
    for (auto &row : data)
        for (auto &c : row) c.load(s, context);
}

void Cipher2d::modSwitchToNext(const Evaluator &ev) {
    for (auto &row : data)
        for (auto &c : row) ev.modSwitchToNextInplace(c);
}

void Cipher2d::addInplace(const Evaluator &ev, const Cipher2d &x) {
    check_rect(data.size(), x.data.size());
    for (std::size_t i = 0; i < data.size(); i++) {
        check_rect(data[i].size(), x[i].size());
        for (std::size_t j = 0; j < data[i].size(); j++) ev.addInplace(data[i][j], x[i][j]);
    }
}

void Cipher2d::addPlainInplace(const Evaluator &ev, const Plain2d &x) {
    check_rect(data.size(), x.data.size());
    for (std::size_t i = 0; i < data.size(); i++) {
        check_rect(data[i].size(), x[i].size());
        for (std::size_t j = 0; j < data[i].size(); j++) ev.addPlainInplace(data[i][j], x[i][j]);
    }
}

Cipher2d Cipher2d::addPlain(const Evaluator &ev, const Plain2d &x) const {
    Cipher2d out = *this;
    out.addPlainInplace(ev, x);
    return out;
}

// ------------------------------------------------------------------ fused sums of products

std::vector<Ciphertext> sumOfProducts(const Evaluator &ev, const std::vector<const Ciphertext *> &cts,
                                      const std::vector<const Plaintext *> &pts, const std::vector<uint32_t> &off,
                                      const std::vector<uint32_t> &ia, const std::vector<uint32_t> &iw) {
    const SEALContext &ctx = ev.context();
    if (ctx.scheme() != SchemeType::bfv && ctx.scheme() != SchemeType::bgv) throw std::logic_error("unsupported scheme");
    if (cts.empty() || off.size() < 2) throw std::invalid_argument("no products");
    const Ciphertext &first = *cts[0];
    auto d = ctx.getContextData(first.parmsID());
    if (!d) throw std::invalid_argument("encrypted is not valid for encryption parameters");
    const int L = d->levelLimbs();
    const std::size_t n = ctx.polyModulusDegree(), ctw = 2 * (std::size_t)L * n, ptw = (std::size_t)L * n;
    const std::size_t na = cts.size(), np = pts.size(), no = off.size() - 1;
    for (std::size_t k = 0; k < ia.size(); k++)
        if (ia[k] >= na || iw[k] >= np) throw std::invalid_argument("product index out of range");
    DeviceBuffer A(na * ctw), Wr(np * n), Wn(np * ptw), O(no * ctw);
    for (std::size_t i = 0; i < na; i++) {
        const Ciphertext &c = *cts[i];
        if (c.parmsID() != first.parmsID() || c.size() != 2 || c.isNttForm() ||
            c.correctionFactor() != first.correctionFactor())
            throw std::invalid_argument("ciphertexts must be size-2, coefficient form, one level and correction factor");
        cuda_ok(cudaMemcpyAsync(A.get() + i * ctw, c.data(), ctw * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
    }
    Wr.zero();
    for (std::size_t j = 0; j < np; j++) {
        const Plaintext &pt = *pts[j];
        if (pt.isNttForm() || pt.coeffCount() > n) throw std::invalid_argument("plaintexts must be in coefficient form");
        if (pt.coeffCount())
            cuda_ok(cudaMemcpyAsync(Wr.get() + j * n, pt.data(), pt.coeffCount() * 8, cudaMemcpyDeviceToDevice, 0),
                    "device copy");
    }
    DeviceBuffer doff = upload_u32(off), dia = upload_u32(ia), diw = upload_u32(iw);
    tb_context *h = ctx.handle();
    tb_ok(tb_ntt_forward(h, A.get(), A.get(), 2 * na, 0, L, 0, nullptr));
    tb_ok(tb_plain_to_ntt(h, L, Wr.get(), n, n, Wn.get(), np, nullptr));
    tb_ok(tb_dyadic_accumulate(h, L, 2, A.get(), 0, Wn.get(), 0, O.get(), 0, (const uint32_t *)doff.get(),
                               (const uint32_t *)dia.get(), (const uint32_t *)diw.get(), (uint32_t)no, nullptr));
    tb_ok(tb_ntt_inverse(h, O.get(), O.get(), 2 * no, 0, L, 0, nullptr));
    std::vector<Ciphertext> out;
    out.reserve(no);
    for (std::size_t o = 0; o < no; o++) {
        Ciphertext c(ctx, first.parmsID(), 2);
        cuda_ok(cudaMemcpyAsync(c.data(), O.get() + o * ctw, ctw * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
        c.correctionFactor() = first.correctionFactor();
        out.push_back(std::move(c));
    }
    return out;
}

// ------------------------------------------------------------------ MatmulHelper

MatmulPlan MatmulPlan::make(std::size_t batch, std::size_t in, std::size_t out, std::size_t slots) {
    if (!batch || !in || !out || !slots) throw std::invalid_argument("matmul dimensions must be positive");
    MatmulPlan p;
    p.batch = batch;
    p.in = in;
    p.out = out;
    p.slots = slots;
    std::size_t best = 2147483647;
    for (std::size_t b = batch; b >= 1; b--) {
        const std::size_t bc = ceil_div(batch, b);
        if (b >= slots) continue;
        if (bc * 2 > best) continue;
        for (std::size_t i = 1; i < slots / b; i++) {
            const std::size_t o = std::min(slots / b / i, out);
            if (i > in || o < 1) continue;
            const std::size_t c = bc * (ceil_div(in, i) + ceil_div(out, o));
            if (c >= best) continue;
            p.batchBlock = b;
            p.inputBlock = i;
            p.outputBlock = o;
            best = c;
        }
    }
    if (!p.batchBlock) throw std::invalid_argument("matmul shape does not fit the slot count");
    return p;
}

Plain2d MatmulHelper::encodeWeights(const BatchEncoder &encoder, const uint64_t *weights) const {
    const auto &p = plan_;
    Plain2d out;
    for (std::size_t li = 0; li < p.in; li += p.inputBlock) {
        const std::size_t ui = std::min(li + p.inputBlock, p.in);
        std::vector<Plaintext> row;
        for (std::size_t lj = 0; lj < p.out; lj += p.outputBlock) {
            const std::size_t uj = std::min(lj + p.outputBlock, p.out);
            std::vector<uint64_t> vec(p.inputBlock * p.outputBlock, 0);
            for (std::size_t j = lj; j < uj; j++)
                for (std::size_t i = li; i < ui; i++)
                    vec[(j - lj) * p.inputBlock + p.inputBlock - (i - li) - 1] = weights[i * p.out + j];
            Plaintext pt;
            encoder.encodePolynomial(vec, pt);
            row.push_back(std::move(pt));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

Plain2d MatmulHelper::encodeInputs(const BatchEncoder &encoder, const uint64_t *inputs) const {
    const auto &p = plan_;
    Plain2d out;
    for (std::size_t li = 0; li < p.batch; li += p.batchBlock) {
        const std::size_t ui = std::min(li + p.batchBlock, p.batch);
        std::vector<Plaintext> row;
        for (std::size_t lj = 0; lj < p.in; lj += p.inputBlock) {
            const std::size_t uj = std::min(lj + p.inputBlock, p.in);
            std::vector<uint64_t> vec(p.slots, 0);
            for (std::size_t i = li; i < ui; i++)
                for (std::size_t j = lj; j < uj; j++)
                    vec[(i - li) * p.inputBlock * p.outputBlock + (j - lj)] = inputs[i * p.in + j];
            Plaintext pt;
            encoder.encodePolynomial(vec, pt);
            row.push_back(std::move(pt));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

Cipher2d MatmulHelper::encryptInputs(const Encryptor &encryptor, const BatchEncoder &encoder,
                                     const uint64_t *inputs) const {
    return encodeInputs(encoder, inputs).encrypt(encryptor);
}

// matmul (app/LinearHelper.cuh:323-346): output (b, j) = sum_i a[b][i] * w[i][j].
Cipher2d MatmulHelper::matmul(const Evaluator &ev, const Cipher2d &a, const Plain2d &w) const {
    const auto &p = plan_;
    const std::size_t nb = p.batchBlocks(), ni = p.inputBlocks(), no = p.outputBlocks();
    if (a.data.size() != nb) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != ni) throw std::invalid_argument("Weight input dimension incorrect.");
    std::vector<const Ciphertext *> cts;
    std::vector<const Plaintext *> pts;
    for (std::size_t b = 0; b < nb; b++) {
        if (a[b].size() != ni) throw std::invalid_argument("Input dimension incorrect.");
        for (auto &c : a[b]) cts.push_back(&c);
    }
    for (std::size_t i = 0; i < ni; i++) {
        if (w[i].size() != no) throw std::invalid_argument("Weight output dimension incorrect.");
        for (auto &pt : w[i]) pts.push_back(&pt);
    }
    std::vector<uint32_t> off{0}, ia, iw;
    for (std::size_t b = 0; b < nb; b++)
        for (std::size_t j = 0; j < no; j++) {
            for (std::size_t i = 0; i < ni; i++) {
                ia.push_back((uint32_t)(b * ni + i));
                iw.push_back((uint32_t)(i * no + j));
            }
            off.push_back((uint32_t)ia.size());
        }
    auto flat = sumOfProducts(ev, cts, pts, off, ia, iw);
    Cipher2d out;
    out.data.resize(nb);
    for (std::size_t b = 0; b < nb; b++)
        for (std::size_t j = 0; j < no; j++) out.data[b].push_back(std::move(flat[b * no + j]));
    return out;
}

// matmulCipher (app/LinearHelper.cuh:348-370): ciphertext weights, one multiply and
// addInplace per pair as the reference (size-3 results).
Cipher2d MatmulHelper::matmulCipher(const Evaluator &ev, const Cipher2d &a, const Cipher2d &w) const {
    const auto &p = plan_;
    const std::size_t nb = p.batchBlocks(), ni = p.inputBlocks(), no = p.outputBlocks();
    if (a.data.size() != nb) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != ni) throw std::invalid_argument("Weight input dimension incorrect.");
    Cipher2d out;
    for (std::size_t b = 0; b < nb; b++) {
        std::vector<Ciphertext> row(no);
        for (std::size_t i = 0; i < ni; i++)
            for (std::size_t j = 0; j < no; j++) {
                Ciphertext prod;
                ev.multiply(a[b][i], w[i][j], prod);
                if (i == 0)
                    row[j] = std::move(prod);
                else
                    ev.addInplace(row[j], prod);
            }
        out.data.push_back(std::move(row));
    }
    return out;
}

// matmulReverse (app/LinearHelper.cuh:372-394): plaintext inputs times ciphertext weights.
Cipher2d MatmulHelper::matmulReverse(const Evaluator &ev, const Plain2d &a, const Cipher2d &w) const {
    const auto &p = plan_;
    const std::size_t nb = p.batchBlocks(), ni = p.inputBlocks(), no = p.outputBlocks();
    if (a.data.size() != nb) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != ni) throw std::invalid_argument("Weight input dimension incorrect.");
    std::vector<const Ciphertext *> cts;
    std::vector<const Plaintext *> pts;
    for (std::size_t i = 0; i < ni; i++) {
        if (w[i].size() != no) throw std::invalid_argument("Weight output dimension incorrect.");
        for (auto &c : w[i]) cts.push_back(&c);
    }
    for (std::size_t b = 0; b < nb; b++) {
        if (a[b].size() != ni) throw std::invalid_argument("Input dimension incorrect.");
        for (auto &pt : a[b]) pts.push_back(&pt);
    }
    std::vector<uint32_t> off{0}, ia, iw;
    for (std::size_t b = 0; b < nb; b++)
        for (std::size_t j = 0; j < no; j++) {
            for (std::size_t i = 0; i < ni; i++) {
                ia.push_back((uint32_t)(i * no + j));
                iw.push_back((uint32_t)(b * ni + i));
            }
            off.push_back((uint32_t)ia.size());
        }
    auto flat = sumOfProducts(ev, cts, pts, off, ia, iw);
    Cipher2d out;
    out.data.resize(nb);
    for (std::size_t b = 0; b < nb; b++)
        for (std::size_t j = 0; j < no; j++) out.data[b].push_back(std::move(flat[b * no + j]));
    return out;
}

std::vector<std::size_t> MatmulHelper::outputTerms(std::size_t li, std::size_t lj) const {
    const auto &p = plan_;
    const std::size_t ui = std::min(li + p.batchBlock, p.batch), uj = std::min(lj + p.outputBlock, p.out);
    std::vector<std::size_t> r;
    for (std::size_t i = li; i < ui; i++)
        for (std::size_t j = lj; j < uj; j++)
            r.push_back((i - li) * p.inputBlock * p.outputBlock + (j - lj) * p.inputBlock + p.inputBlock - 1);
    return r;
}

// encodeOutputs (app/LinearHelper.cuh:396-420): values at the output coefficients.
Plain2d MatmulHelper::encodeOutputs(const BatchEncoder &encoder, const uint64_t *outputs) const {
    const auto &p = plan_;
    Plain2d out;
    for (std::size_t li = 0; li < p.batch; li += p.batchBlock) {
        const std::size_t ui = std::min(li + p.batchBlock, p.batch);
        std::vector<Plaintext> row;
        for (std::size_t lj = 0; lj < p.out; lj += p.outputBlock) {
            const std::size_t uj = std::min(lj + p.outputBlock, p.out);
            std::vector<uint64_t> buf(p.slots, 0);
            for (std::size_t i = li; i < ui; i++)
                for (std::size_t j = lj; j < uj; j++)
                    buf[(i - li) * p.inputBlock * p.outputBlock + (j - lj) * p.inputBlock + p.inputBlock - 1] =
                        outputs[i * p.out + j];
            Plaintext pt;
            encoder.encodePolynomial(buf, pt);
            row.push_back(std::move(pt));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

std::vector<uint64_t> MatmulHelper::decryptOutputs(const BatchEncoder &encoder, Decryptor &decryptor,
                                                   const Cipher2d &outputs) const {
    const auto &p = plan_;
    std::vector<uint64_t> dec(p.batch * p.out);
    std::size_t di = 0;
    for (std::size_t li = 0; li < p.batch; li += p.batchBlock, di++) {
        const std::size_t ui = std::min(li + p.batchBlock, p.batch);
        std::size_t dj = 0;
        for (std::size_t lj = 0; lj < p.out; lj += p.outputBlock, dj++) {
            const std::size_t uj = std::min(lj + p.outputBlock, p.out);
            Plaintext pt;
            decryptor.decrypt(outputs.data.at(di).at(dj), pt);
            std::vector<uint64_t> buf;
            encoder.decodePolynomial(pt, buf);
            for (std::size_t i = li; i < ui; i++)
                for (std::size_t j = lj; j < uj; j++)
                    dec[i * p.out + j] =
                        buf[(i - li) * p.inputBlock * p.outputBlock + (j - lj) * p.inputBlock + p.inputBlock - 1];
        }
    }
    return dec;
}

// serializeOutputs / deserializeOutputs (app/LinearHelper.cuh:490-528).
void MatmulHelper::serializeOutputs(const Evaluator &ev, const Cipher2d &x, std::ostream &s) const {
    const auto &p = plan_;
    std::size_t di = 0;
    for (std::size_t li = 0; li < p.batch; li += p.batchBlock, di++) {
        std::size_t dj = 0;
        for (std::size_t lj = 0; lj < p.out; lj += p.outputBlock, dj++)
            x.data.at(di).at(dj).saveTerms(s, ev, outputTerms(li, lj));
    }
}

Cipher2d MatmulHelper::deserializeOutputs(const Evaluator &ev, std::istream &s) const {
    const auto &p = plan_;
    Cipher2d out;
    for (std::size_t li = 0; li < p.batch; li += p.batchBlock) {
        std::vector<Ciphertext> row;
        for (std::size_t lj = 0; lj < p.out; lj += p.outputBlock) {
            Ciphertext c;
            c.loadTerms(s, ev, outputTerms(li, lj));
            row.push_back(std::move(c));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

// serializeEncodedWeights / deserializeEncodedWeights (app/LinearHelper.cuh:453-488).
void MatmulHelper::serializeEncodedWeights(const Plain2d &w, std::ostream &s) const {
    const std::size_t rows = w.data.size();
    if (!rows) throw std::invalid_argument("No rows in weight matrix.");
    const std::size_t cols = w[0].size();
    if (!cols) throw std::invalid_argument("No columns in weight matrix.");
    for (auto &r : w.data)
        if (r.size() != cols) throw std::invalid_argument("Weight matrix is not rectangular.");
    put(s, rows);
    put(s, cols);
    for (auto &r : w.data)
        for (auto &pt : r) pt.save(s);
}

Plain2d MatmulHelper::deserializeEncodedWeights(std::istream &s) const {
    const auto rows = get<std::size_t>(s), cols = get<std::size_t>(s);
    if (rows > (1u << 24) || cols > (1u << 24)) throw std::invalid_argument("weight matrix too large");
    Plain2d out;
    out.data.assign(rows, std::vector<Plaintext>(cols));
    for (auto &r : out.data)
        for (auto &pt : r) pt.load(s);
    return out;
}

// ------------------------------------------------------------------ Conv2dHelper

Conv2dHelper::Conv2dHelper(std::size_t batch, std::size_t image_height, std::size_t image_width,
                           std::size_t kernel_height, std::size_t kernel_width, std::size_t input_channels,
                           std::size_t output_channels, std::size_t slots)
    : batch_(batch), kh_(kernel_height), kw_(kernel_width), ih_(image_height), iw_(image_width), ic_(input_channels),
      oc_(output_channels), slots_(slots) {
    if (!batch || !image_height || !image_width || !kernel_height || !kernel_width || !input_channels ||
        !output_channels || !slots)
        throw std::invalid_argument("convolution dimensions must be positive");
    if (kernel_height > image_height || kernel_width > image_width) throw std::invalid_argument("kernel larger than image");
    const std::size_t max_size = (std::size_t)std::sqrt((double)slots);
    if (image_height > max_size || image_width > max_size) {
        bh_ = bw_ = max_size;
        blocked_ = true;
    } else {
        bh_ = image_height;
        bw_ = image_width;
        blocked_ = false;
    }
    if (blocked_ && (kernel_height > bh_ || kernel_width > bw_)) throw std::invalid_argument("kernel larger than a block");
}

std::size_t Conv2dHelper::totalBatchSize() const {
    if (!blocked_) return batch_;
    const std::size_t kh = kh_ - 1, kw = kw_ - 1;
    return batch_ * ceil_div(ih_ - kh, bh_ - kh) * ceil_div(iw_ - kw, bw_ - kw);
}

// encodeWeights (app/LinearHelper.cuh:626-661): each output channel's kernels for a
// group of input channels, reversed, in one coefficient-encoded plaintext.
Plain2d Conv2dHelper::encodeWeights(const BatchEncoder &encoder, const std::vector<uint64_t> &weights) const {
    if (weights.size() != ic_ * oc_ * kh_ * kw_) throw std::invalid_argument("Weights shape incorrect.");
    const std::size_t block = bh_ * bw_, channel_slots = slots_ / block;
    Plain2d out;
    for (std::size_t oc = 0; oc < oc_; oc++) {
        std::vector<Plaintext> row;
        for (std::size_t lic = 0; lic < ic_; lic += channel_slots) {
            const std::size_t uic = std::min(lic + channel_slots, ic_);
            std::vector<uint64_t> spread(channel_slots * block, 0);
            for (std::size_t j = lic; j < uic; j++)
                for (std::size_t ki = 0; ki < kh_; ki++)
                    for (std::size_t kj = 0; kj < kw_; kj++)
                        spread[(channel_slots - 1 - (j - lic)) * block + ki * bw_ + kj] =
                            weights[((oc * ic_) + j) * (kh_ * kw_) + (kh_ - ki - 1) * kw_ + (kw_ - kj - 1)];
            Plaintext pt;
            encoder.encodePolynomial(spread, pt);
            row.push_back(std::move(pt));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

// encodeInputs (app/LinearHelper.cuh:674-740): blocks of the images (overlapping by
// kernel - 1 when blocked), channel groups per plaintext.
Plain2d Conv2dHelper::encodeInputs(const BatchEncoder &encoder, const std::vector<uint64_t> &inputs) const {
    if (inputs.size() != batch_ * ic_ * ih_ * iw_) throw std::invalid_argument("Inputs shape incorrect.");
    const std::size_t total = totalBatchSize(), block = bh_ * bw_;
    std::vector<uint64_t> split;
    if (!blocked_) {
        split = inputs;
    } else {
        const std::size_t kh = kh_ - 1, kw = kw_ - 1;
        const std::size_t sh = ceil_div(ih_ - kh, bh_ - kh), sw = ceil_div(iw_ - kw, bw_ - kw);
        split.assign(batch_ * sh * sw * ic_ * block, 0);
        const std::size_t image = ih_ * iw_;
        for (std::size_t b = 0; b < batch_; b++)
            for (std::size_t i = 0; i < sh; i++)
                for (std::size_t j = 0; j < sw; j++) {
                    const std::size_t bid = b * sh * sw + i * sw + j;
                    const std::size_t si = i * (bh_ - kh), sj = j * (bw_ - kw);
                    const std::size_t ui = (si + bh_ >= ih_) ? ih_ : (si + bh_);
                    const std::size_t uj = (sj + bw_ >= iw_) ? iw_ : (sj + bw_);
                    for (std::size_t tc = 0; tc < ic_; tc++)
                        for (std::size_t ti = 0; ti < ui - si; ti++)
                            for (std::size_t tj = 0; tj < uj - sj; tj++)
                                split[bid * block * ic_ + tc * block + ti * bw_ + tj] =
                                    inputs[b * image * ic_ + tc * image + (si + ti) * iw_ + (sj + tj)];
                }
    }
    const std::size_t channel_slots = slots_ / block;
    Plain2d out;
    for (std::size_t b = 0; b < total; b++) {
        std::vector<Plaintext> group;
        for (std::size_t c = 0; c < ic_; c += channel_slots) {
            const std::size_t upper = std::min(c + channel_slots, ic_);
            std::vector<uint64_t> plain(slots_, 0);
            for (std::size_t k = 0; k < upper - c; k++)
                for (std::size_t i = 0; i < bh_; i++)
                    for (std::size_t j = 0; j < bw_; j++)
                        plain[k * block + i * bw_ + j] = split[b * ic_ * block + (c + k) * block + i * bw_ + j];
            Plaintext pt;
            encoder.encodePolynomial(plain, pt);
            group.push_back(std::move(pt));
        }
        out.data.push_back(std::move(group));
    }
    return out;
}

Cipher2d Conv2dHelper::encryptInputs(const Encryptor &encryptor, const BatchEncoder &encoder,
                                     const std::vector<uint64_t> &inputs) const {
    return encodeInputs(encoder, inputs).encrypt(encryptor);
}

// conv2d (app/LinearHelper.cuh:752-773): output (b, oc) = sum_i a[b][i] * w[oc][i].
Cipher2d Conv2dHelper::conv2d(const Evaluator &ev, const Cipher2d &a, const Plain2d &w) const {
    const std::size_t total = totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != oc_) throw std::invalid_argument("Weight output channels incorrect.");
    const std::size_t groups = a[0].size();
    std::vector<const Ciphertext *> cts;
    std::vector<const Plaintext *> pts;
    for (auto &row : a.data) {
        if (row.size() != groups) throw std::invalid_argument("Input channel groups incorrect.");
        for (auto &c : row) cts.push_back(&c);
    }
    for (auto &row : w.data) {
        if (row.size() != groups) throw std::invalid_argument("Weight channel groups incorrect.");
        for (auto &pt : row) pts.push_back(&pt);
    }
    std::vector<uint32_t> off{0}, ia, iw;
    for (std::size_t b = 0; b < total; b++)
        for (std::size_t oc = 0; oc < oc_; oc++) {
            for (std::size_t i = 0; i < groups; i++) {
                ia.push_back((uint32_t)(b * groups + i));
                iw.push_back((uint32_t)(oc * groups + i));
            }
            off.push_back((uint32_t)ia.size());
        }
    auto flat = sumOfProducts(ev, cts, pts, off, ia, iw);
    Cipher2d out;
    out.data.resize(total);
    for (std::size_t b = 0; b < total; b++)
        for (std::size_t oc = 0; oc < oc_; oc++) out.data[b].push_back(std::move(flat[b * oc_ + oc]));
    return out;
}

// conv2dCipher (app/LinearHelper.cuh:775-797): ciphertext kernels, one multiply and
// addInplace per pair as the reference.
Cipher2d Conv2dHelper::conv2dCipher(const Evaluator &ev, const Cipher2d &a, const Cipher2d &w) const {
    const std::size_t total = totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    Cipher2d out;
    for (std::size_t b = 0; b < total; b++) {
        std::vector<Ciphertext> group;
        for (std::size_t oc = 0; oc < oc_; oc++) {
            Ciphertext acc;
            for (std::size_t i = 0; i < a[b].size(); i++) {
                Ciphertext prod;
                ev.multiply(a[b][i], w.data.at(oc).at(i), prod);
                if (i == 0)
                    acc = std::move(prod);
                else
                    ev.addInplace(acc, prod);
            }
            group.push_back(std::move(acc));
        }
        out.data.push_back(std::move(group));
    }
    return out;
}

// conv2dReverse (app/LinearHelper.cuh:799-820): plaintext images, ciphertext kernels.
Cipher2d Conv2dHelper::conv2dReverse(const Evaluator &ev, const Plain2d &a, const Cipher2d &w) const {
    const std::size_t total = totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != oc_) throw std::invalid_argument("Weight output channels incorrect.");
    const std::size_t groups = a[0].size();
    std::vector<const Ciphertext *> cts;
    std::vector<const Plaintext *> pts;
    for (auto &row : w.data) {
        if (row.size() != groups) throw std::invalid_argument("Weight channel groups incorrect.");
        for (auto &c : row) cts.push_back(&c);
    }
    for (auto &row : a.data) {
        if (row.size() != groups) throw std::invalid_argument("Input channel groups incorrect.");
        for (auto &pt : row) pts.push_back(&pt);
    }
    std::vector<uint32_t> off{0}, ia, iw;
    for (std::size_t b = 0; b < total; b++)
        for (std::size_t oc = 0; oc < oc_; oc++) {
            for (std::size_t i = 0; i < groups; i++) {
                ia.push_back((uint32_t)(oc * groups + i));
                iw.push_back((uint32_t)(b * groups + i));
            }
            off.push_back((uint32_t)ia.size());
        }
    auto flat = sumOfProducts(ev, cts, pts, off, ia, iw);
    Cipher2d out;
    out.data.resize(total);
    for (std::size_t b = 0; b < total; b++)
        for (std::size_t oc = 0; oc < oc_; oc++) out.data[b].push_back(std::move(flat[b * oc_ + oc]));
    return out;
}

// encodeOutputs / decryptOutputs (app/LinearHelper.cuh:822-930): the valid output
// window sits in the last channel slot of each output polynomial.
Plain2d Conv2dHelper::encodeOutputs(const BatchEncoder &encoder, const std::vector<uint64_t> &outputs) const {
    const std::size_t block = bh_ * bw_, channel_slots = slots_ / block;
    const std::size_t yh = bh_ - kh_ + 1, yw = bw_ - kw_ + 1, oyh = ih_ - kh_ + 1, oyw = iw_ - kw_ + 1;
    if (outputs.size() != batch_ * oc_ * oyh * oyw) throw std::invalid_argument("Outputs shape incorrect.");
    const std::size_t kh = kh_ - 1, kw = kw_ - 1;
    const std::size_t sh = ceil_div(ih_ - kh, bh_ - kh), sw = ceil_div(iw_ - kw, bw_ - kw);
    std::vector<uint64_t> mask(channel_slots * block, 0);
    Plain2d out;
    for (std::size_t b = 0; b < totalBatchSize(); b++) {
        const std::size_t ob = b / (sh * sw), si = (b % (sh * sw)) / sw, sj = b % sw;
        std::vector<Plaintext> group;
        for (std::size_t c = 0; c < oc_; c++) {
            for (std::size_t i = 0; i < yh; i++)
                for (std::size_t j = 0; j < yw; j++) {
                    const std::size_t mi = (channel_slots - 1) * block + (bh_ - yh + i) * bw_ + (bw_ - yw + j);
                    if (si * yh + i < oyh && sj * yw + j < oyw)
                        mask[mi] = outputs[ob * oc_ * oyh * oyw + c * oyh * oyw + (si * yh + i) * oyw + (sj * yw + j)];
                }
            Plaintext pt;
            encoder.encodePolynomial(mask, pt);
            group.push_back(std::move(pt));
        }
        out.data.push_back(std::move(group));
    }
    return out;
}

std::vector<uint64_t> Conv2dHelper::decryptOutputs(const BatchEncoder &encoder, Decryptor &decryptor,
                                                   const Cipher2d &outputs) const {
    const std::size_t block = bh_ * bw_, channel_slots = slots_ / block;
    const std::size_t yh = bh_ - kh_ + 1, yw = bw_ - kw_ + 1, oyh = ih_ - kh_ + 1, oyw = iw_ - kw_ + 1;
    const std::size_t kh = kh_ - 1, kw = kw_ - 1;
    const std::size_t sh = ceil_div(ih_ - kh, bh_ - kh), sw = ceil_div(iw_ - kw, bw_ - kw);
    std::vector<uint64_t> ret(batch_ * oc_ * oyh * oyw);
    for (std::size_t b = 0; b < totalBatchSize(); b++) {
        const std::size_t ob = b / (sh * sw), si = (b % (sh * sw)) / sw, sj = b % sw;
        for (std::size_t c = 0; c < oc_; c++) {
            Plaintext pt;
            decryptor.decrypt(outputs.data.at(b).at(c), pt);
            std::vector<uint64_t> buf;
            encoder.decodePolynomial(pt, buf);
            for (std::size_t i = 0; i < yh; i++)
                for (std::size_t j = 0; j < yw; j++) {
                    const std::size_t mi = (channel_slots - 1) * block + (bh_ - yh + i) * bw_ + (bw_ - yw + j);
                    if (si * yh + i < oyh && sj * yw + j < oyw)
                        ret[ob * oc_ * oyh * oyw + c * oyh * oyw + (si * yh + i) * oyw + (sj * yw + j)] = buf[mi];
                }
        }
    }
    return ret;
}

// serializeOutputs / deserializeOutputs (app/LinearHelper.cuh:932-972): the whole last
// channel slot of every output travels.
void Conv2dHelper::serializeOutputs(const Evaluator &ev, const Cipher2d &x, std::ostream &s) const {
    const std::size_t block = bh_ * bw_, channel_slots = slots_ / block, st = (channel_slots - 1) * block;
    std::vector<std::size_t> required(block);
    for (std::size_t i = 0; i < block; i++) required[i] = st + i;
    for (std::size_t b = 0; b < totalBatchSize(); b++)
        for (std::size_t oc = 0; oc < oc_; oc++) x.data.at(b).at(oc).saveTerms(s, ev, required);
}

Cipher2d Conv2dHelper::deserializeOutputs(const Evaluator &ev, std::istream &s) const {
    const std::size_t block = bh_ * bw_, channel_slots = slots_ / block, st = (channel_slots - 1) * block;
    std::vector<std::size_t> required(block);
    for (std::size_t i = 0; i < block; i++) required[i] = st + i;
    Cipher2d out;
    for (std::size_t b = 0; b < totalBatchSize(); b++) {
        std::vector<Ciphertext> row(oc_);
        for (auto &c : row) c.loadTerms(s, ev, required);
        out.data.push_back(std::move(row));
    }
    return out;
}

}  // namespace troyn

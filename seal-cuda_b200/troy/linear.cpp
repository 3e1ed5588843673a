// Plain2d, Cipher2d, MatmulHelper and Conv2dHelper (app/LinearHelper.cuh) over the
// library's fused device sum of products.
#include "linear.hpp"

#include "device_util.hpp"

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

using detail::cuda_ok;
using detail::tb_ok;
using detail::upload_u32;

std::size_t ceil_div(std::size_t a, std::size_t b) { return (a + b - 1) / b; }

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
    if (cts.empty() || pts.empty() || off.size() < 2) throw std::invalid_argument("no products");
    const Ciphertext &first = *cts[0];
    auto d = ctx.getContextData(first.parmsID());
    if (!d) throw std::invalid_argument("encrypted is not valid for encryption parameters");
    const int L = d->levelLimbs();
    const bool ntt = first.isNttForm();
    const std::size_t size = first.size();
    if (size < 2) throw std::invalid_argument("encrypted is empty");
    if (!ntt && ctx.scheme() != SchemeType::bfv && ctx.scheme() != SchemeType::bgv)
        throw std::invalid_argument("encrypted must be in NTT form");
    const std::size_t n = ctx.polyModulusDegree(), ctw = size * (std::size_t)L * n, ptw = (std::size_t)L * n;
    const std::size_t na = cts.size(), np = pts.size(), no = off.size() - 1;
    if (off[0] != 0 || off[no] != ia.size() || ia.size() != iw.size()) throw std::invalid_argument("bad term lists");
    for (std::size_t o = 0; o < no; o++)
        if (off[o + 1] <= off[o]) throw std::invalid_argument("every output needs a product");
    for (std::size_t k = 0; k < ia.size(); k++)
        if (ia[k] >= na || iw[k] >= np) throw std::invalid_argument("product index out of range");
    for (const Ciphertext *c : cts)
        if (c->parmsID() != first.parmsID() || c->size() != size || c->isNttForm() != ntt ||
            c->correctionFactor() != first.correctionFactor())
            throw std::invalid_argument("encrypted1 and encrypted2 parameter mismatch");
    // An output's scale is its first product's (addInplace keeps the left operand's);
    // NTT-form products multiply the scales, each within bounds as in multiplyPlain.
    std::vector<double> scales(no);
    for (std::size_t o = 0; o < no; o++) scales[o] = cts[ia[off[o]]]->scale();
    if (ntt) {
        for (const Plaintext *p : pts) {
            if (!p->isNttForm() || p->parmsID() != first.parmsID())
                throw std::invalid_argument("encrypted_ntt and plain_ntt parameter mismatch");
            if (p->coeffCount() != ptw) throw std::invalid_argument("plain is not valid for encryption parameters");
        }
        for (std::size_t k = 0; k < ia.size(); k++)
            if (!isScaleWithinBounds(cts[ia[k]]->scale() * pts[iw[k]]->scale(), *d))
                throw std::invalid_argument("scale out of bounds");
        for (std::size_t o = 0; o < no; o++) scales[o] *= pts[iw[off[o]]]->scale();
    } else {
        for (const Plaintext *p : pts)
            if (p->isNttForm() || p->coeffCount() > n)
                throw std::invalid_argument("plain is not valid for encryption parameters");
    }
    DeviceBuffer A(na * ctw), Wn(np * ptw), O(no * ctw);
    for (std::size_t i = 0; i < na; i++)
        cuda_ok(cudaMemcpyAsync(A.get() + i * ctw, cts[i]->data(), ctw * 8, cudaMemcpyDeviceToDevice, 0),
                "device copy");
    tb_context *h = ctx.handle();
    if (ntt) {
        for (std::size_t j = 0; j < np; j++)
            cuda_ok(cudaMemcpyAsync(Wn.get() + j * ptw, pts[j]->data(), ptw * 8, cudaMemcpyDeviceToDevice, 0),
                    "device copy");
    } else {
        DeviceBuffer Wr(np * n);
        Wr.zero();
        for (std::size_t j = 0; j < np; j++)
            if (pts[j]->coeffCount())
                cuda_ok(cudaMemcpyAsync(Wr.get() + j * n, pts[j]->data(), pts[j]->coeffCount() * 8,
                                        cudaMemcpyDeviceToDevice, 0),
                        "device copy");
        tb_ok(tb_ntt_forward(h, A.get(), A.get(), size * na, 0, L, 0, nullptr));
        tb_ok(tb_plain_to_ntt(h, L, Wr.get(), n, n, Wn.get(), np, nullptr));
    }
    DeviceBuffer doff = upload_u32(off), dia = upload_u32(ia), diw = upload_u32(iw);
    tb_ok(tb_dyadic_accumulate(h, L, (int)size, A.get(), 0, Wn.get(), 0, O.get(), 0, (const uint32_t *)doff.get(),
                               (const uint32_t *)dia.get(), (const uint32_t *)diw.get(), (uint32_t)no, nullptr));
    if (!ntt) tb_ok(tb_ntt_inverse(h, O.get(), O.get(), size * no, 0, L, 0, nullptr));
    std::vector<Ciphertext> out;
    out.reserve(no);
    for (std::size_t o = 0; o < no; o++) {
        Ciphertext c(ctx, first.parmsID(), size);
        cuda_ok(cudaMemcpyAsync(c.data(), O.get() + o * ctw, ctw * 8, cudaMemcpyDeviceToDevice, 0), "device copy");
        c.isNttForm() = ntt;
        c.scale() = scales[o];
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

// ------------------------------------------------------------------ convolution geometry

ConvGeometry::ConvGeometry(std::size_t batch_, std::size_t ih_, std::size_t iw_, std::size_t kh_, std::size_t kw_,
                           std::size_t ic_, std::size_t oc_, std::size_t slots_)
    : batch(batch_), ih(ih_), iw(iw_), kh(kh_), kw(kw_), ic(ic_), oc(oc_), slots(slots_) {
    if (!batch || !ih || !iw || !kh || !kw || !ic || !oc || !slots)
        throw std::invalid_argument("convolution dimensions must be positive");
    if (kh > ih || kw > iw) throw std::invalid_argument("kernel larger than image");
    const std::size_t max_size = (std::size_t)std::sqrt((double)slots);
    blocked = ih > max_size || iw > max_size;
    bh = blocked ? max_size : ih;
    bw = blocked ? max_size : iw;
    if (kh > bh || kw > bw) throw std::invalid_argument("kernel larger than a block");
}

// encodeWeights (app/LinearHelper.cuh:626-661): channel j's kernel, flipped, at
// channel slot channel_slots - 1 - (j - first channel of the group).
template <class T>
std::vector<std::vector<std::vector<T>>> ConvGeometry::weightVectors(const std::vector<T> &weights) const {
    if (weights.size() != ic * oc * kh * kw) throw std::invalid_argument("Weights shape incorrect.");
    const std::size_t blk = block(), cs = channelSlots();
    std::vector<std::vector<std::vector<T>>> out(oc);
    for (std::size_t o = 0; o < oc; o++)
        for (std::size_t lic = 0; lic < ic; lic += cs) {
            std::vector<T> spread(cs * blk, T(0));
            for (std::size_t j = lic; j < std::min(lic + cs, ic); j++)
                for (std::size_t ki = 0; ki < kh; ki++)
                    for (std::size_t kj = 0; kj < kw; kj++)
                        spread[(cs - 1 - (j - lic)) * blk + ki * bw + kj] =
                            weights[((o * ic) + j) * (kh * kw) + (kh - ki - 1) * kw + (kw - kj - 1)];
            out[o].push_back(std::move(spread));
        }
    return out;
}

// encodeInputs (app/LinearHelper.cuh:674-742): block (b, i, j) starts at row
// i * (bh - kh + 1), column j * (bw - kw + 1) of image b; channel c + k of a group at
// channel slot k.
template <class T>
std::vector<std::vector<std::vector<T>>> ConvGeometry::inputVectors(const std::vector<T> &inputs) const {
    if (inputs.size() != batch * ic * ih * iw) throw std::invalid_argument("Inputs shape incorrect.");
    const std::size_t blk = block(), cs = channelSlots(), sh = splitsH(), sw = splitsW(), image = ih * iw;
    std::vector<std::vector<std::vector<T>>> out;
    out.reserve(totalBatchSize());
    for (std::size_t b = 0; b < batch; b++)
        for (std::size_t i = 0; i < sh; i++)
            for (std::size_t j = 0; j < sw; j++) {
                const std::size_t si = i * (bh - kh + 1), sj = j * (bw - kw + 1);
                const std::size_t ui = std::min(si + bh, ih), uj = std::min(sj + bw, iw);
                std::vector<std::vector<T>> groups;
                for (std::size_t c = 0; c < ic; c += cs) {
                    std::vector<T> plain(slots, T(0));
                    for (std::size_t k = 0; k < std::min(cs, ic - c); k++)
                        for (std::size_t ti = 0; ti < ui - si; ti++)
                            for (std::size_t tj = 0; tj < uj - sj; tj++)
                                plain[k * blk + ti * bw + tj] =
                                    inputs[b * image * ic + (c + k) * image + (si + ti) * iw + (sj + tj)];
                    groups.push_back(std::move(plain));
                }
                out.push_back(std::move(groups));
            }
    return out;
}

// decryptOutputs (app/LinearHelper.cuh:886-930): output (i, j) of block b sits at
// (channel_slots - 1) * block + (bh - yh + i) * bw + (bw - yw + j).
std::vector<std::pair<std::size_t, std::size_t>> ConvGeometry::outputMap(std::size_t b, std::size_t c) const {
    const std::size_t yh = bh - kh + 1, yw = bw - kw + 1, oyh = ih - kh + 1, oyw = iw - kw + 1;
    const std::size_t sh = splitsH(), sw = splitsW();
    const std::size_t ob = b / (sh * sw), si = (b % (sh * sw)) / sw, sj = b % sw;
    std::vector<std::pair<std::size_t, std::size_t>> m;
    for (std::size_t i = 0; i < yh; i++)
        for (std::size_t j = 0; j < yw; j++)
            if (si * yh + i < oyh && sj * yw + j < oyw)
                m.emplace_back((channelSlots() - 1) * block() + (bh - yh + i) * bw + (bw - yw + j),
                               ob * oc * oyh * oyw + c * oyh * oyw + (si * yh + i) * oyw + (sj * yw + j));
    return m;
}

std::vector<std::size_t> ConvGeometry::outputTerms() const {
    const std::size_t st = (channelSlots() - 1) * block();
    std::vector<std::size_t> r(block());
    for (std::size_t i = 0; i < r.size(); i++) r[i] = st + i;
    return r;
}

template std::vector<std::vector<std::vector<uint64_t>>> ConvGeometry::weightVectors(const std::vector<uint64_t> &) const;
template std::vector<std::vector<std::vector<double>>> ConvGeometry::weightVectors(const std::vector<double> &) const;
template std::vector<std::vector<std::vector<uint64_t>>> ConvGeometry::inputVectors(const std::vector<uint64_t> &) const;
template std::vector<std::vector<std::vector<double>>> ConvGeometry::inputVectors(const std::vector<double> &) const;

// conv2d (app/LinearHelper.cuh:752-773): output (b, oc) = sum_i a[b][i] * w[oc][i].
Cipher2d convolve(const Evaluator &ev, const ConvGeometry &g, const Cipher2d &a, const Plain2d &w) {
    const std::size_t total = g.totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != g.oc) throw std::invalid_argument("Weight output channels incorrect.");
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
        for (std::size_t oc = 0; oc < g.oc; oc++) {
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
        for (std::size_t oc = 0; oc < g.oc; oc++) out.data[b].push_back(std::move(flat[b * g.oc + oc]));
    return out;
}

// ------------------------------------------------------------------ Conv2dHelper

namespace {

Plain2d encode_rows(const BatchEncoder &encoder, const std::vector<std::vector<std::vector<uint64_t>>> &rows) {
    Plain2d out;
    for (auto &r : rows) {
        std::vector<Plaintext> row;
        for (auto &v : r) {
            Plaintext pt;
            encoder.encodePolynomial(v, pt);
            row.push_back(std::move(pt));
        }
        out.data.push_back(std::move(row));
    }
    return out;
}

}  // namespace

Plain2d Conv2dHelper::encodeWeights(const BatchEncoder &encoder, const std::vector<uint64_t> &weights) const {
    return encode_rows(encoder, g_.weightVectors(weights));
}

Plain2d Conv2dHelper::encodeInputs(const BatchEncoder &encoder, const std::vector<uint64_t> &inputs) const {
    return encode_rows(encoder, g_.inputVectors(inputs));
}

Cipher2d Conv2dHelper::encryptInputs(const Encryptor &encryptor, const BatchEncoder &encoder,
                                     const std::vector<uint64_t> &inputs) const {
    return encodeInputs(encoder, inputs).encrypt(encryptor);
}

Cipher2d Conv2dHelper::conv2d(const Evaluator &ev, const Cipher2d &a, const Plain2d &w) const {
    return convolve(ev, g_, a, w);
}

// conv2dCipher (app/LinearHelper.cuh:775-797): ciphertext kernels, one multiply and
// addInplace per pair as the reference.
Cipher2d Conv2dHelper::conv2dCipher(const Evaluator &ev, const Cipher2d &a, const Cipher2d &w) const {
    const std::size_t total = g_.totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    Cipher2d out;
    for (std::size_t b = 0; b < total; b++) {
        std::vector<Ciphertext> group;
        for (std::size_t oc = 0; oc < g_.oc; oc++) {
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
    const std::size_t total = g_.totalBatchSize();
    if (a.data.size() != total) throw std::invalid_argument("Input batchsize incorrect.");
    if (w.data.size() != g_.oc) throw std::invalid_argument("Weight output channels incorrect.");
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
        for (std::size_t oc = 0; oc < g_.oc; oc++) {
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
        for (std::size_t oc = 0; oc < g_.oc; oc++) out.data[b].push_back(std::move(flat[b * g_.oc + oc]));
    return out;
}

// encodeOutputs (app/LinearHelper.cuh:822-861). As the reference, one mask vector is
// reused across outputs, so positions a later block does not hold keep earlier values.
Plain2d Conv2dHelper::encodeOutputs(const BatchEncoder &encoder, const std::vector<uint64_t> &outputs) const {
    if (outputs.size() != g_.outputCount()) throw std::invalid_argument("Outputs shape incorrect.");
    std::vector<uint64_t> mask(g_.channelSlots() * g_.block(), 0);
    Plain2d out;
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++) {
        std::vector<Plaintext> group;
        for (std::size_t c = 0; c < g_.oc; c++) {
            for (auto &[mi, oi] : g_.outputMap(b, c)) mask[mi] = outputs[oi];
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
    std::vector<uint64_t> ret(g_.outputCount());
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++)
        for (std::size_t c = 0; c < g_.oc; c++) {
            Plaintext pt;
            decryptor.decrypt(outputs.data.at(b).at(c), pt);
            std::vector<uint64_t> buf;
            encoder.decodePolynomial(pt, buf);
            for (auto &[mi, oi] : g_.outputMap(b, c)) ret[oi] = buf[mi];
        }
    return ret;
}

// serializeOutputs / deserializeOutputs (app/LinearHelper.cuh:932-972): the whole last
// channel slot of every output travels.
void Conv2dHelper::serializeOutputs(const Evaluator &ev, const Cipher2d &x, std::ostream &s) const {
    const auto required = g_.outputTerms();
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++)
        for (std::size_t oc = 0; oc < g_.oc; oc++) x.data.at(b).at(oc).saveTerms(s, ev, required);
}

Cipher2d Conv2dHelper::deserializeOutputs(const Evaluator &ev, std::istream &s) const {
    const auto required = g_.outputTerms();
    Cipher2d out;
    for (std::size_t b = 0; b < g_.totalBatchSize(); b++) {
        std::vector<Ciphertext> row(g_.oc);
        for (auto &c : row) c.loadTerms(s, ev, required);
        out.data.push_back(std::move(row));
    }
    return out;
}

}  // namespace troyn

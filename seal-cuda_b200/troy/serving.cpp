// The continuous-batching MatmulServer over the library's batched device operations.
#include "serving.hpp"

#include "device_util.hpp"

#include <cuda_runtime_api.h>

#include <algorithm>
#include <cstring>
#include <stdexcept>
#include <string>

namespace troyn {

namespace {

using detail::cuda_ok;

// Record of tb_matmul_encode_weights: {offset lo, offset hi, in, out, ib, ob, li, lj}.
void push_block(std::vector<uint32_t> &d, uint64_t src, const MatmulPlan &p, std::size_t bi, std::size_t bj) {
    d.push_back((uint32_t)src);
    d.push_back((uint32_t)(src >> 32));
    d.push_back((uint32_t)p.in);
    d.push_back((uint32_t)p.out);
    d.push_back((uint32_t)p.inputBlock);
    d.push_back((uint32_t)p.outputBlock);
    d.push_back((uint32_t)(bi * p.inputBlock));
    d.push_back((uint32_t)(bj * p.outputBlock));
}

}  // namespace

// ------------------------------------------------------------------ server

struct MatmulServer::Wave {
    std::vector<Request> reqs;
    std::vector<std::size_t> out_base;   // first output ciphertext of each request
    std::size_t bytes = 0, out_words = 0;
    void *dev = nullptr;
    cudaEvent_t begin = nullptr, done = nullptr;
    bool failed = false;
};

namespace {

std::size_t align256(std::size_t x) { return (x + 255) & ~std::size_t(255); }

bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

}  // namespace

// Pinned staging of one slot, grown on demand (reused only after the slot's previous
// wave has finished).
struct MatmulServer::Staging {
    void *p = nullptr;
    std::size_t bytes = 0;
    void ensure(std::size_t need) {
        if (need <= bytes) return;
        if (p) cudaFreeHost(p);
        p = nullptr;
        bytes = 0;
        const std::size_t grow = std::max(need, std::max(2 * bytes, std::size_t(1) << 24));
        cuda_ok(cudaHostAlloc(&p, grow, cudaHostAllocDefault), "pinned allocation");
        bytes = grow;
    }
    ~Staging() {
        if (p) cudaFreeHost(p);
    }
};

namespace {
}  // namespace

double MatmulServer::now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

MatmulServer::MatmulServer(const SEALContext &context, Options options) : context_(context), opt_(options) {
    context.requireSet();
    if (context.scheme() != SchemeType::bfv && context.scheme() != SchemeType::bgv)
        throw std::logic_error("unsupported scheme");
    if (opt_.slots < 1 || opt_.slots > 16) throw std::invalid_argument("slots must be in [1, 16]");
    L_ = context.firstContextData()->levelLimbs();
    n_ = context.polyModulusDegree();
    for (int i = 0; i < opt_.slots; i++) {
        cudaStream_t s;
        cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream creation");
        streams_.push_back(s);
        pins_.emplace_back(new Staging());  // records and non-page-locked request data
        pins_.back()->ensure(std::size_t(16) << 20);
        pins_.emplace_back(new Staging());  // outputs, allocated up front
        pins_.back()->ensure(opt_.output_staging);
    }
}

MatmulServer::~MatmulServer() {
    for (auto &kv : running_) {
        cudaEventSynchronize(kv.second->done);
        cudaEventDestroy(kv.second->begin);
        cudaEventDestroy(kv.second->done);
    }
    for (void *s : streams_) {
        cudaStreamSynchronize((cudaStream_t)s);
        cudaStreamDestroy((cudaStream_t)s);
    }
}

// Device bytes of one request: inputs, raw and encoded weights, transformed weights,
// outputs (records and alignment are covered by 64 KiB of slack).
std::size_t MatmulServer::footprint(const MatmulPlan &p) const {
    const std::size_t ni = p.inputBlocks(), no = p.outputBlocks(), nw = ni * no;
    const std::size_t ctw = 2 * (std::size_t)L_ * n_;
    return 8 * (ni * ctw + p.in * p.out + nw * n_ + nw * (std::size_t)L_ * n_ + no * ctw) + (64u << 10);
}

uint64_t MatmulServer::submitBorrowed(std::size_t in, std::size_t out, const uint64_t *inputs, std::size_t input_words,
                                      const uint64_t *weights, double arrival, std::shared_ptr<void> owner,
                                      uint64_t *outputs) {
    MatmulPlan p = MatmulPlan::make(1, in, out, n_);
    const std::size_t ctw = 2 * (std::size_t)L_ * n_;
    if (input_words != p.inputBlocks() * ctw) throw std::invalid_argument("input ciphertext words do not match the shape");
    if (!inputs || !weights) throw std::invalid_argument("null request data");
    Request r;
    r.id = next_id_++;
    r.in = in;
    r.out = out;
    r.plan = p;
    r.in_ptr = inputs;
    r.w_ptr = weights;
    r.owner = std::move(owner);
    r.pinned = is_pinned(inputs) && is_pinned(weights);
    r.out_ptr = outputs;
    r.out_pinned = outputs && is_pinned(outputs);
    r.arrival = arrival;
    r.bytes = footprint(p);
    if (r.bytes > opt_.memory_budget) throw std::invalid_argument("request larger than the memory budget");
    queue_.push_back(std::move(r));
    stats_.submitted++;
    return queue_.back().id;
}

uint64_t MatmulServer::submit(std::size_t in, std::size_t out, const uint64_t *inputs, std::size_t input_words,
                              const uint64_t *weights, double arrival) {
    auto copies = std::make_shared<std::pair<std::vector<uint64_t>, std::vector<uint64_t>>>(
        std::vector<uint64_t>(inputs, inputs + input_words), std::vector<uint64_t>(weights, weights + in * out));
    return submitBorrowed(in, out, copies->first.data(), input_words, copies->second.data(), arrival, copies);
}

bool MatmulServer::launch(int slot) {
    if (queue_.empty()) return false;
    auto w = std::make_unique<Wave>();
    std::size_t bytes = 0, out_bytes = 0;
    const std::size_t ctw_bytes = 16 * (std::size_t)L_ * n_;
    while (!queue_.empty() && w->reqs.size() < opt_.max_wave_requests &&
           in_flight_bytes_ + bytes + queue_.front().bytes <= opt_.memory_budget &&
           (w->reqs.empty() || out_bytes + queue_.front().plan.outputBlocks() * ctw_bytes <= opt_.output_staging)) {
        bytes += queue_.front().bytes;
        out_bytes += queue_.front().plan.outputBlocks() * ctw_bytes;
        w->reqs.push_back(std::move(queue_.front()));
        queue_.pop_front();
    }
    if (w->reqs.empty()) return false;  // the oldest request waits for memory to free up
    const std::size_t ctw = 2 * (std::size_t)L_ * n_, ptw = (std::size_t)L_ * n_;
    // layout: inputs | raw weights | weight records | term offsets | term a | term w  (staged)
    //         encoded weights | transformed weights | outputs                          (device only)
    std::size_t na = 0, nw = 0, no = 0, wwords = 0, nterms = 0;
    std::vector<uint32_t> blocks, off{0}, ia, iw;
    for (auto &r : w->reqs) {
        const auto &p = r.plan;
        const std::size_t ri = p.inputBlocks(), ro = p.outputBlocks();
        for (std::size_t bi = 0; bi < ri; bi++)
            for (std::size_t bj = 0; bj < ro; bj++) push_block(blocks, wwords, p, bi, bj);
        w->out_base.push_back(no);
        for (std::size_t bj = 0; bj < ro; bj++) {
            for (std::size_t bi = 0; bi < ri; bi++) {
                ia.push_back((uint32_t)(na + bi));
                iw.push_back((uint32_t)(nw + bi * ro + bj));
            }
            off.push_back((uint32_t)ia.size());
        }
        na += ri;
        nw += ri * ro;
        no += ro;
        wwords += p.in * p.out;
    }
    nterms = ia.size();
    // device: inputs | raw weights | records (offsets, terms) | encoded weights |
    //         transformed weights | outputs
    // staging (page-locked): records | data of requests whose memory is not page-locked
    const std::size_t o_in = 0, o_wr = align256(o_in + na * ctw * 8), o_bl = align256(o_wr + wwords * 8),
                      o_off = align256(o_bl + blocks.size() * 4), o_ia = align256(o_off + off.size() * 4),
                      o_iw = align256(o_ia + nterms * 4), rec_end = align256(o_iw + nterms * 4);
    const std::size_t o_wp = rec_end, o_wn = align256(o_wp + nw * n_ * 8), o_out = align256(o_wn + nw * ptw * 8),
                      total = align256(o_out + no * ctw * 8);
    const std::size_t rec_bytes = rec_end - o_bl;
    std::size_t staged = rec_bytes;
    for (auto &r : w->reqs)
        if (!r.pinned) staged += 8 * (r.plan.inputBlocks() * ctw + r.in * r.out);
    Staging &pin_in = *pins_[2 * slot], &pin_out = *pins_[2 * slot + 1];
    pin_in.ensure(staged);
    pin_out.ensure(no * ctw * 8);
    char *h = static_cast<char *>(pin_in.p);
    std::memcpy(h + (o_bl - o_bl), blocks.data(), blocks.size() * 4);
    std::memcpy(h + (o_off - o_bl), off.data(), off.size() * 4);
    std::memcpy(h + (o_ia - o_bl), ia.data(), nterms * 4);
    std::memcpy(h + (o_iw - o_bl), iw.data(), nterms * 4);
    std::vector<const char *> src_in, src_w;  // per request: where its data is copied from
    std::size_t hs = rec_bytes;
    for (auto &r : w->reqs) {
        const std::size_t iw_words = r.plan.inputBlocks() * ctw, ww = r.in * r.out;
        if (r.pinned) {
            src_in.push_back(reinterpret_cast<const char *>(r.in_ptr));
            src_w.push_back(reinterpret_cast<const char *>(r.w_ptr));
        } else {
            std::memcpy(h + hs, r.in_ptr, iw_words * 8);
            src_in.push_back(h + hs);
            hs += iw_words * 8;
            std::memcpy(h + hs, r.w_ptr, ww * 8);
            src_w.push_back(h + hs);
            hs += ww * 8;
            if (!r.out_ptr) r.owner.reset();  // staged; the borrowed memory may go
        }
    }

    cudaStream_t s = (cudaStream_t)streams_[slot];
    w->bytes = std::max(bytes, total);
    w->out_words = no * ctw;
    cuda_ok(cudaEventCreate(&w->begin), "event creation");
    cuda_ok(cudaEventCreate(&w->done), "event creation");
    cuda_ok(cudaEventRecord(w->begin, s), "event record");
    const double ta = now();
    int st = cudaMallocAsync(&w->dev, total, s) == cudaSuccess ? TB_OK : TB_ERR_OUT_OF_MEMORY;
    stats_.alloc_host_s += now() - ta;
    char *d = static_cast<char *>(w->dev);
    auto U = [&](std::size_t o) { return reinterpret_cast<uint64_t *>(d + o); };
    auto V = [&](std::size_t o) { return reinterpret_cast<const uint32_t *>(d + o); };
    tb_context *hctx = context_.handle();
    if (st == TB_OK && cudaMemcpyAsync(d + o_bl, h, rec_bytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
        st = TB_ERR_CUDA;
    {
        std::size_t a2 = 0, w2 = 0;
        for (std::size_t k = 0; k < w->reqs.size(); k++) {
            const Request &r = w->reqs[k];
            const std::size_t iw_words = r.plan.inputBlocks() * ctw, ww = r.in * r.out;
            if (st == TB_OK &&
                (cudaMemcpyAsync(d + o_in + a2 * 8, src_in[k], iw_words * 8, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                 cudaMemcpyAsync(d + o_wr + w2 * 8, src_w[k], ww * 8, cudaMemcpyHostToDevice, s) != cudaSuccess))
                st = TB_ERR_CUDA;
            a2 += iw_words;
            w2 += ww;
        }
    }
    if (st == TB_OK && inject_) st = TB_ERR_CUDA;
    inject_ = false;
    if (st == TB_OK) st = tb_ntt_forward(hctx, U(o_in), U(o_in), 2 * na, 0, L_, 0, s);
    if (st == TB_OK) st = tb_matmul_encode_weights(hctx, U(o_wr), V(o_bl), nw, U(o_wp), s);
    if (st == TB_OK) st = tb_plain_to_ntt(hctx, L_, U(o_wp), n_, n_, U(o_wn), nw, s);
    if (st == TB_OK)
        st = tb_dyadic_accumulate(hctx, L_, 2, U(o_in), 0, U(o_wn), 0, U(o_out), 0, V(o_off), V(o_ia), V(o_iw),
                                  (uint32_t)no, s);
    if (st == TB_OK) st = tb_ntt_inverse(hctx, U(o_out), U(o_out), 2 * no, 0, L_, 0, s);
    // results: straight into page-locked caller buffers, the rest through the staging
    for (std::size_t k = 0; k < w->reqs.size() && st == TB_OK; k++) {
        const Request &r = w->reqs[k];
        const std::size_t words = r.plan.outputBlocks() * ctw;
        void *dst = r.out_pinned ? (void *)r.out_ptr : (void *)(static_cast<uint64_t *>(pin_out.p) + w->out_base[k] * ctw);
        if (cudaMemcpyAsync(dst, U(o_out) + w->out_base[k] * ctw, words * 8, cudaMemcpyDeviceToHost, s) != cudaSuccess)
            st = TB_ERR_CUDA;
    }
    w->failed = st != TB_OK;
    if (w->dev) cudaFreeAsync(w->dev, s);
    cuda_ok(cudaEventRecord(w->done, s), "event record");
    in_flight_bytes_ += w->bytes;
    stats_.waves++;
    stats_.max_wave = std::max(stats_.max_wave, w->reqs.size());
    stats_.peak_bytes = std::max(stats_.peak_bytes, in_flight_bytes_);
    running_[slot] = std::move(w);
    return true;
}

void MatmulServer::reap(std::vector<uint64_t> &finished) {
    for (auto it = running_.begin(); it != running_.end();) {
        Wave &w = *it->second;
        const cudaError_t q = cudaEventQuery(w.done);
        if (q == cudaErrorNotReady) {
            ++it;
            continue;
        }
        const bool ok = q == cudaSuccess && !w.failed;
        const double t = now();
        const uint64_t *out = static_cast<const uint64_t *>(pins_[2 * it->first + 1]->p);
        const std::size_t ctw = 2 * (std::size_t)L_ * n_;
        for (std::size_t k = 0; k < w.reqs.size(); k++) {
            const Request &r = w.reqs[k];
            Done d;
            d.arrival = r.arrival;
            d.done = t;
            d.ok = ok;
            if (ok) {
                const std::size_t words = r.plan.outputBlocks() * ctw;
                if (!r.out_ptr)
                    d.outputs.assign(out + w.out_base[k] * ctw, out + w.out_base[k] * ctw + words);
                else if (!r.out_pinned)
                    std::memcpy(r.out_ptr, out + w.out_base[k] * ctw, words * 8);
            }
            done_[r.id] = std::move(d);
            finished.push_back(r.id);
            if (ok)
                stats_.completed++;
            else
                stats_.failed++;
        }
        in_flight_bytes_ -= w.bytes;
        float ms = 0;
        if (cudaEventElapsedTime(&ms, w.begin, w.done) == cudaSuccess) stats_.device_s += ms * 1e-3;
        cudaEventDestroy(w.begin);
        cudaEventDestroy(w.done);
        it = running_.erase(it);
    }
}

std::vector<uint64_t> MatmulServer::step() {
    std::vector<uint64_t> finished;
    double t0 = now();
    reap(finished);
    double t1 = now();
    stats_.reap_host_s += t1 - t0;
    for (int slot = 0; slot < opt_.slots && !queue_.empty(); slot++)
        if (!running_.count(slot)) launch(slot);
    stats_.launch_host_s += now() - t1;
    return finished;
}

bool MatmulServer::drain(double timeout) {
    const double end = now() + timeout;
    while (!idle()) {
        step();
        if (now() > end) return false;
    }
    return true;
}

bool MatmulServer::take(uint64_t id, std::vector<uint64_t> &outputs, double &arrival, double &done, bool &ok) {
    auto it = done_.find(id);
    if (it == done_.end()) return false;
    outputs = std::move(it->second.outputs);
    arrival = it->second.arrival;
    done = it->second.done;
    ok = it->second.ok;
    done_.erase(it);
    return true;
}

bool MatmulServer::result(uint64_t id, std::vector<uint64_t> &outputs, double &arrival, double &done, bool &ok) {
    auto it = done_.find(id);
    if (it == done_.end()) return false;
    outputs = it->second.outputs;
    arrival = it->second.arrival;
    done = it->second.done;
    ok = it->second.ok;
    return true;
}

}  // namespace troyn

// Uneven batches behind the C ABI: ciphertext pairs of several parameter sets (ring
// degree, modulus chain, scheme) through multiply -> relinearize -> one rotation, as
// one object a C or C++ caller creates once and launches per batch.
//
// Each shape group's pipeline is the batched calls of this library (tb_multiply,
// tb_relinearize, tb_apply_galois: one launch sequence per stage for every
// ciphertext of the group) issued on a stream of its own, so the groups overlap on the
// device: a group of small rings fills the SMs a group of large rings leaves idle in
// its short launches. The fork/join of all groups is recorded once as a CUDA graph
// (the library's stream-ordered scratch allocations become graph memory nodes), after
// which one graph launch runs the whole uneven batch. The reference drives these
// operations one ciphertext per call (EvaluatorCuda::multiply / relinearizeInplace /
// rotateRowsInplace, src/evaluator_cuda.cu:262-382, 703-744, 2106-2163); run_per_op
// issues exactly that, and all three forms give identical words (exact arithmetic,
// no state shared between ciphertexts).
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/troy_b200.h"
#include "context.hpp"

namespace tb {
int galois_ntt_table(Context &c, uint32_t elt, const uint32_t **out);  // keyswitch.cu
}

struct tb_uneven {
    std::vector<tb_uneven_group> groups;
    std::vector<uint64_t *> t3;          // [count][3][L][n] products per group
    std::vector<cudaStream_t> streams;   // one per group
    std::vector<cudaEvent_t> done;       // end of each group's pipeline
    cudaEvent_t start = nullptr;
    cudaStream_t capture = nullptr;      // private stream the graph is recorded on
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;

    ~tb_uneven() {
        int prev = -1;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        for (auto *p : t3)
            if (p) cudaFree(p);
        for (auto s : streams) cudaStreamDestroy(s);
        for (auto e : done) cudaEventDestroy(e);
        if (start) cudaEventDestroy(start);
        if (capture) cudaStreamDestroy(capture);
        if (prev >= 0) cudaSetDevice(prev);
    }
};

using tb::set_error;

namespace {

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// One group's pipeline: multiply -> relinearize -> rotation, `count` ciphertexts per
// call (the batched form), or one per call (per_op: the reference's usage).
int group_pipeline(const tb_uneven_group &g, uint64_t *t3, bool per_op, cudaStream_t s) {
    const uint64_t n = g.ctx->c->n;
    const uint64_t w2 = 2ull * g.L * n, w3 = 3ull * g.L * n;
    const uint64_t step = per_op ? 1 : g.count;
    for (uint64_t i = 0; i < g.count; i += step) {
        const uint64_t nb = per_op ? 1 : g.count;
        int st = tb_multiply(g.ctx, g.L, g.a + i * w2, 0, g.b + i * w2, 0, t3 + i * w3, 0, nb, s);
        if (st == TB_OK) st = tb_relinearize(g.ctx, g.L, t3 + i * w3, 0, g.relin_key, nb, s);
        if (st == TB_OK)
            st = tb_apply_galois(g.ctx, g.L, g.galois_elt, t3 + i * w3, w3, g.out + i * w2, 0, g.galois_key, nb, s);
        if (st != TB_OK) return st;
    }
    return TB_OK;
}

int fork_join(tb_uneven *u, cudaStream_t s) {
    cudaError_t e = cudaEventRecord(u->start, s);
    if (e != cudaSuccess) return tb::status_from(e);
    for (size_t g = 0; g < u->groups.size(); g++) {
        e = cudaStreamWaitEvent(u->streams[g], u->start, 0);
        if (e != cudaSuccess) return tb::status_from(e);
        const int st = group_pipeline(u->groups[g], u->t3[g], false, u->streams[g]);
        if (st != TB_OK) return st;
        e = cudaEventRecord(u->done[g], u->streams[g]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, u->done[g], 0);
        if (e != cudaSuccess) return tb::status_from(e);
    }
    return TB_OK;
}

}  // namespace

extern "C" {

int tb_uneven_create(const tb_uneven_group *groups, int count, tb_uneven **out) {
    if (!out) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!groups || count < 1) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "no shape groups");
    const int device = groups[0].ctx && groups[0].ctx->c ? groups[0].ctx->c->device : -1;
    for (int i = 0; i < count; i++) {
        const tb_uneven_group &g = groups[i];
        if (!g.ctx || !g.ctx->c) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null context in a shape group");
        const tb::Context &c = *g.ctx->c;
        if (c.device != device) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "shape groups on different devices");
        if (c.scheme == tb::SCHEME_RAW) return set_error(tb::TB_ERR_UNSUPPORTED, "shape group without a scheme");
        if (g.L < 1 || g.L > (int)c.chain.size() - 1)
            return set_error(tb::TB_ERR_INVALID_ARGUMENT, "shape group level outside the data chain");
        if (!g.count) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "empty shape group");
        if (!g.a || !g.b || !g.out || !g.relin_key || !g.galois_key)
            return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null buffer in a shape group");
        if (!(g.galois_elt & 1) || g.galois_elt >= 2 * c.n)
            return set_error(tb::TB_ERR_INVALID_ARGUMENT, "Galois element is not valid");
    }
    DeviceGuard guard(device);
    auto *u = new tb_uneven();
    u->device = device;
    u->groups.assign(groups, groups + count);
    cudaError_t e = cudaEventCreateWithFlags(&u->start, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&u->capture, cudaStreamNonBlocking);
    for (int i = 0; i < count && e == cudaSuccess; i++) {
        const tb_uneven_group &g = groups[i];
        uint64_t *p = nullptr;
        e = cudaMalloc(&p, 3ull * g.L * g.ctx->c->n * 8 * g.count);
        u->t3.push_back(p);
        cudaStream_t s = nullptr;
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
        u->streams.push_back(s);
        cudaEvent_t ev = nullptr;
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        u->done.push_back(ev);
    }
    if (e != cudaSuccess) {
        delete u;
        return tb::status_from(e);
    }
    // CKKS rotations gather through a per-element table built on first use: build it
    // now, outside any capture
    for (int i = 0; i < count; i++) {
        if (groups[i].ctx->c->scheme != tb::SCHEME_CKKS) continue;
        const uint32_t *tab = nullptr;
        const int st = tb::galois_ntt_table(*groups[i].ctx->c, groups[i].galois_elt, &tab);
        if (st != TB_OK) {
            delete u;
            return st;
        }
    }
    *out = u;
    return TB_OK;
}

int tb_uneven_run(tb_uneven *u, void *stream) {
    if (!u) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null uneven batch");
    DeviceGuard guard(u->device);
    return fork_join(u, reinterpret_cast<cudaStream_t>(stream));
}

int tb_uneven_run_per_op(tb_uneven *u, void *stream) {
    if (!u) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null uneven batch");
    DeviceGuard guard(u->device);
    for (size_t g = 0; g < u->groups.size(); g++) {
        const int st = group_pipeline(u->groups[g], u->t3[g], true, reinterpret_cast<cudaStream_t>(stream));
        if (st != TB_OK) return st;
    }
    return TB_OK;
}

int tb_uneven_capture(tb_uneven *u) {
    if (!u) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null uneven batch");
    DeviceGuard guard(u->device);
    if (u->exec) return TB_OK;
    // one uncaptured run first: every table and pool setting the calls make on first
    // use exists before the capture starts
    int st = fork_join(u, u->capture);
    if (st != TB_OK) return st;
    cudaError_t e = cudaStreamSynchronize(u->capture);
    if (e != cudaSuccess) return tb::status_from(e);
    e = cudaStreamBeginCapture(u->capture, cudaStreamCaptureModeRelaxed);
    if (e != cudaSuccess) return tb::status_from(e);
    st = fork_join(u, u->capture);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(u->capture, &graph);
    if (st != TB_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return tb::status_from(e);
    e = cudaGraphInstantiate(&u->exec, graph, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(graph);
        u->exec = nullptr;
        return tb::status_from(e);
    }
    u->graph = graph;
    return TB_OK;
}

int tb_uneven_replay(tb_uneven *u, void *stream) {
    if (!u) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null uneven batch");
    if (!u->exec) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "uneven batch not captured");
    DeviceGuard guard(u->device);
    return tb::status_from(cudaGraphLaunch(u->exec, reinterpret_cast<cudaStream_t>(stream)));
}

int tb_uneven_destroy(tb_uneven *u) {
    delete u;
    return TB_OK;
}

}  // extern "C"

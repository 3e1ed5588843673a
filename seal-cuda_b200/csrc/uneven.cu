// Uneven batches behind the C ABI: ciphertext pairs of several parameter sets (ring
// degree, modulus chain, scheme) through multiply -> relinearize -> one rotation, as
// one object a C or C++ caller creates once and launches per batch.
//
// Each shape group's pipeline is the batched calls of this library (tb_multiply,
// tb_relinearize, tb_apply_galois: one launch sequence per stage for every
// ciphertext of the group) issued on a stream of its own, so the groups overlap on the
// device: a group of small rings fills the SMs a group of large rings leaves idle in
// its short launches. In the shapes mode (tb_uneven_set_shapes) the products still run
// per group on their streams, and then the relinearizations and rotations of every
// group run as one persistent launch per key-switch step for all degrees and levels
// at once (keyswitch_shapes). Either way the fork/join is recorded once as a CUDA graph
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
int uneven_relin_rotate(Context *const *ctxs, const int *Ls, const uint64_t *Bs, uint64_t *const *t3,
                        const uint64_t *const *rlks, const uint64_t *const *gks, const uint32_t *elts,
                        uint64_t *const *outs, int count, cudaStream_t s);  // keyswitch.cu
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
    bool shapes = false;   // key switching of all groups in one launch per step

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

// Shapes mode: the groups' products on their own streams (joined back to s), then the
// relinearizations and rotations of every group with one launch per key-switch step.
int shapes_pipeline(tb_uneven *u, cudaStream_t s) {
    cudaError_t e = cudaEventRecord(u->start, s);
    if (e != cudaSuccess) return tb::status_from(e);
    const int count = (int)u->groups.size();
    tb::Context *ctxs[tb::MAX_SHAPES];
    int Ls[tb::MAX_SHAPES];
    uint64_t Bs[tb::MAX_SHAPES];
    uint64_t *outs[tb::MAX_SHAPES];
    const uint64_t *rlks[tb::MAX_SHAPES], *gks[tb::MAX_SHAPES];
    uint32_t elts[tb::MAX_SHAPES];
    for (int g = 0; g < count; g++) {
        const tb_uneven_group &G = u->groups[g];
        e = cudaStreamWaitEvent(u->streams[g], u->start, 0);
        if (e != cudaSuccess) return tb::status_from(e);
        const int st = tb_multiply(G.ctx, G.L, G.a, 0, G.b, 0, u->t3[g], 0, G.count, u->streams[g]);
        if (st != TB_OK) return st;
        e = cudaEventRecord(u->done[g], u->streams[g]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(s, u->done[g], 0);
        if (e != cudaSuccess) return tb::status_from(e);
        ctxs[g] = G.ctx->c;
        Ls[g] = G.L;
        Bs[g] = G.count;
        outs[g] = G.out;
        rlks[g] = G.relin_key;
        gks[g] = G.galois_key;
        elts[g] = G.galois_elt;
    }
    return tb::uneven_relin_rotate(ctxs, Ls, Bs, u->t3.data(), rlks, gks, elts, outs, count, s);
}

int fork_join(tb_uneven *u, cudaStream_t s) {
    if (u->shapes) return shapes_pipeline(u, s);
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

// Whether every group can take the one-launch-per-step key switching.
bool shapes_possible(const tb_uneven *u) {
    if (u->groups.size() > (size_t)tb::MAX_SHAPES) return false;
    for (const auto &g : u->groups)
        if (g.ctx->c->logn < 12 || g.ctx->c->logn > tb::MAX_LOGB || g.count > 0x7fffffffull / 4096) return false;
    return true;
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

int tb_uneven_set_shapes(tb_uneven *u, int on) {
    if (!u) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "null uneven batch");
    if (on && !shapes_possible(u))
        return set_error(tb::TB_ERR_UNSUPPORTED, "one-launch key switching takes at most 8 groups of degree 4096 .. 16384");
    if (u->exec) return set_error(tb::TB_ERR_INVALID_ARGUMENT, "uneven batch already captured");
    u->shapes = on != 0;
    return TB_OK;
}

int tb_uneven_destroy(tb_uneven *u) {
    delete u;
    return TB_OK;
}

}  // extern "C"

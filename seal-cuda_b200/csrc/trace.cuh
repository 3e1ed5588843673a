// Optional per-launch device timing. When enabled (tb_trace_enable), every library
// launch site records a CUDA event pair on its stream; tb_trace_collect sums the
// elapsed times per kernel name. Disabled, a scope costs one relaxed load.
#pragma once

#include <atomic>
#include <cuda_runtime.h>

namespace tb {

extern std::atomic<bool> g_trace_on;
void trace_record(const char *name, cudaEvent_t a, cudaEvent_t b);

struct TraceScope {
    const char *name;
    cudaStream_t s;
    cudaEvent_t a = nullptr, b = nullptr;
    TraceScope(const char *nm, cudaStream_t st) : name(nm), s(st) {
        if (g_trace_on.load(std::memory_order_relaxed)) {
            cudaEventCreate(&a);
            cudaEventCreate(&b);
            cudaEventRecord(a, s);
        }
    }
    ~TraceScope() {
        if (a) {
            cudaEventRecord(b, s);
            trace_record(name, a, b);
        }
    }
};

}  // namespace tb

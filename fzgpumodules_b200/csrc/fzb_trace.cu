// fzb_trace.cu -- optional per-kernel timing with CUDA events, the library
// side of the reference's per-node profiling (enableProfiling records a
// start/stop cudaEvent pair per DAG node and collectTimings folds them into
// per-stage milliseconds: src/pipeline/dag.cpp:107-116,418-420,
// include/perf.h:70).
//
// When tracing is off a TraceScope costs one branch.  When it is on, every
// traced launch site records an event before and after its kernel on the
// launching stream; fzb_trace_collect() waits for the recorded events and
// accumulates launches and milliseconds per kernel name.  Events are created
// once and recycled (cudaEventCreate allocates no device memory).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fzb.h"
#include "fzb_kernels.cuh"

namespace fzb {

bool g_trace_on = false;

namespace {

struct Pending {
    const char* name;
    cudaEvent_t a, b;
};

struct Agg {
    uint64_t launches = 0;
    double ms = 0.0;
};

std::mutex g_mu;
std::vector<Pending> g_pending;
std::vector<cudaEvent_t> g_free;
std::map<std::string, Agg> g_agg;

cudaEvent_t take_event() {
    if (!g_free.empty()) {
        cudaEvent_t e = g_free.back();
        g_free.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

}  // namespace

TraceScope::TraceScope(cudaStream_t s, const char* name) : s_(s), end_(nullptr) {
    if (!g_trace_on) return;
    std::lock_guard<std::mutex> lock(g_mu);
    cudaEvent_t a = take_event(), b = take_event();
    if (!a || !b) return;
    cudaEventRecord(a, s);
    g_pending.push_back({name, a, b});
    end_ = b;
}

TraceScope::~TraceScope() {
    if (end_) cudaEventRecord(end_, s_);
}

}  // namespace fzb

using namespace fzb;

extern "C" {

int fzb_trace_enable(int on) {
    std::lock_guard<std::mutex> lock(g_mu);
    const int prev = g_trace_on ? 1 : 0;
    g_trace_on = on != 0;
    return prev;
}

int fzb_trace_collect(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    int rc = FZB_OK;
    for (const Pending& p : g_pending) {
        float ms = 0.0f;
        if (cudaEventSynchronize(p.b) != cudaSuccess || cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) {
            rc = FZB_E_CUDA;
        } else {
            Agg& g = g_agg[p.name];
            g.launches++;
            g.ms += ms;
        }
        g_free.push_back(p.a);
        g_free.push_back(p.b);
    }
    g_pending.clear();
    return rc ? rc : (int)g_agg.size();
}

int fzb_trace_get(int i, char* name, size_t name_cap, uint64_t* launches, double* total_ms) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (i < 0 || i >= (int)g_agg.size() || !name || name_cap == 0) return FZB_E_INVALID;
    auto it = g_agg.begin();
    std::advance(it, i);
    std::strncpy(name, it->first.c_str(), name_cap - 1);
    name[name_cap - 1] = '\0';
    if (launches) *launches = it->second.launches;
    if (total_ms) *total_ms = it->second.ms;
    return FZB_OK;
}

void fzb_trace_reset(void) {
    std::lock_guard<std::mutex> lock(g_mu);
    g_agg.clear();
}

}  // extern "C"

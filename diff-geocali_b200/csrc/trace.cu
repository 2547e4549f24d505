// trace.cu -- optional CUDA-event timing of every kernel libdgc launches.
//
// When enabled (dgc_trace_enable(1)), each launch helper records a start and a
// stop event on the launch stream; dgc_trace_count()/dgc_trace_get() return the
// kernel names and device durations afterwards.  Disabled, the cost is one
// relaxed atomic load per launch.
#include <atomic>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "trace.cuh"

namespace dgc {

namespace {

struct Record {
    std::string name;
    cudaEvent_t start;
    cudaEvent_t stop;
};

std::atomic<int> g_enabled{0};
std::mutex g_mu;
std::vector<Record> g_records;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    return e;
}

}  // namespace

TraceScope::TraceScope(const char* name, cudaStream_t s) : active_(false), stream_(s), index_(-1) {
    if (!g_enabled.load(std::memory_order_relaxed)) return;
    std::lock_guard<std::mutex> lock(g_mu);
    Record r{name, take_event(), take_event()};
    if (!r.start || !r.stop) return;
    cudaEventRecord(r.start, s);
    g_records.push_back(r);
    index_ = (int)g_records.size() - 1;
    active_ = true;
}

TraceScope::~TraceScope() {
    if (!active_) return;
    std::lock_guard<std::mutex> lock(g_mu);
    if (index_ < (int)g_records.size()) cudaEventRecord(g_records[index_].stop, stream_);
}

}  // namespace dgc

extern "C" {

void dgc_trace_enable(int on) { dgc::g_enabled.store(on ? 1 : 0); }

int dgc_trace_count(void) {
    std::lock_guard<std::mutex> lock(dgc::g_mu);
    return (int)dgc::g_records.size();
}

int dgc_trace_get(int index, char* name, int name_len, float* ms) {
    std::lock_guard<std::mutex> lock(dgc::g_mu);
    if (index < 0 || index >= (int)dgc::g_records.size()) return DGC_ERR_INVALID_ARGUMENT;
    const dgc::Record& r = dgc::g_records[index];
    if (name && name_len > 0) {
        strncpy(name, r.name.c_str(), (size_t)name_len - 1);
        name[name_len - 1] = '\0';
    }
    if (ms) {
        cudaError_t e = cudaEventSynchronize(r.stop);
        if (e == cudaSuccess) e = cudaEventElapsedTime(ms, r.start, r.stop);
        if (e != cudaSuccess) {
            dgc::set_error(std::string("trace event: ") + cudaGetErrorString(e));
            return DGC_ERR_CUDA;
        }
    }
    return DGC_OK;
}

void dgc_trace_clear(void) {
    std::lock_guard<std::mutex> lock(dgc::g_mu);
    for (auto& r : dgc::g_records) {
        cudaEventSynchronize(r.stop);
        dgc::g_pool.push_back(r.start);
        dgc::g_pool.push_back(r.stop);
    }
    dgc::g_records.clear();
}

}  // extern "C"

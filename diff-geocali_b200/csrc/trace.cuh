// trace.cuh -- scoped CUDA-event timer around one kernel launch (see trace.cu).
#pragma once

#include <cuda_runtime.h>

namespace dgc {

class TraceScope {
  public:
    TraceScope(const char* name, cudaStream_t s);
    ~TraceScope();
    TraceScope(const TraceScope&) = delete;
    TraceScope& operator=(const TraceScope&) = delete;

  private:
    bool active_;
    cudaStream_t stream_;
    int index_;
};

}  // namespace dgc

#define DGC_TRACE(name, stream) ::dgc::TraceScope dgc_trace_scope__(name, stream)

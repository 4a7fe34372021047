// Launch counting, optional per-stage CUDA-event timing and NVTX ranges.
//
// Every kernel launch site bumps a process-wide counter (read through
// pptkg_launch_count).  When stage timing is enabled, a Stage scope records a
// pair of events on the launching stream around its work; pptkg_profile_get
// later returns the summed milliseconds per stage name.  Every Stage scope
// is also an NVTX range of the same name on the host thread (a no-op unless
// a profiler that collects NVTX is attached).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <atomic>

namespace pptkg {

extern std::atomic<long long> g_launches;
bool profiling_on();
void profile_record(const char* stage, cudaEvent_t a, cudaEvent_t b);

struct Stage {
  const char* name;
  cudaStream_t st;
  cudaEvent_t a = nullptr, b = nullptr;
  Stage(const char* n, cudaStream_t s) : name(n), st(s) {
    nvtxRangePushA(n);
    if (profiling_on() && cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess)
      cudaEventRecord(a, st);
  }
  ~Stage() {
    if (a && b) {
      cudaEventRecord(b, st);
      profile_record(name, a, b);
    }
    nvtxRangePop();
  }
};

}  // namespace pptkg

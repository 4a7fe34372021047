// Stage timing store behind pptkg_profile_enable / pptkg_profile_get.
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "pptkg.h"
#include "profile.cuh"

namespace pptkg {

std::atomic<long long> g_launches{0};
std::atomic<int> g_tune_lane_span{256};
std::atomic<int> g_tune_rnear_warp_queries{262144};
thread_local int* g_status_sink = nullptr;

namespace {
struct Pending {
  std::string name;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
std::map<std::string, std::pair<double, long long>> g_total;

void drain_locked() {
  for (auto& p : g_pending) {
    float ms = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      auto& t = g_total[p.name];
      t.first += ms;
      t.second += 1;
    }
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  g_pending.clear();
}
}  // namespace

void keep_pool_cached(cudaStream_t) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
  static std::atomic<unsigned long long> done{0};
  const unsigned long long bit = 1ull << dev;
  if (done.load() & bit) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    unsigned long long thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  done.fetch_or(bit);
}

bool profiling_on() {
  std::lock_guard<std::mutex> g(g_mu);
  return g_on;
}

void profile_record(const char* stage, cudaEvent_t a, cudaEvent_t b) {
  std::lock_guard<std::mutex> g(g_mu);
  g_pending.push_back({stage, a, b});
}

}  // namespace pptkg

extern "C" {

int pptkg_profile_enable(int on) {
  std::lock_guard<std::mutex> g(pptkg::g_mu);
  pptkg::drain_locked();
  pptkg::g_total.clear();
  pptkg::g_on = on != 0;
  return PPTKG_OK;
}

int pptkg_profile_get(const char* stage, double* total_ms, int64_t* count) {
  std::lock_guard<std::mutex> g(pptkg::g_mu);
  pptkg::drain_locked();
  auto it = pptkg::g_total.find(stage ? stage : "");
  if (total_ms) *total_ms = it == pptkg::g_total.end() ? 0.0 : it->second.first;
  if (count) *count = it == pptkg::g_total.end() ? 0 : it->second.second;
  return PPTKG_OK;
}

int64_t pptkg_launch_count(void) { return pptkg::g_launches.load(); }

int pptkg_tune_set(const char* name, int64_t value) {
  if (!name) return PPTKG_E_INVALID;
  if (std::string(name) == "lane_span") {
    if (value < -1 || value > INT32_MAX) return PPTKG_E_INVALID;
    pptkg::g_tune_lane_span.store((int)value);
    return PPTKG_OK;
  }
  if (std::string(name) == "rnear_warp_queries") {
    if (value < 0 || value > INT32_MAX) return PPTKG_E_INVALID;
    pptkg::g_tune_rnear_warp_queries.store((int)value);
    return PPTKG_OK;
  }
  return PPTKG_E_INVALID;
}

int pptkg_set_status_sink(int* d_word) {
  pptkg::g_status_sink = d_word;
  return PPTKG_OK;
}

int pptkg_tune_get(const char* name, int64_t* value) {
  if (!name || !value) return PPTKG_E_INVALID;
  if (std::string(name) == "lane_span") {
    *value = pptkg::g_tune_lane_span.load();
    return PPTKG_OK;
  }
  if (std::string(name) == "rnear_warp_queries") {
    *value = pptkg::g_tune_rnear_warp_queries.load();
    return PPTKG_OK;
  }
  return PPTKG_E_INVALID;
}

}  // extern "C"

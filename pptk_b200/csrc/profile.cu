// Stage timing store behind pptkg_profile_enable / pptkg_profile_get.
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>
#include <vector>

#include "common.cuh"
#include "pptkg.h"
#include "profile.cuh"
#include "util.cuh"

namespace pptkg {

std::atomic<long long> g_launches{0};
std::atomic<int> g_tune_lane_span{1024};
std::atomic<int> g_tune_rnear_warp_queries{262144};
std::atomic<int> g_tune_warm_bound{1};
std::atomic<int> g_tune_topk_min{0};
std::atomic<int> g_tune_warm_mult{2};
thread_local int* g_status_sink = nullptr;

#ifdef PPTKG_BOUNDS_CHECK
static std::mutex g_bmu;
static std::map<int, int*> g_bwords;
int* bounds_word(int device) {
  std::lock_guard<std::mutex> g(g_bmu);
  auto it = g_bwords.find(device);
  if (it != g_bwords.end()) return it->second;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  int* w = nullptr;
  if (cudaMalloc((void**)&w, sizeof(int)) != cudaSuccess || cudaMemset(w, 0, sizeof(int)) != cudaSuccess) w = nullptr;
  cudaSetDevice(prev);
  g_bwords[device] = w;
  return w;
}
int bounds_take(int device) {
  int* w = bounds_word(device);
  if (!w) return 0;
  int prev = 0, h = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  cudaDeviceSynchronize();
  cudaMemcpy(&h, w, sizeof(int), cudaMemcpyDeviceToHost);
  if (h) cudaMemset(w, 0, sizeof(int));
  cudaSetDevice(prev);
  return h;
}
#else
int* bounds_word(int) { return nullptr; }
int bounds_take(int) { return 0; }
#endif

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

// ------------------------------------------------- device memory cache --
namespace {
struct LiveBlock {
  size_t bytes;
  int device;
};
// A freed block and the event recorded on its stream when it was freed.
struct CachedBlock {
  void* p;
  cudaEvent_t ev;
};
std::mutex g_amu;
// free blocks: (device, stream) -> size -> blocks
std::map<std::pair<int, cudaStream_t>, std::multimap<size_t, CachedBlock>> g_cached;
std::unordered_map<void*, LiveBlock> g_live;

size_t round_block(size_t bytes) {
  if (bytes == 0) bytes = 1;
  const size_t q = bytes <= ((size_t)1 << 20) ? 512 : ((size_t)2 << 20);
  return (bytes + q - 1) / q * q;
}

// Returns every cached block of `device` to the pool (g_amu held).
void flush_device_locked(int device) {
  for (auto it = g_cached.begin(); it != g_cached.end();) {
    if (it->first.first != device) {
      ++it;
      continue;
    }
    for (auto& kv : it->second) {
      cudaFreeAsync(kv.second.p, it->first.second);
      if (kv.second.ev) cudaEventDestroy(kv.second.ev);
    }
    it = g_cached.erase(it);
  }
}

// Takes the smallest block of `list` that fits rb and wastes at most half of
// it; with `ready`, only a block whose free event has completed (its last
// use is over, so no stream needs to wait for it).  False if there is none
// (g_amu held).
bool take_fit(std::multimap<size_t, CachedBlock>& list, size_t rb, bool ready, CachedBlock& out, size_t& bytes) {
  for (auto it = list.lower_bound(rb); it != list.end() && it->first <= rb + rb / 2; ++it) {
    if (ready) {
      const cudaError_t q = it->second.ev ? cudaEventQuery(it->second.ev) : cudaSuccess;
      if (q != cudaSuccess) {
        cudaGetLastError();
        continue;
      }
    }
    out = it->second;
    bytes = it->first;
    list.erase(it);
    return true;
  }
  return false;
}
// True unless `st` is known not to be capturing into a CUDA graph.  A
// captured call gets graph-owned memory from cudaMallocAsync / cudaFreeAsync
// (memory nodes); a cached block would be shared between the graph's replays
// and later calls.
bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return cs != cudaStreamCaptureStatusNone;
}
}  // namespace

// Blocks below this size go straight to the pool (small requests are cheap
// for it); the stalls were measured on requests of tens of MB to 15 GB.
constexpr size_t CACHE_MIN_BYTES = (size_t)1 << 20;

cudaError_t dev_malloc(void** p, size_t bytes, cudaStream_t st) {
  *p = nullptr;
  if (bytes < CACHE_MIN_BYTES || capturing(st)) return cudaMallocAsync(p, bytes ? bytes : 1, st);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const size_t rb = round_block(bytes);
  {
    std::lock_guard<std::mutex> g(g_amu);
    CachedBlock b{nullptr, nullptr};
    size_t got = 0;
    // a block freed on this stream: stream order already protects it
    auto own = g_cached.find({dev, st});
    bool found = own != g_cached.end() && take_fit(own->second, rb, false, b, got);
    if (!found) {
      // a block freed on another stream of the device whose last use has
      // completed: taking one still in use would make this stream wait for
      // the other stream's kernels
      for (auto& kv : g_cached) {
        if (kv.first.first != dev || kv.first.second == st) continue;
        if (take_fit(kv.second, rb, true, b, got)) {
          found = true;
          break;
        }
      }
    }
    if (found && b.ev) cudaEventDestroy(b.ev);
    if (found) {
      *p = b.p;
      g_live[*p] = LiveBlock{got, dev};
      return cudaSuccess;
    }
  }
  e = cudaMallocAsync(p, rb, st);
  if (e == cudaErrorMemoryAllocation) {
    cudaGetLastError();
    {
      std::lock_guard<std::mutex> g(g_amu);
      flush_device_locked(dev);
    }
    e = cudaMallocAsync(p, rb, st);
  }
  if (e != cudaSuccess) {
    *p = nullptr;
    return e;
  }
  std::lock_guard<std::mutex> g(g_amu);
  g_live[*p] = LiveBlock{rb, dev};
  return cudaSuccess;
}

void dev_free(void* p, cudaStream_t st) {
  if (!p) return;
  const bool cap = capturing(st);
  std::lock_guard<std::mutex> g(g_amu);
  auto it = g_live.find(p);
  if (it == g_live.end() || cap) {  // captured, or not from the cache
    if (it != g_live.end()) g_live.erase(it);
    cudaFreeAsync(p, st);
    return;
  }
  CachedBlock b{p, nullptr};
  if (cudaEventCreateWithFlags(&b.ev, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(b.ev, st) != cudaSuccess) {
    // without an event the block can only go back to the pool
    if (b.ev) cudaEventDestroy(b.ev);
    cudaGetLastError();
    cudaFreeAsync(p, st);
    g_live.erase(it);
    return;
  }
  g_cached[{it->second.device, st}].insert({it->second.bytes, b});
  g_live.erase(it);
}

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
  if (std::string(name) == "warm_bound") {
    if (value < 0 || value > 1) return PPTKG_E_INVALID;
    pptkg::g_tune_warm_bound.store((int)value);
    return PPTKG_OK;
  }
  if (std::string(name) == "topk_min") {
    if (value != 0 && value != 4 && value != 8 && value != 16 && value != 32 && value != 64) return PPTKG_E_INVALID;
    pptkg::g_tune_topk_min.store((int)value);
    return PPTKG_OK;
  }
  if (std::string(name) == "warm_mult") {
    if (value < 1 || value > 8) return PPTKG_E_INVALID;
    pptkg::g_tune_warm_mult.store((int)value);
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
  if (std::string(name) == "warm_bound") {
    *value = pptkg::g_tune_warm_bound.load();
    return PPTKG_OK;
  }
  if (std::string(name) == "topk_min") {
    *value = pptkg::g_tune_topk_min.load();
    return PPTKG_OK;
  }
  if (std::string(name) == "warm_mult") {
    *value = pptkg::g_tune_warm_mult.load();
    return PPTKG_OK;
  }
  return PPTKG_E_INVALID;
}

}  // extern "C"

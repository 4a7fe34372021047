// Stream-ordered device memory and small device-wide primitives (exclusive
// scan, block reductions) used by the build and query paths.
#pragma once

#include "common.cuh"

namespace pptkg {

// Keeps freed blocks of the device's default memory pool cached instead of
// returning them to the driver at every synchronisation (the default release
// threshold is 0), so repeated calls reuse their scratch without remapping.
void keep_pool_cached(cudaStream_t st);

// Device memory of trees and of the build path.  Freed blocks of 1 MB and
// more are kept in a cache per (device, stream); smaller ones go back to the
// pool.  An allocation takes a block freed on its own stream
// (stream order makes that safe without any synchronisation), else one freed
// on another stream of the device whose free event (recorded on that stream
// at the free) has completed; misses come from the stream-ordered pool.  On
// a stream that is capturing a CUDA graph both calls go straight to
// cudaMallocAsync / cudaFreeAsync, so captured work keeps graph-owned memory.  The cache exists because cudaMallocAsync, even on
// memory the pool already holds, was measured to stall the calling thread for
// 0.1-1.7 s at times on 1-15 GB requests, leaving the GPU idle.  A request
// that the pool cannot meet empties the cache of every stream of the device
// and is tried once more.  dev_free takes the stream whose order protects
// the block's last use (the stream it was used on).
cudaError_t dev_malloc(void** p, size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);

// ------------------------------------------------------------- DevBuf ----
// Scratch memory that goes back when the buffer goes away, on the stream it
// was allocated for: from the stream-ordered pool, or (CACHED) from
// dev_malloc.  The build path uses the cached form: its scratch is large
// (up to 2 records per point) and allocated on one stream per build.
template <typename T, bool CACHED = false>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DevBuf() = default;
  DevBuf(size_t count, cudaStream_t stream) { alloc(count, stream); }
  void alloc(size_t count, cudaStream_t stream) {
    release();
    s = stream;
    n = count;
    if (count) {
      if (CACHED)
        PPTKG_CUDA(dev_malloc((void**)&p, count * sizeof(T), stream));
      else
        PPTKG_CUDA(cudaMallocAsync((void**)&p, count * sizeof(T), stream));
    }
  }
  void release() {
    if (p) {
      if (CACHED)
        dev_free(p, s);
      else
        cudaFreeAsync(p, s);
    }
    p = nullptr;
    n = 0;
  }
  T* get() const { return p; }
  ~DevBuf() { release(); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
};

// Scratch of the build path.
template <typename T>
using BuildBuf = DevBuf<T, true>;

// ------------------------------------------------------ block primitives --
template <typename V>
__device__ __forceinline__ V warp_incl_scan(V v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    V t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

template <typename V>
__device__ __forceinline__ V warp_sum(V v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Exclusive block scan; returns the exclusive prefix of v and the block total.
// `sh` needs 33 entries.  Every thread of the block must call it.
template <typename V>
__device__ __forceinline__ V block_excl_scan(V v, V* sh, V& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  V inc = warp_incl_scan(v);
  if (lane == 31) sh[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    V w = lane < nw ? sh[lane] : V(0);
    V wi = warp_incl_scan(w);
    if (lane < nw) sh[lane] = wi - w;
    if (lane == nw - 1) sh[32] = wi;
  }
  __syncthreads();
  V r = sh[wid] + inc - v;
  total = sh[32];
  __syncthreads();
  return r;
}

template <typename V>
__device__ __forceinline__ V block_sum(V v, V* sh) {
  V t;
  block_excl_scan(v, sh, t);
  return t;
}

// --------------------------------------------------- device-wide scan ----
constexpr int SCAN_THREADS = 512;
constexpr int SCAN_ITEMS = 8;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

template <typename In>
__global__ void k_scan_reduce(const In* in, int64_t n, int64_t* partial) {
  __shared__ int64_t sh[33];
  int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK + (int64_t)threadIdx.x * SCAN_ITEMS;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++)
    if (base + i < n) s += (int64_t)in[base + i];
  int64_t t = block_sum(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = t;
}

template <typename In, typename Out>
__global__ void k_scan_down(const In* in, int64_t n, const int64_t* partial, Out* out, Out* total) {
  __shared__ int64_t sh[33];
  int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK + (int64_t)threadIdx.x * SCAN_ITEMS;
  int64_t v[SCAN_ITEMS];
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    v[i] = (base + i < n) ? (int64_t)in[base + i] : 0;
    s += v[i];
  }
  int64_t tot;
  int64_t run = block_excl_scan(s, sh, tot) + (partial ? partial[blockIdx.x] : 0);
#pragma unroll
  for (int i = 0; i < SCAN_ITEMS; i++) {
    if (base + i < n) out[base + i] = (Out)run;
    run += v[i];
  }
  if (total && blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) *total = (Out)run;
}

// out[i] = sum(in[0..i-1]); *total (device pointer, optional) = sum(in).
// `in` and `out` may alias.
template <typename In, typename Out>
void exclusive_scan(const In* in, Out* out, int64_t n, Out* total, cudaStream_t st) {
  if (n <= 0) {
    if (total) PPTKG_CUDA(cudaMemsetAsync(total, 0, sizeof(Out), st));
    return;
  }
  int64_t nb = (n + SCAN_CHUNK - 1) / SCAN_CHUNK;
  if (nb == 1) {
    k_scan_down<In, Out><<<1, SCAN_THREADS, 0, st>>>(in, n, nullptr, out, total);
    PPTKG_CHECK_LAUNCH();
    return;
  }
  DevBuf<int64_t> part(nb, st);
  k_scan_reduce<In><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, part.get());
  PPTKG_CHECK_LAUNCH();
  exclusive_scan<int64_t, int64_t>(part.get(), part.get(), nb, nullptr, st);
  k_scan_down<In, Out><<<(unsigned)nb, SCAN_THREADS, 0, st>>>(in, n, part.get(), out, total);
  PPTKG_CHECK_LAUNCH();
}

}  // namespace pptkg

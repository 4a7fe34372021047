// Shared device helpers for the pptk B200 kernels: element-type traits,
// reference-exact arithmetic (no FMA contraction), ordered integer images of
// floating point values for atomic min/max, and error plumbing.
#pragma once

#include <limits>
#include <type_traits>

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cfloat>
#include <climits>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace pptkg {

// ---------------------------------------------------------------- errors --
struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

enum Status {
  OK = 0,
  E_INVALID = 1,     // bad argument (ValueError at the Python boundary)
  E_TYPE = 2,        // unsupported dtype / dim (TypeError)
  E_CUDA = 3,        // CUDA runtime failure
  E_RANGE = 4,       // index outside the point range (RuntimeError)
  E_DEVICE = 5,      // a kernel reported a failed internal check
  E_UNSUPPORTED = 6  // NotImplementedError
};

#define PPTKG_CUDA(call)                                                                        \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::pptkg::Error(::pptkg::E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

// Counts every kernel launch of the library (pptkg_launch_count) and checks it.
extern std::atomic<long long> g_launches;

// Run-time tuning knobs (pptkg_tune_set / pptkg_tune_get), read at launch.
//  lane_span: a kNN warp whose queries span more than this many tree
//    positions walks the tree per lane instead of as a packet (-1: never).
extern std::atomic<int> g_tune_lane_span;
//  rnear_warp_queries: r-near batches of at most this many queries run one
//    warp per query instead of 32-query packets (0: never).
extern std::atomic<int> g_tune_rnear_warp_queries;
//  warm_bound: after the warm start of a kNN list, also lower its bound to
//    the k-th distance of the 32 (k <= 16) or 3 x k tree-order neighbours
//    of the query's anchor (1) or not (0).
extern std::atomic<int> g_tune_warm_bound;
//  topk_min: smallest top-k list capacity used (0: the smallest of 4, 8, 16,
//    32, 64 that holds k; otherwise at least this one) -- the k-tiling of the
//    register lists.
extern std::atomic<int> g_tune_topk_min;
//  warm_mult: float lists whose k equals their capacity start warm from the
//    k nearest of warm_mult x k tree-order neighbours (1: from k of them).
extern std::atomic<int> g_tune_warm_mult;

// Status sink of this host thread (pptkg_set_status_sink): while set, query
// entry points record kernel check failures into this device word and
// neither synchronise nor read it back, so their launches can be captured
// into a CUDA graph.
extern thread_local int* g_status_sink;

// PPTKG_BOUNDS_CHECK builds: the device word (one per device) where the
// query kernels' index checks record the first failing site (TreeView::
// checked), and its read-and-clear; in the normal build bounds_word is null
// and bounds_take 0.
int* bounds_word(int device);
int bounds_take(int device);

#define PPTKG_CHECK_LAUNCH()          \
  do {                                \
    ::pptkg::g_launches++;            \
    PPTKG_CUDA(cudaGetLastError());   \
  } while (0)

// ------------------------------------------------------------ dtype codes --
// Identical to include/pptkg.h.
enum DType { F32 = 0, F64 = 1, I8 = 2, I16 = 3, I32 = 4, I64 = 5, U8 = 6, U16 = 7, U32 = 8, U64 = 9 };

template <typename T>
constexpr int dtype_code() {
  if constexpr (std::is_same<T, float>::value) return F32;
  else if constexpr (std::is_same<T, double>::value) return F64;
  else if constexpr (std::is_signed<T>::value) return sizeof(T) == 1 ? I8 : sizeof(T) == 2 ? I16 : sizeof(T) == 4 ? I32 : I64;
  else return sizeof(T) == 1 ? U8 : sizeof(T) == 2 ? U16 : sizeof(T) == 4 ? U32 : U64;
}

inline int dtype_size(int dt) {
  switch (dt) {
    case F32: case I32: case U32: return 4;
    case F64: case I64: case U64: return 8;
    case I16: case U16: return 2;
    case I8: case U8: return 1;
  }
  return 0;
}

// Distance arithmetic type: float for float32 and all integer types, double
// for float64 (pptk/kdtree/src/accumulator.h:13-27).
template <typename T> struct DistOf { typedef float type; };
template <> struct DistOf<double> { typedef double type; };

// Largest and lowest finite values of a point type (all ten pptk dtypes).
template <typename T> struct Limits {
  __host__ __device__ static constexpr T max() { return std::numeric_limits<T>::max(); }
  __host__ __device__ static constexpr T lowest() { return std::numeric_limits<T>::lowest(); }
};

// --------------------------------------------- exact (uncontracted) math --
// Every operation below rounds once, as the reference's x86-64 SSE build does
// (no -march, hence no FMA; pptk CMakeLists.txt:4).
__device__ __forceinline__ float xsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float xadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float xmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float xdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double xsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double xadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double xmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double xdiv(double a, double b) { return __ddiv_rn(a, b); }

// ------------------------------------------ ordered integer images (min/max)
// Monotone map from a float/double to an unsigned integer so that atomicMin /
// atomicMax on the image order like the values (NaN excluded; -0 < +0).
__host__ __device__ __forceinline__ uint32_t ord_of(float f) {
  uint32_t u = *reinterpret_cast<uint32_t*>(&f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__host__ __device__ __forceinline__ float from_ord(uint32_t u) {
  u = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
  return *reinterpret_cast<float*>(&u);
}
__host__ __device__ __forceinline__ unsigned long long ord_of(double f) {
  unsigned long long u = *reinterpret_cast<unsigned long long*>(&f);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__host__ __device__ __forceinline__ double from_ord(unsigned long long u) {
  u = (u & 0x8000000000000000ull) ? (u & 0x7fffffffffffffffull) : ~u;
  return *reinterpret_cast<double*>(&u);
}

// The same monotone images for every point type (ord_t / from_ord_t):
// floats as above; integers of up to 32 bits as unsigned 32-bit with the
// sign bit flipped for signed types; 64-bit integers likewise in 64 bits.
template <typename T> struct OrdOf {
  typedef typename std::conditional<(sizeof(T) > 4), unsigned long long, uint32_t>::type type;
};

template <typename T>
__host__ __device__ __forceinline__ typename OrdOf<T>::type ord_t(T v) {
  typedef typename OrdOf<T>::type U;
  if constexpr (std::is_floating_point<T>::value) {
    return ord_of(v);
  } else if constexpr (std::is_signed<T>::value) {
    typedef typename std::conditional<(sizeof(T) > 4), long long, int32_t>::type S;
    return (U)(S)v ^ ((U)1 << (sizeof(U) * 8 - 1));
  } else {
    return (U)v;
  }
}

template <typename T>
__host__ __device__ __forceinline__ T from_ord_t(typename OrdOf<T>::type u) {
  typedef typename OrdOf<T>::type U;
  if constexpr (std::is_floating_point<T>::value) {
    return from_ord(u);
  } else if constexpr (std::is_signed<T>::value) {
    typedef typename std::conditional<(sizeof(T) > 4), long long, int32_t>::type S;
    return (T)(S)(u ^ ((U)1 << (sizeof(U) * 8 - 1)));
  } else {
    return (T)u;
  }
}

// A coordinate the reference keeps (ValidPointIndices drops NaN/inf rows;
// integer coordinates are always kept).
template <typename T>
__host__ __device__ __forceinline__ bool valid_coord(T v) {
  if constexpr (std::is_floating_point<T>::value)
    return isfinite(v);
  else
    return true;
}

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }
__host__ __device__ __forceinline__ int div_up_dev(int a, int b) { return (a + b - 1) / b; }

}  // namespace pptkg

// C ABI (include/pptkg.h): argument checks, host/device staging, dispatch on
// element type and dimension, and error reporting.
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "build.cuh"
#include "persist.cuh"
#include "pptkg.h"
#include "profile.cuh"
#include "query.cuh"
#include "util.cuh"

struct pptkg_tree {
  std::unique_ptr<pptkg::TreeBase> t;
};

namespace {

using namespace pptkg;

thread_local std::string g_msg;
thread_local int g_code = 0;

template <typename F>
int guarded(F&& f) {
  try {
    keep_pool_cached(0);
    f();
#ifdef PPTKG_BOUNDS_CHECK
    // index checks of the query kernels (not while a status sink is set:
    // reading the word would synchronise a capture)
    if (!g_status_sink) {
      int dev = 0;
      cudaGetDevice(&dev);
      static const char* const kSite[] = {"", "point record", "index map", "traversal node"};
      if (const int site = bounds_take(dev))
        throw Error(E_DEVICE, std::string("bounds check failed: ") +
                                  (site > 0 && site < 4 ? kSite[site] : "unknown") + " index out of range");
    }
#endif
    return PPTKG_OK;
  } catch (const Error& e) {
    g_msg = e.what();
    g_code = e.code;
  } catch (const std::bad_alloc&) {
    g_msg = "host allocation failed";
    g_code = PPTKG_E_CUDA;
  } catch (const std::exception& e) {
    g_msg = e.what();
    g_code = PPTKG_E_INVALID;
  }
  return g_code;
}

inline cudaStream_t S(void* s) { return (cudaStream_t)s; }

// Device view of a caller array: used in place when it already lives on the
// device, otherwise copied in (and, for outputs, copied back by flush()).
template <typename T>
struct Staged {
  T* d = nullptr;
  void* user = nullptr;
  size_t count = 0;
  bool host = false;
  DevBuf<T> buf;
  Staged(const void* p, size_t n, int mem, bool copy_in, cudaStream_t st) {
    user = const_cast<void*>(p);
    count = n;
    if (!p) return;
    if (mem == PPTKG_MEM_DEVICE) {
      d = (T*)p;
      return;
    }
    if (mem != PPTKG_MEM_HOST) throw Error(E_INVALID, "mem must be PPTKG_MEM_HOST or PPTKG_MEM_DEVICE");
    host = true;
    buf.alloc(std::max<size_t>(n, 1), st);
    d = buf.get();
    if (copy_in && n) {
      Stage s("h2d", st);
      PPTKG_CUDA(cudaMemcpyAsync(d, p, n * sizeof(T), cudaMemcpyDefault, st));
    }
  }
  void flush(cudaStream_t st) {
    if (host && user && count) {
      Stage s("d2h", st);
      PPTKG_CUDA(cudaMemcpyAsync(user, d, count * sizeof(T), cudaMemcpyDefault, st));
    }
  }
};

template <typename F>
void dispatch_float(int dtype, F&& f) {
  if (dtype == F32)
    f(float());
  else if (dtype == F64)
    f(double());
  else
    throw Error(E_TYPE, "points must be float32 or float64 (dtype code " + std::to_string(dtype) + ")");
}

template <int D>
struct Dim {
  static constexpr int value = D;
};

template <typename F>
void dispatch_build(int dtype, int dim, F&& f) {
  dispatch_float(dtype, [&](auto t) {
    if (dim == 2)
      f(t, Dim<2>());
    else if (dim == 3)
      f(t, Dim<3>());
    else if (dim == 4)
      f(t, Dim<4>());
    else
      throw Error(E_TYPE, "k-d tree dim must be 2, 3 or 4 (got " + std::to_string(dim) + ")");
  });
}

// Every point type the reference builds trees of (kdtree_wrapper.cpp:15-55).
template <typename F>
void dispatch_any(int dtype, F&& f) {
  switch (dtype) {
    case F32: f(float()); break;
    case F64: f(double()); break;
    case I8: f(int8_t()); break;
    case I16: f(int16_t()); break;
    case I32: f(int32_t()); break;
    case I64: f(int64_t()); break;
    case U8: f(uint8_t()); break;
    case U16: f(uint16_t()); break;
    case U32: f(uint32_t()); break;
    case U64: f(uint64_t()); break;
    default: throw Error(E_TYPE, "unsupported point dtype code " + std::to_string(dtype));
  }
}

template <typename F>
void dispatch_build_any(int dtype, int dim, F&& f) {
  dispatch_any(dtype, [&](auto t) {
    if (dim == 2)
      f(t, Dim<2>());
    else if (dim == 3)
      f(t, Dim<3>());
    else if (dim == 4)
      f(t, Dim<4>());
    else
      throw Error(E_TYPE, "k-d tree dim must be 2, 3 or 4 (got " + std::to_string(dim) + ")");
  });
}

template <typename F>
void dispatch_query(const TreeBase* t, F&& f) {
  if (t->dim != 3) throw Error(E_UNSUPPORTED, "forest and multi-tree queries need 3-d trees");
  dispatch_float(t->dtype, [&](auto tt) { f(tt, Dim<3>()); });
}

// kNN / r-near on single trees of any built dimension (2, 3, 4).
template <typename F>
void dispatch_query_dims(const TreeBase* t, F&& f) {
  dispatch_float(t->dtype, [&](auto tt) {
    switch (t->dim) {
      case 2: f(tt, Dim<2>()); break;
      case 3: f(tt, Dim<3>()); break;
      case 4: f(tt, Dim<4>()); break;
      default: throw Error(E_TYPE, "k-d tree dim must be 2, 3 or 4");
    }
  });
}

// The tree of a handle, for the capturable forest entries (no host work).
TreeBase* tree_raw(const pptkg_tree* t) {
  if (!t || !t->t) throw Error(E_INVALID, "null tree");
  return t->t.get();
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    PPTKG_CUDA(cudaGetDevice(&prev));
    if (prev != dev) PPTKG_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != prev && prev >= 0) cudaSetDevice(prev);
  }
};

// The tree of a handle with host-side counts that match the device: a
// capture-ready forest's last rebuild is read back first (a device-wide
// synchronisation; these entries are not captured).
const TreeBase* tree_of(const pptkg_tree* h) {
  TreeBase* t = tree_raw(h);
  if (t->capture) {
    DeviceGuard g(t->device);
    PPTKG_CUDA(cudaDeviceSynchronize());
    dispatch_float(t->dtype, [&](auto tt) {
      typedef decltype(tt) T;
      switch (t->dim) {
        case 2: forest_sync<T, 2>(t, 0); break;
        case 3: forest_sync<T, 3>(t, 0); break;
        default: forest_sync<T, 4>(t, 0); break;
      }
    });
  }
  return t;
}


constexpr int DEFAULT_BUCKET = 64;
constexpr double DEFAULT_GAP = 1e-3;

// Preorder serialization of the reference node list (node.h:15-29): each
// record is preceded by its chain of empty-split nodes (kdtree-impl.h:
// 114-158); a record without split or trims adds no node.
template <typename T, int D>
void serialize_nodes(const std::vector<Rec<T, D>>& recs, int r, int64_t base, std::vector<double>& out) {
  if (r < 0) return;
  const Rec<T, D>& rec = recs[r];
  const bool split = rec.split_dim >= 0;
  const int nt = std::min<int>(rec.ntrim, 2 * D);
  for (int i = 0; i < nt; i++) {
    const int dim = rec.trim[i] >> 1, side = rec.trim[i] & 1;
    const bool has_next = (i + 1 < nt) || split;
    out.push_back(dim);
    out.push_back((double)((side == 0 ? rec.begin : rec.end) - base));
    out.push_back(side == 0 ? (double)rec.lo[dim] : (double)rec.hi[dim]);
    out.push_back(side == 1 && has_next ? 1.0 : 0.0);
    out.push_back(side == 0 && has_next ? 1.0 : 0.0);
  }
  if (!split) return;
  auto emits = [&](int c) { return c >= 0 && (recs[c].split_dim >= 0 || recs[c].ntrim > 0); };
  out.push_back(rec.split_dim);
  out.push_back((double)(rec.split_index - base));
  out.push_back((double)rec.split_val);
  out.push_back(emits(rec.left) ? 1.0 : 0.0);
  out.push_back(emits(rec.right) ? 1.0 : 0.0);
  serialize_nodes<T, D>(recs, rec.left, base, out);
  serialize_nodes<T, D>(recs, rec.right, base, out);
}

// Shared staging of an r-near query batch.
struct RnearArgs {
  DevBuf<char> qbuf;
  pptkg::QuerySpec qs;
};

template <int Dm>
static void stage_rnear(RnearArgs& a, const pptkg::TreeBase* t, const void* queries, const int32_t* indices, int64_t m,
                        int qdtype, int mem, cudaStream_t st, std::unique_ptr<Staged<int32_t>>& idx) {
  a.qs.m = m;
  if (queries) {
    if (qdtype != F32 && qdtype != F64) throw Error(E_TYPE, "query points must be float32 or float64");
    a.qs.qdtype = qdtype;
    const size_t bytes = (size_t)m * Dm * dtype_size(qdtype);
    if (mem == PPTKG_MEM_HOST && m) {
      a.qbuf.alloc(bytes, st);
      PPTKG_CUDA(cudaMemcpyAsync(a.qbuf.get(), queries, bytes, cudaMemcpyDefault, st));
      a.qs.pts = a.qbuf.get();
    } else {
      a.qs.pts = queries;
    }
  } else {
    if (!indices && m > t->n) throw Error(E_RANGE, "query rows exceed the point count");
    idx.reset(new Staged<int32_t>(indices, (size_t)m, mem, true, st));
    a.qs.idx = idx->d;
    a.qs.exclude_self = true;
  }
}

static void run_normals(const TreeBase* t, const int32_t* indices, int64_t m, int mem, int k, float r, int num_eigen,
                        int precision, void* out_evecs, void* out_evals, int32_t* out_sizes, cudaStream_t st) {
  if (t->dim != 3) throw Error(E_TYPE, "normals need 3-d points");
  if (t->rec_dtype != F32 && t->rec_dtype != F64) throw Error(E_TYPE, "normals need float32 or float64 points");
  if (num_eigen != 1 && num_eigen != 3) throw Error(E_INVALID, "num_eigen must be 1 or 3");
  if (!(r > 0.0f)) throw Error(E_INVALID, "r must be positive");
  if (k == 0) throw Error(E_INVALID, "k cannot be zero");
  if (k < 0 && r == INFINITY) throw Error(E_INVALID, "invalid combo: r == inf and k < 0");
  if (k < -1) throw Error(E_INVALID, "k must be positive or -1");
  dispatch_float(t->dtype, [&](auto tt) {
    typedef decltype(tt) T;
    Staged<int32_t> qi(indices, (size_t)m, mem, true, st);
    Staged<T> ev(out_evecs, (size_t)m * 3 * num_eigen, mem, false, st);
    Staged<T> ew(out_evals, (size_t)m * num_eigen, mem, false, st);
    Staged<int32_t> sz(out_sizes, (size_t)m, mem, false, st);
    QuerySpec qs;
    qs.m = m;
    qs.idx = qi.d;
    qs.exclude_self = false;
    normals_query<T>(t, qs, k, r, num_eigen, precision, DEFAULT_GAP, ev.d, ew.d, sz.d, st);
    ev.flush(st);
    ew.flush(st);
    sz.flush(st);
    PPTKG_CUDA(cudaStreamSynchronize(st));
  });
}

}  // namespace

extern "C" {

static int ref_nodes(const pptkg_tree* tree, int cloud, double* out, int64_t capacity, int64_t* count);

int pptkg_version(void) { return 100; }

int pptkg_bounds_checked(void) {
#ifdef PPTKG_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

int pptkg_last_error(char* buf, size_t len) {
  if (buf && len) {
    size_t n = std::min(len - 1, g_msg.size());
    memcpy(buf, g_msg.data(), n);
    buf[n] = 0;
  }
  return g_code;
}

int pptkg_tree_build(const void* points, int64_t n, int dim, int dtype, int mem, int max_leaf_size,
                     double empty_split, void* stream, pptkg_tree** out) {
  return guarded([&] {
    if (!out) throw Error(E_INVALID, "out is null");
    *out = nullptr;
    if (n < 0) throw Error(E_INVALID, "negative point count");
    if (n > 0 && !points) throw Error(E_INVALID, "points is null");
    if (!(empty_split >= 0.0)) throw Error(E_INVALID, "emptysplit must be non-negative");
    dispatch_build_any(dtype, dim, [&](auto t, auto d) {
      typedef decltype(t) T;
      constexpr int Dm = decltype(d)::value;
      Staged<T> in(points, (size_t)n * Dm, mem, true, S(stream));
      std::unique_ptr<pptkg_tree> h(new pptkg_tree());
      h->t.reset(build_tree<T, Dm>(in.d, n, max_leaf_size, empty_split, DEFAULT_BUCKET, S(stream)));
      *out = h.release();
    });
  });
}

int pptkg_forest_build(const void* points, int64_t n, int dim, int dtype, int mem, const int64_t* offsets,
                       int ncloud, int max_leaf_size, double empty_split, void* stream, pptkg_tree** out) {
  return guarded([&] {
    if (!out) throw Error(E_INVALID, "out is null");
    *out = nullptr;
    if (n < 0) throw Error(E_INVALID, "negative point count");
    if (n > 0 && !points) throw Error(E_INVALID, "points is null");
    if (ncloud < 1 || !offsets) throw Error(E_INVALID, "need at least one cloud and its offsets");
    if (!(empty_split >= 0.0)) throw Error(E_INVALID, "emptysplit must be non-negative");
    dispatch_build(dtype, dim, [&](auto t, auto d) {
      typedef decltype(t) T;
      constexpr int Dm = decltype(d)::value;
      Staged<T> in(points, (size_t)n * Dm, mem, true, S(stream));
      std::unique_ptr<pptkg_tree> h(new pptkg_tree());
      h->t.reset(build_forest<T, Dm>(in.d, n, offsets, ncloud, max_leaf_size, empty_split, DEFAULT_BUCKET, S(stream)));
      *out = h.release();
    });
  });
}

int pptkg_forest_capture_ready(pptkg_tree* forest, void* stream) {
  return guarded([&] {
    TreeBase* t = const_cast<TreeBase*>(tree_of(forest));
    DeviceGuard g(t->device);
    if (t->rec_dtype != F32 && t->rec_dtype != F64)
      throw Error(E_TYPE, "capture mode needs a float32 or float64 forest");
    dispatch_build(t->dtype, t->dim, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      forest_capture_ready<T, Dm>(t, S(stream));
    });
    forest_slot_map_device(t, S(stream));
    PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
  });
}

int pptkg_forest_rebuild(pptkg_tree* forest, const void* points, void* stream) {
  return guarded([&] {
    TreeBase* t = tree_raw(forest);
    DeviceGuard g(t->device);
    if (!t->capture) throw Error(E_INVALID, "pptkg_forest_rebuild needs a capture-ready forest");
    if (t->n > 0 && !points) throw Error(E_INVALID, "points is null");
    // with a status sink set nothing is read back (the call can be
    // captured); otherwise the status is checked here
    DevBuf<int> own;
    int* status = g_status_sink;
    if (!status) {
      own.alloc(1, S(stream));
      PPTKG_CUDA(cudaMemsetAsync(own.get(), 0, sizeof(int), S(stream)));
      status = own.get();
    }
    dispatch_build(t->dtype, t->dim, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      rebuild_forest<T, Dm>(t, (const T*)points, S(stream), status);
    });
    forest_slot_map_device(t, S(stream));
    if (!g_status_sink) {
      int h = 0;
      PPTKG_CUDA(cudaMemcpyAsync(&h, status, sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
      if (h == 20) throw Error(E_UNSUPPORTED, "forest rebuild: the points need more tree levels than planned");
      if (h == 21) throw Error(E_UNSUPPORTED, "forest rebuild: the points need more tree records than planned");
      if (h) throw Error(E_DEVICE, "forest rebuild: device check failed (code " + std::to_string(h) + ")");
    }
  });
}

int pptkg_forest_info(const pptkg_tree* forest, int* ncloud, int64_t* valid_offsets) {
  return guarded([&] {
    const TreeBase* t = tree_of(forest);
    if (ncloud) *ncloud = t->ncloud;
    if (valid_offsets) std::copy(t->valid_off_h.begin(), t->valid_off_h.end(), valid_offsets);
  });
}

int pptkg_forest_ref_nodes(const pptkg_tree* forest, int cloud, double* out, int64_t capacity, int64_t* count) {
  if (cloud < 0) {
    g_msg = "cloud index out of range";
    g_code = PPTKG_E_INVALID;
    return g_code;
  }
  return ref_nodes(forest, cloud, out, capacity, count);
}

int pptkg_forest_knn(const pptkg_tree* forest, int k, double dmax, int exclude_self, int mem, int32_t* out_idx,
                     int32_t* out_cnt, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_raw(forest);
    DeviceGuard g(t->device);
    if (k < 1) throw Error(E_INVALID, "k must be positive");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (t->n && !out_idx) throw Error(E_INVALID, "out_idx is null");
    dispatch_query(t, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      Staged<int32_t> oi(out_idx, (size_t)t->n * k, mem, false, S(stream));
      Staged<int32_t> oc(out_cnt, (size_t)t->n, mem, false, S(stream));
      forest_knn<T, Dm>(t, k, dmax, exclude_self != 0, oi.d, oc.d, S(stream));
      oi.flush(S(stream));
      oc.flush(S(stream));
      if (!(g_status_sink && mem == PPTKG_MEM_DEVICE)) PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_forest_normals(const pptkg_tree* forest, int k, float r, int num_eigen, int precision, int mem,
                         void* out_evecs, void* out_evals, int32_t* out_sizes, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_raw(forest);
    DeviceGuard g(t->device);
    if (num_eigen != 1 && num_eigen != 3) throw Error(E_INVALID, "num_eigen must be 1 or 3");
    if (!(r > 0.0f)) throw Error(E_INVALID, "r must be positive");
    dispatch_float(t->dtype, [&](auto tt) {
      typedef decltype(tt) T;
      Staged<T> ev(out_evecs, (size_t)t->n * 3 * num_eigen, mem, false, S(stream));
      Staged<T> ew(out_evals, (size_t)t->n * num_eigen, mem, false, S(stream));
      Staged<int32_t> sz(out_sizes, (size_t)t->n, mem, false, S(stream));
      forest_normals<T>(t, k, r, num_eigen, precision, DEFAULT_GAP, ev.d, ew.d, sz.d, S(stream));
      ev.flush(S(stream));
      ew.flush(S(stream));
      sz.flush(S(stream));
      if (!(g_status_sink && mem == PPTKG_MEM_DEVICE)) PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_forest_knn_normals(const pptkg_tree* forest, int k, float r, int num_eigen, int precision, int mem,
                             int32_t* out_idx, int32_t* out_cnt, void* out_evecs, void* out_evals,
                             int32_t* out_sizes, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_raw(forest);
    DeviceGuard g(t->device);
    if (num_eigen != 1 && num_eigen != 3) throw Error(E_INVALID, "num_eigen must be 1 or 3");
    if (!(r > 0.0f)) throw Error(E_INVALID, "r must be positive");
    if (t->n && !out_idx) throw Error(E_INVALID, "out_idx is null");
    dispatch_float(t->dtype, [&](auto tt) {
      typedef decltype(tt) T;
      Staged<int32_t> oi(out_idx, (size_t)t->n * k, mem, false, S(stream));
      Staged<int32_t> oc(out_cnt, (size_t)t->n, mem, false, S(stream));
      Staged<T> ev(out_evecs, (size_t)t->n * 3 * num_eigen, mem, false, S(stream));
      Staged<T> ew(out_evals, (size_t)t->n * num_eigen, mem, false, S(stream));
      Staged<int32_t> sz(out_sizes, (size_t)t->n, mem, false, S(stream));
      forest_normals<T>(t, k, r, num_eigen, precision, DEFAULT_GAP, ev.d, ew.d, sz.d, S(stream), oi.d, oc.d);
      oi.flush(S(stream));
      oc.flush(S(stream));
      ev.flush(S(stream));
      ew.flush(S(stream));
      sz.flush(S(stream));
      if (!(g_status_sink && mem == PPTKG_MEM_DEVICE)) PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

static std::vector<const TreeBase*> tree_list(const pptkg_tree* const* trees, int ntrees) {
  if (ntrees < 1 || !trees) throw Error(E_INVALID, "need at least one tree");
  std::vector<const TreeBase*> v(ntrees);
  for (int g = 0; g < ntrees; g++) v[g] = tree_of(trees[g]);
  for (int g = 1; g < ntrees; g++)
    if (v[g]->device != v[0]->device) throw Error(E_INVALID, "all trees of a batch must live on one device");
  return v;
}

int pptkg_multi_knn(const pptkg_tree* const* trees, int ntrees, const void* queries, const int64_t* row_offsets,
                    int qdtype, int mem, int k, double dmax, int32_t* out_idx, int32_t* out_cnt, void* stream) {
  return guarded([&] {
    std::vector<const TreeBase*> v = tree_list(trees, ntrees);
    DeviceGuard g(v[0]->device);
    if (!row_offsets || row_offsets[0] != 0) throw Error(E_INVALID, "row offsets must start at 0");
    const int64_t m = row_offsets[ntrees];
    if (k < 1) throw Error(E_INVALID, "k must be positive");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (qdtype != F32 && qdtype != F64) throw Error(E_TYPE, "query points must be float32 or float64");
    if (m && (!queries || !out_idx)) throw Error(E_INVALID, "null array");
    dispatch_query(v[0], [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      const size_t bytes = (size_t)m * Dm * dtype_size(qdtype);
      DevBuf<char> qbuf;
      const void* qd = queries;
      if (mem == PPTKG_MEM_HOST && m) {
        qbuf.alloc(bytes, S(stream));
        PPTKG_CUDA(cudaMemcpyAsync(qbuf.get(), queries, bytes, cudaMemcpyDefault, S(stream)));
        qd = qbuf.get();
      }
      Staged<int32_t> oi(out_idx, (size_t)m * k, mem, false, S(stream));
      Staged<int32_t> oc(out_cnt, (size_t)m, mem, false, S(stream));
      multi_knn<T, Dm>(v.data(), ntrees, qd, qdtype, row_offsets, k, dmax, oi.d, oc.d, S(stream));
      oi.flush(S(stream));
      oc.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_multi_normals(const pptkg_tree* const* trees, int ntrees, const int32_t* indices,
                        const int64_t* row_offsets, int mem, int k, float r, int num_eigen, int precision,
                        void* out_evecs, void* out_evals, int32_t* out_sizes, void* stream) {
  return guarded([&] {
    std::vector<const TreeBase*> v = tree_list(trees, ntrees);
    DeviceGuard g(v[0]->device);
    if (!row_offsets || row_offsets[0] != 0) throw Error(E_INVALID, "row offsets must start at 0");
    const int64_t m = row_offsets[ntrees];
    if (v[0]->dim != 3) throw Error(E_TYPE, "normals need 3-d points");
    for (const TreeBase* x : v)
      if (x->rec_dtype != F32 && x->rec_dtype != F64) throw Error(E_TYPE, "normals need float32 or float64 points");
    if (num_eigen != 1 && num_eigen != 3) throw Error(E_INVALID, "num_eigen must be 1 or 3");
    if (!(r > 0.0f)) throw Error(E_INVALID, "r must be positive");
    if (m && !indices) throw Error(E_INVALID, "indices is null");
    dispatch_float(v[0]->dtype, [&](auto tt) {
      typedef decltype(tt) T;
      Staged<int32_t> qi(indices, (size_t)m, mem, true, S(stream));
      Staged<T> ev(out_evecs, (size_t)m * 3 * num_eigen, mem, false, S(stream));
      Staged<T> ew(out_evals, (size_t)m * num_eigen, mem, false, S(stream));
      Staged<int32_t> sz(out_sizes, (size_t)m, mem, false, S(stream));
      multi_normals<T>(v.data(), ntrees, qi.d, row_offsets, k, r, num_eigen, precision, DEFAULT_GAP, ev.d, ew.d,
                       sz.d, S(stream));
      ev.flush(S(stream));
      ew.flush(S(stream));
      sz.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_tree_free(pptkg_tree* tree) {
  return guarded([&] { delete tree; });
}

int pptkg_tree_info(const pptkg_tree* tree, int64_t* n, int64_t* n_valid, int* dim, int* dtype, int64_t* n_records,
                    int* depth) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    if (n) *n = t->n;
    if (n_valid) *n_valid = t->nv;
    if (dim) *dim = t->dim;
    if (dtype) *dtype = t->rec_dtype;
    if (n_records) *n_records = t->n_recs;
    if (depth) *depth = t->depth;
  });
}

int pptkg_tree_reverse_indices(const pptkg_tree* tree, int32_t* out, int mem, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (!out) throw Error(E_INVALID, "out is null");
    dispatch_build(t->dtype, t->dim, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      typedef PointRec<T, Dm> PR;
      const size_t id_off = offsetof(PR, id);
      Staged<int32_t> o(out, t->nv, mem, false, S(stream));
      if (t->nv)
        PPTKG_CUDA(cudaMemcpy2DAsync(o.d, sizeof(int32_t), (const char*)t->pts + id_off, sizeof(PR), sizeof(int32_t),
                                     t->nv, cudaMemcpyDeviceToDevice, S(stream)));
      o.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

static int ref_nodes(const pptkg_tree* tree, int cloud, double* out, int64_t capacity, int64_t* count) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    if (cloud < -1 || cloud >= t->ncloud) throw Error(E_INVALID, "cloud index out of range");
    DeviceGuard g(t->device);
    dispatch_build_any(t->rec_dtype, t->dim, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      std::vector<Rec<T, Dm>> recs(t->n_recs);
      if (t->n_recs)
        PPTKG_CUDA(cudaMemcpy(recs.data(), t->recs, sizeof(Rec<T, Dm>) * t->n_recs, cudaMemcpyDeviceToHost));
      int root = -1;
      PPTKG_CUDA(cudaMemcpy(&root, t->root_rec + (cloud < 0 ? 0 : cloud), sizeof(int), cudaMemcpyDeviceToHost));
      std::vector<double> v;
      const int64_t base = t->valid_off_h.empty() ? 0 : t->valid_off_h[cloud < 0 ? 0 : cloud];
      if (t->n_recs && root >= 0) serialize_nodes<T, Dm>(recs, root, base, v);
      const int64_t cnt = (int64_t)(v.size() / 5);
      if (count) *count = cnt;
      if (out) {
        if (capacity < cnt) throw Error(E_INVALID, "node buffer too small");
        memcpy(out, v.data(), v.size() * sizeof(double));
      }
    });
  });
}

int pptkg_tree_ref_nodes(const pptkg_tree* tree, double* out, int64_t capacity, int64_t* count) {
  return ref_nodes(tree, -1, out, capacity, count);
}

int pptkg_tree_set_bucket(pptkg_tree* tree, int bucket, void* stream) {
  return guarded([&] {
    // (a capture-ready forest's counts are synchronised first)
    TreeBase* t = const_cast<TreeBase*>(tree_of(tree));
    DeviceGuard g(t->device);
    if (bucket < 1 || bucket > 4096) throw Error(E_INVALID, "bucket must be in [1, 4096]");
    dispatch_build_any(t->rec_dtype, t->dim, [&](auto tt, auto d) {
      make_tnodes<decltype(tt), decltype(d)::value>(t, bucket, S(stream));
    });
  });
}

int pptkg_knn(const pptkg_tree* tree, const void* queries, int64_t m, int qdtype, int mem, int k, double dmax,
              int32_t* out_idx, int32_t* out_cnt, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    if (k < 1) throw Error(E_INVALID, "k must be positive");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (qdtype != F32 && qdtype != F64) throw Error(E_TYPE, "query points must be float32 or float64");
    if (m && (!queries || !out_idx)) throw Error(E_INVALID, "null array");
    dispatch_query_dims(t, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      const size_t qn = (size_t)m * Dm;
      QuerySpec qs;
      qs.m = m;
      qs.qdtype = qdtype;
      DevBuf<char> qbuf;
      if (mem == PPTKG_MEM_HOST && m) {
        qbuf.alloc(qn * dtype_size(qdtype), S(stream));
        PPTKG_CUDA(cudaMemcpyAsync(qbuf.get(), queries, qn * dtype_size(qdtype), cudaMemcpyDefault, S(stream)));
        qs.pts = qbuf.get();
      } else {
        qs.pts = queries;
      }
      Staged<int32_t> oi(out_idx, (size_t)m * k, mem, false, S(stream));
      Staged<int32_t> oc(out_cnt, (size_t)m, mem, false, S(stream));
      knn_query<T, Dm>(t, qs, k, dmax, oi.d, oc.d, S(stream));
      oi.flush(S(stream));
      oc.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_knn_self(const pptkg_tree* tree, const int32_t* indices, int64_t m, int mem, int k, double dmax,
                   int32_t* out_idx, int32_t* out_cnt, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    if (k < 1) throw Error(E_INVALID, "k must be positive");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (!indices && m > t->n) throw Error(E_RANGE, "query rows exceed the point count");
    if (m && !out_idx) throw Error(E_INVALID, "out_idx is null");
    dispatch_query_dims(t, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      Staged<int32_t> qi(indices, (size_t)m, mem, true, S(stream));
      QuerySpec qs;
      qs.m = m;
      qs.idx = qi.d;
      qs.exclude_self = true;
      Staged<int32_t> oi(out_idx, (size_t)m * k, mem, false, S(stream));
      Staged<int32_t> oc(out_cnt, (size_t)m, mem, false, S(stream));
      knn_query<T, Dm>(t, qs, k, dmax, oi.d, oc.d, S(stream));
      oi.flush(S(stream));
      oc.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_rnear_count(const pptkg_tree* tree, const void* queries, const int32_t* indices, int64_t m, int qdtype,
                      int mem, double dmax, int64_t* out_offsets, int64_t* total, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (!out_offsets) throw Error(E_INVALID, "out_offsets is null");
    dispatch_query_dims(t, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      RnearArgs a;
      std::unique_ptr<Staged<int32_t>> idx;
      stage_rnear<Dm>(a, t, queries, indices, m, qdtype, mem, S(stream), idx);
      Staged<int64_t> off(out_offsets, (size_t)m + 1, mem, false, S(stream));
      int64_t tot = rnear_count<T, Dm>(t, a.qs, dmax, off.d, S(stream));
      off.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
      if (total) *total = tot;
    });
  });
}

int pptkg_rnear_fill(const pptkg_tree* tree, const void* queries, const int32_t* indices, int64_t m, int qdtype,
                     int mem, double dmax, const int64_t* offsets, int32_t* out_idx, void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    if (!(dmax >= 0.0)) throw Error(E_INVALID, "dmax must be non-negative");
    if (!offsets) throw Error(E_INVALID, "offsets is null");
    dispatch_query_dims(t, [&](auto tt, auto d) {
      typedef decltype(tt) T;
      constexpr int Dm = decltype(d)::value;
      RnearArgs a;
      std::unique_ptr<Staged<int32_t>> idx;
      stage_rnear<Dm>(a, t, queries, indices, m, qdtype, mem, S(stream), idx);
      Staged<int64_t> off(offsets, (size_t)m + 1, mem, true, S(stream));
      int64_t total = 0;
      if (mem == PPTKG_MEM_HOST)
        total = m ? offsets[m] : 0;
      else if (m)
        PPTKG_CUDA(cudaMemcpyAsync(&total, offsets + m, sizeof(int64_t), cudaMemcpyDefault, S(stream)));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
      if (total && !out_idx) throw Error(E_INVALID, "out_idx is null");
      Staged<int32_t> o(out_idx, (size_t)total, mem, false, S(stream));
      rnear_fill<T, Dm>(t, a.qs, dmax, off.d, o.d, S(stream));
      o.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_estimate_normals(const void* points, int64_t n, int dtype, int mem, int k, float r,
                           const int32_t* subsample, int64_t m, int num_eigen, int precision, void* out_evecs,
                           void* out_evals, int32_t* out_sizes, void* stream) {
  return guarded([&] {
    if (n < 0) throw Error(E_INVALID, "negative point count");
    if (n > 0 && !points) throw Error(E_INVALID, "points is null");
    if (!subsample) m = n;
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    dispatch_float(dtype, [&](auto tt) {
      typedef decltype(tt) T;
      Staged<T> in(points, (size_t)n * 3, mem, true, S(stream));
      std::unique_ptr<TreeBase> t(build_tree<T, 3>(in.d, n, 10, 0.2, DEFAULT_BUCKET, S(stream)));
      run_normals(t.get(), subsample, m, mem, k, r, num_eigen, precision, out_evecs, out_evals, out_sizes,
                  S(stream));
    });
  });
}

int pptkg_tree_normals(const pptkg_tree* tree, const int32_t* indices, int64_t m, int mem, int k, float r,
                       int num_eigen, int precision, void* out_evecs, void* out_evals, int32_t* out_sizes,
                       void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    if (t->dim != 3) throw Error(E_TYPE, "normals need 3-d points");
    if (t->rec_dtype != F32 && t->rec_dtype != F64) throw Error(E_TYPE, "normals need float32 or float64 points");
    // NULL indices mean every row: outputs are sized for n rows
    if (!indices && m != 0 && m != t->n)
      throw Error(E_INVALID, "with indices NULL, m must be 0 or the tree's row count (every row is answered)");
    if (!indices) m = t->n;
    if (m < 0 || m > INT32_MAX) throw Error(E_INVALID, "query count out of range");
    run_normals(t, indices, m, mem, k, r, num_eigen, precision, out_evecs, out_evals, out_sizes, S(stream));
  });
}

// The allocation-free entry takes device memory only: a host pointer would be
// read by the kernels as if it were a device address.  Rejects (without
// touching the memory) anything that is not device or managed memory
// reachable from the tree's device.
static void require_device_memory(const void* p, int device, const char* what) {
  if (!p) return;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    (void)cudaGetLastError();
    throw Error(E_INVALID, std::string(what) + ": not a pointer the CUDA runtime knows");
  }
  if (a.type == cudaMemoryTypeManaged) return;
  if (a.type != cudaMemoryTypeDevice)
    throw Error(E_INVALID, std::string(what) + " must point to device memory (host memory given)");
  if (a.device != device) throw Error(E_INVALID, std::string(what) + " lies on another device than the tree");
}

int pptkg_tree_normals_noalloc(const pptkg_tree* tree, const int32_t* indices, int64_t m, int k, float r,
                               int num_eigen, int precision, void* out_evecs, void* out_evals, int32_t* out_sizes,
                               void* stream) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    require_device_memory(indices, t->device, "indices");
    require_device_memory(out_evecs, t->device, "out_evecs");
    require_device_memory(out_evals, t->device, "out_evals");
    require_device_memory(out_sizes, t->device, "out_sizes");
    if (t->dim != 3) throw Error(E_TYPE, "normals need 3-d points");
    if (t->rec_dtype != F32 && t->rec_dtype != F64) throw Error(E_TYPE, "normals need float32 or float64 points");
    if (num_eigen != 1 && num_eigen != 3) throw Error(E_INVALID, "num_eigen must be 1 or 3");
    if (!(r > 0.0f)) throw Error(E_INVALID, "r must be positive");
    if (precision < PPTKG_PREC_AUTO || precision > PPTKG_PREC_FP64) throw Error(E_INVALID, "unknown precision");
    if (!indices && m == 0) m = t->n;
    if (m > 0 && !out_evecs && !out_evals && !out_sizes) throw Error(E_INVALID, "no output requested");
    dispatch_float(t->dtype, [&](auto tt) {
      typedef decltype(tt) T;
      normals_noalloc<T>(t, indices, m, k, r, num_eigen, precision, (T*)out_evecs, (T*)out_evals, out_sizes,
                         S(stream));
    });
  });
}

int pptkg_eigh3(const void* A, int64_t m, int dtype, int mem, void* w, void* V, int layout, void* stream) {
  return guarded([&] {
    if (m < 0) throw Error(E_INVALID, "negative count");
    if (layout != 0 && layout != 1) throw Error(E_INVALID, "layout must be 0 or 1");
    if (m && (!A || !w || !V)) throw Error(E_INVALID, "null array");
    dispatch_float(dtype, [&](auto tt) {
      typedef decltype(tt) T;
      Staged<T> a(A, (size_t)m * 9, mem, true, S(stream));
      Staged<T> ww(w, (size_t)m * 3, mem, false, S(stream));
      Staged<T> vv(V, (size_t)m * 9, mem, false, S(stream));
      eigh3_batched<T>(a.d, m, ww.d, vv.d, layout, S(stream));
      ww.flush(S(stream));
      vv.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_nbhd_covariance(const void* points, int64_t n, int dtype, int mem, const int64_t* offsets,
                          const int32_t* indices, int64_t m, void* out_cov, void* stream) {
  return guarded([&] {
    if (n < 0 || m < 0) throw Error(E_INVALID, "negative count");
    if (m && (!points || !offsets || !out_cov)) throw Error(E_INVALID, "null array");
    dispatch_float(dtype, [&](auto tt) {
      typedef decltype(tt) T;
      int64_t total = 0;
      if (m) {
        if (mem == PPTKG_MEM_HOST) {
          total = offsets[m];
        } else {
          PPTKG_CUDA(cudaMemcpyAsync(&total, offsets + m, sizeof(int64_t), cudaMemcpyDefault, S(stream)));
          PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
        }
      }
      if (total < 0) throw Error(E_INVALID, "negative offsets");
      if (total && !indices) throw Error(E_INVALID, "indices is null");
      Staged<T> p(points, (size_t)n * 3, mem, true, S(stream));
      Staged<int64_t> o(offsets, (size_t)m + 1, mem, true, S(stream));
      Staged<int32_t> ix(indices, (size_t)total, mem, true, S(stream));
      Staged<T> c(out_cov, (size_t)m * 9, mem, false, S(stream));
      nbhd_covariance<T>(p.d, n, o.d, ix.d, total, m, c.d, S(stream));
      c.flush(S(stream));
      PPTKG_CUDA(cudaStreamSynchronize(S(stream)));
    });
  });
}

int pptkg_tree_save(const pptkg_tree* tree, void* buf, int64_t capacity, int64_t* size) {
  return guarded([&] {
    const TreeBase* t = tree_of(tree);
    DeviceGuard g(t->device);
    std::vector<char> blob = save_tree(t, t->stream);
    if (size) *size = (int64_t)blob.size();
    if (buf) {
      if (capacity < (int64_t)blob.size()) throw Error(E_INVALID, "buffer too small for the stored tree");
      memcpy(buf, blob.data(), blob.size());
    }
  });
}

int pptkg_tree_load(const void* buf, int64_t size, void* stream, pptkg_tree** out) {
  return guarded([&] {
    if (!out) throw Error(E_INVALID, "out is null");
    *out = nullptr;
    if (size < 0) throw Error(E_INVALID, "negative size");
    std::unique_ptr<pptkg_tree> h(new pptkg_tree());
    h->t.reset(load_tree((const char*)buf, (size_t)size, S(stream)));
    *out = h.release();
  });
}

}  // extern "C"

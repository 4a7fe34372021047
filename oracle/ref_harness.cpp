// Test infrastructure (oracle side). Never linked into the product library.
//
// A thin C driver around the reference's own header-only k-d tree
// (pptk/kdtree/src/*.h), compiled in place from the reference sources by
// oracle/build_oracle.py into oracle/_ref/libpptk_ref.so.  It exposes the
// reference build, kNN and r-near queries (point and self forms) through
// plain pointers so that tests and the CPU baseline can run the reference
// code itself.  TBB is not installed, so the batch loops are OpenMP
// `parallel for` over the very per-query methods that the reference's TBB
// parallel_for bodies call (kdtree-impl.h:718-770); the build is the serial
// RecursiveBuildHelper, which yields the same tree as the TBB BuildTask
// (both call MakeNode, kdtree-impl.h:306-308 vs :656-663).
//
// estimate_normals is restated here on top of the reference tree because
// Eigen is not installed: the loop, the neighbourhood query and the
// covariance follow estimate_normals.cpp:64-110; the 3x3 symmetric
// eigensolve is cyclic Jacobi (Golub & Van Loan, Matrix Computations,
// 4th ed., Alg. 8.5.2 sym.schur2 + 8.5.3 cyclic Jacobi) in place of Eigen's
// SelfAdjointEigenSolver.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#include "common.h"
#include "kdtree.h"

namespace {

using oracle::dispatch;
using oracle::dispatch_type;

struct Handle {
  void* tree;
  int dtype;
  int dim;
  int64_t n;
};

template <typename T>
void serialize(const pointkd::Node<T>* node, std::vector<double>& out) {
  // preorder; 5 doubles per node: dim, index, value, has_left, has_right
  if (!node) return;
  out.push_back((double)node->split_dim);
  out.push_back((double)node->split_index);
  out.push_back((double)node->split_value);
  out.push_back(node->left ? 1.0 : 0.0);
  out.push_back(node->right ? 1.0 : 0.0);
  serialize(node->left, out);
  serialize(node->right, out);
}

}  // namespace

extern "C" {

// Builds the reference k-d tree over n contiguous AoS points of `dtype`.
void* ref_build(const void* pts, int64_t n, int dim, int dtype, int max_leaf_size, double empty_split) {
  Handle* h = new Handle{nullptr, dtype, dim, n};
  pointkd::BuildParams params;
  params.num_proc = 1;
  params.max_leaf_size = max_leaf_size;
  params.empty_split_threshold = empty_split;
  bool ok = dispatch(dtype, dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    h->tree = new pointkd::KdTree<T, D>((const T*)pts, (int)n, params);
  });
  if (!ok) {
    delete h;
    return nullptr;
  }
  return h;
}

void ref_free(void* hp) {
  Handle* h = (Handle*)hp;
  if (!h) return;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    delete (pointkd::KdTree<T, D>*)h->tree;
  });
  delete h;
}

int64_t ref_num_valid(void* hp) {
  Handle* h = (Handle*)hp;
  int64_t r = 0;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    r = ((pointkd::KdTree<T, D>*)h->tree)->num_points();
  });
  return r;
}

// reverse_indices_: tree position -> original index (num_valid entries).
void ref_reverse_indices(void* hp, int32_t* out) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    const auto& v = ((pointkd::KdTree<T, D>*)h->tree)->reverse_indices();
    std::copy(v.begin(), v.end(), out);
  });
}

// Preorder node list, 5 doubles per node (split dim, split index, split
// value, has left, has right).  Returns the node count; `out` may be NULL.
int64_t ref_tree_nodes(void* hp, double* out) {
  Handle* h = (Handle*)hp;
  std::vector<double> v;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    serialize(((pointkd::KdTree<T, D>*)h->tree)->root(), v);
  });
  if (out) std::copy(v.begin(), v.end(), out);
  return (int64_t)(v.size() / 5);
}

static int threads_or_max(int nthreads) { return nthreads > 0 ? nthreads : omp_get_max_threads(); }

// kNN for m point queries (AoS, dtype qdtype); out_idx is m x k, padded -1.
void ref_knn(void* hp, const void* q, int64_t m, int qdtype, int k, double dmax, int32_t* out_idx,
             int32_t* out_cnt, int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    typedef pointkd::KdTree<T, D> Tree;
    const Tree* tree = (const Tree*)h->tree;
    oracle::dispatch_query<T>(qdtype, h->dtype, [&](auto qt) {
      typedef decltype(qt) Q;
      const Q* qp = (const Q*)q;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads_or_max(nthreads))
      for (int64_t i = 0; i < m; i++) {
        pointkd::Indices res;
        tree->KNearestNeighbors(res, qp + i * D, k, (typename Tree::DistT)dmax);
        for (int j = 0; j < k; j++) out_idx[i * k + j] = j < (int)res.size() ? res[j] : -1;
        out_cnt[i] = (int32_t)res.size();
      }
    });
  });
}

void ref_knn_self(void* hp, const int32_t* qidx, int64_t m, int k, double dmax, int32_t* out_idx,
                  int32_t* out_cnt, int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    typedef pointkd::KdTree<T, D> Tree;
    const Tree* tree = (const Tree*)h->tree;
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads_or_max(nthreads))
    for (int64_t i = 0; i < m; i++) {
      pointkd::Indices res;
      tree->KNearestNeighborsSelf(res, qidx[i], k, (typename Tree::DistT)dmax);
      for (int j = 0; j < k; j++) out_idx[i * k + j] = j < (int)res.size() ? res[j] : -1;
      out_cnt[i] = (int32_t)res.size();
    }
  });
}

// r-near.  Call with out == NULL to fill offsets (m + 1 entries, exclusive
// prefix of the per-query counts); call again with out sized offsets[m].
void ref_rnear(void* hp, const void* q, int64_t m, int qdtype, double dmax, int64_t* offsets, int32_t* out,
               int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    typedef pointkd::KdTree<T, D> Tree;
    const Tree* tree = (const Tree*)h->tree;
    oracle::dispatch_query<T>(qdtype, h->dtype, [&](auto qt) {
      typedef decltype(qt) Q;
      const Q* qp = (const Q*)q;
      std::vector<int64_t> cnt(m);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads_or_max(nthreads))
      for (int64_t i = 0; i < m; i++) {
        pointkd::Indices res;
        tree->RNearNeighbors(res, qp + i * D, (typename Tree::DistT)dmax);
        cnt[i] = (int64_t)res.size();
        if (out) std::copy(res.begin(), res.end(), out + offsets[i]);
      }
      if (!out) {
        offsets[0] = 0;
        for (int64_t i = 0; i < m; i++) offsets[i + 1] = offsets[i] + cnt[i];
      }
    });
  });
}

void ref_rnear_self(void* hp, const int32_t* qidx, int64_t m, double dmax, int64_t* offsets, int32_t* out,
                    int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    typedef pointkd::KdTree<T, D> Tree;
    const Tree* tree = (const Tree*)h->tree;
    std::vector<int64_t> cnt(m);
#pragma omp parallel for schedule(dynamic, 256) num_threads(threads_or_max(nthreads))
    for (int64_t i = 0; i < m; i++) {
      pointkd::Indices res;
      tree->RNearNeighborsSelf(res, qidx[i], (typename Tree::DistT)dmax);
      cnt[i] = (int64_t)res.size();
      if (out) std::copy(res.begin(), res.end(), out + offsets[i]);
    }
    if (!out) {
      offsets[0] = 0;
      for (int64_t i = 0; i < m; i++) offsets[i + 1] = offsets[i] + cnt[i];
    }
  });
}

// estimate_normals restated on the reference tree (estimate_normals.cpp:17-120)
// with the Jacobi eigensolve.  pts: n x 3 of dtype (0 = f32, 1 = f64);
// sub: optional query indices (m of them, already wrapped into [0, n));
// outputs sized like the reference (num_eigen 1 or 3).  Returns the build
// time in seconds through *build_s.
void ref_estimate_normals(const void* pts, int64_t n, int dtype, int k, float r, const int32_t* sub, int64_t m,
                          int num_eigen, void* evecs, void* evals, int32_t* sizes, int nthreads,
                          double* build_s) {
  auto run = [&](auto t) {
    typedef decltype(t) T;
    const T* P = (const T*)pts;
    std::vector<T> points(P, P + n * 3);
    pointkd::BuildParams params;
    params.num_proc = 1;
    double t0 = omp_get_wtime();
    pointkd::KdTree<T, 3> tree(points, params);
    if (build_s) *build_s = omp_get_wtime() - t0;
    const T d_max = (T)r;
    int64_t num = sub ? m : n;
    T* ev = (T*)evecs;
    T* ew = (T*)evals;
#pragma omp parallel for schedule(static, 1000) num_threads(threads_or_max(nthreads))
    for (int64_t i = 0; i < num; i++) {
      int64_t i_ = sub ? sub[i] : i;
      pointkd::Indices idx;
      const T* q = &points[i_ * 3];
      if (k == -1)
        tree.RNearNeighbors(idx, q, d_max);
      else
        tree.KNearestNeighbors(idx, q, k, d_max);
      size_t cnt = idx.size();
      // mean then centred X^T X / n, in T (estimate_normals.cpp:84-88)
      T mean[3] = {0, 0, 0};
      for (size_t j = 0; j < cnt; j++)
        for (int c = 0; c < 3; c++) mean[c] += points[idx[j] * 3 + c];
      for (int c = 0; c < 3; c++) mean[c] /= (T)cnt;
      T C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (size_t j = 0; j < cnt; j++) {
        T x[3];
        for (int c = 0; c < 3; c++) x[c] = points[idx[j] * 3 + c] - mean[c];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) C[a * 3 + b] += x[a] * x[b];
      }
      for (int a = 0; a < 9; a++) C[a] /= (T)cnt;
      T w[3], V[9];
      oracle::jacobi3<T>(C, w, V);
      if (ev) {
        if (num_eigen == 1) {
          for (int c = 0; c < 3; c++) ev[i * 3 + c] = V[c * 3 + 0];
        } else {
          for (int e = 0; e < 3; e++)
            for (int c = 0; c < 3; c++) ev[i * 9 + e * 3 + c] = V[c * 3 + e];
        }
      }
      if (ew) {
        if (num_eigen == 1)
          ew[i] = w[0];
        else
          for (int e = 0; e < 3; e++) ew[i * 3 + e] = w[e];
      }
      if (sizes) sizes[i] = (int32_t)cnt;
    }
  };
  if (dtype == oracle::F32)
    run(float());
  else
    run(double());
}

// The normal loop of ref_estimate_normals (estimate_normals.cpp:64-110) over
// an already built reference tree `hp` (float32/float64, dim 3) whose input
// array was `pts` (n x 3, original order): the resident-tree form, so that
// a timed run holds queries only.  sub: m query rows (original indices).
void ref_tree_normals(void* hp, const void* pts, const int32_t* sub, int64_t m, int k, float r, int num_eigen,
                      void* evecs, void* evals, int32_t* sizes, int nthreads) {
  Handle* h = (Handle*)hp;
  auto run = [&](auto t) {
    typedef decltype(t) T;
    const pointkd::KdTree<T, 3>& tree = *(const pointkd::KdTree<T, 3>*)h->tree;
    const T* P = (const T*)pts;
    const T d_max = (T)r;
    T* ev = (T*)evecs;
    T* ew = (T*)evals;
#pragma omp parallel for schedule(static, 1000) num_threads(threads_or_max(nthreads))
    for (int64_t i = 0; i < m; i++) {
      pointkd::Indices idx;
      const T* q = P + (int64_t)sub[i] * 3;
      if (k == -1)
        tree.RNearNeighbors(idx, q, d_max);
      else
        tree.KNearestNeighbors(idx, q, k, d_max);
      size_t cnt = idx.size();
      T mean[3] = {0, 0, 0};
      for (size_t j = 0; j < cnt; j++)
        for (int c = 0; c < 3; c++) mean[c] += P[(int64_t)idx[j] * 3 + c];
      for (int c = 0; c < 3; c++) mean[c] /= (T)cnt;
      T C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (size_t j = 0; j < cnt; j++) {
        T x[3];
        for (int c = 0; c < 3; c++) x[c] = P[(int64_t)idx[j] * 3 + c] - mean[c];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) C[a * 3 + b] += x[a] * x[b];
      }
      for (int a = 0; a < 9; a++) C[a] /= (T)cnt;
      T w[3], V[9];
      oracle::jacobi3<T>(C, w, V);
      if (ev) {
        if (num_eigen == 1) {
          for (int c = 0; c < 3; c++) ev[i * 3 + c] = V[c * 3 + 0];
        } else {
          for (int e = 0; e < 3; e++)
            for (int c = 0; c < 3; c++) ev[i * 9 + e * 3 + c] = V[c * 3 + e];
        }
      }
      if (ew) {
        if (num_eigen == 1)
          ew[i] = w[0];
        else
          for (int e = 0; e < 3; e++) ew[i * 3 + e] = w[e];
      }
      if (sizes) sizes[i] = (int32_t)cnt;
    }
  };
  if (h->dim != 3) return;
  if (h->dtype == oracle::F32)
    run(float());
  else if (h->dtype == oracle::F64)
    run(double());
}

int ref_max_threads() { return omp_get_max_threads(); }

}  // extern "C"

// Host entry points of the query kernels (kNN, r-near, normals).
#pragma once

#include "tree.cuh"

namespace pptkg {

// Which points a query batch asks about.
struct QuerySpec {
  // point queries: m rows of `dim` coordinates of qdtype (F32 or F64), device
  const void* pts = nullptr;
  int qdtype = F32;
  // index queries: original point indices (device), or all of [0, m) when null
  const int32_t* idx = nullptr;
  int64_t m = 0;
  // index queries exclude the query point itself (the reference's *Self forms)
  bool exclude_self = true;
};

constexpr int KNN_MAX_K = 64;

template <typename T, int D>
void knn_query(const TreeBase* t, const QuerySpec& qs, int k, double dmax, int32_t* d_idx, int32_t* d_cnt,
               cudaStream_t st);

// Writes per-query hit counts into d_off[0..m) and turns them into offsets
// (d_off has m + 1 entries); returns the total.
template <typename T, int D>
int64_t rnear_count(const TreeBase* t, const QuerySpec& qs, double dmax, int64_t* d_off, cudaStream_t st);

template <typename T, int D>
void rnear_fill(const TreeBase* t, const QuerySpec& qs, double dmax, const int64_t* d_off, int32_t* d_out,
                cudaStream_t st);

enum Precision { PREC_AUTO = 0, PREC_FP32 = 1, PREC_FP64 = 2 };

// PCA normals of the points with original indices qs.idx (or all n points)
// over their k nearest neighbours including themselves (k == -1: r-near
// neighbourhoods).  Outputs are indexed by query row; any may be null.
template <typename T>
void normals_query(const TreeBase* t, const QuerySpec& qs, int k, float r, int num_eigen, int precision,
                   double gap_thr, T* d_evecs, T* d_evals, int32_t* d_sizes, cudaStream_t st);

// Queries over every valid point of every cloud of a forest, each against
// its own cloud's tree; outputs are indexed by global input row (n rows).
template <typename T, int D>
void forest_knn(const TreeBase* t, int k, double dmax, bool exclude_self, int32_t* d_idx, int32_t* d_cnt,
                cudaStream_t st);
// With d_idx set, forest_normals also answers the self kNN (k, dmax = r,
// the point itself excluded) from the same walk: d_idx n x k, d_cnt n, as
// forest_knn writes them.
template <typename T>
void forest_normals(const TreeBase* t, int k, float r, int num_eigen, int precision, double gap_thr, T* d_evecs,
                    T* d_evals, int32_t* d_sizes, cudaStream_t st, int32_t* d_idx = nullptr,
                    int32_t* d_cnt = nullptr);

// Device-side slot map of a capture-ready forest (after each rebuild).
void forest_slot_map_device(TreeBase* t, cudaStream_t st);

// One launch over several single trees: tree g answers the query rows
// [rows[g], rows[g+1]) (host offsets) of a concatenated batch.
template <typename T, int D>
void multi_knn(const TreeBase* const* trees, int ntrees, const void* d_q, int qdtype, const int64_t* rows, int k,
               double dmax, int32_t* d_idx, int32_t* d_cnt, cudaStream_t st);
template <typename T>
void multi_normals(const TreeBase* const* trees, int ntrees, const int32_t* d_idx, const int64_t* rows, int k, float r,
                   int num_eigen, int precision, double gap_thr, T* d_evecs, T* d_evals, int32_t* d_sizes,
                   cudaStream_t st);

// pptkg_tree_normals_noalloc: the tree-normals path with its scratch in a
// static device array instead of allocated memory (device pointers only).
template <typename T>
void normals_noalloc(const TreeBase* t, const int32_t* d_idx, int64_t m, int k, float r, int num_eigen, int precision,
                     T* d_evecs, T* d_evals, int32_t* d_sizes, cudaStream_t st);

// Batched symmetric 3x3 eigensolve (row-major inputs).
template <typename T>
void eigh3_batched(const T* d_A, int64_t m, T* d_w, T* d_V, int layout, cudaStream_t st);


// Centred covariances of m neighbourhoods given as CSR lists (offsets m+1,
// `total` indices into the n x 3 points); C is m x 3 x 3 row-major (pca.cu).
template <typename T>
void nbhd_covariance(const T* d_pts, int64_t n, const int64_t* d_off, const int32_t* d_idx, int64_t total, int64_t m,
                     T* d_C, cudaStream_t st);

}  // namespace pptkg

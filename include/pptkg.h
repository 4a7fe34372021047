/*
 * pptkg.h -- C ABI of pptk_b200, the B200 implementation of pptk's k-d tree,
 * kNN / r-near queries and PCA normal estimation.
 *
 * Plain pointers and sizes only.  Every function returns PPTKG_OK (0) or a
 * PPTKG_E_* status; pptkg_last_error() returns the message of the last
 * failure on the calling thread.  Array arguments are host memory when
 * `mem` is PPTKG_MEM_HOST and device memory of the current device when it is
 * PPTKG_MEM_DEVICE; `stream` is a cudaStream_t (NULL: the default stream).
 * Calls return once their results are written.
 *
 * The reference interfaces that each entry point replaces are cited with
 * paths relative to the pptk source tree.
 */
#ifndef PPTKG_H_
#define PPTKG_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PPTKG_API __attribute__((visibility("default")))
#else
#define PPTKG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define PPTKG_OK 0
#define PPTKG_E_INVALID 1     /* bad argument value (Python: ValueError) */
#define PPTKG_E_TYPE 2        /* unsupported dtype or dim (TypeError) */
#define PPTKG_E_CUDA 3        /* CUDA runtime failure */
#define PPTKG_E_RANGE 4       /* index outside the point range (RuntimeError) */
#define PPTKG_E_DEVICE 5      /* a kernel's internal check failed */
#define PPTKG_E_UNSUPPORTED 6 /* not implemented (NotImplementedError) */

/* element types (numpy dtypes of the reference's dispatch,
 * pptk/kdtree/kdtree_wrapper.cpp:15-41) */
#define PPTKG_F32 0
#define PPTKG_F64 1
#define PPTKG_I8 2
#define PPTKG_I16 3
#define PPTKG_I32 4
#define PPTKG_I64 5
#define PPTKG_U8 6
#define PPTKG_U16 7
#define PPTKG_U32 8
#define PPTKG_U64 9

#define PPTKG_MEM_HOST 0
#define PPTKG_MEM_DEVICE 1

/* normal-estimation arithmetic */
#define PPTKG_PREC_AUTO 0 /* float32 input: FP32 path; float64 input: FP64 */
#define PPTKG_PREC_FP32 1 /* FP32 covariance (shifted, compensated) + FP32
                             eigensolve, FP64 re-solve of small eigen-gaps */
#define PPTKG_PREC_FP64 2

typedef struct pptkg_tree pptkg_tree;

/* Library version (major * 10000 + minor * 100 + patch). */
PPTKG_API int pptkg_version(void);

/* 1 for the diagnostic build compiled with PPTKG_BOUNDS_CHECK
 * (libpptkg_checked.so), 0 otherwise.  In that build every point-record,
 * index-map and traversal-node index the query kernels read is checked
 * against its array; a failed check records its site in a device word and
 * reads element 0 instead, and the call returns PPTKG_E_DEVICE ("bounds
 * check failed: ...").  Traversal stack depths are checked in every build. */
PPTKG_API int pptkg_bounds_checked(void);

/* Copies the last error message of this thread into buf (NUL-terminated,
 * truncated to len); returns the status of that error. */
PPTKG_API int pptkg_last_error(char* buf, size_t len);

/* Builds a k-d tree over n points of `dim` coordinates (contiguous rows).
 * Replaces pptk.kdtree._build: Build + BuildTreeAction
 * (pptk/kdtree/kdtree_wrapper.cpp:76-104, :281-304) and the KdTree
 * constructor (pptk/kdtree/src/kdtree-impl.h:773-833).  Rows holding a NaN or
 * inf coordinate are left out, as in the reference.  The tree owns a copy of
 * the points.  dtype: any PPTKG_* point type (float32, float64, int8 ...
 * uint64); dim: 2, 3 or 4.  Integer trees are built in their own type, as
 * the reference builds them, and answer queries in float, the reference's
 * distance type for integers (accumulator.h:16-19); pptkg_tree_info reports
 * the input type. */
PPTKG_API int pptkg_tree_build(const void* points, int64_t n, int dim, int dtype, int mem, int max_leaf_size,
                     double empty_split, void* stream, pptkg_tree** out);

/* Frees a tree.  Replaces DeleteKdTree (kdtree_wrapper.cpp:57-74). */
PPTKG_API int pptkg_tree_free(pptkg_tree* tree);

/* Sizes of a tree: input rows, valid rows (the reference's num_points(),
 * kdtree.h:224), dim, dtype, build records, traversal depth bound. */
PPTKG_API int pptkg_tree_info(const pptkg_tree* tree, int64_t* n, int64_t* n_valid, int* dim, int* dtype,
                    int64_t* n_records, int* depth);

/* Tree position -> original row (n_valid entries): the reference's
 * reverse_indices() (kdtree.h:226). */
PPTKG_API int pptkg_tree_reverse_indices(const pptkg_tree* tree, int32_t* out, int mem, void* stream);

/* The reference node list in preorder, 5 doubles per node (split dim, split
 * index, split value, has left child, has right child), empty-split nodes
 * included (pptk/kdtree/src/node.h:15-29).  *count receives the node count;
 * out may be NULL to query it. */
PPTKG_API int pptkg_tree_ref_nodes(const pptkg_tree* tree, double* out, int64_t capacity, int64_t* count);

/* Re-cuts the traversal hierarchy at `bucket` points per leaf bucket (a
 * tuning knob; results do not depend on it). */
PPTKG_API int pptkg_tree_set_bucket(pptkg_tree* tree, int bucket, void* stream);

/* k nearest neighbours of m point queries (rows of `dim` coordinates of
 * qdtype F32/F64) with distance < dmax.  out_idx: m x k original row indices
 * in ascending distance, ties in distance broken by ascending original
 * index, -1 padded; out_cnt (optional): neighbours found.  Replaces
 * QueryWithPoints with k > 0 (kdtree_wrapper.cpp:139-159) /
 * KdTree::KNearestNeighbors (kdtree-impl.h:873-929).  k >= 1 (above 64 the
 * lists live in device-memory heaps). */
PPTKG_API int pptkg_knn(const pptkg_tree* tree, const void* queries, int64_t m, int qdtype, int mem, int k, double dmax,
              int32_t* out_idx, int32_t* out_cnt, void* stream);

/* k nearest neighbours of stored points given by original row index
 * (indices NULL: rows 0..m-1), each point excluding itself.  Replaces
 * QueryWithIndices with k > 0 (kdtree_wrapper.cpp:117-137) /
 * KNearestNeighborsSelf (kdtree-impl.h:931-976).  A row dropped at build
 * time gets no neighbours. */
PPTKG_API int pptkg_knn_self(const pptkg_tree* tree, const int32_t* indices, int64_t m, int mem, int k, double dmax,
                   int32_t* out_idx, int32_t* out_cnt, void* stream);

/* r-near, first step: per-query counts of points with distance < dmax,
 * written as offsets (m + 1 entries, out_offsets[m] = total).  Queries are
 * points (queries != NULL) or stored rows (indices, or rows 0..m-1 when both
 * are NULL; the row itself excluded).  Replaces the counting half of
 * RNearNeighbors[Self] (kdtree-impl.h:978-1069). */
PPTKG_API int pptkg_rnear_count(const pptkg_tree* tree, const void* queries, const int32_t* indices, int64_t m, int qdtype,
                      int mem, double dmax, int64_t* out_offsets, int64_t* total, void* stream);

/* r-near, second step: the hits of each query in ascending tree position
 * (the reference's left-then-right order, kdtree-impl.h:519-558), as original
 * row indices at out_idx[offsets[i] .. offsets[i+1]). */
PPTKG_API int pptkg_rnear_fill(const pptkg_tree* tree, const void* queries, const int32_t* indices, int64_t m, int qdtype,
                     int mem, double dmax, const int64_t* offsets, int32_t* out_idx, void* stream);

/* PCA normals: builds a tree over n x 3 points and, for every point (or the
 * m rows in `subsample`), eigen-decomposes the covariance of its k nearest
 * neighbours including itself within distance r (k = -1: all points within
 * r).  Replaces estimate_normals (pptk/processing/estimate_normals/
 * estimate_normals.cpp:17-120, :259-345).  num_eigen 1: out_evecs m x 3 (the
 * normal), out_evals m; num_eigen 3: m x 3 x 3 ([i, j, :] = j-th eigenvector,
 * ascending eigenvalue) and m x 3.  Outputs may be NULL. */
PPTKG_API int pptkg_estimate_normals(const void* points, int64_t n, int dtype, int mem, int k, float r,
                           const int32_t* subsample, int64_t m, int num_eigen, int precision, void* out_evecs,
                           void* out_evals, int32_t* out_sizes, void* stream);

/* The same PCA over an existing 3-D tree (rows of the tree's input): the
 * rows `indices` (m of them), or every row when indices is NULL (m must then
 * be 0 or the tree's row count; the outputs hold one entry per row). */
PPTKG_API int pptkg_tree_normals(const pptkg_tree* tree, const int32_t* indices, int64_t m, int mem, int k, float r,
                       int num_eigen, int precision, void* out_evecs, void* out_evals, int32_t* out_sizes,
                       void* stream);

/* Allocation-free form of pptkg_tree_normals.  No counterpart in the
 * reference: it serves callers that cannot allocate device memory, such as
 * code running under another framework that has reserved the GPU's memory up
 * front, or latency-critical loops where a cudaMalloc (which can synchronize
 * the device) is not acceptable.  The caller passes device pointers for the
 * query rows (indices, or NULL for rows 0..m-1; m = 0 with NULL means all
 * rows) and for the outputs, as in pptkg_tree_normals with PPTKG_MEM_DEVICE.
 * A pointer that is not device (or managed) memory of the tree's device is
 * rejected with PPTKG_E_INVALID before anything reads it.
 * Limits: m <= PPTKG_NOALLOC_MAX_QUERIES (65536), 1 <= k <= 16; larger sizes
 * are rejected with PPTKG_E_INVALID.  The scratch (about 4.7 MB) is a static
 * device array held by every GPU that loads the library until the process
 * exits; the first call on a device looks up its address, so make that first
 * call before any stream capture.  The address is kept for the rest of the
 * process, like every device pointer the library holds: a cudaDeviceReset
 * invalidates it together with the trees.  Each call waits for its stream at
 * the end, to read the status word of the kernels' checks.  All calls share
 * that one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialized by the caller.  No memory is
 * allocated or freed. */
#define PPTKG_NOALLOC_MAX_QUERIES 65536
#define PPTKG_NOALLOC_MAX_K 16
PPTKG_API int pptkg_tree_normals_noalloc(const pptkg_tree* tree, const int32_t* indices, int64_t m, int k, float r,
                                         int num_eigen, int precision, void* out_evecs, void* out_evals,
                                         int32_t* out_sizes, void* stream);

/* Forests (ragged batches).  Builds one tree per cloud over the consecutive
 * row ranges [offsets[c], offsets[c+1]) of one point array (offsets: host,
 * ncloud + 1 entries, offsets[0] = 0, offsets[ncloud] = n), each tree exactly
 * the one pptkg_tree_build gives for that cloud alone; one build pass serves
 * all clouds.  The reference builds such batches one KdTree per cloud
 * (kdtree-impl.h:773-833).  The handle works with pptkg_tree_info,
 * pptkg_tree_reverse_indices (global positions) and pptkg_tree_set_bucket. */
PPTKG_API int pptkg_forest_build(const void* points, int64_t n, int dim, int dtype, int mem, const int64_t* offsets,
                                 int ncloud, int max_leaf_size, double empty_split, void* stream, pptkg_tree** out);

/* Number of clouds and (optionally, host, ncloud + 1) the first tree position
 * of each cloud's valid points. */
PPTKG_API int pptkg_forest_info(const pptkg_tree* forest, int* ncloud, int64_t* valid_offsets);

/* Reference node list of one cloud's tree (layout of pptkg_tree_ref_nodes). */
PPTKG_API int pptkg_forest_ref_nodes(const pptkg_tree* forest, int cloud, double* out, int64_t capacity,
                                     int64_t* count);

/* k nearest neighbours of every valid point among the points of its own
 * cloud (optionally excluding itself, as KNearestNeighborsSelf does).  Outputs
 * are indexed by global input row: out_idx n x k (global rows, -1 padded),
 * out_cnt n; rows of dropped points get no neighbours. */
PPTKG_API int pptkg_forest_knn(const pptkg_tree* forest, int k, double dmax, int exclude_self, int mem,
                               int32_t* out_idx, int32_t* out_cnt, void* stream);

/* PCA normals of every point over its cloud's k nearest neighbours (itself
 * included, within r), the estimate_normals computation for all clouds at
 * once; outputs indexed by global input row (layouts of pptkg_estimate_normals). */
PPTKG_API int pptkg_forest_normals(const pptkg_tree* forest, int k, float r, int num_eigen, int precision, int mem,
                                   void* out_evecs, void* out_evals, int32_t* out_sizes, void* stream);

/* Self kNN and PCA normals of every point in one walk (no reference
 * counterpart; the reference answers them with two calls): equal to
 * pptkg_forest_knn(k, dmax = r, exclude_self = 1) into out_idx / out_cnt
 * and pptkg_forest_normals(k, r, ...) into out_evecs / out_evals /
 * out_sizes.  out_cnt, out_evals and out_sizes may be NULL. */
PPTKG_API int pptkg_forest_knn_normals(const pptkg_tree* forest, int k, float r, int num_eigen, int precision,
                                       int mem, int32_t* out_idx, int32_t* out_cnt, void* out_evecs,
                                       void* out_evals, int32_t* out_sizes, void* stream);

/* Capture mode of a float32 / float64 forest (no reference counterpart; the
 * rebuild step of a CUDA graph over build and queries).
 * pptkg_forest_capture_ready sizes the forest's device arrays for new
 * coordinates of the same rows and fixes the rebuild's launch shapes, then
 * synchronises.  After it,
 * pptkg_forest_rebuild rebuilds every cloud's tree in place from new
 * coordinates of the same n rows (points: device, the layout of
 * pptkg_forest_build) with no host synchronisation while a status sink is
 * set, so that rebuild, pptkg_forest_knn and pptkg_forest_normals can be
 * captured together; the trees equal those pptkg_forest_build gives for the
 * new coordinates.  The capacities are the first build's tree levels + 8
 * and twice its records and traversal nodes; sink code 20 (more levels) or
 * 21 (more records), without a sink PPTKG_E_UNSUPPORTED, means the
 * coordinates need more than that: the trees of that pass are not the
 * reference trees and the forest must be built again.  Host-side reads
 * (pptkg_forest_info, pptkg_tree_info, ref nodes, save) synchronise the
 * device and take the last rebuild's counts. */
PPTKG_API int pptkg_forest_capture_ready(pptkg_tree* forest, void* stream);
PPTKG_API int pptkg_forest_rebuild(pptkg_tree* forest, const void* points, void* stream);

/* Multi-tree batches (no reference counterpart; the serving loop's batching
 * step).  One launch answers queries for several resident single trees:
 * tree g answers the concatenated query rows [row_offsets[g],
 * row_offsets[g+1]) (row_offsets: host, ntrees + 1 entries).  All trees
 * share dtype and dim.  Results are exactly those of pptkg_knn /
 * pptkg_tree_normals on each tree alone. */
PPTKG_API int pptkg_multi_knn(const pptkg_tree* const* trees, int ntrees, const void* queries,
                              const int64_t* row_offsets, int qdtype, int mem, int k, double dmax, int32_t* out_idx,
                              int32_t* out_cnt, void* stream);
PPTKG_API int pptkg_multi_normals(const pptkg_tree* const* trees, int ntrees, const int32_t* indices,
                                  const int64_t* row_offsets, int mem, int k, float r, int num_eigen, int precision,
                                  void* out_evecs, void* out_evals, int32_t* out_sizes, void* stream);

/* Batched symmetric 3x3 eigensolve of m row-major matrices of dtype F32/F64:
 * w m x 3 ascending; V m x 3 x 3 with layout 0: V[i, :, j] = j-th
 * eigenvector (vfuncs._eigh, pptk/vfuncs/vfuncs.cpp:1241-1293), layout 1:
 * V[i, j, :] = j-th eigenvector (estimate_normals.cpp:96-99). */
PPTKG_API int pptkg_eigh3(const void* A, int64_t m, int dtype, int mem, void* w, void* V, int layout, void* stream);

/* Covariances of neighbourhood lists (replaces the per-neighbourhood
 * vfuncs chain MEAN / DOT(TRANSPOSE(Y), Y) that pptk's expression layer
 * evaluates, pptk/points/expr.py:27-72, vfuncs/vfuncs.cpp `_mean`, `_dot`,
 * `_transpose`): for neighbourhood i, the rows indices[offsets[i] ..
 * offsets[i+1]) of the n x 3 points (F32/F64); out_cov (m x 3 x 3,
 * row-major) = Y^T Y / count with Y the rows minus their mean.  Feed it to
 * pptkg_eigh3 for the `_eigh` step.  An index outside [0, n) is
 * PPTKG_E_RANGE. */
PPTKG_API int pptkg_nbhd_covariance(const void* points, int64_t n, int dtype, int mem, const int64_t* offsets,
                                   const int32_t* indices, int64_t m, void* out_cov, void* stream);

/* Tree persistence (no reference counterpart: the reference keeps trees in
 * process memory only).  pptkg_tree_save writes a tree or forest to one
 * self-describing host buffer (header, the device arrays, a checksum);
 * with buf NULL it only reports the size.  pptkg_tree_load puts such a
 * buffer back on the current device without a rebuild; the header, sizes,
 * checksum and records are checked on the host and every node reference,
 * point id and index-map entry on the device, so a damaged buffer is
 * PPTKG_E_INVALID. */
PPTKG_API int pptkg_tree_save(const pptkg_tree* tree, void* buf, int64_t capacity, int64_t* size);
PPTKG_API int pptkg_tree_load(const void* buf, int64_t size, void* stream, pptkg_tree** out);

/* Instrumentation (no reference counterpart).  Stage timing records CUDA
 * events on the launching stream around each stage ("build", "order",
 * "knn", "normals", "rnear_count", "rnear_fill", "h2d", "d2h");
 * enabling or disabling resets the totals. */
PPTKG_API int pptkg_profile_enable(int on);
PPTKG_API int pptkg_profile_get(const char* stage, double* total_ms, int64_t* count);
/* Kernels launched by this library since it was loaded. */
PPTKG_API int64_t pptkg_launch_count(void);

/* Run-time tuning (no reference counterpart; set by the autotuner,
 * pptk_b200/autotune.py).  Settings are process-wide and read at launch.
 *   "lane_span": a kNN / normals warp whose 32 queries span more than this
 *     many tree positions walks the tree per lane rather than as one packet
 *     (-1: always packets).  Default 1024 (with warm-started lists, packets
 *     won down to about one query per ten tree points: 2M random queries on
 *     a 20M-point scene took 6.3 ms as packets, 10.6-12.0 ms with 256).
 *   "rnear_warp_queries": pptkg_rnear_count / pptkg_rnear_fill calls, and
 *     normals over r-near neighbourhoods (k = -1), with at most this many
 *     queries give each query a whole warp (the lanes split every bucket)
 *     instead of packing 32 queries into a warp (0: never).
 *     Default 262144 (below it, 32-query packets leave B200's 148 SMs short
 *     of warps).  Hit lists and neighbourhood sizes do not depend on it;
 *     normals agree to FP64 rounding (their sums add in another order).
 *   "warm_bound": kNN / normals lists start from the k tree positions
 *     around each query's anchor; with 1 their bound is also lowered to the
 *     k-th distance over a wider window of tree-order neighbours (fewer
 *     list insertions), with 0 not.  Default 1.  Results do not depend on
 *     it.
 *   "warm_mult": float lists whose k equals their capacity (4, 8, 16, 32)
 *     start from the k nearest of warm_mult x k tree-order neighbours of the
 *     query's anchor (1 to 8; 1 gives the k-position start).  Default 2.
 *     Results do not depend on it.
 *   "topk_min": the k-tiling of the register top-k lists: 0 (default) uses
 *     the smallest capacity of 4, 8, 16, 32, 64 that holds k; 4 ... 64 use at
 *     least that capacity.  Results do not depend on it.
 * Unknown names or out-of-range values: PPTKG_E_INVALID. */
PPTKG_API int pptkg_tune_set(const char* name, int64_t value);
PPTKG_API int pptkg_tune_get(const char* name, int64_t* value);

/* Status sink of the calling host thread (no reference counterpart; for
 * capturing forest queries into a CUDA graph).  While d_word (a device int,
 * or NULL to clear) is set, pptkg_forest_knn / pptkg_forest_normals /
 * pptkg_forest_knn_normals / pptkg_forest_rebuild with device buffers
 * record kernel check failures by writing a non-zero code
 * into *d_word and neither synchronise nor read it back; the caller zeroes
 * the word and checks it after the work (or a graph replay) completes.  A
 * forest's first query sets up device tables and must run without a sink. */
PPTKG_API int pptkg_set_status_sink(int* d_word);

#ifdef __cplusplus
}
#endif

#endif /* PPTKG_H_ */

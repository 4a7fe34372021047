// Query kernels: exact kNN (point and self forms), r-near count/fill in the
// reference's order, and fused kNN + PCA normal estimation.
#include <algorithm>
#include <memory>
#include <mutex>
#include <string>

#include "knn.cuh"
#include "normals.cuh"
#include "profile.cuh"
#include "query.cuh"
#include "util.cuh"

namespace pptkg {

constexpr int QWARPS = 4;
constexpr int QTHREADS = QWARPS * 32;

template <typename T, int D>
TreeView<T, D> view_of(const TreeBase* t) {
  TreeView<T, D> v;
  v.pts = (const PointRec<T, D>*)t->pts;
  v.nodes = (const TNode<T, D>*)t->tnodes;
  v.nv = (int)t->nv;
  v.depth = t->tdepth;
  v.n_nodes = t->n_tnodes;
  v.root = t->root_tnode_h.empty() ? 0 : t->root_tnode_h[0];
  v.fwd = t->fwd;
  v.n_in = (int)t->n;
  v.pts_cap = (int)(t->capture ? t->n : t->nv);
  v.err = bounds_word(t->device);
  return v;
}

// Per-warp shared memory: the staging buffer (a leaf chunk in r-near walks,
// the warp's queries in kNN walks), traversal stack, the 32 x 33 distance
// matrix and the 32 candidate ids of the kNN bucket scan, and (normals)
// `logcap` list slots per lane.
template <typename T, int D>
__host__ __device__ constexpr size_t stage_bytes() {
  typedef typename DistOf<T>::type DistT;
  return 32 * (sizeof(PointRec<T, D>) > sizeof(QStage<DistT, D>) ? sizeof(PointRec<T, D>) : sizeof(QStage<DistT, D>));
}

template <typename T, int D>
__host__ __device__ __forceinline__ size_t warp_smem_bytes(int depth, int logcap = 0) {
  typedef typename DistOf<T>::type DistT;
  return stage_bytes<T, D>() + (((size_t)depth * sizeof(StackEnt<T, D>) + 15) & ~(size_t)15) +
         ((32 * 33 * sizeof(DistT) + 15) & ~(size_t)15) + 32 * 4 + (size_t)logcap * 32 * 4;
}

template <typename T, int D>
__device__ __forceinline__ WarpScratch<T, D> warp_scratch(int depth, int logcap = 0) {
  typedef typename DistOf<T>::type DistT;
  extern __shared__ __align__(16) unsigned char qsm[];
  const size_t per = warp_smem_bytes<T, D>(depth, logcap);
  unsigned char* base = qsm + (threadIdx.x >> 5) * per;
  WarpScratch<T, D> ws;
  ws.buf = (PointRec<T, D>*)base;
  base += stage_bytes<T, D>();
  ws.stack = (int*)base;
  base += ((size_t)depth * sizeof(StackEnt<T, D>) + 15) & ~(size_t)15;
  ws.dmat = (DistT*)base;
  base += (32 * 33 * sizeof(DistT) + 15) & ~(size_t)15;
  ws.cid = (int*)base;
  base += 32 * 4;
  ws.log = logcap ? (int*)base : nullptr;
  return ws;
}

// Candidate-log capacity per lane of the normals kernel.
__host__ __device__ constexpr int normals_logcap(int kmax) { return 2 * kmax; }

// ------------------------------------------------------------- loaders ----
// Query i is row i of a user array.
// `anc` (optional): per query row, a tree position near the query (the start
// of the leaf the query falls in), used to seed the search radius.
template <typename Q, int D>
struct PointQueries {
  const Q* q;
  const int* anc = nullptr;
  template <typename T, typename DistT>
  __device__ __forceinline__ bool load(int i, const TreeView<T, D>& tv, DistT* out, int& own,
                                       int* anchor = nullptr) const {
#pragma unroll
    for (int d = 0; d < D; d++) out[d] = (DistT)q[(int64_t)i * D + d];
    own = -1;
    if (anchor) *anchor = anc ? anc[i] : -1;
    return true;
  }
};

// Query i is the stored point with original index idx[i] (or i); EXCL drops
// the point itself from its own result (KNearestNeighborsSelf,
// kdtree-impl.h:931-948; RNearNeighborsSelf, :1028-1043).
//
// `bad` (optional): indices are checked against the tree's rows on the
// device; an index outside [0, n) sets *bad = 4 and leaves the query empty.
template <int D, bool EXCL>
struct IndexQueries {
  const int* idx;
  const int* fwd;
  int* bad = nullptr;
  template <typename T, typename DistT>
  __device__ __forceinline__ bool load(int i, const TreeView<T, D>& tv, DistT* out, int& own,
                                       int* anchor = nullptr) const {
    const int o = idx ? idx[i] : i;
    own = -1;
    if (anchor) *anchor = -1;
    if (bad && (o < 0 || o >= tv.n_in)) {
      atomicExch(bad, 4);
      return false;
    }
    const int p = tv.pos_of(fwd ? fwd : tv.fwd, o);
    if (anchor) *anchor = p;
    if (p < 0) return false;  // the point was dropped (NaN/inf): no neighbours
    const PointRec<T, D> r = tv.pt(p);
#pragma unroll
    for (int d = 0; d < D; d++) out[d] = (DistT)r.c[d];
    own = EXCL ? p : -1;
    return true;
  }
};

// Loaders whose query point is excluded from its own list (self kNN); with
// one, k_normals runs its fused form (kNN outputs + the point put back).
template <typename L>
struct ExcludesSelf : std::false_type {};
template <int D>
struct ExcludesSelf<IndexQueries<D, true>> : std::true_type {};

// Forest queries: every valid point of every cloud, in tree order, each
// cloud's range padded to whole warps so that a warp never mixes trees.
//
// Multi-tree batches (`views` set): group g is a separate tree with its own
// TreeView; its query rows [row_off[g], row_off[g+1]) take the slots from
// slot_off[g], rounded up to whole warps.
struct SlotMap {
  const int* warp_cloud;     // group (cloud or tree) of each warp; null: plain mode
  const int64_t* slot_off;   // first slot of each group
  const int64_t* valid_off;  // forest: first tree position of each cloud
  const int* root_tnode;     // forest: traversal root of each cloud
  const void* views;         // multi-tree: TreeView<T, D> per group
  const int64_t* row_off;    // multi-tree: first query row per group
  const int* order;          // multi-tree: query row of each batch position (null: identity)
};

// Resolves the query of a slot: its output row (-1: padding) and the warp's
// tree (root, or the whole view in multi-tree mode).
template <typename T, int D>
__device__ __forceinline__ int forest_query(int slot, const SlotMap& fm, TreeView<T, D>& tv) {
  const int c = fm.warp_cloud[slot >> 5];
  if (fm.views) {
    tv = static_cast<const TreeView<T, D>*>(fm.views)[c];
    const int64_t row = fm.row_off[c] + (slot - fm.slot_off[c]);
    if (row >= fm.row_off[c + 1]) return -1;
    return fm.order ? fm.order[row] : (int)row;
  }
  tv.root = fm.root_tnode[c];
  const int64_t p = fm.valid_off[c] + (slot - fm.slot_off[c]);
  return p < fm.valid_off[c + 1] ? tv.pt(p).id : -1;
}

// Per-lane stack capacity of the per-lane walk (trees deeper than this use
// packet walks only).
constexpr int LANE_STACK = 64;

// Upper bound on the k-th smallest squared distance from q to the points of
// the tree positions [lo, hi) other than `own`: for a window of w consecutive
// positions containing `anchor` (w = k, plus one when `own` is excluded and
// then skipped), the largest distance from q to its points is such a bound;
// the smallest over three windows is returned.  Infinity when the range
// holds fewer than w points.  Distances use the same arithmetic as the
// search, so the bound is attained exactly by a real candidate.
template <typename T, int D, typename DistT>
__device__ __forceinline__ DistT seed_bound(const TreeView<T, D>& tv, const DistT* q, int anchor, int k, int own,
                                            int lo, int hi) {
  // three windows of w positions: ending at, centred on and starting at the
  // anchor (clamped to [lo, hi)); each gives a bound, the smallest is kept
  const int w = k + (own >= 0 ? 1 : 0);
  if (hi - lo < w || anchor < 0) return (DistT)INFINITY;
  const int a = min(max(anchor, lo), hi - 1);
  const int b0 = min(max(a - w + 1, lo), hi - w);
  const int b1 = min(max(a - w / 2, lo), hi - w);
  const int b2 = min(max(a, lo), hi - w);
  DistT m0 = (DistT)0, m1 = (DistT)0, m2 = (DistT)0;
  for (int p = b0; p < b2 + w; p++) {
    if (p == own) continue;
    const DistT d2 = point_dist2<T, DistT, D>(tv.pt(p).c, q);
    if (p < b0 + w) m0 = d2 > m0 ? d2 : m0;
    if (p >= b1 && p < b1 + w) m1 = d2 > m1 ? d2 : m1;
    if (p >= b2) m2 = d2 > m2 ? d2 : m2;
  }
  const DistT m01 = m0 < m1 ? m0 : m1;
  return m01 < m2 ? m01 : m2;
}

// Tighter seed for float distances and k <= 16: the k-th smallest distance
// from q to the 32 positions of [lo, hi) around `anchor` (`own` excluded),
// sorted in registers by a bitonic network.  The window holds every window
// of seed_bound, so this bound is never looser.  Infinity when fewer than k
// candidates exist.
template <typename T, int D>
__device__ __forceinline__ float seed_bound32(const TreeView<T, D>& tv, const float* q, int anchor, int k, int own,
                                             int lo, int hi) {
  if (hi - lo < k + (own >= 0 ? 1 : 0) || anchor < 0) return INFINITY;
  const int a = min(max(anchor, lo), hi - 1);
  const int b = max(min(a - 16, hi - 32), lo);
  float v[32];
#pragma unroll
  for (int j = 0; j < 32; j++) {
    const int p = b + j;
    v[j] = (p < hi && p != own) ? point_dist2<T, float, D>(tv.pt(p).c, q) : INFINITY;
  }
#pragma unroll
  for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
    for (int stride = size / 2; stride > 0; stride >>= 1)
#pragma unroll
      for (int i = 0; i < 32; i++) {
        const int j = i ^ stride;
        if (j > i) {
          const float x = v[i], y = v[j];
          const float mn = fminf(x, y), mx = fmaxf(x, y);
          if ((i & size) == 0) {
            v[i] = mn;
            v[j] = mx;
          } else {
            v[i] = mx;
            v[j] = mn;
          }
        }
      }
  float r = INFINITY;
#pragma unroll
  for (int j = 0; j < 32; j++)
    if (j == k - 1) r = v[j];
  return r;
}

// Warm start of a query's top-k list from its neighbourhood in tree order:
// the list is filled with the candidates at the w tree positions around the
// query's anchor (w = k, plus one for a self query, whose own position is
// dropped), sorted, and those positions [wlo, wlo + wn) are skipped by the
// walk, so every candidate is still offered exactly once.  The list's bound
// starts at a real k-th distance instead of the radius, which keeps a warp
// of far-apart queries from visiting most of the tree and means that most
// candidates the walk meets are rejected without an insertion.
//
// Slot j of the window gets: a real key (distance < r2), an empty key (no
// candidate: outside the tree, or beyond r2), or a dead key (j >= w, or the
// own position when w = k + 1) -- exactly k live (real or empty) keys, which
// the descending sort moves to the k live slots of the list.
//
// With g_tune_warm_bound, the bound is then lowered to seed_bound32 /
// seed_bound over a wider window (live keys above it become seed keys);
// candidates of the wider window outside [wlo, wlo + wn) are offered by the
// walk as any other.
//
// Float lists with k equal to their capacity (k = 4, 8, 16, 32) start from
// a window of warm_mult x k positions instead (g_tune_warm_mult >= 2): the
// list then holds the k nearest of those tree-order neighbours, all of them
// real candidates.
template <typename T, int D, typename DistT, typename Top>
__device__ __forceinline__ void warm_topk(Top& top, const TreeView<T, D>& tv, const SlotMap& fm, int slot,
                                          const DistT* q, int anchor, int k, int own, DistT r2, bool bound,
                                          int warm_mult, int& wlo, int& wn) {
  constexpr int CAP = Top::CAP;
  wlo = 0;
  wn = 0;
  if (anchor < 0) return;
  int lo = 0, hi = tv.nv;
  if (fm.warp_cloud && !fm.views) {
    const int c = fm.warp_cloud[slot >> 5];
    lo = (int)fm.valid_off[c];
    hi = (int)fm.valid_off[c + 1];
  }
  if (hi <= lo) return;
  if constexpr (std::is_same<DistT, float>::value && CAP <= 32) {
    if (k == CAP && warm_mult >= 2) {
      // a window of warm_mult x k positions: its first k keys fill the
      // list, the rest are sorted apart in blocks of Q and merged in, so the
      // list holds the k nearest of the window's tree-order neighbours (all
      // real unless the window is short) and its bound is their k-th distance
      constexpr int Q = CAP < 16 ? CAP : 16;
      const int W = warm_mult * CAP;
      const int a2 = min(max(anchor, lo), hi - 1);
      const int start = hi - lo >= W ? min(max(a2 - W / 2, lo), hi - W) : lo;
      auto key_at = [&](int p) {
        unsigned long long key = top.key_empty();
        if (p < hi && p != own) {
          const PointRec<T, D> r = tv.pt(p);
          const DistT d2 = point_dist2<T, DistT, D>(r.c, q);
          if (d2 < r2) key = top.key_real(d2, r.id);
        }
        return key;
      };
#pragma unroll
      for (int j = 0; j < CAP; j++) top.s[j] = key_at(start + j);
      top.sort_desc();
      for (int off = CAP; off < W; off += Q) {
        unsigned long long t[Q];
#pragma unroll
        for (int j = 0; j < Q; j++) t[j] = key_at(start + off + j);
        bitonic_sort<Q>(t, false);
        top.merge_smallest(t);
      }
      wlo = start;
      wn = min(W, hi - start);
      // a window narrower than seed_bound32's 32 positions: its bound may
      // be tighter
      if (bound && k <= 16 && W < 32) top.seed(k, seed_bound32<T, D>(tv, q, anchor, k, own, lo, hi), r2);
      return;
    }
  }
  const int w = min(k + (own >= 0 ? 1 : 0), CAP);
  const int a = min(max(anchor, lo), hi - 1);
  const int start = hi - lo >= w ? min(max(a - w / 2, lo), hi - w) : lo;
#pragma unroll
  for (int j = 0; j < CAP; j++) {
    const int p = start + j;
    if (j >= w) {
      top.set_dead(j);
    } else if (p >= hi) {
      top.set_empty(j);
    } else if (p == own) {
      if (w == k + 1)
        top.set_dead(j);
      else
        top.set_empty(j);
    } else {
      const PointRec<T, D> r = tv.pt(p);
      const DistT d2 = point_dist2<T, DistT, D>(r.c, q);
      if (d2 < r2)
        top.set_real(j, d2, r.id);
      else
        top.set_empty(j);
    }
  }
  top.sort_desc();
  wlo = start;
  wn = min(w, hi - start);
  if (bound) {
    DistT b;
    if constexpr (std::is_same<DistT, float>::value)
      b = k <= 16 ? seed_bound32<T, D>(tv, q, anchor, k, own, lo, hi)
                  : seed_bound<T, D, DistT>(tv, q, anchor, k, own, lo, hi);
    else
      b = seed_bound<T, D, DistT>(tv, q, anchor, k, own, lo, hi);
    top.seed(k, b, r2);
  }
}

// order_mode 0: slot = query; 1: order[slot]; 2: tree order (query = the
// original index stored at tree position slot).
template <typename T, int D>
__device__ __forceinline__ int query_of(int slot, const int* order, int order_mode, const TreeView<T, D>& tv) {
  return order_mode == 0 ? slot : (order_mode == 1 ? order[slot] : tv.pt(slot).id);
}

// ----------------------------------------------------------- ordering ----
template <typename T, int D, typename Q>
__global__ void k_locate(TreeView<T, D> tv, const Q* q, int m, int* key) {
  typedef typename DistOf<T>::type DistT;
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  DistT p[D];
#pragma unroll
  for (int d = 0; d < D; d++) p[d] = (DistT)q[(int64_t)i * D + d];
  int cur = tv.root, k = 0;
  for (int step = 0; step <= tv.depth + 1; step++) {
    const TNode<T, D> nd = load_node(tv.nodes, tv.node_index(cur));
    int c;
    if (nd.cnt[1] == 0)
      c = 0;
    else if (nd.cnt[0] == 0)
      c = 1;
    else
      c = box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], p) < box_min_dist2<T, DistT, D>(nd.lo[0], nd.hi[0], p);
    const int ref = nd.ref[c];
    if (ref < 0) {
      k = -ref - 1 + nd.cnt[c] / 2;  // the middle of the leaf bucket
      break;
    }
    cur = ref;
  }
  key[i] = min(max(k, 0), tv.nv);
}

static __global__ void k_check_idx(const int* idx, int m, int n, int* status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m && (idx[i] < 0 || idx[i] >= n)) atomicExch(status, 4);
}

// Rejects index queries outside [0, n) before any kernel dereferences them.
static void check_indices(const TreeBase* t, const QuerySpec& qs, cudaStream_t st) {
  if (qs.pts || !qs.idx || qs.m <= 0) return;
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  k_check_idx<<<div_up(qs.m, 256), 256, 0, st>>>(qs.idx, (int)qs.m, (int)t->n, status.get());
  PPTKG_CHECK_LAUNCH();
  int h = 0;
  PPTKG_CUDA(cudaMemcpyAsync(&h, status.get(), sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (h) throw Error(E_RANGE, "query index outside of [0, n)");
}

// Tree position of each index query (nv for dropped points and, when the
// indices are unchecked, for indices outside [0, n)).
static __global__ void k_idxkey(const int* idx, const int* fwd, int m, int n, int nv, int* key) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int o = idx ? idx[i] : i;
  const int p = o >= 0 && o < n ? fwd[o] : -1;
  key[i] = p < 0 ? nv : p;
}

// Counting sort on key >> shift: queries of the same run of 2^shift tree
// positions share a bin (their relative order within it is immaterial).
// The shift grows as the queries thin out, keeping bins about as many as
// queries.
static int order_shift(int nv, int m) {
  int s = 0;
  while (s < 20 && ((int64_t)m << (s + 1)) <= (int64_t)nv) s++;
  return s;
}

static __global__ void k_hist(const int* key, int m, int shift, int* hist) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) atomicAdd(&hist[key[i] >> shift], 1);
}

static __global__ void k_place(const int* key, int m, int shift, int* cursor, int* order) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) order[atomicAdd(&cursor[key[i] >> shift], 1)] = i;
}

// Builds a processing order in which queries near each other in the tree are
// adjacent (counting sort on the tree position key).  Returns the order mode.
//
// For point queries `anchors` (m ints, optional) receives each query's leaf
// start position (the seed anchor of the search), for every m.
template <typename T, int D>
int make_order(const TreeBase* t, const QuerySpec& qs, DevBuf<int>& order, cudaStream_t st, bool checked = false,
               int* anchors = nullptr) {
  if (!checked) check_indices(t, qs, st);
  Stage stage("order", st);
  const int m = (int)qs.m;
  const int nv = (int)t->nv;
  if (m <= 0) return 0;
  if (!qs.pts && !qs.idx && m == nv && t->n == t->nv) return 2;  // all points, tree order
  const bool locate = qs.pts && (anchors || m >= 2048);
  DevBuf<int> keybuf((locate && anchors) || (!locate && m < 2048) ? 0 : m, st);
  int* key = locate && anchors ? anchors : keybuf.get();
  if (locate) {
    if (qs.qdtype == F64)
      k_locate<T, D, double><<<div_up(m, 256), 256, 0, st>>>(view_of<T, D>(t), (const double*)qs.pts, m, key);
    else
      k_locate<T, D, float><<<div_up(m, 256), 256, 0, st>>>(view_of<T, D>(t), (const float*)qs.pts, m, key);
    PPTKG_CHECK_LAUNCH();
  }
  if (m < 2048) return 0;
  const int shift = order_shift(nv, m);
  const int bins = (nv >> shift) + 1;
  DevBuf<int> hist(bins + 1, st);
  if (!qs.pts) {
    k_idxkey<<<div_up(m, 256), 256, 0, st>>>(qs.idx, t->fwd, m, (int)t->n, nv, key);
    PPTKG_CHECK_LAUNCH();
  }
  PPTKG_CUDA(cudaMemsetAsync(hist.get(), 0, sizeof(int) * (bins + 1), st));
  k_hist<<<div_up(m, 256), 256, 0, st>>>(key, m, shift, hist.get());
  PPTKG_CHECK_LAUNCH();
  exclusive_scan<int, int>(hist.get(), hist.get(), bins, (int*)nullptr, st);
  order.alloc(m, st);
  k_place<<<div_up(m, 256), 256, 0, st>>>(key, m, shift, hist.get(), order.get());
  PPTKG_CHECK_LAUNCH();
  return 1;
}

// ----------------------------------------------------------------- kNN ----
// Blocks per SM the kNN kernel is compiled for: float top-k lists of up to
// 16 entries fit 96 registers (5 blocks of 128 threads); larger lists keep
// the compiler's register count.
constexpr int knn_min_blocks(int kmax, int dist_bytes) { return (dist_bytes == 4 && kmax <= 16) ? 5 : (dist_bytes == 4 && kmax <= 32) ? 4 : 1; }

template <typename T, int D, int KMAX, typename L>
__global__ void __launch_bounds__(QTHREADS, knn_min_blocks(KMAX, sizeof(typename DistOf<T>::type))) k_knn(TreeView<T, D> tv, L ld, const int* order, int order_mode, int m,
                                                  int k, typename DistOf<T>::type r2, int32_t* out_idx,
                                                  int32_t* out_cnt, int* status, SlotMap fm, int lane_span,
                                                  bool warm_bound, int warm_mult) {
  typedef typename DistOf<T>::type DistT;
  const int slot = blockIdx.x * QTHREADS + threadIdx.x;
  if ((slot & ~31) >= m) return;
  WarpScratch<T, D> ws = warp_scratch<T, D>(tv.depth);
  int qid = -1, own = -1, anchor = -1;
  DistT q[D];
  bool active = false;
  if (fm.warp_cloud) {
    qid = forest_query(slot, fm, tv);
    if (qid >= 0) active = ld.load(qid, tv, q, own, &anchor);
  } else if (slot < m) {
    qid = query_of(slot, order, order_mode, tv);
    active = ld.load(qid, tv, q, own, &anchor);
  }
  if (!active)
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = (DistT)0;
  TopK<KMAX, DistT> top;
  top.reset(k, r2);
  int wlo = 0, wn = 0;
  if (active) warm_topk<T, D, DistT>(top, tv, fm, slot, q, anchor, k, own, r2, warm_bound, warm_mult, wlo, wn);
  const bool ok = use_lane_walk<LANE_STACK>(anchor, active, lane_span, tv.depth)
                      ? lane_knn<LANE_STACK, T, D>(tv, q, own, active, r2, top, wlo, wn)
                      : packet_knn<T, D>(tv, q, own, active, r2, top, ws, wlo, wn);
  if (!ok) atomicExch(status, 1);
  if (qid >= 0) {
    int c = 0;
#pragma unroll
    for (int j = 0; j < KMAX; j++) {
      if (j < k) {
        const bool v = active && top.valid(j);
        c += v;
        out_idx[(int64_t)qid * k + (k - 1 - j)] = v ? top.id(j) : -1;
      }
    }
    if (out_cnt) out_cnt[qid] = c;
  }
}

template <typename T, int D, int KMAX, typename L>
void launch_knn(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                int32_t* d_idx, int32_t* d_cnt, int* status, cudaStream_t st, SlotMap fm) {
  if (m <= 0) return;
  const size_t smem = QWARPS * warp_smem_bytes<T, D>(t->tdepth);
  if (smem > 48 * 1024)
    PPTKG_CUDA(cudaFuncSetAttribute(k_knn<T, D, KMAX, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_knn<T, D, KMAX, L><<<div_up(m, QTHREADS), QTHREADS, smem, st>>>(view_of<T, D>(t), ld, order, mode, m, k, r2,
                                                                      d_idx, d_cnt, status, fm,
                                                                      g_tune_lane_span.load(),
                                                                      g_tune_warm_bound.load() != 0,
                                                                      g_tune_warm_mult.load());
  PPTKG_CHECK_LAUNCH();
}

template <typename T, int D, typename L>
void dispatch_knn(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                  int32_t* d_idx, int32_t* d_cnt, int* status, cudaStream_t st, SlotMap fm = SlotMap{}) {
  const int kc = std::max(k, g_tune_topk_min.load());
  if (kc <= 4)
    launch_knn<T, D, 4>(t, ld, order, mode, m, k, r2, d_idx, d_cnt, status, st, fm);
  else if (kc <= 8)
    launch_knn<T, D, 8>(t, ld, order, mode, m, k, r2, d_idx, d_cnt, status, st, fm);
  else if (kc <= 16)
    launch_knn<T, D, 16>(t, ld, order, mode, m, k, r2, d_idx, d_cnt, status, st, fm);
  else if (kc <= 32)
    launch_knn<T, D, 32>(t, ld, order, mode, m, k, r2, d_idx, d_cnt, status, st, fm);
  else
    launch_knn<T, D, 64>(t, ld, order, mode, m, k, r2, d_idx, d_cnt, status, st, fm);
}

template <typename DistT>
DistT radius2(double dmax) {
  // the reference casts dmax to the distance type and squares it there
  // (kdtree_wrapper.cpp:144-146, kdtree-impl.h:881)
  const DistT r = (DistT)dmax;
  return r * r;
}

static void check_status(int* d_status, cudaStream_t st, const char* what) {
  int h = 0;
  PPTKG_CUDA(cudaMemcpyAsync(&h, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (h == 4) throw Error(E_RANGE, std::string(what) + ": query index outside of its tree's [0, n)");
  if (h) throw Error(E_DEVICE, std::string(what) + ": device traversal check failed (code " + std::to_string(h) + ")");
}

// The status word of one query call: the thread's status sink when one is
// set (nothing is read back), else a fresh zeroed word checked at the end.
struct StatusWord {
  DevBuf<int> own;
  int* p = nullptr;
  explicit StatusWord(cudaStream_t st) {
    if (g_status_sink) {
      p = g_status_sink;
    } else {
      own.alloc(1, st);
      PPTKG_CUDA(cudaMemsetAsync(own.get(), 0, sizeof(int), st));
      p = own.get();
    }
  }
  int* get() const { return p; }
  void check(cudaStream_t st, const char* what) {
    if (!g_status_sink) check_status(p, st, what);
  }
};


// kNN for k above the register lists' capacity: one thread per query, the
// per-lane walk with its top-k in a device-memory heap (HeapTop), then a heap
// sort into ascending order.  Queries run in chunks of `m` slots starting
// at slot `m0` of the processing order; hd / hp hold one heap per slot.
constexpr int BIG_STACK = 128;

// POS: write tree positions (through the tree's index map) to chunk rows
// (for the normal pass) instead of original indices to query rows.
template <typename T, int D, typename L, bool POS>
__global__ void k_knn_big(TreeView<T, D> tv, L ld, const int* order, int order_mode, int m0, int m, int k,
                          typename DistOf<T>::type r2, typename DistOf<T>::type* hd, int* hp, int32_t* out_idx,
                          int32_t* out_cnt, int* status) {
  typedef typename DistOf<T>::type DistT;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int qid = query_of(m0 + i, order, order_mode, tv);
  int own = -1;
  DistT q[D];
  const bool active = ld.load(qid, tv, q, own);
  HeapTop<DistT> top{hd + (int64_t)i * k, hp + (int64_t)i * k, k, 0, r2};
  if (active && !lane_knn<BIG_STACK, T, D>(tv, q, own, true, r2, top)) atomicExch(status, 1);
  top.sort();
  const int64_t row = POS ? i : qid;
  int32_t* out = out_idx + row * k;
  for (int j = 0; j < k; j++) out[j] = j < top.size ? (POS ? tv.pos_of(tv.fwd, top.p[j]) : top.p[j]) : -1;
  if (out_cnt) out_cnt[row] = top.size;
}

template <typename T, int D, typename L>
void launch_knn_big(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                    int32_t* d_idx, int32_t* d_cnt, int* status, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (t->tdepth > BIG_STACK) throw Error(E_UNSUPPORTED, "k > 64 on a tree deeper than 128 levels");
  const size_t per_query = (size_t)k * (sizeof(DistT) + sizeof(int));
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)m, ((size_t)2 << 30) / per_query));
  DevBuf<DistT> hd((size_t)chunk * k, st);
  DevBuf<int> hp((size_t)chunk * k, st);
  for (int m0 = 0; m0 < m; m0 += chunk) {
    const int mc = std::min(chunk, m - m0);
    k_knn_big<T, D, L, false><<<div_up(mc, 128), 128, 0, st>>>(view_of<T, D>(t), ld, order, mode, m0, mc, k, r2,
                                                                 hd.get(), hp.get(), d_idx, d_cnt, status);
    PPTKG_CHECK_LAUNCH();
  }
}

template <typename T, int D>
void knn_query(const TreeBase* t, const QuerySpec& qs, int k, double dmax, int32_t* d_idx, int32_t* d_cnt,
               cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k < 1) throw Error(E_INVALID, "k must be positive");
  const int m = (int)qs.m;
  if (m <= 0) return;
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  DevBuf<int> order, anchors(qs.pts ? m : 0, st);
  const int mode = make_order<T, D>(t, qs, order, st, false, anchors.get());
  const DistT r2 = radius2<DistT>(dmax);
  Stage stage("knn", st);
  if (k > KNN_MAX_K) {
    if (qs.pts) {
      if (qs.qdtype == F64)
        launch_knn_big<T, D>(t, PointQueries<double, D>{(const double*)qs.pts}, order.get(), mode, m, k, r2, d_idx,
                             d_cnt, status.get(), st);
      else
        launch_knn_big<T, D>(t, PointQueries<float, D>{(const float*)qs.pts}, order.get(), mode, m, k, r2, d_idx,
                             d_cnt, status.get(), st);
    } else if (qs.exclude_self) {
      launch_knn_big<T, D>(t, IndexQueries<D, true>{qs.idx, t->fwd}, order.get(), mode, m, k, r2, d_idx, d_cnt,
                           status.get(), st);
    } else {
      launch_knn_big<T, D>(t, IndexQueries<D, false>{qs.idx, t->fwd}, order.get(), mode, m, k, r2, d_idx, d_cnt,
                           status.get(), st);
    }
    check_status(status.get(), st, "knn");
    return;
  }
  if (qs.pts) {
    if (qs.qdtype == F64)
      dispatch_knn<T, D>(t, PointQueries<double, D>{(const double*)qs.pts, anchors.get()}, order.get(), mode, m, k,
                         r2, d_idx, d_cnt, status.get(), st);
    else
      dispatch_knn<T, D>(t, PointQueries<float, D>{(const float*)qs.pts, anchors.get()}, order.get(), mode, m, k, r2,
                         d_idx, d_cnt, status.get(), st);
  } else if (qs.exclude_self) {
    dispatch_knn<T, D>(t, IndexQueries<D, true>{qs.idx, t->fwd}, order.get(), mode, m, k, r2, d_idx, d_cnt,
                       status.get(), st);
  } else {
    dispatch_knn<T, D>(t, IndexQueries<D, false>{qs.idx, t->fwd}, order.get(), mode, m, k, r2, d_idx, d_cnt,
                       status.get(), st);
  }
  check_status(status.get(), st, "knn");
}

// -------------------------------------------------------------- r-near ----
template <typename T, int D, typename L>
__global__ void __launch_bounds__(QTHREADS) k_rnear_count(TreeView<T, D> tv, L ld, const int* order, int order_mode,
                                                          int m, typename DistOf<T>::type r2, int64_t* counts,
                                                          int* status) {
  typedef typename DistOf<T>::type DistT;
  const int slot = blockIdx.x * QTHREADS + threadIdx.x;
  if ((slot & ~31) >= m) return;
  WarpScratch<T, D> ws = warp_scratch<T, D>(tv.depth);
  int qid = -1, own = -1;
  DistT q[D];
  bool active = false;
  if (slot < m) {
    qid = query_of(slot, order, order_mode, tv);
    active = ld.load(qid, tv, q, own);
  }
  if (!active)
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = (DistT)0;
  long long cnt = 0;
  auto none = [](int, const PointRec<T, D>&) {};
  if (!packet_rnear<T, D, DistT, true>(tv, q, active, r2, ws, cnt, none)) atomicExch(status, 1);
  if (own >= 0 && cnt > 0) cnt -= 1;  // the point itself is always a hit when r2 > 0
  if (slot < m) counts[qid] = active ? cnt : 0;
}

template <typename T, int D, typename L>
__global__ void __launch_bounds__(QTHREADS) k_rnear_fill(TreeView<T, D> tv, L ld, const int* order, int order_mode,
                                                         int m, typename DistOf<T>::type r2, const int64_t* off,
                                                         int32_t* out, int* status) {
  typedef typename DistOf<T>::type DistT;
  const int slot = blockIdx.x * QTHREADS + threadIdx.x;
  if ((slot & ~31) >= m) return;
  WarpScratch<T, D> ws = warp_scratch<T, D>(tv.depth);
  int qid = -1, own = -1;
  DistT q[D];
  bool active = false;
  if (slot < m) {
    qid = query_of(slot, order, order_mode, tv);
    active = ld.load(qid, tv, q, own);
  }
  if (!active)
#pragma unroll
    for (int d = 0; d < D; d++) q[d] = (DistT)0;
  int64_t w = active ? off[qid] : 0;
  const int64_t wend = active ? off[qid + 1] : 0;
  bool overflow = false;
  long long unused = 0;
  auto emit = [&](int pos, const PointRec<T, D>& pr) {
    if (pos == own) return;
    if (w < wend)
      out[w++] = pr.id;
    else
      overflow = true;
  };
  if (!packet_rnear<T, D, DistT, false>(tv, q, active, r2, ws, unused, emit)) atomicExch(status, 1);
  if (overflow || w != wend) atomicExch(status, 2);
}

// r-near walk with one warp per query, for batches too small to fill the
// GPU as 32-query packets (a packet lane walks its own hits one by one, so a
// few thousand queries with 1e4-1e5 hits each leave most of the GPU idle).
// The warp walks its query's path once, with all lanes in step, and calls
// visit(begin, n, whole) warp-uniformly for every leaf bucket the ball
// touches and every child box inside the ball (whole = true: all of its
// positions are hits), positions [begin, begin + n).  Children are visited
// left before right, so the ranges come in ascending tree position, the
// order of the reference's left-then-right walk (kdtree-impl.h:519-558).
// Subtree start positions are carried down the walk (a left child starts
// where its parent does, a right child cnt[0] later) and checked against
// every leaf reached.  visit returns false to stop the walk; the result is
// false then, or on a corrupt tree or a full stack.
template <typename T, int D, typename DistT, typename Visit>
__device__ __forceinline__ bool warp_rnear_walk(const TreeView<T, D>& tv, const DistT* q, DistT r2, int* stk,
                                                int stack_ints, Visit visit) {
  const int lane = threadIdx.x & 31;
  bool bad = false;
  // child c of nd, whose positions start at cb: visits it, or returns the
  // inner node to descend into (-1: nothing to descend into)
  auto take = [&](const TNode<T, D>& nd, int c, int cb) -> int {
    const int n = nd.cnt[c];
    if (n == 0 || !(box_min_dist2<T, DistT, D>(nd.lo[c], nd.hi[c], q) < r2)) return -1;
    if (box_max_dist2<T, DistT, D>(nd.lo[c], nd.hi[c], q) < r2) {
      if (!visit(cb, n, true)) bad = true;
      return -1;
    }
    if (nd.ref[c] < 0) {
      if (-nd.ref[c] - 1 != cb || !visit(cb, n, false)) bad = true;
      return -1;
    }
    return nd.ref[c];
  };
  int sp = 0, cur = tv.root, b = 0, visits = 0;
  while (!bad) {
    if (++visits > tv.n_nodes) {  // a tree is acyclic: more visits mean a corrupt node array
      bad = true;
      break;
    }
    const TNode<T, D> nd = load_node(tv.nodes, tv.node_index(cur));
    const int b1 = b + nd.cnt[0];
    int next = take(nd, 0, b);
    if (next >= 0) {
      // into the left subtree; the right child waits if the ball reaches it
      if (nd.cnt[1] > 0 && box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], q) < r2) {
        if (2 * sp + 2 > stack_ints) {
          bad = true;
          break;
        }
        __syncwarp();
        if (lane == 0) {
          stk[2 * sp] = cur * 2 + 1;
          stk[2 * sp + 1] = b1;
        }
        __syncwarp();
        sp++;
      }
      cur = next;
      continue;
    }
    next = take(nd, 1, b1);
    if (next >= 0) {
      cur = next;
      b = b1;
      continue;
    }
    bool found = false;
    while (sp > 0 && !bad) {
      --sp;
      const int e = stk[2 * sp], eb = stk[2 * sp + 1];
      const int r = take(load_node(tv.nodes, tv.node_index(e >> 1)), e & 1, eb);
      if (r >= 0) {
        cur = r;
        b = eb;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  return !bad;
}

// r-near counts or hit lists with one warp per query (warp_rnear_walk):
// lane j tests position base + j of each chunk of a leaf bucket, a box
// inside the ball is taken whole (the fill reads only its ids, the count adds
// its size), and hits are written at their ballot rank, so they come out in
// ascending tree position: the same set and order as the packet walk.
// COUNT: counts[qid] = hits, the query's own point excluded as in
// k_rnear_count; otherwise out[off[qid] ...] = original indices of the hits.
template <typename T, int D, typename L, bool COUNT>
__global__ void __launch_bounds__(QTHREADS) k_rnear_warp(TreeView<T, D> tv, L ld, const int* order, int order_mode,
                                                         int m, typename DistOf<T>::type r2, int stack_ints,
                                                         int64_t* counts, const int64_t* off, int32_t* out,
                                                         int* status) {
  typedef typename DistOf<T>::type DistT;
  extern __shared__ __align__(16) int rw_stack[];
  const int w = blockIdx.x * QWARPS + (threadIdx.x >> 5);
  if (w >= m) return;
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  const unsigned lt = (1u << lane) - 1u;
  int* stk = rw_stack + (threadIdx.x >> 5) * stack_ints;
  const int qid = query_of(w, order, order_mode, tv);
  DistT q[D];
  int own = -1;
  const bool active = ld.load(qid, tv, q, own);
  long long cnt = 0;
  int64_t wp = 0, wend = 0;
  if (!COUNT && active) {
    wp = off[qid];
    wend = off[qid + 1];
  }
  auto visit = [&](int begin, int n, bool whole) -> bool {
    if (COUNT && whole) {
      cnt += n;
      return true;
    }
    bool bad = false;
    for (int base = begin; base < begin + n; base += 32) {
      const int p = base + lane;
      bool hit = false;
      int32_t id = 0;
      if (p < begin + n) {
        if (whole) {
          hit = p != own;
          if (hit) id = tv.pt(p).id;
        } else {
          const PointRec<T, D> pr = tv.pt(p);
          hit = point_dist2<T, DistT, D>(pr.c, q) < r2 && (COUNT || p != own);
          id = pr.id;
        }
      }
      const unsigned hm = __ballot_sync(FULL, hit);
      if (COUNT) {
        cnt += __popc(hm);
      } else {
        if (hit) {
          const int64_t at = wp + __popc(hm & lt);
          if (at < wend)
            out[at] = id;
          else
            bad = true;
        }
        wp += __popc(hm);
      }
    }
    return !__any_sync(FULL, bad);  // warp-uniform
  };
  const bool ok = !active || warp_rnear_walk<T, D, DistT>(tv, q, r2, stk, stack_ints, visit);
  if (lane != 0) return;
  if (COUNT) {
    if (own >= 0 && cnt > 0) cnt -= 1;  // the point itself is always a hit when r2 > 0
    counts[qid] = active ? cnt : 0;
    if (!ok) atomicExch(status, 1);
  } else if (!ok || wp != wend) {
    atomicExch(status, 2);
  }
}

// Per-warp stack of k_rnear_warp: (child ref, start position) pairs, one per
// level at most.
inline int rnear_warp_stack_ints(int depth) { return (2 * (depth + 1) + 3) & ~3; }

template <typename T, int D, typename L, bool COUNT>
void launch_rnear_warp(const TreeBase* t, L ld, const int* order, int mode, int m, typename DistOf<T>::type r2,
                       int64_t* counts, const int64_t* off, int32_t* out, int* status, cudaStream_t st) {
  const int si = rnear_warp_stack_ints(t->tdepth);
  const size_t smem = (size_t)QWARPS * si * sizeof(int);
  if (smem > 48 * 1024)
    PPTKG_CUDA(cudaFuncSetAttribute(k_rnear_warp<T, D, L, COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  k_rnear_warp<T, D, L, COUNT><<<div_up(m, QWARPS), QTHREADS, smem, st>>>(view_of<T, D>(t), ld, order, mode, m, r2,
                                                                            si, counts, off, out, status);
  PPTKG_CHECK_LAUNCH();
}

template <typename T, int D, typename F>
void with_loader(const TreeBase* t, const QuerySpec& qs, F&& f) {
  if (qs.pts) {
    if (qs.qdtype == F64)
      f(PointQueries<double, D>{(const double*)qs.pts});
    else
      f(PointQueries<float, D>{(const float*)qs.pts});
  } else if (qs.exclude_self) {
    f(IndexQueries<D, true>{qs.idx, t->fwd});
  } else {
    f(IndexQueries<D, false>{qs.idx, t->fwd});
  }
}

template <typename T, int D>
int64_t rnear_count(const TreeBase* t, const QuerySpec& qs, double dmax, int64_t* d_off, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  const int m = (int)qs.m;
  if (m <= 0) {
    PPTKG_CUDA(cudaMemsetAsync(d_off, 0, sizeof(int64_t), st));
    return 0;
  }
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  DevBuf<int> order;
  const int mode = make_order<T, D>(t, qs, order, st);
  const DistT r2 = radius2<DistT>(dmax);
  const size_t smem = QWARPS * warp_smem_bytes<T, D>(t->tdepth);
  Stage stage("rnear_count", st);
  with_loader<T, D>(t, qs, [&](auto ld) {
    typedef decltype(ld) L;
    if (m <= g_tune_rnear_warp_queries.load()) {
      launch_rnear_warp<T, D, L, true>(t, ld, order.get(), mode, m, r2, d_off, nullptr, nullptr, status.get(), st);
      return;
    }
    if (smem > 48 * 1024)
      PPTKG_CUDA(cudaFuncSetAttribute(k_rnear_count<T, D, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rnear_count<T, D, L><<<div_up(m, QTHREADS), QTHREADS, smem, st>>>(view_of<T, D>(t), ld, order.get(), mode, m,
                                                                          r2, d_off, status.get());
    PPTKG_CHECK_LAUNCH();
  });
  exclusive_scan<int64_t, int64_t>(d_off, d_off, m, d_off + m, st);
  check_status(status.get(), st, "rnear_count");
  int64_t total = 0;
  PPTKG_CUDA(cudaMemcpyAsync(&total, d_off + m, sizeof(int64_t), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  return total;
}

template <typename T, int D>
void rnear_fill(const TreeBase* t, const QuerySpec& qs, double dmax, const int64_t* d_off, int32_t* d_out,
                cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  const int m = (int)qs.m;
  if (m <= 0) return;
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  DevBuf<int> order;
  const int mode = make_order<T, D>(t, qs, order, st);
  const DistT r2 = radius2<DistT>(dmax);
  const size_t smem = QWARPS * warp_smem_bytes<T, D>(t->tdepth);
  Stage stage("rnear_fill", st);
  with_loader<T, D>(t, qs, [&](auto ld) {
    typedef decltype(ld) L;
    if (m <= g_tune_rnear_warp_queries.load()) {
      launch_rnear_warp<T, D, L, false>(t, ld, order.get(), mode, m, r2, nullptr, d_off, d_out, status.get(), st);
      return;
    }
    if (smem > 48 * 1024)
      PPTKG_CUDA(cudaFuncSetAttribute(k_rnear_fill<T, D, L>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_rnear_fill<T, D, L><<<div_up(m, QTHREADS), QTHREADS, smem, st>>>(view_of<T, D>(t), ld, order.get(), mode, m, r2,
                                                                         d_off, d_out, status.get());
    PPTKG_CHECK_LAUNCH();
  });
  check_status(status.get(), st, "rnear_fill");
}

// ------------------------------------------------------------- normals ----
// Covariance of the neighbourhood in precision P, each neighbour shifted to
// the query point first (p - q, formed in the input type's precision or
// better), then mean-centred in a second pass with compensated sums.  The
// neighbours are the tree positions log[i * 32], i < n.
template <typename T, typename P, typename DistT>
__device__ __forceinline__ Sym3<P> log_covariance(const TreeView<T, 3>& tv, const int* log, int n, const DistT* q) {
  typedef typename std::conditional<(sizeof(T) > sizeof(P)), T, P>::type W;
  P s0 = 0, s1 = 0, s2 = 0;
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> r = tv.pt(log[j * 32]);
    s0 += (P)((W)r.c[0] - (W)q[0]);
    s1 += (P)((W)r.c[1] - (W)q[1]);
    s2 += (P)((W)r.c[2] - (W)q[2]);
  }
  const P inv = n > 0 ? (P)1 / (P)n : (P)0;
  const P m0 = s0 * inv, m1 = s1 * inv, m2 = s2 * inv;
  CSum<P> c00, c01, c02, c11, c12, c22;
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> r = tv.pt(log[j * 32]);
    const P e0 = (P)((W)r.c[0] - (W)q[0]) - m0;
    const P e1 = (P)((W)r.c[1] - (W)q[1]) - m1;
    const P e2 = (P)((W)r.c[2] - (W)q[2]) - m2;
    c00.add(e0 * e0);
    c01.add(e0 * e1);
    c02.add(e0 * e2);
    c11.add(e1 * e1);
    c12.add(e1 * e2);
    c22.add(e2 * e2);
  }
  Sym3<P> C;
  C.a00 = c00.value() * inv;
  C.a01 = c01.value() * inv;
  C.a02 = c02.value() * inv;
  C.a11 = c11.value() * inv;
  C.a12 = c12.value() * inv;
  C.a22 = c22.value() * inv;
  return C;
}

template <typename T, typename P>
__device__ __forceinline__ void write_pca(int row, int n, const P w[3], const P V[9], int num_eigen, T* evecs, T* evals,
                                          int32_t* sizes) {
  if (num_eigen == 1) {
    if (evecs) {
      evecs[(int64_t)row * 3 + 0] = (T)V[0];
      evecs[(int64_t)row * 3 + 1] = (T)V[3];
      evecs[(int64_t)row * 3 + 2] = (T)V[6];
    }
    if (evals) evals[row] = (T)w[0];
  } else {
    if (evecs)
#pragma unroll
      for (int e = 0; e < 3; e++)
#pragma unroll
        for (int c = 0; c < 3; c++) evecs[(int64_t)row * 9 + e * 3 + c] = (T)V[c * 3 + e];
    if (evals)
#pragma unroll
      for (int e = 0; e < 3; e++) evals[(int64_t)row * 3 + e] = (T)w[e];
  }
  if (sizes) sizes[row] = n;
}

template <typename T>
__device__ __forceinline__ void write_invalid(int row, int num_eigen, T* evecs, T* evals, int32_t* sizes) {
  const T nan = (T)NAN;
  const int nv = num_eigen == 1 ? 3 : 9;
  if (evecs)
    for (int c = 0; c < nv; c++) evecs[(int64_t)row * nv + c] = nan;
  if (evals)
    for (int c = 0; c < num_eigen; c++) evals[(int64_t)row * num_eigen + c] = nan;
  if (sizes) sizes[row] = 0;
}

// Blocks per SM that the register budget of a normals kernel aims for: the
// top-k list takes 2 (float) or 3 (double) registers per slot.
constexpr int normals_min_blocks(int kmax, int dist_bytes, int prec) {
  const int need = kmax * (dist_bytes == 4 ? 2 : 3) + (prec == PREC_FP32 ? 64 : 72);
  const int b = 65536 / (QTHREADS * need);
  return b < 1 ? 1 : (b > 8 ? 8 : b);
}

// Fused kNN + PCA.  In the FP32 precision mode a neighbourhood whose two
// smallest eigenvalues nearly coincide (relative gap < gap_thr) is queued in
// `fix` for an FP64 re-solve by a second launch of this kernel in FP64 mode.
//
// With a loader that excludes the query point, own (ExcludesSelf; the
// forest's fused query, knn_idx set), one walk answers both a self kNN and
// the normal: the list is
// the k nearest other points, written to knn_idx / knn_cnt as k_knn writes
// them, and the neighbourhood of the normal is that list with the query
// point put in at its place in (dist2, id) order and cut to k -- the k
// nearest including the query point, in the order the normal-only walk
// gathers them, so both results equal the separate calls.
template <typename T, int KMAX, typename L, int PREC>
__global__ void __launch_bounds__(QTHREADS, normals_min_blocks(KMAX, sizeof(typename DistOf<T>::type), PREC))
k_normals(TreeView<T, 3> tv, L ld, const int* order, int order_mode, int m,
                                                      int k, typename DistOf<T>::type r2, int num_eigen,
                                                      double gap_thr, T* evecs, T* evals, int32_t* sizes,
                                                      int* fix, int* nfix, int* status, SlotMap fm, int lane_span,
                                                      bool warm_bound, int warm_mult, int32_t* knn_idx,
                                                      int32_t* knn_cnt) {
  typedef typename DistOf<T>::type DistT;
  constexpr int LOGCAP = normals_logcap(KMAX);
  const int slot = blockIdx.x * QTHREADS + threadIdx.x;
  if ((slot & ~31) >= m) return;
  WarpScratch<T, 3> ws = warp_scratch<T, 3>(tv.depth, LOGCAP);
  const int lane = threadIdx.x & 31;
  int qid = -1, own = -1, grp = 0, anchor = -1;
  DistT q[3];
  bool active = false;
  if (fm.warp_cloud) {
    grp = fm.views ? fm.warp_cloud[slot >> 5] : 0;
    qid = forest_query(slot, fm, tv);
    if (qid >= 0) active = ld.load(qid, tv, q, own, &anchor);
  } else if (slot < m) {
    qid = query_of(slot, order, order_mode, tv);
    active = ld.load(qid, tv, q, own, &anchor);
  }
  if (!active) q[0] = q[1] = q[2] = (DistT)0;
  int* lane_log = ws.log + lane;
  TopK<KMAX, DistT> top;
  top.reset(k, r2);
  int wlo = 0, wn = 0;
  if (active) warm_topk<T, 3, DistT>(top, tv, fm, slot, q, anchor, k, own, r2, warm_bound, warm_mult, wlo, wn);
  const bool ok = use_lane_walk<LANE_STACK>(anchor, active, lane_span, tv.depth)
                      ? lane_knn<LANE_STACK, T, 3>(tv, q, own, active, r2, top, wlo, wn)
                      : packet_knn<T, 3>(tv, q, own, active, r2, top, ws, wlo, wn);
  if (!ok) atomicExch(status, 1);
  if (qid < 0) return;
  if (!active) {
    write_invalid<T>(qid, num_eigen, evecs, evals, sizes);
    if constexpr (ExcludesSelf<L>::value) {
      for (int j = 0; j < k; j++) knn_idx[(int64_t)qid * k + j] = -1;
      if (knn_cnt) knn_cnt[qid] = 0;
    }
    return;
  }
  // the list holds point ids; the neighbours are gathered from their tree
  // positions (the index map's loads are independent and overlap)
  int n = 0;
  if constexpr (ExcludesSelf<L>::value) {
    int c = 0;
    bool placed = false;
#pragma unroll
    for (int j = KMAX - 1; j >= 0; j--) {
      if (j < k) {
        const bool v = top.valid(j);
        knn_idx[(int64_t)qid * k + (k - 1 - j)] = v ? top.id(j) : -1;
        if (v) {
          c++;
          if (!placed && !top.below_zero(j, qid)) {
            lane_log[(n++) * 32] = own;
            placed = true;
          }
          if (n < k) lane_log[(n++) * 32] = tv.pos_of(tv.fwd, top.id(j));
        }
      }
    }
    if (!placed && n < k) lane_log[(n++) * 32] = own;
    if (knn_cnt) knn_cnt[qid] = c;
  } else {
    (void)knn_idx;
    (void)knn_cnt;
#pragma unroll
    for (int j = KMAX - 1; j >= 0; j--)
      if (j < k && top.valid(j)) lane_log[(n++) * 32] = tv.pos_of(tv.fwd, top.id(j));
  }
  if (PREC == PREC_FP64) {
    Sym3<double> C = log_covariance<T, double, DistT>(tv, lane_log, n, q);
    double w[3], V[9];
    eigh3<double>(C, w, V);
    write_pca<T, double>(qid, n, w, V, num_eigen, evecs, evals, sizes);
  } else {
    Sym3<float> C = log_covariance<T, float, DistT>(tv, lane_log, n, q);
    float w[3], V[9];
    eigh3<float>(C, w, V);
    write_pca<T, float>(qid, n, w, V, num_eigen, evecs, evals, sizes);
    if (fix && n > 0 && !(rel_gap<float>(w) >= (float)gap_thr)) {
      // queue [query, count, neighbour positions] for the FP64 re-solve
      int* e = fix + (int64_t)atomicAdd(nfix, 1) * (KMAX + 2);
      e[0] = qid;
      e[1] = n | (grp << 8);
      for (int j = 0; j < n; j++) e[2 + j] = lane_log[j * 32];
    }
  }
}

// r-near neighbourhoods (k == -1): moments accumulated during the traversal
// in FP64, shifted to the query point.
template <typename T, typename L>
__global__ void __launch_bounds__(QTHREADS) k_normals_rnear(TreeView<T, 3> tv, L ld, const int* order, int order_mode,
                                                            int m, typename DistOf<T>::type r2, int num_eigen,
                                                            T* evecs, T* evals, int32_t* sizes, int* status) {
  typedef typename DistOf<T>::type DistT;
  const int slot = blockIdx.x * QTHREADS + threadIdx.x;
  if ((slot & ~31) >= m) return;
  WarpScratch<T, 3> ws = warp_scratch<T, 3>(tv.depth);
  int qid = -1, own = -1;
  DistT q[3];
  bool active = false;
  if (slot < m) {
    qid = query_of(slot, order, order_mode, tv);
    active = ld.load(qid, tv, q, own);
  }
  if (!active) q[0] = q[1] = q[2] = (DistT)0;
  double s[3] = {0, 0, 0}, ss[6] = {0, 0, 0, 0, 0, 0};
  long long n = 0;
  auto emit = [&](int pos, const PointRec<T, 3>& pr) {
    const double e0 = (double)pr.c[0] - (double)q[0], e1 = (double)pr.c[1] - (double)q[1],
                 e2 = (double)pr.c[2] - (double)q[2];
    s[0] += e0;
    s[1] += e1;
    s[2] += e2;
    ss[0] += e0 * e0;
    ss[1] += e0 * e1;
    ss[2] += e0 * e2;
    ss[3] += e1 * e1;
    ss[4] += e1 * e2;
    ss[5] += e2 * e2;
    n++;
  };
  long long unused = 0;
  if (!packet_rnear<T, 3, DistT, false>(tv, q, active, r2, ws, unused, emit)) atomicExch(status, 1);
  if (slot >= m) return;
  if (!active || n == 0) {
    write_invalid<T>(qid, num_eigen, evecs, evals, sizes);
    return;
  }
  const double inv = 1.0 / (double)n;
  const double m0 = s[0] * inv, m1 = s[1] * inv, m2 = s[2] * inv;
  Sym3<double> C;
  C.a00 = ss[0] * inv - m0 * m0;
  C.a01 = ss[1] * inv - m0 * m1;
  C.a02 = ss[2] * inv - m0 * m2;
  C.a11 = ss[3] * inv - m1 * m1;
  C.a12 = ss[4] * inv - m1 * m2;
  C.a22 = ss[5] * inv - m2 * m2;
  double w[3], V[9];
  eigh3<double>(C, w, V);
  write_pca<T, double>(qid, (int)n, w, V, num_eigen, evecs, evals, sizes);
}

// k_normals_rnear with one warp per query (warp_rnear_walk), for batches
// too small to fill the GPU as packets: each lane accumulates the shifted
// FP64 sums of the hits it tests (boxes inside the ball are summed without
// distance tests), the warp adds the lanes' sums, and lane 0 solves.  The
// neighbourhood (every point within r, the query point included) and its
// size are those of the packet kernel; the sums add in another order, so
// results agree to FP64 rounding.
template <typename T, typename L>
__global__ void __launch_bounds__(QTHREADS) k_normals_rnear_warp(TreeView<T, 3> tv, L ld, const int* order,
                                                                 int order_mode, int m, typename DistOf<T>::type r2,
                                                                 int stack_ints, int num_eigen, T* evecs, T* evals,
                                                                 int32_t* sizes, int* status) {
  typedef typename DistOf<T>::type DistT;
  extern __shared__ __align__(16) int rw_stack[];
  const int w = blockIdx.x * QWARPS + (threadIdx.x >> 5);
  if (w >= m) return;
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  int* stk = rw_stack + (threadIdx.x >> 5) * stack_ints;
  const int qid = query_of(w, order, order_mode, tv);
  DistT q[3];
  int own = -1;
  const bool active = ld.load(qid, tv, q, own);
  double s[3] = {0, 0, 0}, ss[6] = {0, 0, 0, 0, 0, 0};
  long long n = 0;
  auto visit = [&](int begin, int cnt, bool whole) -> bool {
    for (int base = begin; base < begin + cnt; base += 32) {
      const int p = base + lane;
      if (p >= begin + cnt) continue;
      const PointRec<T, 3> pr = tv.pt(p);
      if (!whole && !(point_dist2<T, DistT, 3>(pr.c, q) < r2)) continue;
      const double e0 = (double)pr.c[0] - (double)q[0], e1 = (double)pr.c[1] - (double)q[1],
                   e2 = (double)pr.c[2] - (double)q[2];
      s[0] += e0;
      s[1] += e1;
      s[2] += e2;
      ss[0] += e0 * e0;
      ss[1] += e0 * e1;
      ss[2] += e0 * e2;
      ss[3] += e1 * e1;
      ss[4] += e1 * e2;
      ss[5] += e2 * e2;
      n++;
    }
    __syncwarp();
    return true;
  };
  const bool ok = !active || warp_rnear_walk<T, 3, DistT>(tv, q, r2, stk, stack_ints, visit);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
    for (int d = 0; d < 3; d++) s[d] += __shfl_xor_sync(FULL, s[d], o);
#pragma unroll
    for (int d = 0; d < 6; d++) ss[d] += __shfl_xor_sync(FULL, ss[d], o);
    n += __shfl_xor_sync(FULL, n, o);
  }
  if (lane != 0) return;
  if (!ok) atomicExch(status, 1);
  if (!active || n == 0) {
    write_invalid<T>(qid, num_eigen, evecs, evals, sizes);
    return;
  }
  const double inv = 1.0 / (double)n;
  const double m0 = s[0] * inv, m1 = s[1] * inv, m2 = s[2] * inv;
  Sym3<double> C;
  C.a00 = ss[0] * inv - m0 * m0;
  C.a01 = ss[1] * inv - m0 * m1;
  C.a02 = ss[2] * inv - m0 * m2;
  C.a11 = ss[3] * inv - m1 * m1;
  C.a12 = ss[4] * inv - m1 * m2;
  C.a22 = ss[5] * inv - m2 * m2;
  double wv[3], V[9];
  eigh3<double>(C, wv, V);
  write_pca<T, double>(qid, (int)n, wv, V, num_eigen, evecs, evals, sizes);
}

// FP64 re-solve of queued neighbourhoods: one thread per entry, a gather of
// the stored neighbour positions, float64 covariance (shifted to the first
// neighbour, centred) and eigensolve; overwrites the FP32 results of that
// output row.
//
// Entry layout: [output row, count | group << 8, positions...] with
// 1 <= count <= KMAX; in a multi-tree batch the group selects the tree whose
// points the positions refer to (views[group]), otherwise `pts` is the
// tree's own.
template <typename T, int KMAX>
__global__ void k_refine64(const PointRec<T, 3>* pts, const int* fix, const int* nfix, int num_eigen, T* evecs,
                           T* evals, int32_t* sizes, const TreeView<T, 3>* views) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= *nfix) return;
  const int* e = fix + (int64_t)i * (KMAX + 2);
  const int qid = e[0], n = e[1] & 0xff, grp = e[1] >> 8;
  if (views) pts = views[grp].pts;
  const PointRec<T, 3> qr = pts[e[2]];
  double s0 = 0, s1 = 0, s2 = 0;
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> r = pts[e[2 + j]];
    s0 += (double)r.c[0] - (double)qr.c[0];
    s1 += (double)r.c[1] - (double)qr.c[1];
    s2 += (double)r.c[2] - (double)qr.c[2];
  }
  const double inv = 1.0 / (double)n, m0 = s0 * inv, m1 = s1 * inv, m2 = s2 * inv;
  Sym3<double> C{0, 0, 0, 0, 0, 0};
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> r = pts[e[2 + j]];
    const double a = (double)r.c[0] - (double)qr.c[0] - m0, b = (double)r.c[1] - (double)qr.c[1] - m1,
                 c = (double)r.c[2] - (double)qr.c[2] - m2;
    C.a00 += a * a;
    C.a01 += a * b;
    C.a02 += a * c;
    C.a11 += b * b;
    C.a12 += b * c;
    C.a22 += c * c;
  }
  C.a00 *= inv;
  C.a01 *= inv;
  C.a02 *= inv;
  C.a11 *= inv;
  C.a12 *= inv;
  C.a22 *= inv;
  double w[3], V[9];
  eigh3<double>(C, w, V);
  write_pca<T, double>(qid, n, w, V, num_eigen, evecs, evals, sizes);
}

template <typename T, int KMAX, typename L, int PREC>
void launch_normals(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                    int num_eigen, double gap_thr, T* ev, T* ew, int32_t* sz, int* fix, int* nfix, int* status,
                    cudaStream_t st, SlotMap fm = SlotMap{}, int32_t* kidx = nullptr, int32_t* kcnt = nullptr) {
  if (m <= 0) return;
  const size_t smem = QWARPS * warp_smem_bytes<T, 3>(t->tdepth, normals_logcap(KMAX));
  if (smem > 48 * 1024)
    PPTKG_CUDA(
        cudaFuncSetAttribute(k_normals<T, KMAX, L, PREC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_normals<T, KMAX, L, PREC><<<div_up(m, QTHREADS), QTHREADS, smem, st>>>(
      view_of<T, 3>(t), ld, order, mode, m, k, r2, num_eigen, gap_thr, ev, ew, sz, fix, nfix, status, fm,
      g_tune_lane_span.load(), g_tune_warm_bound.load() != 0, g_tune_warm_mult.load(), kidx, kcnt);
  PPTKG_CHECK_LAUNCH();
}

template <typename T, int KMAX, typename L>
void normals_pass(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                  int num_eigen, int prec, double gap_thr, T* ev, T* ew, int32_t* sz, int* status, cudaStream_t st,
                  SlotMap fm = SlotMap{}, int32_t* kidx = nullptr, int32_t* kcnt = nullptr) {
  if (prec == PREC_FP64) {
    launch_normals<T, KMAX, L, PREC_FP64>(t, ld, order, mode, m, k, r2, num_eigen, gap_thr, ev, ew, sz, nullptr,
                                          nullptr, status, st, fm, kidx, kcnt);
    return;
  }
  // FP32 pass, then an FP64 re-solve of the queued small-gap neighbourhoods
  DevBuf<int> fix((size_t)std::max(m, 1) * (KMAX + 2), st), nfix(1, st);
  PPTKG_CUDA(cudaMemsetAsync(nfix.get(), 0, sizeof(int), st));
  launch_normals<T, KMAX, L, PREC_FP32>(t, ld, order, mode, m, k, r2, num_eigen, gap_thr, ev, ew, sz, fix.get(),
                                        nfix.get(), status, st, fm, kidx, kcnt);
  {
    Stage s("normals.refine64", st);
    k_refine64<T, KMAX><<<div_up(m, 256), 256, 0, st>>>((const PointRec<T, 3>*)t->pts, fix.get(), nfix.get(),
                                                        num_eigen, ev, ew, sz,
                                                        static_cast<const TreeView<T, 3>*>(fm.views));
    PPTKG_CHECK_LAUNCH();
  }
}

template <typename T, typename L>
void dispatch_normals(const TreeBase* t, L ld, const int* order, int mode, int m, int k,
                      typename DistOf<T>::type r2, int num_eigen, int prec, double gap_thr, T* ev, T* ew,
                      int32_t* sz, int* status, cudaStream_t st, SlotMap fm = SlotMap{}, int32_t* kidx = nullptr,
                      int32_t* kcnt = nullptr) {
  const int kc = std::max(k, g_tune_topk_min.load());
  if (kc <= 4)
    normals_pass<T, 4, L>(t, ld, order, mode, m, k, r2, num_eigen, prec, gap_thr, ev, ew, sz, status, st, fm, kidx,
                          kcnt);
  else if (kc <= 8)
    normals_pass<T, 8, L>(t, ld, order, mode, m, k, r2, num_eigen, prec, gap_thr, ev, ew, sz, status, st, fm, kidx,
                          kcnt);
  else if (kc <= 16)
    normals_pass<T, 16, L>(t, ld, order, mode, m, k, r2, num_eigen, prec, gap_thr, ev, ew, sz, status, st, fm, kidx,
                           kcnt);
  else if (kc <= 32)
    normals_pass<T, 32, L>(t, ld, order, mode, m, k, r2, num_eigen, prec, gap_thr, ev, ew, sz, status, st, fm, kidx,
                           kcnt);
  else
    normals_pass<T, 64, L>(t, ld, order, mode, m, k, r2, num_eigen, prec, gap_thr, ev, ew, sz, status, st, fm, kidx,
                           kcnt);
}

// Normals of neighbourhoods held as tree positions (pos: m x k, counts cnt),
// the large-k path: float64 covariance shifted to the query point and
// centred, float64 eigensolve, results in T.
template <typename T, typename L>
__global__ void k_normals_pos(TreeView<T, 3> tv, L ld, const int* order, int order_mode, int m0, int m, int k,
                              const int32_t* pos, const int32_t* cnt, int num_eigen, T* evecs, T* evals,
                              int32_t* sizes) {
  typedef typename DistOf<T>::type DistT;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const int qid = query_of(m0 + i, order, order_mode, tv);
  int own = -1;
  DistT q[3];
  const bool active = ld.load(qid, tv, q, own);
  const int n = cnt[i];
  if (!active || n <= 0) {
    write_invalid<T>(qid, num_eigen, evecs, evals, sizes);
    return;
  }
  const int32_t* P = pos + (int64_t)i * k;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> rp = tv.pt(P[j]);
    s0 += (double)rp.c[0] - (double)q[0];
    s1 += (double)rp.c[1] - (double)q[1];
    s2 += (double)rp.c[2] - (double)q[2];
  }
  const double inv = 1.0 / (double)n, a0 = s0 * inv, a1 = s1 * inv, a2 = s2 * inv;
  Sym3<double> C{0, 0, 0, 0, 0, 0};
  for (int j = 0; j < n; j++) {
    const PointRec<T, 3> rp = tv.pt(P[j]);
    const double x = (double)rp.c[0] - (double)q[0] - a0, y = (double)rp.c[1] - (double)q[1] - a1,
                 z = (double)rp.c[2] - (double)q[2] - a2;
    C.a00 += x * x;
    C.a01 += x * y;
    C.a02 += x * z;
    C.a11 += y * y;
    C.a12 += y * z;
    C.a22 += z * z;
  }
  C.a00 *= inv;
  C.a01 *= inv;
  C.a02 *= inv;
  C.a11 *= inv;
  C.a12 *= inv;
  C.a22 *= inv;
  double w[3], V[9];
  eigh3<double>(C, w, V);
  write_pca<T, double>(qid, n, w, V, num_eigen, evecs, evals, sizes);
}

// estimate_normals with k above the register lists: the large-k walk writes
// each chunk's neighbourhoods as tree positions, k_normals_pos solves them.
template <typename T, typename L>
void normals_big(const TreeBase* t, L ld, const int* order, int mode, int m, int k, typename DistOf<T>::type r2,
                 int num_eigen, T* ev, T* ew, int32_t* sz, int* status, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (t->tdepth > BIG_STACK) throw Error(E_UNSUPPORTED, "k > 64 on a tree deeper than 128 levels");
  const size_t per_query = (size_t)k * (sizeof(DistT) + 2 * sizeof(int)) + sizeof(int);
  const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)m, ((size_t)2 << 30) / per_query));
  DevBuf<DistT> hd((size_t)chunk * k, st);
  DevBuf<int> hp((size_t)chunk * k, st), pos((size_t)chunk * k, st), cnt(chunk, st);
  for (int m0 = 0; m0 < m; m0 += chunk) {
    const int mc = std::min(chunk, m - m0);
    k_knn_big<T, 3, L, true><<<div_up(mc, 128), 128, 0, st>>>(view_of<T, 3>(t), ld, order, mode, m0, mc, k, r2,
                                                                hd.get(), hp.get(), pos.get(), cnt.get(), status);
    PPTKG_CHECK_LAUNCH();
    k_normals_pos<T, L><<<div_up(mc, 128), 128, 0, st>>>(view_of<T, 3>(t), ld, order, mode, m0, mc, k, pos.get(),
                                                          cnt.get(), num_eigen, ev, ew, sz);
    PPTKG_CHECK_LAUNCH();
  }
}

template <typename T>
void normals_query(const TreeBase* t, const QuerySpec& qs_in, int k, float r, int num_eigen, int precision,
                   double gap_thr, T* d_evecs, T* d_evals, int32_t* d_sizes, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k == 0 || k < -1) throw Error(E_INVALID, "k must be positive or -1");
  QuerySpec qs = qs_in;
  qs.pts = nullptr;
  qs.exclude_self = false;
  const int m = (int)qs.m;
  if (m <= 0) return;
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  DevBuf<int> order;
  int mode = make_order<T, 3>(t, qs, order, st);
  if (mode == 2) {
    // tree order covers valid points only: rows of dropped points (none when
    // n == nv) need no separate pass
  }
  // the radius travels as a C float (estimate_normals.cpp:264) and is cast to
  // the input type (:17-22) before being squared in the distance type
  const DistT rr = (DistT)(T)r;
  const DistT r2 = rr * rr;
  IndexQueries<3, false> ld{qs.idx, t->fwd};
  Stage stage("normals", st);
  if (k == -1 && m <= g_tune_rnear_warp_queries.load()) {
    const int si = rnear_warp_stack_ints(t->tdepth);
    const size_t smem = (size_t)QWARPS * si * sizeof(int);
    if (smem > 48 * 1024)
      PPTKG_CUDA(cudaFuncSetAttribute(k_normals_rnear_warp<T, IndexQueries<3, false>>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_normals_rnear_warp<T, IndexQueries<3, false>><<<div_up(m, QWARPS), QTHREADS, smem, st>>>(
        view_of<T, 3>(t), ld, order.get(), mode, m, r2, si, num_eigen, d_evecs, d_evals, d_sizes, status.get());
    PPTKG_CHECK_LAUNCH();
  } else if (k == -1) {
    const size_t smem = QWARPS * warp_smem_bytes<T, 3>(t->tdepth);
    if (smem > 48 * 1024)
      PPTKG_CUDA(cudaFuncSetAttribute(k_normals_rnear<T, IndexQueries<3, false>>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_normals_rnear<T, IndexQueries<3, false>><<<div_up(m, QTHREADS), QTHREADS, smem, st>>>(
        view_of<T, 3>(t), ld, order.get(), mode, m, r2, num_eigen, d_evecs, d_evals, d_sizes, status.get());
    PPTKG_CHECK_LAUNCH();
  } else if (k > KNN_MAX_K) {
    normals_big<T, IndexQueries<3, false>>(t, ld, order.get(), mode, m, k, r2, num_eigen, d_evecs, d_evals, d_sizes,
                                          status.get(), st);
  } else {
    int prec = precision;
    if (prec == PREC_AUTO) prec = sizeof(T) == 4 ? PREC_FP32 : PREC_FP64;
    dispatch_normals<T, IndexQueries<3, false>>(t, ld, order.get(), mode, m, k, r2, num_eigen, prec, gap_thr, d_evecs,
                                                d_evals, d_sizes, status.get(), st);
  }
  check_status(status.get(), st, "normals");
}

// --------------------------------------------------------------- eigh3 ----
template <typename T>
__global__ void k_eigh3(const T* A, int64_t m, T* w, T* V, int layout) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  const T* a = A + i * 9;
  Sym3<T> S;
  S.a00 = a[0];
  S.a01 = a[1];
  S.a02 = a[2];
  S.a11 = a[4];
  S.a12 = a[5];
  S.a22 = a[8];
  T ww[3], VV[9];
  eigh3<T>(S, ww, VV);
  for (int e = 0; e < 3; e++) w[i * 3 + e] = ww[e];
  // layout 0: V[i, r, c] = component r of eigenvector c (columns, as
  // vfuncs._eigh returns them); layout 1: [i, e, :] = eigenvector e
  for (int r = 0; r < 3; r++)
    for (int c = 0; c < 3; c++) V[i * 9 + r * 3 + c] = layout == 0 ? VV[r * 3 + c] : VV[c * 3 + r];
}

template <typename T>
void eigh3_batched(const T* d_A, int64_t m, T* d_w, T* d_V, int layout, cudaStream_t st) {
  if (m <= 0) return;
  k_eigh3<T><<<(unsigned)((m + 255) / 256), 256, 0, st>>>(d_A, m, d_w, d_V, layout);
  PPTKG_CHECK_LAUNCH();
}

// ------------------------------------------------------------ forests ----
static __global__ void k_warp_cloud(const int64_t* slot_off, int ncloud, int64_t nwarps, int* warp_cloud) {
  const int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwarps) return;
  const int64_t s = w * 32;
  int lo = 0, hi = ncloud - 1;  // last cloud whose first slot is <= s
  while (lo < hi) {
    const int mid = (lo + hi + 1) / 2;
    if (slot_off[mid] <= s)
      lo = mid;
    else
      hi = mid - 1;
  }
  warp_cloud[w] = lo;
}

// Slot map of a forest (cached on the tree): cloud c's valid points take the
// slots [slot_off[c], slot_off[c] + count), rounded up to whole warps.
static SlotMap slot_map(const TreeBase* t, int64_t& n_slots, cudaStream_t st) {
  TreeBase* mt = const_cast<TreeBase*>(t);
  if (!mt->warp_cloud && g_status_sink)
    throw Error(E_INVALID, "a forest's first query must run without a status sink (it synchronises once)");
  if (!mt->warp_cloud) {
    std::vector<int64_t> so(t->ncloud + 1, 0);
    for (int c = 0; c < t->ncloud; c++) {
      const int64_t cnt = t->valid_off_h[c + 1] - t->valid_off_h[c];
      so[c + 1] = so[c] + (cnt + 31) / 32 * 32;
    }
    mt->n_slots = so[t->ncloud];
    if (mt->n_slots > INT32_MAX) throw Error(E_INVALID, "forest too large for one query pass");
    PPTKG_CUDA(dev_malloc((void**)&mt->slot_off, sizeof(int64_t) * (t->ncloud + 1), st));
    PPTKG_CUDA(cudaMemcpyAsync(mt->slot_off, so.data(), sizeof(int64_t) * (t->ncloud + 1), cudaMemcpyHostToDevice, st));
    const int64_t nw = std::max<int64_t>(mt->n_slots / 32, 1);
    PPTKG_CUDA(dev_malloc((void**)&mt->warp_cloud, sizeof(int) * nw, st));
    if (mt->n_slots > 0) {
      k_warp_cloud<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(mt->slot_off, t->ncloud, nw, mt->warp_cloud);
      PPTKG_CHECK_LAUNCH();
    }
    PPTKG_CUDA(cudaStreamSynchronize(st));
  }
  n_slots = mt->n_slots;
  return SlotMap{mt->warp_cloud, mt->slot_off, t->valid_off, t->root_tnode, nullptr, nullptr, nullptr};
}

#ifndef PPTKG_QUERY_DIM
// Slots of each cloud rounded up to whole warps (capture mode: from the
// device's valid offsets).
static __global__ void k_slot_counts(const int64_t* valid_off, int ncloud, int64_t* cnt) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < ncloud) cnt[c] = (valid_off[c + 1] - valid_off[c] + 31) / 32 * 32;
}

// The slot map of a capture-ready forest, computed on the device from its
// current valid offsets over a fixed slot capacity (every cloud's input rows
// rounded up to whole warps); warps beyond the live slots find no query.
void forest_slot_map_device(TreeBase* t, cudaStream_t st) {
  int64_t cap = 0;
  for (int c = 0; c < t->ncloud; c++) cap += (t->orig_off_h[c + 1] - t->orig_off_h[c] + 31) / 32 * 32;
  if (cap > INT32_MAX) throw Error(E_INVALID, "forest too large for one query pass");
  const int64_t nw = std::max<int64_t>(cap / 32, 1);
  if (!t->slot_off) PPTKG_CUDA(dev_malloc((void**)&t->slot_off, sizeof(int64_t) * (t->ncloud + 1), st));
  if (!t->warp_cloud || t->n_slots != cap) {
    if (t->warp_cloud) dev_free(t->warp_cloud, st);
    PPTKG_CUDA(dev_malloc((void**)&t->warp_cloud, sizeof(int) * nw, st));
  }
  t->n_slots = cap;
  DevBuf<int64_t> cnt(t->ncloud, st);
  k_slot_counts<<<div_up(t->ncloud, 256), 256, 0, st>>>(t->valid_off, t->ncloud, cnt.get());
  PPTKG_CHECK_LAUNCH();
  exclusive_scan<int64_t, int64_t>(cnt.get(), t->slot_off, t->ncloud, t->slot_off + t->ncloud, st);
  k_warp_cloud<<<(unsigned)((nw + 255) / 256), 256, 0, st>>>(t->slot_off, t->ncloud, nw, t->warp_cloud);
  PPTKG_CHECK_LAUNCH();
}
#endif  // PPTKG_QUERY_DIM

template <typename T, int D>
void forest_knn(const TreeBase* t, int k, double dmax, bool exclude_self, int32_t* d_idx, int32_t* d_cnt,
                cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k < 1) throw Error(E_INVALID, "k must be positive");
  if (k > KNN_MAX_K) throw Error(E_UNSUPPORTED, "k > 64 is not supported by the GPU kNN kernels");
  int64_t n_slots = 0;
  const SlotMap fm = slot_map(t, n_slots, st);
  // rows of dropped (NaN/inf) points are not visited: no neighbours
  PPTKG_CUDA(cudaMemsetAsync(d_idx, 0xff, sizeof(int32_t) * (size_t)t->n * k, st));
  if (d_cnt) PPTKG_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (size_t)t->n, st));
  if (n_slots == 0) return;
  StatusWord status(st);
  const DistT r2 = radius2<DistT>(dmax);
  Stage stage("forest.knn", st);
  if (exclude_self)
    dispatch_knn<T, D>(t, IndexQueries<D, true>{nullptr, t->fwd}, nullptr, 0, (int)n_slots, k, r2, d_idx, d_cnt,
                       status.get(), st, fm);
  else
    dispatch_knn<T, D>(t, IndexQueries<D, false>{nullptr, t->fwd}, nullptr, 0, (int)n_slots, k, r2, d_idx, d_cnt,
                       status.get(), st, fm);
  status.check(st, "forest knn");
}

template <typename T>
__global__ void k_fill_invalid(int64_t n, int num_eigen, T* evecs, T* evals, int32_t* sizes) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) write_invalid<T>((int)i, num_eigen, evecs, evals, sizes);
}

template <typename T>
void forest_normals(const TreeBase* t, int k, float r, int num_eigen, int precision, double gap_thr, T* d_evecs,
                    T* d_evals, int32_t* d_sizes, cudaStream_t st, int32_t* d_idx, int32_t* d_cnt) {
  typedef typename DistOf<T>::type DistT;
  if (t->dim != 3) throw Error(E_TYPE, "normals need 3-d points");
  if (k < 1) throw Error(E_INVALID, "forest normals need k >= 1");
  if (k > KNN_MAX_K) throw Error(E_UNSUPPORTED, "k > 64 is not supported by the GPU normal kernels");
  int64_t n_slots = 0;
  const SlotMap fm = slot_map(t, n_slots, st);
  // rows of dropped points get NaN and size 0 (a capture-ready forest
  // cannot tell from the host whether it has such rows)
  if ((t->capture || t->n > t->nv) && t->n > 0) {
    k_fill_invalid<T><<<(unsigned)((t->n + 255) / 256), 256, 0, st>>>(t->n, num_eigen, d_evecs, d_evals, d_sizes);
    PPTKG_CHECK_LAUNCH();
    // (and no neighbours, for the fused kNN)
    if (d_idx) PPTKG_CUDA(cudaMemsetAsync(d_idx, 0xff, sizeof(int32_t) * (size_t)t->n * k, st));
    if (d_cnt) PPTKG_CUDA(cudaMemsetAsync(d_cnt, 0, sizeof(int32_t) * (size_t)t->n, st));
  }
  if (n_slots == 0) return;
  StatusWord status(st);
  const DistT rr = (DistT)(T)r;
  const DistT r2 = rr * rr;
  int prec = precision == PREC_AUTO ? (sizeof(T) == 4 ? PREC_FP32 : PREC_FP64) : precision;
  if (d_idx) {
    // one walk for the self kNN (the list excludes the query point) and
    // the normal (the query point put back in)
    Stage stage("forest.knn_normals", st);
    dispatch_normals<T, IndexQueries<3, true>>(t, IndexQueries<3, true>{nullptr, t->fwd}, nullptr, 0, (int)n_slots,
                                               k, r2, num_eigen, prec, gap_thr, d_evecs, d_evals, d_sizes,
                                               status.get(), st, fm, d_idx, d_cnt);
    status.check(st, "forest kNN + normals");
    return;
  }
  Stage stage("forest.normals", st);
  dispatch_normals<T, IndexQueries<3, false>>(t, IndexQueries<3, false>{nullptr, t->fwd}, nullptr, 0, (int)n_slots,
                                              k, r2, num_eigen, prec, gap_thr, d_evecs, d_evals, d_sizes, status.get(),
                                              st, fm);
  status.check(st, "forest normals");
}

#ifndef PPTKG_QUERY_DIM
template void forest_knn<float, 3>(const TreeBase*, int, double, bool, int32_t*, int32_t*, cudaStream_t);
template void forest_knn<double, 3>(const TreeBase*, int, double, bool, int32_t*, int32_t*, cudaStream_t);
template void forest_normals<float>(const TreeBase*, int, float, int, int, double, float*, float*, int32_t*,
                                    cudaStream_t, int32_t*, int32_t*);
template void forest_normals<double>(const TreeBase*, int, float, int, int, double, double*, double*, int32_t*,
                                     cudaStream_t, int32_t*, int32_t*);
#endif  // PPTKG_QUERY_DIM


// ---------------------------------------------------- multi-tree batches --
// Device tables of a multi-tree batch: TreeViews, per-warp group, slot and
// row offsets, uploaded as one block.  `rows` are host offsets (ntrees + 1)
// of each tree's queries.
template <typename T, int D>
struct MultiTables {
  DevBuf<char> blob;
  const TreeView<T, D>* views = nullptr;
  const int64_t *slot_off = nullptr, *row_off = nullptr;
  const int* warp_tree = nullptr;
  DevBuf<int> order, anchor;
  bool ordered = false;
  int64_t n_slots = 0;
  int depth = 0, n_nodes = 0;
  SlotMap map() const {
    return SlotMap{warp_tree, slot_off, nullptr, nullptr, views, row_off, ordered ? order.get() : nullptr};
  }
};

template <typename T, int D>
void multi_tables(const TreeBase* const* trees, int ntrees, const int64_t* rows, MultiTables<T, D>& mt, cudaStream_t st) {
  std::vector<TreeView<T, D>> v(ntrees);
  std::vector<int64_t> so(ntrees + 1, 0);
  for (int g = 0; g < ntrees; g++) {
    const TreeBase* t = trees[g];
    if (t->dtype != (sizeof(T) == 4 ? F32 : F64) || t->dim != D)
      throw Error(E_TYPE, "all trees of a batch must share dtype and dim");
    if (t->ncloud != 1) throw Error(E_INVALID, "multi-tree batches take single trees, not forests");
    v[g] = view_of<T, D>(t);
    mt.depth = std::max(mt.depth, t->tdepth);
    mt.n_nodes = std::max(mt.n_nodes, t->n_tnodes);
    const int64_t m = rows[g + 1] - rows[g];
    if (m < 0) throw Error(E_INVALID, "query offsets must not decrease");
    so[g + 1] = so[g] + (m + 31) / 32 * 32;
  }
  mt.n_slots = so[ntrees];
  if (mt.n_slots > INT32_MAX) throw Error(E_INVALID, "batch too large for one pass");
  // every view uses the batch-wide stack bound (shared memory is sized once)
  for (auto& x : v) x.depth = mt.depth;
  const size_t nw = (size_t)std::max<int64_t>(mt.n_slots / 32, 1);
  auto up = [](size_t b) { return (b + 255) / 256 * 256; };
  const size_t o_views = 0, o_so = up(sizeof(TreeView<T, D>) * ntrees), o_ro = o_so + up(8 * (ntrees + 1)),
               o_wt = o_ro + up(8 * (ntrees + 1)), total = o_wt + up(4 * nw);
  std::vector<char> h(total, 0);
  memcpy(h.data() + o_views, v.data(), sizeof(TreeView<T, D>) * ntrees);
  memcpy(h.data() + o_so, so.data(), 8 * (ntrees + 1));
  memcpy(h.data() + o_ro, rows, 8 * (ntrees + 1));
  int* wt = reinterpret_cast<int*>(h.data() + o_wt);
  for (int g = 0; g < ntrees; g++)
    for (int64_t w = so[g] / 32; w < so[g + 1] / 32; w++) wt[w] = g;
  mt.blob.alloc(total, st);
  // pageable source: the call returns once the bytes are staged, so `h` may
  // go out of scope without a synchronisation
  PPTKG_CUDA(cudaMemcpyAsync(mt.blob.get(), h.data(), total, cudaMemcpyHostToDevice, st));
  mt.views = reinterpret_cast<const TreeView<T, D>*>(mt.blob.get() + o_views);
  mt.slot_off = reinterpret_cast<const int64_t*>(mt.blob.get() + o_so);
  mt.row_off = reinterpret_cast<const int64_t*>(mt.blob.get() + o_ro);
  mt.warp_tree = reinterpret_cast<const int*>(mt.blob.get() + o_wt);
}

// A stand-in tree carrying the batch-wide traversal bounds for the launch
// helpers (which size shared memory from the tree they are given).
static TreeBase* bounds_tree(int depth, int n_nodes) {
  TreeBase* b = new TreeBase();
  b->tdepth = depth;
  b->n_tnodes = n_nodes;
  return b;
}

static __global__ void k_order_rows(const int* local, int m, int base, int* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) out[i] = base + (local ? local[i] : i);
}

// Processing order of a multi-tree batch: each tree's queries sorted by
// tree position (as for a single tree) within that tree's rows, so a warp's
// queries are neighbours.  `spec(g)` gives the QuerySpec of group g.
template <typename T, int D, typename Spec>
void multi_order(const TreeBase* const* trees, int ntrees, const int64_t* rows, MultiTables<T, D>& mt, Spec spec,
                 cudaStream_t st, bool anchors = false) {
  const int64_t m_all = rows[ntrees];
  bool any = false;
  for (int g = 0; g < ntrees && !any; g++) any = rows[g + 1] - rows[g] >= 2048;
  if (!any && !anchors) return;
  if (anchors) mt.anchor.alloc(m_all, st);
  if (any) mt.order.alloc(m_all, st);
  for (int g = 0; g < ntrees; g++) {
    const int64_t m = rows[g + 1] - rows[g];
    if (m <= 0) continue;
    DevBuf<int> local;
    const int mode = make_order<T, D>(trees[g], spec(g), local, st, true, anchors ? mt.anchor.get() + rows[g] : nullptr);
    if (any) {
      k_order_rows<<<div_up(m, 256), 256, 0, st>>>(mode == 1 ? local.get() : nullptr, (int)m, (int)rows[g],
                                                   mt.order.get() + rows[g]);
      PPTKG_CHECK_LAUNCH();
    }
  }
  mt.ordered = any;
}

template <typename T, int D>
void multi_knn(const TreeBase* const* trees, int ntrees, const void* d_q, int qdtype, const int64_t* rows, int k,
               double dmax, int32_t* d_idx, int32_t* d_cnt, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k < 1) throw Error(E_INVALID, "k must be positive");
  if (k > KNN_MAX_K) throw Error(E_UNSUPPORTED, "k > 64 is not supported by the GPU kNN kernels");
  MultiTables<T, D> mt;
  multi_tables<T, D>(trees, ntrees, rows, mt, st);
  if (mt.n_slots == 0) return;
  const size_t qbytes = (qdtype == F64 ? sizeof(double) : sizeof(float)) * D;
  multi_order<T, D>(trees, ntrees, rows, mt, [&](int g) {
    QuerySpec qs;
    qs.pts = (const char*)d_q + rows[g] * qbytes;
    qs.qdtype = qdtype;
    qs.m = rows[g + 1] - rows[g];
    return qs;
  }, st, true);
  std::unique_ptr<TreeBase> bt(bounds_tree(mt.depth, mt.n_nodes));
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  const DistT r2 = radius2<DistT>(dmax);
  Stage stage("multi.knn", st);
  if (qdtype == F64)
    dispatch_knn<T, D>(bt.get(), PointQueries<double, D>{(const double*)d_q, mt.anchor.get()}, nullptr, 0,
                       (int)mt.n_slots, k, r2, d_idx, d_cnt, status.get(), st, mt.map());
  else
    dispatch_knn<T, D>(bt.get(), PointQueries<float, D>{(const float*)d_q, mt.anchor.get()}, nullptr, 0,
                       (int)mt.n_slots, k, r2, d_idx, d_cnt, status.get(), st, mt.map());
  check_status(status.get(), st, "multi-tree knn");
}

template <typename T>
void multi_normals(const TreeBase* const* trees, int ntrees, const int32_t* d_idx, const int64_t* rows, int k, float r,
                   int num_eigen, int precision, double gap_thr, T* d_evecs, T* d_evals, int32_t* d_sizes,
                   cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k < 1) throw Error(E_INVALID, "batched normals need k >= 1");
  if (k > KNN_MAX_K) throw Error(E_UNSUPPORTED, "k > 64 is not supported by the GPU normal kernels");
  MultiTables<T, 3> mt;
  multi_tables<T, 3>(trees, ntrees, rows, mt, st);
  if (mt.n_slots == 0) return;
  // query indices are checked against their own tree's rows by the kernels
  // (status 4); the ordering pass maps bad ones to the end of the order
  multi_order<T, 3>(trees, ntrees, rows, mt, [&](int g) {
    QuerySpec qs;
    qs.idx = d_idx + rows[g];
    qs.m = rows[g + 1] - rows[g];
    qs.exclude_self = false;
    return qs;
  }, st);
  std::unique_ptr<TreeBase> bt(bounds_tree(mt.depth, mt.n_nodes));
  DevBuf<int> status(1, st);
  PPTKG_CUDA(cudaMemsetAsync(status.get(), 0, sizeof(int), st));
  const DistT rr = (DistT)(T)r;
  const DistT r2 = rr * rr;
  int prec = precision == PREC_AUTO ? (sizeof(T) == 4 ? PREC_FP32 : PREC_FP64) : precision;
  Stage stage("multi.normals", st);
  // fwd comes from each warp's TreeView (null here)
  dispatch_normals<T, IndexQueries<3, false>>(bt.get(), IndexQueries<3, false>{d_idx, nullptr, status.get()}, nullptr,
                                              0, (int)mt.n_slots, k, r2, num_eigen, prec, gap_thr, d_evecs, d_evals,
                                              d_sizes, status.get(), st, mt.map());
  check_status(status.get(), st, "multi-tree normals");
}

#ifndef PPTKG_QUERY_DIM
template void multi_knn<float, 3>(const TreeBase* const*, int, const void*, int, const int64_t*, int, double, int32_t*,
                                  int32_t*, cudaStream_t);
template void multi_knn<double, 3>(const TreeBase* const*, int, const void*, int, const int64_t*, int, double,
                                   int32_t*, int32_t*, cudaStream_t);
template void multi_normals<float>(const TreeBase* const*, int, const int32_t*, const int64_t*, int, float, int, int,
                                   double, float*, float*, int32_t*, cudaStream_t);
template void multi_normals<double>(const TreeBase* const*, int, const int32_t*, const int64_t*, int, float, int, int,
                                    double, double*, double*, int32_t*, cudaStream_t);
#endif  // PPTKG_QUERY_DIM


#ifndef PPTKG_QUERY_DIM
// ------------------------------------------- allocation-free normals ----
// Scratch of pptkg_tree_normals_noalloc, resident on every GPU that loads the
// library: [0] status word, [1] FP64 re-solve queue length, then (from int 64,
// 256-byte aligned) the queue itself, NOALLOC_MAX_QUERIES entries of up to
// NOALLOC_MAX_K + 2 ints.  About 4.7 MB.
constexpr int NOALLOC_MAX_QUERIES = 65536;
constexpr int NOALLOC_MAX_K = 16;
constexpr int NOALLOC_QUEUE_OFFSET = 64;
static __device__ __align__(256) int g_noalloc_scratch[NOALLOC_QUEUE_OFFSET +
                                                       NOALLOC_MAX_QUERIES * (NOALLOC_MAX_K + 2)];

// Device address of the scratch array on the current device.  Host code
// cannot use the symbol itself (it names a host-side stand-in), so the
// address is looked up once per device with that device current.
static int* noalloc_scratch() {
  static std::mutex mu;
  static int* addr[64] = {};
  int dev = 0;
  PPTKG_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw Error(E_CUDA, "device ordinal out of range");
  std::lock_guard<std::mutex> g(mu);
  if (!addr[dev]) {
    int* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      throw Error(E_CUDA, std::string("cudaGetSymbolAddress(noalloc scratch): ") + cudaGetErrorString(e));
    addr[dev] = p;
  }
  return addr[dev];
}

template <typename T, int KMAX>
static void normals_noalloc_k(const TreeBase* t, const int32_t* idx, int m, int k, typename DistOf<T>::type r2,
                              int num_eigen, int prec, T* ev, T* ew, int32_t* sz, int* scratch, cudaStream_t st) {
  typedef IndexQueries<3, false> L;
  L ld{idx, t->fwd};
  const int mode = (!idx && m == t->nv && t->n == t->nv) ? 2 : 0;
  int* status = scratch;
  int* nfix = scratch + 1;
  int* fix = scratch + NOALLOC_QUEUE_OFFSET;
  if (prec == PREC_FP64) {
    launch_normals<T, KMAX, L, PREC_FP64>(t, ld, nullptr, mode, m, k, r2, num_eigen, 0.0, ev, ew, sz, nullptr,
                                          nullptr, status, st);
    return;
  }
  launch_normals<T, KMAX, L, PREC_FP32>(t, ld, nullptr, mode, m, k, r2, num_eigen, 1e-3, ev, ew, sz, fix, nfix,
                                        status, st);
  k_refine64<T, KMAX><<<div_up(m, 256), 256, 0, st>>>((const PointRec<T, 3>*)t->pts, fix, nfix, num_eigen, ev, ew,
                                                      sz, nullptr);
  PPTKG_CHECK_LAUNCH();
}

template <typename T>
void normals_noalloc(const TreeBase* t, const int32_t* d_idx, int64_t m, int k, float r, int num_eigen, int precision,
                     T* d_evecs, T* d_evals, int32_t* d_sizes, cudaStream_t st) {
  typedef typename DistOf<T>::type DistT;
  if (k < 1 || k > NOALLOC_MAX_K)
    throw Error(E_INVALID, "k must be in [1, " + std::to_string(NOALLOC_MAX_K) + "] for the allocation-free entry");
  if (m < 0 || m > NOALLOC_MAX_QUERIES)
    throw Error(E_INVALID, "query count " + std::to_string(m) + " exceeds the allocation-free limit of " +
                               std::to_string(NOALLOC_MAX_QUERIES));
  if (!d_idx && m > t->n) throw Error(E_RANGE, "query rows exceed the point count");
  int* scratch = noalloc_scratch();
  if (m == 0) return;
  // status and queue length start at zero; the queue itself needs no clearing
  PPTKG_CUDA(cudaMemsetAsync(scratch, 0, 2 * sizeof(int), st));
  int h = 0;
  if (d_idx) {
    k_check_idx<<<div_up(m, 256), 256, 0, st>>>(d_idx, (int)m, (int)t->n, scratch);
    PPTKG_CHECK_LAUNCH();
    PPTKG_CUDA(cudaMemcpyAsync(&h, scratch, sizeof(int), cudaMemcpyDeviceToHost, st));
    PPTKG_CUDA(cudaStreamSynchronize(st));
    if (h) throw Error(E_RANGE, "query index outside of [0, n)");
  }
  const DistT rr = (DistT)(T)r;
  const DistT r2 = rr * rr;
  int prec = precision == PREC_AUTO ? (sizeof(T) == 4 ? PREC_FP32 : PREC_FP64) : precision;
  const int mi = (int)m;
  if (k <= 4)
    normals_noalloc_k<T, 4>(t, d_idx, mi, k, r2, num_eigen, prec, d_evecs, d_evals, d_sizes, scratch, st);
  else if (k <= 8)
    normals_noalloc_k<T, 8>(t, d_idx, mi, k, r2, num_eigen, prec, d_evecs, d_evals, d_sizes, scratch, st);
  else
    normals_noalloc_k<T, 16>(t, d_idx, mi, k, r2, num_eigen, prec, d_evecs, d_evals, d_sizes, scratch, st);
  PPTKG_CUDA(cudaMemcpyAsync(&h, scratch, sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (h) throw Error(E_DEVICE, "normals (allocation-free): device traversal check failed (code " +
                                   std::to_string(h) + ")");
}

template void normals_noalloc<float>(const TreeBase*, const int32_t*, int64_t, int, float, int, int, float*, float*,
                                     int32_t*, cudaStream_t);
template void normals_noalloc<double>(const TreeBase*, const int32_t*, int64_t, int, float, int, int, double*,
                                      double*, int32_t*, cudaStream_t);

#endif  // PPTKG_QUERY_DIM

#define PPTKG_INST_Q(T, D)                                                                                 \
  template void knn_query<T, D>(const TreeBase*, const QuerySpec&, int, double, int32_t*, int32_t*,        \
                                cudaStream_t);                                                             \
  template int64_t rnear_count<T, D>(const TreeBase*, const QuerySpec&, double, int64_t*, cudaStream_t);   \
  template void rnear_fill<T, D>(const TreeBase*, const QuerySpec&, double, const int64_t*, int32_t*,      \
                                 cudaStream_t);

// This file builds the 3-d query paths and everything 3-d only (normals,
// forests, multi-tree batches, the allocation-free entry point).
// query_d2.cu / query_d4.cu include it with PPTKG_QUERY_DIM set and build
// only the kNN and r-near paths of that dimension, in parallel.
#ifndef PPTKG_QUERY_DIM
PPTKG_INST_Q(float, 3)
PPTKG_INST_Q(double, 3)

template void normals_query<float>(const TreeBase*, const QuerySpec&, int, float, int, int, double, float*, float*,
                                   int32_t*, cudaStream_t);
template void normals_query<double>(const TreeBase*, const QuerySpec&, int, float, int, int, double, double*, double*,
                                    int32_t*, cudaStream_t);
template void eigh3_batched<float>(const float*, int64_t, float*, float*, int, cudaStream_t);
template void eigh3_batched<double>(const double*, int64_t, double*, double*, int, cudaStream_t);
#else
PPTKG_INST_Q(float, PPTKG_QUERY_DIM)
PPTKG_INST_Q(double, PPTKG_QUERY_DIM)
#endif

}  // namespace pptkg

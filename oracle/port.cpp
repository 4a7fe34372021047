// Test infrastructure (oracle side): a CPU restatement of the reference's
// k-d tree and normal-estimation algorithms.  It is the checker that the
// GPU tests compare against; it is never linked into the product library,
// and the product never calls it.
//
// Every function cites the reference code it restates (paths relative to
// the pptk project).  Two semantics are deliberately pinned here, and the
// GPU path follows the same ones:
//  * kNN results are the k smallest (dist2, original index) pairs among the
//    points with dist2 < r^2, in that order: ties in distance are broken by
//    point index.  The reference keeps whichever equal-dist2 candidate its
//    std::priority_queue happens to keep (kdtree-impl.h:360-373, :894-899);
//    outside of exact distance ties the two agree, and the tests compare
//    against the reference after sorting each equal-dist2 run and allowing
//    the choice among points tied at the k-th distance.
//  * eigenvectors are signed so that their largest-magnitude component is
//    positive (Eigen's sign is an implementation artefact; the reference's
//    own test pins only +[1,0,0] on collinear input, which this convention
//    reproduces).
//
// Built by oracle/build_oracle.py into oracle/libpptk_port.so.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <type_traits>
#include <vector>

#include "common.h"

namespace {

using oracle::dispatch;
using oracle::dispatch_type;

// Distance arithmetic type: float for float32 and every integer type, double
// for float64 (accumulator.h:13-27).
template <typename T>
struct DistOf {
  typedef float type;
};
template <>
struct DistOf<double> {
  typedef double type;
};

template <typename T, int D>
struct Box {
  T lo[D], hi[D];
  // empty box as in Box::Reset (box.h:107-110)
  void reset() {
    for (int i = 0; i < D; i++) {
      lo[i] = std::numeric_limits<T>::max();
      hi[i] = std::numeric_limits<T>::lowest();
    }
  }
  // box.h:99-105 (std::min / std::max argument order kept)
  void add(const T* p) {
    for (int i = 0; i < D; i++) {
      lo[i] = std::min(p[i], lo[i]);
      hi[i] = std::max(p[i], hi[i]);
    }
  }
  bool is_point() const {  // box.h:112-121
    for (int i = 0; i < D; i++)
      if (lo[i] != hi[i]) return false;
    return true;
  }
};

// Squared distance from q to the nearest / farthest point of a box, per axis
// in DistT, summed in axis order from zero (box.h:157-198).
template <typename DistT, typename Q, typename T, int D>
DistT min_dist2(const Q* q, const Box<T, D>& b) {
  DistT s = (DistT)0.0;
  for (int i = 0; i < D; i++) {
    DistT a = (DistT)b.lo[i] - (DistT)q[i];
    DistT c = (DistT)b.hi[i] - (DistT)q[i];
    DistT v;
    if (a > (DistT)0.0)
      v = a * a;
    else if (c < (DistT)0.0)
      v = c * c;
    else
      v = (DistT)0.0;
    s += v;
  }
  return s;
}

template <typename DistT, typename Q, typename T, int D>
DistT max_dist2(const Q* q, const Box<T, D>& b) {
  DistT s = (DistT)0.0;
  for (int i = 0; i < D; i++) {
    DistT a = (DistT)b.lo[i] - (DistT)q[i];
    a = a * a;
    DistT c = (DistT)b.hi[i] - (DistT)q[i];
    c = c * c;
    s += std::max(a, c);
  }
  return s;
}

// Point-to-point squared distance (kdtree-impl.h:331-339): each axis
// difference (point - query) squared and added in axis order, no FMA.
template <typename DistT, typename Q, typename T, int D>
DistT point_dist2(const Q* q, const T* p) {
  DistT s = (DistT)0.0;
  for (int i = 0; i < D; i++) {
    DistT t = (DistT)p[i] - (DistT)q[i];
    s += t * t;
  }
  return s;
}

// midpoint() (kdtree-impl.h:160-173), unsigned and signed/float forms.
template <typename T>
typename std::enable_if<std::is_unsigned<T>::value, T>::type mid(T a, T b) {
  if (a < b) std::swap(a, b);
  return (a - b) / 2 + b;
}
template <typename T>
typename std::enable_if<!std::is_unsigned<T>::value, T>::type mid(T a, T b) {
  if ((a >= 0 && b >= 0) || (a < 0 && b < 0)) return (b - a) / (T)2 + a;
  return (a + b) / (T)2;
}

template <typename T, int D>
struct Tree {
  typedef typename DistOf<T>::type DistT;
  struct Node {
    int dim;
    int index;
    T value;
    int child[2];  // -1: none (leaf range / empty)
  };
  int64_t n_orig = 0;
  std::vector<int> rev;  // tree position -> original index
  std::vector<int> fwd;  // original index -> tree position, -1 if dropped
  std::vector<T> pts;    // tree-ordered AoS copy
  Box<T, D> root_box;
  std::vector<Node> nodes;  // preorder, empty-split (trim) nodes included
  int root = -1;
};

template <typename T, int D>
struct Builder {
  typedef Tree<T, D> TreeT;
  typedef typename TreeT::Node Node;
  const T* P;
  std::vector<int>& idx;
  int64_t n_orig;
  int max_leaf;
  double thr;
  std::vector<Node>& nodes;

  const T* at(int i) const { return P + (int64_t)idx[i] * D; }

  // Two-pass three-way partition of idx[b, b+count) about split value s
  // along axis d (kdtree-impl.h:192-246): first pass moves values < s to the
  // front with a pair of converging cursors, second pass does the same for
  // values <= s on the remainder; the split position follows the rule that
  // balances runs of values equal to s (:234-244).
  int partition(int b, int count, int d, T s) {
    int* a = &idx[b];
    auto v = [&](int i) { return P[(int64_t)a[i] * D + d]; };
    int lo = 0, hi = count - 1;
    while (true) {
      while (lo <= hi && v(lo) < s) ++lo;
      while (lo <= hi && v(hi) >= s) --hi;
      if (lo >= hi) break;
      std::swap(a[lo++], a[hi--]);
    }
    const int lim1 = lo;
    hi = count - 1;
    while (true) {
      while (lo <= hi && v(lo) <= s) ++lo;
      while (lo <= hi && v(hi) > s) --hi;
      if (lo >= hi) break;
      std::swap(a[lo++], a[hi--]);
    }
    const int lim2 = lo;
    int nl = count / 2;
    if (lim1 > count / 2)
      nl = lim1;
    else if (lim2 < count / 2)
      nl = lim2;
    if (lim1 == count && lim2 == 0) nl = count / 2;
    return nl;
  }

  void link(int parent, int child, int b) {
    // an empty split whose index is the range start has its empty side on
    // the left, so its only child hangs on the right (kdtree-impl.h:143-151)
    if (nodes[parent].index == b)
      nodes[parent].child[1] = child;
    else
      nodes[parent].child[0] = child;
  }

  // One subtree over idx[b, e) with loose extent `box` (MakeNode +
  // RecursiveBuildHelper, kdtree-impl.h:248-329).  Returns the id of its first
  // node, or -1 when the range is a plain leaf.
  int make(int b, int e, Box<T, D> box) {
    const int size = e - b;
    Box<T, D> tight = box;
    int head = -1, tail = -1;
    if ((int64_t)size != n_orig) {
      tight.reset();
      for (int i = b; i < e; i++) tight.add(at(i));
      // empty-space trimming (TrimEmptyGaps / LargestEmptyGap, :99-158)
      while (true) {
        int gdim = -1, gside = -1;
        double gsize = 0.0;
        for (int i = 0; i < D; i++) {
          double g = std::max(0.0, (double)box.hi[i] - (double)tight.hi[i]);
          if (g >= gsize) gdim = i, gside = 1, gsize = g;
          g = std::max(0.0, (double)tight.lo[i] - (double)box.lo[i]);
          if (g >= gsize) gdim = i, gside = 0, gsize = g;
        }
        if (gsize == 0.0) break;
        double width = (double)box.hi[gdim] - (double)box.lo[gdim];
        if (gsize / width <= thr) break;
        Node t;
        t.dim = gdim;
        t.child[0] = t.child[1] = -1;
        if (gside == 0) {
          t.value = tight.lo[gdim];
          t.index = b;
          box.lo[gdim] = t.value;
        } else {
          t.value = tight.hi[gdim];
          t.index = e;
          box.hi[gdim] = t.value;
        }
        int id = (int)nodes.size();
        nodes.push_back(t);
        if (tail >= 0)
          link(tail, id, b);
        else
          head = id;
        tail = id;
      }
    }
    if (!tight.is_point() && size > max_leaf) {
      // widest axis, the last one on ties (ComputeSplit, :175-190)
      int sd = 0;
      T sv = T();
      T maxw = (T)0;
      for (int i = 0; i < D; i++) {
        T w = tight.hi[i] - tight.lo[i];
        if (w >= maxw) {
          maxw = w;
          sd = i;
          sv = (tight.lo[i] == tight.hi[i]) ? tight.lo[i] : mid<T>(tight.lo[i], tight.hi[i]);
        }
      }
      int nl = partition(b, size, sd, sv);
      Node s;
      s.dim = sd;
      s.value = sv;
      s.index = b + nl;
      s.child[0] = s.child[1] = -1;
      int id = (int)nodes.size();
      nodes.push_back(s);
      if (tail >= 0)
        link(tail, id, b);
      else
        head = id;
      const int si = b + nl;
      if (b < si) {
        Box<T, D> lb = box;
        lb.hi[sd] = sv;
        int c = make(b, si, lb);
        nodes[id].child[0] = c;
      }
      if (si < e) {
        Box<T, D> rb = box;
        rb.lo[sd] = sv;
        int c = make(si, e, rb);
        nodes[id].child[1] = c;
      }
    }
    return head;
  }
};

// BuildTree (kdtree-impl.h:773-818): drop rows with a NaN/inf coordinate
// (floating types only, :53-75), bound the rest, build, then reorder.
template <typename T, int D>
Tree<T, D>* build(const T* P, int64_t n, int max_leaf, double thr) {
  Tree<T, D>* t = new Tree<T, D>();
  t->n_orig = n;
  std::vector<int> idx;
  for (int64_t i = 0; i < n; i++) {
    bool ok = true;
    if (std::is_floating_point<T>::value)
      for (int d = 0; d < D; d++) {
        double v = (double)P[i * D + d];
        if (std::isnan(v) || std::isinf(v)) ok = false;
      }
    if (ok) idx.push_back((int)i);
  }
  t->root_box.reset();
  for (int i : idx) t->root_box.add(P + (int64_t)i * D);
  Builder<T, D> bld{P, idx, n, max_leaf, thr, t->nodes};
  t->root = bld.make(0, (int)idx.size(), t->root_box);
  t->pts.resize(idx.size() * D);
  for (size_t i = 0; i < idx.size(); i++)
    for (int d = 0; d < D; d++) t->pts[i * D + d] = P[(int64_t)idx[i] * D + d];
  t->fwd.assign(n, -1);
  for (size_t i = 0; i < idx.size(); i++) t->fwd[idx[i]] = (int)i;
  t->rev = idx;
  return t;
}

// Sorted candidate list of (dist2, original index), at most k long.
template <typename DistT>
struct TopK {
  int k;
  std::vector<std::pair<DistT, int>> v;
  bool full() const { return (int)v.size() >= k; }
  DistT worst() const { return v.back().first; }
  void offer(DistT d, int id) {
    std::pair<DistT, int> c(d, id);
    if (full() && !(c < v.back())) return;
    auto it = std::upper_bound(v.begin(), v.end(), c);
    v.insert(it, c);
    if ((int)v.size() > k) v.pop_back();
  }
};

// Near-child-first depth-first kNN over the same tree and the same loose
// node extents as KNearestNeighborsHelper (kdtree-impl.h:348-429), with the
// far child visited while its box can still hold a candidate that ties or
// beats the current k-th (dist2, index).
template <typename T, int D, typename Q>
void knn_rec(const Tree<T, D>& t, int node, int b, int e, Box<T, D>& box, const Q* q,
             typename Tree<T, D>::DistT r2, TopK<typename Tree<T, D>::DistT>& top) {
  typedef typename Tree<T, D>::DistT DistT;
  if (node < 0) {
    for (int i = b; i < e; i++) {
      DistT d2 = point_dist2<DistT, Q, T, D>(q, &t.pts[(size_t)i * D]);
      if (d2 < r2) top.offer(d2, t.rev[i]);
    }
    return;
  }
  const auto& nd = t.nodes[node];
  const int sd = nd.dim;
  const int near = (q[sd] < nd.value) ? 0 : 1;
  const int rb[2] = {b, nd.index}, re[2] = {nd.index, e};
  for (int pass = 0; pass < 2; pass++) {
    const int c = pass == 0 ? near : 1 - near;
    if (rb[c] >= re[c]) continue;
    T saved = c == 0 ? box.hi[sd] : box.lo[sd];
    if (c == 0)
      box.hi[sd] = nd.value;
    else
      box.lo[sd] = nd.value;
    bool visit = true;
    if (pass == 1) {
      DistT md = min_dist2<DistT, Q, T, D>(q, box);
      visit = md < r2 && (!top.full() || md <= top.worst());
    }
    if (visit) knn_rec(t, nd.child[c], rb[c], re[c], box, q, r2, top);
    if (c == 0)
      box.hi[sd] = saved;
    else
      box.lo[sd] = saved;
  }
}

template <typename T, int D, typename Q>
void knn_one(const Tree<T, D>& t, const Q* q, int k, typename Tree<T, D>::DistT r,
             std::vector<std::pair<typename Tree<T, D>::DistT, int>>& out) {
  typedef typename Tree<T, D>::DistT DistT;
  out.clear();
  // KNearestNeighbors early outs (kdtree-impl.h:878-881)
  if (k < 1 || r < (DistT)0.0) return;
  Box<T, D> box = t.root_box;
  const DistT r2 = r * r;
  if (min_dist2<DistT, Q, T, D>(q, box) >= r2) return;
  // a NaN coordinate makes every distance NaN: no candidate qualifies
  TopK<DistT> top{k, {}};
  top.v.reserve(k + 1);
  knn_rec<T, D, Q>(t, t.root, 0, (int)t.rev.size(), box, q, r2, top);
  out = top.v;
}

// RNearNeighborsHelper (kdtree-impl.h:519-558): prune by the box's nearest
// distance, accept whole boxes inside the ball, test leaf points; left child
// before right child, so hits come out in ascending tree position.
template <typename T, int D, typename Q>
void rnear_rec(const Tree<T, D>& t, int node, int b, int e, Box<T, D>& box, const Q* q,
               typename Tree<T, D>::DistT r2, std::vector<int>& out) {
  typedef typename Tree<T, D>::DistT DistT;
  if (min_dist2<DistT, Q, T, D>(q, box) >= r2) return;
  if (max_dist2<DistT, Q, T, D>(q, box) < r2) {
    for (int i = b; i < e; i++) out.push_back(i);
    return;
  }
  if (node < 0) {
    for (int i = b; i < e; i++)
      if (point_dist2<DistT, Q, T, D>(q, &t.pts[(size_t)i * D]) < r2) out.push_back(i);
    return;
  }
  const auto& nd = t.nodes[node];
  const int sd = nd.dim;
  if (nd.index > b) {
    T s = box.hi[sd];
    box.hi[sd] = nd.value;
    rnear_rec(t, nd.child[0], b, nd.index, box, q, r2, out);
    box.hi[sd] = s;
  }
  if (nd.index < e) {
    T s = box.lo[sd];
    box.lo[sd] = nd.value;
    rnear_rec(t, nd.child[1], nd.index, e, box, q, r2, out);
    box.lo[sd] = s;
  }
}

template <typename T, int D, typename Q>
void rnear_one(const Tree<T, D>& t, const Q* q, typename Tree<T, D>::DistT r, std::vector<int>& out) {
  typedef typename Tree<T, D>::DistT DistT;
  out.clear();
  if (r < (DistT)0.0) return;  // kdtree-impl.h:982
  Box<T, D> box = t.root_box;
  rnear_rec<T, D, Q>(t, t.root, 0, (int)t.rev.size(), box, q, r * r, out);
}

struct Handle {
  void* tree;
  int dtype;
  int dim;
};

template <typename T, int D>
Tree<T, D>& tree_of(Handle* h) {
  return *(Tree<T, D>*)h->tree;
}

static int nthreads_or_max(int n) { return n > 0 ? n : omp_get_max_threads(); }

}  // namespace

extern "C" {

void* port_build(const void* pts, int64_t n, int dim, int dtype, int max_leaf_size, double empty_split) {
  Handle* h = new Handle{nullptr, dtype, dim};
  bool ok = dispatch(dtype, dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    h->tree = build<T, D>((const T*)pts, n, max_leaf_size, empty_split);
  });
  if (!ok) {
    delete h;
    return nullptr;
  }
  return h;
}

void port_free(void* hp) {
  Handle* h = (Handle*)hp;
  if (!h) return;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    delete (Tree<T, D>*)h->tree;
  });
  delete h;
}

int64_t port_num_valid(void* hp) {
  Handle* h = (Handle*)hp;
  int64_t r = 0;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    r = (int64_t)tree_of<decltype(t), decltype(d)::value>(h).rev.size();
  });
  return r;
}

void port_reverse_indices(void* hp, int32_t* out) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    const auto& v = tree_of<decltype(t), decltype(d)::value>(h).rev;
    std::copy(v.begin(), v.end(), out);
  });
}

// Tree-ordered point copy, as float64 (num_valid x dim).
void port_tree_points(void* hp, double* out) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    const auto& v = tree_of<decltype(t), decltype(d)::value>(h).pts;
    for (size_t i = 0; i < v.size(); i++) out[i] = (double)v[i];
  });
}

// Preorder node list in the same 5-double layout as ref_tree_nodes.
int64_t port_tree_nodes(void* hp, double* out) {
  Handle* h = (Handle*)hp;
  int64_t cnt = 0;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    const auto& tr = tree_of<decltype(t), decltype(d)::value>(h);
    cnt = (int64_t)tr.nodes.size();
    if (!out) return;
    for (size_t i = 0; i < tr.nodes.size(); i++) {
      const auto& nd = tr.nodes[i];
      out[i * 5 + 0] = nd.dim;
      out[i * 5 + 1] = nd.index;
      out[i * 5 + 2] = (double)nd.value;
      out[i * 5 + 3] = nd.child[0] >= 0 ? 1.0 : 0.0;
      out[i * 5 + 4] = nd.child[1] >= 0 ? 1.0 : 0.0;
    }
  });
  return cnt;
}

// kNN of m point queries (AoS of qdtype).  out_idx: m x k original indices,
// -1 padded; out_pos (optional): tree positions; out_d2 (optional): dist2.
void port_knn(void* hp, const void* q, int64_t m, int qdtype, int k, double dmax, int32_t* out_idx,
              int32_t* out_cnt, int32_t* out_pos, double* out_d2, int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    const auto& tr = tree_of<T, D>(h);
    typedef typename Tree<T, D>::DistT DistT;
    oracle::dispatch_query<T>(qdtype, h->dtype, [&](auto qt) {
      typedef decltype(qt) Q;
      const Q* qp = (const Q*)q;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads_or_max(nthreads))
      for (int64_t i = 0; i < m; i++) {
        std::vector<std::pair<DistT, int>> res;
        knn_one<T, D, Q>(tr, qp + i * D, k, (DistT)dmax, res);
        for (int j = 0; j < k; j++) {
          bool ok = j < (int)res.size();
          out_idx[i * k + j] = ok ? res[j].second : -1;
          if (out_pos) out_pos[i * k + j] = ok ? tr.fwd[res[j].second] : -1;
          if (out_d2) out_d2[i * k + j] = ok ? (double)res[j].first : -1.0;
        }
        out_cnt[i] = (int32_t)res.size();
      }
    });
  });
}

// Self queries by original index (KNearestNeighborsSelf, kdtree-impl.h:931-948):
// a dropped (NaN/inf) point has no neighbours; otherwise k+1 neighbours of
// its own coordinates, minus the query index itself, first k kept.
void port_knn_self(void* hp, const int32_t* qidx, int64_t m, int k, double dmax, int32_t* out_idx,
                   int32_t* out_cnt, int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    const auto& tr = tree_of<T, D>(h);
    typedef typename Tree<T, D>::DistT DistT;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads_or_max(nthreads))
    for (int64_t i = 0; i < m; i++) {
      int qi = qidx[i];
      int cnt = 0;
      if (tr.fwd[qi] >= 0) {
        std::vector<std::pair<DistT, int>> res;
        knn_one<T, D, T>(tr, &tr.pts[(size_t)tr.fwd[qi] * D], k + 1, (DistT)dmax, res);
        for (size_t j = 0; j < res.size() && cnt < k; j++) {
          int oi = res[j].second;
          if (oi != qi) out_idx[i * k + cnt++] = oi;
        }
      }
      for (int j = cnt; j < k; j++) out_idx[i * k + j] = -1;
      out_cnt[i] = cnt;
    }
  });
}

// r-near, two calls: out == NULL fills offsets (m + 1), then out is filled.
void port_rnear(void* hp, const void* q, int64_t m, int qdtype, double dmax, int64_t* offsets, int32_t* out,
                int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    const auto& tr = tree_of<T, D>(h);
    typedef typename Tree<T, D>::DistT DistT;
    oracle::dispatch_query<T>(qdtype, h->dtype, [&](auto qt) {
      typedef decltype(qt) Q;
      const Q* qp = (const Q*)q;
      std::vector<int64_t> cnt(m);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads_or_max(nthreads))
      for (int64_t i = 0; i < m; i++) {
        std::vector<int> res;
        rnear_one<T, D, Q>(tr, qp + i * D, (DistT)dmax, res);
        cnt[i] = (int64_t)res.size();
        if (out)
          for (size_t j = 0; j < res.size(); j++) out[offsets[i] + j] = tr.rev[res[j]];
      }
      if (!out) {
        offsets[0] = 0;
        for (int64_t i = 0; i < m; i++) offsets[i + 1] = offsets[i] + cnt[i];
      }
    });
  });
}

// RNearNeighborsSelf (kdtree-impl.h:1028-1043): own coordinates, own index removed.
void port_rnear_self(void* hp, const int32_t* qidx, int64_t m, double dmax, int64_t* offsets, int32_t* out,
                     int nthreads) {
  Handle* h = (Handle*)hp;
  dispatch(h->dtype, h->dim, [&](auto t, auto d) {
    typedef decltype(t) T;
    const int D = decltype(d)::value;
    const auto& tr = tree_of<T, D>(h);
    typedef typename Tree<T, D>::DistT DistT;
    std::vector<int64_t> cnt(m);
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads_or_max(nthreads))
    for (int64_t i = 0; i < m; i++) {
      int qi = qidx[i];
      std::vector<int> res, keep;
      if (tr.fwd[qi] >= 0) rnear_one<T, D, T>(tr, &tr.pts[(size_t)tr.fwd[qi] * D], (DistT)dmax, res);
      for (int p : res)
        if (tr.rev[p] != qi) keep.push_back(tr.rev[p]);
      cnt[i] = (int64_t)keep.size();
      if (out) std::copy(keep.begin(), keep.end(), out + offsets[i]);
    }
    if (!out) {
      offsets[0] = 0;
      for (int64_t i = 0; i < m; i++) offsets[i + 1] = offsets[i] + cnt[i];
    }
  });
}

// estimate_normals (estimate_normals.cpp:17-120) over the restated tree: for
// each query point (all points, or the subsample indices) take its k nearest
// neighbours including itself (or its r-near set when k == -1), mean-centre,
// C = X^T X / n in the input type, Jacobi eigensolve in the input type.
// nbr_idx (optional, m x k) receives the neighbourhoods for the FP64 oracle.
void port_estimate_normals(const void* pts, int64_t n, int dtype, int k, float r, const int32_t* sub, int64_t m,
                           int num_eigen, void* evecs, void* evals, int32_t* sizes, int32_t* nbr_idx,
                           int nthreads) {
  auto run = [&](auto tt) {
    typedef decltype(tt) T;
    const T* P = (const T*)pts;
    Tree<T, 3>* tr = build<T, 3>(P, n, 10, 0.2);
    typedef typename Tree<T, 3>::DistT DistT;
    const int64_t num = sub ? m : n;
    T* ev = (T*)evecs;
    T* ew = (T*)evals;
#pragma omp parallel for schedule(dynamic, 64) num_threads(nthreads_or_max(nthreads))
    for (int64_t i = 0; i < num; i++) {
      const int64_t src = sub ? sub[i] : i;
      const T* q = P + src * 3;
      std::vector<int> nb;
      if (k == -1) {
        std::vector<int> pos;
        rnear_one<T, 3, T>(*tr, q, (DistT)(T)r, pos);
        for (int p : pos) nb.push_back(tr->rev[p]);
      } else {
        std::vector<std::pair<DistT, int>> res;
        knn_one<T, 3, T>(*tr, q, k, (DistT)(T)r, res);
        for (auto& pr : res) nb.push_back(pr.second);
      }
      if (nbr_idx && k > 0)
        for (int j = 0; j < k; j++) nbr_idx[i * k + j] = j < (int)nb.size() ? nb[j] : -1;
      const size_t cnt = nb.size();
      T mean[3] = {0, 0, 0};
      for (size_t j = 0; j < cnt; j++)
        for (int c = 0; c < 3; c++) mean[c] += P[(int64_t)nb[j] * 3 + c];
      for (int c = 0; c < 3; c++) mean[c] /= (T)cnt;
      T C[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      for (size_t j = 0; j < cnt; j++) {
        T x[3];
        for (int c = 0; c < 3; c++) x[c] = P[(int64_t)nb[j] * 3 + c] - mean[c];
        for (int a = 0; a < 3; a++)
          for (int b = 0; b < 3; b++) C[a * 3 + b] += x[a] * x[b];
      }
      for (int a = 0; a < 9; a++) C[a] /= (T)cnt;
      T w[3], V[9];
      oracle::jacobi3<T>(C, w, V);
      if (ev) {
        if (num_eigen == 1)
          for (int c = 0; c < 3; c++) ev[i * 3 + c] = V[c * 3 + 0];
        else
          for (int e = 0; e < 3; e++)
            for (int c = 0; c < 3; c++) ev[i * 9 + e * 3 + c] = V[c * 3 + e];
      }
      if (ew) {
        if (num_eigen == 1)
          ew[i] = w[0];
        else
          for (int e = 0; e < 3; e++) ew[i * 3 + e] = w[e];
      }
      if (sizes) sizes[i] = (int32_t)cnt;
    }
    delete tr;
  };
  if (dtype == oracle::F32)
    run(float());
  else
    run(double());
}

// Batched symmetric 3x3 eigensolve in float32 or float64 (row-major inputs),
// eigenvalues ascending, eigenvectors as columns.
void port_eigh3(const void* A, int64_t m, int dtype, void* w, void* V) {
  auto run = [&](auto tt) {
    typedef decltype(tt) T;
    for (int64_t i = 0; i < m; i++) oracle::jacobi3<T>((const T*)A + i * 9, (T*)w + i * 3, (T*)V + i * 9);
  };
  if (dtype == oracle::F32)
    run(float());
  else
    run(double());
}

int port_max_threads() { return omp_get_max_threads(); }

}  // extern "C"

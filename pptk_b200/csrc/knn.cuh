// Warp-packet k-d tree traversal for kNN and r-near queries.
//
// A warp carries 32 queries that are close in tree order (queries are sorted
// by the tree position of the point or of the bucket they fall in), so the
// packet walks one shared path: each node is one broadcast load, the two
// children are tested per lane, and a child is entered when any lane can
// still improve its result there.  Leaf buckets are staged in shared memory
// with one coalesced 16 B load per lane and then read back as broadcasts.
//
// Distances follow the reference exactly (kdtree-impl.h:331-339): per-axis
// (point - query) in the distance type, squared, summed in axis order, each
// operation rounded separately.  Box distances use the same operations, so a
// box's nearest distance never exceeds the distance of a point inside it and
// pruning can never drop an answer.
#pragma once

#include "tree.cuh"

namespace pptkg {

// ------------------------------------------------------------- distances --
template <typename T, typename DistT, int D>
__device__ __forceinline__ DistT point_dist2(const T* p, const DistT* q) {
  DistT s = xmul(xsub((DistT)p[0], q[0]), xsub((DistT)p[0], q[0]));
#pragma unroll
  for (int d = 1; d < D; d++) {
    DistT t = xsub((DistT)p[d], q[d]);
    s = xadd(s, xmul(t, t));
  }
  return s;
}

template <typename T, typename DistT, int D>
__device__ __forceinline__ DistT box_min_dist2(const T* lo, const T* hi, const DistT* q) {
  DistT s = (DistT)0;
#pragma unroll
  for (int d = 0; d < D; d++) {
    DistT a = xsub((DistT)lo[d], q[d]);
    DistT c = xsub((DistT)hi[d], q[d]);
    DistT v = a > (DistT)0 ? xmul(a, a) : (c < (DistT)0 ? xmul(c, c) : (DistT)0);
    s = xadd(s, v);
  }
  return s;
}

template <typename T, typename DistT, int D>
__device__ __forceinline__ DistT box_max_dist2(const T* lo, const T* hi, const DistT* q) {
  DistT s = (DistT)0;
#pragma unroll
  for (int d = 0; d < D; d++) {
    DistT a = xsub((DistT)lo[d], q[d]);
    DistT c = xsub((DistT)hi[d], q[d]);
    a = xmul(a, a);
    c = xmul(c, c);
    s = xadd(s, a > c ? a : c);
  }
  return s;
}

// ---------------------------------------------------------------- top-k ---
// The k best (dist2, point id) pairs, held in registers in descending order
// so that the current k-th best is always slot 0.  The id is the point's
// original index, so among equal distances the smaller index wins -- both
// for the order of a result and for which point takes the k-th slot.  (The
// reference keeps whichever equal-distance candidate its std::priority_queue
// happens to retain, kdtree-impl.h:360-373, 894-899; an index order makes the
// answer a function of the input alone.)  KMAX is the compile time capacity;
// for a run-time k < KMAX the slots [k, KMAX) hold entries that compare below
// every candidate and never move.
template <int KMAX, typename DistT>
struct TopK;

// Bitonic sort of N 64-bit keys held in registers (fully unrolled), into
// descending (desc = true) or ascending order.
template <int N>
__device__ __forceinline__ void bitonic_sort(unsigned long long (&a)[N], bool desc) {
#pragma unroll
  for (int size = 2; size <= N; size <<= 1)
#pragma unroll
    for (int stride = size / 2; stride > 0; stride >>= 1)
#pragma unroll
      for (int i = 0; i < N; i++) {
        const int j = i ^ stride;
        if (j > i) {
          const unsigned long long x = a[i], y = a[j];
          // blocks alternate direction; the last stage (size == N) has the
          // requested one
          const bool up = ((i & size) != 0) == desc;
          const bool sw = up ? (x > y) : (x < y);
          a[i] = sw ? y : x;
          a[j] = sw ? x : y;
        }
      }
}

// float distances: (dist2 bits << 32 | id) packed into one 64-bit key;
// non-negative floats order like their bit patterns.
template <int KMAX>
struct TopK<KMAX, float> {
  static constexpr int CAP = KMAX;
  unsigned long long s[KMAX];
  unsigned long long lim;
  __device__ __forceinline__ void reset(int k, float r2) {
    lim = (unsigned long long)__float_as_uint(r2) << 32;
#pragma unroll
    for (int j = 0; j < KMAX; j++) s[j] = j < k ? lim : 0ull;
  }
  __device__ __forceinline__ float worst() const { return __uint_as_float((unsigned)(s[0] >> 32)); }
  __device__ __forceinline__ void offer(float d2, int id) {
    unsigned long long c = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
    if (c < s[0]) insert(c);
  }
  __device__ __forceinline__ void insert(unsigned long long c) {
#pragma unroll
    for (int j = 0; j < KMAX - 1; j++) {
      unsigned long long nx = s[j + 1];
      s[j] = nx > c ? nx : (s[j] > c ? c : s[j]);
    }
    s[KMAX - 1] = s[KMAX - 1] > c ? c : s[KMAX - 1];
  }
  // Lowers the bound of the k live slots to b, inclusively (distances equal
  // to b still enter): live keys above the seed key become the seed key,
  // which sorts after every real key of distance b, so the list stays
  // sorted.  Only valid when at least k real candidates with distance <= b
  // are in the list or will be offered, so that every seed key is pushed out
  // by the end of the search.
  __device__ __forceinline__ void seed(int k, float b, float) {
    const unsigned long long key = ((unsigned long long)__float_as_uint(b) << 32) | 0xffffffffull;
    if (!(b >= 0.f) || key >= lim) return;
#pragma unroll
    for (int j = 0; j < KMAX; j++)
      if (j < k && s[j] > key) s[j] = key;
  }
  __device__ __forceinline__ void reserve(int) {}
  __device__ __forceinline__ bool valid(int j) const { return s[j] < lim && (unsigned)s[j] != 0xffffffffu; }
  __device__ __forceinline__ int id(int j) const { return (int)(unsigned)(s[j] & 0xffffffffull); }
  // Slot j sorts before the key (0, id0) of a point at distance 0.
  __device__ __forceinline__ bool below_zero(int j, int id0) const {
    return s[j] < (unsigned long long)(unsigned)id0;
  }
  __device__ __forceinline__ float dist(int j) const { return __uint_as_float((unsigned)(s[j] >> 32)); }
  // Warm start (see warm_topk): slot j holds a real candidate, an empty
  // live slot (no candidate yet) or a dead slot (beyond k); sort_desc()
  // then restores the list order.
  __device__ __forceinline__ void set_real(int j, float d2, int id) {
    s[j] = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
  }
  __device__ __forceinline__ void set_empty(int j) { s[j] = lim; }
  __device__ __forceinline__ void set_dead(int j) { s[j] = 0ull; }
  __device__ __forceinline__ void sort_desc() { bitonic_sort<KMAX>(s, true); }
  // The KMAX smallest of this list (sorted descending) and t (Q <= KMAX
  // keys sorted ascending, read as padded with keys above every list key),
  // sorted descending: the element-wise minimum of the two is a bitonic
  // sequence holding them, and a bitonic merge sorts it.
  template <int Q>
  __device__ __forceinline__ void merge_smallest(const unsigned long long (&t)[Q]) {
    static_assert(Q <= KMAX, "merge of at most KMAX keys");
#pragma unroll
    for (int j = 0; j < Q; j++) s[j] = t[j] < s[j] ? t[j] : s[j];
#pragma unroll
    for (int stride = KMAX / 2; stride > 0; stride >>= 1)
#pragma unroll
      for (int i = 0; i < KMAX; i++) {
        const int j = i ^ stride;
        if (j > i) {
          const unsigned long long x = s[i], y = s[j];
          const bool sw = x < y;
          s[i] = sw ? y : x;
          s[j] = sw ? x : y;
        }
      }
  }
  __device__ __forceinline__ unsigned long long key_real(float d2, int id) const {
    return ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)id;
  }
  __device__ __forceinline__ unsigned long long key_empty() const { return lim; }
};

// double distances: parallel (dist2, id) arrays compared lexicographically.
template <int KMAX>
struct TopK<KMAX, double> {
  static constexpr int CAP = KMAX;
  double d[KMAX];
  int p[KMAX];
  double lim_d;
  __device__ __forceinline__ void reset(int k, double r2) {
    lim_d = r2;
#pragma unroll
    for (int j = 0; j < KMAX; j++) {
      d[j] = j < k ? r2 : -1.0;
      p[j] = -1;
    }
  }
  __device__ __forceinline__ double worst() const { return d[0]; }
  __device__ __forceinline__ static bool gt(double da, int pa, double db, int pb) {
    return da > db || (da == db && pa > pb);
  }
  __device__ __forceinline__ void offer(double d2, int id) {
    if (gt(d[0], p[0], d2, id)) insert(d2, id);
  }
  __device__ __forceinline__ void insert(double cd, int cp) {
#pragma unroll
    for (int j = 0; j < KMAX - 1; j++) {
      const bool nx = gt(d[j + 1], p[j + 1], cd, cp);
      const bool cur = gt(d[j], p[j], cd, cp);
      d[j] = nx ? d[j + 1] : (cur ? cd : d[j]);
      p[j] = nx ? p[j + 1] : (cur ? cp : p[j]);
    }
    if (gt(d[KMAX - 1], p[KMAX - 1], cd, cp)) {
      d[KMAX - 1] = cd;
      p[KMAX - 1] = cp;
    }
  }
  // As TopK<KMAX, float>::seed; r2 is the bound the slots were reset to.
  __device__ __forceinline__ void seed(int k, double b, double r2) {
    if (!(b >= 0.0) || !(b < r2)) return;
#pragma unroll
    for (int j = 0; j < KMAX; j++)
      if (j < k && gt(d[j], p[j], b, 0x7fffffff)) {
        d[j] = b;
        p[j] = 0x7fffffff;
      }
  }
  __device__ __forceinline__ void reserve(int) {}
  __device__ __forceinline__ bool valid(int j) const { return p[j] >= 0 && p[j] != 0x7fffffff && d[j] >= 0.0; }
  __device__ __forceinline__ int id(int j) const { return p[j]; }
  __device__ __forceinline__ bool below_zero(int j, int id0) const { return d[j] == 0.0 && p[j] < id0; }
  __device__ __forceinline__ double dist(int j) const { return d[j]; }
  __device__ __forceinline__ void set_real(int j, double d2, int id) {
    d[j] = d2;
    p[j] = id;
  }
  __device__ __forceinline__ void set_empty(int j) {
    d[j] = lim_d;
    p[j] = -1;
  }
  __device__ __forceinline__ void set_dead(int j) {
    d[j] = -1.0;
    p[j] = -1;
  }
  __device__ __forceinline__ void sort_desc() {
#pragma unroll
    for (int size = 2; size <= KMAX; size <<= 1)
#pragma unroll
      for (int stride = size / 2; stride > 0; stride >>= 1)
#pragma unroll
        for (int i = 0; i < KMAX; i++) {
          const int j = i ^ stride;
          if (j > i) {
            const double da = d[i], db = d[j];
            const int pa = p[i], pb = p[j];
            const bool up = (i & size) != 0;
            const bool sw = up ? gt(da, pa, db, pb) : gt(db, pb, da, pa);
            d[i] = sw ? db : da;
            d[j] = sw ? da : db;
            p[i] = sw ? pb : pa;
            p[j] = sw ? pa : pb;
          }
        }
  }
};

// ----------------------------------------------------- packet traversal --
// Per-warp shared memory: the traversal stack and one leaf staging buffer.
template <typename T, int D>
struct WarpScratch {
  int* stack;
  PointRec<T, D>* buf;                   // 32 entries (r-near staging)
  int* log;                              // per-lane neighbour lists, lane-strided; null when unused
  typename DistOf<T>::type* dmat;        // 32 x 33 distances (kNN bucket scan); null when unused
  int* cid;                              // 32 candidate ids of the chunk being scanned (kNN)
};

// A lane's query as the rest of its warp reads it during a bucket scan:
// the coordinates and the entry bound (a candidate enters the list iff its
// dist2 <= thr).
template <typename DistT, int D>
struct alignas(16) QStage {
  DistT q[D];
  DistT thr;
};

// The largest value below r2 (r2 > 0), -1 for r2 <= 0, so that for every
// distance d2 >= 0: d2 < r2  <=>  d2 <= below(r2).
__device__ __forceinline__ float below(float r2) {
  if (!(r2 > 0.f)) return -1.f;
  return __uint_as_float(__float_as_uint(r2) - 1u);  // +inf -> FLT_MAX
}
__device__ __forceinline__ double below(double r2) {
  if (!(r2 > 0.0)) return -1.0;
  return __longlong_as_double(__double_as_longlong(r2) - 1ll);  // +inf -> DBL_MAX
}

// Entry bound of a list whose k-th distance is `worst` (worst <= r2 always):
// d2 <= entry_bound  <=>  d2 <= worst && d2 < r2.
template <typename DistT>
__device__ __forceinline__ DistT entry_bound(DistT worst, DistT r2_below) {
  return worst < r2_below ? worst : r2_below;
}

// One deferred child on the per-warp traversal stack: its box travels with
// it, so a pop re-tests the box from shared memory without touching the node
// array.  ref >= 0: inner node; ref < 0: leaf bucket starting at -ref - 1.
template <typename T, int D>
struct StackEnt {
  T lo[D], hi[D];
  int ref, cnt;
};

template <typename T, int D>
__device__ __forceinline__ TNode<T, D> load_node(const TNode<T, D>* nodes, int i) {
  static_assert(sizeof(TNode<T, D>) % 16 == 0, "TNode must be a multiple of 16 bytes");
  TNode<T, D> n;
  const float4* src = reinterpret_cast<const float4*>(nodes + i);
  float4* dst = reinterpret_cast<float4*>(&n);
#pragma unroll
  for (int j = 0; j < (int)(sizeof(TNode<T, D>) / 16); j++) dst[j] = __ldg(src + j);
  return n;
}

// Bits [a, a + n) of a 32-bit chunk mask (clipped to the chunk; 0 if empty).
__device__ __forceinline__ unsigned window_bits(int a, int n) {
  const int lo = max(a, 0), hi = min(a + n, 32);
  if (hi <= lo) return 0u;
  const unsigned top = hi >= 32 ? 0xffffffffu : ((1u << hi) - 1u);
  return top & ~((1u << lo) - 1u);
}

// The packet traversal shared by the kNN walks: near child first by majority
// vote, a child entered when any lane needs it (need(md): the lane's query
// can still improve from a box at squared distance md), leaf buckets handed
// to scan(begin, count, mine) warp-uniformly.  Returns false when the
// traversal stack would overflow (the host sizes it from the tree depth, so
// this is a safety net that reports instead of corrupting memory) or the
// node array is corrupt.
//
// The walk hides the latency of the dependent node loads: the node to
// descend into is loaded before the sibling bucket is scanned, and deferred
// children carry their boxes on the stack.
template <typename T, int D, typename DistT, typename Need, typename Scan>
__device__ __forceinline__ bool packet_walk(const TreeView<T, D>& tv, const DistT* q, bool active,
                                            WarpScratch<T, D> ws, Need need, Scan scan) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  StackEnt<T, D>* stk = reinterpret_cast<StackEnt<T, D>*>(ws.stack);
  int sp = 0;
  bool ok = true;
  int visits = 0;
  auto push = [&](const T* lo, const T* hi, int ref, int cnt) {
    if (sp >= tv.depth) {
      ok = false;
      return;
    }
    __syncwarp();
    if (lane == 0) {
      StackEnt<T, D> e;
#pragma unroll
      for (int d = 0; d < D; d++) {
        e.lo[d] = lo[d];
        e.hi[d] = hi[d];
      }
      e.ref = ref;
      e.cnt = cnt;
      stk[sp] = e;
    }
    sp++;
  };
  TNode<T, D> nd = load_node(tv.nodes, tv.node_index(tv.root));
  while (true) {
    if (++visits > tv.n_nodes) {  // a tree is acyclic: more visits mean a corrupt node array
      ok = false;
      break;
    }
    DistT md[2];
    md[0] = nd.cnt[0] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[0], nd.hi[0], q) : (DistT)INFINITY;
    md[1] = nd.cnt[1] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], q) : (DistT)INFINITY;
    // near child first, by majority vote; children unpacked with selects
    // (no run-time register indexing)
    const bool sw = __popc(__ballot_sync(FULL, active && md[1] < md[0])) > __popc(__ballot_sync(FULL, active)) / 2;
    const DistT md0 = sw ? md[1] : md[0], md1 = sw ? md[0] : md[1];
    const int ref0 = sw ? nd.ref[1] : nd.ref[0], ref1 = sw ? nd.ref[0] : nd.ref[1];
    const int cnt0 = sw ? nd.cnt[1] : nd.cnt[0], cnt1 = sw ? nd.cnt[0] : nd.cnt[1];
    const bool m0 = need(md0);
    const bool a0 = __any_sync(FULL, m0);
    const bool a1 = __any_sync(FULL, need(md1));
    int next = -1;
    TNode<T, D> nn;
    if (a0 && ref0 >= 0) {
      // near child is an inner node: fetch it now, defer the far child
      next = ref0;
      nn = load_node(tv.nodes, tv.node_index(next));
      if (a1) {
        T lo1[D], hi1[D];
#pragma unroll
        for (int d = 0; d < D; d++) {
          lo1[d] = sw ? nd.lo[0][d] : nd.lo[1][d];
          hi1[d] = sw ? nd.hi[0][d] : nd.hi[1][d];
        }
        push(lo1, hi1, ref1, cnt1);
      }
    } else {
      if (a1 && ref1 >= 0) {
        // far child is an inner node: its fetch overlaps the near bucket scan
        next = ref1;
        nn = load_node(tv.nodes, tv.node_index(next));
      }
      if (a0) scan(-ref0 - 1, cnt0, m0);
      const bool m1 = need(md1);  // re-test against the tightened threshold
      if (!__any_sync(FULL, m1)) {
        next = -1;
      } else if (ref1 < 0) {
        scan(-ref1 - 1, cnt1, m1);
      }
    }
    if (next >= 0) {
      nd = nn;
      continue;
    }
    __syncwarp();
    bool found = false;
    while (sp > 0) {
      --sp;
      const StackEnt<T, D> e = stk[sp];
      __syncwarp();
      const bool me = need(box_min_dist2<T, DistT, D>(e.lo, e.hi, q));
      if (!__any_sync(FULL, me)) continue;
      if (e.ref < 0) {
        scan(-e.ref - 1, e.cnt, me);
        continue;
      }
      nd = load_node(tv.nodes, tv.node_index(e.ref));
      found = true;
      break;
    }
    __syncwarp();
    if (!found) break;
  }
  return ok;
}

// Exact kNN of the lane's query over the whole tree, ties in dist2 broken by
// point id, with the top-k list in the lane's registers.  `own` (tree
// position or -1) is skipped, which is how self queries exclude the query
// point itself; so are the tree positions [wlo, wlo + wn), the warm-start
// window whose candidates the list holds.
template <typename T, int D, typename Top, typename DistT>
__device__ bool packet_knn(const TreeView<T, D>& tv, const DistT* q, int own, bool active, DistT r2, Top& top,
                           WarpScratch<T, D> ws, int wlo = 0, int wn = 0) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  auto need = [&](DistT md) { return active && md < r2 && md <= top.worst(); };
  // Leaf bucket scan, transposed: lane j holds candidate j of the chunk
  // (one coalesced 16 B load), and the warp loops only over the lanes whose
  // query needs this bucket.  For such a query i every lane computes its
  // candidate's distance to q_i; the row goes to dmat[i][*] and the ballot of
  // candidates that can enter list i becomes lane i's mark mask.  Each lane
  // then inserts its marked candidates, reading distances from its row and
  // the candidates' ids from the chunk's id row.
  // The queries sit in the warp's staging buffer (unused by kNN walks) so
  // that lane i's coordinates and bound arrive as one shared broadcast.
  QStage<DistT, D>* qst = reinterpret_cast<QStage<DistT, D>*>(ws.buf);
  const DistT r2_below = below(r2);
#pragma unroll
  for (int d = 0; d < D; d++) qst[lane].q[d] = q[d];
  auto scan = [&](int begin, int count, bool mine) {
    const unsigned needm = __ballot_sync(FULL, mine);
    for (int base = begin; base < begin + count; base += 32) {
      const int nb = min(32, begin + count - base);
      PointRec<T, D> pr;
      if (lane < nb) {
        pr = tv.pt(base + lane);
      } else {
#pragma unroll
        for (int d = 0; d < D; d++) pr.c[d] = (T)0;
        pr.id = -1;
      }
      // each needing lane publishes its entry bound for this chunk; the
      // loop below reads a query and its bound as one broadcast
      __syncwarp();
      qst[lane].thr = entry_bound(top.worst(), r2_below);
      ws.cid[lane] = pr.id;
      __syncwarp();
      const unsigned valid = nb == 32 ? FULL : (1u << nb) - 1u;
      unsigned mark = 0;
      unsigned rem = needm;
      while (rem) {
        const int i = __ffs(rem) - 1;
        rem &= rem - 1;
        const QStage<DistT, D> qi = qst[i];
        const DistT d2 = point_dist2<T, DistT, D>(pr.c, qi.q);
        ws.dmat[i * 33 + lane] = d2;
        const unsigned m = __ballot_sync(FULL, d2 <= qi.thr) & valid;
        if (lane == i) mark = m;
      }
      // the query's own point never enters its list, and the positions of
      // its warm-start window are in it already
      if (own >= base && own < base + nb) mark &= ~(1u << (own - base));
      mark &= ~window_bits(wlo - base, wn);
      __syncwarp();
      top.reserve(__popc(mark));
      while (mark) {
        const int t = __ffs(mark) - 1;
        mark &= mark - 1;
        top.offer(ws.dmat[lane * 33 + t], ws.cid[t]);
      }
      __syncwarp();
    }
  };
  return packet_walk<T, D, DistT>(tv, q, active, ws, need, scan);
}

// Per-lane traversal for warps whose queries lie far apart, where a packet
// walk would visit the union of 32 unrelated paths one node at a time.  Each
// lane walks its own near-first depth-first path with a private stack of
// deferred children (reference, size and box distance, re-tested on pop), so
// the 32 walks advance side by side and their node loads overlap.  The set of
// candidates each query accepts is the same as in the packet walk: every
// point whose distance is within the query's final bound is offered, so the
// result (the k smallest (dist2, id) pairs) is identical.
// Requires tv.depth <= LSTACK (the caller checks); false on a corrupt tree.
template <int LSTACK, typename T, int D, typename DistT, typename Top>
__device__ bool lane_knn(const TreeView<T, D>& tv, const DistT* q, int own, bool active, DistT r2, Top& top,
                         int wlo = 0, int wn = 0) {
  if (!active) return true;
  int sref[LSTACK], scnt[LSTACK];
  DistT smd[LSTACK];
  int sp = 0;
  auto need = [&](DistT md) { return md < r2 && md <= top.worst(); };
  // a bucket is read four points at a time so that the loads overlap; the
  // offers then go in position order against the current bound, as one by one
  auto scan = [&](int begin, int count) {
    const int end = begin + count;
    int p = begin;
    for (; p + 4 <= end; p += 4) {
      PointRec<T, D> r[4];
      DistT d2[4];
#pragma unroll
      for (int j = 0; j < 4; j++) {
        r[j] = tv.pt(p + j);
        d2[j] = point_dist2<T, DistT, D>(r[j].c, q);
      }
#pragma unroll
      for (int j = 0; j < 4; j++)
        if (d2[j] <= top.worst() && d2[j] < r2 && p + j != own && (unsigned)(p + j - wlo) >= (unsigned)wn)
          top.offer(d2[j], r[j].id);
    }
    for (; p < end; p++) {
      const PointRec<T, D> r = tv.pt(p);
      const DistT d2 = point_dist2<T, DistT, D>(r.c, q);
      if (d2 <= top.worst() && d2 < r2 && p != own && (unsigned)(p - wlo) >= (unsigned)wn) top.offer(d2, r.id);
    }
  };
  int cur = tv.root, visits = 0;
  while (true) {
    if (++visits > tv.n_nodes) return false;  // a tree is acyclic: more visits mean a corrupt node array
    const TNode<T, D> nd = load_node(tv.nodes, tv.node_index(cur));
    const DistT md0 = nd.cnt[0] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[0], nd.hi[0], q) : (DistT)INFINITY;
    const DistT md1 = nd.cnt[1] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], q) : (DistT)INFINITY;
    const bool sw = md1 < md0;
    const DistT mdn = sw ? md1 : md0, mdf = sw ? md0 : md1;
    const int refn = sw ? nd.ref[1] : nd.ref[0], reff = sw ? nd.ref[0] : nd.ref[1];
    const int cntn = sw ? nd.cnt[1] : nd.cnt[0], cntf = sw ? nd.cnt[0] : nd.cnt[1];
    int next = -1;
    // the far child is never nearer than the near one, so it is needed only
    // when the near one is
    if (need(mdn)) {
      if (refn >= 0) {
        next = refn;
        if (need(mdf)) {
          if (sp >= LSTACK) return false;
          sref[sp] = reff;
          scnt[sp] = cntf;
          smd[sp] = mdf;
          sp++;
        }
      } else {
        scan(-refn - 1, cntn);
        if (need(mdf)) {
          if (reff >= 0)
            next = reff;
          else
            scan(-reff - 1, cntf);
        }
      }
    }
    while (next < 0 && sp > 0) {
      --sp;
      if (!need(smd[sp])) continue;
      if (sref[sp] < 0)
        scan(-sref[sp] - 1, scnt[sp]);
      else
        next = sref[sp];
    }
    if (next < 0) return true;
    cur = next;
  }
}

// Top-k of any size k for the per-lane walk: a binary max-heap of
// (dist2, id) pairs in device memory, ordered like the register lists
// ((dist2, id) lexicographic), so the k kept are the same k smallest.
// Slot 0 holds the current k-th once the heap is full.
template <typename DistT>
struct HeapTop {
  DistT* d;
  int* p;
  int k, size;
  DistT r2;
  __device__ __forceinline__ static bool gt(DistT da, int pa, DistT db, int pb) {
    return da > db || (da == db && pa > pb);
  }
  __device__ __forceinline__ DistT worst() const { return size < k ? r2 : d[0]; }
  __device__ void sift_down(int i, int n) {
    const DistT di = d[i];
    const int pi = p[i];
    while (true) {
      int c = 2 * i + 1;
      if (c >= n) break;
      if (c + 1 < n && gt(d[c + 1], p[c + 1], d[c], p[c])) c++;
      if (!gt(d[c], p[c], di, pi)) break;
      d[i] = d[c];
      p[i] = p[c];
      i = c;
    }
    d[i] = di;
    p[i] = pi;
  }
  __device__ void offer(DistT d2, int id) {
    if (size < k) {
      int i = size++;
      while (i > 0) {
        const int par = (i - 1) / 2;
        if (!gt(d2, id, d[par], p[par])) break;
        d[i] = d[par];
        p[i] = p[par];
        i = par;
      }
      d[i] = d2;
      p[i] = id;
    } else if (gt(d[0], p[0], d2, id)) {
      d[0] = d2;
      p[0] = id;
      sift_down(0, size);
    }
  }
  // Sorts the kept pairs ascending in place (heap sort).
  __device__ void sort() {
    for (int e = size - 1; e > 0; e--) {
      const DistT td = d[0];
      const int tp = p[0];
      d[0] = d[e];
      p[0] = p[e];
      d[e] = td;
      p[e] = tp;
      sift_down(0, e);
    }
  }
};

// Warp-uniform choice of the traversal: per-lane walks when the warp's
// queries span more than `span` tree positions (anchors: tree positions near
// each query; -1 unknown), packet walks otherwise.
template <int LSTACK>
__device__ __forceinline__ bool use_lane_walk(int anchor, bool active, int span, int depth) {
  const unsigned FULL = 0xffffffffu;
  const bool known = active && anchor >= 0;
  const int lo = __reduce_min_sync(FULL, known ? anchor : 0x7fffffff);
  const int hi = __reduce_max_sync(FULL, known ? anchor : -1);
  return span >= 0 && depth <= LSTACK && hi > lo && hi - lo > span;
}

// r-near over the whole tree in ascending tree position (the reference's
// left-then-right order, kdtree-impl.h:519-558).  In COUNT mode a lane whose
// ball contains a whole child box adds the child's size without distance
// tests (every point of the box is provably inside, see box_max_dist2);
// otherwise every point with dist2 < r2 is passed to emit(pos) in ascending
// position.  The own position is not excluded here: for self queries the
// caller subtracts it (it is always a hit when r2 > 0).
template <typename T, int D, typename DistT, bool COUNT, typename Emit>
__device__ bool packet_rnear(const TreeView<T, D>& tv, const DistT* q, bool active, DistT r2, WarpScratch<T, D> ws,
                             long long& count, Emit emit) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  int sp = 0;
  int cur = tv.root;
  bool ok = true;
  auto scan = [&](int begin, int cnt, bool mine) {
    for (int base = begin; base < begin + cnt; base += 32) {
      const int nb = min(32, begin + cnt - base);
      __syncwarp();
      if (lane < nb) ws.buf[lane] = tv.pt(base + lane);
      __syncwarp();
      if (mine) {
        for (int t = 0; t < nb; t++) {
          const PointRec<T, D> pr = ws.buf[t];
          const DistT d2 = point_dist2<T, DistT, D>(pr.c, q);
          if (d2 < r2) {
            if (COUNT)
              count++;
            else
              emit(base + t, pr);
          }
        }
      }
    }
  };
  // A lane that counted a whole inner child is muted while the warp walks
  // that child's subtree for other lanes: `mute` is the stack depth at which
  // the subtree was entered, and the lane rejoins once a pop goes below it.
  int mute = -1;
  auto live = [&]() { return active && mute < 0; };
  // Handles child c of nd; returns the node to descend into, or -1.
  auto process = [&](const TNode<T, D>& nd, int c, bool& took) -> int {
    took = false;
    if (nd.cnt[c] == 0) return -1;
    bool mine = live() && box_min_dist2<T, DistT, D>(nd.lo[c], nd.hi[c], q) < r2;
    if (COUNT && mine && box_max_dist2<T, DistT, D>(nd.lo[c], nd.hi[c], q) < r2) {
      count += nd.cnt[c];
      mine = false;
      took = true;
    }
    if (!__any_sync(FULL, mine)) return -1;
    const int ref = nd.ref[c];
    if (ref < 0) {
      scan(-ref - 1, nd.cnt[c], mine);
      return -1;
    }
    return ref;
  };
  int visits = 0;
  while (true) {
    if (++visits > tv.n_nodes) {
      ok = false;
      break;
    }
    const TNode<T, D>& nd = tv.nodes[cur];
    const bool w0 = live() && nd.cnt[0] > 0 && box_min_dist2<T, DistT, D>(nd.lo[0], nd.hi[0], q) < r2;
    const bool w1 = live() && nd.cnt[1] > 0 && box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], q) < r2;
    const bool a0 = __any_sync(FULL, w0), a1 = __any_sync(FULL, w1);
    int next = -1;
    bool took = false;
    if (a0) {
      next = process(nd, 0, took);
      if (next >= 0 && a1) {
        if (sp >= tv.depth) {
          ok = false;
        } else {
          __syncwarp();
          if (lane == 0) ws.stack[sp] = (cur << 1) | 1;
          sp++;
        }
      }
    }
    if (next < 0 && a1) next = process(nd, 1, took);
    if (next >= 0) {
      if (took) mute = sp;
      cur = next;
      continue;
    }
    __syncwarp();
    bool found = false;
    while (sp > 0) {
      const int e = ws.stack[--sp];
      __syncwarp();
      if (mute >= 0 && sp < mute) mute = -1;
      const int r = process(tv.nodes[e >> 1], e & 1, took);
      if (r >= 0) {
        if (took) mute = sp;
        cur = r;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  return ok;
}

}  // namespace pptkg

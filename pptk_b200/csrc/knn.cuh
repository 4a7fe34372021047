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
// The k best (dist2, tree position) pairs, held in registers in descending
// order so that the current k-th best is always slot 0.  KMAX is the compile
// time capacity; for a run-time k < KMAX the slots [k, KMAX) hold entries
// that compare below every candidate and never move.
template <int KMAX, typename DistT>
struct TopK;

// float distances: (dist2 bits << 32 | position) packed into one 64-bit key;
// non-negative floats order like their bit patterns.
template <int KMAX>
struct TopK<KMAX, float> {
  unsigned long long s[KMAX];
  unsigned long long lim;
  __device__ __forceinline__ void reset(int k, float r2) {
    lim = (unsigned long long)__float_as_uint(r2) << 32;
#pragma unroll
    for (int j = 0; j < KMAX; j++) s[j] = j < k ? lim : 0ull;
  }
  __device__ __forceinline__ float worst() const { return __uint_as_float((unsigned)(s[0] >> 32)); }
  __device__ __forceinline__ void offer(float d2, int pos) {
    unsigned long long c = ((unsigned long long)__float_as_uint(d2) << 32) | (unsigned)pos;
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
  __device__ __forceinline__ bool valid(int j) const { return s[j] < lim; }
  __device__ __forceinline__ int pos(int j) const { return (int)(unsigned)(s[j] & 0xffffffffull); }
  __device__ __forceinline__ float dist(int j) const { return __uint_as_float((unsigned)(s[j] >> 32)); }
};

// double distances: parallel (dist2, position) arrays compared lexicographically.
template <int KMAX>
struct TopK<KMAX, double> {
  double d[KMAX];
  int p[KMAX];
  __device__ __forceinline__ void reset(int k, double r2) {
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
  __device__ __forceinline__ void offer(double d2, int pos) {
    if (gt(d[0], p[0], d2, pos)) insert(d2, pos);
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
  __device__ __forceinline__ bool valid(int j) const { return p[j] >= 0 && d[j] >= 0.0; }
  __device__ __forceinline__ int pos(int j) const { return p[j]; }
  __device__ __forceinline__ double dist(int j) const { return d[j]; }
};

// ----------------------------------------------------- packet traversal --
// Per-warp shared memory: the traversal stack and one leaf staging buffer.
template <typename T, int D>
struct WarpScratch {
  int* stack;
  PointRec<T, D>* buf;  // 32 entries
};

// Exact kNN of the lane's query over the whole tree, ties in dist2 broken by
// tree position.  `own` (tree position or -1) is skipped, which is how self
// queries exclude the query point itself.  Returns false when the traversal
// stack would overflow (the host sizes it from the tree depth, so this is a
// safety net that reports instead of corrupting memory).
template <typename T, int D, int KMAX, typename DistT>
__device__ bool packet_knn(const TreeView<T, D>& tv, const DistT* q, int own, bool active, DistT r2,
                           TopK<KMAX, DistT>& top, WarpScratch<T, D> ws) {
  const int lane = threadIdx.x & 31;
  const unsigned FULL = 0xffffffffu;
  int sp = 0;
  int cur = 0;
  bool ok = true;
  int visits = 0;
  auto need = [&](DistT md) { return active && md < r2 && md <= top.worst(); };
  // Leaf bucket scan in two steps: every lane first marks the candidates that
  // can enter its list (distance at most its current k-th), with no
  // divergent branch, then inserts only those.  The warp pays for insertions
  // once per bucket (the largest count over lanes) rather than once per
  // candidate that some lane accepts.
  auto scan = [&](int begin, int count) {
    for (int base = begin; base < begin + count; base += 32) {
      const int nb = min(32, begin + count - base);
      __syncwarp();
      if (lane < nb) ws.buf[lane] = tv.pts[base + lane];
      __syncwarp();
      unsigned mark = 0;
      if (active) {
        const DistT thr = top.worst();
        for (int t = 0; t < nb; t++) {
          const DistT d2 = point_dist2<T, DistT, D>(ws.buf[t].c, q);
          const bool take = d2 < r2 && d2 <= thr && base + t != own;
          mark |= (unsigned)take << t;
        }
      }
      while (mark) {
        const int t = __ffs(mark) - 1;
        mark &= mark - 1;
        const DistT d2 = point_dist2<T, DistT, D>(ws.buf[t].c, q);
        top.offer(d2, base + t);
      }
    }
  };
  while (true) {
    if (++visits > tv.n_nodes) {  // a tree is acyclic: more visits mean a corrupt node array
      ok = false;
      break;
    }
    const TNode<T, D>& nd = tv.nodes[cur];
    DistT md[2];
    md[0] = nd.cnt[0] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[0], nd.hi[0], q) : (DistT)INFINITY;
    md[1] = nd.cnt[1] > 0 ? box_min_dist2<T, DistT, D>(nd.lo[1], nd.hi[1], q) : (DistT)INFINITY;
    const int first = __popc(__ballot_sync(FULL, active && md[1] < md[0])) > __popc(__ballot_sync(FULL, active)) / 2;
    int next = -1;
#pragma unroll
    for (int o = 0; o < 2; o++) {
      const int c = o == 0 ? first : 1 - first;
      if (!__any_sync(FULL, need(md[c]))) continue;
      const int ref = nd.ref[c];
      if (ref < 0) {
        scan(-ref - 1, nd.cnt[c]);
      } else if (next < 0) {
        next = ref;
      } else {
        if (sp >= tv.depth) {
          ok = false;
        } else {
          if (lane == 0) ws.stack[sp] = (cur << 1) | c;
          sp++;
        }
      }
    }
    if (next >= 0) {
      cur = next;
      continue;
    }
    __syncwarp();
    bool found = false;
    while (sp > 0) {
      const int e = ws.stack[--sp];
      __syncwarp();
      const TNode<T, D>& pn = tv.nodes[e >> 1];
      const int c = e & 1;
      const DistT m = box_min_dist2<T, DistT, D>(pn.lo[c], pn.hi[c], q);
      if (__any_sync(FULL, need(m))) {
        cur = pn.ref[c];
        found = true;
        break;
      }
    }
    __syncwarp();
    if (!found) break;
  }
  return ok;
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
  int cur = 0;
  bool ok = true;
  auto scan = [&](int begin, int cnt, bool mine) {
    for (int base = begin; base < begin + cnt; base += 32) {
      const int nb = min(32, begin + cnt - base);
      __syncwarp();
      if (lane < nb) ws.buf[lane] = tv.pts[base + lane];
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

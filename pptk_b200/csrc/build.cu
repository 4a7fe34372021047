// Level-synchronous device builder that reproduces the reference k-d tree
// exactly (pptk/kdtree/src/kdtree-impl.h:248-329 MakeNode /
// RecursiveBuildHelper, :773-818 BuildTree).
//
// The reference builds depth first; every node only permutes the indices of
// its own range, so building all nodes of a level at once gives the same
// permutation.  Nodes with more than `small_cap` points are processed by
// grid-wide kernels over 4096-point tiles; smaller subtrees are finished by
// one CTA each, entirely in shared memory.
//
// The reference partition (PartitionIndices, kdtree-impl.h:192-246) is two
// Hoare passes with converging cursors.  Each pass pairs the j-th misplaced
// element of the left zone (ascending) with the j-th misplaced element of the
// right zone (descending), so it is reproduced by ranking the two kinds of
// misplaced elements with scans and swapping rank-matched pairs.
#include <algorithm>
#include <vector>

#include "build.cuh"
#include "profile.cuh"
#include "util.cuh"

namespace pptkg {

constexpr int BT = 256;     // threads per tile block
constexpr int SWAP_U = 4;   // pairs a k_swap thread has in flight
constexpr int TILE = 4096;  // points per tile
constexpr int TITEMS = TILE / BT;

template <typename T, int D>
struct Seg {
  int b, e;
  int parent, side;  // parent record and side; a cloud's root has parent = -1 - cloud
  int lvl;
  int rec;
  long long n_orig;  // input rows of the segment's cloud (the reference's num_points)
  T lo[D], hi[D];  // loose extent (the reference's node_box), trimmed in place
  typename OrdOf<T>::type tlo[D], thi[D];
  int act;
  int sd;
  T sv;
  int L1, L2;
  int G;
  int tile0, ntiles;
};

constexpr int MAX_LEVELS = 4096;  // grid-wide levels (segments above small_cap points)

struct BuildCtl {
  int status;
  int n_tiles;
  int nsmall;
  int small_next;
  int rec_count;
  int depth;
  int level_cnt[MAX_LEVELS + 1];  // large segments per level
  int rec_base[MAX_LEVELS + 1];
};

// ----------------------------------------------------------------- helpers
template <typename T>
__device__ __forceinline__ T midpoint_ref(T a, T b) {
  if constexpr (std::is_unsigned<T>::value) {
    // kdtree-impl.h:161-164 (unsigned form), in C++ integer promotion
    if (a < b) {
      const T t = a;
      a = b;
      b = t;
    }
    return (T)((a - b) / 2 + b);
  } else if constexpr (std::is_integral<T>::value) {
    // kdtree-impl.h:167-173 (signed form), in C++ integer promotion
    if ((a >= 0 && b >= 0) || (a < 0 && b < 0)) return (T)((b - a) / (T)2 + a);
    return (T)((a + b) / (T)2);
  } else {
    // the same signed form in floating point, one rounding per operation
    if ((a >= (T)0 && b >= (T)0) || (a < (T)0 && b < (T)0)) return xadd(xdiv(xsub(b, a), (T)2), a);
    return xdiv(xadd(a, b), (T)2);
  }
}

// `T width = max - min` of ComputeSplit (kdtree-impl.h:179): integer types
// wrap as the reference's conversion back to T does.
template <typename T>
__device__ __forceinline__ T width_ref(T lo, T hi) {
  if constexpr (std::is_integral<T>::value)
    return (T)(hi - lo);
  else
    return xsub(hi, lo);
}

__device__ __forceinline__ double max0(double x) { return (0.0 < x) ? x : 0.0; }

// MakeNode's per-node decisions (kdtree-impl.h:248-297): empty-space trims of
// the loose extent against the tight box (TrimEmptyGaps, :114-158, in double),
// then the leaf test and the widest-axis midpoint split (ComputeSplit,
// :175-190, in T).  Writes the record except split_index and children.
template <typename T, int D>
__device__ void node_logic(int size, long long n_orig, bool is_top, T lo[D], T hi[D], const T tlo[D], const T thi[D],
                           int max_leaf, double thr, Rec<T, D>& rec, int& act, int& sd, T& sv) {
  for (int i = 0; i < D; i++) {
    rec.lo[i] = tlo[i];
    rec.hi[i] = thi[i];
  }
  if (is_top)
    for (int i = 0; i < D; i++) {
      lo[i] = tlo[i];
      hi[i] = thi[i];
    }
  rec.ntrim = 0;
  rec.split_dim = -1;
  rec.split_val = (T)0;
  rec.split_index = -1;
  rec.left = rec.right = -1;
  if ((long long)size != n_orig) {
    for (int guard = 0; guard <= 2 * D; guard++) {
      int gdim = -1, gside = -1;
      double gsize = 0.0;
      for (int i = 0; i < D; i++) {
        double g = max0(__dsub_rn((double)hi[i], (double)thi[i]));
        if (g >= gsize) gdim = i, gside = 1, gsize = g;
        g = max0(__dsub_rn((double)tlo[i], (double)lo[i]));
        if (g >= gsize) gdim = i, gside = 0, gsize = g;
      }
      if (gsize == 0.0) break;
      double width = __dsub_rn((double)hi[gdim], (double)lo[gdim]);
      if (__ddiv_rn(gsize, width) <= thr) break;
      if (rec.ntrim < 2 * D) rec.trim[rec.ntrim] = (uint8_t)(gdim * 2 + gside);
      rec.ntrim++;
      if (gside == 0)
        lo[gdim] = tlo[gdim];
      else
        hi[gdim] = thi[gdim];
    }
  }
  bool point = true;
  for (int i = 0; i < D; i++)
    if (tlo[i] != thi[i]) point = false;
  act = 0;
  if (!point && size > max_leaf) {
    T maxw = (T)0;
    sd = 0;
    sv = (T)0;
    for (int i = 0; i < D; i++) {
      T w = width_ref(tlo[i], thi[i]);
      if (w >= maxw) {
        maxw = w;
        sd = i;
        sv = (tlo[i] == thi[i]) ? tlo[i] : midpoint_ref(tlo[i], thi[i]);
      }
    }
    act = 1;
    rec.split_dim = (int8_t)sd;
    rec.split_val = sv;
  }
}

// num_left rule of PartitionIndices (kdtree-impl.h:234-244).
__device__ __forceinline__ int num_left_rule(int lim1, int lim2, int count) {
  int nl;
  if (lim1 > count / 2)
    nl = lim1;
  else if (lim2 < count / 2)
    nl = lim2;
  else
    nl = count / 2;
  if (lim1 == count && lim2 == 0) nl = count / 2;
  return nl;
}

// ------------------------------------------------------- input staging ----
template <typename T, int D>
__global__ void k_valid(const T* __restrict__ in, int64_t n, int* __restrict__ flag) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool ok = true;
#pragma unroll
  for (int d = 0; d < D; d++) ok = ok && valid_coord(in[i * D + d]);
  flag[i] = ok ? 1 : 0;
}

template <typename T, int D>
__global__ void k_compact(const T* __restrict__ in, int64_t n, const int* __restrict__ flag,
                          const int* __restrict__ off, SoA<T, D> soa) {
  int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  int j = off[i];
#pragma unroll
  for (int d = 0; d < D; d++) soa.x[d][j] = in[i * D + d];
  soa.id[j] = (int)i;
}

// valid_off[c] = number of valid rows before cloud c (the stable compaction
// keeps every cloud's valid rows together, in order).
static __global__ void k_cloud_off(const int* off, const int64_t* orig_off, int ncloud, int64_t* valid_off) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c <= ncloud) valid_off[c] = off[orig_off[c]];
}

// ------------------------------------------------------ grid-wide levels --
// Level `lvl` works on list segs (ctl->level_cnt[lvl] entries).  Kernels are
// launched with upper-bound grids and read the live counts from the device,
// so the host never waits between levels.
template <typename T, int D>
__global__ void k_roots(const int64_t* valid_off, const int64_t* orig_off, int ncloud, int small_cap, Seg<T, D>* lvl0,
                        Seg<T, D>* small, int small_capn, BuildCtl* ctl) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncloud) return;
  const int b = (int)valid_off[c], e = (int)valid_off[c + 1];
  if (e <= b) return;
  Seg<T, D> g;
  g.b = b;
  g.e = e;
  g.parent = -1 - c;
  g.side = 0;
  g.lvl = 0;
  g.rec = -1;
  g.n_orig = orig_off[c + 1] - orig_off[c];
  for (int d = 0; d < D; d++) {
    g.lo[d] = Limits<T>::max();  // replaced by the tight box at a root
    g.hi[d] = Limits<T>::lowest();
  }
  if (e - b > small_cap) {
    lvl0[atomicAdd(&ctl->level_cnt[0], 1)] = g;
  } else {
    const int slot = atomicAdd(&ctl->nsmall, 1);
    if (slot < small_capn)
      small[slot] = g;
    else
      atomicExch(&ctl->status, 7);
  }
}

template <typename T, int D>
__global__ void k_tiles(Seg<T, D>* segs, int lvl, int* tile_seg, BuildCtl* ctl) {
  __shared__ int sh[33];
  const int nseg = ctl->level_cnt[lvl];
  int carry = 0;
  for (int c0 = 0; c0 < nseg; c0 += blockDim.x) {
    int i = c0 + threadIdx.x;
    int nt = 0;
    if (i < nseg) nt = div_up_dev(segs[i].e - segs[i].b, TILE);
    int tot;
    int ex = block_excl_scan(nt, sh, tot);
    if (i < nseg) {
      segs[i].tile0 = carry + ex;
      segs[i].ntiles = nt;
    }
    carry += tot;
  }
  if (threadIdx.x == 0) {
    ctl->n_tiles = carry;
    ctl->rec_base[lvl] = ctl->rec_count;
    ctl->rec_count += nseg;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = wid; i < nseg; i += nw) {
    int t0 = segs[i].tile0, nt = segs[i].ntiles;
    for (int t = lane; t < nt; t += 32) tile_seg[t0 + t] = i;
  }
}

// The tiles of a level are walked grid-stride by a grid of a few blocks per
// SM, so a level with few tiles (or none: the trailing levels of a
// capture-mode rebuild) costs a few hundred idle blocks, not one per tile of
// the largest level.
template <typename T, int D>
__device__ __forceinline__ void tile_at(const Seg<T, D>* segs, const int* tile_seg, int t, int& s, int& start,
                                        int& end) {
  s = tile_seg[t];
  start = segs[s].b + (t - segs[s].tile0) * TILE;
  end = min(start + TILE, segs[s].e);
}

template <typename T, int D>
__global__ void k_seg_init(Seg<T, D>* segs, int lvl, const BuildCtl* ctl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ctl->level_cnt[lvl]) return;
  for (int d = 0; d < D; d++) {
    segs[i].tlo[d] = ord_t<T>(Limits<T>::max());
    segs[i].thi[d] = ord_t<T>(Limits<T>::lowest());
  }
  segs[i].L1 = segs[i].L2 = 0;
  segs[i].act = 0;
  segs[i].G = 0;
}

template <typename T>
__device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T>
__device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T, int D>
__global__ void __launch_bounds__(BT) k_bbox(Seg<T, D>* segs, const int* tile_seg, const BuildCtl* ctl, SoA<T, D> soa) {
  __shared__ T shmn[D][BT / 32], shmx[D][BT / 32];
  const int ntiles = ctl->n_tiles;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int s, start, end;
    tile_at(segs, tile_seg, t, s, start, end);
    T mn[D], mx[D];
#pragma unroll
    for (int d = 0; d < D; d++) {
      mn[d] = Limits<T>::max();
      mx[d] = Limits<T>::lowest();
    }
    for (int i = start + threadIdx.x; i < end; i += BT) {
#pragma unroll
      for (int d = 0; d < D; d++) {
        T v = soa.x[d][i];
        mn[d] = min(mn[d], v);
        mx[d] = max(mx[d], v);
      }
    }
#pragma unroll
    for (int d = 0; d < D; d++) {
      mn[d] = warp_min(mn[d]);
      mx[d] = warp_max(mx[d]);
      if (lane == 0) {
        shmn[d][wid] = mn[d];
        shmx[d][wid] = mx[d];
      }
    }
    __syncthreads();
    if (threadIdx.x < D) {
      int d = threadIdx.x;
      T a = shmn[d][0], b = shmx[d][0];
      for (int w = 1; w < BT / 32; w++) {
        a = min(a, shmn[d][w]);
        b = max(b, shmx[d][w]);
      }
      atomicMin(&segs[s].tlo[d], ord_t<T>(a));
      atomicMax(&segs[s].thi[d], ord_t<T>(b));
    }
    __syncthreads();
  }
}

template <typename T, int D>
__global__ void k_node(Seg<T, D>* segs, int lvl, BuildCtl* ctl, Rec<T, D>* recs, int rec_cap, int* root_rec,
                       int max_leaf, double thr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ctl->level_cnt[lvl]) return;
  Seg<T, D>& g = segs[i];
  T tlo[D], thi[D], lo[D], hi[D];
  for (int d = 0; d < D; d++) {
    tlo[d] = from_ord_t<T>(g.tlo[d]);
    thi[d] = from_ord_t<T>(g.thi[d]);
    lo[d] = g.lo[d];
    hi[d] = g.hi[d];
  }
  Rec<T, D> rec;
  int act, sd = 0;
  T sv = (T)0;
  node_logic<T, D>(g.e - g.b, g.n_orig, g.parent < 0, lo, hi, tlo, thi, max_leaf, thr, rec, act, sd, sv);
  rec.begin = g.b;
  rec.end = g.e;
  const int id = ctl->rec_base[lvl] + i;
  if (id >= rec_cap) {
    atomicExch(&ctl->status, 6);
    g.act = 0;
    return;
  }
  recs[id] = rec;
  if (g.parent >= 0) {
    if (g.side == 0)
      recs[g.parent].left = id;
    else
      recs[g.parent].right = id;
  } else {
    root_rec[-g.parent - 1] = id;
  }
  g.rec = id;
  g.act = act;
  g.sd = sd;
  g.sv = sv;
  for (int d = 0; d < D; d++) {
    g.lo[d] = lo[d];
    g.hi[d] = hi[d];
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(BT) k_count(Seg<T, D>* segs, const int* tile_seg, const BuildCtl* ctl, SoA<T, D> soa) {
  __shared__ long long sh[33];
  const int ntiles = ctl->n_tiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int s, start, end;
    tile_at(segs, tile_seg, t, s, start, end);
    if (!segs[s].act) continue;  // (uniform over the block)
    const T sv = segs[s].sv;
    const T* v = soa.x[segs[s].sd];
    int c1 = 0, c2 = 0;
    for (int i = start + threadIdx.x; i < end; i += BT) {
      T x = v[i];
      c1 += x < sv;
      c2 += x <= sv;
    }
    long long packed = ((long long)c2 << 32) | (long long)c1;
    long long tot = block_sum(packed, sh);
    if (threadIdx.x == 0) {
      atomicAdd(&segs[s].L1, (int)(tot & 0xffffffffll));
      atomicAdd(&segs[s].L2, (int)(tot >> 32));
    }
  }
}

// Misplaced-element predicates of the two partition passes.
template <typename T>
__device__ __forceinline__ void pass_flags(int pass, int i, T x, T sv, int b, int L1, int L2, bool& bl, bool& gr) {
  if (pass == 1) {
    const int Z = b + L1;
    bl = (i < Z) && !(x < sv);
    gr = (i >= Z) && (x < sv);
  } else {
    const int Z = b + L2;
    bl = (i >= b + L1) && (i < Z) && (x > sv);
    gr = (i >= Z) && (x <= sv);
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(BT) k_flags(int pass, Seg<T, D>* segs, const int* tile_seg, const BuildCtl* ctl,
                                              SoA<T, D> soa, long long* tile_cnt) {
  __shared__ long long sh[33];
  const int ntiles = ctl->n_tiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int s, start, end;
    tile_at(segs, tile_seg, t, s, start, end);
    long long c = 0;
    // the second pass moves the points equal to the split value; with none
    // (L1 == L2, the usual case for float data) it has nothing to do
    if (segs[s].act && !(pass == 2 && segs[s].L1 == segs[s].L2)) {
      const T sv = segs[s].sv;
      const T* v = soa.x[segs[s].sd];
      const int b = segs[s].b, L1 = segs[s].L1, L2 = segs[s].L2;
      for (int i = start + threadIdx.x; i < end; i += BT) {
        bool bl, gr;
        pass_flags(pass, i, v[i], sv, b, L1, L2, bl, gr);
        c += (long long)bl + ((long long)gr << 32);
      }
    }
    long long tot = block_sum(c, sh);
    if (threadIdx.x == 0) tile_cnt[t] = tot;
  }
}

template <typename T, int D>
__global__ void k_tscan(Seg<T, D>* segs, int lvl, const long long* tile_cnt, long long* tile_off, BuildCtl* ctl) {
  __shared__ long long sh[33];
  const int nseg = ctl->level_cnt[lvl];
  for (int si = blockIdx.x; si < nseg; si += gridDim.x) {
    Seg<T, D>& g = segs[si];
    if (!g.act) continue;  // (uniform over the block)
    long long carry = 0;
    for (int c0 = 0; c0 < g.ntiles; c0 += blockDim.x) {
      int t = c0 + threadIdx.x;
      long long v = t < g.ntiles ? tile_cnt[g.tile0 + t] : 0;
      long long tot;
      long long ex = block_excl_scan(v, sh, tot);
      if (t < g.ntiles) tile_off[g.tile0 + t] = carry + ex;
      carry += tot;
    }
    if (threadIdx.x == 0) {
      int nbl = (int)(carry & 0xffffffffll), ngr = (int)(carry >> 32);
      g.G = nbl;
      if (nbl != ngr) atomicExch(&ctl->status, 1);
    }
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(BT) k_scatter(int pass, Seg<T, D>* segs, const int* tile_seg, const BuildCtl* ctl,
                                                SoA<T, D> soa, const long long* tile_off, int* blpos, int* grpos) {
  __shared__ long long sh[33];
  const int ntiles = ctl->n_tiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int s, start, end;
    tile_at(segs, tile_seg, t, s, start, end);
    if (!segs[s].act || (pass == 2 && segs[s].L1 == segs[s].L2)) continue;  // (uniform over the block)
    const T sv = segs[s].sv;
    const T* v = soa.x[segs[s].sd];
    const int b = segs[s].b, L1 = segs[s].L1, L2 = segs[s].L2, G = segs[s].G;
    const int i0 = start + threadIdx.x * TITEMS;
    unsigned mbl = 0, mgr = 0;
#pragma unroll
    for (int j = 0; j < TITEMS; j++) {
      int i = i0 + j;
      if (i < end) {
        bool bl, gr;
        pass_flags(pass, i, v[i], sv, b, L1, L2, bl, gr);
        mbl |= (unsigned)bl << j;
        mgr |= (unsigned)gr << j;
      }
    }
    long long mine = (long long)__popc(mbl) + ((long long)__popc(mgr) << 32);
    long long tot;
    long long ex = block_excl_scan(mine, sh, tot) + tile_off[t];
    int rb = (int)(ex & 0xffffffffll), rg = (int)(ex >> 32);
    const int size = segs[s].e - b;
#pragma unroll
    for (int j = 0; j < TITEMS; j++) {
      if (mbl >> j & 1) {
        if (rb < size) blpos[b + rb] = i0 + j;
        rb++;
      }
      if (mgr >> j & 1) {
        const int slot = G - 1 - rg;
        if (slot >= 0 && slot < size) grpos[b + slot] = i0 + j;
        rg++;
      }
    }
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(BT) k_swap(Seg<T, D>* segs, const int* tile_seg, BuildCtl* ctl, SoA<T, D> soa,
                                             const int* blpos, const int* grpos) {
  const int ntiles = ctl->n_tiles;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    int s, start, end;
    tile_at(segs, tile_seg, t, s, start, end);
    if (!segs[s].act) continue;
    const int b = segs[s].b, e = segs[s].e, G = segs[s].G;
    // pair j of this tile: j = start - b + threadIdx.x + u * BT.  Every
    // position belongs to one pair only, so the loads of SWAP_U pairs are
    // issued before their stores: the swap is bound by memory latency, and
    // one pair in flight per thread left most of it exposed
    const int jend = min(end - b, G);
    for (int j0 = start - b + threadIdx.x; j0 < jend; j0 += SWAP_U * BT) {
      int x[SWAP_U], y[SWAP_U];
      bool ok[SWAP_U];
#pragma unroll
      for (int u = 0; u < SWAP_U; u++) {
        const int j = j0 + u * BT;
        ok[u] = j < jend;
        x[u] = ok[u] ? blpos[b + j] : b;
        y[u] = ok[u] ? grpos[b + j] : b;
        if (ok[u] && (x[u] < b || x[u] >= e || y[u] < b || y[u] >= e)) {
          atomicExch(&ctl->status, 4);
          ok[u] = false;
        }
      }
      T vx[SWAP_U][D], vy[SWAP_U][D];
      int ix[SWAP_U], iy[SWAP_U];
#pragma unroll
      for (int u = 0; u < SWAP_U; u++) {
        if (!ok[u]) continue;
#pragma unroll
        for (int d = 0; d < D; d++) {
          vx[u][d] = soa.x[d][x[u]];
          vy[u][d] = soa.x[d][y[u]];
        }
        ix[u] = soa.id[x[u]];
        iy[u] = soa.id[y[u]];
      }
#pragma unroll
      for (int u = 0; u < SWAP_U; u++) {
        if (!ok[u]) continue;
#pragma unroll
        for (int d = 0; d < D; d++) {
          soa.x[d][x[u]] = vy[u][d];
          soa.x[d][y[u]] = vx[u][d];
        }
        soa.id[x[u]] = iy[u];
        soa.id[y[u]] = ix[u];
      }
    }
  }
}

template <typename T, int D>
__global__ void k_children(Seg<T, D>* segs, int lvl, Rec<T, D>* recs, Seg<T, D>* next, Seg<T, D>* small,
                           int small_capn, int small_cap_pts, BuildCtl* ctl) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ctl->level_cnt[lvl]) return;
  const Seg<T, D>& g = segs[i];
  if (!g.act) return;
  const int count = g.e - g.b;
  const int si = g.b + num_left_rule(g.L1, g.L2, count);
  recs[g.rec].split_index = si;
  for (int side = 0; side < 2; side++) {
    int cb = side ? si : g.b, ce = side ? g.e : si;
    if (cb >= ce) continue;
    Seg<T, D> c;
    c.b = cb;
    c.e = ce;
    c.parent = g.rec;
    c.side = side;
    c.lvl = g.lvl + 1;
    c.rec = -1;
    c.n_orig = g.n_orig;
    for (int d = 0; d < D; d++) {
      c.lo[d] = g.lo[d];
      c.hi[d] = g.hi[d];
    }
    if (side == 0)
      c.hi[g.sd] = g.sv;
    else
      c.lo[g.sd] = g.sv;
    if (ce - cb > small_cap_pts) {
      next[atomicAdd(&ctl->level_cnt[lvl + 1], 1)] = c;
    } else {
      const int slot = atomicAdd(&ctl->nsmall, 1);
      if (slot < small_capn)
        small[slot] = c;
      else
        atomicExch(&ctl->status, 7);
    }
  }
}

// -------------------------------------------------- per-CTA subtrees ----
template <typename T, int D>
struct Entry {
  int b, e, parent, side;
  T lo[D], hi[D];
};

constexpr int SUB_THREADS = 256;
// k_subtree nodes of at most this many points are split by one thread
constexpr int LANE_NODE = 32;

// Finishes small segments' whole subtrees in shared memory, level by level:
// one warp per node above LANE_NODE points, one thread per smaller node.
// Persistent: each CTA takes segments from the small list until it is
// exhausted.  (Splitting the first levels' few nodes with
// the whole block instead was measured slower: a third more subtree time on
// a 4,096-cloud forest; the warps of the SM's other CTAs already fill the
// issue slots those levels leave idle.)
template <typename T, int D>
__global__ void __launch_bounds__(SUB_THREADS) k_subtree(const Seg<T, D>* small, SoA<T, D> soa, Rec<T, D>* recs,
                                                         int* root_rec, int cap_pts, int cap_list, int max_leaf,
                                                         double thr, int rec_cap, BuildCtl* ctl) {
  extern __shared__ __align__(16) unsigned char smem[];
  T* X[D];
  unsigned char* p = smem;
  for (int d = 0; d < D; d++) {
    X[d] = (T*)p;
    p += sizeof(T) * cap_pts;
  }
  int* ID = (int*)p;
  p += sizeof(int) * cap_pts;
  int* S = (int*)p;
  p += sizeof(int) * cap_pts;
  p = (unsigned char*)(((uintptr_t)p + 15) & ~(uintptr_t)15);
  Entry<T, D>* LA0 = (Entry<T, D>*)p;
  Entry<T, D>* LB0 = LA0 + cap_list;
  int* cnt = (int*)(LB0 + cap_list);  // [0] nA, [1] nB, [2] base, [3] overflow, [4] item
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const unsigned lt = (1u << lane) - 1u;
  const int nsmall = min(ctl->nsmall, INT_MAX);

  while (true) {
    if (threadIdx.x == 0) cnt[4] = atomicAdd(&ctl->small_next, 1);
    __syncthreads();
    const int item = cnt[4];
    __syncthreads();
    if (item >= nsmall) break;
    const Seg<T, D> seg = small[item];
    const int n = seg.e - seg.b;
    Entry<T, D>* LA = LA0;
    Entry<T, D>* LB = LB0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      for (int d = 0; d < D; d++) X[d][i] = soa.x[d][seg.b + i];
      ID[i] = soa.id[seg.b + i];
    }
    if (threadIdx.x == 0) {
      Entry<T, D> r;
      r.b = 0;
      r.e = n;
      r.parent = seg.parent;
      r.side = seg.side;
      for (int d = 0; d < D; d++) {
        r.lo[d] = seg.lo[d];
        r.hi[d] = seg.hi[d];
      }
      LA[0] = r;
      cnt[0] = 1;
      cnt[3] = 0;
    }
    __syncthreads();
    int levels = 0;
    while (true) {
      const int nA = cnt[0];
      if (nA == 0) break;
      if (levels > n + 1) {  // every level splits ranges into strictly smaller ones
        if (threadIdx.x == 0) atomicExch(&ctl->status, 5);
        break;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        cnt[1] = 0;
        cnt[2] = atomicAdd(&ctl->rec_count, nA);
      }
      __syncthreads();
      const int base = cnt[2];
      levels++;
      for (int ei = wid; ei < nA; ei += nw) {
        Entry<T, D> en = LA[ei];
        const int b = en.b, e = en.e, size = e - b;
        if (size <= LANE_NODE) continue;  // (warp-uniform) one thread's node, below
        T mn[D], mx[D];
        for (int d = 0; d < D; d++) {
          mn[d] = Limits<T>::max();
          mx[d] = Limits<T>::lowest();
        }
        for (int q = b + lane; q < e; q += 32)
          for (int d = 0; d < D; d++) {
            T v = X[d][q];
            mn[d] = min(mn[d], v);
            mx[d] = max(mx[d], v);
          }
        for (int d = 0; d < D; d++) {
          mn[d] = warp_min(mn[d]);
          mx[d] = warp_max(mx[d]);
        }
        int act = 0, sd = 0;
        T sv = (T)0;
        const int id = base + ei;
        if (lane == 0) {
          Rec<T, D> rec;
          node_logic<T, D>(size, seg.n_orig, en.parent < 0, en.lo, en.hi, mn, mx, max_leaf, thr, rec, act, sd, sv);
          rec.begin = seg.b + b;
          rec.end = seg.b + e;
          if (id >= rec_cap) {
            atomicExch(&ctl->status, 6);
            act = 0;
          } else {
            recs[id] = rec;
            if (en.parent >= 0) {
              if (en.side == 0)
                recs[en.parent].left = id;
              else
                recs[en.parent].right = id;
            } else {
              root_rec[-en.parent - 1] = id;
            }
          }
          LA[ei] = en;  // keep the trimmed extent for the children
        }
        act = __shfl_sync(0xffffffffu, act, 0);
        if (!act) continue;
        sd = __shfl_sync(0xffffffffu, sd, 0);
        sv = __shfl_sync(0xffffffffu, sv, 0);
        T* v = X[sd];
        int L1 = 0, L2 = 0;
        for (int q0 = b; q0 < e; q0 += 32) {
          int q = q0 + lane;
          T x = q < e ? v[q] : sv;
          bool in = q < e;
          L1 += __popc(__ballot_sync(0xffffffffu, in && x < sv));
          L2 += __popc(__ballot_sync(0xffffffffu, in && x <= sv));
        }
        const int half = size / 2;
        for (int pass = 1; pass <= (L1 == L2 ? 1 : 2); pass++) {
          const int zlo = pass == 1 ? b : b + L1;
          const int Z = pass == 1 ? b + L1 : b + L2;
          int G = 0;
          for (int q0 = zlo; q0 < Z; q0 += 32) {
            int q = q0 + lane;
            bool f = false;
            if (q < Z) {
              T x = v[q];
              f = pass == 1 ? !(x < sv) : (x > sv);
            }
            unsigned bal = __ballot_sync(0xffffffffu, f);
            if (f && G + __popc(bal & lt) < half) S[b + G + __popc(bal & lt)] = q;
            G += __popc(bal);
          }
          int a = 0;
          for (int q0 = Z; q0 < e; q0 += 32) {
            int q = q0 + lane;
            bool f = false;
            if (q < e) {
              T x = v[q];
              f = pass == 1 ? (x < sv) : (x <= sv);
            }
            unsigned bal = __ballot_sync(0xffffffffu, f);
            if (f) {
              int r = a + __popc(bal & lt);
              if (r < G && G <= half) S[b + half + (G - 1 - r)] = q;
            }
            a += __popc(bal);
          }
          if ((a != G || G > half) && lane == 0) atomicExch(&ctl->status, 2);
          __syncwarp();
          if (a == G && G <= half)
            for (int j = lane; j < G; j += 32) {
              int x = S[b + j], y = S[b + half + j];
              for (int d = 0; d < D; d++) {
                T t = X[d][x];
                X[d][x] = X[d][y];
                X[d][y] = t;
              }
              int t = ID[x];
              ID[x] = ID[y];
              ID[y] = t;
            }
          __syncwarp();
        }
        if (lane == 0) {
          const int si = b + num_left_rule(L1, L2, size);
          if (id < rec_cap) recs[id].split_index = seg.b + si;
          const Entry<T, D> par = LA[ei];
          for (int side = 0; side < 2; side++) {
            int cb = side ? si : b, ce = side ? e : si;
            if (cb >= ce) continue;
            Entry<T, D> c;
            c.b = cb;
            c.e = ce;
            c.parent = id;
            c.side = side;
            for (int d = 0; d < D; d++) {
              c.lo[d] = par.lo[d];
              c.hi[d] = par.hi[d];
            }
            if (side == 0)
              c.hi[sd] = sv;
            else
              c.lo[sd] = sv;
            int slot = atomicAdd(&cnt[1], 1);
            if (slot < cap_list)
              LB[slot] = c;
            else
              atomicExch(&cnt[3], 1);
          }
        }
      }
      // nodes of at most LANE_NODE points: one thread each, with the
      // reference's two converging cursors over shared memory (the pairs a
      // warp forms by ranks), so that the many small nodes of the last
      // levels do not each pay a warp's fixed per-node work
      for (int ei = threadIdx.x; ei < nA; ei += blockDim.x) {
        Entry<T, D> en = LA[ei];
        const int b = en.b, e = en.e, size = e - b;
        if (size > LANE_NODE) continue;
        T mn[D], mx[D];
        for (int d = 0; d < D; d++) {
          mn[d] = Limits<T>::max();
          mx[d] = Limits<T>::lowest();
        }
        for (int q = b; q < e; q++)
          for (int d = 0; d < D; d++) {
            const T x = X[d][q];
            mn[d] = min(mn[d], x);
            mx[d] = max(mx[d], x);
          }
        const int id = base + ei;
        Rec<T, D> rec;
        int act = 0, sd = 0;
        T sv = (T)0;
        node_logic<T, D>(size, seg.n_orig, en.parent < 0, en.lo, en.hi, mn, mx, max_leaf, thr, rec, act, sd, sv);
        rec.begin = seg.b + b;
        rec.end = seg.b + e;
        if (id >= rec_cap) {
          atomicExch(&ctl->status, 6);
          continue;
        }
        recs[id] = rec;
        if (en.parent >= 0) {
          if (en.side == 0)
            recs[en.parent].left = id;
          else
            recs[en.parent].right = id;
        } else {
          root_rec[-en.parent - 1] = id;
        }
        if (!act) continue;
        const T* v = X[sd];
        int L1 = 0, L2 = 0;
        for (int q = b; q < e; q++) {
          L1 += v[q] < sv;
          L2 += v[q] <= sv;
        }
        for (int pass = 1; pass <= (L1 == L2 ? 1 : 2); pass++) {
          const int Z = pass == 1 ? b + L1 : b + L2;
          int i = pass == 1 ? b : b + L1, j = e - 1;
          while (true) {
            while (i < Z && !(pass == 1 ? !(v[i] < sv) : (v[i] > sv))) i++;
            while (j >= Z && !(pass == 1 ? (v[j] < sv) : (v[j] <= sv))) j--;
            if (i >= Z || j < Z) break;
            for (int d = 0; d < D; d++) {
              const T t = X[d][i];
              X[d][i] = X[d][j];
              X[d][j] = t;
            }
            const int t = ID[i];
            ID[i] = ID[j];
            ID[j] = t;
            i++;
            j--;
          }
        }
        const int si = b + num_left_rule(L1, L2, size);
        recs[id].split_index = seg.b + si;
        for (int side = 0; side < 2; side++) {
          const int cb = side ? si : b, ce = side ? e : si;
          if (cb >= ce) continue;
          Entry<T, D> c;
          c.b = cb;
          c.e = ce;
          c.parent = id;
          c.side = side;
          for (int d = 0; d < D; d++) {
            c.lo[d] = en.lo[d];
            c.hi[d] = en.hi[d];
          }
          if (side == 0)
            c.hi[sd] = sv;
          else
            c.lo[sd] = sv;
          const int slot = atomicAdd(&cnt[1], 1);
          if (slot < cap_list)
            LB[slot] = c;
          else
            atomicExch(&cnt[3], 1);
        }
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        cnt[0] = min(cnt[1], cap_list);
        if (cnt[3]) atomicExch(&ctl->status, 3);
      }
      __syncthreads();
      Entry<T, D>* tmp = LA;
      LA = LB;
      LB = tmp;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      for (int d = 0; d < D; d++) soa.x[d][seg.b + i] = X[d][i];
      soa.id[seg.b + i] = ID[i];
    }
    if (threadIdx.x == 0) atomicMax(&ctl->depth, seg.lvl + levels);
    __syncthreads();
  }
}

// ------------------------------------------------------- finishing ----
template <typename T, int D>
__global__ void k_finish(SoA<T, D> soa, int nv, PointRec<T, D>* pts, int* fwd, const int64_t* nv_dev = nullptr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (nv_dev) nv = (int)*nv_dev;  // capture mode: the valid count is on the device
  if (i >= nv) return;
  PointRec<T, D> r;
#pragma unroll
  for (int d = 0; d < D; d++) r.c[d] = soa.x[d][i];
  r.id = soa.id[i];
  pts[i] = r;
  fwd[r.id] = i;
}

template <typename T, int D>
__global__ void k_tflag(const Rec<T, D>* recs, int n_recs, int bucket, int* flag, const int* n_dev = nullptr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_recs) return;
  if (n_dev && i >= *n_dev) {  // capture mode: records beyond the live count
    flag[i] = 0;
    return;
  }
  const Rec<T, D>& r = recs[i];
  flag[i] = (r.split_dim >= 0 && r.end - r.begin > bucket && r.left >= 0 && r.right >= 0) ? 1 : 0;
}

template <typename T, int D>
__global__ void k_tfill(const Rec<T, D>* recs, int n_recs, const int* flag, const int* tid, TNode<T, D>* nodes,
                        const int* n_dev = nullptr, int node_lim = INT_MAX, int* status = nullptr) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_recs || (n_dev && i >= *n_dev) || !flag[i]) return;
  // capture mode: nodes beyond the capacity are left out (their parents
  // see them as buckets: the walks stay exact) and reported
  if (tid[i] >= node_lim) {
    atomicExch(status, 21);
    return;
  }
  const Rec<T, D>& r = recs[i];
  TNode<T, D> t;
  for (int c = 0; c < 2; c++) {
    int ch = c ? r.right : r.left;
    const Rec<T, D>& cr = recs[ch];
    for (int d = 0; d < D; d++) {
      t.lo[c][d] = cr.lo[d];
      t.hi[c][d] = cr.hi[d];
    }
    t.cnt[c] = cr.end - cr.begin;
    t.ref[c] = (flag[ch] && tid[ch] < node_lim) ? tid[ch] : -cr.begin - 1;
  }
  nodes[tid[i]] = t;
}

// Per-cloud traversal roots: the root record's node when it is an inner
// node, otherwise a dedicated node (index nt + c) whose first child is the
// whole cloud as one bucket (or nothing, for a cloud without valid points).
template <typename T, int D>
__global__ void k_troots(const Rec<T, D>* recs, const int* root_rec, const int64_t* valid_off, int ncloud,
                         const int* flag, const int* tid, int nt, TNode<T, D>* nodes, int* root_tnode,
                         const int* nt_dev = nullptr) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncloud) return;
  if (nt_dev) nt = *nt_dev;  // the node count on the device
  const int r = root_rec[c];
  TNode<T, D> t;
  for (int k = 0; k < 2; k++)
    for (int d = 0; d < D; d++) {
      t.lo[k][d] = Limits<T>::max();
      t.hi[k][d] = Limits<T>::lowest();
    }
  t.ref[0] = t.ref[1] = -1;
  t.cnt[0] = t.cnt[1] = 0;
  if (r >= 0 && flag[r] && tid[r] < nt) {
    // the root record has its own node; the reserved slot stays an empty
    // node (nothing refers to it, but every slot holds a well-formed node)
    nodes[nt + c] = t;
    root_tnode[c] = tid[r];
    return;
  }
  if (r >= 0) {
    for (int d = 0; d < D; d++) {
      t.lo[0][d] = recs[r].lo[d];
      t.hi[0][d] = recs[r].hi[d];
    }
    t.ref[0] = -(int)valid_off[c] - 1;
    t.cnt[0] = (int)(valid_off[c + 1] - valid_off[c]);
  }
  nodes[nt + c] = t;
  root_tnode[c] = nt + c;
}

// ------------------------------------------------------------ host side ----
// Grid of the grid-stride level kernels: eight 256-thread blocks per SM.
static int level_grid(int device) {
  int nsm = 148;
  PPTKG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  return std::max(nsm, 1) * 8;
}

template <typename T, int D>
int small_capacity(int max_leaf, int& cap_list, size_t& smem) {
  const size_t budget = 72 * 1024;
  int cap = sizeof(T) == 4 ? 2048 : 1024;
  while (true) {
    cap_list = 2 * (cap / (max_leaf + 1)) + 2;
    smem = (sizeof(T) * D + 2 * sizeof(int)) * (size_t)cap + 16 + 2 * sizeof(Entry<T, D>) * (size_t)cap_list +
           8 * sizeof(int);
    if (smem <= budget || cap <= 64) break;
    cap /= 2;
  }
  return cap;
}

// ------------------------------------------------ integer point types ----
// The reference computes every distance of an integer tree in float
// (Accumulator, accumulator.h:16-19): each coordinate and box bound is
// converted to float where it is read (kdtree-impl.h:331-339, box.h:157-198).
// After the build (done exactly in T), the tree-ordered points and the
// traversal boxes are stored as those float values, so the float query
// kernels answer integer trees; the records stay in T.
template <typename T, int D>
__global__ void k_lower_points(const PointRec<T, D>* in, int64_t nv, PointRec<float, D>* out) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nv) return;
  PointRec<float, D> r;
#pragma unroll
  for (int d = 0; d < D; d++) r.c[d] = (float)in[i].c[d];
  r.id = in[i].id;
  out[i] = r;
}

template <typename T, int D>
__global__ void k_lower_tnodes(const TNode<T, D>* in, int n, TNode<float, D>* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  TNode<float, D> t;
#pragma unroll
  for (int k = 0; k < 2; k++) {
#pragma unroll
    for (int d = 0; d < D; d++) {
      t.lo[k][d] = (float)in[i].lo[k][d];
      t.hi[k][d] = (float)in[i].hi[k][d];
    }
    t.ref[k] = in[i].ref[k];
    t.cnt[k] = in[i].cnt[k];
  }
  out[i] = t;
}

template <typename T, int D>
void lower_points(TreeBase* tree, cudaStream_t st) {
  PointRec<float, D>* out = nullptr;
  PPTKG_CUDA(dev_malloc((void**)&out, std::max<int64_t>(tree->nv, 1) * sizeof(PointRec<float, D>), st));
  if (tree->nv > 0) {
    k_lower_points<T, D><<<(unsigned)((tree->nv + 255) / 256), 256, 0, st>>>((const PointRec<T, D>*)tree->pts,
                                                                             tree->nv, out);
    PPTKG_CHECK_LAUNCH();
  }
  dev_free(tree->pts, st);
  tree->pts = out;
  tree->dtype = F32;
}

template <typename T, int D>
void lower_tnodes(TreeBase* tree, cudaStream_t st) {
  TNode<float, D>* out = nullptr;
  const int n = tree->n_tnodes;
  PPTKG_CUDA(dev_malloc((void**)&out, std::max(n, 1) * sizeof(TNode<float, D>), st));
  if (n > 0) {
    k_lower_tnodes<T, D><<<(unsigned)((n + 255) / 256), 256, 0, st>>>((const TNode<T, D>*)tree->tnodes, n, out);
    PPTKG_CHECK_LAUNCH();
  }
  dev_free(tree->tnodes, st);
  tree->tnodes = out;
}

template <typename T, int D>
TreeBase* build_forest(const T* d_in, int64_t n, const int64_t* orig_off_h, int ncloud, int max_leaf, double thr,
                       int bucket, cudaStream_t st) {
  if (n > (int64_t)INT32_MAX / 2 - 64) throw Error(E_INVALID, "k-d tree supports at most 2^30 points");
  if (ncloud < 1) throw Error(E_INVALID, "at least one cloud");
  if (max_leaf < 1) max_leaf = 1;
  Stage stage("build", st);
  keep_pool_cached(st);
  std::unique_ptr<TreeBase> tree(new TreeBase());
  tree->stream = st;
  tree->dtype = std::is_same<T, double>::value ? F64 : F32;
  tree->rec_dtype = dtype_code<T>();
  tree->dim = D;
  tree->n = n;
  tree->max_leaf = max_leaf;
  tree->empty_split = thr;
  tree->bucket = bucket;
  tree->ncloud = ncloud;
  PPTKG_CUDA(cudaGetDevice(&tree->device));
  tree->orig_off_h.assign(orig_off_h, orig_off_h + ncloud + 1);
  if (tree->orig_off_h[0] != 0 || tree->orig_off_h[ncloud] != n)
    throw Error(E_INVALID, "cloud offsets must start at 0 and end at n");
  for (int c = 0; c < ncloud; c++)
    if (tree->orig_off_h[c + 1] < tree->orig_off_h[c]) throw Error(E_INVALID, "cloud offsets must not decrease");
  PPTKG_CUDA(dev_malloc((void**)&tree->orig_off, sizeof(int64_t) * (ncloud + 1), st));
  PPTKG_CUDA(dev_malloc((void**)&tree->valid_off, sizeof(int64_t) * (ncloud + 1), st));
  PPTKG_CUDA(dev_malloc((void**)&tree->root_rec, sizeof(int) * ncloud, st));
  PPTKG_CUDA(dev_malloc((void**)&tree->root_tnode, sizeof(int) * ncloud, st));
  PPTKG_CUDA(cudaMemcpyAsync(tree->orig_off, orig_off_h, sizeof(int64_t) * (ncloud + 1), cudaMemcpyHostToDevice, st));
  PPTKG_CUDA(cudaMemsetAsync(tree->root_rec, 0xff, sizeof(int) * ncloud, st));

  // valid-point compaction (ValidPointIndices, kdtree-impl.h:53-75), per cloud
  std::unique_ptr<Stage> st_prep(new Stage("build.prep", st));
  BuildBuf<int> flag(n + 1, st), off(n + 1, st);
  if (n > 0) {
    k_valid<T, D><<<div_up(n, 256), 256, 0, st>>>(d_in, n, flag.get());
    PPTKG_CHECK_LAUNCH();
  }
  exclusive_scan<int, int>(flag.get(), off.get(), n, off.get() + n, st);
  k_cloud_off<<<div_up(ncloud + 1, 256), 256, 0, st>>>(off.get(), tree->orig_off, ncloud, tree->valid_off);
  PPTKG_CHECK_LAUNCH();
  tree->valid_off_h.resize(ncloud + 1);
  PPTKG_CUDA(cudaMemcpyAsync(tree->valid_off_h.data(), tree->valid_off, sizeof(int64_t) * (ncloud + 1),
                             cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  const int nv = (int)tree->valid_off_h[ncloud];
  tree->nv = nv;

  BuildBuf<T> xs((size_t)D * nv + 1, st);
  BuildBuf<int> ids(nv + 1, st);
  SoA<T, D> soa;
  for (int d = 0; d < D; d++) soa.x[d] = xs.get() + (size_t)d * nv;
  soa.id = ids.get();
  if (n > 0) {
    k_compact<T, D><<<div_up(n, 256), 256, 0, st>>>(d_in, n, flag.get(), off.get(), soa);
    PPTKG_CHECK_LAUNCH();
  }
  flag.release();
  off.release();
  st_prep.reset();

  int cap_list;
  size_t smem;
  const int small_cap = small_capacity<T, D>(max_leaf, cap_list, smem);
  // a binary tree over nv points has at most 2 nv - 1 records
  const size_t rec_cap = 2 * (size_t)nv + 64;
  std::unique_ptr<Stage> st_scr(new Stage("build.scratch", st));
  BuildBuf<Rec<T, D>> recbuf(rec_cap, st);
  Rec<T, D>* recs = recbuf.get();
  st_scr.reset();

  // large segments per level are disjoint and above small_cap points
  const int seg_cap = nv / (small_cap + 1) + 2;
  const int max_tiles = nv / TILE + seg_cap + 2;
  int small_capn = ncloud + 2 * 64 * (seg_cap + 1);
  int depth = 0;
  for (int attempt = 0; attempt < 4; attempt++, small_capn *= 4) {
    Stage st_att("build.attempt", st);
    BuildBuf<BuildCtl> ctl(1, st);
    PPTKG_CUDA(cudaMemsetAsync(ctl.get(), 0, sizeof(BuildCtl), st));
    BuildBuf<Seg<T, D>> segL[2] = {BuildBuf<Seg<T, D>>(seg_cap, st), BuildBuf<Seg<T, D>>(seg_cap, st)};
    BuildBuf<Seg<T, D>> smallL(small_capn, st);
    if (nv > 0) {
      k_roots<T, D><<<div_up(ncloud, 128), 128, 0, st>>>(tree->valid_off, tree->orig_off, ncloud, small_cap,
                                                          segL[0].get(), smallL.get(), small_capn, ctl.get());
      PPTKG_CHECK_LAUNCH();
    }
    int levels = 0;
    {
      Stage st_levels("build.levels", st);
      BuildBuf<int> blpos(nv + 1, st), grpos(nv + 1, st);
      BuildBuf<int> tile_seg(max_tiles, st);
      BuildBuf<long long> tile_cnt(max_tiles, st), tile_off(max_tiles, st);
      const unsigned gt = (unsigned)std::min(max_tiles, level_grid(tree->device));
      const unsigned gq = (unsigned)std::min(seg_cap, level_grid(tree->device));
      const unsigned gs = (unsigned)div_up(seg_cap, 128);
      int h0 = 0;
      if (nv > 0) {
        PPTKG_CUDA(cudaMemcpyAsync(&h0, &ctl.get()->level_cnt[0], sizeof(int), cudaMemcpyDeviceToHost, st));
        PPTKG_CUDA(cudaStreamSynchronize(st));
      }
      for (int lvl = 0; h0 > 0 && lvl < MAX_LEVELS; lvl++) {
        Seg<T, D>* A = segL[lvl & 1].get();
        Seg<T, D>* B = segL[(lvl + 1) & 1].get();
        k_tiles<T, D><<<1, 1024, 0, st>>>(A, lvl, tile_seg.get(), ctl.get());
        PPTKG_CHECK_LAUNCH();
        k_seg_init<T, D><<<gs, 128, 0, st>>>(A, lvl, ctl.get());
        PPTKG_CHECK_LAUNCH();
        k_bbox<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa);
        PPTKG_CHECK_LAUNCH();
        k_node<T, D><<<gs, 128, 0, st>>>(A, lvl, ctl.get(), recs, (int)rec_cap, tree->root_rec, max_leaf, thr);
        PPTKG_CHECK_LAUNCH();
        k_count<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa);
        PPTKG_CHECK_LAUNCH();
        for (int pass = 1; pass <= 2; pass++) {
          k_flags<T, D><<<gt, BT, 0, st>>>(pass, A, tile_seg.get(), ctl.get(), soa, tile_cnt.get());
          PPTKG_CHECK_LAUNCH();
          k_tscan<T, D><<<gq, 256, 0, st>>>(A, lvl, tile_cnt.get(), tile_off.get(), ctl.get());
          PPTKG_CHECK_LAUNCH();
          k_scatter<T, D><<<gt, BT, 0, st>>>(pass, A, tile_seg.get(), ctl.get(), soa, tile_off.get(), blpos.get(),
                                            grpos.get());
          PPTKG_CHECK_LAUNCH();
          k_swap<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa, blpos.get(), grpos.get());
          PPTKG_CHECK_LAUNCH();
        }
        k_children<T, D><<<gs, 128, 0, st>>>(A, lvl, recs, B, smallL.get(), small_capn, small_cap, ctl.get());
        PPTKG_CHECK_LAUNCH();
        levels = lvl + 1;
        // the host looks at the next level's size every fourth level only;
        // kernels of a level without segments exit at once
        if (levels % 4 == 0) {
          int h = 0;
          PPTKG_CUDA(cudaMemcpyAsync(&h, &ctl.get()->level_cnt[lvl + 1], sizeof(int), cudaMemcpyDeviceToHost, st));
          PPTKG_CUDA(cudaStreamSynchronize(st));
          if (h == 0) break;
        }
      }
    }
    BuildCtl hctl;
    PPTKG_CUDA(cudaMemcpyAsync(&hctl, ctl.get(), sizeof(BuildCtl), cudaMemcpyDeviceToHost, st));
    PPTKG_CUDA(cudaStreamSynchronize(st));
    if (hctl.status == 7) continue;  // small list too short: retry with more room
    if (hctl.status) throw Error(E_DEVICE, "device build: partition check failed (code " + std::to_string(hctl.status) + ")");
    if (levels >= MAX_LEVELS) throw Error(E_DEVICE, "device build: more than 4096 levels of large nodes");
    depth = levels;
    if (hctl.nsmall > 0) {
      Stage st_sub("build.subtree", st);
      PPTKG_CUDA(cudaFuncSetAttribute(k_subtree<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      int per_sm = 1, nsm = 1;
      PPTKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subtree<T, D>, SUB_THREADS, smem));
      PPTKG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, tree->device));
      const int grid = std::max(1, std::min(hctl.nsmall, std::max(per_sm, 1) * nsm));
      k_subtree<T, D><<<grid, SUB_THREADS, smem, st>>>(smallL.get(), soa, recs, tree->root_rec, small_cap, cap_list,
                                                       max_leaf, thr, (int)rec_cap, ctl.get());
      PPTKG_CHECK_LAUNCH();
      PPTKG_CUDA(cudaMemcpyAsync(&hctl, ctl.get(), sizeof(BuildCtl), cudaMemcpyDeviceToHost, st));
      PPTKG_CUDA(cudaStreamSynchronize(st));
      if (hctl.status)
        throw Error(E_DEVICE, "device build: subtree check failed (code " + std::to_string(hctl.status) + ")");
    }
    tree->n_recs = hctl.rec_count;
    tree->levels = levels;
    depth = std::max(depth, hctl.depth);
    break;
  }
  if ((size_t)tree->n_recs > rec_cap) throw Error(E_DEVICE, "device build: record capacity exceeded");
  tree->depth = depth;
  std::unique_ptr<Stage> st_rec(new Stage("build.records", st));
  PPTKG_CUDA(dev_malloc(&tree->recs, std::max(tree->n_recs, 1) * sizeof(Rec<T, D>), st));
  if (tree->n_recs)
    PPTKG_CUDA(cudaMemcpyAsync(tree->recs, recs, tree->n_recs * sizeof(Rec<T, D>), cudaMemcpyDeviceToDevice, st));
  recbuf.release();
  st_rec.reset();

  // tree-ordered points and the forward map
  std::unique_ptr<Stage> st_fin(new Stage("build.finish", st));
  PointRec<T, D>* pts = nullptr;
  PPTKG_CUDA(dev_malloc((void**)&pts, std::max<int64_t>(nv, 1) * sizeof(PointRec<T, D>), st));
  tree->pts = pts;
  PPTKG_CUDA(dev_malloc((void**)&tree->fwd, std::max<int64_t>(n, 1) * sizeof(int), st));
  if (n > 0) PPTKG_CUDA(cudaMemsetAsync(tree->fwd, 0xff, n * sizeof(int), st));
  if (nv > 0) {
    k_finish<T, D><<<div_up(nv, 256), 256, 0, st>>>(soa, nv, pts, tree->fwd);
    PPTKG_CHECK_LAUNCH();
  }

  st_fin.reset();
  // traversal hierarchy cut at `bucket` points
  {
    Stage st_tn("build.tnodes", st);
    make_tnodes<T, D>(tree.get(), bucket, st);
  }

  Stage st_root("build.root", st);
  Rec<T, D> r0;
  int root0 = -1;
  PPTKG_CUDA(cudaMemcpyAsync(&root0, tree->root_rec, sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (root0 >= 0) {
    PPTKG_CUDA(cudaMemcpyAsync(&r0, (Rec<T, D>*)tree->recs + root0, sizeof(r0), cudaMemcpyDeviceToHost, st));
    PPTKG_CUDA(cudaStreamSynchronize(st));
    for (int d = 0; d < D; d++) {
      tree->root_lo[d] = (double)r0.lo[d];
      tree->root_hi[d] = (double)r0.hi[d];
    }
  }
  if constexpr (std::is_integral<T>::value) lower_points<T, D>(tree.get(), st);
  return tree.release();
}

template <typename T, int D>
TreeBase* build_tree(const T* d_in, int64_t n, int max_leaf, double thr, int bucket, cudaStream_t st) {
  const int64_t off[2] = {0, n};
  return build_forest<T, D>(d_in, n, off, 1, max_leaf, thr, bucket, st);
}

template <typename T, int D>
void make_tnodes(TreeBase* tree, int bucket, cudaStream_t st) {
  if (tree->tnodes) {
    dev_free(tree->tnodes, st);
    tree->tnodes = nullptr;
  }
  if (bucket < 1) bucket = 1;
  tree->bucket = bucket;
  const int nr = tree->n_recs;
  const Rec<T, D>* recs = (const Rec<T, D>*)tree->recs;
  BuildBuf<int> flag(nr + 1, st), tid(nr + 1, st);
  int nt = 0;
  if (nr > 0) {
    k_tflag<T, D><<<div_up(nr, 256), 256, 0, st>>>(recs, nr, bucket, flag.get());
    PPTKG_CHECK_LAUNCH();
    exclusive_scan<int, int>(flag.get(), tid.get(), nr, tid.get() + nr, st);
    PPTKG_CUDA(cudaMemcpyAsync(&nt, tid.get() + nr, sizeof(int), cudaMemcpyDeviceToHost, st));
    PPTKG_CUDA(cudaStreamSynchronize(st));
  }
  TNode<T, D>* nodes = nullptr;
  // a capture-ready forest keeps the capacity that its rebuilds fill
  const int64_t cap = tree->capture ? std::max<int64_t>(tree->cap_tnodes, (int64_t)nt + tree->ncloud)
                                    : (int64_t)nt + tree->ncloud;
  if (tree->capture) tree->cap_tnodes = cap;
  PPTKG_CUDA(dev_malloc((void**)&nodes, (size_t)cap * sizeof(TNode<T, D>), st));
  tree->tnodes = nodes;
  tree->n_tnodes = (int)cap;
  if (nt > 0) {
    k_tfill<T, D><<<div_up(nr, 256), 256, 0, st>>>(recs, nr, flag.get(), tid.get(), nodes);
    PPTKG_CHECK_LAUNCH();
  }
  k_troots<T, D><<<div_up(tree->ncloud, 128), 128, 0, st>>>(recs, tree->root_rec, tree->valid_off, tree->ncloud,
                                                            nr > 0 ? flag.get() : nullptr, tid.get(), nt, nodes,
                                                            tree->root_tnode);
  PPTKG_CHECK_LAUNCH();
  tree->root_tnode_h.resize(tree->ncloud);
  PPTKG_CUDA(cudaMemcpyAsync(tree->root_tnode_h.data(), tree->root_tnode, sizeof(int) * tree->ncloud,
                             cudaMemcpyDeviceToHost, st));
  if (!tree->capture) tree->tdepth = tree->depth + 2;
  if constexpr (std::is_integral<T>::value) lower_tnodes<T, D>(tree, st);
  PPTKG_CUDA(cudaStreamSynchronize(st));
}

#ifndef PPTKG_BUILD_INT
// ------------------------------------------------------ capture mode ----
// Build status of a rebuild: the device checks of the build kernels, code
// 20 when the new data needs a deeper tree than the capacity planned for
// (large segments left after the last of the cap_levels levels, or a depth
// beyond the traversal stacks' tdepth) and 21 when it needs more records.
// meta: valid points, records, depth.
static __global__ void k_rebuild_status(const BuildCtl* ctl, int levels_cap, int tdepth, int* status, int64_t* meta,
                                        const int64_t* valid_off, int ncloud) {
  int levels = 0;
  for (int l = 0; l < levels_cap; l++)
    if (ctl->level_cnt[l] > 0) levels = l + 1;
  const int depth = ctl->depth > levels ? ctl->depth : levels;
  if (ctl->status) atomicExch(status, ctl->status == 6 ? 21 : 10 + ctl->status);
  if (ctl->level_cnt[levels_cap] > 0 || depth + 2 > tdepth) atomicExch(status, 20);
  meta[0] = valid_off[ncloud];
  meta[1] = ctl->rec_count;
  meta[2] = depth;
  meta[3] = 0;
}

template <typename T, int D>
void forest_capture_ready(TreeBase* t, cudaStream_t st) {
  if (t->capture) return;
  if (t->rec_dtype != F32 && t->rec_dtype != F64) throw Error(E_TYPE, "capture mode needs float32 or float64 points");
  int cap_list;
  size_t smem;
  const int small_cap = small_capacity<T, D>(t->max_leaf, cap_list, smem);
  const int64_t n = t->n;
  t->cap_levels = std::min(t->levels + 8, MAX_LEVELS);
  const int64_t seg_cap = n / (small_cap + 1) + 2;
  // small segments: at most two children of every large segment of every
  // level, plus the clouds' roots
  const int64_t small = 2 * (int64_t)t->cap_levels * (seg_cap + 1) + t->ncloud + 64;
  if (small > INT32_MAX) throw Error(E_INVALID, "forest too large for capture mode");
  t->cap_small = (int)small;
  // records and traversal nodes: twice the first build's counts (a tree
  // over n points has at most 2n - 1 records); a rebuild that needs more
  // stops with code 21
  t->cap_recs = std::min<int64_t>(2 * n + 64, 2 * (int64_t)t->n_recs + 4096);
  // (the direct build's inner traversal nodes: n_tnodes less the clouds'
  // root slots)
  const int64_t live_tnodes = std::max<int64_t>((int64_t)t->n_tnodes - t->ncloud, 0);
  t->cap_tnodes = std::min<int64_t>(t->cap_recs, 2 * live_tnodes + 4096) + t->ncloud;
  if (t->cap_recs > INT32_MAX / 2 || t->cap_tnodes > INT32_MAX / 2)
    throw Error(E_INVALID, "forest too large for capture mode");
  int per_sm = 1, nsm = 1;
  PPTKG_CUDA(cudaFuncSetAttribute(k_subtree<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  PPTKG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_subtree<T, D>, SUB_THREADS, smem));
  PPTKG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, t->device));
  t->cap_subgrid = std::max(per_sm, 1) * nsm;
  // capacity-sized arrays, current contents kept
  auto grow = [&](void** p, size_t have, size_t want) {
    void* q = nullptr;
    PPTKG_CUDA(dev_malloc(&q, std::max<size_t>(want, 1), st));
    if (have) PPTKG_CUDA(cudaMemcpyAsync(q, *p, have, cudaMemcpyDeviceToDevice, st));
    if (*p) dev_free(*p, st);
    *p = q;
  };
  grow(&t->pts, (size_t)t->nv * sizeof(PointRec<T, D>), (size_t)n * sizeof(PointRec<T, D>));
  grow(&t->recs, (size_t)t->n_recs * sizeof(Rec<T, D>), (size_t)t->cap_recs * sizeof(Rec<T, D>));
  grow(&t->tnodes, (size_t)t->n_tnodes * sizeof(TNode<T, D>), (size_t)t->cap_tnodes * sizeof(TNode<T, D>));
  t->n_tnodes = (int)t->cap_tnodes;
  t->tdepth += 8;
  if (!t->dev_meta) PPTKG_CUDA(dev_malloc((void**)&t->dev_meta, 4 * sizeof(int64_t), st));
  t->capture = true;
  PPTKG_CUDA(cudaStreamSynchronize(st));
}

template <typename T, int D>
void rebuild_forest(TreeBase* t, const T* d_in, cudaStream_t st, int* status) {
  if (!t->capture) throw Error(E_INVALID, "rebuild needs a capture-ready forest");
  Stage stage("rebuild", st);
  const int64_t n = t->n;
  const int ncloud = t->ncloud;
  // valid rows and per-cloud valid offsets, all on the device
  BuildBuf<int> flag(n + 1, st), off(n + 1, st);
  if (n > 0) {
    k_valid<T, D><<<div_up(n, 256), 256, 0, st>>>(d_in, n, flag.get());
    PPTKG_CHECK_LAUNCH();
  }
  exclusive_scan<int, int>(flag.get(), off.get(), n, off.get() + n, st);
  k_cloud_off<<<div_up(ncloud + 1, 256), 256, 0, st>>>(off.get(), t->orig_off, ncloud, t->valid_off);
  PPTKG_CHECK_LAUNCH();
  BuildBuf<T> xs((size_t)D * n + 1, st);
  BuildBuf<int> ids(n + 1, st);
  SoA<T, D> soa;
  for (int d = 0; d < D; d++) soa.x[d] = xs.get() + (size_t)d * n;
  soa.id = ids.get();
  if (n > 0) {
    k_compact<T, D><<<div_up(n, 256), 256, 0, st>>>(d_in, n, flag.get(), off.get(), soa);
    PPTKG_CHECK_LAUNCH();
  }
  flag.release();
  off.release();
  int cap_list;
  size_t smem;
  const int small_cap = small_capacity<T, D>(t->max_leaf, cap_list, smem);
  const int rec_cap = (int)t->cap_recs;
  Rec<T, D>* recs = (Rec<T, D>*)t->recs;
  const int seg_cap = (int)(n / (small_cap + 1) + 2);
  const int max_tiles = (int)(n / TILE) + seg_cap + 2;
  BuildBuf<BuildCtl> ctl(1, st);
  PPTKG_CUDA(cudaMemsetAsync(ctl.get(), 0, sizeof(BuildCtl), st));
  PPTKG_CUDA(cudaMemsetAsync(t->root_rec, 0xff, sizeof(int) * ncloud, st));
  BuildBuf<Seg<T, D>> segL[2] = {BuildBuf<Seg<T, D>>(seg_cap, st), BuildBuf<Seg<T, D>>(seg_cap, st)};
  BuildBuf<Seg<T, D>> smallL(t->cap_small, st);
  k_roots<T, D><<<div_up(ncloud, 128), 128, 0, st>>>(t->valid_off, t->orig_off, ncloud, small_cap, segL[0].get(),
                                                      smallL.get(), t->cap_small, ctl.get());
  PPTKG_CHECK_LAUNCH();
  {
    // a fixed number of levels; the kernels of a level without segments
    // return at once
    BuildBuf<int> blpos(n + 1, st), grpos(n + 1, st);
    BuildBuf<int> tile_seg(max_tiles, st);
    BuildBuf<long long> tile_cnt(max_tiles, st), tile_off(max_tiles, st);
    const unsigned gt = (unsigned)std::min(max_tiles, level_grid(t->device));
    const unsigned gq = (unsigned)std::min(seg_cap, level_grid(t->device));
    const unsigned gs = (unsigned)div_up(seg_cap, 128);
    for (int lvl = 0; lvl < t->cap_levels; lvl++) {
      Seg<T, D>* A = segL[lvl & 1].get();
      Seg<T, D>* B = segL[(lvl + 1) & 1].get();
      k_tiles<T, D><<<1, 1024, 0, st>>>(A, lvl, tile_seg.get(), ctl.get());
      PPTKG_CHECK_LAUNCH();
      k_seg_init<T, D><<<gs, 128, 0, st>>>(A, lvl, ctl.get());
      PPTKG_CHECK_LAUNCH();
      k_bbox<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa);
      PPTKG_CHECK_LAUNCH();
      k_node<T, D><<<gs, 128, 0, st>>>(A, lvl, ctl.get(), recs, rec_cap, t->root_rec, t->max_leaf, t->empty_split);
      PPTKG_CHECK_LAUNCH();
      k_count<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa);
      PPTKG_CHECK_LAUNCH();
      for (int pass = 1; pass <= 2; pass++) {
        k_flags<T, D><<<gt, BT, 0, st>>>(pass, A, tile_seg.get(), ctl.get(), soa, tile_cnt.get());
        PPTKG_CHECK_LAUNCH();
        k_tscan<T, D><<<gq, 256, 0, st>>>(A, lvl, tile_cnt.get(), tile_off.get(), ctl.get());
        PPTKG_CHECK_LAUNCH();
        k_scatter<T, D><<<gt, BT, 0, st>>>(pass, A, tile_seg.get(), ctl.get(), soa, tile_off.get(), blpos.get(),
                                          grpos.get());
        PPTKG_CHECK_LAUNCH();
        k_swap<T, D><<<gt, BT, 0, st>>>(A, tile_seg.get(), ctl.get(), soa, blpos.get(), grpos.get());
        PPTKG_CHECK_LAUNCH();
      }
      k_children<T, D><<<gs, 128, 0, st>>>(A, lvl, recs, B, smallL.get(), t->cap_small, small_cap, ctl.get());
      PPTKG_CHECK_LAUNCH();
    }
  }
  // the persistent subtree kernel takes the small segments; blocks without
  // work return
  k_subtree<T, D><<<t->cap_subgrid, SUB_THREADS, smem, st>>>(smallL.get(), soa, recs, t->root_rec, small_cap, cap_list,
                                                             t->max_leaf, t->empty_split, rec_cap, ctl.get());
  PPTKG_CHECK_LAUNCH();
  k_rebuild_status<<<1, 1, 0, st>>>(ctl.get(), t->cap_levels, t->tdepth, status, t->dev_meta, t->valid_off, ncloud);
  PPTKG_CHECK_LAUNCH();
  // tree-ordered points and the forward map
  if (n > 0) {
    PPTKG_CUDA(cudaMemsetAsync(t->fwd, 0xff, n * sizeof(int), st));
    k_finish<T, D><<<div_up(n, 256), 256, 0, st>>>(soa, (int)n, (PointRec<T, D>*)t->pts, t->fwd,
                                                   t->valid_off + ncloud);
    PPTKG_CHECK_LAUNCH();
  }
  // traversal hierarchy over the live records
  BuildBuf<int> tflag(rec_cap + 1, st), tid(rec_cap + 1, st);
  const int* nrec_dev = &ctl.get()->rec_count;
  k_tflag<T, D><<<div_up(rec_cap, 256), 256, 0, st>>>(recs, rec_cap, t->bucket, tflag.get(), nrec_dev);
  PPTKG_CHECK_LAUNCH();
  exclusive_scan<int, int>(tflag.get(), tid.get(), rec_cap, tid.get() + rec_cap, st);
  TNode<T, D>* nodes = (TNode<T, D>*)t->tnodes;
  // inner nodes take the slots below cap_tnodes - ncloud, the clouds' root
  // slots the last ncloud
  const int node_lim = (int)(t->cap_tnodes - ncloud);
  k_tfill<T, D><<<div_up(rec_cap, 256), 256, 0, st>>>(recs, rec_cap, tflag.get(), tid.get(), nodes, nrec_dev,
                                                      node_lim, status);
  PPTKG_CHECK_LAUNCH();
  k_troots<T, D><<<div_up(ncloud, 128), 128, 0, st>>>(recs, t->root_rec, t->valid_off, ncloud, tflag.get(),
                                                      tid.get(), node_lim, nodes, t->root_tnode);
  PPTKG_CHECK_LAUNCH();
}

template <typename T, int D>
void forest_sync(TreeBase* t, cudaStream_t st) {
  if (!t->capture) return;
  int64_t meta[4] = {0, 0, 0, 0};
  PPTKG_CUDA(cudaMemcpyAsync(meta, t->dev_meta, sizeof(meta), cudaMemcpyDeviceToHost, st));
  t->valid_off_h.resize(t->ncloud + 1);
  PPTKG_CUDA(cudaMemcpyAsync(t->valid_off_h.data(), t->valid_off, sizeof(int64_t) * (t->ncloud + 1),
                             cudaMemcpyDeviceToHost, st));
  t->root_tnode_h.resize(t->ncloud);
  PPTKG_CUDA(cudaMemcpyAsync(t->root_tnode_h.data(), t->root_tnode, sizeof(int) * t->ncloud, cudaMemcpyDeviceToHost,
                             st));
  int root0 = -1;
  PPTKG_CUDA(cudaMemcpyAsync(&root0, t->root_rec, sizeof(int), cudaMemcpyDeviceToHost, st));
  PPTKG_CUDA(cudaStreamSynchronize(st));
  if (meta[1] > 0) {  // a rebuild ran
    t->nv = meta[0];
    t->n_recs = (int)std::min<int64_t>(meta[1], t->cap_recs);  // (a rebuild past the capacity stops there)
    t->depth = (int)meta[2];
  }
  if (root0 >= 0 && root0 < t->n_recs) {  // the first cloud's root box (saved with the tree)
    Rec<T, D> r0;
    PPTKG_CUDA(cudaMemcpyAsync(&r0, (const Rec<T, D>*)t->recs + root0, sizeof(r0), cudaMemcpyDeviceToHost, st));
    PPTKG_CUDA(cudaStreamSynchronize(st));
    for (int d = 0; d < D; d++) {
      t->root_lo[d] = (double)r0.lo[d];
      t->root_hi[d] = (double)r0.hi[d];
    }
  }
}
#endif  // PPTKG_BUILD_INT

#ifndef PPTKG_BUILD_INT
size_t TreeBase::device_bytes() const {
  size_t ps = (dtype == F64 ? 8 : 4) * dim + 4;
  ps = (ps + 15) / 16 * 16;
  return ps * nv + 4 * n;
}

TreeBase::~TreeBase() {
  // stream-ordered release on the stream the tree was built on
  if (pts) dev_free(pts, stream);
  if (recs) dev_free(recs, stream);
  if (tnodes) dev_free(tnodes, stream);
  if (fwd) dev_free(fwd, stream);
  if (root_rec) dev_free(root_rec, stream);
  if (root_tnode) dev_free(root_tnode, stream);
  if (valid_off) dev_free(valid_off, stream);
  if (orig_off) dev_free(orig_off, stream);
  if (slot_off) dev_free(slot_off, stream);
  if (warp_cloud) dev_free(warp_cloud, stream);
  if (dev_meta) dev_free(dev_meta, stream);
}

#endif  // PPTKG_BUILD_INT

#define PPTKG_INST_BUILD(T, D)                                                                                  \
  template TreeBase* build_tree<T, D>(const T*, int64_t, int, double, int, cudaStream_t);                      \
  template TreeBase* build_forest<T, D>(const T*, int64_t, const int64_t*, int, int, double, int, cudaStream_t); \
  template void make_tnodes<T, D>(TreeBase*, int, cudaStream_t);

#define PPTKG_INST_CAPTURE(T, D)                                              \
  template void forest_capture_ready<T, D>(TreeBase*, cudaStream_t);          \
  template void rebuild_forest<T, D>(TreeBase*, const T*, cudaStream_t, int*); \
  template void forest_sync<T, D>(TreeBase*, cudaStream_t);

// This file builds float32 / float64 trees; build_int.cu includes it with
// PPTKG_BUILD_INT set and builds the eight integer point types.
#ifndef PPTKG_BUILD_INT
PPTKG_INST_CAPTURE(float, 3)
PPTKG_INST_CAPTURE(double, 3)
PPTKG_INST_CAPTURE(float, 2)
PPTKG_INST_CAPTURE(double, 2)
PPTKG_INST_CAPTURE(float, 4)
PPTKG_INST_CAPTURE(double, 4)
PPTKG_INST_BUILD(float, 3)
PPTKG_INST_BUILD(double, 3)
PPTKG_INST_BUILD(float, 2)
PPTKG_INST_BUILD(double, 2)
PPTKG_INST_BUILD(float, 4)
PPTKG_INST_BUILD(double, 4)
#else
#define PPTKG_INST_BUILD_DIMS(T) PPTKG_INST_BUILD(T, 2) PPTKG_INST_BUILD(T, 3) PPTKG_INST_BUILD(T, 4)
PPTKG_INST_BUILD_DIMS(int8_t)
PPTKG_INST_BUILD_DIMS(int16_t)
PPTKG_INST_BUILD_DIMS(int32_t)
PPTKG_INST_BUILD_DIMS(int64_t)
PPTKG_INST_BUILD_DIMS(uint8_t)
PPTKG_INST_BUILD_DIMS(uint16_t)
PPTKG_INST_BUILD_DIMS(uint32_t)
PPTKG_INST_BUILD_DIMS(uint64_t)
#endif

}  // namespace pptkg

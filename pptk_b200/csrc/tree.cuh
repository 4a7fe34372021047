// Device-resident k-d tree layout.
//
// The build reproduces the reference tree exactly (pptk/kdtree/src/
// kdtree-impl.h:248-329, 773-818): the same point permutation, the same
// split and empty-split ("trim") nodes.  It leaves three products in HBM:
//
//  * PointRec[nv]  -- the valid points in tree order, each with its original
//                     index (the reference's points_ + reverse_indices_,
//                     kdtree.h:236-248), 16 B for float32 xyz;
//  * Rec[n_recs]   -- one record per reference split node or leaf range, with
//                     its tight bounding box and the empty-split chain that
//                     precedes it (kept to prove tree identity);
//  * TNode[n_tnodes] -- the traversal hierarchy: the reference tree cut at
//                     nodes of at most `bucket` points, each node holding both
//                     children's tight boxes, so one 64 B broadcast load per
//                     warp decides both children.
//
// The traversal only needs boxes that contain their points: every result is
// decided by point distances computed exactly as the reference does, so the
// tighter boxes change the amount of work, never an answer.
#pragma once

#include <vector>

#include "common.cuh"

namespace pptkg {

template <typename T, int D>
struct alignas(16) PointRec {
  T c[D];
  int32_t id;  // original index of the point
};

// Build record of one reference node range [begin, end).
template <typename T, int D>
struct Rec {
  T lo[D], hi[D];   // tight bounding box of the range
  T split_val;      // valid when split_dim >= 0
  int32_t begin, end;
  int32_t split_index;
  int32_t left, right;  // child records, -1 when absent
  int8_t split_dim;     // -1: leaf range
  int8_t ntrim;         // empty splits performed before this node (<= 2D)
  uint8_t trim[2 * D];  // each: dim * 2 + side (0: low side trimmed, 1: high)
};

// Traversal node: two children, each either an inner node or a leaf bucket.
template <typename T, int D>
struct alignas(16) TNode {
  T lo[2][D], hi[2][D];  // children's tight boxes
  int32_t ref[2];        // >= 0: TNode index; < 0: leaf, begin = -ref - 1
  int32_t cnt[2];        // points under the child (0: no child)
};

template <typename T, int D>
struct TreeView {
  const PointRec<T, D>* pts;
  const TNode<T, D>* nodes;
  int32_t nv;
  int32_t depth;    // traversal stack bound (TNode levels)
  int32_t n_nodes;  // TNode count: no traversal visits more nodes than this
  int32_t root;     // TNode where this tree's traversals start
  const int32_t* fwd;  // original row -> tree position
  int32_t n_in;        // original rows (entries of fwd)
  int32_t pts_cap;     // point records allocated (nv, or n for a capture-ready forest)
  int* err;            // PPTKG_BOUNDS_CHECK builds: first failed check (site code); else null

  // Index checks of the PPTKG_BOUNDS_CHECK build: an index outside [0, n)
  // records `site` in *err (the first failure wins) and reads element 0
  // instead, so a corrupt index is reported, never dereferenced.  In the
  // normal build they are the identity.
  __device__ __forceinline__ int checked(int i, int n, int site) const {
#ifdef PPTKG_BOUNDS_CHECK
    if (i < 0 || i >= n) {
      if (err) atomicCAS(err, 0, site);
      return 0;
    }
#endif
    return i;
  }
  __device__ __forceinline__ const PointRec<T, D>& pt(int i) const { return pts[checked(i, pts_cap, 1)]; }
  __device__ __forceinline__ int pos_of(const int32_t* map, int o) const { return map[checked(o, n_in, 2)]; }
  __device__ __forceinline__ int node_index(int i) const { return checked(i, n_nodes, 3); }
};

// Host-side owner of one device tree, or of a forest of independent trees
// built together over consecutive row ranges (clouds) of one point array.
// Tree positions, record ranges and leaf references are global over the
// concatenated array; cloud c's points occupy positions
// [valid_off[c], valid_off[c+1]) and its traversals start at root_tnode[c].
struct TreeBase {
  // dtype: type of the traversal data (points, TNodes), F32 or F64.
  // rec_dtype: the input point type, in which the tree was built and its
  // records are kept; an integer tree's traversal data is stored as the
  // float values the reference's distance type (float) gives its coordinates.
  int dtype = F32, dim = 3, rec_dtype = F32;
  int64_t n = 0, nv = 0;
  int n_recs = 0, n_tnodes = 0, depth = 0, tdepth = 0, bucket = 32;
  int max_leaf = 10;
  double empty_split = 0.2;
  int device = 0;
  cudaStream_t stream = 0;  // allocations are stream-ordered on this stream
  void* pts = nullptr;      // PointRec<T, D>[nv]
  void* recs = nullptr;     // Rec<T, D>[n_recs]
  void* tnodes = nullptr;   // TNode<T, D>[n_tnodes]
  int32_t* fwd = nullptr;   // original index -> tree position, -1 if dropped
  int ncloud = 1;
  int32_t* root_rec = nullptr;    // device [ncloud]: root record per cloud (-1: no valid point)
  int32_t* root_tnode = nullptr;  // device [ncloud]
  int64_t* valid_off = nullptr;   // device [ncloud + 1]
  int64_t* orig_off = nullptr;    // device [ncloud + 1]
  std::vector<int32_t> root_tnode_h;
  int64_t n_slots = 0;             // forest query slots (cached slot map)
  int64_t* slot_off = nullptr;     // device [ncloud + 1]
  int32_t* warp_cloud = nullptr;   // device [n_slots / 32]
  std::vector<int64_t> valid_off_h, orig_off_h;
  double root_lo[4] = {0, 0, 0, 0}, root_hi[4] = {0, 0, 0, 0};
  int levels = 0;  // grid-wide build levels of the last direct build
  // Capture mode (forest_capture_ready): the arrays have their capacities
  // (points n, records cap_recs, traversal nodes cap_tnodes, query slots
  // n_slots) and rebuild_forest issues no host synchronisation and no
  // allocation whose size depends on device data, so it can be captured
  // into a CUDA graph.  The host-side counts (nv, valid_off_h, n_recs,
  // depth) are those of the last direct build or forest_sync; dev_meta
  // holds the device's {nv, n_recs, depth, 0} of the last rebuild.
  bool capture = false;
  int cap_levels = 0, cap_small = 0, cap_subgrid = 0;
  int64_t cap_recs = 0, cap_tnodes = 0;
  int64_t* dev_meta = nullptr;
  size_t device_bytes() const;
  ~TreeBase();
};

}  // namespace pptkg

// Device k-d tree builder (exact replica of the reference tree).
#pragma once

#include <memory>

#include "tree.cuh"

namespace pptkg {

// Working structure-of-arrays copy of the valid points during the build.
template <typename T, int D>
struct SoA {
  T* x[D];
  int* id;
};

// Builds the tree over n contiguous AoS points already on the device.
// Rows with a NaN/inf coordinate are dropped, as in the reference.
template <typename T, int D>
TreeBase* build_tree(const T* d_points, int64_t n, int max_leaf, double empty_split, int bucket, cudaStream_t st);

// Builds one tree per cloud over the consecutive row ranges
// [orig_off[c], orig_off[c+1]) of the same point array (host offsets,
// ncloud + 1 entries), each exactly the tree the reference builds for that
// cloud alone.
template <typename T, int D>
TreeBase* build_forest(const T* d_points, int64_t n, const int64_t* orig_off_h, int ncloud, int max_leaf,
                       double empty_split, int bucket, cudaStream_t st);

// (Re)derives the traversal hierarchy for a bucket size.
template <typename T, int D>
void make_tnodes(TreeBase* tree, int bucket, cudaStream_t st);

// Capture mode of a forest built by build_forest (float32 / float64):
// forest_capture_ready gives its arrays their capacities and fixes the
// launch shapes (at most the direct build's levels + 8 grid-wide levels);
// rebuild_forest then rebuilds every cloud's tree from new coordinates of
// the same rows (d_points, device) into those arrays with no host
// synchronisation, so that it can be captured into a CUDA graph.  Its
// device checks land in *status (code 20: the data needs more levels than
// planned).  forest_sync reads the counts of the last rebuild back into the
// host fields (nv, valid offsets, records, depth).
template <typename T, int D>
void forest_capture_ready(TreeBase* t, cudaStream_t st);
template <typename T, int D>
void rebuild_forest(TreeBase* t, const T* d_points, cudaStream_t st, int* status);
template <typename T, int D>
void forest_sync(TreeBase* t, cudaStream_t st);

}  // namespace pptkg

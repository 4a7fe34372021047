// Trees of integer point types (int8 ... uint64; kdtree_wrapper.cpp:15-55):
// the builder of build.cu instantiated for them in a translation unit of its
// own.  Their traversal data is lowered to float after the build (see
// lower_points / lower_tnodes), so queries use the float kernels.
#define PPTKG_BUILD_INT 1
#include "build.cu"

// kNN and r-near query paths of 4-d trees (kdtree_wrapper.cpp:15-55 builds
// and queries trees of dim 2, 3 and 4): the templates of query.cu,
// instantiated for dimension 4 in a translation unit of their own.
#define PPTKG_QUERY_DIM 4
#include "query.cu"

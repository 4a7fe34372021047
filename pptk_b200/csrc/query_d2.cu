// kNN and r-near query paths of 2-d trees (kdtree_wrapper.cpp:15-55 builds
// and queries trees of dim 2, 3 and 4): the templates of query.cu,
// instantiated for dimension 2 in a translation unit of their own.
#define PPTKG_QUERY_DIM 2
#include "query.cu"

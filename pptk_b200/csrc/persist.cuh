// Tree persistence (persist.cu): save a built tree to one host buffer and
// load it back onto the current device.
#pragma once

#include <vector>

#include "tree.cuh"

namespace pptkg {

std::vector<char> save_tree(const TreeBase* t, cudaStream_t st);
TreeBase* load_tree(const char* buf, size_t size, cudaStream_t st);

}  // namespace pptkg

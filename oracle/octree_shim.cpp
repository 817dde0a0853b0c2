// Test infrastructure: exposes the library's balanced coarse aggregation
// (urban-sph_a100_b200/csrc/octree.h, host code that coarse.cu runs before
// it assembles the coarse operator) to the CPU tests through a C entry point,
// so that its invariants are checked without a GPU.  Nothing in the library
// links this file.
#include <cstring>
#include <vector>

#include "octree.h"

extern "C" int octree_aggregates_c(const int *cell, int nmem, int B, int NI, int NJ, int NK, int maxagg, int *box) {
    if (!cell || !box || nmem < 0 || B < 1 || NI < 1 || NJ < 1 || NK < 1 || maxagg < 1) return -1;
    const std::vector<int> c(cell, cell + 3 * (size_t)nmem);
    const std::vector<int> out = sph::octree_aggregates(c, nmem, B, NI, NJ, NK, maxagg);
    if (!out.empty()) std::memcpy(box, out.data(), sizeof(int) * out.size());
    return 0;
}

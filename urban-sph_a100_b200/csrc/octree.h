// Balanced coarse aggregates of the two-level preconditioner (host code,
// used by coarse.cu; also compiled on its own by the CPU tests).
#pragma once
#include <algorithm>
#include <utility>
#include <vector>

namespace sph {

// Balanced aggregates (ppe_coarse_block = -B): start from blocks of B^3
// cells and split the block holding the most rows into its (up to eight)
// non-empty octants, again and again, while the aggregate count stays within
// maxagg (ppe_coarse_max) and the block is wider than one cell.  On an
// APR-refined deck a block of the refined zone holds eight times the rows of
// a block outside it; splitting by row count gives every aggregate about the
// same number of rows, i.e. aggregates about twice finer (in cells) where the
// particles are.  cell[3k], cell[3k+1], cell[3k+2] are the cell coordinates
// (x, y, z) of member k, in [0, NI) x [0, NJ) x [0, NK); returns the box of
// every member, numbered 0.. (the caller renumbers them by first row).
// Ties between equally full boxes go to the lower box index, so the result
// does not depend on anything but the input.
inline std::vector<int> octree_aggregates(const std::vector<int> &cell, int nmem, int B, int NI, int NJ, int NK,
                                          int maxagg) {
    struct Box {
        int x0, x1, y0, y1, z0, z1;
        std::vector<int> mem;
    };
    std::vector<Box> boxes;
    {
        const int NBx = (NI + B - 1) / B, NBy = (NJ + B - 1) / B;
        std::vector<int> id((size_t)NBx * NBy * ((NK + B - 1) / B), -1);
        for (int k = 0; k < nmem; ++k) {
            const int bx = cell[3 * k] / B, by = cell[3 * k + 1] / B, bz = cell[3 * k + 2] / B;
            int &b = id[((size_t)bz * NBy + by) * NBx + bx];
            if (b < 0) {
                b = (int)boxes.size();
                boxes.push_back(Box{bx * B, std::min(NI, bx * B + B), by * B, std::min(NJ, by * B + B), bz * B,
                                    std::min(NK, bz * B + B), {}});
            }
            boxes[b].mem.push_back(k);
        }
    }
    if ((int)boxes.size() <= maxagg) {
        // largest first (ties: lower box index), each split replaces one box by its non-empty octants
        auto larger = [&](int a, int b) {
            return boxes[a].mem.size() != boxes[b].mem.size() ? boxes[a].mem.size() < boxes[b].mem.size() : a > b;
        };
        std::vector<int> heap;
        for (int b = 0; b < (int)boxes.size(); ++b) heap.push_back(b);
        std::make_heap(heap.begin(), heap.end(), larger);
        while (!heap.empty()) {
            std::pop_heap(heap.begin(), heap.end(), larger);
            const int b = heap.back();
            heap.pop_back();
            Box &bx = boxes[b];
            if (bx.mem.size() < 2) break;   // every remaining box holds at most one row
            const int mx = bx.x1 - bx.x0 > 1 ? bx.x0 + (bx.x1 - bx.x0 + 1) / 2 : bx.x1;
            const int my = bx.y1 - bx.y0 > 1 ? bx.y0 + (bx.y1 - bx.y0 + 1) / 2 : bx.y1;
            const int mz = bx.z1 - bx.z0 > 1 ? bx.z0 + (bx.z1 - bx.z0 + 1) / 2 : bx.z1;
            if (mx == bx.x1 && my == bx.y1 && mz == bx.z1) continue;   // one cell wide: cannot split
            std::vector<int> part[8];
            for (int k : bx.mem)
                part[(cell[3 * k] >= mx ? 1 : 0) | (cell[3 * k + 1] >= my ? 2 : 0) | (cell[3 * k + 2] >= mz ? 4 : 0)]
                    .push_back(k);
            int nonempty = 0;
            for (int q = 0; q < 8; ++q) nonempty += part[q].empty() ? 0 : 1;
            if ((int)boxes.size() + nonempty - 1 > maxagg) break;   // the largest box cannot split any more
            const Box parent = Box{bx.x0, bx.x1, bx.y0, bx.y1, bx.z0, bx.z1, {}};
            bool first = true;
            for (int q = 0; q < 8; ++q) {
                if (part[q].empty()) continue;
                Box child{(q & 1) ? mx : parent.x0, (q & 1) ? parent.x1 : mx, (q & 2) ? my : parent.y0,
                          (q & 2) ? parent.y1 : my, (q & 4) ? mz : parent.z0, (q & 4) ? parent.z1 : mz,
                          std::move(part[q])};
                int id;
                if (first) { boxes[b] = std::move(child); id = b; first = false; }
                else { boxes.push_back(std::move(child)); id = (int)boxes.size() - 1; }
                heap.push_back(id);
                std::push_heap(heap.begin(), heap.end(), larger);
            }
        }
    }
    std::vector<int> agg(nmem, -1);
    for (int b = 0; b < (int)boxes.size(); ++b)
        for (int k : boxes[b].mem) agg[k] = b;
    return agg;
}

}  // namespace sph

// Space-filling-curve renumbering of the mesh at upload time.
#pragma once
#include <cstdint>
#include <vector>

namespace titan {

struct Renumbering {
    // new index -> original index, and the inverse
    std::vector<int32_t> cell_n2o, cell_o2n;
    std::vector<int32_t> face_n2o, face_o2n;
    std::vector<int32_t> node_n2o, node_o2n;
};

// 63-bit Morton key of a point quantised to 21 bits per axis inside [lo, hi].
uint64_t morton3(const double p[3], const double lo[3], const double hi[3]);

// Cells sorted by the Morton key of their centre (mean of the 8 nodes), ties
// by original index; faces by (new index of cells[0], original index); nodes
// by the Morton key of their position. Pure integer permutations: applying
// them and their inverses is bit-exact.
Renumbering sfc_renumber(int64_t nnode, int64_t ncell, int64_t nface, const double* node_xyz,
                         const int32_t* cell_nodes, const int32_t* face_cells);

}  // namespace titan

// Space-filling-curve (Morton / Z-order) renumbering of cells, faces and nodes.
//
// The reference addresses cells, faces and nodes through pointers in
// construction order (Setka::Renumerate, TITAN/source/Setka.cpp:443-465
// assigns the 1-based `number`). On the GPU the face kernel gathers the two
// cells of every face and the cell kernel gathers its six faces, so the
// numbering decides how often those gathers hit the same cache lines. Sorting
// cells along a Z-order curve keeps face neighbours close in memory; faces
// follow their cells[0]; nodes follow the same curve.
#include "renumber.h"

#include <algorithm>
#include <cmath>
#include <numeric>

namespace titan {

static inline uint64_t spread21(uint64_t v) {
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

uint64_t morton3(const double p[3], const double lo[3], const double hi[3]) {
    uint64_t q[3];
    for (int k = 0; k < 3; ++k) {
        const double span = hi[k] - lo[k];
        double u = span > 0.0 ? (p[k] - lo[k]) / span : 0.0;
        u = std::min(std::max(u, 0.0), 1.0);
        q[k] = (uint64_t)std::floor(u * 2097151.0);
    }
    return spread21(q[0]) | (spread21(q[1]) << 1) | (spread21(q[2]) << 2);
}

static std::vector<int32_t> sort_by_key(std::vector<uint64_t>& key) {
    const int64_t n = (int64_t)key.size();
    std::vector<int32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](int32_t a, int32_t b) {
        return key[a] < key[b] || (key[a] == key[b] && a < b);
    });
    return idx;
}

static std::vector<int32_t> invert(const std::vector<int32_t>& p) {
    std::vector<int32_t> q(p.size());
    for (size_t i = 0; i < p.size(); ++i) q[p[i]] = (int32_t)i;
    return q;
}

Renumbering sfc_renumber(int64_t nnode, int64_t ncell, int64_t nface, const double* xyz, const int32_t* cell_nodes,
                         const int32_t* face_cells) {
    Renumbering R;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < nnode; ++i)
        for (int k = 0; k < 3; ++k) {
            lo[k] = std::min(lo[k], xyz[3 * i + k]);
            hi[k] = std::max(hi[k], xyz[3 * i + k]);
        }
    std::vector<uint64_t> key(ncell);
    for (int64_t c = 0; c < ncell; ++c) {
        double p[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < 8; ++j)
            for (int k = 0; k < 3; ++k) p[k] += xyz[3 * (int64_t)cell_nodes[8 * c + j] + k];
        for (int k = 0; k < 3; ++k) p[k] /= 8.0;
        key[c] = morton3(p, lo, hi);
    }
    R.cell_n2o = sort_by_key(key);
    R.cell_o2n = invert(R.cell_n2o);

    key.assign(nface, 0);
    for (int64_t f = 0; f < nface; ++f) key[f] = (uint64_t)R.cell_o2n[face_cells[2 * f]];
    R.face_n2o = sort_by_key(key);
    R.face_o2n = invert(R.face_n2o);

    key.assign(nnode, 0);
    for (int64_t i = 0; i < nnode; ++i) key[i] = morton3(xyz + 3 * i, lo, hi);
    R.node_n2o = sort_by_key(key);
    R.node_o2n = invert(R.node_n2o);
    return R;
}

}  // namespace titan

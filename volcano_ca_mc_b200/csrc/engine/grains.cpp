// grains.cpp -- grain labelling for the MC statistics: connected components of equal orientation
// (> 0), von Neumann or Moore connectivity, periodic axes joined, every grain represented by its
// smallest globalIndex (engine/src/mc/Grains.cpp:33-150).  Union-find with path halving; the
// components do not depend on the order of the joins.
#include <stdexcept>

#include "model.hpp"

namespace eng {

namespace {

uint32_t find_root(std::vector<uint32_t>& parent, uint32_t i) {
    while (parent[i] != i) {
        parent[i] = parent[parent[i]];
        i = parent[i];
    }
    return i;
}

int wrap_or_out(int v, int n, bool periodic) {
    if (v >= 0 && v < n) return v;
    if (!periodic) return -1;
    return v < 0 ? v + n : v - n;
}

}  // namespace

GrainLabels label_grains(const CrystalMap& m, bool moore, const bool periodic[3]) {
    const Dims& d = m.dims;
    const size_t n = (size_t)d.cells();
    if (n >= GrainLabels::kNone) throw std::invalid_argument("too many cells to label grains (limit 2^32 - 1)");
    // forward half of the connectivity (the dz, dy, dx order of Neighborhood, in the plane of the
    // two axes of size > 1 for 2D)
    struct Off {
        int dx, dy, dz;
    };
    std::vector<Off> forward;
    const int sizes[3] = {d.nx, d.ny, d.nz};
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                if (dx == 0 && dy == 0 && dz == 0) continue;
                const int o[3] = {dx, dy, dz};
                bool ok = true;
                for (int a = 0; a < 3; ++a)
                    if (sizes[a] == 1 && o[a] != 0) ok = false;
                if (!ok) continue;
                if (!moore && std::abs(dx) + std::abs(dy) + std::abs(dz) != 1) continue;
                if (dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0)))) forward.push_back(Off{dx, dy, dz});
            }
    GrainLabels g;
    g.root.resize(n);
    for (size_t i = 0; i < n; ++i) g.root[i] = (uint32_t)i;
    size_t i = 0;
    for (int z = 0; z < d.nz; ++z)
        for (int y = 0; y < d.ny; ++y)
            for (int x = 0; x < d.nx; ++x, ++i) {
                const int32_t s = m.crystal[i];
                if (s <= 0) continue;
                uint32_t ri = find_root(g.root, (uint32_t)i);
                for (const Off& o : forward) {
                    const int qx = wrap_or_out(x + o.dx, d.nx, periodic[0]);
                    const int qy = wrap_or_out(y + o.dy, d.ny, periodic[1]);
                    const int qz = wrap_or_out(z + o.dz, d.nz, periodic[2]);
                    if (qx < 0 || qy < 0 || qz < 0) continue;
                    const size_t j = (size_t)qx + (size_t)d.nx * ((size_t)qy + (size_t)d.ny * qz);
                    if (m.crystal[j] != s) continue;
                    const uint32_t rj = find_root(g.root, (uint32_t)j);
                    if (rj < ri) {
                        g.root[ri] = rj;
                        ri = rj;
                    } else if (ri < rj) {
                        g.root[rj] = ri;
                    }
                }
            }
    g.size.assign(n, 0);
    for (size_t k = 0; k < n; ++k) {
        if (m.crystal[k] <= 0) {
            g.root[k] = GrainLabels::kNone;
            continue;
        }
        const uint32_t r = find_root(g.root, (uint32_t)k);
        g.root[k] = r;
        ++g.size[r];
        ++g.cells;
        g.grains += (r == k) ? 1 : 0;
    }
    return g;
}

}  // namespace eng

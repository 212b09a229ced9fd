// common.cu -- host helpers shared by the CA and MC halves of libvca.so: the error channel of the
// C ABI, neighbourhood tables and the spill-level priority flood.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <queue>
#include <string>
#include <utility>
#include <vector>

#include "vca.h"
#include "vca_device.cuh"
#include "vca_internal.h"

namespace vca {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

vca_status cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VCA_ERR_NOMEM : VCA_ERR_CUDA;
}

// TerrainGenerator::fillDepressions (engine/src/terrain/TerrainGenerator.cpp:86-161): priority
// flood from the outlets (non-periodic edges; on a fully wrapped map, the lowest columns).  A column
// is closed by the first open neighbour taken from the queue, at level max(own height, that
// neighbour's level); levels are taken in nondecreasing order, so the filled surface (the lowest
// level over all paths to an outlet of the highest column on the path) does not depend on the order
// inside one level.  Heights are small integers, so the queue is a bucket per level (a stack of
// columns linked through `next`): linear time.  A height range too wide for buckets uses a heap.
std::vector<int32_t> fill_depressions(const std::vector<int32_t>& h, int nx, int ny, bool px, bool py) {
    const size_t n = h.size();
    std::vector<int32_t> filled = h;
    if (n == 0) return filled;
    std::vector<char> closed(n, 0);
    const auto mm = std::minmax_element(h.begin(), h.end());
    const int32_t lo = *mm.first;
    const uint64_t range = (uint64_t)((int64_t)*mm.second - lo) + 1;
    const bool buckets = range <= (uint64_t)std::max<size_t>(n, 1u << 16);
    std::vector<int64_t> head(buckets ? range : 0, -1);
    std::vector<int64_t> next(buckets ? n : 0, -1);
    using Item = std::pair<int32_t, size_t>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> open;
    auto push = [&](size_t i, int32_t level) {
        if (buckets) {
            const size_t b = (size_t)((int64_t)level - lo);
            next[i] = head[b];
            head[b] = (int64_t)i;
        } else {
            open.push({level, i});
        }
    };
    auto seed = [&](size_t i) {
        if (!closed[i]) {
            closed[i] = 1;
            push(i, h[i]);
        }
    };
    bool any = false;
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const bool ex = !px && nx > 1 && (x == 0 || x == nx - 1);
            const bool ey = !py && ny > 1 && (y == 0 || y == ny - 1);
            if (ex || ey) {
                seed((size_t)x + (size_t)nx * y);
                any = true;
            }
        }
    if (!any)
        for (size_t i = 0; i < n; ++i)
            if (h[i] == lo) seed(i);
    const int dx[4] = {-1, 1, 0, 0}, dy[4] = {0, 0, -1, 1};
    size_t cur = 0;  // lowest bucket that may hold columns
    for (;;) {
        size_t i;
        int32_t level;
        if (buckets) {
            while (cur < range && head[cur] < 0) ++cur;
            if (cur == range) break;
            i = (size_t)head[cur];
            head[cur] = next[i];
            level = (int32_t)((int64_t)cur + lo);
        } else {
            if (open.empty()) break;
            i = open.top().second;
            level = open.top().first;
            open.pop();
        }
        const int x = (int)(i % (size_t)nx), y = (int)(i / (size_t)nx);
        for (int d = 0; d < 4; ++d) {
            int sx = x + dx[d], sy = y + dy[d];
            if (sx < 0 || sx >= nx) {
                if (!px || nx == 1) continue;
                sx = (sx + nx) % nx;
            }
            if (sy < 0 || sy >= ny) {
                if (!py || ny == 1) continue;
                sy = (sy + ny) % ny;
            }
            const size_t j = (size_t)sx + (size_t)nx * sy;
            if (closed[j]) continue;
            closed[j] = 1;
            filled[j] = std::max(h[j], level);
            push(j, filled[j]);
        }
    }
    return filled;
}

// Neighbourhood tables (engine/src/core/Neighborhood.cpp:18-119): 2D in the plane of the two
// axes of size > 1 (v outer, u inner), 3D in dz, dy, dx order.
bool build_nb(int kind, int nx, int ny, int nz, NbTable& t) {
    std::memset(&t, 0, sizeof(t));
    const int sizes[3] = {nx, ny, nz};
    int plane[3] = {0, 0, 0}, axes = 0;
    for (int a = 0; a < 3; ++a)
        if (sizes[a] > 1) plane[axes++] = a;
    if (axes < 2) return false;
    auto keep2 = [&](int var, int u, int v) -> bool {
        switch (kind) {
            case VCA_NB_VON_NEUMANN: return std::abs(u) + std::abs(v) == 1;
            case VCA_NB_MOORE: return true;
            case VCA_NB_PENTAGONAL: return var == 0 ? u != -1 : var == 1 ? u != 1 : var == 2 ? v != -1 : v != 1;
            default:
                return var == 0 ? !((u == -1 && v == -1) || (u == 1 && v == 1)) : !((u == -1 && v == 1) || (u == 1 && v == -1));
        }
    };
    auto keep3 = [&](int var, int dx, int dy, int dz) -> bool {
        switch (kind) {
            case VCA_NB_VON_NEUMANN: return std::abs(dx) + std::abs(dy) + std::abs(dz) == 1;
            case VCA_NB_MOORE: return true;
            default: {
                const int c[6] = {dx != -1, dx != 1, dy != -1, dy != 1, dz != -1, dz != 1};
                return c[var] != 0;
            }
        }
    };
    if (axes == 2) {
        t.variants = kind == VCA_NB_PENTAGONAL ? 4 : kind == VCA_NB_HEXAGONAL ? 2 : 1;
        for (int var = 0; var < t.variants; ++var) {
            int k = 0;
            for (int v = -1; v <= 1; ++v)
                for (int u = -1; u <= 1; ++u) {
                    if ((u == 0 && v == 0) || !keep2(var, u, v)) continue;
                    int d[3] = {0, 0, 0};
                    d[plane[0]] = u;
                    d[plane[1]] = v;
                    for (int a = 0; a < 3; ++a) t.off[var][k][a] = (int8_t)d[a];
                    ++k;
                }
            t.count[var] = k;
        }
    } else {
        if (kind == VCA_NB_HEXAGONAL) return false;
        t.variants = kind == VCA_NB_PENTAGONAL ? 6 : 1;
        for (int var = 0; var < t.variants; ++var) {
            int k = 0;
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if ((dx == 0 && dy == 0 && dz == 0) || !keep3(var, dx, dy, dz)) continue;
                        t.off[var][k][0] = (int8_t)dx;
                        t.off[var][k][1] = (int8_t)dy;
                        t.off[var][k][2] = (int8_t)dz;
                        ++k;
                    }
            t.count[var] = k;
        }
    }
    return true;
}

}  // namespace vca

extern "C" {
const char* vca_last_error(void) { return vca::g_last_error.c_str(); }
const char* vca_version(void) { return "vca 2 sm_100a (lava CA + Potts checkerboard MC)"; }
}

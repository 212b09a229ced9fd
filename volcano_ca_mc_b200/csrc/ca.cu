// ca.cu -- lava cellular automaton on sm_100a: kernels and the vca_ca_* half of the C ABI.
//
// One CA step (LavaCA::step, engine/src/ca/LavaCA.hpp:230-247) is three launches on the handle's
// stream:
//   ca_schedule_kernel  (ACTIVE sweep only) -- which 64 x TY x TZ tiles can change this step;
//   ca_descent_kernel   -- D(n) of every supported LAVA cell (computeDescent, LavaCA.hpp:551-566);
//   ca_rules_kernel     -- the rules cur -> next for every cell of the scheduled tiles
//                          (updateLava / updateClassic, LavaCA.hpp:1109-1201), the step counters,
//                          and, in its last block, finishStep (LavaCA.hpp:1206-1229).
// The state is double-buffered SoA planes (type u8, flowId i32, temp f32, solidStep u16,
// arrivalStep u16) in pitched rows; which buffer is current is the parity of the device-side
// step counter, so a run of steps needs no host round trip until the stop test.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
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

constexpr int kThreads = 256;   // threads of a tile block: 16 per 64-cell row, 16 rows
constexpr int kTileX = 64;
constexpr int kMaxDrop = 16;    // LavaCA::kMaxDrop (LavaCA.hpp:1293)
constexpr int kSmemRowBytes = 72;  // 4 pad + 64 cells + 4 pad
constexpr int kMaxHaloRows = 36;   // (TY + 2) * (TZ + 2) for TY = TZ = 4

// ------------------------------------------------------------------------------------------
// Addressing with the reference's frame semantics: a coordinate one step outside the interior
// is the opposite layer on a periodic axis, else the VOID frame (Boundary::applyWith,
// engine/src/core/Boundary.hpp:75-131).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int64_t pidx(const CaGeom& g, int x, int y, int z) {
    return (int64_t)x + (int64_t)g.P * ((int64_t)y + (int64_t)g.ny * z);
}
__device__ __forceinline__ bool wrap_axis(int& v, int n, int periodic) {
    if (v >= 0 && v < n) return true;
    if (!periodic || n == 1) return false;
    v = v < 0 ? v + n : v - n;
    return true;
}
__device__ __forceinline__ bool resolve(const CaGeom& g, int& x, int& y, int& z) {
    return wrap_axis(x, g.nx, g.per[0]) && wrap_axis(y, g.ny, g.per[1]) && wrap_axis(z, g.nz, g.per[2]);
}
__device__ __forceinline__ int type_at(const CaGeom& g, const uint8_t* T, int x, int y, int z) {
    if (!resolve(g, x, y, z)) return kVoid;
    return __ldg(T + pidx(g, x, y, z));
}
// LavaCA::spillAt (LavaCA.hpp:383): the column wraps.
__device__ __forceinline__ int spill_at(const CaKernelArgs& k, int x, int y) {
    const int nx = k.g.nx, ny = k.g.ny;
    x = x < 0 ? x + nx : (x >= nx ? x - nx : x);
    y = y < 0 ? y + ny : (y >= ny ? y - ny : y);
    return __ldg(k.spill + x + (int64_t)nx * y);
}
__device__ __forceinline__ bool solid_ground(int t) { return t == kRock || t == kBasalt; }

// LavaCA::hasSupport (LavaCA.hpp:390-399).
__device__ bool has_support(const CaKernelArgs& k, const uint8_t* T, int x, int y, int z) {
    if (z == 0) return true;
    const int below = type_at(k.g, T, x, y, z - 1);
    if (solid_ground(below)) return true;
    return below == kLava && k.spill != nullptr && z - 1 < spill_at(k, x, y);
}
// LavaCA::dropDepth (LavaCA.hpp:404-414).
__device__ int drop_depth(const CaKernelArgs& k, const uint8_t* T, int x, int y, int z) {
    for (int d = 0; d <= kMaxDrop && z - d >= 0; ++d) {
        if (d > 0 && type_at(k.g, T, x, y, z - d) != kAir) return -1;
        if (has_support(k, T, x, y, z - d)) return d;
    }
    return kMaxDrop;
}
// LavaCA::descent (LavaCA.hpp:421-429).
__device__ int descent(const CaKernelArgs& k, const uint8_t* T, int x, int y, int z) {
    int best = 0;
    const CaTables* tb = k.tables;
    const int nside = tb->nside;
    for (int s = 0; s < nside; ++s) {
        const int ax = x + tb->side[s][0], ay = y + tb->side[s][1];
        if (type_at(k.g, T, ax, ay, z) == kAir) best = max(best, drop_depth(k, T, ax, ay, z));
    }
    return best;
}

// CandidateVote (engine/src/ca/CaRules.hpp:127-183).
struct Vote {
    int n;
    int32_t ids[26];
    int counts[26];
    float max_temp[26];
    __device__ void add(int32_t id, float t) {
        for (int i = 0; i < n; ++i)
            if (ids[i] == id) {
                ++counts[i];
                max_temp[i] = fmaxf(max_temp[i], t);
                return;
            }
        ids[n] = id;
        counts[n] = 1;
        max_temp[n] = t;
        ++n;
    }
    // Most votes; ties: tied ids ascending, pick hashRand(seed, t, idx, TieBreak) % k.
    __device__ int winner(uint64_t prefix, uint64_t gidx) const {
        if (n == 1) return 0;
        int best = 0;
        for (int i = 0; i < n; ++i) best = max(best, counts[i]);
        int tied[26];
        int k = 0;
        for (int i = 0; i < n; ++i)
            if (counts[i] == best) tied[k++] = i;
        if (k == 1) return tied[0];
        for (int i = 1; i < k; ++i) {
            const int t = tied[i];
            int j = i;
            while (j > 0 && ids[tied[j - 1]] > ids[t]) {
                tied[j] = tied[j - 1];
                --j;
            }
            tied[j] = t;
        }
        const uint64_t r = hash_salt(hash_index(prefix, gidx), kSaltTieBreak);
        return tied[(int)(r % (uint64_t)k)];
    }
};

__device__ __forceinline__ int variant_of(const CaKernelArgs& k, uint64_t prefix, uint64_t gidx) {
    if (k.tables->nb.variants == 1) return 0;
    return (int)fast_mod(hash_salt(hash_index(prefix, gidx), kSaltNeighborhood), k.var_mod);
}

// LavaCA::tryPonding (LavaCA.hpp:443-461).
__device__ void try_ponding(const CaKernelArgs& k, const uint8_t* T, const int32_t* F, const float* Te, int x, int y,
                            int z, Vote& v) {
    if (k.spill == nullptr || z > __ldg(k.spill + x + (int64_t)k.g.nx * y)) return;
    const int bz = z - 1;
    if (type_at(k.g, T, x, y, bz) != kLava) return;
    if (!has_support(k, T, x, y, bz)) return;
    const int nh = k.g.ny > 1 ? 4 : 2;
    const int hx[4] = {-1, 1, 0, 0}, hy[4] = {0, 0, -1, 1};
    for (int h = 0; h < nh; ++h) {
        const int n = type_at(k.g, T, x + hx[h], y + hy[h], bz);
        if (n == kAir || n == kVoid) return;
    }
    const int64_t b = pidx(k.g, x, y, bz);
    v.add(__ldg(F + b), __fsub_rn(__ldg(Te + b), k.cool_lateral));
}

// LavaCA::gatherLavaCandidates (LavaCA.hpp:465-519).
__device__ void gather_lava(const CaKernelArgs& k, const uint8_t* T, const int32_t* F, const float* Te, int x, int y,
                            int z, uint64_t prefix, uint64_t gidx, Vote& v) {
    v.n = 0;
    const NbTable& nb = k.tables->nb;
    const int var = variant_of(k, prefix, gidx);
    const int cnt = nb.count[var];
    int c_drop = -100;
    for (int i = 0; i < cnt; ++i) {
        const int dx = nb.off[var][i][0], dy = nb.off[var][i][1], dz = nb.off[var][i][2];
        if (dz < 0) {
            if (k.ponding && dx == 0 && dy == 0) try_ponding(k, T, F, Te, x, y, z, v);
            continue;
        }
        int sx = x + dx, sy = y + dy, sz = z + dz;
        if (!resolve(k.g, sx, sy, sz)) continue;
        const int64_t s = pidx(k.g, sx, sy, sz);
        if (__ldg(T + s) != kLava) continue;
        float cooling;
        if (dz > 0 && dx == 0 && dy == 0) {
            cooling = k.cool_fall;
        } else {
            const int d = k.desc[s];
            if (d < 0) continue;
            if (c_drop == -100) c_drop = drop_depth(k, T, x, y, z);
            if (dz > 0) {
                if (c_drop != 0 || d != 1) continue;
                cooling = k.cool_fall;
            } else {
                if (c_drop != d || (d == 1 && k.diag_falls)) continue;
                cooling = k.cool_lateral;
            }
        }
        v.add(__ldg(F + s), __fsub_rn(__ldg(Te + s), cooling));
    }
}

// updateClassic's vote (LavaCA.hpp:1176-1182).
__device__ void gather_classic(const CaKernelArgs& k, const uint8_t* T, const int32_t* F, int x, int y, int z,
                               uint64_t prefix, uint64_t gidx, Vote& v) {
    v.n = 0;
    const NbTable& nb = k.tables->nb;
    const int var = variant_of(k, prefix, gidx);
    for (int i = 0; i < nb.count[var]; ++i) {
        int sx = x + nb.off[var][i][0], sy = y + nb.off[var][i][1], sz = z + nb.off[var][i][2];
        if (!resolve(k.g, sx, sy, sz)) continue;
        const int64_t s = pidx(k.g, sx, sy, sz);
        if (__ldg(T + s) == kLava) v.add(__ldg(F + s), 0.0f);
    }
}

// ------------------------------------------------------------------------------------------
// Tile decoding.  Tile id = tx + tiles_x * (ty + tiles_y * tz).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void tile_origin(const CaGeom& g, uint32_t tile, int& x0, int& y0, int& z0) {
    const int tx = (int)(tile % (uint32_t)g.tiles_x);
    const uint32_t r = tile / (uint32_t)g.tiles_x;
    const int ty = (int)(r % (uint32_t)g.tiles_y);
    const int tz = (int)(r / (uint32_t)g.tiles_y);
    x0 = tx * kTileX;
    y0 = ty * g.TY;
    z0 = tz * g.TZ;
}

// ------------------------------------------------------------------------------------------
// Schedule (ACTIVE sweep): tile t is processed in step s when a tile within one tile of it held
// LAVA after step s-1 (only cells within one cell of LAVA, and LAVA itself, can change: the
// front set of LavaCA::frontCandidates, LavaCA.hpp:907-940), or when t changed in step s-1
// (its two buffers differ and next must be refreshed).  Other tiles keep both buffers equal.
// ------------------------------------------------------------------------------------------
__global__ void ca_schedule_kernel(CaKernelArgs k) {
    const CaCtrl* ctrl = k.ctrl;
    if (ctrl->stop) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1, nxt = cur ^ 1;
    const CaGeom& g = k.g;
    if (blockIdx.x == 0 && threadIdx.x == 0) k.ctrl->list_count[nxt] = 0;
    const uint32_t* fin = k.tile_flags[cur];
    uint32_t* fout = k.tile_flags[nxt];
    // Warp-uniform loop: every lane of a warp runs the same iterations, so the ballot below sees all 32.
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < k.ntiles; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t tile = base + threadIdx.x;
        bool process = false;
        if (tile < k.ntiles) {
            const int tx = (int)(tile % g.tiles_x);
            const uint64_t r = tile / g.tiles_x;
            const int ty = (int)(r % g.tiles_y);
            const int tz = (int)(r / g.tiles_y);
            process = (fin[tile] & 2u) != 0;
            for (int dz = -1; dz <= 1 && !process; ++dz) {
                int zz = tz + dz;
                if (!wrap_axis(zz, g.tiles_z, g.per[2])) continue;
                for (int dy = -1; dy <= 1 && !process; ++dy) {
                    int yy = ty + dy;
                    if (!wrap_axis(yy, g.tiles_y, g.per[1])) continue;
                    for (int dx = -1; dx <= 1; ++dx) {
                        int xx = tx + dx;
                        if (!wrap_axis(xx, g.tiles_x, g.per[0])) continue;
                        if (fin[xx + (uint64_t)g.tiles_x * (yy + (uint64_t)g.tiles_y * zz)] & 1u) {
                            process = true;
                            break;
                        }
                    }
                }
            }
            fout[tile] = 0;
        }
        // Warp-aggregated append keeps neighbouring tiles next to each other in the list.
        const unsigned ballot = __ballot_sync(0xFFFFFFFFu, process);
        const unsigned lane = threadIdx.x & 31;
        unsigned slot = 0;
        if (lane == 0 && ballot) slot = atomicAdd(&k.ctrl->list_count[cur], (unsigned)__popc(ballot));
        slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
        if (process) k.tile_list[cur][slot + __popc(ballot & ((1u << lane) - 1u))] = (uint32_t)tile;
    }
}

// ------------------------------------------------------------------------------------------
// D(n) of the LAVA cells of the scheduled tiles (computeDescent / frontDescent,
// LavaCA.hpp:551-566, 877-888).  Only cells that are LAVA now are read back by the rules.
// ------------------------------------------------------------------------------------------
__global__ __launch_bounds__(kThreads) void ca_descent_kernel(CaKernelArgs k) {
    const CaCtrl* ctrl = k.ctrl;
    if (ctrl->stop) return;
    if (k.classic) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1;
    const CaGeom& g = k.g;
    const uint8_t* T = k.type[cur];
    const uint64_t count = k.dense ? k.ntiles : ctrl->list_count[cur];
    const int xq = threadIdx.x & 15, row = threadIdx.x >> 4;
    const int ly = row % g.TY, lz = row / g.TY;
    for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t tile = k.dense ? (uint32_t)i : k.tile_list[cur][i];
        int x0, y0, z0;
        tile_origin(g, tile, x0, y0, z0);
        const int y = y0 + ly, z = z0 + lz, x = x0 + 4 * xq;
        if (y >= g.ny || z >= g.nz) continue;
        const int64_t p = pidx(g, x, y, z);
        const uint32_t w = *reinterpret_cast<const uint32_t*>(T + p);
        uint32_t lava = __vcmpeq4(w, 0x02020202u);
        while (lava) {
            const int j = (__ffs(lava) - 1) >> 3;
            lava &= ~(0xFFu << (8 * j));
            const int xx = x + j;
            int8_t d = -1;
            if (has_support(k, T, xx, y, z)) d = (int8_t)descent(k, T, xx, y, z);
            k.desc[p + j] = d;
        }
    }
}

// ------------------------------------------------------------------------------------------
// Rules.  A block handles one 64 x TY x TZ tile at a time (persistent loop over the schedule):
//   1. stage the tile's cell types with a one-cell halo in shared memory (frame semantics at the
//      grid edges), and mark per cell whether LAVA lies within one cell (3x3x3): only such AIR
//      cells can gain lava (CaRules.hpp:69-79);
//   2. each thread updates 4 consecutive cells of a row: 128-bit loads and stores of the flowId
//      and temp planes, 64-bit of the two step planes, 32-bit of the type plane;
//   3. AIR cells next to lava run the exact candidate gathering and vote from global memory.
// ------------------------------------------------------------------------------------------
__global__ __launch_bounds__(kThreads) void ca_rules_kernel(CaKernelArgs k) {
    __shared__ __align__(16) uint8_t s_type[kMaxHaloRows * kSmemRowBytes];
    __shared__ uint32_t s_dil[kMaxHaloRows * 16];
    __shared__ unsigned long long s_red[4][kThreads / 32];
    __shared__ bool s_last;

    CaCtrl* ctrl = k.ctrl;
    if (ctrl->stop) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1, nxt = cur ^ 1;
    const CaGeom& g = k.g;
    const uint8_t* T = k.type[cur];
    const int32_t* F = k.flow[cur];
    const float* Te = k.temp[cur];
    const uint64_t count = k.dense ? k.ntiles : ctrl->list_count[cur];

    // StepCtx (LavaCA.hpp:542-546)
    const bool erupting = (int64_t)t < (int64_t)k.eruption_steps;
    const uint16_t stamp = (uint16_t)min(t, 65535u);
    uint64_t prefix = 0;
    bool have_prefix = false;

    const int tid = threadIdx.x;
    const int xq = tid & 15, row = tid >> 4;
    const int ly = row % g.TY, lz = row / g.TY;
    const int hy_on = g.ny > 1 ? 1 : 0, hz_on = g.nz > 1 ? 1 : 0;
    const int HY = hy_on ? g.TY + 2 : 1, HZ = hz_on ? g.TZ + 2 : 1;
    const int halo_rows = HY * HZ;

    unsigned int my_active = 0, my_changed = 0, my_born = 0;
    unsigned int tiles_done = 0;

    for (uint64_t i = blockIdx.x; i < count; i += gridDim.x) {
        const uint32_t tile = k.dense ? (uint32_t)i : k.tile_list[cur][i];
        int x0, y0, z0;
        tile_origin(g, tile, x0, y0, z0);
        ++tiles_done;

        // 1. stage types with halo
        for (int w = tid; w < halo_rows * 16; w += kThreads) {
            const int r = w >> 4, word = w & 15;
            int yy = y0 - hy_on + r % HY, zz = z0 - hz_on + r / HY;
            uint32_t v = 0xFFFFFFFFu;
            int xw = x0 + 4 * word;
            if (wrap_axis(yy, g.ny, g.per[1]) && wrap_axis(zz, g.nz, g.per[2])) {
                v = *reinterpret_cast<const uint32_t*>(T + pidx(g, xw, yy, zz));
                // Periodic x with padded rows: the frame cell x = nx inside this word is the copy of x = 0.
                if (g.per[0] && g.nx < g.P && xw <= g.nx && g.nx < xw + 4) {
                    const int b = g.nx - xw;
                    const uint32_t c0 = T[pidx(g, 0, yy, zz)];
                    v = (v & ~(0xFFu << (8 * b))) | (c0 << (8 * b));
                }
            }
            *reinterpret_cast<uint32_t*>(s_type + r * kSmemRowBytes + 4 + 4 * word) = v;
        }
        for (int e = tid; e < halo_rows * 2; e += kThreads) {
            const int r = e >> 1, right = e & 1;
            int yy = y0 - hy_on + r % HY, zz = z0 - hz_on + r / HY;
            int xx = right ? x0 + kTileX : x0 - 1;
            uint8_t v = kVoid;
            if (right && xx > g.nx) {
                v = kVoid;  // beyond the frame: only padding cells see it
            } else if (wrap_axis(xx, g.nx, g.per[0]) && wrap_axis(yy, g.ny, g.per[1]) && wrap_axis(zz, g.nz, g.per[2])) {
                v = T[pidx(g, xx, yy, zz)];
            }
            s_type[r * kSmemRowBytes + (right ? 4 + kTileX : 3)] = v;
        }
        __syncthreads();
        for (int w = tid; w < halo_rows * 16; w += kThreads) {
            const int r = w >> 4, word = w & 15;
            const uint8_t* rowp = s_type + r * kSmemRowBytes + 4 + 4 * word;
            const uint32_t m = __vcmpeq4(*reinterpret_cast<const uint32_t*>(rowp), 0x02020202u);
            const uint32_t left = rowp[-1] == kLava ? 0xFFu : 0u;
            const uint32_t rightb = rowp[4] == kLava ? 0xFF000000u : 0u;
            s_dil[w] = m | (m << 8) | (m >> 8) | left | rightb;
        }
        __syncthreads();

        const int y = y0 + ly, z = z0 + lz, x = x0 + 4 * xq;
        bool any_lava = false, any_changed = false;
        if (y < g.ny && z < g.nz) {
            const int hr = (ly + hy_on) + HY * (lz + hz_on);
            uint32_t w = *reinterpret_cast<const uint32_t*>(s_type + hr * kSmemRowBytes + 4 + 4 * xq);
            // Padding cells (x >= nx) are VOID: the staged copy may hold the periodic image of x = 0 there.
            if (x + 4 > g.nx) {
                const int keep = max(0, g.nx - x);
                w |= 0xFFFFFFFFu << (8 * keep);
            }
            uint32_t near = 0;
            for (int dz = -hz_on; dz <= hz_on; ++dz)
                for (int dy = -hy_on; dy <= hy_on; ++dy) near |= s_dil[(hr + dy + HY * dz) * 16 + xq];

            const int64_t p = pidx(g, x, y, z);
            int4 f4 = *reinterpret_cast<const int4*>(F + p);
            float4 t4 = *reinterpret_cast<const float4*>(Te + p);
            uint2 s2 = *reinterpret_cast<const uint2*>(k.solid[cur] + p);
            uint2 a2 = *reinterpret_cast<const uint2*>(k.arrival[cur] + p);
            int32_t fl[4] = {f4.x, f4.y, f4.z, f4.w};
            float te[4] = {t4.x, t4.y, t4.z, t4.w};
            uint16_t so[4] = {(uint16_t)(s2.x & 0xFFFF), (uint16_t)(s2.x >> 16), (uint16_t)(s2.y & 0xFFFF),
                              (uint16_t)(s2.y >> 16)};
            uint16_t ar[4] = {(uint16_t)(a2.x & 0xFFFF), (uint16_t)(a2.x >> 16), (uint16_t)(a2.y & 0xFFFF),
                              (uint16_t)(a2.y >> 16)};
            uint32_t wout = w;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const uint8_t ty = (w >> (8 * j)) & 0xFF;
                if (ty == kAir) {
                    if ((near >> (8 * j)) & 0xFF) {
                        const int xx = x + j;
                        const uint64_t gi = (uint64_t)xx + (uint64_t)g.nx * ((uint64_t)y + (uint64_t)g.ny * z);
                        if (!have_prefix) {
                            prefix = hash_prefix(k.seed, t);
                            have_prefix = true;
                        }
                        Vote v;
                        if (!k.classic) {
                            gather_lava(k, T, F, Te, xx, y, z, prefix, gi, v);
                        } else {
                            gather_classic(k, T, F, xx, y, z, prefix, gi, v);
                        }
                        if (v.n > 0) {
                            const int wi = v.winner(prefix, gi);
                            const float wt = k.classic ? 0.0f : v.max_temp[wi];
                            if (k.classic || wt >= k.solidus) {
                                wout = (wout & ~(0xFFu << (8 * j))) | ((uint32_t)kLava << (8 * j));
                                fl[j] = v.ids[wi];
                                te[j] = wt;
                                so[j] = 0;
                                ar[j] = stamp;
                                ++my_active;
                                ++my_changed;
                                ++my_born;
                                any_changed = true;
                                any_lava = true;
                            }
                        }
                    }
                } else if (ty == kLava) {
                    if (!k.classic) {
                        const float before = te[j];
                        float nt;
                        bool vent = false;
                        const int32_t f = fl[j];
                        if (erupting && f > 0 && f < k.vent_slots) {
                            const int4 vc = __ldg(k.vents + f);
                            vent = vc.x == x + j && vc.y == y && vc.z == z;
                        }
                        nt = vent ? k.erupt_temp : __fsub_rn(before, k.cool_ambient);
                        if (nt < k.solidus) {
                            wout = (wout & ~(0xFFu << (8 * j))) | ((uint32_t)kBasalt << (8 * j));
                            so[j] = stamp;
                            te[j] = nt;
                            ++my_changed;
                            any_changed = true;
                        } else {
                            te[j] = nt;
                            ++my_active;
                            any_lava = true;
                            if (nt != before) {
                                ++my_changed;
                                any_changed = true;
                            }
                        }
                    } else {
                        ++my_active;
                        any_lava = true;
                    }
                }
            }
            *reinterpret_cast<uint32_t*>(k.type[nxt] + p) = wout;
            *reinterpret_cast<int4*>(k.flow[nxt] + p) = make_int4(fl[0], fl[1], fl[2], fl[3]);
            *reinterpret_cast<float4*>(k.temp[nxt] + p) = make_float4(te[0], te[1], te[2], te[3]);
            *reinterpret_cast<uint2*>(k.solid[nxt] + p) =
                make_uint2((uint32_t)so[0] | ((uint32_t)so[1] << 16), (uint32_t)so[2] | ((uint32_t)so[3] << 16));
            *reinterpret_cast<uint2*>(k.arrival[nxt] + p) =
                make_uint2((uint32_t)ar[0] | ((uint32_t)ar[1] << 16), (uint32_t)ar[2] | ((uint32_t)ar[3] << 16));
        }
        const int tl = __syncthreads_or(any_lava);
        const int tc = __syncthreads_or(any_changed);
        if (tid == 0 && !k.dense) k.tile_flags[nxt][tile] = (tl ? 1u : 0u) | (tc ? 2u : 0u);
    }

    // Block sums of the step counters, then finishStep in the last block (LavaCA.hpp:1206-1229).
    const unsigned lane = tid & 31, warp = tid >> 5;
    unsigned a = __reduce_add_sync(0xFFFFFFFFu, my_active);
    unsigned c = __reduce_add_sync(0xFFFFFFFFu, my_changed);
    unsigned b = __reduce_add_sync(0xFFFFFFFFu, my_born);
    if (lane == 0) {
        s_red[0][warp] = a;
        s_red[1][warp] = c;
        s_red[2][warp] = b;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long sa = 0, sc = 0, sb = 0;
        for (int w = 0; w < kThreads / 32; ++w) {
            sa += s_red[0][w];
            sc += s_red[1][w];
            sb += s_red[2][w];
        }
        if (sa) atomicAdd(&ctrl->acc_active, sa);
        if (sc) atomicAdd(&ctrl->acc_changed, sc);
        if (sb) atomicAdd(&ctrl->acc_born, sb);
        if (tiles_done) atomicAdd(&ctrl->acc_tiles, (unsigned long long)tiles_done);
        __threadfence();
        const unsigned ticket = atomicAdd(&ctrl->ticket, 1u);
        s_last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last && tid == 0) {
        __threadfence();
        const unsigned long long active = atomicExch(&ctrl->acc_active, 0ull);
        const unsigned long long changed = atomicExch(&ctrl->acc_changed, 0ull);
        const unsigned long long born = atomicExch(&ctrl->acc_born, 0ull);
        const unsigned long long tiles = atomicExch(&ctrl->acc_tiles, 0ull);
        ctrl->ticket = 0;
        const uint64_t air = ctrl->air - born;
        ctrl->air = air;
        ctrl->lava = active;
        ctrl->tiles_processed += tiles;
        k.hist_active[t] = active;
        k.hist_changed[t] = changed;
        const uint32_t steps = t + 1;
        int stop = VCA_STOP_RUNNING;
        if (!ctrl->classic && active == 0) stop = VCA_STOP_NO_LAVA;
        else if (ctrl->classic && air == 0) stop = VCA_STOP_NO_AIR;
        else if (changed == 0 && !ctrl->random_nb) stop = VCA_STOP_NO_CHANGE;
        else if ((int)steps >= ctrl->max_steps) stop = VCA_STOP_MAX_STEPS;
        ctrl->stop = stop;
        ctrl->steps = steps;
        __threadfence();
    }
}

// ------------------------------------------------------------------------------------------
// Set-up kernels.
// ------------------------------------------------------------------------------------------
// Per-tile LAVA flag of the current state and the LAVA / AIR totals (countInitialState,
// LavaCA.hpp:1252-1280).  One block per tile.
__global__ __launch_bounds__(kThreads) void ca_tile_init_kernel(CaKernelArgs k, int cur) {
    const CaGeom& g = k.g;
    const int xq = threadIdx.x & 15, row = threadIdx.x >> 4;
    const int ly = row % g.TY, lz = row / g.TY;
    __shared__ unsigned long long s_cnt[2];
    if (threadIdx.x == 0) s_cnt[0] = s_cnt[1] = 0;
    __syncthreads();
    for (uint64_t tile = blockIdx.x; tile < k.ntiles; tile += gridDim.x) {
        int x0, y0, z0;
        tile_origin(g, (uint32_t)tile, x0, y0, z0);
        const int y = y0 + ly, z = z0 + lz, x = x0 + 4 * xq;
        unsigned lava = 0, air = 0;
        if (y < g.ny && z < g.nz) {
            const uint32_t w = *reinterpret_cast<const uint32_t*>(k.type[cur] + pidx(g, x, y, z));
            lava = __popc(__vcmpeq4(w, 0x02020202u)) >> 3;
            air = __popc(__vcmpeq4(w, 0u)) >> 3;
            // padding cells are VOID, so they count as neither
        }
        const int any = __syncthreads_or(lava > 0);
        if (threadIdx.x == 0) {
            k.tile_flags[cur][tile] = any ? 1u : 0u;
            k.tile_flags[cur ^ 1][tile] = 0u;
        }
        const unsigned la = __reduce_add_sync(0xFFFFFFFFu, lava);
        const unsigned ai = __reduce_add_sync(0xFFFFFFFFu, air);
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&s_cnt[0], (unsigned long long)la);
            atomicAdd(&s_cnt[1], (unsigned long long)ai);
        }
        __syncthreads();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        atomicAdd(&k.ctrl->acc_active, s_cnt[0]);
        atomicAdd(&k.ctrl->acc_born, s_cnt[1]);
    }
}

// Fill the padding cells x in [nx, P) of every row with VOID (both buffers).
__global__ void ca_pad_kernel(uint8_t* t0, uint8_t* t1, int nx, int P, int64_t rows) {
    const int pad = P - nx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows * pad; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = i / pad;
        const int x = nx + (int)(i % pad);
        t0[r * P + x] = kVoid;
        t1[r * P + x] = kVoid;
    }
}

// ROCK for z < h(x, y) (LavaCA::applyTerrain, LavaCA.hpp:185-194).
__global__ void ca_terrain_kernel(uint8_t* type, const int32_t* heights, int nx, int ny, int nz, int P) {
    const int64_t n = (int64_t)nx * ny * nz;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t r = i / nx;
        const int y = (int)(r % ny);
        const int z = (int)(r / ny);
        const int h = min(heights[x + (int64_t)nx * y], nz);
        if (z < h) type[x + (int64_t)P * r] = kRock;
    }
}

}  // namespace vca

// ============================================================================================
// Host side
// ============================================================================================
using namespace vca;

namespace vca {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

vca_status cuda_fail(cudaError_t e, const char* what) {
    set_error(std::string("CUDA error in ") + what + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? VCA_ERR_NOMEM : VCA_ERR_CUDA;
}

// TerrainGenerator::fillDepressions (engine/src/terrain/TerrainGenerator.cpp:86-161): priority
// flood from the outlets (non-periodic edges; on a fully wrapped map, the lowest columns).
std::vector<int32_t> fill_depressions(const std::vector<int32_t>& h, int nx, int ny, bool px, bool py) {
    const size_t n = h.size();
    std::vector<int32_t> filled = h;
    std::vector<char> closed(n, 0);
    using Item = std::pair<int32_t, size_t>;
    std::priority_queue<Item, std::vector<Item>, std::greater<Item>> open;
    auto seed = [&](size_t i) {
        if (!closed[i]) {
            closed[i] = 1;
            open.push({h[i], i});
        }
    };
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const bool ex = !px && nx > 1 && (x == 0 || x == nx - 1);
            const bool ey = !py && ny > 1 && (y == 0 || y == ny - 1);
            if (ex || ey) seed((size_t)x + (size_t)nx * y);
        }
    if (open.empty() && n > 0) {
        const int32_t lowest = *std::min_element(h.begin(), h.end());
        for (size_t i = 0; i < n; ++i)
            if (h[i] == lowest) seed(i);
    }
    const int dx[4] = {-1, 1, 0, 0}, dy[4] = {0, 0, -1, 1};
    while (!open.empty()) {
        const Item it = open.top();
        open.pop();
        const int x = (int)(it.second % (size_t)nx), y = (int)(it.second / (size_t)nx);
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
            filled[j] = std::max(h[j], it.first);
            open.push({filled[j], j});
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
            default: return var == 0 ? !((u == -1 && v == -1) || (u == 1 && v == 1)) : !((u == -1 && v == 1) || (u == 1 && v == -1));
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

namespace {

CaKernelArgs make_args(const vca_ca* h) {
    CaKernelArgs k;
    std::memset(&k, 0, sizeof(k));
    k.g = h->geom;
    k.classic = h->desc.mode == VCA_MODE_CLASSIC;
    k.ponding = h->desc.ponding != 0;
    k.dense = h->desc.sweep == VCA_SWEEP_DENSE;
    k.seed = h->desc.seed;
    k.max_steps = h->desc.max_steps;
    k.eruption_steps = h->desc.eruption_steps;
    k.erupt_temp = h->desc.erupt_temp;
    k.solidus = h->desc.solidus_temp;
    k.cool_ambient = h->desc.cooling_ambient;
    k.cool_lateral = h->desc.cooling_lateral;
    k.cool_fall = h->desc.cooling_fall;
    k.var_mod = make_fastmod((uint64_t)h->tables_host.nb.variants);
    bool diag = false;
    for (int v = 0; v < h->tables_host.nb.variants; ++v)
        for (int i = 0; i < h->tables_host.nb.count[v]; ++i) {
            const int8_t* o = h->tables_host.nb.off[v][i];
            if (o[2] == -1 && (o[0] != 0 || o[1] != 0)) diag = true;
        }
    k.diag_falls = diag;
    for (int b = 0; b < 2; ++b) {
        k.type[b] = h->type[b];
        k.flow[b] = h->flow[b];
        k.temp[b] = h->temp[b];
        k.solid[b] = h->solid[b];
        k.arrival[b] = h->arrival[b];
        k.tile_flags[b] = h->tile_flags[b];
        k.tile_list[b] = h->tile_list[b];
    }
    k.desc = h->desc_plane;
    k.spill = h->has_terrain ? h->spill : nullptr;
    k.vents = h->vents;
    k.vent_slots = h->vent_slots;
    k.tables = h->tables;
    k.ctrl = h->ctrl;
    k.hist_active = h->hist_active;
    k.hist_changed = h->hist_changed;
    k.ntiles = h->ntiles;
    return k;
}

vca_status check(const vca_ca* h) {
    if (h == nullptr) {
        set_error("null vca_ca handle");
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

// Pull the control block to the host mirror.
vca_status sync_ctrl(vca_ca* h) {
    VCA_CUDA(cudaMemcpyAsync(h->ctrl_host, h->ctrl, sizeof(CaCtrl), cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = (int)h->ctrl_host->steps;
    h->stop = h->ctrl_host->stop;
    return VCA_OK;
}

// Tile flags, LAVA/AIR totals and the initial stop state of the current buffer, and a copy of the
// current buffer into the other one (both buffers equal: the ACTIVE schedule relies on it).
vca_status init_state(vca_ca* h, int steps_done) {
    const int cur = steps_done & 1, oth = cur ^ 1;
    const size_t n = h->plane_cells;
    VCA_CUDA(cudaMemcpyAsync(h->type[oth], h->type[cur], n, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->flow[oth], h->flow[cur], n * 4, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->temp[oth], h->temp[cur], n * 4, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->solid[oth], h->solid[cur], n * 2, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->arrival[oth], h->arrival[cur], n * 2, cudaMemcpyDeviceToDevice, h->stream));
    CaCtrl c;
    std::memset(&c, 0, sizeof(c));
    c.steps = (uint32_t)steps_done;
    c.max_steps = h->desc.max_steps;
    c.random_nb = h->tables_host.nb.variants > 1;
    c.classic = h->desc.mode == VCA_MODE_CLASSIC;
    VCA_CUDA(cudaMemcpyAsync(h->ctrl, &c, sizeof(c), cudaMemcpyHostToDevice, h->stream));
    CaKernelArgs k = make_args(h);
    const int blocks = (int)std::min<uint64_t>(h->ntiles, (uint64_t)h->grid_blocks * 4);
    ca_tile_init_kernel<<<blocks, kThreads, 0, h->stream>>>(k, cur);
    VCA_CUDA(cudaGetLastError());
    if (vca_status s_ = sync_ctrl(h)) return s_;
    CaCtrl* m = h->ctrl_host;
    const uint64_t lava = m->acc_active, air = m->acc_born;
    m->acc_active = 0;
    m->acc_born = 0;
    m->lava = lava;
    m->air = air;
    // LavaCA::countInitialState (LavaCA.hpp:1272-1279)
    int stop = VCA_STOP_RUNNING;
    if (!c.classic && lava == 0) stop = VCA_STOP_NO_LAVA;
    else if (c.classic && air == 0) stop = VCA_STOP_NO_AIR;
    else if (h->desc.max_steps <= steps_done) stop = VCA_STOP_MAX_STEPS;
    m->stop = stop;
    VCA_CUDA(cudaMemcpyAsync(h->ctrl, m, sizeof(CaCtrl), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = steps_done;
    h->stop = stop;
    return VCA_OK;
}

vca_status run_steps(vca_ca* h, int max_new_steps, bool until_stop) {
    if (!h->seeded) {
        set_error("vca_ca: place_seeds or set_state must come before stepping");
        return VCA_ERR_STATE;
    }
    if (h->stop != VCA_STOP_RUNNING) return VCA_OK;
    const CaKernelArgs k = make_args(h);
    VCA_CUDA(cudaEventRecord(h->ev_a, h->stream));
    int chunk = 4;
    int done = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof;
    size_t ev_used = 0;
    while (true) {
        const int n = until_stop ? chunk : std::min(chunk, max_new_steps - done);
        for (int s = 0; s < n; ++s) {
            if (!k.dense) {
                const int threads = 256;
                const int blocks = (int)std::min<uint64_t>((h->ntiles + threads - 1) / threads, 148 * 8);
                ca_schedule_kernel<<<blocks, threads, 0, h->stream>>>(k);
            }
            ca_descent_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k);
            if (h->profile_kernels) {
                while (h->prof_events.size() < ev_used + 2) {
                    cudaEvent_t e;
                    VCA_CUDA(cudaEventCreate(&e));
                    h->prof_events.push_back(e);
                }
                cudaEvent_t e0 = h->prof_events[ev_used], e1 = h->prof_events[ev_used + 1];
                ev_used += 2;
                VCA_CUDA(cudaEventRecord(e0, h->stream));
                ca_rules_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k);
                VCA_CUDA(cudaEventRecord(e1, h->stream));
                prof.push_back({e0, e1});
            } else {
                ca_rules_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k);
            }
        }
        VCA_CUDA(cudaGetLastError());
        done += n;
        if (vca_status s_ = sync_ctrl(h)) return s_;
        if (h->stop != VCA_STOP_RUNNING) break;
        if (!until_stop && done >= max_new_steps) break;
        chunk = std::min(chunk * 2, 256);
    }
    VCA_CUDA(cudaEventRecord(h->ev_b, h->stream));
    VCA_CUDA(cudaEventSynchronize(h->ev_b));
    float ms = 0.f;
    VCA_CUDA(cudaEventElapsedTime(&ms, h->ev_a, h->ev_b));
    h->total_ms += ms;
    if (h->profile_kernels) {
        // Only launches that did work (steps actually taken) count; launches after the stop exit at once.
        const uint64_t real = std::min<uint64_t>(prof.size(), (uint64_t)h->steps);
        for (size_t i = 0; i < prof.size(); ++i) {
            float m = 0.f;
            VCA_CUDA(cudaEventElapsedTime(&m, prof[i].first, prof[i].second));
            if (i < real) {
                h->rules_ms += m;
                ++h->rules_launches;
            }
        }
    }
    return VCA_OK;
}

void free_all(vca_ca* h) {
    if (h->device >= 0) cudaSetDevice(h->device);
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->type[b]);
        cudaFree(h->flow[b]);
        cudaFree(h->temp[b]);
        cudaFree(h->solid[b]);
        cudaFree(h->arrival[b]);
        cudaFree(h->tile_flags[b]);
        cudaFree(h->tile_list[b]);
    }
    cudaFree(h->desc_plane);
    cudaFree(h->spill);
    cudaFree(h->vents);
    cudaFree(h->tables);
    cudaFree(h->ctrl);
    cudaFree(h->hist_active);
    cudaFree(h->hist_changed);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->ev_a) cudaEventDestroy(h->ev_a);
    if (h->ev_b) cudaEventDestroy(h->ev_b);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
}

vca_status upload_vents(vca_ca* h, const vca_vent* vents, int count) {
    int slots = 1;
    for (int i = 0; i < count; ++i) slots = std::max(slots, vents[i].flow_id + 1);
    std::vector<int4> table((size_t)slots, make_int4(-1, -1, -1, 0));
    for (int i = 0; i < count; ++i)
        if (vents[i].flow_id > 0) table[(size_t)vents[i].flow_id] = make_int4(vents[i].x, vents[i].y, vents[i].z, 0);
    cudaFree(h->vents);
    h->vents = nullptr;
    VCA_CUDA(cudaMalloc(&h->vents, sizeof(int4) * table.size()));
    VCA_CUDA(cudaMemcpyAsync(h->vents, table.data(), sizeof(int4) * table.size(), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->vent_slots = slots;
    return VCA_OK;
}

// Copy host planes (unpitched) into the pitched current buffer.
template <class T>
vca_status put_plane(vca_ca* h, T* dst, const T* src) {
    const auto& g = h->geom;
    VCA_CUDA(cudaMemcpy2DAsync(dst, sizeof(T) * (size_t)g.P, src, sizeof(T) * (size_t)g.nx, sizeof(T) * (size_t)g.nx,
                               (size_t)g.ny * g.nz, cudaMemcpyHostToDevice, h->stream));
    return VCA_OK;
}
template <class T>
vca_status get_plane(vca_ca* h, T* dst, const T* src) {
    const auto& g = h->geom;
    VCA_CUDA(cudaMemcpy2DAsync(dst, sizeof(T) * (size_t)g.nx, src, sizeof(T) * (size_t)g.P, sizeof(T) * (size_t)g.nx,
                               (size_t)g.ny * g.nz, cudaMemcpyDeviceToHost, h->stream));
    return VCA_OK;
}

}  // namespace

extern "C" {

const char* vca_last_error(void) { return g_last_error.c_str(); }

const char* vca_version(void) { return "vca 1 sm_100a (lava CA + Potts checkerboard MC)"; }

vca_status vca_ca_create(const vca_ca_desc* d, vca_ca** out) {
    if (d == nullptr || out == nullptr) {
        set_error("vca_ca_create: null argument");
        return VCA_ERR_ARG;
    }
    *out = nullptr;
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    if (nx < 1 || ny < 1 || nz < 1 || (nx > 1) + (ny > 1) + (nz > 1) < 2) {
        set_error("vca_ca_create: the space must be 2D (exactly one size equal to 1) or 3D");
        return VCA_ERR_ARG;
    }
    if ((uint64_t)nx * ny * nz > 2000000000ULL) {
        set_error("vca_ca_create: more than 2 000 000 000 cells");
        return VCA_ERR_ARG;
    }
    if (d->mode == VCA_MODE_LAVA && (nx > 1) + (ny > 1) + (nz > 1) == 2 && ny != 1) {
        set_error("vca_ca_create: a 2D lava space is the x-z cross-section (ny = 1)");
        return VCA_ERR_ARG;
    }
    if (d->max_steps < 0 || d->max_steps > 65535) {
        set_error("vca_ca_create: max_steps must be in 0..65535");
        return VCA_ERR_ARG;
    }
    if (d->neighborhood < 0 || d->neighborhood > 3 || d->boundary < 0 || d->boundary > 1 || d->mode < 0 || d->mode > 1 ||
        d->sweep < 0 || d->sweep > 1) {
        set_error("vca_ca_create: unknown neighborhood, boundary, mode or sweep");
        return VCA_ERR_ARG;
    }
    vca_ca* h = new vca_ca();
    h->desc = *d;
    h->device = d->device;
    if (!build_nb(d->neighborhood, nx, ny, nz, h->tables_host.nb)) {
        delete h;
        set_error("vca_ca_create: the hexagonal neighbourhood is defined in 2D only");
        return VCA_ERR_ARG;
    }
    // side offsets: union of dz == 0 offsets over all variants (LavaCA.hpp:104-112)
    h->tables_host.nside = 0;
    for (int v = 0; v < h->tables_host.nb.variants; ++v)
        for (int i = 0; i < h->tables_host.nb.count[v]; ++i) {
            const int8_t* o = h->tables_host.nb.off[v][i];
            if (o[2] != 0) continue;
            bool dup = false;
            for (int s = 0; s < h->tables_host.nside; ++s)
                dup = dup || (h->tables_host.side[s][0] == o[0] && h->tables_host.side[s][1] == o[1]);
            if (!dup) {
                std::memcpy(h->tables_host.side[h->tables_host.nside], o, 3);
                ++h->tables_host.nside;
            }
        }
    auto fail = [&](vca_status s) {
        free_all(h);
        delete h;
        return s;
    };
    cudaError_t e = cudaSetDevice(d->device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
    cudaDeviceProp prop;
    e = cudaGetDeviceProperties(&prop, d->device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaGetDeviceProperties"));
    if (prop.major < 10) {
        set_error("vca_ca_create: needs an sm_100 (Blackwell) device, found sm_" + std::to_string(prop.major) +
                  std::to_string(prop.minor));
        return fail(VCA_ERR_CUDA);
    }
    auto& g = h->geom;
    g.nx = nx;
    g.ny = ny;
    g.nz = nz;
    g.P = (nx + kTileX - 1) / kTileX * kTileX;
    const bool periodic = d->boundary == VCA_BC_PERIODIC;
    g.per[0] = periodic && nx > 1;
    g.per[1] = periodic && ny > 1;
    g.per[2] = periodic && d->mode == VCA_MODE_CLASSIC && nz > 1;
    if (ny > 1 && nz > 1) {
        g.TY = 4;
        g.TZ = 4;
    } else if (ny == 1) {
        g.TY = 1;
        g.TZ = 16;
    } else {
        g.TY = 16;
        g.TZ = 1;
    }
    g.tiles_x = g.P / kTileX;
    g.tiles_y = (ny + g.TY - 1) / g.TY;
    g.tiles_z = (nz + g.TZ - 1) / g.TZ;
    h->ntiles = (uint64_t)g.tiles_x * g.tiles_y * g.tiles_z;
    h->plane_cells = (size_t)g.P * ny * nz;
    const size_t n = h->plane_cells;
#define ALLOC(ptr, bytes)                                   \
    do {                                                    \
        e = cudaMalloc(&(ptr), (bytes));                    \
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc " #ptr)); \
    } while (0)
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
    for (int b = 0; b < 2; ++b) {
        ALLOC(h->type[b], n);
        ALLOC(h->flow[b], n * 4);
        ALLOC(h->temp[b], n * 4);
        ALLOC(h->solid[b], n * 2);
        ALLOC(h->arrival[b], n * 2);
        ALLOC(h->tile_flags[b], h->ntiles * 4);
        ALLOC(h->tile_list[b], h->ntiles * 4);
    }
    ALLOC(h->desc_plane, n);
    ALLOC(h->tables, sizeof(CaTables));
    ALLOC(h->ctrl, sizeof(CaCtrl));
    ALLOC(h->hist_active, sizeof(unsigned long long) * (size_t)std::max(1, d->max_steps));
    ALLOC(h->hist_changed, sizeof(unsigned long long) * (size_t)std::max(1, d->max_steps));
#undef ALLOC
    e = cudaMallocHost(&h->ctrl_host, sizeof(CaCtrl));
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMallocHost"));
    for (int b = 0; b < 2; ++b) {
        if ((e = cudaMemsetAsync(h->type[b], 0, n, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->flow[b], 0, n * 4, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->temp[b], 0, n * 4, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->solid[b], 0, n * 2, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->arrival[b], 0, n * 2, h->stream)) != cudaSuccess ||
            (e = cudaMemsetAsync(h->tile_flags[b], 0, h->ntiles * 4, h->stream)) != cudaSuccess)
            return fail(cuda_fail(e, "cudaMemsetAsync"));
    }
    if ((e = cudaMemsetAsync(h->desc_plane, 0xFF, n, h->stream)) != cudaSuccess) return fail(cuda_fail(e, "cudaMemsetAsync"));
    if (g.P > nx) {
        ca_pad_kernel<<<256, 256, 0, h->stream>>>(h->type[0], h->type[1], nx, g.P, (int64_t)ny * nz);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(cuda_fail(e, "ca_pad_kernel"));
    }
    e = cudaMemcpyAsync(h->tables, &h->tables_host, sizeof(CaTables), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemcpyAsync tables"));
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ca_rules_kernel, kThreads, 0);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    h->grid_blocks = (int)std::min<uint64_t>(h->ntiles, (uint64_t)prop.multiProcessorCount * std::max(1, per_sm));
    if ((e = cudaEventCreate(&h->ev_a)) != cudaSuccess || (e = cudaEventCreate(&h->ev_b)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaEventCreate"));
    const char* prof = std::getenv("VCA_PROFILE_KERNELS");
    h->profile_kernels = prof != nullptr && prof[0] == '1';
    // An empty vent table and an initial control block (no seeds yet).
    vca_vent none{0, 0, 0, 0};
    vca_status s = upload_vents(h, &none, 0);
    if (s != VCA_OK) return fail(s);
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamSynchronize"));
    *out = h;
    return VCA_OK;
}

vca_status vca_ca_apply_terrain(vca_ca* h, const int32_t* heights) {
    if (vca_status s = check(h)) return s;
    if (heights == nullptr) {
        set_error("vca_ca_apply_terrain: null heights");
        return VCA_ERR_ARG;
    }
    if (h->desc.mode != VCA_MODE_LAVA) {
        set_error("vca_ca_apply_terrain: terrain exists in lava mode only");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const auto& g = h->geom;
    const size_t cols = (size_t)g.nx * g.ny;
    std::vector<int32_t> hv(heights, heights + cols);
    for (auto& v : hv) {
        if (v < 0) {
            set_error("vca_ca_apply_terrain: negative height");
            return VCA_ERR_ARG;
        }
    }
    const std::vector<int32_t> spill = fill_depressions(hv, g.nx, g.ny, g.per[0] != 0, g.per[1] != 0);
    if (h->spill == nullptr) VCA_CUDA(cudaMalloc(&h->spill, sizeof(int32_t) * cols));
    int32_t* dh = nullptr;
    VCA_CUDA(cudaMalloc(&dh, sizeof(int32_t) * cols));
    VCA_CUDA(cudaMemcpyAsync(dh, hv.data(), sizeof(int32_t) * cols, cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->spill, spill.data(), sizeof(int32_t) * cols, cudaMemcpyHostToDevice, h->stream));
    const int cur = h->steps & 1;
    ca_terrain_kernel<<<1184, 256, 0, h->stream>>>(h->type[cur], dh, g.nx, g.ny, g.nz, g.P);
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    cudaFree(dh);
    h->has_terrain = true;
    return VCA_OK;
}

vca_status vca_ca_place_seeds(vca_ca* h, const vca_vent* vents, int count) {
    if (vca_status s = check(h)) return s;
    if (count < 0 || (count > 0 && vents == nullptr)) {
        set_error("vca_ca_place_seeds: bad vent list");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const auto& g = h->geom;
    const int cur = h->steps & 1;
    const float temp = h->desc.mode == VCA_MODE_LAVA ? h->desc.erupt_temp : 0.0f;
    for (int i = 0; i < count; ++i) {
        const vca_vent& v = vents[i];
        if (v.x < 0 || v.x >= g.nx || v.y < 0 || v.y >= g.ny || v.z < 0 || v.z >= g.nz) {
            set_error("vca_ca_place_seeds: vent " + std::to_string(i) + " lies outside the grid");
            return VCA_ERR_ARG;
        }
        // CellState{Lava, flowId, temp, 0, 0} (LavaCA.hpp:219)
        const size_t p = (size_t)v.x + (size_t)g.P * ((size_t)v.y + (size_t)g.ny * v.z);
        const uint8_t lava = VCA_LAVA;
        const uint16_t zero16 = 0;
        VCA_CUDA(cudaMemcpyAsync(h->type[cur] + p, &lava, 1, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaMemcpyAsync(h->flow[cur] + p, &v.flow_id, 4, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaMemcpyAsync(h->temp[cur] + p, &temp, 4, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaMemcpyAsync(h->solid[cur] + p, &zero16, 2, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaMemcpyAsync(h->arrival[cur] + p, &zero16, 2, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaStreamSynchronize(h->stream));  // the sources live on this stack frame
    }
    if (vca_status s = upload_vents(h, vents, count)) return s;
    h->seeded = true;
    return init_state(h, h->steps);
}

vca_status vca_ca_set_state(vca_ca* h, const uint8_t* type, const int32_t* flow_id, const float* temp,
                            const uint16_t* solid_step, const uint16_t* arrival_step, const int32_t* spill,
                            const vca_vent* vents, int vent_count, int steps_done) {
    if (vca_status s = check(h)) return s;
    if (!type || !flow_id || !temp || !solid_step || !arrival_step || steps_done < 0 || vent_count < 0 ||
        (vent_count > 0 && !vents)) {
        set_error("vca_ca_set_state: bad argument");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const auto& g = h->geom;
    const int cur = steps_done & 1;
    if (vca_status s = put_plane(h, h->type[cur], type)) return s;
    if (vca_status s = put_plane(h, h->flow[cur], flow_id)) return s;
    if (vca_status s = put_plane(h, h->temp[cur], temp)) return s;
    if (vca_status s = put_plane(h, h->solid[cur], solid_step)) return s;
    if (vca_status s = put_plane(h, h->arrival[cur], arrival_step)) return s;
    if (spill != nullptr) {
        const size_t cols = (size_t)g.nx * g.ny;
        if (h->spill == nullptr) VCA_CUDA(cudaMalloc(&h->spill, sizeof(int32_t) * cols));
        VCA_CUDA(cudaMemcpyAsync(h->spill, spill, sizeof(int32_t) * cols, cudaMemcpyHostToDevice, h->stream));
        h->has_terrain = true;
    } else {
        h->has_terrain = false;
    }
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    if (vca_status s = upload_vents(h, vents, vent_count)) return s;
    h->seeded = true;
    return init_state(h, steps_done);
}

vca_status vca_ca_step(vca_ca* h, int* running) {
    if (vca_status s = check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = run_steps(h, 1, false)) return s;
    if (running) *running = h->stop == VCA_STOP_RUNNING;
    return VCA_OK;
}

vca_status vca_ca_run(vca_ca* h) {
    if (vca_status s = check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    return run_steps(h, 0, true);
}

vca_status vca_ca_get_info(vca_ca* h, vca_ca_info* out) {
    if (vca_status s = check(h)) return s;
    if (!out) {
        set_error("vca_ca_get_info: null output");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    out->steps = h->steps;
    out->stop_reason = h->stop;
    out->lava_cells = h->ctrl_host->lava;
    out->air_cells = h->ctrl_host->air;
    out->tiles_total = h->ntiles;
    out->tiles_processed = h->ctrl_host->tiles_processed;
    out->cells_per_tile = (uint64_t)kTileX * h->geom.TY * h->geom.TZ;
    return VCA_OK;
}

vca_status vca_ca_history(vca_ca* h, uint64_t* active, uint64_t* changed, int capacity, int* count) {
    if (vca_status s = check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    const int n = std::min(std::max(capacity, 0), h->steps);
    if (n > 0 && active) VCA_CUDA(cudaMemcpyAsync(active, h->hist_active, 8 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    if (n > 0 && changed) VCA_CUDA(cudaMemcpyAsync(changed, h->hist_changed, 8 * (size_t)n, cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    if (count) *count = h->steps;
    return VCA_OK;
}

vca_status vca_ca_download(vca_ca* h, uint8_t* type, int32_t* flow_id, float* temp, uint16_t* solid_step,
                           uint16_t* arrival_step) {
    if (vca_status s = check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    const int cur = h->steps & 1;
    if (type) if (vca_status s = get_plane(h, type, h->type[cur])) return s;
    if (flow_id) if (vca_status s = get_plane(h, flow_id, h->flow[cur])) return s;
    if (temp) if (vca_status s = get_plane(h, temp, h->temp[cur])) return s;
    if (solid_step) if (vca_status s = get_plane(h, solid_step, h->solid[cur])) return s;
    if (arrival_step) if (vca_status s = get_plane(h, arrival_step, h->arrival[cur])) return s;
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_ca_get_spill(vca_ca* h, int32_t* spill) {
    if (vca_status s = check(h)) return s;
    if (!h->has_terrain) {
        set_error("vca_ca_get_spill: no terrain");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemcpy(spill, h->spill, sizeof(int32_t) * (size_t)h->geom.nx * h->geom.ny, cudaMemcpyDeviceToHost));
    return VCA_OK;
}

vca_status vca_ca_timing(vca_ca* h, double* total_ms, double* rules_kernel_ms, uint64_t* rules_launches) {
    if (vca_status s = check(h)) return s;
    if (total_ms) *total_ms = h->total_ms;
    if (rules_kernel_ms) *rules_kernel_ms = h->rules_launches ? h->rules_ms / (double)h->rules_launches : 0.0;
    if (rules_launches) *rules_launches = h->rules_launches;
    return VCA_OK;
}

void vca_ca_destroy(vca_ca* h) {
    if (!h) return;
    free_all(h);
    delete h;
}

}  // extern "C"

// Accessors used by the MC half (mc.cu) to build the crystallisation domain on the device.
namespace vca {
struct CaView {
    const uint8_t* type;
    const uint16_t* solid;
    const uint16_t* arrival;
    int nx, ny, nz, P;
    cudaStream_t stream;
    int device;
};
vca_status ca_view(vca_ca* h, CaView* v) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = sync_ctrl(h)) return s;
    const int cur = h->steps & 1;
    v->type = h->type[cur];
    v->solid = h->solid[cur];
    v->arrival = h->arrival[cur];
    v->nx = h->geom.nx;
    v->ny = h->geom.ny;
    v->nz = h->geom.nz;
    v->P = h->geom.P;
    v->stream = h->stream;
    v->device = h->device;
    return VCA_OK;
}
}  // namespace vca

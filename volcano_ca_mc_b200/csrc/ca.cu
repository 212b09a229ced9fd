// ca.cu -- lava cellular automaton on sm_100a: kernels and the vca_ca_* half of the C ABI.
//
// One CA step (LavaCA::step, engine/src/ca/LavaCA.hpp:230-247) is three launches on the handle's
// stream:
//   ca_drop_kernel  -- brings the drop-depth plane (dropDepth of every AIR cell, LavaCA.hpp:404-414)
//                      up to date by rescanning the column segments above last step's type changes;
//   ca_rules_kernel -- a persistent streaming loop over 64 x TY x TZ tiles (TY * TZ = 16): every
//                      cell of the tile is read and written to the next buffer, LAVA cools
//                      (updateLava, LavaCA.hpp:1135-1151), AIR cells with LAVA within one cell are
//                      listed as candidates, the tiles of the next step are scheduled;
//   ca_cand_kernel  -- the candidates: gatherLavaCandidates, vote and solidus test (LavaCA.hpp:
//                      443-519, 1121-1134) with D(n) of each lava source evaluated from the
//                      drop-depth plane (descent / computeDescent, LavaCA.hpp:421-429, 551-566);
//                      in its last block, finishStep (LavaCA.hpp:1206-1229).
// State: double-buffered SoA planes (type u8, flowId i32, temp f32, solidStep u16, arrivalStep u16)
// in pitched rows; the current buffer is the parity of the device-side step counter, so a run of
// steps needs no host round trip until the stop test.
//
// ACTIVE schedule: only LAVA cells and AIR cells with LAVA within one cell can change in a step
// (the front set of LavaCA::frontCandidatesLayer, LavaCA.hpp:907-940).  A tile is processed in step
// t+1 when a tile within one tile of it holds LAVA after step t, or when it changed in step t (its
// two buffers then differ).  Every other tile keeps both buffers equal and is skipped; the result is
// bit-identical to the DENSE schedule, which processes every tile every step.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <utility>
#include <vector>

#include "vca.h"
#include "vca_device.cuh"
#include "vca_internal.h"

namespace vca {

constexpr int kThreads = 256;       // threads of a tile block: 16 per 64-cell row, 16 rows
constexpr int kTileX = 64;
constexpr int kMaxDrop = 16;        // LavaCA::kMaxDrop (LavaCA.hpp:1293)
constexpr int kSmemRowBytes = 96;   // 16 pad (left frame byte at 15) + 64 cells + right frame byte + pad
constexpr int kRowOff = 16;         // first cell of a staged row (16-byte aligned for cp.async)

// ------------------------------------------------------------------------------------------
// Addressing with the reference's frame semantics: a coordinate one step outside the interior is
// the opposite layer on a periodic axis, else the VOID frame (Boundary::applyWith,
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
// A halo coordinate of a tile: up to one cell outside [0, n) maps through the frame; further out
// (past a partial last tile) is outside the grid.
__device__ __forceinline__ bool halo_axis(int& v, int n, int periodic) {
    if (v > n) return false;
    return wrap_axis(v, n, periodic);
}
__device__ __forceinline__ bool solid_ground(int t) { return t == kRock || t == kBasalt; }
// resolve() for a neighbour one cell away, as selects instead of branches, so that the loads of
// all neighbours of a cell can be issued together.  v is only meaningful when the result is true.
__device__ __forceinline__ bool wrap1_sel(int& v, int n, int periodic) {
    const bool in = (unsigned)v < (unsigned)n;
    const int w = v < 0 ? v + n : v - n;
    v = in ? v : w;
    return in | ((periodic != 0) & (n > 1));
}
__device__ __forceinline__ bool resolve1_sel(const CaGeom& g, int& x, int& y, int& z) {
    const bool a = wrap1_sel(x, g.nx, g.per[0]), b = wrap1_sel(y, g.ny, g.per[1]), c = wrap1_sel(z, g.nz, g.per[2]);
    return a & b & c;
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
    __device__ bool overflow() const { return false; }
    __device__ void pick(uint64_t prefix, uint64_t gidx, int32_t* id, float* t) const {
        const int w = winner(prefix, gidx);
        *id = ids[w];
        *t = max_temp[w];
    }
};

// The same vote for up to 4 distinct flowIds, held in registers (every index is a compile-time
// constant after unrolling).  A fifth distinct id sets overflow; the caller then recounts with Vote.
struct SmallVote {
    int n;
    bool over;
    int32_t ids[4];
    int counts[4];
    float max_temp[4];
    __device__ void add(int32_t id, float t) {
        bool hit = false;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            if (s < n && ids[s] == id) {
                ++counts[s];
                max_temp[s] = fmaxf(max_temp[s], t);
                hit = true;
            }
        if (hit) return;
        if (n == 4) {
            over = true;
            return;
        }
#pragma unroll
        for (int s = 0; s < 4; ++s)
            if (s == n) {
                ids[s] = id;
                counts[s] = 1;
                max_temp[s] = t;
            }
        ++n;
    }
    __device__ bool overflow() const { return over; }
    // Most votes; ties: the (r % k)-th smallest tied id, r = hashRand(seed, t, idx, TieBreak).
    __device__ void pick(uint64_t prefix, uint64_t gidx, int32_t* id, float* t) const {
        int best = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s)
            if (s < n) best = max(best, counts[s]);
        int k = 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) k += (s < n && counts[s] == best) ? 1 : 0;
        int want = 0;
        if (k > 1) want = (int)(hash_salt(hash_index(prefix, gidx), kSaltTieBreak) % (uint64_t)k);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (!(s < n && counts[s] == best)) continue;
            int rank = 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) rank += (u < n && counts[u] == best && ids[u] < ids[s]) ? 1 : 0;
            if (rank == want) {
                *id = ids[s];
                *t = max_temp[s];
            }
        }
    }
};

__device__ __forceinline__ void tile_origin(const CaGeom& g, uint32_t tile, int& x0, int& y0, int& z0) {
    uint32_t tx, ty;
    const uint32_t r = fast_divmod(tile, g.div_tx, tx);
    const uint32_t tz = fast_divmod(r, g.div_ty, ty);
    x0 = (int)tx * kTileX;
    y0 = (int)ty * g.TY;
    z0 = (int)tz * g.TZ;
}

// ------------------------------------------------------------------------------------------
// Drop depth (LavaCA::dropDepth, LavaCA.hpp:404-414), kept current for every AIR cell.
//
// dropDepth of an AIR cell z only looks down its own column.  With k the number of AIR cells
// directly below z (the run of AIR from its bottom cell w = z - k up to z), the loop can only find
// support at w, so
//     dropDepth(z) = 16 if k > 16;  k if hasSupport(w);  16 if k == 16;  -1 otherwise
// (when w has no support the cell under w exists and is not AIR).  An upward scan of a column
// segment [lo, hi) from lo - 17 yields it for every cell of the segment: a run that reaches below
// the scan start is longer than 16 either way.  dropDepth(z) depends only on the types in
// [z - 17, z], so after a step only the 18 cells above each cell whose type changed need a
// rescan; the rules kernel lists those cells.  Non-AIR cells hold -1.
// ------------------------------------------------------------------------------------------
__device__ void drop_scan(const CaKernelArgs& k, const uint8_t* T, int x, int y, int lo, int hi) {
    const CaGeom& g = k.g;
    const bool has_spill = k.spill != nullptr;
    const int sp = has_spill ? __ldg(k.spill + x + (int64_t)g.nx * y) : 0;
    const int zb = max(0, lo - (kMaxDrop + 1));
    int prev = zb > 0 ? T[pidx(g, x, y, zb - 1)] : kVoid;
    int run_start = 0;
    bool in_run = false, run_sup = false;
#pragma unroll 4
    for (int z = zb; z < hi; ++z) {
        const int tz = T[pidx(g, x, y, z)];
        // hasSupport(z) (LavaCA.hpp:390-399)
        const bool hs = z == 0 || solid_ground(prev) || (prev == kLava && has_spill && z - 1 < sp);
        int dd = -1;
        if (tz == kAir) {
            if (!in_run) {
                in_run = true;
                if (z == zb && prev == kAir) {
                    run_start = z - 4 * kMaxDrop;  // the run goes on below the scan: longer than 16
                    run_sup = false;
                } else {
                    run_start = z;
                    run_sup = hs;
                }
            }
            const int kk = z - run_start;
            dd = kk > kMaxDrop ? kMaxDrop : (run_sup ? kk : (kk == kMaxDrop ? kMaxDrop : -1));
        } else {
            in_run = false;
        }
        if (z >= lo) k.drop[pidx(g, x, y, z)] = (int8_t)dd;
        prev = tz;
    }
}

// The same closed form for the 18 cells [zc, zc + 18) above one changed cell, from one batch of
// independent loads: the types of the window [zc - 17, zc + 18) become bit masks (bit i = cell
// zc - 17 + i; cells below the grid floor count as solid), the run bottom w of an AIR cell is one
// above the highest non-AIR bit below it.  A run that reaches below the window is longer than 16.
__device__ void drop_rescan18(const CaKernelArgs& k, const uint8_t* T, int x, int y, int zc) {
    const CaGeom& g = k.g;
    constexpr int kWin = 2 * (kMaxDrop + 1) + 1;  // 35 cells
    const int b = zc - (kMaxDrop + 1);
    const int64_t col = pidx(g, x, y, 0), zs = (int64_t)g.P * g.ny;
    const int sp = k.spill != nullptr ? __ldg(k.spill + x + (int64_t)g.nx * y) : 0;
    uint64_t air = 0, solid = 0, lava = 0;
#pragma unroll
    for (int i = 0; i < kWin; ++i) {
        // clamped loads without branches, so that all 35 are in flight together
        const int z = b + i;
        const bool in = z >= 0 && z < g.nz;
        const int t = __ldg(T + col + zs * min(max(z, 0), g.nz - 1));
        air |= (uint64_t)(in && t == kAir) << i;
        solid |= (uint64_t)(z < 0 || (in && (t == kRock || t == kBasalt))) << i;
        lava |= (uint64_t)(in && t == kLava) << i;
    }
    const int hi = min(g.nz, zc + kMaxDrop + 2);
    for (int z = zc; z < hi; ++z) {
        const int i = z - b;
        int dd = -1;
        if ((air >> i) & 1ull) {
            const uint64_t below = ~air & ((1ull << i) - 1ull);
            if (below == 0) {
                dd = kMaxDrop;  // i >= 17 AIR cells below z
            } else {
                const int j = 63 - __clzll((long long)below);  // the cell under the run bottom
                const int kk = i - j - 1;
                const int under = b + j;  // its z (-1: the grid floor)
                const bool sup = ((solid >> j) & 1ull) || (((lava >> j) & 1ull) && k.spill != nullptr && under < sp);
                dd = kk > kMaxDrop ? kMaxDrop : (sup ? kk : (kk == kMaxDrop ? kMaxDrop : -1));
            }
        }
        k.drop[col + zs * z] = (int8_t)dd;
    }
}

// Rescans the columns above last step's type changes (or every column when forced or when the
// change list overflowed), and clears the change list this step's rules will fill.  Block `bid` of
// `nblk` blocks working on this grid.
__device__ __forceinline__ void drop_body(const CaKernelArgs& k, int force_full, uint32_t bid, uint32_t nblk) {
    CaCtrl* ctrl = k.ctrl;
    if (!force_full && (ctrl->stop || ctrl->error)) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1, nxt = cur ^ 1;
    if (!force_full && bid == 0 && threadIdx.x == 0) {
        ctrl->chg_count[nxt] = 0;   // filled by this step's rules
        ctrl->list_count[nxt] = 0;  // tiles of the next step, scheduled by this step's rules
        ctrl->tile_next = 0;        // tiles handed out at run time by this step's rules (DENSE)
    }
    if (k.classic) return;
    const CaGeom& g = k.g;
    const uint8_t* T = k.type[cur];
    const unsigned n = force_full ? 0u : ctrl->chg_count[cur];
    const uint64_t stride = (uint64_t)nblk * blockDim.x;
    const uint64_t gtid = bid * (uint64_t)blockDim.x + threadIdx.x;
    // a slab's halo layers change by copies from its neighbours, outside the change list: rescan all
    if (force_full || n > k.chg_cap || k.slab) {
        const uint64_t cols = (uint64_t)g.nx * g.ny;
        for (uint64_t c = gtid; c < cols; c += stride) drop_scan(k, T, (int)(c % g.nx), (int)(c / g.nx), 0, g.nz);
        return;
    }
    for (uint64_t j = gtid; j < n; j += stride) {
        const uint32_t gi = k.chg_list[cur][j];
        const uint32_t r = gi / (uint32_t)g.nx;
        const int x = (int)(gi - r * (uint32_t)g.nx);
        const int y = (int)(r % (uint32_t)g.ny);
        const int z = (int)(r / (uint32_t)g.ny);
        drop_rescan18(k, T, x, y, z);
    }
}
__global__ void ca_drop_kernel(const __grid_constant__ CaKernelArgs k, int force_full) {
    drop_body(k, force_full, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------------------------------
// Rules, candidate pass: an AIR cell with LAVA within one cell (listed by the streaming pass).
// ------------------------------------------------------------------------------------------

// gatherLavaCandidates + tryPonding (LavaCA.hpp:443-519) or updateClassic's vote (1176-1182), the
// winner (CaRules.hpp:152-173) and the solidus test.  Returns true when the cell becomes LAVA.
// Memory rounds: the cell's own drop depth and the neighbour types of its variant are fetched
// together (independent loads); then, for up to 8 LAVA neighbours at a time, their D(n), flowId and
// temperature together.  The vote does not depend on the order in which sources are added.
template <class V>
__device__ __forceinline__ bool gather_vote(const CaKernelArgs& k, const uint8_t* T, const int32_t* F, const float* Te,
                                            int x, int y, int z, uint64_t prefix, uint64_t gidx, V& v, int32_t* out_flow,
                                            float* out_temp) {
    const CaGeom& g = k.g;
    const NbTable& nb = k.tables.nb;
    const int var = nb.variants == 1 ? 0 : (int)fast_mod(hash_salt(hash_index(prefix, gidx), kSaltNeighborhood), k.var_mod);
    const int cnt = nb.count[var];
    const int64_t self = pidx(g, x, y, z);
    const int c_drop = k.classic ? 0 : (int)k.drop[self];
    // one round of independent loads: a neighbour outside the grid (or past the variant's count)
    // reads the cell itself, which is AIR
    uint32_t lava_mask = 0;
#pragma unroll
    for (int i = 0; i < 26; ++i) {
        int sx = x + nb.off[var][i][0], sy = y + nb.off[var][i][1], sz = z + nb.off[var][i][2];
        const bool ok = (i < cnt) & resolve1_sel(g, sx, sy, sz);
        const int tv = __ldg(T + (ok ? pidx(g, sx, sy, sz) : self));
        lava_mask |= (uint32_t)(tv == kLava) << i;
    }
    // tryPonding's cells (LavaCA.hpp:443-461), fetched in the same round: the spill level, the cell
    // under the one below (its support), the cells beside the one below (4 in 3D, 2 in 2D; outside
    // the grid they are VOID, i.e. open) and the flowId and temperature of the one below
    const bool pond = !k.classic && k.ponding && k.spill != nullptr && z >= 1;
    int p_spill = 0, p_under = kRock;
    bool p_closed = true;
    int32_t p_flow = 0;
    float p_temp = 0.0f;
    if (pond) {
        const int bz = z - 1;
        p_spill = __ldg(k.spill + x + (int64_t)g.nx * y);
        if (bz > 0) p_under = __ldg(T + pidx(g, x, y, bz - 1));  // bz == 0 stands on the grid floor
        const int nh = g.ny > 1 ? 4 : 2;
        const int hx[4] = {-1, 1, 0, 0}, hy[4] = {0, 0, -1, 1};
#pragma unroll
        for (int h = 0; h < 4; ++h) {
            int sx = x + hx[h], sy = y + hy[h], sz = bz;
            const bool ok = (h < nh) & resolve1_sel(g, sx, sy, sz);
            const int n = __ldg(T + (ok ? pidx(g, sx, sy, sz) : self));
            const bool open = h < nh && (!ok || n == kAir || n == kVoid);
            p_closed = p_closed && !open;
        }
        const int64_t b = pidx(g, x, y, bz);
        p_flow = __ldg(F + b);
        p_temp = __ldg(Te + b);
    }
    if (!lava_mask) return false;
    v.n = 0;
    while (lava_mask) {
        int src[8];
        int8_t dsc[8];
        int32_t fl[8];
        float te[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            src[q] = -1;
            if (lava_mask) {
                const int i = __ffs(lava_mask) - 1;
                lava_mask &= lava_mask - 1;
                const int dx = nb.off[var][i][0], dy = nb.off[var][i][1], dz = nb.off[var][i][2];
                if (dz < 0 && !k.classic) {
                    // a LAVA cell below feeds only by ponding (straight below), resolved on its own
                    if (k.ponding && dx == 0 && dy == 0) src[q] = 26;
                    continue;
                }
                src[q] = i;
            }
        }
        // the sources' flowId, temperature and D(n), again in one round (unused slots read the cell)
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const bool use = src[q] >= 0 && src[q] != 26;
            const int i = use ? src[q] : 0;
            int sx = x + nb.off[var][i][0], sy = y + nb.off[var][i][1], sz = z + nb.off[var][i][2];
            resolve1_sel(g, sx, sy, sz);
            const int64_t sp = use ? pidx(g, sx, sy, sz) : self;
            fl[q] = __ldg(F + sp);
            te[q] = __ldg(Te + sp);
            dsc[q] = __ldg(k.desc + sp);
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            if (src[q] < 0) continue;
            if (k.classic) {
                v.add(fl[q], 0.0f);
                continue;
            }
            if (src[q] == 26) {
                // tryPonding (LavaCA.hpp:443-461): at or below the spill level, the cell below
                // supported (hasSupport of z - 1: the grid floor, solid ground, or LAVA below the
                // spill level) and closed on every side
                if (!pond || z > p_spill) continue;
                const bool sup = solid_ground(p_under) || (p_under == kLava && z - 2 < p_spill);
                if (!sup || !p_closed) continue;
                v.add(p_flow, __fsub_rn(p_temp, k.cool_lateral));
                continue;
            }
            const int i = src[q];
            const int dx = nb.off[var][i][0], dy = nb.off[var][i][1], dz = nb.off[var][i][2];
            float cooling;
            if (dz > 0 && dx == 0 && dy == 0) {
                cooling = k.cool_fall;
            } else {
                const int d = dsc[q];
                if (d < 0) continue;
                if (dz > 0) {
                    if (c_drop != 0 || d != 1) continue;
                    cooling = k.cool_fall;
                } else {
                    if (c_drop != d || (d == 1 && k.diag_falls)) continue;
                    cooling = k.cool_lateral;
                }
            }
            v.add(fl[q], __fsub_rn(te[q], cooling));
        }
    }
    if (v.n == 0 || v.overflow()) return false;
    int32_t wid = 0;
    float wt = 0.0f;
    v.pick(prefix, gidx, &wid, &wt);
    if (k.classic) {
        *out_flow = wid;
        *out_temp = 0.0f;
        return true;
    }
    if (!(wt >= k.solidus)) return false;
    *out_flow = wid;
    *out_temp = wt;
    return true;
}

// A cell with five or more distinct flowIds among its sources: the vote with room for 26.
__device__ __noinline__ bool air_gains_lava_wide(const CaKernelArgs& k, const uint8_t* T, const int32_t* F,
                                                 const float* Te, int x, int y, int z, uint64_t prefix, uint64_t gidx,
                                                 int32_t* out_flow, float* out_temp) {
    Vote v;
    return gather_vote(k, T, F, Te, x, y, z, prefix, gidx, v, out_flow, out_temp);
}

__device__ __forceinline__ bool air_gains_lava(const CaKernelArgs& k, const uint8_t* T, const int32_t* F,
                                               const float* Te, int x, int y, int z, uint64_t prefix, uint64_t gidx,
                                               int32_t* out_flow, float* out_temp) {
    SmallVote v;
    v.over = false;
    const bool gained = gather_vote(k, T, F, Te, x, y, z, prefix, gidx, v, out_flow, out_temp);
    if (v.over) return air_gains_lava_wide(k, T, F, Te, x, y, z, prefix, gidx, out_flow, out_temp);
    return gained;
}

// Whether a tile whose LAVA touches the faces `f` (bits 2-7: -x, +x, -y, +y, -z, +z) can reach its
// neighbour (dx, dy, dz) = lane's offset in the next step: LAVA lies within one cell of it only when it
// touches the faces towards it.  In lava mode an AIR cell takes LAVA only from its own level, from
// the level above, or by ponding from the cell straight below (gatherLavaCandidates,
// LavaCA.hpp:462-519), so a tile above is reached only straight up and only by ponding (bit 7 is
// then set only for LAVA that can pond upwards).
__device__ __forceinline__ bool faces_reach(unsigned f, int lane, bool lava_mode) {
    const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
    if (lava_mode && dz > 0 && (dx != 0 || dy != 0)) return false;
    return (dx == 0 || ((f >> (dx < 0 ? 2 : 3)) & 1u)) && (dy == 0 || ((f >> (dy < 0 ? 4 : 5)) & 1u)) &&
           (dz == 0 || ((f >> (dz < 0 ? 6 : 7)) & 1u));
}

// The face bits of a LAVA cell (x, y, z) of the tile with origin (x0, y0, z0): the faces it lies on;
// the top face only when `up` (the cell can feed the one above it).
__device__ __forceinline__ unsigned cell_faces(const CaGeom& g, int x, int y, int z, int x0, int y0, int z0, bool up) {
    unsigned f = 0;
    if (x == x0) f |= 1u << 2;
    if (x == min(x0 + kTileX, g.nx) - 1) f |= 1u << 3;
    if (y == y0) f |= 1u << 4;
    if (y == min(y0 + g.TY, g.ny) - 1) f |= 1u << 5;
    if (z == z0) f |= 1u << 6;
    if (up && z == min(z0 + g.TZ, g.nz) - 1) f |= 1u << 7;
    return f;
}
// A LAVA cell at (x, y, z) can feed the AIR cell above it: in classic mode always, in lava mode by
// ponding when that cell lies at or below its column's spill level (LavaCA.hpp:443-461).
__device__ __forceinline__ bool feeds_up(const CaKernelArgs& k, int spill_level, int z) {
    return k.classic || (k.ponding && k.spill != nullptr && z + 1 <= spill_level);
}

// Schedule the tiles within one tile of `tile` for step t + 1; lanes 0..26 of a warp each try one
// target, `want` says which lanes take part.  The mark of a tile scheduled for step s is
// 2 (s + 1) plus a lava bit: the bit says that LAVA lies within one tile, so the tile's cells may
// change; without it the tile is only refreshed (its two buffers differ) by a plain copy.  Marks
// are kept per step parity, so a mark read during step s is never raised during step s.
__device__ __forceinline__ void schedule_around(const CaKernelArgs& k, uint32_t tile, uint32_t t, int nxt, int lane,
                                                bool want, bool lava) {
    const CaGeom& g = k.g;
    bool first = false;
    uint32_t target = 0;
    if (want && lane < 27) {
        const int dx = lane % 3 - 1, dy = (lane / 3) % 3 - 1, dz = lane / 9 - 1;
        uint32_t ux, uy;
        const uint32_t r = fast_divmod(tile, g.div_tx, ux);
        const uint32_t uz = fast_divmod(r, g.div_ty, uy);
        int tx = (int)ux + dx, ty = (int)uy + dy, tz = (int)uz + dz;
        if (wrap_axis(tx, g.tiles_x, g.per[0]) && wrap_axis(ty, g.tiles_y, g.per[1]) && wrap_axis(tz, g.tiles_z, g.per[2])) {
            target = (uint32_t)tx + (uint32_t)g.tiles_x * ((uint32_t)ty + (uint32_t)g.tiles_y * tz);
            const uint32_t m = 2u * (t + 2u);
            first = atomicMax(&k.tile_mark[nxt][target], m + (lava ? 1u : 0u)) < m;
        }
    }
    if (k.dense) return;  // every tile runs anyway; the marks only choose its path
    const unsigned ballot = __ballot_sync(0xFFFFFFFFu, first);
    unsigned slot = 0;
    if (lane == 0 && ballot) slot = atomicAdd(&k.ctrl->list_count[nxt], (unsigned)__popc(ballot));
    slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
    const unsigned pos = slot + __popc(ballot & ((1u << lane) - 1u));
    if (first && pos < k.ntiles) k.tile_list[nxt][pos] = target;  // a tile is listed once per step
}

// Asynchronous global -> shared copies (cp.async): the data lands without passing through registers;
// cp_async_wait_all waits for all of this thread's copies.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(smem)), "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// all committed groups but the most recent one are complete
__device__ __forceinline__ void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Shared-memory row of the tile cell (ly, lz) in the staged halo layout.
__device__ __forceinline__ int hr_of(int ly, int lz, int hy_on, int hz_on, int HY) { return (ly + hy_on) + HY * (lz + hz_on); }

// Warp-aggregated append of n entries (values v[0..n-1], n <= 4) per lane to list/count.
__device__ __forceinline__ void warp_append(uint32_t* list, unsigned int* count, uint32_t cap, int lane, unsigned n,
                                            const uint32_t* v) {
    unsigned incl = n;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const unsigned u = __shfl_up_sync(0xFFFFFFFFu, incl, off);
        if (lane >= off) incl += u;
    }
    unsigned base = 0;
    if (lane == 31 && incl) base = atomicAdd(count, incl);
    base = __shfl_sync(0xFFFFFFFFu, base, 31) + incl - n;
    for (unsigned j = 0; j < n; ++j)
        if (base + j < cap) list[base + j] = v[j];
}

constexpr int kMaxDeferred = 64;   // tiles a rules block schedules in one batch
constexpr int kTileCells = 1024;   // 64 x TY x TZ, TY * TZ = 16
constexpr int kCandBuf = 2 * kTileCells;  // candidates a rules block gathers before one flush

// ------------------------------------------------------------------------------------------
// TMA and mbarrier primitives (PTX ISA: cp.async.bulk.tensor, mbarrier).  Tiled loads land in shared
// memory and complete transaction bytes on an mbarrier; tiled stores read shared memory as bulk
// groups.  Every wait is bounded: a wait that runs out reports failure to the caller.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Waits for the completion of the phase with the given parity; false after ~2^20 suspended tries.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity), "r"(1000u)
            : "memory");
        if (done) return true;
    }
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, int x, int y, int z, const void* src) {
    asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3}], [%4];\n" ::"l"(map), "r"(x),
                 "r"(y), "r"(z), "r"(smem_u32(src))
                 : "memory");
}
// 4D boxes {x, y, z, plane}: two planes of one allocation (flowId + temperature, solidStep +
// arrivalStep) move in one copy
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];\n" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_store_4d(const CUtensorMap* map, int x, int y, int z, const void* src) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%1, %2, %3, %4}], [%5];\n" ::"l"(map),
                 "r"(x), "r"(y), "r"(z), "r"(0), "r"(smem_u32(src))
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;\n" ::: "memory"); }
// the shared-memory sources of all committed bulk stores have been read
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory"); }
// orders this thread's generic-proxy shared-memory accesses before later async-proxy (TMA) ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

// ------------------------------------------------------------------------------------------
// Rules, streaming pass.  A persistent block walks its tiles through a two-slot pipeline in
// shared memory.  Thread 0 issues the TMA box copies of tile i + 1 into one slot while tile i is
// computed from the other: the tile's state boxes (flowId, temp, solidStep, arrivalStep), its types
// with a one-cell halo (one box, x from x0 - 16 so that both frame bytes come along), and in lava
// mode the drop depths of its levels; the threads add the spill levels of its columns (cp.async).
// The control loads run two tiles ahead (tile id of i + 2, mark of i + 1).  Results are written back
// into the slot and leave by TMA stores, which clip at the grid edges.
// Per tile:
//   1. LAVA cells cool (updateLava's LAVA branch, LavaCA.hpp:1135-1151) and get their D(n)
//      (descent / computeDescent, LavaCA.hpp:421-429, 551-566) from byte windows of the staged
//      types and drop depths; AIR cells that a source could reach are gathered in shared memory and
//      appended to the candidate list in batches, resolved by the candidate pass;
//   2. LAVA -> BASALT cells are listed for the drop-depth rescan;
//   3. the block batches its tiles' flags and, after the loop, schedules the next step's tiles:
//      with LAVA a tile and its neighbours, changed only the tile itself.
// A tile without LAVA within one tile (mark without lava bit, or not scheduled at all in the DENSE
// schedule) cannot change: thread 0 alone moves its state boxes from the current to the next buffer.
// Tiles at the grid edge get their frame cells (VOID, or the periodic copy) patched after the load.
// ------------------------------------------------------------------------------------------
// Shared-memory room of the rules pass for a family of tile shapes 64 x TY x TZ (TY * TZ = 16):
// staged halo rows (HY * HZ, HY = TY + 2 and HZ = TZ + 2 on axes of size > 1), drop-depth rows
// (HY * TZ) and spill columns (64 * TY).  Halo rows are a multiple of 4, so that the drop rows after
// them start 128-byte aligned.
template <int HALO, int DROP, int TYMAX>
struct RulesShape {
    static constexpr int halo = HALO, drop = DROP, ty = TYMAX;
    static_assert(HALO % 4 == 0 && HALO * 4 <= kThreads && DROP * 4 <= kThreads, "frame patch threads");
};
using ShapeA = RulesShape<36, 24, 4>;   // 4 x 4 in 3D; 1 x 16 (x-z) and 16 x 1 (x-y) in 2D
using ShapeB = RulesShape<40, 32, 8>;   // 2 x 8 and 8 x 2 in 3D
using ShapeC = RulesShape<56, 48, 16>;  // 1 x 16 and 16 x 1 in 3D
// a wrapped-x column buffer: 16 bytes per halo row (or drop row), each buffer 128-byte aligned
constexpr int xside_bytes(int rows) { return (rows * 16 + 127) / 128 * 128; }

template <class S>
struct __align__(128) RulesSlot {
    int32_t flow[kTileCells];
    float temp[kTileCells];
    uint16_t solid[kTileCells];
    uint16_t arrival[kTileCells];
    uint8_t own_type[kTileCells];
    uint8_t type[S::halo * kSmemRowBytes];
    int8_t drop[S::drop * kSmemRowBytes];
    int32_t spill[kTileX * S::ty];
    // wrapped x columns (periodic x): [0] the 16 cells ending at x = nx - 1 (left frame, byte 15 of
    // each row), [1] the 16 cells from x = 0 (right frame or padded-row copy, byte 0)
    __align__(128) uint8_t xside[2][xside_bytes(S::halo)];
    __align__(128) int8_t xside_drop[2][xside_bytes(S::drop)];
};
template <class S>
constexpr bool slot_layout_ok() {
    using T = RulesSlot<S>;
    return offsetof(T, temp) == offsetof(T, flow) + 4 * kTileCells && offsetof(T, arrival) == offsetof(T, solid) + 2 * kTileCells &&
           offsetof(T, type) % 128 == 0 && offsetof(T, drop) % 128 == 0 && offsetof(T, own_type) % 128 == 0 &&
           offsetof(T, solid) % 128 == 0 && offsetof(T, xside) % 128 == 0 && offsetof(T, xside_drop) % 128 == 0;
}
static_assert(slot_layout_ok<ShapeA>() && slot_layout_ok<ShapeB>() && slot_layout_ok<ShapeC>(),
              "the planes of a pair follow each other in a slot, as a 4D box lands them; TMA destinations are "
              "128-byte aligned");
template <class S>
constexpr size_t rules_dyn_smem() { return 2 * sizeof(RulesSlot<S>) + 128; }
constexpr size_t kRulesDynSmem = rules_dyn_smem<ShapeA>();

// Bytes x-1 .. x+2 / x .. x+3 / x+1 .. x+4 of a staged row around the 4 cells at p (p = row start +
// kRowOff + 4 * xq; the frame bytes sit at kRowOff - 1 and kRowOff + 64).
__device__ __forceinline__ uint32_t win_left(const uint8_t* p) {
    return __funnelshift_r(*reinterpret_cast<const uint32_t*>(p - 4), *reinterpret_cast<const uint32_t*>(p), 24);
}
__device__ __forceinline__ uint32_t win_mid(const uint8_t* p) { return *reinterpret_cast<const uint32_t*>(p); }
__device__ __forceinline__ uint32_t win_right(const uint8_t* p) {
    return __funnelshift_r(*reinterpret_cast<const uint32_t*>(p), *reinterpret_cast<const uint32_t*>(p + 4), 8);
}

template <class S, bool kDyn>
__device__ __forceinline__ void rules_body(const CaTensorMaps& tm, const CaKernelArgs& k, uint32_t bid, uint32_t nblk) {
    using RulesSlot = vca::RulesSlot<S>;
    // Declared with the 16-byte alignment that dynamic shared memory is guaranteed to have, so that
    // the rounding below is computed at run time: the dynamic part starts after the kernel's static
    // shared variables, whose total need not be a multiple of 128 bytes (the batched kernel adds its
    // member's arguments).
    extern __shared__ __align__(16) uint8_t s_dyn[];
    // the slots start on a 128-byte boundary (TMA destinations); the launch adds 128 bytes of slack
    RulesSlot* slots = reinterpret_cast<RulesSlot*>(s_dyn + ((128u - (smem_u32(s_dyn) & 127u)) & 127u));
    __shared__ __align__(8) uint64_t s_bar[2];
    __shared__ unsigned s_flags[2];
    __shared__ unsigned s_wtot[kThreads / 32];
    __shared__ uint32_t s_sched_tile[kMaxDeferred];
    __shared__ uint32_t s_cand[kCandBuf];
    __shared__ unsigned s_cand_base;
    __shared__ uint8_t s_sched_flag[kMaxDeferred];
    __shared__ unsigned long long s_red[2][kThreads / 32];

    CaCtrl* ctrl = k.ctrl;
    if (ctrl->stop || ctrl->error) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1, nxt = cur ^ 1;
    const CaGeom& g = k.g;
    const uint8_t* T = k.type[cur];
    const uint64_t count = k.dense ? k.ntiles : ctrl->list_count[cur];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int xq = tid & 15, row = tid >> 4;
    const int ly = row % g.TY, lz = row / g.TY;
    const int hy_on = g.ny > 1 ? 1 : 0, hz_on = g.nz > 1 ? 1 : 0;
    const int HY = hy_on ? g.TY + 2 : 1, HZ = hz_on ? g.TZ + 2 : 1;
    const int halo_rows = HY * HZ;
    const int drop_rows = HY * g.TZ;
    const bool lava_mode = !k.classic;
    const bool stage_spill = lava_mode && hz_on && k.spill != nullptr;
    const bool erupting = (int64_t)t < (int64_t)k.eruption_steps;
    const uint32_t stamp = min(t, 65535u);
    const uint32_t live_mark = 2u * (t + 1u) + 1u;
    // transaction bytes of one slot fill
    const uint32_t tx_copy = kTileCells * (1 + 4 + 4 + 2 + 2);
    const uint32_t tx_rules = kTileCells * (4 + 4 + 2 + 2) + kSmemRowBytes * halo_rows + (lava_mode ? kSmemRowBytes * drop_rows : 0);
    const bool xwrap = g.per[0] && (g.nx & 15) == 0;  // the wrapped x columns come by TMA (16-cell aligned)
    const uint32_t tx_xside = 16u * halo_rows + (lava_mode ? 16u * drop_rows : 0u);
    if (tid == 0) {
        s_flags[0] = s_flags[1] = 0;
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        fence_proxy_async();
    }
    __syncthreads();

    unsigned int my_active = 0, my_changed = 0, tiles_done = 0;
    int nsched = 0, rit = 0;  // rit: rules tiles so far (parity of s_flags)
    unsigned nbuf = 0;        // candidates in s_cand (block-uniform)
    bool failed = false;      // a bounded wait ran out (block-uniform once set)

    auto flush_schedule = [&]() {
        __syncthreads();
        // lane (dx, dy, dz) of a tile with LAVA schedules that neighbour when the LAVA touches the
        // faces towards it; a tile that changed schedules itself
        for (int e = warp; e < nsched; e += kThreads / 32) {
            const unsigned f = s_sched_flag[e];
            schedule_around(k, s_sched_tile[e], t, nxt, lane,
                            ((f & 1u) && faces_reach(f, lane, !k.classic)) || ((f & 2u) && lane == 13), (f & 1u) != 0);
        }
        __syncthreads();
        nsched = 0;
    };
    auto flush_cands = [&]() {
        __syncthreads();
        if (tid == 0) s_cand_base = atomicAdd(&ctrl->cand_count, nbuf);
        __syncthreads();
        const unsigned base = s_cand_base;
        for (unsigned j = tid; j < nbuf; j += kThreads) k.cand_list[base + j] = s_cand[j];
        __syncthreads();
        nbuf = 0;
    };
    auto tile_at = [&](uint64_t i) -> uint32_t { return k.dense ? (uint32_t)i : k.tile_list[cur][i]; };
    // Rules (not the plain copy) for a tile: its mark says LAVA lies within one tile.  A z slab's
    // halo layers are rewritten by copies from the neighbouring slabs, which the marks never see, so
    // there the tiles within one tile of a halo layer take the rules every step.
    auto takes_rules = [&](uint32_t tile, uint32_t mark) -> bool {
        if (mark == live_mark) return true;
        if (!k.slab) return false;
        int tx0, ty0, tz0;
        tile_origin(g, tile, tx0, ty0, tz0);
        return tz0 < k.own_z0 + g.TZ || tz0 + 2 * g.TZ > k.own_z1;
    };

    // Fill a slot: TMA boxes by thread 0 (the slot's earlier stores must have been read first),
    // spill levels by the threads.
    auto stage = [&](int s, uint32_t tile, bool rules) {
        RulesSlot& sl = slots[s];
        int x0, y0, z0;
        tile_origin(g, tile, x0, y0, z0);
        if (tid == 0) {
            bulk_wait_read_all();
            fence_proxy_async();
            // periodic x: an x-edge tile also loads the column that holds its wrapped frame cells
            const bool wl = rules && xwrap && x0 == 0, wr = rules && xwrap && x0 + kTileX >= g.nx;
            mbar_arrive_expect_tx(&s_bar[s], (rules ? tx_rules : tx_copy) + (wl ? tx_xside : 0u) + (wr ? tx_xside : 0u));
            tma_load_4d(sl.flow, &tm.ft[cur], x0, y0, z0, &s_bar[s]);   // flowId and temperature
            tma_load_4d(sl.solid, &tm.sa[cur], x0, y0, z0, &s_bar[s]);  // solidStep and arrivalStep
            if (rules) {
                tma_load_3d(sl.type, &tm.halo_type[cur], x0 - 16, y0 - hy_on, z0 - hz_on, &s_bar[s]);
                if (lava_mode) tma_load_3d(sl.drop, &tm.drop, x0 - 16, y0 - hy_on, z0, &s_bar[s]);
                if (wl) {
                    tma_load_3d(sl.xside[0], &tm.xside_type[cur], g.nx - 16, y0 - hy_on, z0 - hz_on, &s_bar[s]);
                    if (lava_mode) tma_load_3d(sl.xside_drop[0], &tm.xside_drop, g.nx - 16, y0 - hy_on, z0, &s_bar[s]);
                }
                if (wr) {
                    tma_load_3d(sl.xside[1], &tm.xside_type[cur], 0, y0 - hy_on, z0 - hz_on, &s_bar[s]);
                    if (lava_mode) tma_load_3d(sl.xside_drop[1], &tm.xside_drop, 0, y0 - hy_on, z0, &s_bar[s]);
                }
            } else {
                tma_load_3d(sl.own_type, &tm.own_type[cur], x0, y0, z0, &s_bar[s]);
            }
        }
        if (rules && stage_spill) {
            for (int c = tid; c < kTileX * g.TY; c += kThreads) {
                const int xx = x0 + (c & (kTileX - 1)), yy = y0 + c / kTileX;
                if (xx < g.nx && yy < g.ny)
                    cp_async4(&sl.spill[c], k.spill + xx + (int64_t)g.nx * yy);
                else
                    sl.spill[c] = 0;
            }
        }
    };
    auto store_tile = [&](int s, int x0, int y0, int z0) {  // thread 0
        RulesSlot& sl = slots[s];
        tma_store_3d(&tm.own_type[nxt], x0, y0, z0, sl.own_type);
        tma_store_4d(&tm.ft[nxt], x0, y0, z0, sl.flow);
        tma_store_4d(&tm.sa[nxt], x0, y0, z0, sl.solid);
        bulk_commit();
    };

    // control pipeline: the indices of this iteration and the next three, the tile ids of the next
    // two, the mark of the next.  Iteration m of a block takes index bid + m nblk.  With kDyn (DENSE
    // over many tiles per block, where a tile costs a plain copy or the whole rules pass) the indices
    // from the fifth on are handed out at run time from a per-step counter instead, so that blocks
    // that drew cheap tiles take more of them; each block's indices still increase, so it stops at
    // the first one past the end, and every index below that is taken by exactly one block.
    const uint64_t G = nblk;
    uint64_t i0 = bid, r1 = 0, r2 = 0, r3 = 0;  // kDyn: the indices of iterations it + 1 .. it + 3
    __shared__ uint64_t s_next[2];               // kDyn: the index of iteration m, at [m & 1]
    auto hand_out = [&]() -> uint64_t {
        return 4 * G < count ? 4 * G + atomicAdd(&ctrl->tile_next, 1u) : count;
    };
    if constexpr (kDyn) {
        r1 = bid + G;
        r2 = bid + 2 * G;
        r3 = bid + 3 * G;
        if (tid == 0) s_next[0] = hand_out();  // iteration 4
    }
    auto at1 = [&]() -> uint64_t { if constexpr (kDyn) return r1; else return i0 + G; };
    auto at2 = [&]() -> uint64_t { if constexpr (kDyn) return r2; else return i0 + 2 * G; };
    auto at3 = [&]() -> uint64_t { if constexpr (kDyn) return r3; else return i0 + 3 * G; };
    uint32_t tile_a = 0, mark_a = 0, vent_a = 0;  // iteration it
    uint32_t tile_b = 0, mark_b = 0, vent_b = 0;  // it + 1
    uint32_t tile_c = 0;                          // it + 2
    if (i0 < count) {
        tile_a = tile_at(i0);
        mark_a = k.tile_mark[cur][tile_a];
        vent_a = k.tile_flags[tile_a];
        if (at1() < count) tile_b = tile_at(at1());
        if (at2() < count) tile_c = tile_at(at2());
        stage(0, tile_a, takes_rules(tile_a, mark_a));
    }
    cp_async_commit();
    if (at1() < count) {
        mark_b = k.tile_mark[cur][tile_b];
        vent_b = k.tile_flags[tile_b];
    }

    for (int it = 0; i0 < count; ++it) {
        const int si = it & 1;
        RulesSlot& sl = slots[si];
        const uint32_t tile = tile_a;
        const bool rules = takes_rules(tile_a, mark_a);
        const bool tile_vent = (vent_a & 2u) != 0;
        // next tile into the other slot, then the control loads of the tiles after it
        if (at1() < count) stage(si ^ 1, tile_b, takes_rules(tile_b, mark_b));
        cp_async_commit();
        uint32_t mark_c = 0, vent_c = 0, tile_d = 0;
        if (at2() < count) {
            mark_c = k.tile_mark[cur][tile_c];
            vent_c = k.tile_flags[tile_c];
        }
        if (at3() < count) tile_d = tile_at(at3());

        int x0, y0, z0;
        tile_origin(g, tile, x0, y0, z0);
        ++tiles_done;
        const uint32_t parity = (uint32_t)(it >> 1) & 1u;
        const bool ok = mbar_wait(&s_bar[si], parity);
        if (rules) cp_async_wait_prior();  // this thread's spill copies
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicOr(&ctrl->error, 1);
                // the copies of the next slot, if any were issued, before the block gives up
                if (at1() < count) mbar_wait(&s_bar[si ^ 1], (uint32_t)((it + 1) >> 1) & 1u);
            }
            failed = true;
            break;
        }
        // kDyn: the index of iteration it + 4 (handed out during iteration it - 1, or before the
        // loop), and the hand-out of iteration it + 5 into the other word, read after the next barrier
        uint64_t i4 = 0;
        if constexpr (kDyn) {
            i4 = s_next[it & 1];
            if (tid == 0) s_next[(it + 1) & 1] = hand_out();
        }
        if (!rules) {
            // No LAVA within one tile: nothing can change, the boxes go to the next buffer as they are.
            if (tid == 0) {
                fence_proxy_async();
                store_tile(si, x0, y0, z0);
            }
        } else {
            const bool edge_tile = x0 == 0 || x0 + kTileX >= g.nx || (hy_on && (y0 == 0 || y0 + g.TY >= g.ny)) ||
                                   (hz_on && (z0 == 0 || z0 + g.TZ >= g.nz));
            if (edge_tile) {
                // Frame cells of the staged rows.  Outside the tensor the TMA filled zeros; the
                // reference's frame is VOID (absorbing) or the opposite layer (periodic,
                // Boundary.hpp:75-131).  Rows outside in y or z are whole-row copies or VOID; the two
                // frame bytes of every row and, for periodic x with padded rows, the copy of x = 0 at
                // x = nx are recomputed one by one.  One round of loads, then the stores.
                const int xpad = (g.per[0] && g.nx < g.P && x0 < g.nx && x0 + kTileX > g.nx) ? g.nx : -1;
                const bool drop_wrap = lava_mode && (g.per[0] || g.per[1]);
                int row_at = -1, frame_at = -1, drow_at = -1, dframe_at = -1;
                uint4 row_v = make_uint4(~0u, ~0u, ~0u, ~0u), drow_v = row_v;
                uint8_t frame_v = kVoid;
                int8_t dframe_v = -1;
                if (tid < halo_rows * 4) {
                    const int r = tid >> 2, ch = tid & 3;
                    int yy = y0 - hy_on + r % HY, zz = z0 - hz_on + r / HY;
                    if (!(yy >= 0 && yy < g.ny && zz >= 0 && zz < g.nz)) {
                        row_at = r * kSmemRowBytes + kRowOff + 16 * ch;
                        if (halo_axis(yy, g.ny, g.per[1]) && halo_axis(zz, g.nz, g.per[2]))
                            row_v = *reinterpret_cast<const uint4*>(T + pidx(g, x0 + 16 * ch, yy, zz));
                    }
                }
                if (tid < halo_rows * 3) {
                    const int r = tid / 3, which = tid % 3;
                    int xx = which == 0 ? x0 - 1 : (which == 1 ? x0 + kTileX : xpad);
                    int yy = y0 - hy_on + r % HY, zz = z0 - hz_on + r / HY;
                    if (!(which == 2 && xpad < 0) &&
                        !(xx >= 0 && xx < g.nx && yy >= 0 && yy < g.ny && zz >= 0 && zz < g.nz)) {
                        frame_at = r * kSmemRowBytes + kRowOff + (xx - x0);
                        const bool yz_in = yy >= 0 && yy < g.ny && zz >= 0 && zz < g.nz;
                        if (xwrap && yz_in && (xx == -1 || xx == g.nx))
                            frame_v = xx < 0 ? sl.xside[0][r * 16 + 15] : sl.xside[1][r * 16];  // loaded with the boxes
                        else if (halo_axis(xx, g.nx, g.per[0]) && halo_axis(yy, g.ny, g.per[1]) && halo_axis(zz, g.nz, g.per[2]))
                            frame_v = T[pidx(g, xx, yy, zz)];
                    }
                }
                if (drop_wrap) {
                    // drop depths are read only where the staged type is AIR: only periodic copies matter
                    const int c = tid - (kThreads - 4 * drop_rows);  // the last 4 * drop_rows threads
                    if (c >= 0 && c < drop_rows * 4) {
                        const int r = c >> 2, ch = c & 3;
                        int yy = y0 - hy_on + r % HY;
                        const int zz = z0 + r / HY;
                        if (zz < g.nz && !(yy >= 0 && yy < g.ny) && halo_axis(yy, g.ny, g.per[1])) {
                            drow_at = r * kSmemRowBytes + kRowOff + 16 * ch;
                            drow_v = *reinterpret_cast<const uint4*>(k.drop + pidx(g, x0 + 16 * ch, yy, zz));
                        }
                    }
                    const int f = tid - (kThreads - 3 * drop_rows);  // the last 3 * drop_rows threads
                    if (f >= 0 && f < drop_rows * 3) {
                        const int r = f / 3, which = f % 3;
                        int xx = which == 0 ? x0 - 1 : (which == 1 ? x0 + kTileX : xpad);
                        int yy = y0 - hy_on + r % HY;
                        const int zz = z0 + r / HY;
                        const int at = r * kSmemRowBytes + kRowOff + (xx - x0);
                        if (!(which == 2 && xpad < 0) && zz < g.nz && !(xx >= 0 && xx < g.nx && yy >= 0 && yy < g.ny)) {
                            if (xwrap && yy >= 0 && yy < g.ny && (xx == -1 || xx == g.nx)) {
                                dframe_at = at;
                                dframe_v = sl.xside_drop[xx < 0 ? 0 : 1][r * 16 + (xx < 0 ? 15 : 0)];
                            } else if (halo_axis(xx, g.nx, g.per[0]) && halo_axis(yy, g.ny, g.per[1])) {
                                dframe_at = at;
                                dframe_v = k.drop[pidx(g, xx, yy, zz)];
                            }
                        }
                    }
                }
                if (row_at >= 0) *reinterpret_cast<uint4*>(sl.type + row_at) = row_v;
                if (drow_at >= 0) *reinterpret_cast<uint4*>(sl.drop + drow_at) = drow_v;
                __syncthreads();  // frame bytes after the row copies (a frame byte of an outside row)
                if (frame_at >= 0) sl.type[frame_at] = frame_v;
                if (dframe_at >= 0) sl.drop[dframe_at] = dframe_v;
                __syncthreads();
            }

            const int y = y0 + ly, z = z0 + lz, x = x0 + 4 * xq;
            const bool valid = y < g.ny && z < g.nz;
            const unsigned own = (z >= k.own_z0 && z < k.own_z1) ? 1u : 0u;  // counted in the step's sums
            const int64_t p = pidx(g, valid ? x : 0, valid ? y : 0, valid ? z : 0);
            const int hr = hr_of(ly, lz, hy_on, hz_on, HY);
            const uint8_t* rowp = sl.type + hr * kSmemRowBytes + kRowOff + 4 * xq;
            uint32_t w = valid ? win_mid(rowp) : 0xFFFFFFFFu;
            if (x + 4 > g.nx) w |= 0xFFFFFFFFu << (8 * max(0, g.nx - x));  // padding cells stay VOID
            const int cell = row * kTileX + 4 * xq;

            bool any_lava = false, any_changed = false;
            uint32_t surv = 0;  // bytes of the thread's cells that are LAVA after the step
            unsigned nbas = 0, ncand = 0;
            uint32_t bas[4], cand[4];
            const uint32_t g0 = (uint32_t)(x + g.nx * (y + g.ny * z));
            const uint32_t lava_m = __vcmpeq4(w, 0x02020202u);
            uint32_t cand_m = __vcmpeq4(w, 0u);
            if (cand_m) {
                // An AIR cell can gain LAVA only from a source at its own level or above (same-level
                // spread, falls), or, in lava mode, by ponding from the cell straight below when it lies at
                // or below its column's spill level (gatherLavaCandidates, LavaCA.hpp:462-519); in classic
                // mode from any LAVA neighbour.
                uint32_t near = 0;
                if (lava_mode) {
                    // A same-level source needs dropDepth(c) == D(n) >= 0, a diagonal one above needs
                    // dropDepth(c) == 0; a LAVA cell straight above always feeds (a fall).  Most AIR
                    // cells next to LAVA lie over it (dropDepth -1) and are left out here.
                    const uint32_t dc = win_mid(reinterpret_cast<const uint8_t*>(sl.drop) +
                                                ((ly + hy_on) + HY * lz) * kSmemRowBytes + kRowOff + 4 * xq);
                    const uint32_t lands = __vcmpges4(dc, 0u), flat = __vcmpeq4(dc, 0u);
                    // the same-level sources count only where the cell lands, the ones above only where
                    // it is flat: a thread whose cells do neither (AIR over LAVA) skips those windows
                    uint32_t level = 0, above = 0, fall = 0;
                    for (int dy = -hy_on; dy <= hy_on; ++dy) {
                        const uint8_t* rp = sl.type + (hr + dy) * kSmemRowBytes + kRowOff + 4 * xq;
                        if (lands)
                            level |= __vcmpeq4(win_left(rp), 0x02020202u) | __vcmpeq4(win_mid(rp), 0x02020202u) |
                                     __vcmpeq4(win_right(rp), 0x02020202u);
                        if (hz_on) {
                            const uint8_t* ap = rp + HY * kSmemRowBytes;
                            if (dy == 0) fall = __vcmpeq4(win_mid(ap), 0x02020202u);
                            if (flat)
                                above |= __vcmpeq4(win_left(ap), 0x02020202u) | __vcmpeq4(win_right(ap), 0x02020202u) |
                                         (dy != 0 ? __vcmpeq4(win_mid(ap), 0x02020202u) : 0u);
                        }
                    }
                    near = (level & lands) | (above & flat) | fall;
                } else {
                    for (int dz = -hz_on; dz <= hz_on; ++dz)
                        for (int dy = -hy_on; dy <= hy_on; ++dy) {
                            const uint8_t* rp = sl.type + (hr + dy + HY * dz) * kSmemRowBytes + kRowOff + 4 * xq;
                            near |= __vcmpeq4(win_left(rp), 0x02020202u) | __vcmpeq4(win_mid(rp), 0x02020202u) |
                                    __vcmpeq4(win_right(rp), 0x02020202u);
                        }
                }
                if (stage_spill && k.ponding) {
                    uint32_t m = __vcmpeq4(win_mid(rowp - HY * kSmemRowBytes), 0x02020202u);
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        if (z > sl.spill[ly * kTileX + 4 * xq + j]) m &= ~(0xFFu << (8 * j));
                    near |= m;
                }
                cand_m &= near;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if ((cand_m >> (8 * j)) & 0xFF) cand[ncand++] = g0 + j;
            }
            uint32_t wout = w;
            if (lava_m && lava_mode) {
                // D(n) of the LAVA cells: support from the cell below, then the largest drop depth of
                // the AIR side cells (dz = 0 offsets of every variant), -1 without support.
                uint32_t sup = 0xFFFFFFFFu;
                if (z > 0) {
                    const uint32_t below = win_mid(rowp - HY * kSmemRowBytes);
                    sup = __vcmpeq4(below, 0x01010101u) | __vcmpeq4(below, 0x03030303u);
                    uint32_t lb = __vcmpeq4(below, 0x02020202u);
                    if (lb && stage_spill) {
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            if (!(z - 1 < sl.spill[ly * kTileX + 4 * xq + j])) lb &= ~(0xFFu << (8 * j));
                        sup |= lb;
                    }
                }
                uint32_t acc = 0;
                const uint8_t* dropc =
                    reinterpret_cast<const uint8_t*>(sl.drop) + ((ly + hy_on) + HY * lz) * kSmemRowBytes + kRowOff + 4 * xq;
                // without support no side cell matters: D(n) is -1 for every unsupported LAVA cell
                // (and D(n) of the thread's other cells is never read)
                const bool scan = (sup & lava_m) != 0;
#pragma unroll
                for (int sy = -1; sy <= 1 && scan; ++sy) {
                    const unsigned bits = (k.side_mask >> (3 * (sy + 1))) & 7u;
                    if (!bits) continue;
                    const uint8_t* tp = rowp + sy * kSmemRowBytes;
                    const uint8_t* dp = dropc + sy * kSmemRowBytes;
                    if (bits & 1u) acc = __vmaxs4(acc, win_left(dp) & __vcmpeq4(win_left(tp), 0u));
                    if (bits & 2u) acc = __vmaxs4(acc, win_mid(dp) & __vcmpeq4(win_mid(tp), 0u));
                    if (bits & 4u) acc = __vmaxs4(acc, win_right(dp) & __vcmpeq4(win_right(tp), 0u));
                }
                *reinterpret_cast<uint32_t*>(k.desc + p) = (acc & sup) | ~sup;
            }
            if (lava_m) {
                if (k.classic) {
                    my_active += own * (__popc(lava_m) >> 3);
                    any_lava = true;
                    surv = lava_m;
                } else {
                    // the state of the thread's four cells, read only where one of them is LAVA
                    const int4 f4 = *reinterpret_cast<const int4*>(&sl.flow[cell]);
                    const float4 t4 = *reinterpret_cast<const float4*>(&sl.temp[cell]);
                    const uint2 s2 = *reinterpret_cast<const uint2*>(&sl.solid[cell]);
                    float te[4] = {t4.x, t4.y, t4.z, t4.w};
                    const int32_t fl[4] = {f4.x, f4.y, f4.z, f4.w};
                    uint32_t so[2] = {s2.x, s2.y};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        if (!((lava_m >> (8 * j)) & 0xFF)) continue;
                        const float before = te[j];
                        bool vent = false;
                        if (erupting && tile_vent && fl[j] > 0 && fl[j] < k.vent_slots) {
                            const int4 vc = __ldg(k.vents + fl[j]);
                            vent = vc.x == x + j && vc.y == y && vc.z == z;
                        }
                        const float nt = vent ? k.erupt_temp : __fsub_rn(before, k.cool_ambient);
                        te[j] = nt;
                        if (nt < k.solidus) {
                            const uint32_t half = (j & 1) * 16;
                            wout = (wout & ~(0xFFu << (8 * j))) | ((uint32_t)kBasalt << (8 * j));
                            so[j >> 1] = (so[j >> 1] & ~(0xFFFFu << half)) | (stamp << half);
                            my_changed += own;
                            bas[nbas++] = g0 + j;
                            any_changed = true;
                        } else {
                            my_active += own;
                            any_lava = true;
                            surv |= 0xFFu << (8 * j);
                            if (nt != before) {
                                my_changed += own;
                                any_changed = true;
                            }
                        }
                    }
                    *reinterpret_cast<float4*>(&sl.temp[cell]) = make_float4(te[0], te[1], te[2], te[3]);
                    *reinterpret_cast<uint2*>(&sl.solid[cell]) = make_uint2(so[0], so[1]);
                }
            }
            *reinterpret_cast<uint32_t*>(&sl.own_type[cell]) = wout;
            if (__any_sync(0xFFFFFFFFu, nbas != 0))
                warp_append(k.chg_list[nxt], &ctrl->chg_count[nxt], k.chg_cap, lane, nbas, bas);

            // candidates: block-wide positions in the shared buffer
            unsigned incl = ncand;
            if (__any_sync(0xFFFFFFFFu, ncand != 0)) {  // most warps of a tile list no candidate
#pragma unroll
                for (int off = 1; off < 32; off <<= 1) {
                    const unsigned u = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                    if (lane >= off) incl += u;
                }
            }
            if (lane == 31) s_wtot[warp] = incl;
            // the faces of the tile that LAVA after the step touches (bits 2-7: -x, +x, -y, +y, -z,
            // +z): a neighbouring tile can change in the next step only if LAVA lies within one cell
            // of it, so the schedule visits only the neighbours across touched faces
            unsigned faces = 0;
            if (surv && valid) {
                const int xlast = min(kTileX, g.nx - x0) - 1, jl = xlast - 4 * xq;
                if (xq == 0 && (surv & 0xFFu)) faces |= 1u << 2;
                if (jl >= 0 && jl < 4 && ((surv >> (8 * jl)) & 0xFFu)) faces |= 1u << 3;
                if (ly == 0) faces |= 1u << 4;
                if (ly == min(g.TY, g.ny - y0) - 1) faces |= 1u << 5;
                if (lz == 0) faces |= 1u << 6;
                if (lz == min(g.TZ, g.nz - z0) - 1) {
                    bool up = k.classic;
                    if (!up && stage_spill && k.ponding)
#pragma unroll
                        for (int j = 0; j < 4; ++j)
                            up = up || (((surv >> (8 * j)) & 0xFFu) && z + 1 <= sl.spill[ly * kTileX + 4 * xq + j]);
                    if (up) faces |= 1u << 7;
                }
            }
            unsigned bits = (any_lava ? 1u : 0u) | (any_changed ? 2u : 0u) | faces;
            bits = __reduce_or_sync(0xFFFFFFFFu, bits);
            if (lane == 0 && bits) atomicOr(&s_flags[rit & 1], bits);
            fence_proxy_async();  // the slot's results are read by the TMA stores below
            __syncthreads();
            if (tid == 0) store_tile(si, x0, y0, z0);
            const unsigned tf = s_flags[rit & 1];
            if (tid == 32) s_flags[(rit + 1) & 1] = 0;
            ++rit;
            unsigned wbase = 0, total = 0;
            for (int w2 = 0; w2 < kThreads / 32; ++w2) {
                const unsigned v = s_wtot[w2];
                wbase += w2 < warp ? v : 0u;
                total += v;
            }
            for (unsigned j = 0, pos = nbuf + wbase + incl - ncand; j < ncand; ++j) s_cand[pos + j] = cand[j];
            nbuf += total;
            if (tid == 0 && tf) {
                s_sched_tile[nsched] = tile;
                s_sched_flag[nsched] = (uint8_t)tf;
            }
            if (tf) ++nsched;
            if (nsched == kMaxDeferred) flush_schedule();
            if (nbuf > kCandBuf - kTileCells) flush_cands();
        }
        tile_a = tile_b;
        mark_a = mark_b;
        vent_a = vent_b;
        tile_b = tile_c;
        mark_b = mark_c;
        vent_b = vent_c;
        tile_c = tile_d;
        if constexpr (kDyn) {
            i0 = r1;
            r1 = r2;
            r2 = r3;
            r3 = i4;
        } else {
            i0 += G;
        }
    }
    cp_async_wait_all();
    if (tid == 0) {
        // every slot fill that was issued has completed or is abandoned with the error flag set; the
        // stores must have left shared memory before the block exits
        bulk_wait_all();
    }
    if (failed) return;
    if (__syncthreads_or(nsched > 0)) flush_schedule();
    if (nbuf) flush_cands();

    const unsigned a = __reduce_add_sync(0xFFFFFFFFu, my_active);
    const unsigned c = __reduce_add_sync(0xFFFFFFFFu, my_changed);
    if (lane == 0) {
        s_red[0][warp] = a;
        s_red[1][warp] = c;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long sa = 0, sc = 0;
        for (int wv = 0; wv < kThreads / 32; ++wv) {
            sa += s_red[0][wv];
            sc += s_red[1][wv];
        }
        if (sa) atomicAdd(&ctrl->acc_active, sa);
        if (sc) atomicAdd(&ctrl->acc_changed, sc);
        if (tiles_done) atomicAdd(&ctrl->acc_tiles, (unsigned long long)tiles_done);
    }
}
template <class S>
__global__ __launch_bounds__(kThreads, 4) void ca_rules_kernel(const __grid_constant__ CaTensorMaps tm,
                                                               const __grid_constant__ CaKernelArgs k) {
    rules_body<S, false>(tm, k, blockIdx.x, gridDim.x);
}
// DENSE over many tiles per block: tiles handed out at run time (rules_body, kDyn)
template <class S>
__global__ __launch_bounds__(kThreads, 4) void ca_rules_dyn_kernel(const __grid_constant__ CaTensorMaps tm,
                                                                   const __grid_constant__ CaKernelArgs k) {
    rules_body<S, true>(tm, k, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------------------------------
// Rules, candidate pass: resolves the listed AIR cells (gatherLavaCandidates / vote / solidus,
// updateLava's AIR branch, LavaCA.hpp:1121-1134), writes the ones that gain LAVA into the next
// buffer, lists their type change, schedules their tiles' neighbourhoods, and the last block
// finishes the step (finishStep, LavaCA.hpp:1206-1229).
// ------------------------------------------------------------------------------------------
constexpr int kCandThreads = 128;
__device__ __forceinline__ void cand_body(const CaKernelArgs& k, uint32_t bid, uint32_t nblk) {
    __shared__ unsigned long long s_red[kCandThreads / 32];
    __shared__ bool s_last;
    CaCtrl* ctrl = k.ctrl;
    if (ctrl->stop || ctrl->error) return;
    const uint32_t t = ctrl->steps;
    const int cur = t & 1, nxt = cur ^ 1;
    const CaGeom& g = k.g;
    const uint8_t* T = k.type[cur];
    const int32_t* F = k.flow[cur];
    const float* Te = k.temp[cur];
    const uint32_t stamp = min(t, 65535u);
    const uint64_t prefix = hash_prefix(k.seed, t);
    const unsigned n = ctrl->cand_count;
    // the blocks that hold listed cells take part (at least one, which finishes the step); the others
    // leave at once, so a short list costs a few blocks instead of the whole grid
    const unsigned parts = max(1u, min(nblk, (n + kCandThreads - 1) / kCandThreads));
    if (bid >= parts) return;
    const int lane = threadIdx.x & 31;
    unsigned born = 0;
    const uint64_t stride = (uint64_t)nblk * kCandThreads;
    // warp-uniform loop (the appends below use full-warp collectives)
    for (uint64_t base = bid * (uint64_t)kCandThreads; base < n; base += stride) {
        const uint64_t j = base + threadIdx.x;
        bool gained = false;
        uint32_t gi = 0, tile = 0;
        unsigned faces = 0;  // of the gained cell in its tile
        if (j < n) {
            gi = k.cand_list[j];
            const uint32_t r = gi / (uint32_t)g.nx;
            const int x = (int)(gi - r * (uint32_t)g.nx);
            const int y = (int)(r % (uint32_t)g.ny);
            const int z = (int)(r / (uint32_t)g.ny);
            int32_t nf;
            float nt;
            if (air_gains_lava(k, T, F, Te, x, y, z, prefix, gi + k.gidx_base, &nf, &nt)) {
                const int64_t p = pidx(g, x, y, z);
                k.type[nxt][p] = kLava;
                k.flow[nxt][p] = nf;
                k.temp[nxt][p] = nt;
                k.solid[nxt][p] = 0;
                k.arrival[nxt][p] = (uint16_t)stamp;
                gained = true;
                born += (z >= k.own_z0 && z < k.own_z1) ? 1u : 0u;
                const int tx = x / kTileX, ty = y / g.TY, tz = z / g.TZ;
                tile = (uint32_t)tx + (uint32_t)g.tiles_x * ((uint32_t)ty + (uint32_t)g.tiles_y * (uint32_t)tz);
                const int sp = (!k.classic && k.spill != nullptr) ? __ldg(k.spill + x + (int64_t)g.nx * y) : 0;
                faces = cell_faces(g, x, y, z, tx * kTileX, ty * g.TY, tz * g.TZ, feeds_up(k, sp, z));
            }
        }
        if (!k.classic && __any_sync(0xFFFFFFFFu, gained))
            warp_append(k.chg_list[nxt], &ctrl->chg_count[nxt], k.chg_cap, lane, gained ? 1u : 0u, &gi);
        // the tiles that gained lava have their neighbourhoods scheduled by the whole warp, once each:
        // the tile itself and the neighbours across the faces its new LAVA cells lie on
        unsigned todo = __ballot_sync(0xFFFFFFFFu, gained);
        while (todo) {
            const int src = __ffs(todo) - 1;
            const uint32_t tl = __shfl_sync(0xFFFFFFFFu, tile, src);
            const bool mine = gained && tile == tl;
            todo &= ~__ballot_sync(0xFFFFFFFFu, mine);
            const unsigned f = __reduce_or_sync(0xFFFFFFFFu, mine ? faces : 0u);
            schedule_around(k, tl, t, nxt, lane, faces_reach(f, lane, !k.classic), true);
        }
    }
    const unsigned b = __reduce_add_sync(0xFFFFFFFFu, born);
    if (lane == 0) s_red[threadIdx.x >> 5] = b;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sb = 0;
        for (int wv = 0; wv < kCandThreads / 32; ++wv) sb += s_red[wv];
        if (sb) {
            atomicAdd(&ctrl->acc_active, sb);
            atomicAdd(&ctrl->acc_changed, sb);
            atomicAdd(&ctrl->acc_born, sb);
        }
        // the ticket with acquire-release semantics: this block's sums are visible before its ticket,
        // and the last block sees every other block's sums after its own
        unsigned old;
        asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;\n" : "=r"(old) : "l"(&ctrl->ticket) : "memory");
        s_last = old == parts - 1;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        const unsigned long long active = atomicExch(&ctrl->acc_active, 0ull);
        const unsigned long long changed = atomicExch(&ctrl->acc_changed, 0ull);
        const unsigned long long nborn = atomicExch(&ctrl->acc_born, 0ull);
        const unsigned long long tiles = atomicExch(&ctrl->acc_tiles, 0ull);
        ctrl->ticket = 0;
        ctrl->cand_count = 0;
        const uint64_t air = ctrl->air - nborn;
        ctrl->air = air;
        ctrl->lava = active;
        ctrl->tiles_processed += tiles;
        k.hist_active[t] = active;
        k.hist_changed[t] = changed;
        const uint32_t steps = t + 1;
        int stop = VCA_STOP_RUNNING;
        if (k.slab) {
            // the stop rule needs the sums over all slabs: the caller decides (vca_ca_slab_stop)
        } else if (!ctrl->classic && active == 0) stop = VCA_STOP_NO_LAVA;
        else if (ctrl->classic && air == 0) stop = VCA_STOP_NO_AIR;
        else if (changed == 0 && !ctrl->random_nb) stop = VCA_STOP_NO_CHANGE;
        else if ((int)steps >= ctrl->max_steps) stop = VCA_STOP_MAX_STEPS;
        ctrl->stop = stop;
        ctrl->steps = steps;  // read by the next kernels, after this launch has completed
    }
}
__global__ __launch_bounds__(kCandThreads, 4) void ca_cand_kernel(const __grid_constant__ CaKernelArgs k) {
    cand_body(k, blockIdx.x, gridDim.x);
}

// ------------------------------------------------------------------------------------------
// Simulation::flowSums (Simulation.cpp:408-466) over the current state: per flowId f in 1..flows
// the LAVA and BASALT cells and the largest squared horizontal distance from the vent of f.  With
// few flows each block sums into shared memory first (one global atomic per flow and block).
// ------------------------------------------------------------------------------------------
constexpr int kFlowPrivMax = 1024;  // flows summed in shared memory (3 * 8 B each)
__global__ void ca_flow_stats_kernel(const uint8_t* T, const int32_t* F, CaGeom g, const int4* vents, int vent_slots,
                                     int flows, unsigned long long* out) {
    extern __shared__ unsigned long long s_sum[];  // [3][flows + 1] when flows <= kFlowPrivMax
    const bool priv = flows <= kFlowPrivMax;
    const int m = flows + 1;
    unsigned long long* acc = priv ? s_sum : out;
    if (priv) {
        for (int i = threadIdx.x; i < 3 * m; i += blockDim.x) s_sum[i] = 0ull;
        __syncthreads();
    }
    const uint64_t cells = (uint64_t)g.nx * g.ny * g.nz;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cells; i += stride) {
        const uint64_t r = i / (uint64_t)g.nx;
        const int x = (int)(i - r * (uint64_t)g.nx);
        const int64_t p = (int64_t)x + (int64_t)g.P * (int64_t)r;
        const int t = T[p];
        if (t != kLava && t != kBasalt) continue;
        const int32_t f = F[p];
        if (f <= 0 || f > flows) continue;
        const int y = (int)(r % (uint64_t)g.ny);
        atomicAdd(&acc[(t == kLava ? 0 : m) + f], 1ull);
        if (f < vent_slots) {
            const int4 v = vents[f];
            const long long dx = x - v.x, dy = y - v.y;
            atomicMax(&acc[2 * m + f], (unsigned long long)(dx * dx + dy * dy));
        }
    }
    if (priv) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * m; i += blockDim.x) {
            const unsigned long long v = s_sum[i];
            if (v == 0ull) continue;
            if (i < 2 * m) atomicAdd(&out[i], v);
            else atomicMax(&out[i], v);
        }
    }
}

// ------------------------------------------------------------------------------------------
// Set-up kernels.
// ------------------------------------------------------------------------------------------
// Per-tile LAVA flag of the current state and the LAVA / AIR totals (countInitialState,
// LavaCA.hpp:1252-1280), accumulated into ctrl->acc_active / acc_born.
__global__ __launch_bounds__(kThreads) void ca_tile_init_kernel(const __grid_constant__ CaKernelArgs k, int cur) {
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
            air = __popc(__vcmpeq4(w, 0u)) >> 3;  // padding cells are VOID, so they count as neither
        }
        const int any = __syncthreads_or(lava > 0);
        if (threadIdx.x == 0) k.tile_flags[tile] = (k.tile_flags[tile] & 2u) | (any ? 1u : 0u);
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

// The tile list of the first step: every tile within one tile of a tile holding LAVA.
__global__ void ca_init_schedule_kernel(const __grid_constant__ CaKernelArgs k, uint32_t t0) {
    const CaGeom& g = k.g;
    const int cur = t0 & 1;
    for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x; base < k.ntiles; base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t tile = base + threadIdx.x;
        bool process = false;
        if (tile < k.ntiles) {
            const int tx = (int)(tile % g.tiles_x);
            const uint64_t r = tile / g.tiles_x;
            const int ty = (int)(r % g.tiles_y), tz = (int)(r / g.tiles_y);
            for (int dz = -1; dz <= 1 && !process; ++dz)
                for (int dy = -1; dy <= 1 && !process; ++dy)
                    for (int dx = -1; dx <= 1 && !process; ++dx) {
                        int xx = tx + dx, yy = ty + dy, zz = tz + dz;
                        if (!wrap_axis(xx, g.tiles_x, g.per[0]) || !wrap_axis(yy, g.tiles_y, g.per[1]) ||
                            !wrap_axis(zz, g.tiles_z, g.per[2]))
                            continue;
                        process = (k.tile_flags[xx + (uint64_t)g.tiles_x * (yy + (uint64_t)g.tiles_y * zz)] & 1u) != 0;
                    }
            if (process) k.tile_mark[cur][tile] = 2u * (t0 + 1u) + 1u;
        }
        const unsigned ballot = __ballot_sync(0xFFFFFFFFu, process);
        const unsigned lane = threadIdx.x & 31;
        unsigned slot = 0;
        if (lane == 0 && ballot) slot = atomicAdd(&k.ctrl->list_count[cur], (unsigned)__popc(ballot));
        slot = __shfl_sync(0xFFFFFFFFu, slot, 0);
        if (process) k.tile_list[cur][slot + __popc(ballot & ((1u << lane) - 1u))] = (uint32_t)tile;
    }
}

// Fill the padding cells x in [nx, P) of every row with VOID (both buffers).
// The control block copied by one warp into host-mapped pinned memory.  A kernel, not a
// device-to-host copy: such a copy queues on the copy engines behind any large download of another
// handle on the same device, and the next step graph would wait behind it.
__global__ void ca_ctrl_snapshot_kernel(const CaCtrl* src, CaCtrl* dst) {
    static_assert(sizeof(CaCtrl) % sizeof(uint32_t) == 0, "CaCtrl is copied as words");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    volatile uint32_t* d = reinterpret_cast<volatile uint32_t*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(CaCtrl) / sizeof(uint32_t)); i += 32) d[i] = s[i];
}

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

// ------------------------------------------------------------------------------------------
// Batched stepping: one launch of each step kernel for many grids.  Every block serves one member
// grid: the block maps give, per block of a launch, the member slot and the block's index among that
// member's blocks (slot -1: idle).  A block copies its member's arguments into shared memory and
// runs the same body as the single-grid kernel with that block index and count, so each member steps
// exactly as it would alone.  The tensor maps stay in global memory (TMA reads them from there).
// ------------------------------------------------------------------------------------------
struct CaBatchView {
    const CaTensorMaps* tm;    // per member slot
    const CaKernelArgs* args;  // per member slot
    const int2* rules_map;     // per block of the drop / rules launches: (slot, block within the member)
    const int2* cand_map;      // per block of the candidate launch
    const int* rules_n;        // per slot: its blocks in the drop / rules launches (0: free slot)
    const int* cand_n;         // per slot: its blocks in the candidate launch
    int4* status;              // per slot after a graph: (stop, error, steps, next tiles) or (-1, 0, 0, 0)
    int slots;
};

__device__ __forceinline__ void load_args(CaKernelArgs& dst, const CaKernelArgs& src) {
    static_assert(sizeof(CaKernelArgs) % sizeof(uint2) == 0, "copied as 8-byte words");
    const uint2* from = reinterpret_cast<const uint2*>(&src);
    uint2* to = reinterpret_cast<uint2*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(CaKernelArgs) / sizeof(uint2)); i += blockDim.x) to[i] = from[i];
    __syncthreads();
}

__global__ __launch_bounds__(kThreads, 4) void ca_drop_batch_kernel(const __grid_constant__ CaBatchView b) {
    const int2 m = b.rules_map[blockIdx.x];
    if (m.x < 0) return;
    __shared__ __align__(16) CaKernelArgs s_k;
    load_args(s_k, b.args[m.x]);
    drop_body(s_k, 0, (uint32_t)m.y, (uint32_t)b.rules_n[m.x]);
}

__global__ __launch_bounds__(kThreads, 4) void ca_rules_batch_kernel(const __grid_constant__ CaBatchView b) {
    const int2 m = b.rules_map[blockIdx.x];
    if (m.x < 0) return;
    __shared__ __align__(16) CaKernelArgs s_k;
    const CaTensorMaps& tm = b.tm[m.x];
    if (threadIdx.x == 0) {
        // the maps were written into global memory by a copy since the last launch: order the
        // tensor-map proxy's reads after that write
        const char* base = reinterpret_cast<const char*>(&tm);
        for (int off = 0; off < (int)sizeof(CaTensorMaps); off += (int)sizeof(CUtensorMap))
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(base + off) : "memory");
    }
    load_args(s_k, b.args[m.x]);
    rules_body<ShapeA, false>(tm, s_k, (uint32_t)m.y, (uint32_t)b.rules_n[m.x]);
}

__global__ __launch_bounds__(kCandThreads, 4) void ca_cand_batch_kernel(const __grid_constant__ CaBatchView b) {
    const int2 m = b.cand_map[blockIdx.x];
    if (m.x < 0) return;
    __shared__ __align__(16) CaKernelArgs s_k;
    load_args(s_k, b.args[m.x]);
    cand_body(s_k, (uint32_t)m.y, (uint32_t)b.cand_n[m.x]);
}

// Stop state of every member after a graph of steps, and the tiles its next step will visit,
// gathered for one copy to the host.
__global__ void ca_batch_status_kernel(const __grid_constant__ CaBatchView b) {
    for (int i = threadIdx.x; i < b.slots; i += blockDim.x) {
        int4 st = make_int4(-1, 0, 0, 0);
        if (b.rules_n[i] > 0) {
            const CaCtrl* c = b.args[i].ctrl;
            st = make_int4(c->stop, c->error, (int)c->steps, (int)c->list_count[c->steps & 1u]);
        }
        b.status[i] = st;
    }
}

// Vents / seeds: CellState{Lava, flowId, temp, 0, 0} (LavaCA::placeSeeds, LavaCA.hpp:215-220).
__global__ void ca_seed_kernel(const __grid_constant__ CaKernelArgs k, const int4* seeds, int count, int cur, float temp) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const int4 s = seeds[i];
        const int64_t p = pidx(k.g, s.x, s.y, s.z);
        k.type[cur][p] = kLava;
        k.flow[cur][p] = s.w;
        k.temp[cur][p] = temp;
        k.solid[cur][p] = 0;
        k.arrival[cur][p] = 0;
    }
}

}  // namespace vca

// ============================================================================================
// Host side
// ============================================================================================
using namespace vca;

namespace {

// batched: the arguments of a batch member, whose blocks the batch shares out.  A single grid whose
// every tile has a rules block of its own runs every tile every step under VCA_SWEEP_ACTIVE (the
// tile list and its atomics buy nothing there, and the results are the same either way).
CaKernelArgs make_args(const vca_ca* h, bool batched = false) {
    CaKernelArgs k;
    std::memset(&k, 0, sizeof(k));
    k.g = h->geom;
    k.classic = h->desc.mode == VCA_MODE_CLASSIC;
    k.ponding = h->desc.ponding != 0;
    k.dense = h->desc.sweep == VCA_SWEEP_DENSE ||
              (h->desc.sweep == VCA_SWEEP_ACTIVE && !batched && h->ntiles <= (uint64_t)h->grid_blocks);
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
    k.side_mask = 0;
    for (int i = 0; i < h->tables_host.nside; ++i)
        k.side_mask |= 1u << (3 * (h->tables_host.side[i][1] + 1) + (h->tables_host.side[i][0] + 1));
    for (int b = 0; b < 2; ++b) {
        k.type[b] = h->type[b];
        k.flow[b] = h->flow[b];
        k.temp[b] = h->temp[b];
        k.solid[b] = h->solid[b];
        k.arrival[b] = h->arrival[b];
        k.tile_list[b] = h->tile_list[b];
    }
    k.tile_flags = h->tile_flags;
    k.tile_mark[0] = h->tile_mark[0];
    k.tile_mark[1] = h->tile_mark[1];
    k.desc = h->desc_plane;
    k.drop = h->drop_plane;
    k.chg_list[0] = h->chg_list[0];
    k.chg_list[1] = h->chg_list[1];
    k.chg_cap = h->chg_cap;
    k.cand_list = h->cand_list;
    k.spill = h->has_terrain ? h->spill : nullptr;
    k.vents = h->vents;
    k.vent_slots = h->vent_slots;
    k.tables = h->tables_host;
    k.ctrl = h->ctrl;
    k.hist_active = h->hist_active;
    k.hist_changed = h->hist_changed;
    k.ntiles = h->ntiles;
    k.slab = h->slab ? 1 : 0;
    k.gidx_base = h->slab ? (uint64_t)h->geom.nx * h->geom.ny * (uint64_t)h->slab_z0 : 0;
    k.own_z0 = h->slab ? h->own_z0 : 0;
    k.own_z1 = h->slab ? h->own_z1 : h->geom.nz;
    return k;
}

vca_status check(const vca_ca* h) {
    if (h == nullptr) {
        set_error("null vca_ca handle");
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

// A handle that a batch is stepping takes no other call until it leaves the batch.
vca_status not_in_batch(const vca_ca* h, const char* who) {
    if (h->batch != nullptr) {
        set_error(std::string(who) + ": the handle is a member of a batch (vca_ca_batch_remove, or wait for it to stop)");
        return VCA_ERR_STATE;
    }
    return VCA_OK;
}

void drop_graph(vca_ca* h) {
    if (h->graph_exec) cudaGraphExecDestroy(h->graph_exec);
    h->graph_exec = nullptr;
}

// Pull the control block to the host mirror.
vca_status sync_ctrl(vca_ca* h) {
    ca_ctrl_snapshot_kernel<<<1, 32, 0, h->stream>>>(h->ctrl, h->ctrl_host_dev);
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = (int)h->ctrl_host->steps;
    h->stop = h->ctrl_host->stop;
    if (h->ctrl_host->error) {
        set_error("vca_ca: a bounded device wait (TMA tile copy) ran out; the run was stopped");
        return VCA_ERR_TIMEOUT;
    }
    return VCA_OK;
}

// Totals and initial stop state of the current buffer, the first tile list, and a copy of the
// current buffer into the other one (both buffers equal: the ACTIVE schedule relies on it).
vca_status init_state(vca_ca* h, int steps_done) {
    const int cur = steps_done & 1, oth = cur ^ 1;
    const size_t n = h->plane_cells;
    VCA_CUDA(cudaMemcpyAsync(h->type[oth], h->type[cur], n, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->flow[oth], h->flow[cur], n * 4, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->temp[oth], h->temp[cur], n * 4, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->solid[oth], h->solid[cur], n * 2, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->arrival[oth], h->arrival[cur], n * 2, cudaMemcpyDeviceToDevice, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->tile_mark[0], 0, h->ntiles * 4, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->tile_mark[1], 0, h->ntiles * 4, h->stream));
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
    ca_drop_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k, 1);
    VCA_CUDA(cudaGetLastError());
    {
        const int sb = (int)std::min<uint64_t>((h->ntiles + 255) / 256, 4096);
        ca_init_schedule_kernel<<<sb, 256, 0, h->stream>>>(k, (uint32_t)steps_done);
        VCA_CUDA(cudaGetLastError());
    }
    if (vca_status s = sync_ctrl(h)) return s;
    CaCtrl* m = h->ctrl_host;
    const uint64_t lava = m->acc_active, air = m->acc_born;
    m->acc_active = 0;
    m->acc_born = 0;
    m->lava = lava;
    m->air = air;
    // LavaCA::countInitialState (LavaCA.hpp:1272-1279)
    int stop = VCA_STOP_RUNNING;
    if (h->slab) {  // the counts of one slab do not decide: the caller sets the stop (vca_ca_slab_stop)
        if (h->desc.max_steps <= steps_done) stop = VCA_STOP_MAX_STEPS;
    } else if (!c.classic && lava == 0) stop = VCA_STOP_NO_LAVA;
    else if (c.classic && air == 0) stop = VCA_STOP_NO_AIR;
    else if (h->desc.max_steps <= steps_done) stop = VCA_STOP_MAX_STEPS;
    m->stop = stop;
    VCA_CUDA(cudaMemcpyAsync(h->ctrl, m, sizeof(CaCtrl), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->steps = steps_done;
    h->stop = stop;
    return VCA_OK;
}

// The rules pass of the handle's tile-shape family.
// Tiles handed out at run time pay where a block has many tiles of uneven cost: DENSE with at
// least 64 tiles per block (measured: c3 DENSE -20 %; with 14 tiles per block, c2, +12 %).
constexpr uint64_t kDynTilesPerBlock = 64;

template <class S>
void launch_rules_shape(const vca_ca* h, const CaKernelArgs& k) {
    const bool dyn = k.dense && h->ntiles >= kDynTilesPerBlock * (uint64_t)h->grid_blocks;
    if (dyn)
        ca_rules_dyn_kernel<S><<<h->grid_blocks, kThreads, rules_dyn_smem<S>(), h->stream>>>(h->tmaps, k);
    else
        ca_rules_kernel<S><<<h->grid_blocks, kThreads, rules_dyn_smem<S>(), h->stream>>>(h->tmaps, k);
}
void launch_rules(const vca_ca* h, const CaKernelArgs& k) {
    switch (h->geom.shape) {
        case 0: launch_rules_shape<ShapeA>(h, k); break;
        case 1: launch_rules_shape<ShapeB>(h, k); break;
        default: launch_rules_shape<ShapeC>(h, k); break;
    }
}

// Resident rules blocks per SM of a shape family: the smaller of the two forms' (they differ by
// 16 bytes of static shared memory).
template <class S>
cudaError_t rules_occupancy(int* per_sm) {
    int a = 0, b = 0;
    cudaError_t e = cudaFuncSetAttribute(ca_rules_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rules_dyn_smem<S>());
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(ca_rules_dyn_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rules_dyn_smem<S>());
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&a, ca_rules_kernel<S>, kThreads, rules_dyn_smem<S>());
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, ca_rules_dyn_kernel<S>, kThreads, rules_dyn_smem<S>());
    *per_sm = std::min(a, b);
    return e;
}

constexpr int kGraphSteps = 16;  // steps captured in one CUDA graph

// The launches of kGraphSteps steps, captured once per state set-up (the kernel arguments only
// change with the terrain, the vents or the state).  Launches after the stop exit at once.
vca_status ensure_graph(vca_ca* h, const CaKernelArgs& k) {
    // A captured graph stays valid while the arguments and launch shapes it was captured with are
    // unchanged (a resident handle running job after job on one space keeps them; make_args zeroes
    // the padding, so a byte comparison is exact).
    if (h->graph_exec && std::memcmp(&h->graph_args, &k, sizeof(k)) == 0 &&
        std::memcmp(&h->graph_tm, &h->tmaps, sizeof(h->tmaps)) == 0 && h->graph_grid == h->grid_blocks &&
        h->graph_cand == h->cand_blocks)
        return VCA_OK;
    drop_graph(h);
    VCA_CUDA(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < kGraphSteps; ++s) {
        ca_drop_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k, 0);
        launch_rules(h, k);
        ca_cand_kernel<<<h->cand_blocks, kCandThreads, 0, h->stream>>>(k);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(h->stream, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&h->graph_exec, graph, 0);
    h->graph_args = k;
    h->graph_tm = h->tmaps;
    h->graph_grid = h->grid_blocks;
    h->graph_cand = h->cand_blocks;
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        h->graph_exec = nullptr;
        return cuda_fail(e2, "cudaGraphInstantiate");
    }
    return VCA_OK;
}

// Whole-run path: graphs of kGraphSteps steps; the stop test of graph i is read while graph i+1 runs.
vca_status run_graphs(vca_ca* h, const CaKernelArgs& k) {
    if (vca_status s = ensure_graph(h, k)) return s;
    VCA_CUDA(cudaEventRecord(h->ev_a, h->stream));
    // graphs that can still do a step before max_steps (the stop rule can only end the run sooner)
    const int left = std::max(0, h->desc.max_steps - h->steps);
    const int needed = (left + kGraphSteps - 1) / kGraphSteps;
    int pending = -1;
    for (int launched = 0; launched < needed; ++launched) {
        const int slot = launched & 1;
        VCA_CUDA(cudaGraphLaunch(h->graph_exec, h->stream));
        ca_ctrl_snapshot_kernel<<<1, 32, 0, h->stream>>>(h->ctrl, h->ctrl_ring_dev + slot);
        VCA_CUDA(cudaGetLastError());
        VCA_CUDA(cudaEventRecord(h->ring_ev[slot], h->stream));
        h->launches += 3 * kGraphSteps + 1;
        if (pending >= 0) {
            VCA_CUDA(cudaEventSynchronize(h->ring_ev[pending]));
            if (h->ctrl_ring[pending].stop != VCA_STOP_RUNNING || h->ctrl_ring[pending].error) break;
        }
        pending = slot;
    }
    VCA_CUDA(cudaEventRecord(h->ev_b, h->stream));
    VCA_CUDA(cudaEventSynchronize(h->ev_b));
    float ms = 0.f;
    VCA_CUDA(cudaEventElapsedTime(&ms, h->ev_a, h->ev_b));
    h->total_ms += ms;
    return sync_ctrl(h);
}

vca_status run_steps(vca_ca* h, int max_new_steps, bool until_stop) {
    if (!h->seeded) {
        set_error("vca_ca: place_seeds or set_state must come before stepping");
        return VCA_ERR_STATE;
    }
    if (h->stop != VCA_STOP_RUNNING) return VCA_OK;
    const CaKernelArgs k = make_args(h);
    if (until_stop && !h->profile_kernels) return run_graphs(h, k);
    VCA_CUDA(cudaEventRecord(h->ev_a, h->stream));
    int chunk = 4;
    int done = 0;
    std::vector<cudaEvent_t> prof;  // profile mode: 4 events a step around drop, rules, cand
    size_t ev_used = 0;
    const int steps_before = h->steps;
    auto mark = [&]() -> cudaError_t {
        while (h->prof_events.size() < ev_used + 1) {
            cudaEvent_t e;
            const cudaError_t ce = cudaEventCreate(&e);
            if (ce != cudaSuccess) return ce;
            h->prof_events.push_back(e);
        }
        cudaEvent_t e = h->prof_events[ev_used++];
        prof.push_back(e);
        return cudaEventRecord(e, h->stream);
    };
    while (true) {
        const int n = until_stop ? chunk : std::min(chunk, max_new_steps - done);
        for (int s = 0; s < n; ++s) {
            if (h->profile_kernels) VCA_CUDA(mark());
            ca_drop_kernel<<<h->grid_blocks, kThreads, 0, h->stream>>>(k, 0);
            if (h->profile_kernels) VCA_CUDA(mark());
            launch_rules(h, k);
            if (h->profile_kernels) VCA_CUDA(mark());
            ca_cand_kernel<<<h->cand_blocks, kCandThreads, 0, h->stream>>>(k);
            if (h->profile_kernels) VCA_CUDA(mark());
        }
        VCA_CUDA(cudaGetLastError());
        h->launches += (uint64_t)n * 3;
        done += n;
        if (vca_status s = sync_ctrl(h)) return s;
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
        // Launches after the stop exit at once; only the ones that did a step count.
        const uint64_t real = std::min<uint64_t>(prof.size() / 4, (uint64_t)(h->steps - steps_before));
        for (size_t i = 0; i < real; ++i) {
            float m[3] = {0.f, 0.f, 0.f};
            for (int j = 0; j < 3; ++j) VCA_CUDA(cudaEventElapsedTime(&m[j], prof[4 * i + j], prof[4 * i + j + 1]));
            h->drop_ms += m[0];
            h->rules_ms += m[1];
            h->cand_ms += m[2];
            ++h->rules_launches;
        }
    }
    return VCA_OK;
}

void free_all(vca_ca* h) {
    if (h->device >= 0) cudaSetDevice(h->device);
    for (int b = 0; b < 2; ++b) {
        cudaFree(h->type[b]);
        cudaFree(h->flow[b]);   // temp[b] lies in the same allocation
        cudaFree(h->solid[b]);  // and arrival[b]
        cudaFree(h->tile_list[b]);
    }
    cudaFree(h->tile_flags);
    cudaFree(h->tile_mark[0]);
    cudaFree(h->tile_mark[1]);
    cudaFree(h->desc_plane);
    cudaFree(h->drop_plane);
    cudaFree(h->chg_list[0]);
    cudaFree(h->chg_list[1]);
    cudaFree(h->cand_list);
    cudaFree(h->spill);
    cudaFree(h->heights_dev);
    cudaFree(h->vents);
    cudaFree(h->seeds_dev);
    cudaFree(h->flow_sums);
    cudaFree(h->ctrl);
    cudaFree(h->hist_active);
    cudaFree(h->hist_changed);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->ev_a) cudaEventDestroy(h->ev_a);
    if (h->ev_b) cudaEventDestroy(h->ev_b);
    for (cudaEvent_t e : h->ring_ev)
        if (e) cudaEventDestroy(e);
    if (h->ctrl_ring) cudaFreeHost(h->ctrl_ring);
    drop_graph(h);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// All cells AIR (padding VOID), drop depths and D(n) -1, no tile scheduled: the state of a new handle.
vca_status clear_planes(vca_ca* h) {
    const auto& g = h->geom;
    const size_t n = h->plane_cells;
    for (int b = 0; b < 2; ++b) {
        VCA_CUDA(cudaMemsetAsync(h->type[b], 0, n, h->stream));
        VCA_CUDA(cudaMemsetAsync(h->flow[b], 0, n * 4, h->stream));
        VCA_CUDA(cudaMemsetAsync(h->temp[b], 0, n * 4, h->stream));
        VCA_CUDA(cudaMemsetAsync(h->solid[b], 0, n * 2, h->stream));
        VCA_CUDA(cudaMemsetAsync(h->arrival[b], 0, n * 2, h->stream));
    }
    VCA_CUDA(cudaMemsetAsync(h->drop_plane, 0xFF, n, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->desc_plane, 0xFF, n, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->tile_mark[0], 0, h->ntiles * 4, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->tile_mark[1], 0, h->ntiles * 4, h->stream));
    if (g.P > g.nx) {
        ca_pad_kernel<<<256, 256, 0, h->stream>>>(h->type[0], h->type[1], g.nx, g.P, (int64_t)g.ny * g.nz);
        VCA_CUDA(cudaGetLastError());
    }
    return VCA_OK;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                   const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// A pitched plane as a 3D tensor (P, ny, nz) of elem-byte cells with a box of (bx, by, bz) cells.
vca_status encode_plane(CUtensorMap* m, CUtensorMapDataType type, size_t elem, void* base, const CaGeom& g, uint32_t bx,
                        uint32_t by, uint32_t bz, const char* what) {
    const EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("vca_ca_create: cuTensorMapEncodeTiled is not available from the driver");
        return VCA_ERR_CUDA;
    }
    const cuuint64_t dims[3] = {(cuuint64_t)g.P, (cuuint64_t)g.ny, (cuuint64_t)g.nz};
    const cuuint64_t strides[2] = {(cuuint64_t)g.P * elem, (cuuint64_t)g.P * g.ny * elem};
    const cuuint32_t box[3] = {bx, by, bz};
    const cuuint32_t step[3] = {1, 1, 1};
    const CUresult r = fn(m, type, 3, base, dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error(std::string("vca_ca_create: cuTensorMapEncodeTiled failed for ") + what + " (CUresult " + std::to_string((int)r) + ")");
        return VCA_ERR_CUDA;
    }
    return VCA_OK;
}

// Two planes of one allocation as a 4D tensor (P, ny, nz, 2), the plane stride given in elements.
vca_status encode_pair(CUtensorMap* m, CUtensorMapDataType type, size_t elem, void* base, const CaGeom& g, size_t plane_stride,
                       uint32_t bx, uint32_t by, uint32_t bz, const char* what) {
    const EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("vca_ca_create: cuTensorMapEncodeTiled is not available from the driver");
        return VCA_ERR_CUDA;
    }
    const cuuint64_t dims[4] = {(cuuint64_t)g.P, (cuuint64_t)g.ny, (cuuint64_t)g.nz, 2};
    const cuuint64_t strides[3] = {(cuuint64_t)g.P * elem, (cuuint64_t)g.P * g.ny * elem, (cuuint64_t)plane_stride * elem};
    const cuuint32_t box[4] = {bx, by, bz, 2};
    const cuuint32_t step[4] = {1, 1, 1, 1};
    const CUresult r = fn(m, type, 4, base, dims, strides, box, step, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error(std::string("vca_ca_create: cuTensorMapEncodeTiled failed for ") + what + " (CUresult " + std::to_string((int)r) + ")");
        return VCA_ERR_CUDA;
    }
    return VCA_OK;
}

// Tensor maps of the rules pass (boxes of one 64 x TY x TZ tile, halo rows 96 bytes from x0 - 16).
vca_status encode_maps(vca_ca* h) {
    const CaGeom& g = h->geom;
    CaTensorMaps& m = h->tmaps;
    const uint32_t TY = (uint32_t)g.TY, TZ = (uint32_t)g.TZ;
    const uint32_t HY = g.ny > 1 ? TY + 2 : 1, HZ = g.nz > 1 ? TZ + 2 : 1;
    for (int b = 0; b < 2; ++b) {
        if (vca_status s = encode_plane(&m.own_type[b], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, h->type[b], g, kTileX, TY, TZ, "type")) return s;
        if (vca_status s = encode_plane(&m.halo_type[b], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, h->type[b], g, kTileX + 32, HY, HZ, "type halo"))
            return s;
        const size_t stride = h->cap.plane_cells;  // temp[b] - flow[b], arrival[b] - solid[b]
        if (vca_status s = encode_pair(&m.ft[b], CU_TENSOR_MAP_DATA_TYPE_INT32, 4, h->flow[b], g, stride, kTileX, TY, TZ,
                                       "flowId + temp"))
            return s;
        if (vca_status s = encode_pair(&m.sa[b], CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, h->solid[b], g, stride, kTileX, TY, TZ,
                                       "solidStep + arrivalStep"))
            return s;
    }
    for (int b = 0; b < 2; ++b)
        if (vca_status s = encode_plane(&m.xside_type[b], CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, h->type[b], g, 16, HY, HZ, "type column"))
            return s;
    if (vca_status s = encode_plane(&m.xside_drop, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, h->drop_plane, g, 16, HY, TZ, "drop column"))
        return s;
    return encode_plane(&m.drop, CU_TENSOR_MAP_DATA_TYPE_UINT8, 1, h->drop_plane, g, kTileX + 32, HY, TZ, "drop depth");
}

vca_status upload_vents(vca_ca* h, const vca_vent* vents, int count) {
    int slots = 1;
    for (int i = 0; i < count; ++i) slots = std::max(slots, vents[i].flow_id + 1);
    std::vector<int4> table((size_t)slots, make_int4(-1, -1, -1, 0));
    for (int i = 0; i < count; ++i)
        if (vents[i].flow_id > 0) table[(size_t)vents[i].flow_id] = make_int4(vents[i].x, vents[i].y, vents[i].z, 0);
    if ((size_t)slots > h->vent_cap) {  // grows only: a resident handle keeps its buffer
        cudaFree(h->vents);
        h->vents = nullptr;
        const size_t cap = std::max<size_t>((size_t)slots, 64);
        VCA_CUDA(cudaMalloc(&h->vents, sizeof(int4) * cap));
        h->vent_cap = cap;
    }
    VCA_CUDA(cudaMemcpyAsync(h->vents, table.data(), sizeof(int4) * table.size(), cudaMemcpyHostToDevice, h->stream));
    // bit 1 of the tile flags: the tiles that hold a vent (the only ones whose LAVA can be reheated)
    const auto& g = h->geom;
    std::vector<uint32_t> flags(h->ntiles, 0u);
    for (int i = 0; i < count; ++i) {
        const vca_vent& v = vents[i];
        if (v.x < 0 || v.x >= g.nx || v.y < 0 || v.y >= g.ny || v.z < 0 || v.z >= g.nz) continue;
        flags[(size_t)(v.x / kTileX) + (size_t)g.tiles_x * ((size_t)(v.y / g.TY) + (size_t)g.tiles_y * (size_t)(v.z / g.TZ))] = 2u;
    }
    VCA_CUDA(cudaMemcpyAsync(h->tile_flags, flags.data(), 4 * flags.size(), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->vent_slots = slots;
    return VCA_OK;
}

// Host planes (unpitched) <-> pitched device planes.
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

namespace vca {

vca_status validate_desc(const vca_ca_desc* d, const char* who) {
    const int nx = d->nx, ny = d->ny, nz = d->nz;
    auto bad = [&](const std::string& m) {
        set_error(std::string(who) + ": " + m);
        return VCA_ERR_ARG;
    };
    if (nx < 1 || ny < 1 || nz < 1 || (nx > 1) + (ny > 1) + (nz > 1) < 2)
        return bad("the space must be 2D (exactly one size equal to 1) or 3D");
    if ((uint64_t)nx * ny * nz > 2000000000ULL) return bad("more than 2 000 000 000 cells");
    if (d->mode == VCA_MODE_LAVA && (nx > 1) + (ny > 1) + (nz > 1) == 2 && ny != 1)
        return bad("a 2D lava space is the x-z cross-section (ny = 1)");
    if (d->max_steps < 0 || d->max_steps > 65535) return bad("max_steps must be in 0..65535");
    if (d->neighborhood < 0 || d->neighborhood > 3 || d->boundary < 0 || d->boundary > 1 || d->mode < 0 || d->mode > 1 ||
        d->sweep < 0 || d->sweep > 2)
        return bad("unknown neighborhood, boundary, mode or sweep");
    NbTable nb;
    if (!build_nb(d->neighborhood, nx, ny, nz, nb)) return bad("the hexagonal neighbourhood is defined in 2D only");
    if (d->tile_y != 0 || d->tile_z != 0) {
        const int ty = d->tile_y, tz = d->tile_z;
        const bool pow2 = ty > 0 && tz > 0 && (ty & (ty - 1)) == 0 && (tz & (tz - 1)) == 0;
        if (!pow2 || ty * tz != 16) return bad("tile_y x tile_z must be 16 cells (1 x 16, 2 x 8, 4 x 4, 8 x 2, 16 x 1)");
        if (ny == 1 && ty != 1) return bad("a 2D x-z section takes tiles with tile_y = 1");
        if (nz == 1 && tz != 1) return bad("a 2D x-y plane takes tiles with tile_z = 1");
    }
    if (d->rules_blocks_per_sm < 0) return bad("rules_blocks_per_sm must be >= 0");
    return VCA_OK;
}

// Pitched geometry and tile shape of a space (tiles 64 x TY x TZ, TY * TZ = 16).
CaGeom geometry_of(const vca_ca_desc* d) {
    CaGeom g{};
    g.nx = d->nx;
    g.ny = d->ny;
    g.nz = d->nz;
    g.P = (d->nx + kTileX - 1) / kTileX * kTileX;
    const bool periodic = d->boundary == VCA_BC_PERIODIC;
    g.per[0] = periodic && d->nx > 1;
    g.per[1] = periodic && d->ny > 1;
    g.per[2] = periodic && d->mode == VCA_MODE_CLASSIC && d->nz > 1;
    if (d->tile_y != 0 && d->tile_z != 0) {
        g.TY = d->tile_y;
        g.TZ = d->tile_z;
    } else if (d->ny > 1 && d->nz > 1) {
        g.TY = 4;
        g.TZ = 4;
    } else if (d->ny == 1) {
        g.TY = 1;
        g.TZ = 16;
    } else {
        g.TY = 16;
        g.TZ = 1;
    }
    {
        // the shared-memory family that holds this tile's staged rows (RulesShape)
        const int hy = d->ny > 1 ? g.TY + 2 : 1, hz = d->nz > 1 ? g.TZ + 2 : 1;
        const int halo = hy * hz, drop = hy * g.TZ;
        const int spill_ty = d->nz > 1 ? g.TY : 1;  // spill levels are staged only with a z axis
        g.shape = (halo <= ShapeA::halo && drop <= ShapeA::drop && spill_ty <= ShapeA::ty)   ? 0
                  : (halo <= ShapeB::halo && drop <= ShapeB::drop && spill_ty <= ShapeB::ty) ? 1
                                                                                              : 2;
    }
    g.tiles_x = g.P / kTileX;
    g.tiles_y = (d->ny + g.TY - 1) / g.TY;
    g.tiles_z = (d->nz + g.TZ - 1) / g.TZ;
    g.div_tx = make_fastdiv32((uint32_t)g.tiles_x);
    g.div_ty = make_fastdiv32((uint32_t)g.tiles_y);
    return g;
}

CaSizes sizes_of(const vca_ca_desc* d) {
    const CaGeom g = geometry_of(d);
    CaSizes z;
    z.plane_cells = (size_t)g.P * d->ny * d->nz;
    z.ntiles = (uint64_t)g.tiles_x * g.tiles_y * g.tiles_z;
    z.chg_cap = (uint32_t)std::min<uint64_t>((uint64_t)d->nx * d->ny * d->nz, 1u << 22);
    z.cols = (size_t)d->nx * d->ny;
    z.hist = std::max(1, d->max_steps);
    return z;
}

// Everything of a handle that depends on the space and the parameters: geometry, neighbourhood
// tables, TMA descriptors, grids, all cells AIR, no vents, step 0.  Allocates nothing.
vca_status configure(vca_ca* h, const vca_ca_desc* d) {
    h->desc = *d;
    h->geom = geometry_of(d);
    const CaGeom& g = h->geom;
    h->ntiles = (uint64_t)g.tiles_x * g.tiles_y * g.tiles_z;
    h->plane_cells = (size_t)g.P * g.ny * g.nz;
    h->chg_cap = h->cap.chg_cap;
    std::memset(&h->tables_host, 0, sizeof(h->tables_host));
    build_nb(d->neighborhood, d->nx, d->ny, d->nz, h->tables_host.nb);
    // side offsets: union of dz == 0 offsets over all variants (LavaCA.hpp:104-112)
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
    int per_sm = std::max(1, h->rules_per_sm[g.shape]);
    if (d->rules_blocks_per_sm > 0) per_sm = std::min(per_sm, d->rules_blocks_per_sm);
    h->grid_blocks = (int)std::min<uint64_t>(h->ntiles, (uint64_t)h->sms * per_sm);
    // one wave, and no more blocks than the grid could ever list candidates for (small grids share the GPU)
    h->cand_blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->sms * std::max(1, h->cand_per_sm),
                                                                  (h->ntiles * kTileCells + kCandThreads - 1) / kCandThreads));
    if (vca_status s = encode_maps(h)) return s;
    if (vca_status s = clear_planes(h)) return s;
    vca_vent none{0, 0, 0, 0};
    if (vca_status s = upload_vents(h, &none, 0)) return s;  // synchronizes the stream
    h->has_terrain = false;
    h->seeded = false;
    h->steps = 0;
    h->stop = VCA_STOP_RUNNING;
    return VCA_OK;
}

}  // namespace vca

extern "C" {

vca_status vca_ca_create(const vca_ca_desc* d, vca_ca** out) {
    if (d == nullptr || out == nullptr) {
        set_error("vca_ca_create: null argument");
        return VCA_ERR_ARG;
    }
    *out = nullptr;
    if (vca_status s = validate_desc(d, "vca_ca_create")) return s;
    const CaSizes need = sizes_of(d);
    vca_ca* h = new vca_ca();
    h->desc = *d;
    h->device = d->device;
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
    h->sms = prop.multiProcessorCount;
#define ALLOC(ptr, bytes)                                                         \
    do {                                                                          \
        e = cudaMalloc(&(ptr), (bytes));                                          \
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc " #ptr));      \
    } while (0)
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
    const size_t n = need.plane_cells;
    for (int b = 0; b < 2; ++b) {
        ALLOC(h->type[b], n);
        // flowId then temperature, solidStep then arrivalStep: one allocation each, so that one 4D
        // TMA box moves both planes of a pair (the plane stride is the capacity's plane size)
        ALLOC(h->flow[b], n * 8);
        h->temp[b] = reinterpret_cast<float*>(h->flow[b] + n);
        ALLOC(h->solid[b], n * 4);
        h->arrival[b] = h->solid[b] + n;
        ALLOC(h->tile_list[b], need.ntiles * 4);
    }
    ALLOC(h->tile_flags, need.ntiles * 4);
    ALLOC(h->tile_mark[0], need.ntiles * 4);
    ALLOC(h->tile_mark[1], need.ntiles * 4);
    ALLOC(h->desc_plane, n);
    ALLOC(h->drop_plane, n);
    ALLOC(h->chg_list[0], sizeof(uint32_t) * (size_t)need.chg_cap);
    ALLOC(h->chg_list[1], sizeof(uint32_t) * (size_t)need.chg_cap);
    ALLOC(h->cand_list, sizeof(uint32_t) * (size_t)need.ntiles * kTileCells);  // never overflows
    ALLOC(h->ctrl, sizeof(CaCtrl));
    ALLOC(h->hist_active, sizeof(unsigned long long) * (size_t)need.hist);
    ALLOC(h->hist_changed, sizeof(unsigned long long) * (size_t)need.hist);
    ALLOC(h->spill, sizeof(int32_t) * need.cols);
    ALLOC(h->heights_dev, sizeof(int32_t) * need.cols);
#undef ALLOC
    h->cap = need;
    if ((e = cudaHostAlloc(&h->ctrl_host, sizeof(CaCtrl), cudaHostAllocMapped)) != cudaSuccess ||
        (e = cudaHostGetDevicePointer(&h->ctrl_host_dev, h->ctrl_host, 0)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaHostAlloc (mapped)"));
    if ((e = rules_occupancy<ShapeA>(&h->rules_per_sm[0])) != cudaSuccess ||
        (e = rules_occupancy<ShapeB>(&h->rules_per_sm[1])) != cudaSuccess ||
        (e = rules_occupancy<ShapeC>(&h->rules_per_sm[2])) != cudaSuccess)
        return fail(cuda_fail(e, "rules-pass occupancy"));
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&h->cand_per_sm, ca_cand_kernel, kCandThreads, 0);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    if ((e = cudaEventCreate(&h->ev_a)) != cudaSuccess || (e = cudaEventCreate(&h->ev_b)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->ring_ev[0], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&h->ring_ev[1], cudaEventDisableTiming)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaEventCreate"));
    if ((e = cudaHostAlloc(&h->ctrl_ring, 2 * sizeof(CaCtrl), cudaHostAllocMapped)) != cudaSuccess ||
        (e = cudaHostGetDevicePointer(&h->ctrl_ring_dev, h->ctrl_ring, 0)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaHostAlloc (mapped)"));
    const char* prof = std::getenv("VCA_PROFILE_KERNELS");
    h->profile_kernels = prof != nullptr && prof[0] == '1';
    if (vca_status s = configure(h, d)) return fail(s);
    *out = h;
    return VCA_OK;
}

vca_status vca_ca_reconfigure(vca_ca* h, const vca_ca_desc* d) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_reconfigure")) return s;
    if (d == nullptr) {
        set_error("vca_ca_reconfigure: null desc");
        return VCA_ERR_ARG;
    }
    if (vca_status s = validate_desc(d, "vca_ca_reconfigure")) return s;
    if (d->device != h->device) {
        set_error("vca_ca_reconfigure: the handle lives on another device");
        return VCA_ERR_ARG;
    }
    const CaSizes need = sizes_of(d);
    if (need.plane_cells > h->cap.plane_cells || need.ntiles > h->cap.ntiles || need.chg_cap > h->cap.chg_cap ||
        need.cols > h->cap.cols || need.hist > h->cap.hist) {
        set_error("vca_ca_reconfigure: the grid does not fit the handle's device memory (vca_ca_footprint)");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    h->slab = false;
    return configure(h, d);
}

vca_status vca_ca_footprint(const vca_ca_desc* d, uint64_t* bytes) {
    if (d == nullptr || bytes == nullptr) {
        set_error("vca_ca_footprint: null argument");
        return VCA_ERR_ARG;
    }
    if (vca_status s = validate_desc(d, "vca_ca_footprint")) return s;
    const CaSizes z = sizes_of(d);
    *bytes = 2 * 13 * (uint64_t)z.plane_cells + 2 * (uint64_t)z.plane_cells  // state x 2, desc, drop
             + 4 * 5 * (uint64_t)z.ntiles                                     // tile lists, flags, marks
             + 4 * (uint64_t)z.ntiles * kTileCells                            // candidate list
             + 2 * 4 * (uint64_t)z.chg_cap + 2 * 8 * (uint64_t)z.hist + 2 * 4 * (uint64_t)z.cols + sizeof(CaCtrl);
    return VCA_OK;
}

vca_status vca_ca_reset(vca_ca* h) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_reset")) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = clear_planes(h)) return s;
    vca_vent none{0, 0, 0, 0};
    if (vca_status s = upload_vents(h, &none, 0)) return s;  // synchronizes the stream
    h->has_terrain = false;
    h->seeded = false;
    h->steps = 0;
    h->stop = VCA_STOP_RUNNING;
    return VCA_OK;
}

vca_status vca_ca_apply_terrain(vca_ca* h, const int32_t* heights) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_apply_terrain")) return s;
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
    std::vector<int32_t> spill = fill_depressions(hv, g.nx, g.ny, g.per[0] != 0, g.per[1] != 0);
    if (h->slab) {
        // heights and spill levels of the whole grid, seen from this slab's layer 0: every test
        // against them (z < h, z - 1 < spill, z <= spill) keeps its truth with both sides shifted
        for (auto& v : hv) v -= h->slab_z0;
        for (auto& v : spill) v -= h->slab_z0;
    }
    VCA_CUDA(cudaMemcpyAsync(h->heights_dev, hv.data(), sizeof(int32_t) * cols, cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->spill, spill.data(), sizeof(int32_t) * cols, cudaMemcpyHostToDevice, h->stream));
    const int cur = h->steps & 1;
    ca_terrain_kernel<<<1184, 256, 0, h->stream>>>(h->type[cur], h->heights_dev, g.nx, g.ny, g.nz, g.P);
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->has_terrain = true;
    h->launches += 1;
    return VCA_OK;
}

vca_status vca_ca_place_seeds(vca_ca* h, const vca_vent* vents, int count) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_place_seeds")) return s;
    if (count < 0 || (count > 0 && vents == nullptr)) {
        set_error("vca_ca_place_seeds: bad vent list");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const auto& g = h->geom;
    const int cur = h->steps & 1;
    const float temp = h->desc.mode == VCA_MODE_LAVA ? h->desc.erupt_temp : 0.0f;
    std::vector<int4> seeds((size_t)count);
    for (int i = 0; i < count; ++i) {
        const vca_vent& v = vents[i];
        if (v.x < 0 || v.x >= g.nx || v.y < 0 || v.y >= g.ny || v.z < 0 || v.z >= g.nz) {
            set_error("vca_ca_place_seeds: vent " + std::to_string(i) + " lies outside the grid");
            return VCA_ERR_ARG;
        }
        seeds[(size_t)i] = make_int4(v.x, v.y, v.z, v.flow_id);
    }
    if (count > 0) {
        // A repeated cell keeps its last entry, as the reference's sequential writes do; the
        // remaining cells are distinct, so the scatter below is order-free.
        std::vector<std::pair<uint64_t, int>> keyed((size_t)count);
        for (int i = 0; i < count; ++i) {
            const int4& s = seeds[(size_t)i];
            keyed[(size_t)i] = {(uint64_t)s.x + (uint64_t)g.nx * ((uint64_t)s.y + (uint64_t)g.ny * s.z), i};
        }
        std::sort(keyed.begin(), keyed.end());
        std::vector<int4> uniq;
        uniq.reserve((size_t)count);
        for (size_t i = 0; i < keyed.size(); ++i)
            if (i + 1 == keyed.size() || keyed[i + 1].first != keyed[i].first) uniq.push_back(seeds[(size_t)keyed[i].second]);
        const int nu = (int)uniq.size();
        // a grow-only buffer: a cudaFree per call would wait for every stream of the device
        if ((size_t)nu > h->seed_cap) {
            VCA_CUDA(cudaStreamSynchronize(h->stream));
            cudaFree(h->seeds_dev);
            h->seeds_dev = nullptr;
            h->seed_cap = 0;
            const size_t cap = std::max<size_t>((size_t)nu, 1024);
            VCA_CUDA(cudaMalloc(&h->seeds_dev, sizeof(int4) * cap));
            h->seed_cap = cap;
        }
        VCA_CUDA(cudaMemcpyAsync(h->seeds_dev, uniq.data(), sizeof(int4) * (size_t)nu, cudaMemcpyHostToDevice,
                                 h->stream));
        ca_seed_kernel<<<std::min(1184, (nu + 255) / 256), 256, 0, h->stream>>>(make_args(h), h->seeds_dev, nu, cur,
                                                                                 temp);
        VCA_CUDA(cudaGetLastError());
        VCA_CUDA(cudaStreamSynchronize(h->stream));
        h->launches += 1;
    }
    if (vca_status s = upload_vents(h, vents, count)) return s;
    h->seeded = true;
    return init_state(h, h->steps);
}

vca_status vca_ca_set_state(vca_ca* h, const uint8_t* type, const int32_t* flow_id, const float* temp,
                            const uint16_t* solid_step, const uint16_t* arrival_step, const int32_t* spill,
                            const vca_vent* vents, int vent_count, int steps_done) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_set_state")) return s;
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
    if (vca_status s = not_in_batch(h, "vca_ca_step")) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = run_steps(h, 1, false)) return s;
    if (running) *running = h->stop == VCA_STOP_RUNNING;
    return VCA_OK;
}

vca_status vca_ca_run(vca_ca* h) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_run")) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    return run_steps(h, 0, true);
}

vca_status vca_ca_get_info(vca_ca* h, vca_ca_info* out) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_get_info")) return s;
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
    out->kernel_launches = h->launches;
    return VCA_OK;
}

vca_status vca_ca_history(vca_ca* h, uint64_t* active, uint64_t* changed, int capacity, int* count) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_history")) return s;
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
    if (vca_status s = not_in_batch(h, "vca_ca_download")) return s;
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
    if (vca_status s = not_in_batch(h, "vca_ca_get_spill")) return s;
    if (!h->has_terrain) {
        set_error("vca_ca_get_spill: no terrain");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemcpy(spill, h->spill, sizeof(int32_t) * (size_t)h->geom.nx * h->geom.ny, cudaMemcpyDeviceToHost));
    return VCA_OK;
}

vca_status vca_ca_flow_stats(vca_ca* h, int flows, uint64_t* lava, uint64_t* basalt, uint64_t* reach2) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_flow_stats")) return s;
    if (flows < 0 || (flows > 0 && (lava == nullptr || basalt == nullptr || reach2 == nullptr))) {
        set_error("vca_ca_flow_stats: bad flow count or null array");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    const size_t m = (size_t)flows + 1;
    if (3 * m > h->flow_sums_cap) {  // grows only
        VCA_CUDA(cudaStreamSynchronize(h->stream));
        cudaFree(h->flow_sums);
        h->flow_sums = nullptr;
        h->flow_sums_cap = 0;
        VCA_CUDA(cudaMalloc(&h->flow_sums, sizeof(unsigned long long) * 3 * m));
        h->flow_sums_cap = 3 * m;
    }
    VCA_CUDA(cudaMemsetAsync(h->flow_sums, 0, sizeof(unsigned long long) * 3 * m, h->stream));
    const int cur = h->steps & 1;
    const auto& g = h->geom;
    const size_t smem = flows <= kFlowPrivMax ? sizeof(unsigned long long) * 3 * m : 0;
    const uint64_t cells = (uint64_t)g.nx * g.ny * g.nz;
    const int blocks = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)h->sms * 8, (cells + 255) / 256));
    ca_flow_stats_kernel<<<blocks, 256, smem, h->stream>>>(h->type[cur], h->flow[cur], g, h->vents, h->vent_slots, flows,
                                                            h->flow_sums);
    VCA_CUDA(cudaGetLastError());
    h->launches += 1;
    std::vector<unsigned long long> host(3 * m);
    VCA_CUDA(cudaMemcpyAsync(host.data(), h->flow_sums, sizeof(unsigned long long) * 3 * m, cudaMemcpyDeviceToHost,
                             h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    for (size_t f = 0; f < m; ++f) {
        lava[f] = f ? host[f] : 0;
        basalt[f] = f ? host[m + f] : 0;
        reach2[f] = f ? host[2 * m + f] : 0;
    }
    return VCA_OK;
}

vca_status vca_ca_set_slab(vca_ca* h, int z_offset, int own_z0, int own_z1) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_set_slab")) return s;
    const auto& g = h->geom;
    if (h->desc.mode != VCA_MODE_LAVA || g.nz < 2 || z_offset < 0 || own_z0 < 0 || own_z1 > g.nz || own_z0 >= own_z1) {
        set_error("vca_ca_set_slab: a slab is a lava grid with nz > 1, z_offset >= 0 and 0 <= own_z0 < own_z1 <= nz");
        return VCA_ERR_ARG;
    }
    if (h->seeded || h->has_terrain) {
        set_error("vca_ca_set_slab: set the slab before the terrain and the seeds");
        return VCA_ERR_STATE;
    }
    h->slab = true;
    h->slab_z0 = z_offset;
    h->own_z0 = own_z0;
    h->own_z1 = own_z1;
    h->desc.sweep = VCA_SWEEP_DENSE;  // halo copies change cells outside the tile scheduler's view
    return VCA_OK;
}

vca_status vca_ca_slab_step(vca_ca* h, uint64_t* active, uint64_t* changed) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_slab_step")) return s;
    if (!h->slab) {
        set_error("vca_ca_slab_step: the handle is not a slab (vca_ca_set_slab)");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const int before = h->steps;
    if (vca_status s = run_steps(h, 1, false)) return s;
    unsigned long long a = 0, c = 0;
    if (h->steps > before) {
        VCA_CUDA(cudaMemcpyAsync(&a, h->hist_active + before, 8, cudaMemcpyDeviceToHost, h->stream));
        VCA_CUDA(cudaMemcpyAsync(&c, h->hist_changed + before, 8, cudaMemcpyDeviceToHost, h->stream));
        VCA_CUDA(cudaStreamSynchronize(h->stream));
    }
    if (active) *active = a;
    if (changed) *changed = c;
    return VCA_OK;
}

vca_status vca_ca_slab_stop(vca_ca* h, int stop_reason) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_slab_stop")) return s;
    if (!h->slab || stop_reason < VCA_STOP_RUNNING || stop_reason > VCA_STOP_MAX_STEPS) {
        set_error("vca_ca_slab_stop: a slab handle and a VCA_STOP_* value");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const int32_t v = stop_reason;
    VCA_CUDA(cudaMemcpyAsync(&h->ctrl->stop, &v, sizeof(v), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->stop = stop_reason;
    return VCA_OK;
}

vca_status vca_ca_layers(vca_ca* h, void** type, void** flow_id, void** temp, void** solid_step, void** arrival_step,
                         uint64_t* layer_cells) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_ca_layers")) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    const int cur = h->steps & 1;
    if (type) *type = h->type[cur];
    if (flow_id) *flow_id = h->flow[cur];
    if (temp) *temp = h->temp[cur];
    if (solid_step) *solid_step = h->solid[cur];
    if (arrival_step) *arrival_step = h->arrival[cur];
    if (layer_cells) *layer_cells = (uint64_t)h->geom.P * h->geom.ny;
    return VCA_OK;
}

// Halo message of a slab: `types` type layers from local layer z0, then the flowId, temperature,
// solidStep and arrivalStep of local layer `full` (full < 0: none).  Layers are whole pitched
// layers (their padding cells are VOID on every slab alike).
static vca_status layers_check(vca_ca* h, int z0, int types, int full, const void* buf, const char* who) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, who)) return s;
    if (buf == nullptr || types < 0 || z0 < 0 || z0 + types > h->geom.nz || full >= h->geom.nz) {
        set_error(std::string(who) + ": layers outside the grid or null buffer");
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

static vca_status copy_layers(vca_ca* h, int z0, int types, int full, void* buf, bool to_buf) {
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s = sync_ctrl(h)) return s;
    const int cur = h->steps & 1;
    const size_t L = (size_t)h->geom.P * h->geom.ny;
    char* b = static_cast<char*>(buf);
    auto move = [&](void* plane, size_t elem, int z, int n, size_t at) -> cudaError_t {
        char* dev = static_cast<char*>(plane) + (size_t)z * L * elem;
        return to_buf ? cudaMemcpyAsync(b + at, dev, (size_t)n * L * elem, cudaMemcpyDefault, h->stream)
                      : cudaMemcpyAsync(dev, b + at, (size_t)n * L * elem, cudaMemcpyDefault, h->stream);
    };
    size_t at = 0;
    if (types > 0) VCA_CUDA(move(h->type[cur], 1, z0, types, at));
    at += (size_t)types * L;
    if (full >= 0) {
        VCA_CUDA(move(h->flow[cur], 4, full, 1, at));
        VCA_CUDA(move(h->temp[cur], 4, full, 1, at + 4 * L));
        VCA_CUDA(move(h->solid[cur], 2, full, 1, at + 8 * L));
        VCA_CUDA(move(h->arrival[cur], 2, full, 1, at + 10 * L));
    }
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_ca_pack_layers(vca_ca* h, int z0, int types, int full, void* buf) {
    if (vca_status s = layers_check(h, z0, types, full, buf, "vca_ca_pack_layers")) return s;
    return copy_layers(h, z0, types, full, buf, true);
}

vca_status vca_ca_unpack_layers(vca_ca* h, int z0, int types, int full, const void* buf) {
    if (vca_status s = layers_check(h, z0, types, full, buf, "vca_ca_unpack_layers")) return s;
    return copy_layers(h, z0, types, full, const_cast<void*>(buf), false);
}

vca_status vca_ca_kernel_times(vca_ca* h, double* drop_ms, double* rules_ms, double* cand_ms, uint64_t* steps) {
    if (vca_status s = check(h)) return s;
    const double n = h->rules_launches ? (double)h->rules_launches : 1.0;
    if (drop_ms) *drop_ms = h->drop_ms / n;
    if (rules_ms) *rules_ms = h->rules_ms / n;
    if (cand_ms) *cand_ms = h->cand_ms / n;
    if (steps) *steps = h->rules_launches;
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
    if (h->batch) vca_ca_batch_remove(h->batch, h);
    free_all(h);
    delete h;
}

}  // extern "C"

// Accessor used by the MC half (mc.cu) to build the crystallisation domain on the device.
namespace vca {
vca_status ca_view(vca_ca* h, CaView* v) {
    if (vca_status s = check(h)) return s;
    if (vca_status s = not_in_batch(h, "vca_mc_set_domain_from_ca / vca_mc_set_mobility_from_ca")) return s;
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

// ============================================================================================
// Batched stepping (vca_ca_batch_*): many member grids stepped by shared launches.
// ============================================================================================
struct vca_ca_batch {
    int device = 0;
    int cap = 0;                  // member slots
    int rules_grid = 0, cand_grid = 0;
    cudaStream_t stream = nullptr;
    // device tables
    CaTensorMaps* d_tm = nullptr;
    CaKernelArgs* d_args = nullptr;
    int2* d_rules_map = nullptr;
    int2* d_cand_map = nullptr;
    int* d_rules_n = nullptr;
    int* d_cand_n = nullptr;
    int4* d_status = nullptr;
    int4* h_status = nullptr;     // pinned, two ring slots of cap entries: (stop, error, steps, next tiles)
    std::vector<uint64_t> weight; // per slot: tiles of the member's next step (its share of the blocks)
    cudaEvent_t status_ev[2] = {nullptr, nullptr};
    cudaEvent_t sync_ev = nullptr;
    cudaGraphExec_t graph = nullptr;
    std::vector<vca_ca*> slots;   // member of each slot (nullptr: free)
    std::vector<vca_ca*> snap[2]; // the slots when the graph of a ring slot was launched
    std::vector<vca_ca*> early;   // members that had stopped before they were added
    std::vector<vca_ca*> done;    // stopped members not yet handed out
    bool dirty = true;            // tables on the device are out of date
    int pending = -1;             // ring slot whose status is not read yet
    int ring = 0;
    uint64_t graphs = 0, launches = 0;
};

namespace {

vca_status batch_check(vca_ca_batch* b) {
    if (b == nullptr) {
        set_error("null vca_ca_batch");
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

// Blocks of a launch of `grid` blocks shared among the members by weight (at least one each).
void split_blocks(const std::vector<uint64_t>& w, int grid, std::vector<int>& n) {
    const size_t m = w.size();
    n.assign(m, 1);
    if (m == 0) return;
    uint64_t total = 0;
    for (uint64_t v : w) total += v;
    int used = 0;
    for (size_t i = 0; i < m; ++i) {
        n[i] = std::max<int>(1, (int)((double)grid * (double)w[i] / (double)std::max<uint64_t>(1, total)));
        used += n[i];
    }
    while (used > grid) {  // take back from the largest shares
        size_t big = 0;
        for (size_t i = 1; i < m; ++i)
            if (n[i] > n[big]) big = i;
        if (n[big] <= 1) break;
        --n[big];
        --used;
    }
    while (used < grid) {  // the rest to the heaviest members, round robin by weight order
        size_t best = 0;
        double best_r = -1.0;
        for (size_t i = 0; i < m; ++i) {
            const double r = (double)w[i] / (double)n[i];
            if (r > best_r) {
                best_r = r;
                best = i;
            }
        }
        ++n[best];
        ++used;
    }
}

// Member arguments and block maps to the device (on the batch stream, ordered after the graphs
// already launched and before the next).
vca_status batch_upload(vca_ca_batch* b) {
    std::vector<CaTensorMaps> tm((size_t)b->cap);
    std::vector<CaKernelArgs> args((size_t)b->cap);
    std::vector<int> rn((size_t)b->cap, 0), cn((size_t)b->cap, 0);
    std::vector<int2> rmap((size_t)b->rules_grid, make_int2(-1, 0)), cmap((size_t)b->cand_grid, make_int2(-1, 0));
    std::vector<int> members;
    std::vector<uint64_t> w;
    for (int i = 0; i < b->cap; ++i) {
        vca_ca* h = b->slots[(size_t)i];
        std::memset(&args[(size_t)i], 0, sizeof(CaKernelArgs));
        if (!h) continue;
        tm[(size_t)i] = h->tmaps;
        args[(size_t)i] = make_args(h, true);
        members.push_back(i);
        w.push_back(std::max<uint64_t>(1, b->weight[(size_t)i]));
    }
    std::vector<int> nr, nc;
    split_blocks(w, b->rules_grid, nr);
    split_blocks(w, b->cand_grid, nc);
    int at_r = 0, at_c = 0;
    for (size_t j = 0; j < members.size(); ++j) {
        const int slot = members[j];
        rn[(size_t)slot] = nr[j];
        cn[(size_t)slot] = nc[j];
        for (int q = 0; q < nr[j]; ++q) rmap[(size_t)(at_r + q)] = make_int2(slot, q);
        for (int q = 0; q < nc[j]; ++q) cmap[(size_t)(at_c + q)] = make_int2(slot, q);
        at_r += nr[j];
        at_c += nc[j];
    }
    // pageable sources: each copy is staged before the call returns, so the vectors may go
    VCA_CUDA(cudaMemcpyAsync(b->d_tm, tm.data(), sizeof(CaTensorMaps) * tm.size(), cudaMemcpyHostToDevice, b->stream));
    VCA_CUDA(cudaMemcpyAsync(b->d_args, args.data(), sizeof(CaKernelArgs) * args.size(), cudaMemcpyHostToDevice, b->stream));
    VCA_CUDA(cudaMemcpyAsync(b->d_rules_n, rn.data(), sizeof(int) * rn.size(), cudaMemcpyHostToDevice, b->stream));
    VCA_CUDA(cudaMemcpyAsync(b->d_cand_n, cn.data(), sizeof(int) * cn.size(), cudaMemcpyHostToDevice, b->stream));
    VCA_CUDA(cudaMemcpyAsync(b->d_rules_map, rmap.data(), sizeof(int2) * rmap.size(), cudaMemcpyHostToDevice, b->stream));
    VCA_CUDA(cudaMemcpyAsync(b->d_cand_map, cmap.data(), sizeof(int2) * cmap.size(), cudaMemcpyHostToDevice, b->stream));
    b->dirty = false;
    return VCA_OK;
}

// A member leaves: its slot is freed and its own stream waits for everything the batch launched so
// far, so the member's next calls see its final state.
vca_status batch_detach(vca_ca_batch* b, vca_ca* h, const int4* st) {
    b->slots[(size_t)h->batch_slot] = nullptr;
    b->dirty = true;
    VCA_CUDA(cudaEventRecord(b->sync_ev, b->stream));
    VCA_CUDA(cudaStreamWaitEvent(h->stream, b->sync_ev, 0));
    if (st) {
        h->steps = st->z;
        h->stop = st->x;
    }
    h->batch = nullptr;
    h->batch_slot = -1;
    return VCA_OK;
}

// Reads the status of the graph in ring slot r (waits for it) and takes the members that stopped
// out of the batch.
vca_status batch_collect(vca_ca_batch* b, int r) {
    VCA_CUDA(cudaEventSynchronize(b->status_ev[r]));
    const int4* st = b->h_status + (size_t)r * b->cap;
    for (int i = 0; i < b->cap; ++i) {
        vca_ca* h = b->snap[r][(size_t)i];
        if (!h || b->slots[(size_t)i] != h || st[i].x < 0) continue;
        if (st[i].x != VCA_STOP_RUNNING || st[i].y != 0) {
            if (vca_status s = batch_detach(b, h, &st[i])) return s;
            b->done.push_back(h);
            continue;
        }
        // the blocks follow the work: re-split when a member's visited tiles moved by more than 1/8
        const uint64_t now = std::max<uint64_t>(1, (uint64_t)std::max(0, st[i].w));
        uint64_t& was = b->weight[(size_t)i];
        if (now > was + was / 8 || now + now / 8 < was) {
            was = now;
            b->dirty = true;
        }
    }
    return VCA_OK;
}

vca_status batch_capture(vca_ca_batch* b) {
    CaBatchView v{b->d_tm, b->d_args, b->d_rules_map, b->d_cand_map, b->d_rules_n, b->d_cand_n, b->d_status, b->cap};
    VCA_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    for (int s = 0; s < kGraphSteps; ++s) {
        ca_drop_batch_kernel<<<b->rules_grid, kThreads, 0, b->stream>>>(v);
        ca_rules_batch_kernel<<<b->rules_grid, kThreads, kRulesDynSmem, b->stream>>>(v);
        ca_cand_batch_kernel<<<b->cand_grid, kCandThreads, 0, b->stream>>>(v);
    }
    ca_batch_status_kernel<<<1, 256, 0, b->stream>>>(v);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) {
        b->graph = nullptr;
        return cuda_fail(e2, "cudaGraphInstantiate");
    }
    return VCA_OK;
}

void batch_free(vca_ca_batch* b) {
    cudaSetDevice(b->device);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_tm);
    cudaFree(b->d_args);
    cudaFree(b->d_rules_map);
    cudaFree(b->d_cand_map);
    cudaFree(b->d_rules_n);
    cudaFree(b->d_cand_n);
    cudaFree(b->d_status);
    if (b->h_status) cudaFreeHost(b->h_status);
    for (cudaEvent_t e : b->status_ev)
        if (e) cudaEventDestroy(e);
    if (b->sync_ev) cudaEventDestroy(b->sync_ev);
    if (b->stream) cudaStreamDestroy(b->stream);
}

}  // namespace

extern "C" {

vca_status vca_ca_batch_create(int device, int max_members, vca_ca_batch** out) {
    if (out == nullptr || max_members < 1) {
        set_error("vca_ca_batch_create: null output or max_members < 1");
        return VCA_ERR_ARG;
    }
    *out = nullptr;
    vca_ca_batch* b = new vca_ca_batch();
    b->device = device;
    auto fail = [&](vca_status s) {
        batch_free(b);
        delete b;
        return s;
    };
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, device)) != cudaSuccess) return fail(cuda_fail(e, "cudaGetDeviceProperties"));
    if (prop.major < 10) {
        set_error("vca_ca_batch_create: needs an sm_100 (Blackwell) device");
        return fail(VCA_ERR_CUDA);
    }
    int rules_per_sm = 0, cand_per_sm = 0;
    if ((e = cudaFuncSetAttribute(ca_rules_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRulesDynSmem)) !=
        cudaSuccess)
        return fail(cuda_fail(e, "cudaFuncSetAttribute"));
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rules_per_sm, ca_rules_batch_kernel, kThreads, kRulesDynSmem)) !=
        cudaSuccess)
        return fail(cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cand_per_sm, ca_cand_batch_kernel, kCandThreads, 0)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor"));
    b->rules_grid = prop.multiProcessorCount * std::max(1, rules_per_sm);
    b->cand_grid = prop.multiProcessorCount * std::max(1, cand_per_sm);
    b->cap = std::min(max_members, std::min(b->rules_grid, b->cand_grid));
    b->slots.assign((size_t)b->cap, nullptr);
    b->weight.assign((size_t)b->cap, 1);
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaStreamCreate"));
#define BALLOC(ptr, bytes)                                                    \
    do {                                                                      \
        e = cudaMalloc(&(ptr), (bytes));                                      \
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMalloc " #ptr));  \
    } while (0)
    BALLOC(b->d_tm, sizeof(CaTensorMaps) * (size_t)b->cap);
    BALLOC(b->d_args, sizeof(CaKernelArgs) * (size_t)b->cap);
    BALLOC(b->d_rules_map, sizeof(int2) * (size_t)b->rules_grid);
    BALLOC(b->d_cand_map, sizeof(int2) * (size_t)b->cand_grid);
    BALLOC(b->d_rules_n, sizeof(int) * (size_t)b->cap);
    BALLOC(b->d_cand_n, sizeof(int) * (size_t)b->cap);
    BALLOC(b->d_status, sizeof(int4) * (size_t)b->cap);
#undef BALLOC
    if ((e = cudaMallocHost(&b->h_status, sizeof(int4) * 2 * (size_t)b->cap)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaMallocHost"));
    if ((e = cudaEventCreateWithFlags(&b->status_ev[0], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->status_ev[1], cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->sync_ev, cudaEventDisableTiming)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaEventCreate"));
    if (vca_status s = batch_upload(b)) return fail(s);
    if (vca_status s = batch_capture(b)) return fail(s);
    *out = b;
    return VCA_OK;
}

vca_status vca_ca_batch_add(vca_ca_batch* b, vca_ca* h) {
    if (vca_status s = batch_check(b)) return s;
    if (vca_status s = check(h)) return s;
    if (h->batch != nullptr) {
        set_error("vca_ca_batch_add: the handle is already in a batch");
        return VCA_ERR_ARG;
    }
    if (h->device != b->device) {
        set_error("vca_ca_batch_add: the handle lives on another device");
        return VCA_ERR_ARG;
    }
    if (!h->seeded) {
        set_error("vca_ca_batch_add: place_seeds or set_state must come before stepping");
        return VCA_ERR_STATE;
    }
    if (h->geom.shape != 0) {
        set_error("vca_ca_batch_add: batched launches take the tile shapes of 4 x 4 or smaller halos "
                  "(4 x 4 in 3D, the 2D tiles); this handle uses " + std::to_string(h->geom.TY) + " x " +
                  std::to_string(h->geom.TZ));
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(b->device));
    if (h->stop != VCA_STOP_RUNNING) {  // nothing to step: reported by the next advance
        h->batch = b;
        b->early.push_back(h);
        return VCA_OK;
    }
    int slot = -1;
    for (int i = 0; i < b->cap && slot < 0; ++i)
        if (!b->slots[(size_t)i]) slot = i;
    if (slot < 0) {
        set_error("vca_ca_batch_add: the batch is full (" + std::to_string(b->cap) + " members)");
        return VCA_ERR_ARG;
    }
    // the batch's next launches come after the member's set-up work
    VCA_CUDA(cudaEventRecord(b->sync_ev, h->stream));
    VCA_CUDA(cudaStreamWaitEvent(b->stream, b->sync_ev, 0));
    b->slots[(size_t)slot] = h;
    b->weight[(size_t)slot] = std::max<uint64_t>(1, h->ntiles);  // until its first status
    h->batch = b;
    h->batch_slot = slot;
    b->dirty = true;
    return VCA_OK;
}

vca_status vca_ca_batch_advance(vca_ca_batch* b, int max_graphs, vca_ca** finished, int capacity, int* count,
                                int* running) {
    if (vca_status s = batch_check(b)) return s;
    if (capacity < 0 || (capacity > 0 && finished == nullptr)) {
        set_error("vca_ca_batch_advance: bad output list");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(b->device));
    for (vca_ca* h : b->early) {
        h->batch = nullptr;
        b->done.push_back(h);
    }
    b->early.clear();
    auto members = [&]() {
        int n = 0;
        for (vca_ca* h : b->slots) n += h != nullptr;
        return n;
    };
    for (int g = 0; g < max_graphs && b->done.empty(); ++g) {
        if (members() == 0) break;
        if (b->dirty)
            if (vca_status s = batch_upload(b)) return s;
        const int r = b->ring;
        VCA_CUDA(cudaGraphLaunch(b->graph, b->stream));
        VCA_CUDA(cudaMemcpyAsync(b->h_status + (size_t)r * b->cap, b->d_status, sizeof(int4) * (size_t)b->cap,
                                 cudaMemcpyDeviceToHost, b->stream));
        VCA_CUDA(cudaEventRecord(b->status_ev[r], b->stream));
        b->snap[r] = b->slots;
        b->graphs += 1;
        b->launches += 3 * kGraphSteps + 1;
        b->ring ^= 1;
        if (b->pending >= 0) {
            if (vca_status s = batch_collect(b, b->pending)) return s;
        }
        b->pending = r;
    }
    // with nothing left to launch, the last graph's status is read now
    if (b->done.empty() && b->pending >= 0) {
        if (vca_status s = batch_collect(b, b->pending)) return s;
        b->pending = -1;
    }
    int n = 0;
    while (n < capacity && !b->done.empty()) {
        finished[n++] = b->done.front();
        b->done.erase(b->done.begin());
    }
    if (count) *count = n;
    if (running) *running = members();
    return VCA_OK;
}

vca_status vca_ca_batch_remove(vca_ca_batch* b, vca_ca* h) {
    if (vca_status s = batch_check(b)) return s;
    if (vca_status s = check(h)) return s;
    if (h->batch != b) {
        set_error("vca_ca_batch_remove: the handle is not in this batch");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(b->device));
    for (size_t i = 0; i < b->early.size(); ++i)
        if (b->early[i] == h) {
            b->early.erase(b->early.begin() + (long)i);
            h->batch = nullptr;
            return VCA_OK;
        }
    if (vca_status s = batch_detach(b, h, nullptr)) return s;
    return sync_ctrl(h);  // steps and stop of the member as it left
}

vca_status vca_ca_batch_info(vca_ca_batch* b, uint64_t* graphs, uint64_t* launches, int* members) {
    if (vca_status s = batch_check(b)) return s;
    if (graphs) *graphs = b->graphs;
    if (launches) *launches = b->launches;
    if (members) {
        int n = 0;
        for (vca_ca* h : b->slots) n += h != nullptr;
        *members = n;
    }
    return VCA_OK;
}

void vca_ca_batch_destroy(vca_ca_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    std::vector<vca_ca*> left;
    for (vca_ca* h : b->slots)
        if (h) {
            batch_detach(b, h, nullptr);
            left.push_back(h);
        }
    for (vca_ca* h : b->early) h->batch = nullptr;
    for (vca_ca* h : b->done) h->batch = nullptr;
    cudaStreamSynchronize(b->stream);
    for (vca_ca* h : left) sync_ctrl(h);  // steps and stop of each member as it left
    batch_free(b);
    delete b;
}

}  // extern "C"

// mc.cu -- Potts Monte Carlo crystallisation with the checkerboard update on sm_100a, and the
// vca_mc_* half of the C ABI.
//
// One MCS (PottsMC::sweep -> sweepColors, engine/src/mc/PottsMC.cpp:451-533) is one launch per
// colour.  The domain cells of a colour are a compact list of global indices (built once, in
// globalIndex order, by a device stream compaction), so a colour pass touches only domain cells:
// per trial it reads the list entry, the cell's mobility and spin, and its neighbours' spins
// (shared with the neighbouring trials through L1/L2), and writes the spin when accepted.
// Cells of one colour are never neighbours in any variant (PottsMC.cpp:160-165), so the trials
// of a colour are independent and the order inside the pass does not matter.
//
// Acceptance is decided in integers: the reference accepts an uphill move when
// toUniform(r) < exp(-dE/kT), i.e. (r >> 11) * 2^-53 < p.  Scaling by 2^53 is exact, so this is
// (r >> 11) < ceil(p * 2^53); the thresholds are built on the host with the host's exp(), once
// per (unlikeBefore, unlikeAfter) pair, and the device compares 64-bit integers.
#include <cuda_runtime.h>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "vca.h"
#include "vca_device.cuh"
#include "vca_internal.h"

namespace vca {

constexpr int kMcThreads = 256;
constexpr int kTableSide = 27;  // unlike counts 0..26

// Exact 32-bit division by a runtime divisor (n < 2^32): q = (c * n) >> 64 with c = ceil(2^64 / d).
struct FastDiv {
    uint32_t d;
    uint64_t c;
};
inline FastDiv make_fastdiv(uint32_t d) { return FastDiv{d, d <= 1 ? 0 : ~0ULL / d + 1}; }
__device__ __forceinline__ uint32_t fdiv(uint32_t n, FastDiv f) { return f.d <= 1 ? n : (uint32_t)__umul64hi(f.c, (uint64_t)n); }

struct McCtrl {
    uint32_t sweeps;
    uint32_t ticket;
    unsigned long long attempts;
    unsigned long long accepted;
    unsigned long long uphill;
    unsigned long long energy_acc;
    unsigned long long sweep_accepted;  // accepted in the running sweep
    unsigned long long bar_arrived;     // grid barrier of the fused sweep kernel: arrivals so far
                                        // (zeroed before each launch)
    int error;                          // bit 0: a bounded barrier wait ran out
    int pad;
};

struct McArgs {
    int nx, ny, nz;
    int per[3];
    FastDiv div_nx, div_ny;
    int parity_colors;
    int classes[3];
    uint64_t seed;
    FastMod q_mod;       // % Q (initial orientation)
    FastMod qm1_mod;     // % (Q - 1) (proposal)
    FastMod var_mod;     // % variants
    int variants;
    int32_t* spin;
    const uint32_t* list;
    const float* list_mob;
    const unsigned long long* table;  // 27 x 27 acceptance thresholds
    const NbTable* nb;
    McCtrl* ctrl;
    // z slab of a taller grid (vca_mc_set_slab): hashRand takes local index + gidx_base, colours
    // the global z = local z + zoff
    uint64_t gidx_base;
    int zoff;
};

__device__ __forceinline__ bool mc_wrap(int& v, int n, int periodic) {
    if (v >= 0 && v < n) return true;
    if (!periodic || n == 1) return false;
    v = v < 0 ? v + n : v - n;
    return true;
}
// Spin of a neighbour through the frame: periodic copy or 0 (PottsMC::fillFrame, PottsMC.cpp:226-277).
__device__ __forceinline__ int32_t spin_at(const McArgs& a, int x, int y, int z) {
    if (!mc_wrap(x, a.nx, a.per[0]) || !mc_wrap(y, a.ny, a.per[1]) || !mc_wrap(z, a.nz, a.per[2])) return 0;
    return a.spin[(uint64_t)x + (uint64_t)a.nx * ((uint64_t)y + (uint64_t)a.ny * z)];
}

// unlikeBeforeAfter's neighbour counts (PottsMC.cpp:394-430, PottsMC.hpp:191-204) for the cell
// (x, y, z) and variant var, one neighbour after another through the frame (the per-colour launches).
__device__ __forceinline__ void nb_counts_loop(const McArgs& a, const NbTable& nb, int var, int x, int y, int z,
                                               int32_t cur, int32_t prop, int& in_dom, int& same_a, int& same_b) {
    in_dom = same_a = same_b = 0;
    const int cnt = nb.count[var];
    for (int k = 0; k < cnt; ++k) {
        const int32_t sj = spin_at(a, x + nb.off[var][k][0], y + nb.off[var][k][1], z + nb.off[var][k][2]);
        in_dom += sj != 0;
        same_a += sj == cur;
        same_b += sj == prop;
    }
}
__device__ __forceinline__ void stage_nb(const McArgs& a, NbTable& s_nb) {
    const int* src = reinterpret_cast<const int*>(a.nb);
    int* dst = reinterpret_cast<int*>(&s_nb);
    for (int i = threadIdx.x; i < (int)(sizeof(NbTable) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
}
static_assert(sizeof(NbTable) % sizeof(int) == 0, "NbTable is copied as ints");

// PottsMC::axisClass / colorOf (PottsMC.cpp:145-158), colour numbering of buildColors (173-193).
__host__ __device__ inline int axis_class(int c, int n, int periodic) {
    if (periodic && (n % 2) == 1 && c == n - 1) return 2;
    return c & 1;
}
__host__ __device__ inline int color_of(const McArgs& a, int x, int y, int z) {
    z += a.zoff;  // a slab colours by global z (its z axis is never periodic)
    if (a.parity_colors) return (x + y + z) & 1;
    const int cx = axis_class(x, a.nx, a.per[0]), cy = axis_class(y, a.ny, a.per[1]), cz = axis_class(z, a.nz, a.per[2]);
    return cx + a.classes[0] * (cy + a.classes[1] * cz);
}

__device__ __forceinline__ void decode(const McArgs& a, uint32_t g, int& x, int& y, int& z) {
    const uint32_t r = fdiv(g, a.div_nx);
    x = (int)(g - r * (uint32_t)a.nx);
    const uint32_t zz = fdiv(r, a.div_ny);
    y = (int)(r - zz * (uint32_t)a.ny);
    z = (int)zz;
}

// PottsMC::initialize (PottsMC.cpp:104-143): 1 + hashRand(seed, 0, g, McInit) % Q in the domain.
__global__ void mc_init_kernel(McArgs a, const uint8_t* domain, uint64_t n) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        int32_t s = 0;
        if (domain[g])
            s = 1 + (int32_t)fast_mod(hash_salt(hash_index(hash_prefix(a.seed, 0), g + a.gidx_base), kSaltMcInit), a.q_mod);
        a.spin[g] = s;
    }
}

// Cells of each colour in the domain (buildColors' class sizes, PottsMC.cpp:194-223).
__global__ void mc_color_count_kernel(McArgs a, const uint8_t* domain, uint64_t n, int colors, unsigned long long* counts) {
    __shared__ unsigned int s_cnt[28];
    for (int c = threadIdx.x; c < 28; c += blockDim.x) s_cnt[c] = 0;
    __syncthreads();
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        if (!domain[g]) continue;
        int x, y, z;
        decode(a, (uint32_t)g, x, y, z);
        atomicAdd(&s_cnt[color_of(a, x, y, z)], 1u);
    }
    __syncthreads();
    for (int c = threadIdx.x; c < colors; c += blockDim.x)
        if (s_cnt[c]) atomicAdd(&counts[c], (unsigned long long)s_cnt[c]);
}

struct ColorPred {
    McArgs a;
    const uint8_t* domain;
    int color;
    __device__ bool operator()(uint32_t g) const {
        if (!domain[g]) return false;
        int x, y, z;
        decode(a, g, x, y, z);
        return color_of(a, x, y, z) == color;
    }
};

__global__ void mc_gather_mob_kernel(const uint32_t* list, const float* mob, float* out, uint64_t n) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x)
        out[j] = mob[list[j]];
}

// One colour of one MCS: colorTrials (PottsMC.cpp:394-448) for the list entries [0, count).
template <bool kMobility, bool kRandomNb>
__global__ __launch_bounds__(kMcThreads) void mc_color_kernel(McArgs a, const uint32_t* list, const float* list_mob,
                                                              uint64_t count, int last_color) {
    __shared__ unsigned long long s_table[kTableSide * kTableSide];
    __shared__ unsigned long long s_red[3][kMcThreads / 32];
    __shared__ bool s_last;
    __shared__ NbTable s_nb;
    for (int i = threadIdx.x; i < kTableSide * kTableSide; i += kMcThreads) s_table[i] = a.table[i];
    stage_nb(a, s_nb);
    __syncthreads();
    McCtrl* ctrl = a.ctrl;
    const uint32_t t = ctrl->sweeps;
    const uint64_t prefix = hash_prefix(a.seed, t);
    const NbTable& nb = s_nb;
    unsigned my_att = 0, my_acc = 0, my_up = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)kMcThreads + threadIdx.x; j < count; j += (uint64_t)gridDim.x * kMcThreads) {
        const uint32_t g = list[j];
        const uint64_t h = hash_index(prefix, g + a.gidx_base);
        if (kMobility) {
            const uint64_t r = hash_salt(h, kSaltMcMobility);
            if (__dmul_rn((double)(r >> 11), 1.0 / 9007199254740992.0) >= (double)list_mob[j]) continue;
        }
        ++my_att;
        int var = 0;
        if (kRandomNb) var = (int)fast_mod(hash_salt(h, kSaltNeighborhood), a.var_mod);
        int x, y, z;
        decode(a, g, x, y, z);
        const int32_t cur = a.spin[g];
        int32_t prop = 1 + (int32_t)fast_mod(hash_salt(h, kSaltMcOrient), a.qm1_mod);
        if (prop >= cur) ++prop;
        int in_dom, same_a, same_b;
        nb_counts_loop(a, nb, var, x, y, z, cur, prop, in_dom, same_a, same_b);
        const int before = in_dom - same_a, after = in_dom - same_b;
        const unsigned long long e = s_table[before * kTableSide + after];
        bool accept;
        if (e >> 63) {
            accept = true;
        } else {
            accept = e != 0 && (hash_salt(h, kSaltMcAccept) >> 11) < e;
            my_up += accept ? 1u : 0u;
        }
        if (accept) {
            a.spin[g] = prop;
            ++my_acc;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned ra = __reduce_add_sync(0xFFFFFFFFu, my_att);
    const unsigned rc = __reduce_add_sync(0xFFFFFFFFu, my_acc);
    const unsigned ru = __reduce_add_sync(0xFFFFFFFFu, my_up);
    if (lane == 0) {
        s_red[0][warp] = ra;
        s_red[1][warp] = rc;
        s_red[2][warp] = ru;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sa = 0, sc = 0, su = 0;
        for (int w = 0; w < kMcThreads / 32; ++w) {
            sa += s_red[0][w];
            sc += s_red[1][w];
            su += s_red[2][w];
        }
        if (sa) atomicAdd(&ctrl->attempts, sa);
        if (sc) {
            atomicAdd(&ctrl->accepted, sc);
            atomicAdd(&ctrl->sweep_accepted, sc);
        }
        if (su) atomicAdd(&ctrl->uphill, su);
        s_last = false;
        if (last_color) {
            __threadfence();
            s_last = atomicAdd(&ctrl->ticket, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        __threadfence();
        ctrl->ticket = 0;
        ctrl->sweeps = t + 1;   // ++sweeps_ (PottsMC.cpp:531)
        __threadfence();
    }
}

// Offsets (index 0: coordinate - 1, 1: the cell, 2: coordinate + 1, times `stride`) and presence of
// the two neighbours of coordinate c on an axis of n cells: wrapped on a periodic axis (a 2-cell axis
// sees its other cell on both sides), absent at the frame otherwise (PottsMC::fillFrame,
// PottsMC.cpp:226-277).
__device__ __forceinline__ void mc_axis_nb(int c, int n, int per, int64_t stride, int64_t o[3], bool k[3]) {
    const bool wrap = per && n > 1;
    o[0] = c > 0 ? -stride : (int64_t)(n - 1) * stride;
    o[1] = 0;
    o[2] = c < n - 1 ? stride : -(int64_t)(n - 1) * stride;
    k[0] = c > 0 || wrap;
    k[1] = true;
    k[2] = c < n - 1 || wrap;
}

// unlikeBeforeAfter's counts (PottsMC.cpp:394-430) of the cell g = (x, y, z) over the neighbours
// whose bit (dx + 1) + 3 (dy + 1) + 9 (dz + 1) is set in `mask` (the variant's neighbourhood), on one
// path for every cell: nine row addresses and three x offsets, wrapped on periodic axes, a missing
// neighbour (frame) read as `none`.  All loads of the cell go out together.  A neighbour counts as in
// the domain when its value is not `none` (orientations: 0 outside the domain; the byte copy of a
// whole-space domain: every existing cell).
template <typename T>
__device__ __forceinline__ void mc_count_block(const McArgs& a, const T* base, uint32_t g, int x, int y, int z, uint32_t mask,
                                               uint32_t none, uint32_t cur, uint32_t prop, int& in_dom, int& same_a,
                                               int& same_b) {
    int64_t ox[3], oy[3], oz[3];
    bool kx[3], ky[3], kz[3];
    mc_axis_nb(x, a.nx, a.per[0], 1, ox, kx);
    mc_axis_nb(y, a.ny, a.per[1], a.nx, oy, ky);
    mc_axis_nb(z, a.nz, a.per[2], (int64_t)a.nx * a.ny, oz, kz);
    const T* p = base + g;
    uint32_t sv[27];
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) {
            const T* r = p + oz[dz] + oy[dy];
            const bool rk = kz[dz] && ky[dy];
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int bit = dx + 3 * dy + 9 * dz;
                const bool k = rk && kx[dx] && ((mask >> bit) & 1u);
                sv[bit] = k ? (uint32_t)r[ox[dx]] : none;
            }
        }
    in_dom = same_a = same_b = 0;
#pragma unroll
    for (int bit = 0; bit < 27; ++bit) {
        if (bit == 13) continue;  // the cell itself
        in_dom += sv[bit] != none;
        same_a += sv[bit] == cur;
        same_b += sv[bit] == prop;
    }
}

// Colour classes of the domain list: colour c is list[off[c] .. off[c + 1]).  Thread i of the sweep
// launch (T threads) takes the entries off[c] + i + k T, k < rounds[c], of colour c; with `cached`
// set, each block keeps its threads' entries (and their mobilities) in shared memory for the whole
// launch, round r of the launch at [round0[c] + k] x kMcThreads.
struct McColors {
    int colors;
    int cached;
    int pre;           // cached and at most kPreRounds rounds per colour: draws computed a pass ahead
    int total_rounds;
    int rounds[28];
    int round0[28];
    uint64_t off[28];
    uint32_t mask[6];  // per variant: bit (dx + 1) + 3 (dy + 1) + 9 (dz + 1) of each neighbour
};

// Grid barrier of the cooperative sweep launches, in two halves so that a block can do work of its
// own between them.  Arrive: after __syncthreads (the block's writes of the pass are ordered before
// it), thread 0 adds one arrival with release semantics.  Wait: thread 0 polls the count with
// acquire loads until every block has arrived `epoch` times, then __syncthreads.  The count only
// grows during a launch and is zeroed before it.  The wait is bounded; a block that gives up, or
// sees that another gave up, returns false (ctrl->error is then set).
__device__ __forceinline__ void mc_barrier_arrive(McCtrl* ctrl) {
    __syncthreads();
    if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u64 [%0], 1;\n" ::"l"(&ctrl->bar_arrived) : "memory");
}
__device__ bool mc_barrier_wait(McCtrl* ctrl, unsigned nblocks, unsigned long long epoch) {
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        const unsigned long long* cnt = &ctrl->bar_arrived;
        volatile int* err = &ctrl->error;
        const unsigned long long target = epoch * nblocks;
        int ok = 1;
        long long spins = 0;
        for (;;) {
            unsigned long long v;
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];\n" : "=l"(v) : "l"(cnt) : "memory");
            if (v >= target) break;
            if (*err || ++spins > (1ll << 26)) {
                ok = 0;
                atomicOr(&ctrl->error, 1);
                break;
            }
            __nanosleep(20);
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// The random draws of one trial (hashRand of its sweep and cell: mobility test, neighbourhood
// variant, proposed orientation, acceptance number), which do not depend on any orientation.
struct McDraws {
    bool attempt;     // passed the mobility test
    int var;          // neighbourhood variant
    int32_t prop_raw; // 1 + r % (Q - 1), before the skip over the current orientation
    uint64_t acc;     // hashRand(..., McAccept)
};
template <bool kMobility, bool kRandomNb>
__device__ __forceinline__ McDraws mc_draws(const McArgs& a, uint64_t prefix, uint32_t g, float mob) {
    McDraws d;
    const uint64_t h = hash_index(prefix, g + a.gidx_base);
    d.attempt = true;
    if (kMobility) {
        const uint64_t r = hash_salt(h, kSaltMcMobility);
        d.attempt = __dmul_rn((double)(r >> 11), 1.0 / 9007199254740992.0) < (double)mob;
    }
    d.var = kRandomNb ? (int)fast_mod(hash_salt(h, kSaltNeighborhood), a.var_mod) : 0;
    d.prop_raw = 1 + (int32_t)fast_mod(hash_salt(h, kSaltMcOrient), a.qm1_mod);
    d.acc = hash_salt(h, kSaltMcAccept);
    return d;
}

// `sweeps` checkerboard MCS in one cooperative launch: the colour classes in ascending order
// (sweepColors, PottsMC.cpp:495-514), a grid barrier after each, the same trial as mc_color_kernel
// (colorTrials, PottsMC.cpp:394-493).  Replaces `sweeps` x `colors` launches.  A colour pass costs
// the latency of its rounds: the entry and mobility come from shared memory (staged once per
// launch); the draws of the trial were computed while the block waited at the previous barrier
// (col.pre: kept in shared memory, one slot per thread and round); the cell's spin and all its
// neighbours' spins are loaded together (one round trip to L2), then the decision and the store.
constexpr int kPreRounds = 4;  // rounds per colour whose draws are computed ahead
template <bool kMobility, bool kRandomNb>
__global__ __launch_bounds__(kMcThreads, 2) void mc_sweeps_kernel(const __grid_constant__ McArgs a,
                                                                  const __grid_constant__ McColors col, int sweeps) {
    // [total_rounds][kMcThreads] entries, then mobilities; then with col.pre the draws of the next
    // pass: [kPreRounds][kMcThreads] acceptance numbers, proposals, flags (bit 7 attempt, variant)
    extern __shared__ __align__(16) uint32_t s_ent[];
    __shared__ unsigned long long s_table[kTableSide * kTableSide];
    __shared__ unsigned long long s_red[3][kMcThreads / 32];
    for (int i = threadIdx.x; i < kTableSide * kTableSide; i += kMcThreads) s_table[i] = a.table[i];
    const uint64_t T = (uint64_t)gridDim.x * kMcThreads;
    const uint64_t me = (uint64_t)blockIdx.x * kMcThreads + threadIdx.x;
    const size_t cache_words = (size_t)col.total_rounds * kMcThreads * (kMobility ? 2 : 1);
    float* s_mob = reinterpret_cast<float*>(s_ent + (size_t)col.total_rounds * kMcThreads);
    uint64_t* s_pacc = reinterpret_cast<uint64_t*>(s_ent + cache_words);
    int32_t* s_pprop = reinterpret_cast<int32_t*>(s_pacc + kPreRounds * kMcThreads);
    uint8_t* s_pflag = reinterpret_cast<uint8_t*>(s_pprop + kPreRounds * kMcThreads);
    if (col.cached) {
        for (int c = 0; c < col.colors; ++c)
            for (int k = 0; k < col.rounds[c]; ++k) {
                const uint64_t j = col.off[c] + me + (uint64_t)k * T;
                const int slot = (col.round0[c] + k) * kMcThreads + threadIdx.x;
                const bool in = j < col.off[c + 1];
                s_ent[slot] = in ? a.list[j] : 0xFFFFFFFFu;
                if (kMobility) s_mob[slot] = in ? a.list_mob[j] : 0.f;
            }
    }
    __syncthreads();
    McCtrl* ctrl = a.ctrl;
    const uint32_t t0 = ctrl->sweeps;
    // this thread's draws of pass (sweep s, colour c) into its slots (col.pre only)
    auto precompute = [&](int s, int c) {
        const uint64_t prefix = hash_prefix(a.seed, t0 + (uint32_t)s);
        for (int k = 0; k < col.rounds[c]; ++k) {
            const int slot = (col.round0[c] + k) * kMcThreads + threadIdx.x;
            const uint32_t g = s_ent[slot];
            if (g == 0xFFFFFFFFu) continue;
            const McDraws d = mc_draws<kMobility, kRandomNb>(a, prefix, g, kMobility ? s_mob[slot] : 0.f);
            const int ps = k * kMcThreads + threadIdx.x;
            s_pacc[ps] = d.acc;
            s_pprop[ps] = d.prop_raw;
            s_pflag[ps] = (uint8_t)((d.attempt ? 0x80 : 0) | d.var);
        }
    };
    unsigned long long my_att = 0, my_acc = 0, my_up = 0;
    bool ok = true;
    unsigned long long epoch = 0;  // grid barriers passed in this launch
    if (col.pre && sweeps > 0) precompute(0, 0);
    for (int s = 0; s < sweeps && ok; ++s) {
        const uint64_t prefix = hash_prefix(a.seed, t0 + (uint32_t)s);
        for (int c = 0; c < col.colors && ok; ++c) {
            for (int k = 0; k < col.rounds[c]; ++k) {
                uint32_t g;
                float mob = 0.f;
                if (col.cached) {
                    const int slot = (col.round0[c] + k) * kMcThreads + threadIdx.x;
                    g = s_ent[slot];
                    if (kMobility && !col.pre) mob = s_mob[slot];
                } else {
                    const uint64_t j = col.off[c] + me + (uint64_t)k * T;
                    g = j < col.off[c + 1] ? a.list[j] : 0xFFFFFFFFu;
                    if (kMobility && g != 0xFFFFFFFFu) mob = a.list_mob[j];
                }
                if (g == 0xFFFFFFFFu) continue;
                McDraws d;
                if (col.pre) {
                    const int ps = k * kMcThreads + threadIdx.x;
                    const unsigned f = s_pflag[ps];
                    d.attempt = (f & 0x80u) != 0;
                    d.var = (int)(f & 0x7Fu);
                    d.prop_raw = s_pprop[ps];
                    d.acc = s_pacc[ps];
                } else {
                    d = mc_draws<kMobility, kRandomNb>(a, prefix, g, mob);
                }
                if (!d.attempt) continue;
                ++my_att;
                const int var = d.var;
                int x, y, z;
                decode(a, g, x, y, z);
                const int32_t cur = a.spin[g];
                int32_t prop = d.prop_raw;
                if (prop >= cur) ++prop;
                int in_dom, same_a, same_b;
                mc_count_block(a, a.spin, g, x, y, z, col.mask[var], 0u, (uint32_t)cur, (uint32_t)prop, in_dom,
                                     same_a, same_b);
                const unsigned long long th = s_table[(in_dom - same_a) * kTableSide + (in_dom - same_b)];
                bool accept;
                if (th >> 63) {
                    accept = true;
                } else {
                    accept = th != 0 && (d.acc >> 11) < th;
                    my_up += accept ? 1u : 0u;
                }
                if (accept) {
                    a.spin[g] = prop;
                    ++my_acc;
                }
            }
            mc_barrier_arrive(ctrl);
            if (col.pre) {  // the next pass's draws while the other blocks finish this one
                const bool last_c = c + 1 == col.colors;
                if (!last_c) precompute(s, c + 1);
                else if (s + 1 < sweeps) precompute(s + 1, 0);
            }
            ok = mc_barrier_wait(ctrl, gridDim.x, ++epoch);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long ra = my_att, rc = my_acc, ru = my_up;
    for (int off = 16; off > 0; off >>= 1) {
        ra += __shfl_down_sync(0xFFFFFFFFu, ra, off);
        rc += __shfl_down_sync(0xFFFFFFFFu, rc, off);
        ru += __shfl_down_sync(0xFFFFFFFFu, ru, off);
    }
    if (lane == 0) {
        s_red[0][warp] = ra;
        s_red[1][warp] = rc;
        s_red[2][warp] = ru;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sa = 0, sc = 0, su = 0;
        for (int w = 0; w < kMcThreads / 32; ++w) {
            sa += s_red[0][w];
            sc += s_red[1][w];
            su += s_red[2][w];
        }
        if (sa) atomicAdd(&ctrl->attempts, sa);
        if (sc) {
            atomicAdd(&ctrl->accepted, sc);
            atomicAdd(&ctrl->sweep_accepted, sc);
        }
        if (su) atomicAdd(&ctrl->uphill, su);
        // every block passed the last barrier, so no block reads ctrl->sweeps any more
        if (blockIdx.x == 0 && ok) ctrl->sweeps = t0 + (uint32_t)sweeps;
    }
}

// ------------------------------------------------------------------------------------------
// Whole-space domain (mc.domain = full, every cell a trial each MCS) with Q <= 256: the sweeps run on
// a one-byte copy of the orientations (orientation - 1, so 67 M cells take 67 MB and stay in L2) and
// enumerate the cells of each colour class directly instead of reading a list.  A cell's neighbours
// are loaded at fixed linear offsets when the cell is away from every face (no wrap or frame test),
// else through the frame as everywhere else.  Same trials, same order of colours, same results.
// ------------------------------------------------------------------------------------------
struct McDense {
    uint8_t* sp;             // orientation - 1 of every cell
    const float* mob;        // mobility of every cell (kMobility)
    int cnt[3][3];           // per axis and class: coordinates of the class
    FastDiv32 div[2][3];     // / cnt[0][c] and / cnt[1][c]
    uint32_t mask[6];        // per variant: bit (dx + 1) + 3 (dy + 1) + 9 (dz + 1) of each neighbour
};

// Coordinate i of class c on an axis of n cells split into `classes` classes (axisClass,
// PottsMC.cpp:145-151): every coordinate (1 class), c + 2 i (classes 0 and 1), the last cell (class 2
// of a periodic odd axis).
__device__ __forceinline__ int class_coord(int i, int c, int classes, int n) {
    return classes == 1 ? i : (c == 2 ? n - 1 : 2 * i + c);
}

__global__ void mc_pack8_kernel(const int32_t* spin, uint8_t* sp, uint64_t n) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x)
        sp[g] = (uint8_t)(spin[g] - 1);
}
__global__ void mc_unpack8_kernel(const uint8_t* sp, int32_t* spin, uint64_t n) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x)
        spin[g] = (int32_t)sp[g] + 1;
}

// kMoore3: the 26-cell Moore neighbourhood of a 3D space, whose interior cells read their 26
// neighbours from nine row addresses and immediate offsets.
template <bool kMobility, bool kRandomNb, bool kParity, bool kMoore3>
__global__ __launch_bounds__(kMcThreads, 3) void mc_dense_sweeps_kernel(const __grid_constant__ McArgs a,
                                                                        const __grid_constant__ McDense d, int sweeps) {
    __shared__ unsigned long long s_table[kTableSide * kTableSide];
    __shared__ unsigned long long s_red[3][kMcThreads / 32];
    for (int i = threadIdx.x; i < kTableSide * kTableSide; i += kMcThreads) s_table[i] = a.table[i];
    __syncthreads();
    McCtrl* ctrl = a.ctrl;
    const uint32_t t0 = ctrl->sweeps;
    const uint8_t* sp = d.sp;
    const uint64_t T = (uint64_t)gridDim.x * kMcThreads;
    const uint64_t me = (uint64_t)blockIdx.x * kMcThreads + threadIdx.x;
    const int colors = kParity ? 2 : a.classes[0] * a.classes[1] * a.classes[2];
    unsigned long long my_att = 0, my_acc = 0, my_up = 0;
    bool ok = true;
    unsigned long long epoch = 0;
    for (int s = 0; s < sweeps && ok; ++s) {
        const uint64_t prefix = hash_prefix(a.seed, t0 + (uint32_t)s);
        for (int c = 0; c < colors && ok; ++c) {
            int cx = 0, cy = 0, cz = 0;
            if (!kParity) {
                cx = c % a.classes[0];
                const int r = c / a.classes[0];
                cy = r % a.classes[1];
                cz = r / a.classes[1];
            }
            const uint32_t nxc = (uint32_t)d.cnt[0][cx], nyc = (uint32_t)d.cnt[1][cy];
            const uint64_t total = (uint64_t)nxc * nyc * (uint32_t)d.cnt[2][cz];
            for (uint64_t i = me; i < total; i += T) {
                uint32_t ix, iy;
                const uint32_t r = fast_divmod((uint32_t)i, d.div[0][cx], ix);
                const uint32_t iz = fast_divmod(r, d.div[1][cy], iy);
                int x, y, z;
                if (kParity) {
                    y = (int)iy;
                    z = (int)iz;
                    x = 2 * (int)ix + ((c + y + z + a.zoff) & 1);
                    if (x >= a.nx) continue;
                } else {
                    x = class_coord((int)ix, cx, a.classes[0], a.nx);
                    y = class_coord((int)iy, cy, a.classes[1], a.ny);
                    z = class_coord((int)iz, cz, a.classes[2], a.nz);
                }
                const uint32_t g = (uint32_t)x + (uint32_t)a.nx * ((uint32_t)y + (uint32_t)a.ny * (uint32_t)z);
                const uint64_t h = hash_index(prefix, g + a.gidx_base);
                if (kMobility) {
                    const uint64_t rr = hash_salt(h, kSaltMcMobility);
                    if (__dmul_rn((double)(rr >> 11), 1.0 / 9007199254740992.0) >= (double)d.mob[g]) continue;
                }
                ++my_att;
                int var = 0;
                if (kRandomNb) var = (int)fast_mod(hash_salt(h, kSaltNeighborhood), a.var_mod);
                const int cur = (int)sp[g] + 1;
                int prop = 1 + (int)fast_mod(hash_salt(h, kSaltMcOrient), a.qm1_mod);
                if (prop >= cur) ++prop;
                const uint32_t cb = (uint32_t)(cur - 1), pb = (uint32_t)(prop - 1);
                int in_dom, same_a, same_b;
                mc_count_block(a, sp, g, x, y, z, kMoore3 ? 0x7FFFFFFu & ~(1u << 13) : d.mask[var], 0x100u, cb, pb,
                                      in_dom, same_a, same_b);
                const unsigned long long th = s_table[(in_dom - same_a) * kTableSide + (in_dom - same_b)];
                bool accept;
                if (th >> 63) {
                    accept = true;
                } else {
                    accept = th != 0 && (hash_salt(h, kSaltMcAccept) >> 11) < th;
                    my_up += accept ? 1u : 0u;
                }
                if (accept) {
                    d.sp[g] = (uint8_t)pb;
                    ++my_acc;
                }
            }
            mc_barrier_arrive(ctrl);
            ok = mc_barrier_wait(ctrl, gridDim.x, ++epoch);
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned long long ra = my_att, rc = my_acc, ru = my_up;
    for (int off = 16; off > 0; off >>= 1) {
        ra += __shfl_down_sync(0xFFFFFFFFu, ra, off);
        rc += __shfl_down_sync(0xFFFFFFFFu, rc, off);
        ru += __shfl_down_sync(0xFFFFFFFFu, ru, off);
    }
    if (lane == 0) {
        s_red[0][warp] = ra;
        s_red[1][warp] = rc;
        s_red[2][warp] = ru;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sa = 0, sc = 0, su = 0;
        for (int w = 0; w < kMcThreads / 32; ++w) {
            sa += s_red[0][w];
            sc += s_red[1][w];
            su += s_red[2][w];
        }
        if (sa) atomicAdd(&ctrl->attempts, sa);
        if (sc) {
            atomicAdd(&ctrl->accepted, sc);
            atomicAdd(&ctrl->sweep_accepted, sc);
        }
        if (su) atomicAdd(&ctrl->uphill, su);
        if (blockIdx.x == 0 && ok) ctrl->sweeps = t0 + (uint32_t)sweeps;
    }
}

// PottsMC::totalEnergy (PottsMC.cpp:590-664): unlike pairs.  Deterministic neighbourhoods count
// each pair once through the forward offsets; random ones sum E_i over the cells with the
// variant of MCS t (the caller halves it).
__global__ __launch_bounds__(kMcThreads) void mc_energy_kernel(McArgs a, const uint32_t* list, uint64_t count, int forward) {
    __shared__ unsigned long long s_sum;
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    const NbTable& nb = *a.nb;
    const uint64_t prefix = hash_prefix(a.seed, a.ctrl->sweeps);
    unsigned long long mine = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)kMcThreads + threadIdx.x; j < count; j += (uint64_t)gridDim.x * kMcThreads) {
        const uint32_t g = list[j];
        int x, y, z;
        decode(a, g, x, y, z);
        const int32_t s = a.spin[g];
        int var = 0;
        if (!forward && a.variants > 1)
            var = (int)fast_mod(hash_salt(hash_index(prefix, g + a.gidx_base), kSaltNeighborhood), a.var_mod);
        int in_dom = 0, same = 0;
        for (int k = 0; k < nb.count[var]; ++k) {
            const int dx = nb.off[var][k][0], dy = nb.off[var][k][1], dz = nb.off[var][k][2];
            if (forward && !(dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0))))) continue;
            const int32_t sj = spin_at(a, x + dx, y + dy, z + dz);
            in_dom += sj != 0;
            same += sj == s;
        }
        mine += (unsigned long long)(in_dom - same);
    }
    for (int off = 16; off > 0; off >>= 1) mine += __shfl_down_sync(0xFFFFFFFFu, mine, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_sum, mine);
    __syncthreads();
    if (threadIdx.x == 0 && s_sum) atomicAdd(&a.ctrl->energy_acc, s_sum);
}

// ------------------------------------------------------------------------------------------
// Grain statistics on the device (labelGrains, engine/src/mc/Grains.cpp:33-150; the majority
// classes by mobility of McStage, engine/src/app/McStage.cpp:38-66).  A grain is a connected set
// of domain cells of one orientation (von Neumann or Moore connectivity, periodic axes joined).
// Lock-free union-find over the domain list: a root is only ever linked to a smaller root by
// compare-and-swap, so parents only decrease and every loop ends; the components do not depend on
// the order of the unions.  Loops are bounded anyway; running out sets an error flag.
// ------------------------------------------------------------------------------------------
struct GrainAcc {
    unsigned long long grains, cells, largest, high_cells;
    unsigned long long high_grains, high_in, high_largest, low_grains, low_in, low_largest;
    unsigned int error;
};

__device__ __forceinline__ uint32_t gr_find(uint32_t* parent, uint32_t x, unsigned* err) {
    for (int i = 0; i < (1 << 24); ++i) {
        const uint32_t p = parent[x];
        if (p == x) return x;
        const uint32_t gp = parent[p];
        if (gp != p) parent[x] = gp;  // path halving: gp is an ancestor of x, so the write is benign
        x = gp;
    }
    atomicOr(err, 1u);
    return x;
}

__device__ __forceinline__ void gr_union(uint32_t* parent, uint32_t a, uint32_t b, unsigned* err) {
    for (int i = 0; i < (1 << 20); ++i) {
        uint32_t ra = gr_find(parent, a, err), rb = gr_find(parent, b, err);
        if (ra == rb) return;
        if (ra > rb) {
            const uint32_t t = ra;
            ra = rb;
            rb = t;
        }
        if (atomicCAS(&parent[rb], rb, ra) == rb) return;  // rb was still a root: linked under ra
        a = ra;
        b = rb;
    }
    atomicOr(err, 1u);
}

__global__ void mc_grain_init_kernel(const uint32_t* list, uint64_t count, uint32_t* parent, uint32_t* gsize, uint32_t* ghigh) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = list[j];
        parent[g] = g;
        gsize[g] = 0;
        ghigh[g] = 0;
    }
}

// Forward offsets of the connectivity (dz, dy, dx order, forward half) on the axes of size > 1.
__global__ void mc_grain_union_kernel(McArgs a, const uint32_t* list, uint64_t count, int moore, uint32_t* parent, GrainAcc* acc) {
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = list[j];
        const int32_t sg = a.spin[g];
        if (sg <= 0) continue;
        int x, y, z;
        decode(a, g, x, y, z);
        for (int dz = 0; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!(dz > 0 || (dz == 0 && (dy > 0 || (dy == 0 && dx > 0))))) continue;
                    if ((a.nx == 1 && dx) || (a.ny == 1 && dy) || (a.nz == 1 && dz)) continue;
                    if (!moore && abs(dx) + abs(dy) + abs(dz) != 1) continue;
                    int qx = x + dx, qy = y + dy, qz = z + dz;
                    if (!mc_wrap(qx, a.nx, a.per[0]) || !mc_wrap(qy, a.ny, a.per[1]) || !mc_wrap(qz, a.nz, a.per[2])) continue;
                    const uint32_t q = (uint32_t)qx + (uint32_t)a.nx * ((uint32_t)qy + (uint32_t)a.ny * (uint32_t)qz);
                    if (a.spin[q] == sg) gr_union(parent, g, q, &acc->error);
                }
    }
}

__global__ void mc_grain_count_kernel(McArgs a, const uint32_t* list, uint64_t count, const float* mob, double threshold,
                                      uint32_t* parent, uint32_t* gsize, uint32_t* ghigh, GrainAcc* acc) {
    unsigned long long cells = 0, high = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = list[j];
        if (a.spin[g] <= 0) continue;
        const uint32_t r = gr_find(parent, g, &acc->error);
        parent[g] = r;
        atomicAdd(&gsize[r], 1u);
        ++cells;
        if (mob != nullptr && (double)mob[g] >= threshold) {
            atomicAdd(&ghigh[r], 1u);
            ++high;
        }
    }
    cells = __reduce_add_sync(0xFFFFFFFFu, (unsigned)cells);
    high = __reduce_add_sync(0xFFFFFFFFu, (unsigned)high);
    if ((threadIdx.x & 31) == 0) {
        if (cells) atomicAdd(&acc->cells, cells);
        if (high) atomicAdd(&acc->high_cells, high);
    }
}

__global__ void mc_grain_reduce_kernel(McArgs a, const uint32_t* list, uint64_t count, const uint32_t* parent,
                                       const uint32_t* gsize, const uint32_t* ghigh, GrainAcc* acc) {
    unsigned long long grains = 0, largest = 0, hg = 0, hin = 0, hl = 0, lg = 0, lin = 0, ll = 0;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < count; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = list[j];
        if (a.spin[g] <= 0 || parent[g] != g) continue;
        const unsigned long long sz = gsize[g];
        ++grains;
        largest = max(largest, sz);
        if (2ull * ghigh[g] >= sz) {  // the class of the majority of its cells (ties: high)
            ++hg;
            hin += sz;
            hl = max(hl, sz);
        } else {
            ++lg;
            lin += sz;
            ll = max(ll, sz);
        }
    }
    if (grains) {
        atomicAdd(&acc->grains, grains);
        atomicMax(&acc->largest, largest);
        atomicAdd(&acc->high_grains, hg);
        atomicAdd(&acc->high_in, hin);
        atomicMax(&acc->high_largest, hl);
        atomicAdd(&acc->low_grains, lg);
        atomicAdd(&acc->low_in, lin);
        atomicMax(&acc->low_largest, ll);
    }
}

// CoolingMobility (engine/src/mc/CoolingMobility.cpp) on the device.
__global__ void mc_domain_from_ca_kernel(const uint8_t* type, int nx, int P, uint64_t rows, uint8_t* domain) {
    const uint64_t n = (uint64_t)nx * rows;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = g / nx;
        const int x = (int)(g - r * nx);
        const uint8_t t = type[r * P + x];
        domain[g] = (t == kBasalt || t == kLava) ? 1 : 0;  // basaltDomain (CoolingMobility.cpp:8-14)
    }
}

// endStep: largest solidStep / arrivalStep in the domain (CoolingMobility.cpp:16-25).
__global__ void mc_end_step_kernel(const uint16_t* solid, const uint16_t* arrival, const uint8_t* domain, int nx, int P,
                                   uint64_t rows, unsigned int* end_step) {
    unsigned m = 0;
    const uint64_t n = (uint64_t)nx * rows;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        if (!domain[g]) continue;
        const uint64_t r = g / nx;
        const uint64_t p = r * P + (g - r * nx);
        m = max(m, (unsigned)max(solid[p], arrival[p]));
    }
    m = __reduce_max_sync(0xFFFFFFFFu, m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(end_step, m);
}

// liquidTime (CoolingMobility.cpp:32-45) and its range (timeRange, 47-56): mm[0] = min, mm[1] = max.
__global__ void mc_time_range_kernel(const uint8_t* type, const uint16_t* solid, const uint16_t* arrival,
                                     const uint8_t* domain, int nx, int P, uint64_t rows, const unsigned int* end_step,
                                     unsigned int* time, unsigned int* mm) {
    unsigned lo = 0xFFFFFFFFu, hi = 0;
    const unsigned end = *end_step;
    const uint64_t n = (uint64_t)nx * rows;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        unsigned tm = 0;
        if (domain[g]) {
            const uint64_t r = g / nx;
            const uint64_t p = r * P + (g - r * nx);
            const unsigned s = type[p] == kBasalt ? solid[p] : end;
            const unsigned ar = arrival[p];
            tm = s > ar ? s - ar : 0;
            lo = min(lo, tm);
            hi = max(hi, tm);
        }
        time[g] = tm;
    }
    lo = __reduce_min_sync(0xFFFFFFFFu, lo);
    hi = __reduce_max_sync(0xFFFFFFFFu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&mm[0], lo);
        atomicMax(&mm[1], hi);
    }
}

// normalize (CoolingMobility.cpp:58-74): mobilityMin + (1 - mobilityMin) * (t - tMin) / (tMax - tMin)
// in double, each operation rounded once (no contraction), then to float.
__global__ void mc_normalize_kernel(const unsigned int* time, const uint8_t* domain, const unsigned int* mm,
                                    double mobility_min, uint64_t n, float* mobility) {
    const unsigned lo = mm[0], hi = mm[1];
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        float m = 0.0f;
        if (domain[g]) {
            if (hi == lo) {
                m = 1.0f;
            } else {
                const double norm = __ddiv_rn((double)(time[g] - lo), (double)(hi - lo));
                m = __double2float_rn(__dadd_rn(mobility_min, __dmul_rn(__dsub_rn(1.0, mobility_min), norm)));
            }
        }
        mobility[g] = m;
    }
}

}  // namespace vca

using namespace vca;

struct vca_mc {
    vca_mc_desc desc;
    int device = 0;
    cudaStream_t stream = nullptr;
    NbTable nb_host;
    NbTable* nb = nullptr;
    int per[3] = {0, 0, 0};
    int colors = 0;
    int parity_colors = 0;
    int classes[3] = {1, 1, 1};
    uint64_t n = 0;
    uint64_t cap_n = 0;                  // cells the per-cell buffers hold (a resident handle runs smaller spaces)
    int32_t* spin = nullptr;
    uint8_t* domain = nullptr;
    float* mobility = nullptr;     // N floats when set
    bool mobility_set = false;
    bool mobility_on = false;
    uint32_t* list = nullptr;      // domain cells by colour
    float* list_mob = nullptr;
    std::vector<uint64_t> color_off;
    unsigned long long* table = nullptr;
    McCtrl* ctrl = nullptr;
    McCtrl* ctrl_host = nullptr;      // pinned, host-mapped mirror
    McCtrl* ctrl_host_dev = nullptr;  // its device address
    bool domain_set = false;
    bool initialized = false;
    int sms = 148;
    // set-up buffers, allocated on first use and kept (no cudaMalloc / cudaFree per call)
    size_t list_cap = 0;                 // cells that list / list_mob can hold
    unsigned int* scratch = nullptr;     // mobility: [end, min, max] + time[n]
    void* cub_temp = nullptr;
    size_t cub_temp_bytes = 0;
    unsigned long long* d_count = nullptr;  // 28 colour counts
    uint32_t* gparent = nullptr;         // grain statistics: parent, size, high count per cell (n each)
    uint32_t* gsize = nullptr;
    uint32_t* ghigh = nullptr;
    void* gacc = nullptr;                // GrainAcc
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    double total_ms = 0.0;
    double color_ms = 0.0;
    uint64_t color_launches = 0;
    uint64_t launches = 0;
    int profile_kernels = 0;
    std::vector<cudaEvent_t> prof_events;
    int slab_zoff = -1;                  // z slab of a taller grid (vca_mc_set_slab), -1: none
    uint8_t* sp8 = nullptr;              // orientation - 1 per cell, for the whole-space sweeps (cap_n bytes)
};

namespace {

vca_status mc_check(const vca_mc* h) {
    if (!h) {
        set_error("null vca_mc handle");
        return VCA_ERR_ARG;
    }
    return VCA_OK;
}

McArgs mc_args(const vca_mc* h) {
    McArgs a;
    std::memset(&a, 0, sizeof(a));
    a.nx = h->desc.nx;
    a.ny = h->desc.ny;
    a.nz = h->desc.nz;
    for (int i = 0; i < 3; ++i) {
        a.per[i] = h->per[i];
        a.classes[i] = h->classes[i];
    }
    a.div_nx = make_fastdiv((uint32_t)a.nx);
    a.div_ny = make_fastdiv((uint32_t)a.ny);
    a.parity_colors = h->parity_colors;
    a.seed = h->desc.seed;
    a.q_mod = make_fastmod((uint64_t)h->desc.Q);
    a.qm1_mod = make_fastmod((uint64_t)(h->desc.Q - 1));
    a.var_mod = make_fastmod((uint64_t)h->nb_host.variants);
    a.variants = h->nb_host.variants;
    a.spin = h->spin;
    a.list = h->list;
    a.list_mob = h->list_mob;
    a.table = h->table;
    a.nb = h->nb;
    a.ctrl = h->ctrl;
    a.zoff = h->slab_zoff > 0 ? h->slab_zoff : 0;
    a.gidx_base = (uint64_t)h->desc.nx * h->desc.ny * (uint64_t)a.zoff;
    return a;
}

// The control block copied by one warp into host-mapped pinned memory (not a device-to-host copy,
// which would queue behind another handle's large download on the copy engines).
__global__ void mc_ctrl_snapshot_kernel(const McCtrl* src, McCtrl* dst) {
    static_assert(sizeof(McCtrl) % sizeof(uint32_t) == 0, "McCtrl is copied as words");
    const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
    volatile uint32_t* d = reinterpret_cast<volatile uint32_t*>(dst);
    for (int i = threadIdx.x; i < (int)(sizeof(McCtrl) / sizeof(uint32_t)); i += 32) d[i] = s[i];
}

vca_status mc_sync(vca_mc* h) {
    mc_ctrl_snapshot_kernel<<<1, 32, 0, h->stream>>>(h->ctrl, h->ctrl_host_dev);
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

int grid_for(uint64_t work, int sms) {
    const uint64_t b = (work + kMcThreads - 1) / kMcThreads;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)sms * 16));
}

void mc_free(vca_mc* h) {
    cudaSetDevice(h->device);
    cudaFree(h->nb);
    cudaFree(h->spin);
    cudaFree(h->domain);
    cudaFree(h->mobility);
    cudaFree(h->list);
    cudaFree(h->list_mob);
    cudaFree(h->table);
    cudaFree(h->ctrl);
    cudaFree(h->scratch);
    cudaFree(h->cub_temp);
    cudaFree(h->d_count);
    cudaFree(h->gparent);
    cudaFree(h->gsize);
    cudaFree(h->ghigh);
    cudaFree(h->gacc);
    cudaFree(h->sp8);
    if (h->ctrl_host) cudaFreeHost(h->ctrl_host);
    if (h->ev_a) cudaEventDestroy(h->ev_a);
    if (h->ev_b) cudaEventDestroy(h->ev_b);
    for (cudaEvent_t e : h->prof_events) cudaEventDestroy(e);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// A variant's neighbours as bits (dx + 1) + 3 (dy + 1) + 9 (dz + 1) of the 3 x 3 x 3 block.
uint32_t nb_mask(const NbTable& nb, int v) {
    uint32_t m = 0;
    if (v < nb.variants)
        for (int k = 0; k < nb.count[v]; ++k)
            m |= 1u << ((nb.off[v][k][0] + 1) + 3 * (nb.off[v][k][1] + 1) + 9 * (nb.off[v][k][2] + 1));
    return m;
}

using SweepsKernel = void (*)(McArgs, McColors, int);

SweepsKernel sweeps_kernel_of(const vca_mc* h) {
    const bool random_nb = h->nb_host.variants > 1;
    if (h->mobility_on) return random_nb ? mc_sweeps_kernel<true, true> : mc_sweeps_kernel<true, false>;
    return random_nb ? mc_sweeps_kernel<false, true> : mc_sweeps_kernel<false, false>;
}

constexpr size_t kMcEntryCacheMax = 160 * 1024;  // shared memory a block may spend on its entries

// The sweep kernel's cooperative grid (all blocks resident at once, no more blocks than the widest
// colour needs), its rounds per colour, and whether the blocks' entries fit in shared memory at
// that occupancy (then the dynamic shared memory size in *smem).
vca_status sweeps_launch_shape(vca_mc* h, SweepsKernel kernel, McColors* col, int* grid, size_t* smem) {
    uint64_t widest = 0;
    for (int c = 0; c < h->colors; ++c) widest = std::max<uint64_t>(widest, h->color_off[c + 1] - h->color_off[c]);
    const uint64_t need = std::max<uint64_t>(1, (widest + kMcThreads - 1) / kMcThreads);
    const size_t per_entry = h->mobility_on ? 8 : 4;
    VCA_CUDA(cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMcEntryCacheMax));
    int per_sm_max = 0;
    VCA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_max, kernel, kMcThreads, 0));
    per_sm_max = std::max(1, per_sm_max);
    auto rounds_for = [&](uint64_t threads) {
        int total = 0;
        for (int c = 0; c < h->colors; ++c) {
            const uint64_t n = h->color_off[c + 1] - h->color_off[c];
            col->rounds[c] = (int)((n + threads - 1) / threads);
            col->round0[c] = total;
            total += col->rounds[c];
        }
        col->total_rounds = total;
    };
    for (int per_sm = per_sm_max; per_sm >= 1; --per_sm) {
        const int g = (int)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)h->sms * per_sm));
        rounds_for((uint64_t)g * kMcThreads);
        int most = 0;
        for (int c = 0; c < h->colors; ++c) most = std::max(most, col->rounds[c]);
        const bool pre = most <= kPreRounds;
        const size_t bytes = (size_t)col->total_rounds * kMcThreads * per_entry +
                             (pre ? (size_t)kPreRounds * kMcThreads * (8 + 4 + 1) : 0);
        if (bytes > kMcEntryCacheMax) continue;
        int fit = 0;
        VCA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, kernel, kMcThreads, bytes));
        if ((uint64_t)fit * h->sms < (uint64_t)g) continue;
        col->cached = 1;
        col->pre = pre;
        *grid = g;
        *smem = bytes;
        return VCA_OK;
    }
    // entries from global memory at full occupancy
    const int g = (int)std::max<uint64_t>(1, std::min<uint64_t>(need, (uint64_t)h->sms * per_sm_max));
    rounds_for((uint64_t)g * kMcThreads);
    col->cached = 0;
    col->pre = 0;
    *grid = g;
    *smem = 0;
    return VCA_OK;
}

using DenseKernel = void (*)(McArgs, McDense, int);

template <bool kParity>
DenseKernel dense_kernel_of(const vca_mc* h) {
    const bool random_nb = h->nb_host.variants > 1;
    const bool moore3 = !kParity && !random_nb && h->nb_host.count[0] == 26;
    if (moore3) return h->mobility_on ? mc_dense_sweeps_kernel<true, false, false, true> : mc_dense_sweeps_kernel<false, false, false, true>;
    if (h->mobility_on)
        return random_nb ? mc_dense_sweeps_kernel<true, true, kParity, false> : mc_dense_sweeps_kernel<true, false, kParity, false>;
    return random_nb ? mc_dense_sweeps_kernel<false, true, kParity, false> : mc_dense_sweeps_kernel<false, false, kParity, false>;
}

// The whole-space sweeps apply when every cell is in the domain and an orientation fits a byte.
bool dense_applies(const vca_mc* h) {
    return !h->profile_kernels && h->slab_zoff < 0 && h->desc.Q <= 256 && !h->color_off.empty() &&
           h->color_off.back() == h->n && h->n > 0;
}

McDense dense_args(const vca_mc* h) {
    McDense d;
    std::memset(&d, 0, sizeof(d));
    d.sp = h->sp8;
    d.mob = h->mobility_on ? h->mobility : nullptr;
    const int dims[3] = {h->desc.nx, h->desc.ny, h->desc.nz};
    for (int a = 0; a < 3; ++a) {
        const int n = dims[a];
        int* c = d.cnt[a];
        c[0] = c[1] = c[2] = 1;
        if (h->parity_colors) {
            c[0] = a == 0 ? (n + 1) / 2 : n;
        } else if (h->classes[a] == 1) {
            c[0] = n;
        } else if (h->classes[a] == 2) {
            c[0] = (n + 1) / 2;
            c[1] = n / 2;
        } else {
            c[0] = c[1] = (n - 1) / 2;
            c[2] = 1;
        }
    }
    for (int a = 0; a < 2; ++a)
        for (int c = 0; c < 3; ++c) d.div[a][c] = make_fastdiv32((uint32_t)std::max(1, d.cnt[a][c]));
    for (int v = 0; v < 6; ++v) d.mask[v] = nb_mask(h->nb_host, v);
    return d;
}

}  // namespace

namespace {

vca_status mc_validate(const vca_mc_desc* d, const char* who) {
    auto bad = [&](const std::string& m) {
        set_error(std::string(who) + ": " + m);
        return VCA_ERR_ARG;
    };
    if (d->nx < 1 || d->ny < 1 || d->nz < 1 || (d->nx > 1) + (d->ny > 1) + (d->nz > 1) < 2)
        return bad("the space must be 2D or 3D");
    if ((uint64_t)d->nx * d->ny * d->nz > 2000000000ULL) return bad("more than 2 000 000 000 cells");
    if (d->Q < 2) return bad("Q must be at least 2 (PottsMC needs two orientations)");
    if (!(d->J > 0.0) || !(d->kT >= 0.0)) return bad("J must be > 0 and kT >= 0");
    NbTable nb;
    if (!build_nb(d->neighborhood, d->nx, d->ny, d->nz, nb)) return bad("the hexagonal neighbourhood is defined in 2D only");
    return VCA_OK;
}

// The space and parameters of an MC handle: neighbourhood, periodic axes, colours, acceptance
// table; orientations and domain cleared.  Allocates nothing.
vca_status mc_configure(vca_mc* h, const vca_mc_desc* d) {
    h->desc = *d;
    h->n = (uint64_t)d->nx * d->ny * d->nz;
    build_nb(d->neighborhood, d->nx, d->ny, d->nz, h->nb_host);
    h->slab_zoff = -1;
    // Periodic axes: PottsMC ctor (PottsMC.cpp:18) with the Boundary of McStage::run (McStage.cpp:106).
    const bool periodic = d->boundary == VCA_BC_PERIODIC;
    h->per[0] = periodic && d->nx > 1;
    h->per[1] = periodic && d->ny > 1;
    h->per[2] = periodic && d->domain_full && d->nz > 1;
    // Colours (PottsMC::buildColors, PottsMC.cpp:160-193).
    const int dims[3] = {d->nx, d->ny, d->nz};
    bool odd = false;
    for (int a = 0; a < 3; ++a) odd = odd || (h->per[a] && dims[a] % 2 == 1);
    h->parity_colors = d->neighborhood == VCA_NB_VON_NEUMANN && !odd;
    for (int a = 0; a < 3; ++a) h->classes[a] = 1;
    if (h->parity_colors) {
        h->colors = 2;
    } else {
        h->colors = 1;
        for (int a = 0; a < 3; ++a) {
            h->classes[a] = dims[a] == 1 ? 1 : (h->per[a] && dims[a] % 2 == 1 ? 3 : 2);
            h->colors *= h->classes[a];
        }
    }
    // Acceptance thresholds for every (unlikeBefore, unlikeAfter): dE = J*after - J*before
    // (PottsMC.cpp:431); dE <= 0 always (bit 63), else ceil(exp(-dE/kT) * 2^53), or 0 when kT = 0.
    std::vector<unsigned long long> table(kTableSide * kTableSide, 0);
    for (int b = 0; b < kTableSide; ++b)
        for (int a = 0; a < kTableSide; ++a) {
            const double dE = d->J * a - d->J * b;
            unsigned long long v = 0;
            if (dE <= 0.0) {
                v = 1ULL << 63;
            } else if (d->kT > 0.0) {
                const double p = std::exp(-dE / d->kT);
                v = (unsigned long long)std::ceil(p * 9007199254740992.0);
            }
            table[b * kTableSide + a] = v;
        }
    VCA_CUDA(cudaMemcpyAsync(h->nb, &h->nb_host, sizeof(NbTable), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaMemcpyAsync(h->table, table.data(), 8 * table.size(), cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->spin, 0, 4 * h->n, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->domain, 0, h->n, h->stream));
    VCA_CUDA(cudaMemsetAsync(h->ctrl, 0, sizeof(McCtrl), h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->domain_set = false;
    h->mobility_set = false;
    h->mobility_on = false;
    h->initialized = false;
    h->color_off.assign(1, 0);
    return VCA_OK;
}

}  // namespace

extern "C" {

vca_status vca_mc_create(const vca_mc_desc* d, vca_mc** out) {
    if (!d || !out) {
        set_error("vca_mc_create: null argument");
        return VCA_ERR_ARG;
    }
    *out = nullptr;
    if (vca_status s = mc_validate(d, "vca_mc_create")) return s;
    const uint64_t n = (uint64_t)d->nx * d->ny * d->nz;
    vca_mc* h = new vca_mc();
    h->device = d->device;
    h->cap_n = n;
    auto fail = [&](vca_status s) {
        mc_free(h);
        delete h;
        return s;
    };
    cudaError_t e = cudaSetDevice(d->device);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaSetDevice"));
    cudaDeviceProp prop;
    if ((e = cudaGetDeviceProperties(&prop, d->device)) != cudaSuccess) return fail(cuda_fail(e, "cudaGetDeviceProperties"));
    if (prop.major < 10) {
        set_error("vca_mc_create: needs an sm_100 (Blackwell) device");
        return fail(VCA_ERR_CUDA);
    }
    h->sms = prop.multiProcessorCount;
    e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail(cuda_fail(e, "cudaStreamCreate"));
    if ((e = cudaMalloc(&h->nb, sizeof(NbTable))) != cudaSuccess || (e = cudaMalloc(&h->spin, 4 * n)) != cudaSuccess ||
        (e = cudaMalloc(&h->domain, n)) != cudaSuccess ||
        (e = cudaMalloc(&h->table, 8 * kTableSide * kTableSide)) != cudaSuccess ||
        (e = cudaMalloc(&h->ctrl, sizeof(McCtrl))) != cudaSuccess)
        return fail(cuda_fail(e, "cudaMalloc"));
    if ((e = cudaHostAlloc(&h->ctrl_host, sizeof(McCtrl), cudaHostAllocMapped)) != cudaSuccess ||
        (e = cudaHostGetDevicePointer(&h->ctrl_host_dev, h->ctrl_host, 0)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaHostAlloc (mapped)"));
    if ((e = cudaEventCreate(&h->ev_a)) != cudaSuccess || (e = cudaEventCreate(&h->ev_b)) != cudaSuccess)
        return fail(cuda_fail(e, "cudaEventCreate"));
    const char* prof = std::getenv("VCA_PROFILE_KERNELS");
    h->profile_kernels = prof != nullptr && prof[0] == '1';
    if (vca_status s = mc_configure(h, d)) return fail(s);
    *out = h;
    return VCA_OK;
}

vca_status vca_mc_reconfigure(vca_mc* h, const vca_mc_desc* d) {
    if (vca_status s = mc_check(h)) return s;
    if (!d) {
        set_error("vca_mc_reconfigure: null desc");
        return VCA_ERR_ARG;
    }
    if (vca_status s = mc_validate(d, "vca_mc_reconfigure")) return s;
    if (d->device != h->device || (uint64_t)d->nx * d->ny * d->nz > h->cap_n) {
        set_error("vca_mc_reconfigure: the space does not fit the handle (more cells, or another device)");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    return mc_configure(h, d);
}

vca_status vca_mc_footprint(const vca_mc_desc* d, uint64_t* bytes) {
    if (!d || !bytes) {
        set_error("vca_mc_footprint: null argument");
        return VCA_ERR_ARG;
    }
    if (vca_status s = mc_validate(d, "vca_mc_footprint")) return s;
    const uint64_t n = (uint64_t)d->nx * d->ny * d->nz;
    // spin 4 + domain 1 + mobility 4 + mobility scratch 4 + colour lists 8 + grain labels 12 bytes per cell,
    // the list-selection scratch (bounded by 4 bytes per cell), tables and counters
    *bytes = 37 * n + 8 * kTableSide * kTableSide + sizeof(McCtrl) + 8 * 28 + sizeof(NbTable) + 4096;
    return VCA_OK;
}

vca_status vca_mc_set_domain(vca_mc* h, const uint8_t* in_domain) {
    if (vca_status s = mc_check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (in_domain) {
        std::vector<uint8_t> d(in_domain, in_domain + h->n);
        for (auto& v : d) v = v ? 1 : 0;
        VCA_CUDA(cudaMemcpyAsync(h->domain, d.data(), h->n, cudaMemcpyHostToDevice, h->stream));
        VCA_CUDA(cudaStreamSynchronize(h->stream));
    } else {
        VCA_CUDA(cudaMemsetAsync(h->domain, 1, h->n, h->stream));
    }
    h->domain_set = true;
    h->initialized = false;
    return VCA_OK;
}

vca_status vca_mc_set_mobility(vca_mc* h, const float* mobility) {
    if (vca_status s = mc_check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (!mobility) {
        h->mobility_on = false;
        return VCA_OK;
    }
    if (!h->mobility) VCA_CUDA(cudaMalloc(&h->mobility, 4 * h->cap_n));
    VCA_CUDA(cudaMemcpyAsync(h->mobility, mobility, 4 * h->n, cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->mobility_set = true;
    h->mobility_on = true;
    h->initialized = false;
    return VCA_OK;
}

vca_status vca_mc_set_domain_from_ca(vca_mc* h, vca_ca* ca) {
    if (vca_status s = mc_check(h)) return s;
    CaView v;
    if (vca_status s = ca_view(ca, &v)) return s;
    if (v.nx != h->desc.nx || v.ny != h->desc.ny || v.nz != h->desc.nz) {
        set_error("vca_mc_set_domain_from_ca: CA and MC dimensions differ");
        return VCA_ERR_ARG;
    }
    if (v.device != h->device) {
        set_error("vca_mc_set_domain_from_ca: CA and MC handles live on different devices");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaStreamSynchronize(v.stream));
    mc_domain_from_ca_kernel<<<h->sms * 8, 256, 0, h->stream>>>(v.type, v.nx, v.P, (uint64_t)v.ny * v.nz, h->domain);
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->domain_set = true;
    h->initialized = false;
    return VCA_OK;
}

vca_status vca_mc_set_mobility_from_ca(vca_mc* h, vca_ca* ca, double mobility_min, int use_in_dynamics) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->domain_set) {
        set_error("vca_mc_set_mobility_from_ca: set the domain first");
        return VCA_ERR_STATE;
    }
    CaView v;
    if (vca_status s = ca_view(ca, &v)) return s;
    if (v.nx != h->desc.nx || v.ny != h->desc.ny || v.nz != h->desc.nz || v.device != h->device) {
        set_error("vca_mc_set_mobility_from_ca: CA and MC handles do not match");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaStreamSynchronize(v.stream));
    if (!h->mobility) VCA_CUDA(cudaMalloc(&h->mobility, 4 * h->cap_n));
    if (!h->scratch) VCA_CUDA(cudaMalloc(&h->scratch, 4 * (3 + h->cap_n)));
    unsigned int* scratch = h->scratch;  // [end, min, max] + time[n]
    const unsigned int init[3] = {0u, 0xFFFFFFFFu, 0u};
    VCA_CUDA(cudaMemcpyAsync(scratch, init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
    const uint64_t rows = (uint64_t)v.ny * v.nz;
    const int blocks = h->sms * 8;
    mc_end_step_kernel<<<blocks, 256, 0, h->stream>>>(v.solid, v.arrival, h->domain, v.nx, v.P, rows, scratch);
    mc_time_range_kernel<<<blocks, 256, 0, h->stream>>>(v.type, v.solid, v.arrival, h->domain, v.nx, v.P, rows, scratch,
                                                        scratch + 3, scratch + 1);
    mc_normalize_kernel<<<blocks, 256, 0, h->stream>>>(scratch + 3, h->domain, scratch + 1, mobility_min, h->n, h->mobility);
    cudaError_t e = cudaGetLastError();
    cudaError_t e2 = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_fail(e, "mobility kernels");
    if (e2 != cudaSuccess) return cuda_fail(e2, "mobility kernels");
    h->mobility_set = true;
    h->mobility_on = use_in_dynamics != 0;
    h->initialized = false;
    return VCA_OK;
}

vca_status vca_mc_mobility(vca_mc* h, float* out) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->mobility_set) {
        set_error("vca_mc_mobility: no mobility was set");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemcpyAsync(out, h->mobility, 4 * h->n, cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_mc_initialize(vca_mc* h) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->domain_set) {
        set_error("vca_mc_initialize: set the domain first");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    McArgs a = mc_args(h);
    mc_init_kernel<<<h->sms * 8, 256, 0, h->stream>>>(a, h->domain, h->n);
    VCA_CUDA(cudaGetLastError());
    // Colour lists, colour by colour, globalIndex ascending inside a colour (PottsMC.cpp:194-223):
    // count the cells of each colour, then select each colour into its place of one list.
    if (!h->d_count) VCA_CUDA(cudaMalloc(&h->d_count, 8 * 28));
    VCA_CUDA(cudaMemsetAsync(h->d_count, 0, 8 * 28, h->stream));
    mc_color_count_kernel<<<h->sms * 8, 256, 0, h->stream>>>(a, h->domain, h->n, h->colors, h->d_count);
    VCA_CUDA(cudaGetLastError());
    std::vector<unsigned long long> counts((size_t)h->colors, 0);
    VCA_CUDA(cudaMemcpyAsync(counts.data(), h->d_count, 8 * (size_t)h->colors, cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->color_off.assign((size_t)h->colors + 1, 0);
    uint64_t total = 0;
    for (int c = 0; c < h->colors; ++c) {
        h->color_off[c] = total;
        total += counts[c];
    }
    h->color_off[h->colors] = total;
    if (total > h->list_cap || (h->mobility_on && !h->list_mob)) {
        cudaFree(h->list);
        cudaFree(h->list_mob);
        h->list = nullptr;
        h->list_mob = nullptr;
        h->list_cap = std::max<uint64_t>(std::max<uint64_t>(total, h->cap_n), 1);  // once per handle
        VCA_CUDA(cudaMalloc(&h->list, 4 * h->list_cap));
        VCA_CUDA(cudaMalloc(&h->list_mob, 4 * h->list_cap));
    }
    ColorPred pred{a, h->domain, 0};
    thrust::counting_iterator<uint32_t> it(0);
    size_t temp_bytes = 0;
    // sized for the capacity, so that later, larger spaces on a resident handle allocate nothing
    VCA_CUDA(cub::DeviceSelect::If(nullptr, temp_bytes, it, h->list, h->d_count, (int64_t)h->cap_n, pred, h->stream));
    if (temp_bytes > h->cub_temp_bytes) {
        cudaFree(h->cub_temp);
        h->cub_temp = nullptr;
        VCA_CUDA(cudaMalloc(&h->cub_temp, temp_bytes));
        h->cub_temp_bytes = temp_bytes;
    }
    for (int c = 0; c < h->colors; ++c) {
        if (counts[c] == 0) continue;
        pred.color = c;
        VCA_CUDA(cub::DeviceSelect::If(h->cub_temp, temp_bytes, it, h->list + h->color_off[c], h->d_count + c, (int64_t)h->n, pred,
                                       h->stream));
    }
    if (h->mobility_on && total) {
        mc_gather_mob_kernel<<<grid_for(total, h->sms), 256, 0, h->stream>>>(h->list, h->mobility, h->list_mob, total);
        VCA_CUDA(cudaGetLastError());
    }
    VCA_CUDA(cudaMemsetAsync(h->ctrl, 0, sizeof(McCtrl), h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    h->initialized = true;
    return VCA_OK;
}

vca_status vca_mc_sweep(vca_mc* h, int count, uint64_t* accepted) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->initialized) {
        set_error("vca_mc_sweep: initialize first");
        return VCA_ERR_STATE;
    }
    if (count < 0) {
        set_error("vca_mc_sweep: negative count");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    McArgs a = mc_args(h);
    VCA_CUDA(cudaMemsetAsync(&h->ctrl->sweep_accepted, 0, 8, h->stream));
    // a cooperative sweep launch: its barrier count starts at zero
    auto barrier_reset = [&](int) -> vca_status {
        VCA_CUDA(cudaMemsetAsync(&h->ctrl->bar_arrived, 0, sizeof(unsigned long long), h->stream));
        return VCA_OK;
    };
    if (!h->profile_kernels) {
        // all sweeps in one cooperative launch (colour passes separated by grid barriers)
        McColors col;
        std::memset(&col, 0, sizeof(col));
        col.colors = h->colors;
        for (int c = 0; c <= h->colors; ++c) col.off[c] = h->color_off[c];
        for (int v = 0; v < 6; ++v) col.mask[v] = nb_mask(h->nb_host, v);
        int grid = 1;
        size_t smem = 0;
        SweepsKernel kernel = sweeps_kernel_of(h);
        if (vca_status s = sweeps_launch_shape(h, kernel, &col, &grid, &smem)) return s;
        const bool dense = dense_applies(h);
        if (dense && !h->sp8) VCA_CUDA(cudaMalloc(&h->sp8, h->cap_n));
        VCA_CUDA(cudaEventRecord(h->ev_a, h->stream));
        if (count > 0 && dense) {
            // whole space: sweeps on the byte copy of the orientations, copied back after
            const McDense d = dense_args(h);
            DenseKernel dk = h->parity_colors ? dense_kernel_of<true>(h) : dense_kernel_of<false>(h);
            int per_sm = 0;
            VCA_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dk, kMcThreads, 0));
            const int dgrid = h->sms * std::max(1, per_sm);
            const int blocks = grid_for(h->n, h->sms);
            mc_pack8_kernel<<<blocks, 256, 0, h->stream>>>(h->spin, h->sp8, h->n);
            VCA_CUDA(cudaGetLastError());
            int n = count;
            McDense dd = d;
            void* args[] = {&a, &dd, &n};
            if (vca_status s = barrier_reset(dgrid)) return s;
            VCA_CUDA(cudaLaunchCooperativeKernel((const void*)dk, dgrid, kMcThreads, args, 0, h->stream));
            mc_unpack8_kernel<<<blocks, 256, 0, h->stream>>>(h->sp8, h->spin, h->n);
            VCA_CUDA(cudaGetLastError());
            h->launches += 3;
        } else if (count > 0 && h->color_off.back() > 0) {
            int n = count;
            void* args[] = {&a, &col, &n};
            if (vca_status s = barrier_reset(grid)) return s;
            VCA_CUDA(cudaLaunchCooperativeKernel((const void*)kernel, grid, kMcThreads, args, smem, h->stream));
            h->launches += 1;
        } else if (count > 0) {
            // empty domain: the sweeps still count (sweepsDone)
            McCtrl* c = h->ctrl_host;
            VCA_CUDA(cudaMemcpyAsync(c, h->ctrl, sizeof(McCtrl), cudaMemcpyDeviceToHost, h->stream));
            VCA_CUDA(cudaStreamSynchronize(h->stream));
            c->sweeps += (uint32_t)count;
            VCA_CUDA(cudaMemcpyAsync(h->ctrl, c, sizeof(McCtrl), cudaMemcpyHostToDevice, h->stream));
        }
        VCA_CUDA(cudaEventRecord(h->ev_b, h->stream));
        VCA_CUDA(cudaEventSynchronize(h->ev_b));
        float ms = 0.f;
        VCA_CUDA(cudaEventElapsedTime(&ms, h->ev_a, h->ev_b));
        h->total_ms += ms;
        if (vca_status s_ = mc_sync(h)) return s_;
        if (h->ctrl_host->error) {
            set_error("vca_mc_sweep: a bounded grid-barrier wait ran out");
            return VCA_ERR_TIMEOUT;
        }
        if (accepted) *accepted = h->ctrl_host->sweep_accepted;
        return VCA_OK;
    }
    VCA_CUDA(cudaEventRecord(h->ev_a, h->stream));
    const bool random_nb = h->nb_host.variants > 1;
    size_t ev_used = 0;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof;
    for (int s = 0; s < count; ++s) {
        for (int c = 0; c < h->colors; ++c) {
            const uint64_t b = h->color_off[c], e = h->color_off[c + 1];
            const uint64_t cnt = e - b;
            const int grid = grid_for(cnt, h->sms);
            const uint32_t* list = h->list + b;
            const float* mob = h->mobility_on ? h->list_mob + b : nullptr;
            const int last = c == h->colors - 1;
            cudaEvent_t e0 = nullptr, e1 = nullptr;
            if (h->profile_kernels) {
                while (h->prof_events.size() < ev_used + 2) {
                    cudaEvent_t ev;
                    VCA_CUDA(cudaEventCreate(&ev));
                    h->prof_events.push_back(ev);
                }
                e0 = h->prof_events[ev_used];
                e1 = h->prof_events[ev_used + 1];
                ev_used += 2;
                VCA_CUDA(cudaEventRecord(e0, h->stream));
            }
            if (h->mobility_on) {
                if (random_nb) mc_color_kernel<true, true><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
                else mc_color_kernel<true, false><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
            } else {
                if (random_nb) mc_color_kernel<false, true><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
                else mc_color_kernel<false, false><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
            }
            if (h->profile_kernels) {
                VCA_CUDA(cudaEventRecord(e1, h->stream));
                prof.push_back({e0, e1});
            }
        }
        h->launches += (uint64_t)h->colors;
        if (h->profile_kernels && prof.size() > 2048) break;  // bounded event pool per call
    }
    VCA_CUDA(cudaGetLastError());
    VCA_CUDA(cudaEventRecord(h->ev_b, h->stream));
    VCA_CUDA(cudaEventSynchronize(h->ev_b));
    float ms = 0.f;
    VCA_CUDA(cudaEventElapsedTime(&ms, h->ev_a, h->ev_b));
    h->total_ms += ms;
    for (auto& pr : prof) {
        float m = 0.f;
        VCA_CUDA(cudaEventElapsedTime(&m, pr.first, pr.second));
        h->color_ms += m;
        ++h->color_launches;
    }
    if (vca_status s_ = mc_sync(h)) return s_;
    if (accepted) *accepted = h->ctrl_host->sweep_accepted;
    return VCA_OK;
}

vca_status vca_mc_get_info(vca_mc* h, vca_mc_info* out) {
    if (vca_status s = mc_check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    if (vca_status s_ = mc_sync(h)) return s_;
    out->sweeps = (int)h->ctrl_host->sweeps;
    out->colors = h->colors;
    out->domain_cells = h->initialized ? h->color_off.back() : 0;
    out->attempts = h->ctrl_host->attempts;
    out->accepted = h->ctrl_host->accepted;
    out->uphill = h->ctrl_host->uphill;
    out->kernel_launches = h->launches;
    return VCA_OK;
}

vca_status vca_mc_grains(vca_mc* h, int moore, double mobility_threshold, vca_mc_grain_stats* out) {
    if (vca_status s = mc_check(h)) return s;
    if (!out) {
        set_error("vca_mc_grains: null output");
        return VCA_ERR_ARG;
    }
    if (!h->initialized) {
        set_error("vca_mc_grains: initialize first");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    if (!h->gparent) {
        VCA_CUDA(cudaMalloc(&h->gparent, 4 * h->cap_n));
        VCA_CUDA(cudaMalloc(&h->gsize, 4 * h->cap_n));
        VCA_CUDA(cudaMalloc(&h->ghigh, 4 * h->cap_n));
        VCA_CUDA(cudaMalloc(&h->gacc, sizeof(GrainAcc)));
    }
    GrainAcc* acc = static_cast<GrainAcc*>(h->gacc);
    VCA_CUDA(cudaMemsetAsync(acc, 0, sizeof(GrainAcc), h->stream));
    const uint64_t total = h->color_off.back();
    const McArgs a = mc_args(h);
    const float* mob = h->mobility_set ? h->mobility : nullptr;
    if (total) {
        const int grid = grid_for(total, h->sms);
        mc_grain_init_kernel<<<grid, kMcThreads, 0, h->stream>>>(h->list, total, h->gparent, h->gsize, h->ghigh);
        mc_grain_union_kernel<<<grid, kMcThreads, 0, h->stream>>>(a, h->list, total, moore, h->gparent, acc);
        mc_grain_count_kernel<<<grid, kMcThreads, 0, h->stream>>>(a, h->list, total, mob, mobility_threshold, h->gparent, h->gsize,
                                                                  h->ghigh, acc);
        mc_grain_reduce_kernel<<<grid, kMcThreads, 0, h->stream>>>(a, h->list, total, h->gparent, h->gsize, h->ghigh, acc);
        VCA_CUDA(cudaGetLastError());
        h->launches += 4;
    }
    GrainAcc r;
    VCA_CUDA(cudaMemcpyAsync(&r, acc, sizeof(r), cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    if (r.error) {
        set_error("vca_mc_grains: a bounded union-find loop ran out");
        return VCA_ERR_TIMEOUT;
    }
    out->grains = r.grains;
    out->cells = r.cells;
    out->largest = r.largest;
    out->high_cells = r.high_cells;
    out->high_grains = r.high_grains;
    out->high_grain_cells = r.high_in;
    out->high_largest = r.high_largest;
    out->low_grains = r.low_grains;
    out->low_grain_cells = r.low_in;
    out->low_largest = r.low_largest;
    return VCA_OK;
}

vca_status vca_mc_set_mobility_values(vca_mc* h, const float* mobility, int use_in_dynamics) {
    if (vca_status s = vca_mc_set_mobility(h, mobility)) return s;
    if (mobility) h->mobility_on = use_in_dynamics != 0;
    return VCA_OK;
}

vca_status vca_mc_energy(vca_mc* h, double* energy) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->initialized) {
        set_error("vca_mc_energy: initialize first");
        return VCA_ERR_STATE;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemsetAsync(&h->ctrl->energy_acc, 0, 8, h->stream));
    const uint64_t total = h->color_off.back();
    const bool forward = h->nb_host.variants == 1;
    if (total) mc_energy_kernel<<<grid_for(total, h->sms), kMcThreads, 0, h->stream>>>(mc_args(h), h->list, total, forward);
    h->launches += total ? 1 : 0;
    VCA_CUDA(cudaGetLastError());
    if (vca_status s_ = mc_sync(h)) return s_;
    const double unlike = (double)h->ctrl_host->energy_acc;
    *energy = forward ? h->desc.J * unlike : 0.5 * h->desc.J * unlike;
    return VCA_OK;
}

vca_status vca_mc_crystals(vca_mc* h, int32_t* out) {
    if (vca_status s = mc_check(h)) return s;
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemcpyAsync(out, h->spin, 4 * h->n, cudaMemcpyDeviceToHost, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_mc_set_spins(vca_mc* h, const int32_t* spins) {
    if (vca_status s = mc_check(h)) return s;
    if (!spins) {
        set_error("vca_mc_set_spins: null spins");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    VCA_CUDA(cudaMemcpyAsync(h->spin, spins, 4 * h->n, cudaMemcpyHostToDevice, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_mc_set_slab(vca_mc* h, int z_offset) {
    if (vca_status s = mc_check(h)) return s;
    if (z_offset < 0 || h->per[2] || h->desc.nz < 2) {
        set_error("vca_mc_set_slab: a slab needs z_offset >= 0, nz > 1 and no periodic z axis");
        return VCA_ERR_ARG;
    }
    if (h->initialized) {
        set_error("vca_mc_set_slab: set the slab before vca_mc_initialize");
        return VCA_ERR_STATE;
    }
    h->slab_zoff = z_offset;
    return VCA_OK;
}

vca_status vca_mc_color_pass(vca_mc* h, int color) {
    if (vca_status s = mc_check(h)) return s;
    if (!h->initialized) {
        set_error("vca_mc_color_pass: initialize first");
        return VCA_ERR_STATE;
    }
    if (color < 0 || color >= h->colors) {
        set_error("vca_mc_color_pass: colour out of range");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const McArgs a = mc_args(h);
    const uint64_t b = h->color_off[color], cnt = h->color_off[color + 1] - b;
    const int grid = grid_for(cnt, h->sms);
    const uint32_t* list = h->list + b;
    const float* mob = h->mobility_on ? h->list_mob + b : nullptr;
    const int last = color == h->colors - 1;
    const bool random_nb = h->nb_host.variants > 1;
    if (h->mobility_on) {
        if (random_nb) mc_color_kernel<true, true><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
        else mc_color_kernel<true, false><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
    } else {
        if (random_nb) mc_color_kernel<false, true><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
        else mc_color_kernel<false, false><<<grid, kMcThreads, 0, h->stream>>>(a, list, mob, cnt, last);
    }
    VCA_CUDA(cudaGetLastError());
    h->launches += 1;
    return VCA_OK;
}

static vca_status spin_layers(vca_mc* h, int z0, int layers, void* buf, bool to_buf, const char* who) {
    if (vca_status s = mc_check(h)) return s;
    if (buf == nullptr || z0 < 0 || layers < 0 || z0 + layers > h->desc.nz) {
        set_error(std::string(who) + ": layers outside the grid or null buffer");
        return VCA_ERR_ARG;
    }
    VCA_CUDA(cudaSetDevice(h->device));
    const size_t L = (size_t)h->desc.nx * h->desc.ny;
    int32_t* dev = h->spin + (size_t)z0 * L;
    const size_t bytes = (size_t)layers * L * sizeof(int32_t);
    if (to_buf)
        VCA_CUDA(cudaMemcpyAsync(buf, dev, bytes, cudaMemcpyDefault, h->stream));
    else
        VCA_CUDA(cudaMemcpyAsync(dev, buf, bytes, cudaMemcpyDefault, h->stream));
    VCA_CUDA(cudaStreamSynchronize(h->stream));
    return VCA_OK;
}

vca_status vca_mc_pack_spins(vca_mc* h, int z0, int layers, void* buf) {
    return spin_layers(h, z0, layers, buf, true, "vca_mc_pack_spins");
}

vca_status vca_mc_unpack_spins(vca_mc* h, int z0, int layers, const void* buf) {
    return spin_layers(h, z0, layers, const_cast<void*>(buf), false, "vca_mc_unpack_spins");
}

vca_status vca_mc_timing(vca_mc* h, double* total_ms, double* color_kernel_ms, uint64_t* color_launches) {
    if (vca_status s = mc_check(h)) return s;
    if (total_ms) *total_ms = h->total_ms;
    if (color_kernel_ms) *color_kernel_ms = h->color_launches ? h->color_ms / (double)h->color_launches : 0.0;
    if (color_launches) *color_launches = h->color_launches;
    return VCA_OK;
}

void vca_mc_destroy(vca_mc* h) {
    if (!h) return;
    mc_free(h);
    delete h;
}

}  // extern "C"

// vca_internal.h -- handle layouts and helpers shared by the CA and MC halves of libvca.so.
#pragma once

#include <cuda.h>  // CUtensorMap (encoded through the runtime's driver entry point, no libcuda link)
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "vca.h"
#include "vca_device.cuh"

namespace vca {

// Error channel of the C ABI: the message of the last failure on this host thread.
void set_error(const std::string& msg);
vca_status cuda_fail(cudaError_t e, const char* what);
std::vector<int32_t> fill_depressions(const std::vector<int32_t>& h, int nx, int ny, bool px, bool py);
bool build_nb(int kind, int nx, int ny, int nz, NbTable& t);

#define VCA_CUDA(call)                                              \
    do {                                                            \
        cudaError_t e__ = (call);                                   \
        if (e__ != cudaSuccess) return ::vca::cuda_fail(e__, #call); \
    } while (0)

// Device-side control block of a CA handle: step counter, stop state, per-step accumulators and
// the active-tile list lengths.  Written by the last block of each rules launch.
struct CaCtrl {
    uint32_t steps;           // steps done (t of the next step)
    int32_t stop;             // VCA_STOP_*
    uint64_t lava;            // LAVA cells after the last step (classic: grains)
    uint64_t air;             // AIR cells after the last step
    unsigned long long acc_active;   // accumulators of the running step
    unsigned long long acc_changed;
    unsigned long long acc_born;
    unsigned long long acc_tiles;
    unsigned int ticket;      // blocks finished in the running rules launch
    unsigned int list_count[2];
    unsigned int chg_count[2];  // cells whose type changed in the step that wrote them
    unsigned int cand_count;    // AIR cells listed for the candidate pass of the running step
    unsigned long long tiles_processed;  // tiles visited over all steps
    int32_t max_steps;
    int32_t random_nb;
    int32_t classic;
    int32_t error;            // bit 0: a bounded device wait ran out (the run stops, VCA_ERR_TIMEOUT)
    uint32_t tile_next;       // rules pass (DENSE): tiles handed out at run time in the running step
};

// Geometry of the pitched device planes.  Each (y, z) row holds P >= nx cells, P a multiple of 64,
// so that every row starts 64-byte aligned in every plane; cells x >= nx are VOID padding.
struct CaGeom {
    int nx, ny, nz;
    int P;                    // row pitch in cells
    int per[3];               // periodic axes (Boundary, engine/src/core/Boundary.cpp:5-11)
    int TY, TZ;               // tile rows: TY * TZ = 16, tile = 64 x TY x TZ cells
    int shape;                // shared-memory family of the rules pass for this tile (0, 1, 2)
    int tiles_x, tiles_y, tiles_z;
    FastDiv32 div_tx, div_ty;  // / tiles_x and / tiles_y (tile id -> tile coordinates)
};

struct CaTables {
    NbTable nb;
    int nside;
    int8_t side[8][3];        // union of the dz == 0 offsets of all variants (LavaCA.hpp:104-112)
};

// TMA descriptors of the pitched planes, seen as 3D tensors (P, ny, nz): per buffer the tile's own
// box {64, TY, TZ} of each plane, the type halo box {96, TY + 2, TZ + 2} from (x0 - 16, y0 - 1,
// z0 - 1), and the drop-depth rows {96, TY + 2, TZ} from (x0 - 16, y0 - 1, z0).
struct CaTensorMaps {
    CUtensorMap own_type[2], halo_type[2], drop;
    // 4D (x, y, z, plane): flowId + temperature, solidStep + arrivalStep (pairs allocated together)
    CUtensorMap ft[2], sa[2];
    // 16-cell-wide columns of the type halo rows {16, TY + 2, TZ + 2} and of the drop rows
    // {16, TY + 2, TZ}: with periodic x (nx a multiple of 16) an x-edge tile loads the column at the
    // other end of its rows, which holds its wrapped frame cell
    CUtensorMap xside_type[2], xside_drop;
};

// Everything a step kernel needs besides the tensor maps (those are a separate kernel parameter, so
// that a batched launch can copy the rest of a grid's arguments into shared memory).
struct CaKernelArgs {
    CaGeom g;
    int classic;
    int ponding;
    int diag_falls;           // LavaCA::diagonalFalls_ (LavaCA.hpp:108-110)
    uint32_t side_mask;       // side offsets (dz = 0) as bits 3 (dy + 1) + (dx + 1)
    int dense;
    uint64_t seed;
    int max_steps;
    int eruption_steps;
    float erupt_temp, solidus, cool_ambient, cool_lateral, cool_fall;
    FastMod var_mod;          // % variant count
    uint8_t* type[2];
    int32_t* flow[2];
    float* temp[2];
    uint16_t* solid[2];
    uint16_t* arrival[2];
    int8_t* drop;             // dropDepth of every AIR cell of the current state (LavaCA.hpp:404-414)
    uint32_t* chg_list[2];    // globalIndex of cells whose type changed (step t writes [(t+1) & 1])
    uint32_t chg_cap;         // capacity of each change list; more changes force a full rescan
    uint32_t* cand_list;      // globalIndex of AIR cells with LAVA within one cell (this step)
    const int32_t* spill;     // nx*ny or nullptr
    const int4* vents;        // (x, y, z, -) per flowId
    int vent_slots;
    CaTables tables;          // by value: read from the kernel parameter (constant) bank
    CaCtrl* ctrl;
    uint32_t* tile_flags;     // bit 0 (set-up only) = LAVA in the tile, bit 1 = a vent in the tile
    uint32_t* tile_mark[2];   // 2 (s + 1) + lava bit of the step s the tile is scheduled for, per parity
    int8_t* desc;             // D(n) of LAVA cells of scheduled tiles (computeDescent, LavaCA.hpp:551-566)
    uint32_t* tile_list[2];   // tiles of step t are tile_list[t & 1]
    unsigned long long* hist_active;
    unsigned long long* hist_changed;
    uint64_t ntiles;
    // z slab of a taller grid (vca_ca_set_slab): globalIndex = local index + gidx_base; the counts of
    // a step cover the owned layers [own_z0, own_z1) only; the caller decides the stop
    uint64_t gidx_base;
    int own_z0, own_z1;
    int slab;
};

// Read-only view of a CA handle's current planes (the MC domain and mobility are built from it).
struct CaView {
    const uint8_t* type;
    const uint16_t* solid;
    const uint16_t* arrival;
    int nx, ny, nz, P;
    cudaStream_t stream;
    int device;
};
vca_status ca_view(vca_ca* h, CaView* v);

}  // namespace vca

namespace vca {
// Device allocation sizes of a CA handle (a resident handle runs any space that fits them).
struct CaSizes {
    size_t plane_cells = 0;   // P * ny * nz
    uint64_t ntiles = 0;
    uint32_t chg_cap = 0;
    size_t cols = 0;          // nx * ny
    int hist = 0;             // steps of history
};
}  // namespace vca

struct vca_ca {
    vca::CaTensorMaps tmaps;  // first member: CUtensorMap needs 64-byte alignment
    vca::CaSizes cap;         // what the device buffers can hold
    int sms = 0, cand_per_sm = 0;
    int rules_per_sm[3] = {0, 0, 0};  // resident rules blocks per SM of each shape family
    size_t vent_cap = 0, seed_cap = 0;
    vca_ca_desc desc;
    vca::CaGeom geom;
    vca::CaTables tables_host;
    int device = 0;
    cudaStream_t stream = nullptr;
    int grid_blocks = 0;      // persistent grid of the tile kernels
    uint64_t ntiles = 0;
    size_t plane_cells = 0;   // P * ny * nz
    // device memory
    uint8_t* type[2] = {nullptr, nullptr};
    int32_t* flow[2] = {nullptr, nullptr};
    float* temp[2] = {nullptr, nullptr};
    uint16_t* solid[2] = {nullptr, nullptr};
    uint16_t* arrival[2] = {nullptr, nullptr};
    int8_t* drop_plane = nullptr;
    uint32_t* chg_list[2] = {nullptr, nullptr};
    uint32_t chg_cap = 0;
    uint32_t* cand_list = nullptr;
    int cand_blocks = 0;      // grid of the candidate pass
    int32_t* spill = nullptr;
    int4* vents = nullptr;
    int4* seeds_dev = nullptr;  // unique seed cells of place_seeds (grows only)
    unsigned long long* flow_sums = nullptr;  // 3 * (flows + 1) sums of vca_ca_flow_stats (grows only)
    size_t flow_sums_cap = 0;
    int vent_slots = 0;
    vca::CaCtrl* ctrl = nullptr;
    vca::CaCtrl* ctrl_host = nullptr;   // pinned, host-mapped mirror
    vca::CaCtrl* ctrl_host_dev = nullptr;  // its device address
    uint32_t* tile_flags = nullptr;
    uint32_t* tile_mark[2] = {nullptr, nullptr};
    int8_t* desc_plane = nullptr;
    uint32_t* tile_list[2] = {nullptr, nullptr};
    unsigned long long* hist_active = nullptr;
    unsigned long long* hist_changed = nullptr;
    int32_t* heights_dev = nullptr;  // nx*ny heights of the last apply_terrain
    bool has_terrain = false;
    bool seeded = false;
    // host mirror of the control state after the last sync
    int steps = 0;
    int stop = VCA_STOP_RUNNING;
    // timing
    cudaEvent_t ev_a = nullptr, ev_b = nullptr;
    double total_ms = 0.0;
    double rules_ms = 0.0;
    uint64_t rules_launches = 0;
    double drop_ms = 0.0, cand_ms = 0.0;  // profile mode: the other two kernels of a step
    uint64_t launches = 0;    // kernel launches issued
    int profile_kernels = 0;  // bracket each rules launch with events (set by VCA_PROFILE_KERNELS=1)
    std::vector<cudaEvent_t> prof_events;
    cudaGraphExec_t graph_exec = nullptr;   // kGraphSteps steps of launches
    vca::CaKernelArgs graph_args;            // the arguments, maps and grids graph_exec was captured with
    vca::CaTensorMaps graph_tm;
    int graph_grid = 0, graph_cand = 0;
    vca::CaCtrl* ctrl_ring = nullptr;       // pinned, host-mapped: two in-flight copies of the control block
    vca::CaCtrl* ctrl_ring_dev = nullptr;   // its device address
    cudaEvent_t ring_ev[2] = {nullptr, nullptr};
    vca_ca_batch* batch = nullptr;          // the batch stepping this handle, if any (vca_ca_batch_add)
    int batch_slot = -1;
    // z slab of a taller grid (vca_ca_set_slab); slab_z0 = global z of local layer 0
    bool slab = false;
    int slab_z0 = 0, own_z0 = 0, own_z1 = 0;
};

/*
 * vca.h -- C ABI of the B200 lava-CA and Potts-MC library (libvca.so).
 *
 * The reference engine has no plugin layer: its hot paths are the C++ classes LavaCA<Storage>
 * (engine/src/ca/LavaCA.hpp) and PottsMC (engine/src/mc/PottsMC.hpp), called directly by
 * Simulation::runWith and McStage::run.  This header is the boundary that replaces those two
 * classes: each entry point names the member function it stands in for.  Everything here is
 * plain C (pointers, sizes, enums); no C++ or CUDA types cross it.
 *
 * Ownership: device buffers belong to the handle; host arrays passed in or out belong to the
 * caller and are only read or written during the call.
 * Threading: a handle is used by one host thread at a time; each handle owns one CUDA stream.
 * Errors: every call returns a vca_status; vca_last_error() gives the message of the last failure
 * on the calling thread.  No exception crosses the boundary.
 * Layout of host planes: unframed, globalIndex order x + nx*(y + ny*z)
 * (engine/src/core/Types.hpp:95-100), as in ca_result.bin.
 */
#ifndef VCA_H
#define VCA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VCA_ABI_VERSION 2

typedef enum {
    VCA_OK = 0,
    VCA_ERR_ARG = 1,      /* invalid argument (maps to the reference's ConfigError, exit code 1) */
    VCA_ERR_STATE = 2,    /* call out of order, e.g. sweep before initialize */
    VCA_ERR_CUDA = 3,     /* CUDA runtime failure or no usable sm_100 device */
    VCA_ERR_NOMEM = 4,    /* device allocation failed */
    VCA_ERR_TIMEOUT = 5   /* a bounded device wait ran out (the context stays usable) */
} vca_status;

/* NeighborhoodKind (engine/src/core/Types.hpp:22) */
enum { VCA_NB_VON_NEUMANN = 0, VCA_NB_MOORE = 1, VCA_NB_PENTAGONAL = 2, VCA_NB_HEXAGONAL = 3 };
/* BoundaryKind (engine/src/core/Types.hpp:25) */
enum { VCA_BC_ABSORBING = 0, VCA_BC_PERIODIC = 1 };
/* CaMode (engine/src/core/Types.hpp:28) */
enum { VCA_MODE_LAVA = 0, VCA_MODE_CLASSIC = 1 };
/* Step schedule.  All give bit-identical results (grids, histories, stop step), like the
 * reference's ca.sweep = front / full (engine/src/ca/LavaCA.hpp:13-29):
 *   ACTIVE      -- tiles with no lava within one cell, and unchanged since the last step, are
 *                  skipped; a grid whose every tile has a rules block of its own runs DENSE;
 *   DENSE       -- every cell of the grid is read and written every step;
 *   ACTIVE_LIST -- ACTIVE with the tile list whatever the grid size. */
enum { VCA_SWEEP_ACTIVE = 0, VCA_SWEEP_DENSE = 1, VCA_SWEEP_ACTIVE_LIST = 2 };
/* StopReason (engine/src/ca/CaRules.hpp:108) */
enum { VCA_STOP_RUNNING = 0, VCA_STOP_NO_LAVA = 1, VCA_STOP_NO_AIR = 2, VCA_STOP_NO_CHANGE = 3,
       VCA_STOP_MAX_STEPS = 4 };
/* CellType (engine/src/core/Types.hpp:13-19) */
enum { VCA_AIR = 0, VCA_ROCK = 1, VCA_LAVA = 2, VCA_BASALT = 3, VCA_VOID = 255 };

typedef struct vca_ca vca_ca;
typedef struct vca_mc vca_mc;
typedef struct vca_ca_batch vca_ca_batch;

/* ------------------------------------------------------------------------------------------
 * Lava cellular automaton -- replaces LavaCA<Storage> (engine/src/ca/LavaCA.hpp:80-271)
 * ---------------------------------------------------------------------------------------- */

/* Dims + CaParams (engine/src/ca/CaRules.hpp:93-105) + Neighborhood kind + Boundary kind.
 * Temperatures are the float values the reference casts from the config
 * (Simulation::caParams, engine/src/app/Simulation.cpp:122-136). */
typedef struct {
    int nx, ny, nz;
    int neighborhood;          /* VCA_NB_* */
    int boundary;              /* VCA_BC_* */
    int mode;                  /* VCA_MODE_* */
    uint64_t seed;             /* rngSeed */
    int max_steps;             /* ca.maxSteps, 0..65535 */
    int eruption_steps;        /* vents.eruptionSteps */
    float erupt_temp;          /* vents.eruptTemp */
    float solidus_temp;        /* ca.solidusTemp */
    float cooling_ambient;     /* ca.coolingAmbient */
    float cooling_lateral;     /* ca.coolingLateral */
    float cooling_fall;        /* ca.coolingFall */
    int ponding;               /* ca.ponding */
    int sweep;                 /* VCA_SWEEP_* */
    int device;                /* CUDA device ordinal */
    /* Launch shape of the step kernels (no counterpart in the reference; results do not depend on
     * it).  Tiles are 64 x tile_y x tile_z cells with tile_y * tile_z = 16: 4 x 4, 2 x 8, 8 x 2,
     * 1 x 16 or 16 x 1 in 3D, 1 x 16 for a 2D x-z section, 16 x 1 for an x-y plane; 0 x 0 picks the
     * default (4 x 4 in 3D).  rules_blocks_per_sm caps the resident blocks of the rules pass per SM
     * (0: as many as fit).  volcano_ca_mc_b200/tuner.py picks them per grid shape. */
    int tile_y, tile_z;
    int rules_blocks_per_sm;
} vca_ca_desc;

/* Vent (engine/src/terrain/VentPlacer.hpp:26-31). */
typedef struct {
    int x, y, z;
    int32_t flow_id;
} vca_vent;

typedef struct {
    int steps;                 /* LavaCA::steps() */
    int stop_reason;           /* LavaCA::stopReason(), VCA_STOP_* */
    uint64_t lava_cells;       /* LAVA cells now (classic: grains) */
    uint64_t air_cells;        /* AIR cells now */
    uint64_t tiles_total;      /* tiles of the grid */
    uint64_t tiles_processed;  /* tile visits summed over all steps (DENSE: steps x tiles) */
    uint64_t cells_per_tile;   /* cells one tile covers */
    uint64_t kernel_launches;  /* CUDA kernel launches issued by this handle so far */
} vca_ca_info;

/* LavaCA ctor (LavaCA.hpp:84-144): all cells AIR, buffers on the device. */
vca_status vca_ca_create(const vca_ca_desc* desc, vca_ca** out);
/* Device bytes a handle of this description allocates (the admission figure of a job server).
 * No counterpart in the reference. */
vca_status vca_ca_footprint(const vca_ca_desc* desc, uint64_t* bytes);
/* Give a handle another space and parameters (any description whose sizes fit the handle's device
 * memory: vca_ca_footprint of it <= that of the creating one, same device), in the state of a new
 * handle.  Allocates nothing; lets a server keep resident handles for jobs of varying size.
 * VCA_ERR_ARG when it does not fit.  No counterpart in the reference. */
vca_status vca_ca_reconfigure(vca_ca* ca, const vca_ca_desc* desc);
/* Back to the state of a new handle (all cells AIR, no terrain, no vents, step 0) without
 * freeing or allocating device memory, so that one resident handle can run job after job of the
 * same dimensions.  No counterpart in the reference (it builds a new LavaCA per run). */
vca_status vca_ca_reset(vca_ca* ca);
/* LavaCA::applyTerrain (LavaCA.hpp:185-211): ROCK for z < h(x,y); spill levels by priority flood
 * (TerrainGenerator::fillDepressions, engine/src/terrain/TerrainGenerator.cpp:86-161).
 * heights: nx*ny values, x fastest.  Lava mode only. */
vca_status vca_ca_apply_terrain(vca_ca* ca, const int32_t* heights);
/* LavaCA::placeSeeds (LavaCA.hpp:215-227): vents become LAVA {flowId, eruptTemp (lava) or 0
 * (classic)}; sets the initial stop state (countInitialState, LavaCA.hpp:1252-1280). */
vca_status vca_ca_place_seeds(vca_ca* ca, const vca_vent* vents, int count);
/* LavaCA::step (LavaCA.hpp:230-247); *running = !finished() afterwards. */
vca_status vca_ca_step(vca_ca* ca, int* running);
/* LavaCA::run (LavaCA.hpp:253-256): steps until the stop rule holds. */
vca_status vca_ca_run(vca_ca* ca);
/* steps(), stopReason() and counters (LavaCA.hpp:258-265). */
vca_status vca_ca_get_info(vca_ca* ca, vca_ca_info* out);
/* activeHistory() / changedHistory() (LavaCA.hpp:263-265): copies min(capacity, steps) entries;
 * either pointer may be NULL. */
vca_status vca_ca_history(vca_ca* ca, uint64_t* active, uint64_t* changed, int capacity, int* count);
/* LavaCA::result() (LavaCA.hpp:271): current planes to host, unframed globalIndex order;
 * any pointer may be NULL to skip that plane. */
vca_status vca_ca_download(vca_ca* ca, uint8_t* type, int32_t* flow_id, float* temp, uint16_t* solid_step,
                           uint16_t* arrival_step);
/* Replace the whole state (test and resume hook; the reference reaches the same state through
 * applyTerrain + placeSeeds + steps).  spill may be NULL (no terrain); vents give the isVent table
 * (LavaCA.hpp:335-341) and are not written into the grid; steps_done is the step counter t. */
vca_status vca_ca_set_state(vca_ca* ca, const uint8_t* type, const int32_t* flow_id, const float* temp,
                            const uint16_t* solid_step, const uint16_t* arrival_step, const int32_t* spill,
                            const vca_vent* vents, int vent_count, int steps_done);
/* Spill levels in use (LavaCA::spill_, set by applyTerrain, LavaCA.hpp:205; read by spillAt, 383):
 * nx*ny values, x fastest; returns VCA_ERR_STATE when there is no terrain. */
vca_status vca_ca_get_spill(vca_ca* ca, int32_t* spill);
/* The per-flow sums of Simulation::flowSums (engine/src/app/Simulation.cpp:408-466) over the current
 * state, on the device: for flowId f in 1..flows, lava[f] and basalt[f] count the LAVA and BASALT
 * cells of flow f and reach2[f] is the largest (x - vx)^2 + (y - vy)^2 over them, (vx, vy) the
 * vent of flow f as given to vca_ca_place_seeds (0 for a flow without cells).  Each array holds
 * flows + 1 entries; entry 0 is set to 0.  The reference's maxReach is the largest hypot over the
 * cells rounded to 0.01, which equals sqrt(reach2[f]) rounded to 0.01. */
vca_status vca_ca_flow_stats(vca_ca* ca, int flows, uint64_t* lava, uint64_t* basalt, uint64_t* reach2);
/* ------------------------------------------------------------------------------------------
 * z slabs of one grid over several GPUs, as the reference's strips (engine/src/parallel/Strip.hpp:1-25,
 * engine/src/mpi/MpiSimulation.cpp): each GPU holds the layers it owns plus 17 halo layers below and
 * 1 above (drop depths look 17 cells down), steps them, and after every step the caller copies the
 * owned boundary layers into its neighbours' halo layers and sums the step's counts over all slabs
 * for the stop rule (finishStep, LavaCA.hpp:1206-1229; LavaCA.hpp:1207-1211 sums the same three
 * counters over the strips).  volcano_ca_mc_b200/slabs.py drives it over torch.distributed.
 * ---------------------------------------------------------------------------------------- */
/* Makes a new lava handle the slab whose layer 0 is global layer z_offset; it owns its layers
 * [own_z0, own_z1).  Call before vca_ca_apply_terrain (which then takes the whole grid's nx*ny
 * heights) and vca_ca_place_seeds (vents in this slab's local coordinates).  A slab steps with the
 * DENSE schedule, hashes global indices, counts only its owned layers and never stops by itself
 * except at max_steps. */
vca_status vca_ca_set_slab(vca_ca* ca, int z_offset, int own_z0, int own_z1);
/* One step of a slab; active / changed get this step's counts over the owned layers. */
vca_status vca_ca_slab_step(vca_ca* ca, uint64_t* active, uint64_t* changed);
/* Sets the stop state the caller decided from the counts of all slabs (VCA_STOP_*). */
vca_status vca_ca_slab_stop(vca_ca* ca, int stop_reason);
/* Device pointers of layer 0 of the current planes (the next step reads them) and the cells of one
 * layer (rows are pitched: layer z starts at z * layer_cells); any pointer may be NULL. */
vca_status vca_ca_layers(vca_ca* ca, void** type, void** flow_id, void** temp, void** solid_step,
                         void** arrival_step, uint64_t* layer_cells);
/* Halo messages between slabs: copies `types` type layers from local layer z0 and, when full >= 0,
 * the flowId, temperature, solidStep and arrivalStep of local layer `full` between the current
 * planes and a buffer of (types + 12 * (full >= 0)) * layer_cells bytes (device, pinned or pageable
 * memory: the copy kind is inferred), in that order.  Unpacking writes the layers back. */
vca_status vca_ca_pack_layers(vca_ca* ca, int z0, int types, int full, void* buf);
vca_status vca_ca_unpack_layers(vca_ca* ca, int z0, int types, int full, const void* buf);
/* Device time of the CA steps so far [ms] (CUDA events around the step launches) and the average
 * duration of one launch of the rules kernel [ms] over the last vca_ca_run / vca_ca_step calls. */
vca_status vca_ca_timing(vca_ca* ca, double* total_ms, double* rules_kernel_ms, uint64_t* rules_launches);
/* With VCA_PROFILE_KERNELS=1 in the environment when the handle was created, runs launch step by
 * step with CUDA events around each kernel: the average device time [ms] of the drop-depth, rules
 * and candidate kernels of a step, and the steps measured.  No counterpart in the reference. */
vca_status vca_ca_kernel_times(vca_ca* ca, double* drop_ms, double* rules_ms, double* cand_ms, uint64_t* steps);
/* ~LavaCA: frees the handle's device memory, stream and graph. */
void vca_ca_destroy(vca_ca* ca);

/* ------------------------------------------------------------------------------------------
 * Batched stepping of many lava CA grids.  No counterpart in the reference: its batch runner
 * (engine/src/app/Batch.cpp:186-246) starts one engine process per config, one after another, and
 * each LavaCA::run (LavaCA.hpp:253-256) steps one grid.  A batch steps every member grid -- of any
 * size, 2D or 3D, neighbourhood, boundary, seed or schedule -- with three launches per step for all
 * of them together (each block of a launch works on one member), captured as a CUDA graph of 16
 * steps.  Each member ends exactly as it would alone (same planes, histories and stop step).
 * ---------------------------------------------------------------------------------------- */

/* A batch of at most max_members grids on a device (max_members is also capped by the blocks of
 * one launch, a few hundred). */
vca_status vca_ca_batch_create(int device, int max_members, vca_ca_batch** out);
/* Adds a handle whose state is set up (place_seeds or set_state done).  While it is a member, every
 * call on the handle except vca_ca_destroy returns VCA_ERR_STATE; it leaves the batch when its stop
 * rule holds (vca_ca_batch_advance reports it) or by vca_ca_batch_remove.  VCA_ERR_ARG when the
 * batch is full or the handle lives on another device or in another batch. */
vca_status vca_ca_batch_add(vca_ca_batch* b, vca_ca* member);
/* Steps the members: launches up to max_graphs graphs of 16 steps, reading each graph's stop flags
 * while the next one runs, and returns once some member has stopped (or all graphs are done, or no
 * member is left).  The members that stopped leave the batch and are written to finished[0..*count)
 * (at most capacity; the others stay queued for the next call); running gets the members still
 * stepping.  A member that had stopped before it was added is reported by the next call. */
vca_status vca_ca_batch_advance(vca_ca_batch* b, int max_graphs, vca_ca** finished, int capacity, int* count,
                                int* running);
/* Takes a member out of the batch now, whatever its state (its last step completes first). */
vca_status vca_ca_batch_remove(vca_ca_batch* b, vca_ca* member);
/* Launch counts: graphs launched, kernel launches issued, members now. */
vca_status vca_ca_batch_info(vca_ca_batch* b, uint64_t* graphs, uint64_t* launches, int* members);
/* Detaches every member (as by vca_ca_batch_remove) and frees the batch. */
void vca_ca_batch_destroy(vca_ca_batch* b);

/* ------------------------------------------------------------------------------------------
 * Potts Monte Carlo, checkerboard update -- replaces PottsMC (engine/src/mc/PottsMC.hpp:52-152)
 * with mc.update = "checkerboard".  mc.update = "random" is sequential by definition
 * (engine/src/mc/McRules.hpp:30-32) and is not offered.
 * ---------------------------------------------------------------------------------------- */

/* PottsMC ctor arguments (PottsMC.cpp:14-46): Dims, McParams (engine/src/mc/McRules.hpp:80-85),
 * Neighborhood kind and Boundary.  domain_full selects the boundary mode: 0 = basalt (lava
 * boundary: z never periodic), 1 = full (classic boundary: all axes periodic when periodic)
 * (McStage::run, engine/src/app/McStage.cpp:104-106). */
typedef struct {
    int nx, ny, nz;
    int neighborhood;
    int boundary;
    int domain_full;
    uint64_t seed;
    int Q;
    double J;
    double kT;
    int device;
} vca_mc_desc;

typedef struct {
    int sweeps;                /* sweepsDone() */
    int colors;                /* colorCount() */
    uint64_t domain_cells;     /* domainCells() */
    uint64_t attempts;         /* attempts() -- trials not skipped by mobility */
    uint64_t accepted;         /* accepted() */
    uint64_t uphill;           /* acceptedUphill() */
    uint64_t kernel_launches;  /* CUDA kernel launches issued by this handle so far */
} vca_mc_info;

vca_status vca_mc_create(const vca_mc_desc* desc, vca_mc** out);
/* Device bytes an MC handle of this description can come to hold (all per-cell buffers).
 * No counterpart in the reference. */
vca_status vca_mc_footprint(const vca_mc_desc* desc, uint64_t* bytes);
/* Another space / parameters on this handle (no more cells than it was created for, same device):
 * orientations cleared, domain and mobility unset.  Allocates nothing.  No counterpart in the
 * reference. */
vca_status vca_mc_reconfigure(vca_mc* mc, const vca_mc_desc* desc);
/* setDomain / setDomainAll (PottsMC.cpp:61-83): in_domain is N bytes, or NULL for all cells. */
vca_status vca_mc_set_domain(vca_mc* mc, const uint8_t* in_domain);
/* setMobility (PottsMC.cpp:85-102): N floats, or NULL to switch mobility off. */
vca_status vca_mc_set_mobility(vca_mc* mc, const float* mobility);
/* CoolingMobility::basaltDomain (engine/src/mc/CoolingMobility.cpp:8-14) of the CA handle's
 * current state, computed on the device without a host round trip. */
vca_status vca_mc_set_domain_from_ca(vca_mc* mc, vca_ca* ca);
/* CoolingMobility::fromCooling (CoolingMobility.cpp:16-83) of the CA handle's state, on the device.
 * If use_in_dynamics is 0 the values are kept only for vca_mc_mobility() (the reference computes
 * them for statistics even when mc.mobilityFromCooling is false). */
vca_status vca_mc_set_mobility_from_ca(vca_mc* mc, vca_ca* ca, double mobility_min, int use_in_dynamics);
/* Current mobility values (PottsMC::mobility_, set by setMobility, PottsMC.cpp:85-102): N floats, 0
 * outside the domain; VCA_ERR_STATE if none were set. */
vca_status vca_mc_mobility(vca_mc* mc, float* out);
/* PottsMC::initialize with setCheckerboard(true) (PottsMC.cpp:104-224). */
vca_status vca_mc_initialize(vca_mc* mc);
/* count x PottsMC::sweep (PottsMC.cpp:516-533); accepted (may be NULL) gets the accepted
 * changes of these sweeps. */
vca_status vca_mc_sweep(vca_mc* mc, int count, uint64_t* accepted);
/* domainCells(), sweepsDone(), attempts(), accepted(), acceptedUphill(), colorCount()
 * (PottsMC.hpp:102-106, 133). */
vca_status vca_mc_get_info(vca_mc* mc, vca_mc_info* out);
/* PottsMC::totalEnergy (PottsMC.cpp:590-664). */
vca_status vca_mc_energy(vca_mc* mc, double* energy);
/* Grain statistics of the current orientations (labelGrains, engine/src/mc/Grains.cpp:33-150, and
 * the majority classes of McStage, engine/src/app/McStage.cpp:38-66): grains are connected sets of
 * one orientation, Moore (moore != 0) or von Neumann connectivity, periodic axes as the sweep's.
 * The high / low split uses the mobility values held by the handle (vca_mc_set_mobility*,
 * vca_mc_set_mobility_from_ca): a grain is high when at least half of its cells have mobility >=
 * mobility_threshold; without mobility values every grain is low. */
typedef struct {
    uint64_t grains;            /* grains */
    uint64_t cells;             /* cells in grains (the domain) */
    uint64_t largest;           /* cells of the largest grain */
    uint64_t high_cells;        /* domain cells with mobility >= threshold */
    uint64_t high_grains;       /* grains of the high class, their cells, the largest */
    uint64_t high_grain_cells;
    uint64_t high_largest;
    uint64_t low_grains;        /* the same for the low class */
    uint64_t low_grain_cells;
    uint64_t low_largest;
} vca_mc_grain_stats;
vca_status vca_mc_grains(vca_mc* mc, int moore, double mobility_threshold, vca_mc_grain_stats* out);
/* setMobility with a choice: the values are kept for vca_mc_grains' classes and, when
 * use_in_dynamics != 0, also gate the trials (vca_mc_set_mobility is use_in_dynamics = 1). */
vca_status vca_mc_set_mobility_values(vca_mc* mc, const float* mobility, int use_in_dynamics);
/* PottsMC::crystals (PottsMC.cpp:666-697): N int32, 0 outside the domain. */
vca_status vca_mc_crystals(vca_mc* mc, int32_t* out);
/* Overwrite all orientations (setOrientation for every cell, PottsMC.cpp:566-576); values
 * outside the domain must be 0 and inside 1..Q. */
vca_status vca_mc_set_spins(vca_mc* mc, const int32_t* spins);
/* Device time of the sweeps so far [ms] and of one colour-pass launch on average [ms]. */
vca_status vca_mc_timing(vca_mc* mc, double* total_ms, double* color_kernel_ms, uint64_t* color_launches);
/* z slabs of the MC stage (the reference's strips exchange one halo layer after every colour,
 * engine/src/mc/PottsMC.cpp:451-460): the handle holds the owned layers and one halo layer on each
 * side, its domain lists only owned cells, and its layer 0 is global layer z_offset (hashRand takes
 * global indices, colours follow the global z).  Set before vca_mc_initialize; the z axis must not be
 * periodic.  The caller sweeps colour by colour (vca_mc_color_pass; the last colour of a sweep ends
 * the MCS) and copies the halo layers between slabs after each colour. */
vca_status vca_mc_set_slab(vca_mc* mc, int z_offset);
vca_status vca_mc_color_pass(vca_mc* mc, int color);
/* Orientations of `layers` layers from local layer z0 to / from a buffer of layers * nx * ny int32
 * (any memory the device can address; the copy kind is inferred). */
vca_status vca_mc_pack_spins(vca_mc* mc, int z0, int layers, void* buf);
vca_status vca_mc_unpack_spins(vca_mc* mc, int z0, int layers, const void* buf);
/* ~PottsMC: frees the handle's device memory and stream. */
void vca_mc_destroy(vca_mc* mc);

/* Potts energy (the quantity of vca_mc_energy) of an nx*ny*nz int32 spin grid that is already in
 * the caller's device memory, written to the caller's device double *energy on the given
 * cudaStream_t (NULL: the legacy default stream).  No counterpart in the reference: it exists for
 * callers that own all device memory and cannot let a library allocate -- a process whose memory
 * pool has reserved the device, or a pipeline that must not take the device-wide synchronisation
 * of cudaMalloc/cudaFree between its launches.  It allocates nothing: its scratch (per-block sums
 * and a counter) is a fixed static device array of 512 KiB + 256 B, so grids above 2^28 cells are
 * rejected with VCA_ERR_ARG.  Spins: 0 outside the domain, 1..Q inside; neighborhood, boundary,
 * domain_full and seed as in vca_mc_desc; mcs = sweeps done (the neighbourhood variant of
 * pentagonal/hexagonal cells at that MCS).  Both pointers must be device memory of the current
 * device, and the stream must belong to that device (VCA_ERR_ARG otherwise).  Outside stream
 * capture every call looks up the scratch's address in the device's current context (a context
 * made again after cudaDeviceReset is followed); during a capture the address of the last call
 * outside capture is used, so make the first call on each device before any stream capture
 * (VCA_ERR_STATE otherwise).  The call returns once the work is queued.  Every call uses the same
 * scratch and the ticket is cleared on the stream before each launch; calls that overlap on one
 * device race on the shared scratch: order them (one stream, or events). */
vca_status vca_mc_energy_noalloc(const int32_t* spins, int nx, int ny, int nz, int neighborhood, int boundary,
                                 int domain_full, uint64_t seed, int mcs, double J, double* energy, void* stream);

/* ------------------------------------------------------------------------------------------ */
/* Message of the last failing call on this host thread (the reference reports errors as C++
 * exceptions; no counterpart). */
const char* vca_last_error(void);
/* ABI version and build string ("vca <abi> sm_100a ..."); no counterpart in the reference. */
const char* vca_version(void);

#ifdef __cplusplus
}
#endif
#endif

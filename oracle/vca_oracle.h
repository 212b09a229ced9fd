/*
 * vca_oracle.h -- CPU restatement of the lava-CA step and the Potts checkerboard sweep.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA path is compared with; it is
 * never linked into the product library (libvca.so) or the engine, and nothing on the product
 * path may call it.  It is pinned against the reference engine's own outputs (step snapshots,
 * final ca_result.bin / mc_result.bin, stats.json histories) by tests/test_oracle_pin.py.
 *
 * Planes are unframed, in the reference's globalIndex order x + nx*(y + ny*z)
 * (engine/src/core/Types.hpp:95-100).  Boundaries are realised by coordinate wrap (periodic)
 * or a VOID answer (absorbing), which is what the reference's 1-cell frame stores
 * (engine/src/core/Boundary.hpp:75-131).
 */
#ifndef VCA_ORACLE_H
#define VCA_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* --- hash (engine/src/core/Rng.hpp:35-74) --- */
uint64_t vo_splitmix64(uint64_t x);
uint64_t vo_hash_rand(uint64_t seed, uint64_t step, uint64_t idx, uint64_t salt);
uint64_t vo_hash_prefix(uint64_t seed, uint64_t step);
uint64_t vo_hash_index(uint64_t prefix, uint64_t idx);
uint64_t vo_hash_salt(uint64_t index_hash, uint64_t salt);

/* --- neighbourhood tables (engine/src/core/Neighborhood.cpp:55-119) ---
 * Writes variants into off[v][k][3] (v < 6, k < 26); returns the variant count, fills
 * counts[v].  kind: 0 von_neumann, 1 moore, 2 pentagonal, 3 hexagonal.  -1 if unsupported. */
int vo_nb_build(int kind, int nx, int ny, int nz, int off[6][26][3], int counts[6]);

/* --- spill levels by priority flood (engine/src/terrain/TerrainGenerator.cpp:86-161) --- */
void vo_fill_depressions(const int32_t* height, int nx, int ny, int periodic_x, int periodic_y,
                         int32_t* filled);

typedef struct {
    int nx, ny, nz;
    int neighborhood;     /* 0..3 as above */
    int periodic;         /* boundary: 0 absorbing, 1 periodic */
    int classic;          /* ca.mode: 0 lava, 1 classic */
    uint64_t seed;
    int max_steps;
    int eruption_steps;
    float erupt_temp, solidus_temp, cooling_ambient, cooling_lateral, cooling_fall;
    int ponding;
} vo_ca_params;

/* One synchronous CA step t (t = steps already done), cur -> next.  spill may be NULL (no
 * terrain).  vent_xyz[3*f .. 3*f+2] is the vent cell of flowId f (f < vent_slots; -1 = none).
 * counts[0] = active (LAVA after step; classic: grains), counts[1] = AIR after, counts[2] = changed.
 * Follows LavaCA::stepLava / updateLava / updateClassic (engine/src/ca/LavaCA.hpp:577-588, 1109-1201). */
void vo_ca_step(const vo_ca_params* p, int t, const int32_t* spill, const int32_t* vent_xyz, int vent_slots,
                const uint8_t* type, const int32_t* flow, const float* temp, const uint16_t* solid,
                const uint16_t* arrival, uint8_t* ntype, int32_t* nflow, float* ntemp, uint16_t* nsolid,
                uint16_t* narrival, uint64_t counts[3]);

/* Stop rule after a step (LavaCA::finishStep, LavaCA.hpp:1206-1229): 0 running, 1 no lava,
 * 2 no air, 3 no change, 4 max steps. */
int vo_ca_stop_after(const vo_ca_params* p, int steps_done, const uint64_t counts[3]);
/* vo_ca_step on a strip of z layers of a taller grid (the reference's MPI strips,
 * engine/src/parallel/Strip.hpp:1-25): global index of local cell 0 = gidx_base (for hashRand),
 * counts over layers [own_z0, own_z1) only; spill levels shifted to local z by the caller. */
void vo_ca_step_strip(const vo_ca_params* p, int t, uint64_t gidx_base, int own_z0, int own_z1, const int32_t* spill,
                      const int32_t* vent_xyz, int vent_slots, const uint8_t* type, const int32_t* flow,
                      const float* temp, const uint16_t* solid, const uint16_t* arrival, uint8_t* ntype,
                      int32_t* nflow, float* ntemp, uint16_t* nsolid, uint16_t* narrival, uint64_t counts[3]);

typedef struct {
    int nx, ny, nz;
    int neighborhood;
    int periodic[3];      /* per axis, already reduced for size-1 axes (PottsMC.cpp:18) */
    uint64_t seed;
    int Q;
    double J, kT;
} vo_mc_params;

/* Initial orientations (PottsMC::initialize, PottsMC.cpp:104-143): spin = 1 + hashRand(seed,0,g,McInit)%Q
 * for domain cells (domain != 0), else 0. */
void vo_mc_init(const vo_mc_params* p, const uint8_t* domain, int32_t* spin);

/* Colour of a cell and the colour count (PottsMC.cpp:145-224). */
int vo_mc_colors(const vo_mc_params* p);
int vo_mc_color_of(const vo_mc_params* p, int x, int y, int z);

/* One checkerboard MCS number t (t = sweeps done) in place.  mobility may be NULL.
 * out[0] attempts, out[1] accepted, out[2] uphill are incremented.
 * Follows PottsMC::sweepColors / colorTrials (PottsMC.cpp:394-514). */
void vo_mc_sweep(const vo_mc_params* p, int t, const uint8_t* domain, const float* mobility, int32_t* spin,
                 uint64_t out[3]);

/* Energy after t sweeps (PottsMC::totalEnergy, PottsMC.cpp:590-664). */
double vo_mc_energy(const vo_mc_params* p, int t, const int32_t* spin);
/* One colour of MCS t on a strip of z layers of a taller grid (PottsMC.cpp:451-460): global index of
 * local cell 0 = gidx_base, global z = local z + zoff. */
void vo_mc_color_strip(const vo_mc_params* p, int t, int col, uint64_t gidx_base, int zoff, const uint8_t* domain,
                       const float* mobility, int32_t* spin, uint64_t out[3]);

#ifdef __cplusplus
}
#endif
#endif

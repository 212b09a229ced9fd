/*
 * vca_oracle.c -- CPU restatement of the reference's lava-CA step and Potts checkerboard sweep.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see vca_oracle.h).  Plain C, one
 * thread, written for clarity, not speed.  Every function cites the reference lines it restates;
 * paths are relative to the reference project root.
 */
#include "vca_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------------------------
 * Hash (engine/src/core/Rng.hpp)
 * ------------------------------------------------------------------------------------------- */
enum { CELL_AIR = 0, CELL_ROCK = 1, CELL_LAVA = 2, CELL_BASALT = 3, CELL_VOID = 255 };

/* Salts: engine/src/core/Rng.hpp:22-31. */
#define SALT_NEIGHBORHOOD 0x4E45494748424F52ULL
#define SALT_TIEBREAK 0x5449455F42524B31ULL
#define SALT_MC_INIT 0x4D43494E49544F52ULL
#define SALT_MC_MOBILITY 0x4D434D4F42494C49ULL
#define SALT_MC_ORIENT 0x4D434F5249454E54ULL
#define SALT_MC_ACCEPT 0x4D43414343455054ULL

/* Rng.hpp:35-40 */
uint64_t vo_splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
/* Rng.hpp:46-52 */
uint64_t vo_hash_rand(uint64_t seed, uint64_t step, uint64_t idx, uint64_t salt) {
    uint64_t h = vo_splitmix64(seed ^ 0xA0761D6478BD642FULL);
    h = vo_splitmix64(h ^ step);
    h = vo_splitmix64(h ^ idx);
    return vo_splitmix64(h ^ salt);
}
/* Rng.hpp:66-72 */
uint64_t vo_hash_prefix(uint64_t seed, uint64_t step) {
    return vo_splitmix64(vo_splitmix64(seed ^ 0xA0761D6478BD642FULL) ^ step);
}
uint64_t vo_hash_index(uint64_t prefix, uint64_t idx) { return vo_splitmix64(prefix ^ idx); }
uint64_t vo_hash_salt(uint64_t h, uint64_t salt) { return vo_splitmix64(h ^ salt); }

/* Rng.hpp:74 — toUniform(r) = (r >> 11) * 2^-53 (exact in double). */
static double to_uniform(uint64_t r) { return (double)(r >> 11) * (1.0 / 9007199254740992.0); }

/* ---------------------------------------------------------------------------------------------
 * Neighbourhoods (engine/src/core/Neighborhood.cpp:18-119)
 * ------------------------------------------------------------------------------------------- */
static int keep2d(int kind, int variant, int u, int v) {
    switch (kind) {
        case 0: return abs(u) + abs(v) == 1;
        case 1: return 1;
        case 2: /* Neighborhood.cpp:94-98 */
            if (variant == 0) return u != -1;
            if (variant == 1) return u != 1;
            if (variant == 2) return v != -1;
            return v != 1;
        case 3: /* Neighborhood.cpp:100-107 */
            if (variant == 0) return !((u == -1 && v == -1) || (u == 1 && v == 1));
            return !((u == -1 && v == 1) || (u == 1 && v == -1));
    }
    return 0;
}
static int keep3d(int kind, int variant, int dx, int dy, int dz) {
    switch (kind) {
        case 0: return abs(dx) + abs(dy) + abs(dz) == 1;
        case 1: return 1;
        case 2: /* Neighborhood.cpp:116-123 */
            switch (variant) {
                case 0: return dx != -1;
                case 1: return dx != 1;
                case 2: return dy != -1;
                case 3: return dy != 1;
                case 4: return dz != -1;
                default: return dz != 1;
            }
    }
    return 0;
}

int vo_nb_build(int kind, int nx, int ny, int nz, int off[6][26][3], int counts[6]) {
    const int sizes[3] = {nx, ny, nz};
    int axes = 0, plane[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) {
        if (sizes[a] > 1) plane[axes++] = a;
    }
    if (axes < 2) return -1;
    int variants;
    if (axes == 2) {
        variants = (kind == 2) ? 4 : (kind == 3) ? 2 : 1;
        for (int var = 0; var < variants; ++var) {
            int k = 0;
            /* build2D: v outer, u inner (Neighborhood.cpp:18-33) */
            for (int v = -1; v <= 1; ++v) {
                for (int u = -1; u <= 1; ++u) {
                    if ((u == 0 && v == 0) || !keep2d(kind, var, u, v)) continue;
                    int d[3] = {0, 0, 0};
                    d[plane[0]] = u;
                    d[plane[1]] = v;
                    off[var][k][0] = d[0];
                    off[var][k][1] = d[1];
                    off[var][k][2] = d[2];
                    ++k;
                }
            }
            counts[var] = k;
        }
    } else {
        if (kind == 3) return -1; /* hexagonal is 2D-only (Neighborhood.cpp:125-127) */
        variants = (kind == 2) ? 6 : 1;
        for (int var = 0; var < variants; ++var) {
            int k = 0;
            /* build3D: dz, dy, dx (Neighborhood.cpp:36-48) */
            for (int dz = -1; dz <= 1; ++dz)
                for (int dy = -1; dy <= 1; ++dy)
                    for (int dx = -1; dx <= 1; ++dx) {
                        if ((dx == 0 && dy == 0 && dz == 0) || !keep3d(kind, var, dx, dy, dz)) continue;
                        off[var][k][0] = dx;
                        off[var][k][1] = dy;
                        off[var][k][2] = dz;
                        ++k;
                    }
            counts[var] = k;
        }
    }
    return variants;
}

/* ---------------------------------------------------------------------------------------------
 * Priority flood (engine/src/terrain/TerrainGenerator.cpp:86-161).  A binary min-heap on
 * (level, column index), like std::priority_queue<pair, ..., greater<pair>>.
 * ------------------------------------------------------------------------------------------- */
typedef struct { int32_t level; int64_t idx; } heap_item;
static int item_less(heap_item a, heap_item b) { return a.level < b.level || (a.level == b.level && a.idx < b.idx); }
static void heap_push(heap_item* h, int64_t* n, heap_item it) {
    int64_t i = (*n)++;
    h[i] = it;
    while (i > 0) {
        int64_t p = (i - 1) / 2;
        if (!item_less(h[i], h[p])) break;
        heap_item t = h[i]; h[i] = h[p]; h[p] = t;
        i = p;
    }
}
static heap_item heap_pop(heap_item* h, int64_t* n) {
    heap_item top = h[0];
    h[0] = h[--(*n)];
    int64_t i = 0;
    for (;;) {
        int64_t l = 2 * i + 1, r = l + 1, m = i;
        if (l < *n && item_less(h[l], h[m])) m = l;
        if (r < *n && item_less(h[r], h[m])) m = r;
        if (m == i) break;
        heap_item t = h[i]; h[i] = h[m]; h[m] = t;
        i = m;
    }
    return top;
}

void vo_fill_depressions(const int32_t* height, int nx, int ny, int periodic_x, int periodic_y, int32_t* filled) {
    const int64_t n = (int64_t)nx * ny;
    char* closed = (char*)calloc((size_t)n, 1);
    heap_item* heap = (heap_item*)malloc(sizeof(heap_item) * (size_t)(n + 1));
    int64_t hn = 0;
    memcpy(filled, height, sizeof(int32_t) * (size_t)n);
    /* Outlets: columns on a non-periodic edge (TerrainGenerator.cpp:110-120). */
    for (int y = 0; y < ny; ++y)
        for (int x = 0; x < nx; ++x) {
            const int edge_x = !periodic_x && nx > 1 && (x == 0 || x == nx - 1);
            const int edge_y = !periodic_y && ny > 1 && (y == 0 || y == ny - 1);
            const int64_t i = x + (int64_t)nx * y;
            if ((edge_x || edge_y) && !closed[i]) {
                closed[i] = 1;
                heap_item it = {height[i], i};
                heap_push(heap, &hn, it);
            }
        }
    if (hn == 0 && n > 0) {
        /* Fully wrapped: the lowest columns drain (TerrainGenerator.cpp:121-131). */
        int32_t lowest = height[0];
        for (int64_t i = 1; i < n; ++i)
            if (height[i] < lowest) lowest = height[i];
        for (int64_t i = 0; i < n; ++i)
            if (height[i] == lowest && !closed[i]) {
                closed[i] = 1;
                heap_item it = {height[i], i};
                heap_push(heap, &hn, it);
            }
    }
    static const int ddx[4] = {-1, 1, 0, 0};
    static const int ddy[4] = {0, 0, -1, 1};
    while (hn > 0) {
        heap_item it = heap_pop(heap, &hn);
        const int x = (int)(it.idx % nx), y = (int)(it.idx / nx);
        for (int k = 0; k < 4; ++k) {
            int sx = x + ddx[k], sy = y + ddy[k];
            if (sx < 0 || sx >= nx) {
                if (!periodic_x || nx == 1) continue;
                sx = (sx + nx) % nx;
            }
            if (sy < 0 || sy >= ny) {
                if (!periodic_y || ny == 1) continue;
                sy = (sy + ny) % ny;
            }
            const int64_t j = sx + (int64_t)nx * sy;
            if (closed[j]) continue;
            closed[j] = 1;
            filled[j] = height[j] > it.level ? height[j] : it.level;
            heap_item nxt = {filled[j], j};
            heap_push(heap, &hn, nxt);
        }
    }
    free(heap);
    free(closed);
}

/* ---------------------------------------------------------------------------------------------
 * Lava CA (engine/src/ca/LavaCA.hpp, engine/src/ca/CaRules.hpp)
 * ------------------------------------------------------------------------------------------- */
typedef struct {
    const vo_ca_params* p;
    int per[3];          /* Boundary periodicity per axis (Boundary.cpp:5-11), frame only on axes of size > 1 */
    const uint8_t* type;
    const int32_t* flow;
    const float* temp;
    const int32_t* spill;
    const int8_t* desc;  /* D(n) plane */
    int nb_off[6][26][3];
    int nb_cnt[6];
    int variants;
    int side[26][3];     /* union of dz == 0 offsets (LavaCA.hpp:104-112) */
    int nside;
    int diagonal_falls;
} ca_ctx;

static int64_t gidx(const vo_ca_params* p, int x, int y, int z) { return x + (int64_t)p->nx * (y + (int64_t)p->ny * z); }

/* Map a coordinate one cell outside the interior through the frame: wrap on a periodic axis
 * of size > 1, else "outside".  Returns 0 when the cell is VOID. */
static int wrap_axis(int* v, int n, int periodic) {
    if (*v >= 0 && *v < n) return 1;
    if (!periodic || n == 1) return 0;
    *v = *v < 0 ? *v + n : *v - n;
    return 1;
}
static int resolve(const ca_ctx* c, int* x, int* y, int* z) {
    return wrap_axis(x, c->p->nx, c->per[0]) && wrap_axis(y, c->p->ny, c->per[1]) && wrap_axis(z, c->p->nz, c->per[2]);
}
static int type_at(const ca_ctx* c, int x, int y, int z) {
    if (!resolve(c, &x, &y, &z)) return CELL_VOID;
    return c->type[gidx(c->p, x, y, z)];
}
static int spill_at(const ca_ctx* c, int x, int y) {
    /* spillAt wraps the column (LavaCA.hpp:383) */
    int xx = x, yy = y;
    if (xx < 0) xx += c->p->nx; else if (xx >= c->p->nx) xx -= c->p->nx;
    if (yy < 0) yy += c->p->ny; else if (yy >= c->p->ny) yy -= c->p->ny;
    return c->spill[xx + (int64_t)c->p->nx * yy];
}
static int solid_ground(int t) { return t == CELL_ROCK || t == CELL_BASALT; }

/* LavaCA::hasSupport (LavaCA.hpp:390-399). */
static int has_support(const ca_ctx* c, int x, int y, int z) {
    if (z == 0) return 1;
    const int below = type_at(c, x, y, z - 1);
    if (solid_ground(below)) return 1;
    return below == CELL_LAVA && c->spill != NULL && z - 1 < spill_at(c, x, y);
}

/* LavaCA::dropDepth (LavaCA.hpp:404-414), kMaxDrop = 16 (LavaCA.hpp:1293). */
static int drop_depth(const ca_ctx* c, int x, int y, int z) {
    for (int d = 0; d <= 16 && z - d >= 0; ++d) {
        if (d > 0 && type_at(c, x, y, z - d) != CELL_AIR) return -1;
        if (has_support(c, x, y, z - d)) return d;
    }
    return 16;
}

/* LavaCA::descent (LavaCA.hpp:421-429). */
static int descent(const ca_ctx* c, int x, int y, int z) {
    int best = 0;
    for (int k = 0; k < c->nside; ++k) {
        const int ax = x + c->side[k][0], ay = y + c->side[k][1];
        if (type_at(c, ax, ay, z) == CELL_AIR) {
            const int d = drop_depth(c, ax, ay, z);
            if (d > best) best = d;
        }
    }
    return best;
}

/* CandidateVote (CaRules.hpp:127-183). */
typedef struct { int32_t ids[32]; int counts[32]; float max_temp[32]; int n; } vote_t;
static void vote_add(vote_t* v, int32_t id, float t) {
    for (int i = 0; i < v->n; ++i)
        if (v->ids[i] == id) {
            ++v->counts[i];
            if (t > v->max_temp[i]) v->max_temp[i] = t; /* std::max(a, b) keeps a unless a < b */
            return;
        }
    v->ids[v->n] = id;
    v->counts[v->n] = 1;
    v->max_temp[v->n] = t;
    ++v->n;
}
static int vote_winner(const vote_t* v, uint64_t seed, uint64_t step, uint64_t cell) {
    if (v->n == 1) return 0;
    int best = 0;
    for (int i = 0; i < v->n; ++i)
        if (v->counts[i] > best) best = v->counts[i];
    int tied[32], k = 0;
    for (int i = 0; i < v->n; ++i)
        if (v->counts[i] == best) tied[k++] = i;
    if (k == 1) return tied[0];
    /* sort tied by id ascending (insertion sort; ids are distinct) */
    for (int i = 1; i < k; ++i) {
        int j = i, t = tied[i];
        while (j > 0 && v->ids[tied[j - 1]] > v->ids[t]) { tied[j] = tied[j - 1]; --j; }
        tied[j] = t;
    }
    const uint64_t r = vo_hash_rand(seed, step, cell, SALT_TIEBREAK);
    return tied[(int)(r % (uint64_t)k)];
}

/* LavaCA::tryPonding (LavaCA.hpp:443-461); horizontal_ offsets (LavaCA.hpp:96-101). */
static void try_ponding(const ca_ctx* c, int x, int y, int z, vote_t* vote) {
    if (c->spill == NULL || z > c->spill[x + (int64_t)c->p->nx * y]) return;
    const int bz = z - 1;
    if (type_at(c, x, y, bz) != CELL_LAVA) return;
    if (!has_support(c, x, y, bz)) return;
    const int hx[4] = {-1, 1, 0, 0}, hy[4] = {0, 0, -1, 1};
    const int nh = c->p->ny > 1 ? 4 : 2;
    for (int k = 0; k < nh; ++k) {
        const int n = type_at(c, x + hx[k], y + hy[k], bz);
        if (n == CELL_AIR || n == CELL_VOID) return;
    }
    const int64_t b = gidx(c->p, x, y, bz);
    vote_add(vote, c->flow[b], c->temp[b] - c->p->cooling_lateral);
}

/* LavaCA::gatherLavaCandidates (LavaCA.hpp:465-519). */
static void gather(const ca_ctx* c, int x, int y, int z, uint64_t prefix, uint64_t idx, vote_t* vote) {
    vote->n = 0;
    int variant = 0;
    if (c->variants > 1) variant = (int)(vo_hash_salt(vo_hash_index(prefix, idx), SALT_NEIGHBORHOOD) % (uint64_t)c->variants);
    int c_drop = -100;
    for (int k = 0; k < c->nb_cnt[variant]; ++k) {
        const int dx = c->nb_off[variant][k][0], dy = c->nb_off[variant][k][1], dz = c->nb_off[variant][k][2];
        if (dz < 0) {
            if (c->p->ponding && dx == 0 && dy == 0) try_ponding(c, x, y, z, vote);
            continue;
        }
        int sx = x + dx, sy = y + dy, sz = z + dz;
        if (!resolve(c, &sx, &sy, &sz)) continue;        /* VOID frame: never lava */
        const int64_t s = gidx(c->p, sx, sy, sz);
        if (c->type[s] != CELL_LAVA) continue;
        float cooling;
        if (dz > 0 && dx == 0 && dy == 0) {
            cooling = c->p->cooling_fall;
        } else {
            const int d = c->desc[s];
            if (d < 0) continue;
            if (c_drop == -100) c_drop = drop_depth(c, x, y, z);
            if (dz > 0) {
                if (c_drop != 0 || d != 1) continue;
                cooling = c->p->cooling_fall;
            } else {
                if (c_drop != d || (d == 1 && c->diagonal_falls)) continue;
                cooling = c->p->cooling_lateral;
            }
        }
        vote_add(vote, c->flow[s], c->temp[s] - cooling);
    }
}

static int is_vent(const int32_t* vent_xyz, int slots, int32_t f, int x, int y, int z) {
    /* LavaCA::isVent (LavaCA.hpp:335-341) */
    if (f <= 0 || f >= slots) return 0;
    return vent_xyz[3 * f] == x && vent_xyz[3 * f + 1] == y && vent_xyz[3 * f + 2] == z;
}

static void ctx_init(ca_ctx* c, const vo_ca_params* p) {
    memset(c, 0, sizeof(*c));
    c->p = p;
    c->per[0] = p->periodic;
    c->per[1] = p->periodic;
    c->per[2] = p->periodic && p->classic;
    c->variants = vo_nb_build(p->neighborhood, p->nx, p->ny, p->nz, c->nb_off, c->nb_cnt);
    for (int v = 0; v < c->variants; ++v)
        for (int k = 0; k < c->nb_cnt[v]; ++k) {
            const int* o = c->nb_off[v][k];
            if (o[2] == 0) {
                int dup = 0;
                for (int j = 0; j < c->nside; ++j)
                    if (c->side[j][0] == o[0] && c->side[j][1] == o[1] && c->side[j][2] == o[2]) dup = 1;
                if (!dup) {
                    c->side[c->nside][0] = o[0];
                    c->side[c->nside][1] = o[1];
                    c->side[c->nside][2] = o[2];
                    ++c->nside;
                }
            } else if (o[2] == -1 && (o[0] != 0 || o[1] != 0)) {
                c->diagonal_falls = 1;
            }
        }
}

/* One step of a grid that may be a strip (z layers) of a taller grid: gidx_base is the global index
 * of local cell 0 (hashRand takes global indices) and only layers [own_z0, own_z1) are counted
 * (the reference's strips sum their counters, engine/src/ca/LavaCA.hpp:1207-1211). */
static void ca_step_impl(const vo_ca_params* p, int t, uint64_t gidx_base, int own_z0, int own_z1, const int32_t* spill,
                         const int32_t* vent_xyz, int vent_slots, const uint8_t* type, const int32_t* flow,
                         const float* temp, const uint16_t* solid, const uint16_t* arrival, uint8_t* ntype,
                         int32_t* nflow, float* ntemp, uint16_t* nsolid, uint16_t* narrival, uint64_t counts[3]) {
    ca_ctx c;
    ctx_init(&c, p);
    c.type = type;
    c.flow = flow;
    c.temp = temp;
    c.spill = spill;
    const int64_t n = (int64_t)p->nx * p->ny * p->nz;
    int8_t* desc = (int8_t*)malloc((size_t)(n > 0 ? n : 1));
    c.desc = desc;
    /* StepCtx (LavaCA.hpp:542-546) */
    const uint64_t tt = (uint64_t)t;
    const int erupting = t < p->eruption_steps;
    const uint16_t stamp = (uint16_t)(t < 65535 ? t : 65535);
    const uint64_t prefix = vo_hash_prefix(p->seed, tt);
    uint64_t active = 0, air = 0, changed = 0;

    if (!p->classic) {
        /* computeDescent (LavaCA.hpp:551-566) */
        for (int z = 0; z < p->nz; ++z)
            for (int y = 0; y < p->ny; ++y)
                for (int x = 0; x < p->nx; ++x) {
                    const int64_t i = gidx(p, x, y, z);
                    int8_t d = -1;
                    if (type[i] == CELL_LAVA && has_support(&c, x, y, z)) d = (int8_t)descent(&c, x, y, z);
                    desc[i] = d;
                }
    }
    vote_t vote;
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t i = gidx(p, x, y, z);
                const uint64_t gi = (uint64_t)i + gidx_base;
                const uint64_t own = (z >= own_z0 && z < own_z1) ? 1 : 0;
                uint8_t ty = type[i];
                int32_t f = flow[i];
                float te = temp[i];
                uint16_t so = solid[i], ar = arrival[i];
                if (!p->classic) {
                    /* updateLava (LavaCA.hpp:1109-1161) */
                    if (ty == CELL_AIR) {
                        gather(&c, x, y, z, prefix, gi, &vote);
                        int became = 0;
                        if (vote.n > 0) {
                            const int w = vote_winner(&vote, p->seed, tt, gi);
                            const float wt = vote.max_temp[w];
                            if (wt >= p->solidus_temp) {
                                ty = CELL_LAVA; f = vote.ids[w]; te = wt; so = 0; ar = stamp;
                                active += own; changed += own;
                                became = 1;
                            }
                        }
                        if (!became) air += own;
                    } else if (ty == CELL_LAVA) {
                        const float before = te;
                        if (erupting && is_vent(vent_xyz, vent_slots, f, x, y, z)) te = p->erupt_temp;
                        else te -= p->cooling_ambient;
                        if (te < p->solidus_temp) {
                            ty = CELL_BASALT; so = stamp; changed += own;
                        } else {
                            active += own;
                            changed += (te != before) ? own : 0;
                        }
                    }
                } else {
                    /* updateClassic (LavaCA.hpp:1164-1201) */
                    if (ty == CELL_AIR) {
                        vote.n = 0;
                        int variant = 0;
                        if (c.variants > 1)
                            variant = (int)(vo_hash_salt(vo_hash_index(prefix, gi), SALT_NEIGHBORHOOD) % (uint64_t)c.variants);
                        for (int k = 0; k < c.nb_cnt[variant]; ++k) {
                            int sx = x + c.nb_off[variant][k][0], sy = y + c.nb_off[variant][k][1], sz = z + c.nb_off[variant][k][2];
                            if (!resolve(&c, &sx, &sy, &sz)) continue;
                            const int64_t s = gidx(p, sx, sy, sz);
                            if (type[s] == CELL_LAVA) vote_add(&vote, flow[s], 0.0f);
                        }
                        if (vote.n > 0) {
                            const int w = vote_winner(&vote, p->seed, tt, gi);
                            ty = CELL_LAVA; f = vote.ids[w]; te = 0.0f; so = 0; ar = stamp;
                            active += own; changed += own;
                        } else {
                            air += own;
                        }
                    } else if (ty == CELL_LAVA) {
                        active += own;
                    }
                }
                ntype[i] = ty; nflow[i] = f; ntemp[i] = te; nsolid[i] = so; narrival[i] = ar;
            }
    free(desc);
    counts[0] = active;
    counts[1] = air;
    counts[2] = changed;
}

void vo_ca_step(const vo_ca_params* p, int t, const int32_t* spill, const int32_t* vent_xyz, int vent_slots,
                const uint8_t* type, const int32_t* flow, const float* temp, const uint16_t* solid,
                const uint16_t* arrival, uint8_t* ntype, int32_t* nflow, float* ntemp, uint16_t* nsolid,
                uint16_t* narrival, uint64_t counts[3]) {
    ca_step_impl(p, t, 0, 0, p->nz, spill, vent_xyz, vent_slots, type, flow, temp, solid, arrival, ntype, nflow, ntemp,
                 nsolid, narrival, counts);
}

void vo_ca_step_strip(const vo_ca_params* p, int t, uint64_t gidx_base, int own_z0, int own_z1, const int32_t* spill,
                      const int32_t* vent_xyz, int vent_slots, const uint8_t* type, const int32_t* flow,
                      const float* temp, const uint16_t* solid, const uint16_t* arrival, uint8_t* ntype,
                      int32_t* nflow, float* ntemp, uint16_t* nsolid, uint16_t* narrival, uint64_t counts[3]) {
    ca_step_impl(p, t, gidx_base, own_z0, own_z1, spill, vent_xyz, vent_slots, type, flow, temp, solid, arrival, ntype,
                 nflow, ntemp, nsolid, narrival, counts);
}

int vo_ca_stop_after(const vo_ca_params* p, int steps_done, const uint64_t counts[3]) {
    const int random_nb = p->neighborhood == 2 || p->neighborhood == 3;
    if (!p->classic && counts[0] == 0) return 1;
    if (p->classic && counts[1] == 0) return 2;
    if (counts[2] == 0 && !random_nb) return 3;
    if (steps_done >= p->max_steps) return 4;
    return 0;
}

/* ---------------------------------------------------------------------------------------------
 * Potts MC, checkerboard update (engine/src/mc/PottsMC.cpp)
 * ------------------------------------------------------------------------------------------- */
static int64_t mgidx(const vo_mc_params* p, int x, int y, int z) { return x + (int64_t)p->nx * (y + (int64_t)p->ny * z); }

/* Spin of a (possibly frame) neighbour: periodic copy or 0 (PottsMC::fillFrame, PottsMC.cpp:226-277). */
static int32_t spin_at(const vo_mc_params* p, const int32_t* spin, int x, int y, int z) {
    if (!wrap_axis(&x, p->nx, p->periodic[0]) || !wrap_axis(&y, p->ny, p->periodic[1]) ||
        !wrap_axis(&z, p->nz, p->periodic[2]))
        return 0;
    return spin[mgidx(p, x, y, z)];
}

void vo_mc_init(const vo_mc_params* p, const uint8_t* domain, int32_t* spin) {
    const uint64_t q = (uint64_t)p->Q;
    const int64_t n = (int64_t)p->nx * p->ny * p->nz;
    for (int64_t g = 0; g < n; ++g)
        spin[g] = domain[g] ? 1 + (int32_t)(vo_hash_rand(p->seed, 0, (uint64_t)g, SALT_MC_INIT) % q) : 0;
}

static int axis_n(const vo_mc_params* p, int a) { return a == 0 ? p->nx : a == 1 ? p->ny : p->nz; }
static int odd_periodic(const vo_mc_params* p) {
    for (int a = 0; a < 3; ++a)
        if (p->periodic[a] && axis_n(p, a) % 2 == 1) return 1;
    return 0;
}
static int parity_colors(const vo_mc_params* p) { return p->neighborhood == 0 && !odd_periodic(p); }
static int classes_of(const vo_mc_params* p, int a) {
    const int n = axis_n(p, a);
    return n == 1 ? 1 : (p->periodic[a] && n % 2 == 1 ? 3 : 2);
}
int vo_mc_colors(const vo_mc_params* p) {
    if (parity_colors(p)) return 2;
    return classes_of(p, 0) * classes_of(p, 1) * classes_of(p, 2);
}
/* axisClass / colorOf / buildColors numbering (PottsMC.cpp:145-193). */
static int axis_class(const vo_mc_params* p, int c, int a) {
    const int n = axis_n(p, a);
    if (p->periodic[a] && n % 2 == 1 && c == n - 1) return 2;
    return c & 1;
}
int vo_mc_color_of(const vo_mc_params* p, int x, int y, int z) {
    if (parity_colors(p)) return (x + y + z) & 1;
    const int cx = axis_class(p, x, 0), cy = axis_class(p, y, 1), cz = axis_class(p, z, 2);
    /* colours numbered by cx + 3cy + 9cz ascending over existing classes, cx fastest */
    return cx + classes_of(p, 0) * (cy + classes_of(p, 1) * cz);
}

/* colorTrials (PottsMC.cpp:394-448) of one colour; order within a colour does not matter.  For a
 * strip of z layers of a taller grid (PottsMC.cpp:451-460): hashRand takes global indices (local +
 * gidx_base) and colours follow the global z (local + zoff). */
static void mc_color_impl(const vo_mc_params* p, int t, int col, uint64_t gidx_base, int zoff, const uint8_t* domain,
                          const float* mobility, int32_t* spin, uint64_t out[3]) {
    int off[6][26][3], cnt[6];
    const int variants = vo_nb_build(p->neighborhood, p->nx, p->ny, p->nz, off, cnt);
    const uint64_t prefix = vo_hash_prefix(p->seed, (uint64_t)t);
    const uint64_t other = (uint64_t)(p->Q - 1);
    {
        for (int z = 0; z < p->nz; ++z)
            for (int y = 0; y < p->ny; ++y)
                for (int x = 0; x < p->nx; ++x) {
                    const int64_t g = mgidx(p, x, y, z);
                    if (!domain[g] || vo_mc_color_of(p, x, y, z + zoff) != col) continue;
                    const uint64_t h = vo_hash_index(prefix, (uint64_t)g + gidx_base);
                    if (mobility != NULL && to_uniform(vo_hash_salt(h, SALT_MC_MOBILITY)) >= (double)mobility[g]) continue;
                    ++out[0];
                    int v = 0;
                    if (variants > 1) v = (int)(vo_hash_salt(h, SALT_NEIGHBORHOOD) % (uint64_t)variants);
                    const int32_t cur = spin[g];
                    int32_t prop = 1 + (int32_t)(vo_hash_salt(h, SALT_MC_ORIENT) % other);
                    if (prop >= cur) ++prop;
                    /* unlikeBeforeAfter (PottsMC.hpp:191-204) */
                    int in_domain = 0, same_a = 0, same_b = 0;
                    for (int k = 0; k < cnt[v]; ++k) {
                        const int32_t sj = spin_at(p, spin, x + off[v][k][0], y + off[v][k][1], z + off[v][k][2]);
                        in_domain += sj != 0;
                        same_a += sj == cur;
                        same_b += sj == prop;
                    }
                    const int before = in_domain - same_a, after = in_domain - same_b;
                    const double dE = p->J * after - p->J * before;
                    int accept = dE <= 0.0;
                    if (!accept && p->kT > 0.0) {
                        accept = to_uniform(vo_hash_salt(h, SALT_MC_ACCEPT)) < exp(-dE / p->kT);
                        out[2] += accept ? 1 : 0;
                    }
                    if (accept) {
                        spin[g] = prop;
                        ++out[1];
                    }
                }
    }
}

void vo_mc_sweep(const vo_mc_params* p, int t, const uint8_t* domain, const float* mobility, int32_t* spin,
                 uint64_t out[3]) {
    const int colors = vo_mc_colors(p);
    for (int col = 0; col < colors; ++col) mc_color_impl(p, t, col, 0, 0, domain, mobility, spin, out);
}

void vo_mc_color_strip(const vo_mc_params* p, int t, int col, uint64_t gidx_base, int zoff, const uint8_t* domain,
                       const float* mobility, int32_t* spin, uint64_t out[3]) {
    mc_color_impl(p, t, col, gidx_base, zoff, domain, mobility, spin, out);
}

double vo_mc_energy(const vo_mc_params* p, int t, const int32_t* spin) {
    int off[6][26][3], cnt[6];
    const int variants = vo_nb_build(p->neighborhood, p->nx, p->ny, p->nz, off, cnt);
    uint64_t unlike = 0;
    if (variants == 1) {
        /* forward pairs (PottsMC.cpp:593-643) */
        for (int z = 0; z < p->nz; ++z)
            for (int y = 0; y < p->ny; ++y)
                for (int x = 0; x < p->nx; ++x) {
                    const int32_t s = spin[mgidx(p, x, y, z)];
                    if (s == 0) continue;
                    uint64_t in_dom = 0, same = 0;
                    for (int k = 0; k < cnt[0]; ++k) {
                        const int* o = off[0][k];
                        if (!(o[2] > 0 || (o[2] == 0 && (o[1] > 0 || (o[1] == 0 && o[0] > 0))))) continue;
                        const int32_t sj = spin_at(p, spin, x + o[0], y + o[1], z + o[2]);
                        in_dom += sj != 0;
                        same += sj == s;
                    }
                    unlike += in_dom - same;
                }
        return p->J * (double)unlike;
    }
    const uint64_t prefix = vo_hash_prefix(p->seed, (uint64_t)t);
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t g = mgidx(p, x, y, z);
                const int32_t s = spin[g];
                if (s == 0) continue;
                const int v = (int)(vo_hash_salt(vo_hash_index(prefix, (uint64_t)g), SALT_NEIGHBORHOOD) % (uint64_t)variants);
                int in_dom = 0, same = 0;
                for (int k = 0; k < cnt[v]; ++k) {
                    const int32_t sj = spin_at(p, spin, x + off[v][k][0], y + off[v][k][1], z + off[v][k][2]);
                    in_dom += sj != 0;
                    same += sj == s;
                }
                unlike += (uint64_t)(in_dom - same);
            }
    return 0.5 * p->J * (double)unlike;
}

// terrain.cpp -- terrain and vents on the host, with the reference's arithmetic so that the
// same config yields the same initial grid: the cone with value noise
// (engine/src/terrain/TerrainGenerator.cpp:16-84), the CSV heightmap loader
// (engine/src/terrain/HeightmapLoader.cpp:37-83) and vent placement by mt19937_64 with a partial
// Fisher-Yates shuffle (engine/src/terrain/VentPlacer.cpp:11-104).  Spill levels (the priority
// flood) are computed by libvca.so in vca_ca_apply_terrain.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <random>
#include <string>

#include "model.hpp"

namespace eng {

namespace {

constexpr uint64_t kSaltTerrain = 0x5445525241494E31ULL;  // engine/src/core/Rng.hpp:25
constexpr uint64_t kSaltVents = 0x56454E5453454544ULL;    // engine/src/core/Rng.hpp:26

// splitmix64 cascade (engine/src/core/Rng.hpp:35-72), host copy of the device hash in vca_device.cuh.
uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}
uint64_t hash_rand(uint64_t seed, uint64_t step, uint64_t idx, uint64_t salt) {
    uint64_t h = splitmix64(seed ^ 0xA0761D6478BD642FULL);
    h = splitmix64(h ^ step);
    h = splitmix64(h ^ idx);
    return splitmix64(h ^ salt);
}

// hashUniform (Rng.hpp:55-59): 53 high bits of hashRand, scaled by 2^-53.
double hash_uniform(uint64_t seed, uint64_t step, uint64_t idx, uint64_t salt) {
    return (double)(hash_rand(seed, step, idx, salt) >> 11) * (1.0 / 9007199254740992.0);
}

// latticeValue / smooth / valueNoise (TerrainGenerator.cpp:16-44).
double lattice_value(uint64_t seed, int octave, int i, int j) {
    const uint64_t key = (uint64_t)(uint32_t)i | ((uint64_t)(uint32_t)j << 32);
    return 2.0 * hash_uniform(seed, (uint64_t)octave, key, kSaltTerrain) - 1.0;
}
double smooth(double t) { return t * t * (3.0 - 2.0 * t); }
double value_noise(uint64_t seed, int octave, int spacing, int x, int y) {
    const int i = x / spacing, j = y / spacing;
    const double fx = smooth((double)(x % spacing) / spacing);
    const double fy = smooth((double)(y % spacing) / spacing);
    const double v00 = lattice_value(seed, octave, i, j);
    const double v10 = lattice_value(seed, octave, i + 1, j);
    const double v01 = lattice_value(seed, octave, i, j + 1);
    const double v11 = lattice_value(seed, octave, i + 1, j + 1);
    const double a = v00 + (v10 - v00) * fx;
    const double b = v01 + (v11 - v01) * fx;
    return a + (b - a) * fy;
}
double smooth_noise(uint64_t seed, int x, int y) {
    const double n = 1.0 * value_noise(seed, 0, 16, x, y) + 0.5 * value_noise(seed, 1, 8, x, y) +
                     0.25 * value_noise(seed, 2, 4, x, y);
    return n / 1.75;
}
double cone_height(const Config& c, double r) { return c.terrain.peak * std::max(0.0, 1.0 - r / c.terrain.base_radius); }

}  // namespace

double distance_from_center(const Dims& d, int x, int y) {
    const double cx = (d.nx - 1) / 2.0, cy = (d.ny - 1) / 2.0;
    return std::hypot(x - cx, y - cy);
}

// TerrainGenerator::cone (TerrainGenerator.cpp:61-84).
Heightmap cone_terrain(const Config& c) {
    const Dims& d = c.space;
    Heightmap hm;
    hm.nx = d.nx;
    hm.ny = d.ny;
    hm.height.resize((size_t)d.nx * d.ny);
    const double amplitude = c.terrain.noise * c.terrain.peak;
    const double crater_floor = cone_height(c, c.terrain.crater_radius) - c.terrain.crater_depth;
    for (int y = 0; y < d.ny; ++y)
        for (int x = 0; x < d.nx; ++x) {
            const double r = distance_from_center(d, x, y);
            double h = (r < c.terrain.crater_radius) ? crater_floor : cone_height(c, r);
            h += amplitude * smooth_noise(c.seed, x, y);
            const int cells = (int)std::ceil(h);
            hm.height[(size_t)x + (size_t)d.nx * y] = std::clamp(cells, 0, d.nz);
        }
    return hm;
}

// HeightmapLoader::loadCsv (HeightmapLoader.cpp:37-83): separators , ; space tab; '#' lines skipped;
// ny data rows of nx non-negative numbers; ROCK count = ceil(value) clamped to nz.
Heightmap load_heightmap_csv(const std::string& path, const Dims& d) {
    std::ifstream in(path);
    if (!in) throw ConfigError("Nie można otworzyć pliku mapy wysokości: " + path);
    Heightmap hm;
    hm.nx = d.nx;
    hm.ny = d.ny;
    hm.height.reserve((size_t)d.nx * d.ny);
    std::string line;
    int line_no = 0, row = 0;
    while (std::getline(in, line)) {
        ++line_no;
        std::vector<std::string> fields;
        std::string cur;
        for (char ch : line) {
            if (ch == ',' || ch == ';' || ch == ' ' || ch == '\t' || ch == '\r') {
                if (!cur.empty()) {
                    fields.push_back(cur);
                    cur.clear();
                }
            } else {
                cur += ch;
            }
        }
        if (!cur.empty()) fields.push_back(cur);
        if (fields.empty() || fields[0][0] == '#') continue;
        if (row >= d.ny) throw ConfigError("Mapa wysokości " + path + " ma więcej wierszy danych niż ny = " + std::to_string(d.ny));
        if ((int)fields.size() != d.nx)
            throw ConfigError("Mapa wysokości " + path + ", wiersz " + std::to_string(line_no) + ": " + std::to_string(fields.size()) +
                              " wartości, oczekiwano nx = " + std::to_string(d.nx));
        for (size_t col = 0; col < fields.size(); ++col) {
            char* end = nullptr;
            const double h = std::strtod(fields[col].c_str(), &end);
            if (end == fields[col].c_str() || *end != '\0' || !std::isfinite(h) || h < 0.0)
                throw ConfigError("Mapa wysokości " + path + ", wiersz " + std::to_string(line_no) + ", kolumna " +
                                  std::to_string(col + 1) + ": oczekiwano nieujemnej liczby, jest \"" + fields[col] + "\"");
            hm.height.push_back(std::min((int)std::ceil(h), d.nz));
        }
        ++row;
    }
    if (row != d.ny)
        throw ConfigError("Mapa wysokości " + path + " ma " + std::to_string(row) + " wierszy danych, oczekiwano ny = " + std::to_string(d.ny));
    return hm;
}

// VentPlacer::placeVents (VentPlacer.cpp:11-58): candidate columns in (y, x) order, then a partial
// Fisher-Yates shuffle driven by mt19937_64(splitmix64(seed ^ kSaltVents)) and gen() % n.
std::vector<Vent> place_vents(const Config& c, const Heightmap& hm) {
    const Dims& d = c.space;
    std::vector<std::pair<int, int>> cand;
    for (int y = 0; y < d.ny; ++y)
        for (int x = 0; x < d.nx; ++x) {
            const int h = hm.at(x, y);
            if (h >= d.nz) continue;
            const double r = distance_from_center(d, x, y);
            bool ok;
            if (c.vents.placement == Placement::Crater) {
                ok = r <= c.terrain.crater_radius;
            } else {
                ok = r > c.terrain.crater_radius && h >= 1 && (c.terrain.type != TerrainType::Cone || r < c.terrain.base_radius);
            }
            if (ok) cand.emplace_back(x, y);
        }
    if ((int)cand.size() < c.vents.count)
        throw ConfigError(std::string("Za mało miejsc na kratery (placement = ") +
                          (c.vents.placement == Placement::Crater ? "crater" : "random") + "): dostępnych " +
                          std::to_string(cand.size()) + ", a vents.count = " + std::to_string(c.vents.count) +
                          (c.vents.placement == Placement::Crater ? "; zwiększ terrain.craterRadius" : ""));
    std::mt19937_64 gen(splitmix64(c.seed ^ kSaltVents));
    std::vector<Vent> vents;
    for (int i = 0; i < c.vents.count; ++i) {
        const size_t remaining = cand.size() - (size_t)i;
        const size_t j = (size_t)i + (size_t)(gen() % remaining);
        std::swap(cand[(size_t)i], cand[j]);
        const auto [x, y] = cand[(size_t)i];
        vents.push_back(Vent{x, y, hm.at(x, y), i + 1});
    }
    return vents;
}

// VentPlacer::placeAt (VentPlacer.cpp:60-81): the first AIR cell of each listed column.
std::vector<Vent> place_at(const std::vector<std::pair<int, int>>& cols, const Dims& d, const Heightmap& hm) {
    std::vector<Vent> vents;
    for (size_t i = 0; i < cols.size(); ++i) {
        const int cx = cols[i].first, cy = cols[i].second;
        const std::string where = "vents.positions[" + std::to_string(i) + "] = [" + std::to_string(cx) + ", " +
                                  std::to_string(cy) + "]";
        if (cx < 0 || cx >= d.nx || cy < 0 || cy >= d.ny)
            throw ConfigError(where + " lies outside the grid " + std::to_string(d.nx) + " x " + std::to_string(d.ny));
        const int h = hm.empty() ? 0 : hm.at(cx, cy);
        if (h >= d.nz)
            throw ConfigError(where + ": the column is all rock (terrain height " + std::to_string(h) +
                              " >= space.nz = " + std::to_string(d.nz) + "), no room for a vent above it");
        vents.push_back(Vent{cx, cy, h, (int32_t)(i + 1)});
    }
    return vents;
}

// VentPlacer::placeSeeds (VentPlacer.cpp:83-104): distinct random cells of the whole space.
std::vector<Vent> place_seeds(int count, const Dims& d, uint64_t seed) {
    const uint64_t n = d.cells();
    std::mt19937_64 gen(splitmix64(seed ^ kSaltVents));
    std::vector<bool> taken((size_t)n, false);
    std::vector<Vent> seeds;
    while ((int)seeds.size() < count) {
        const uint64_t idx = gen() % n;
        if (taken[(size_t)idx]) continue;
        taken[(size_t)idx] = true;
        const int x = (int)(idx % (uint64_t)d.nx);
        const int y = (int)((idx / (uint64_t)d.nx) % (uint64_t)d.ny);
        const int z = (int)(idx / ((uint64_t)d.nx * (uint64_t)d.ny));
        seeds.push_back(Vent{x, y, z, (int32_t)(seeds.size() + 1)});
    }
    return seeds;
}

}  // namespace eng

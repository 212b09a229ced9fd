// model.hpp -- data types of the engine host (the C++17 front end over libvca.so).
//
// The host mirrors the reference engine's surface (engine/src/app, engine/src/io,
// engine/src/terrain): config keys and validation, terrain and vents, result files, statistics.
// All grid compute (CA steps, Potts sweeps, energy, mobility) runs in libvca.so on the GPU.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "json.hpp"

namespace eng {

// Exit codes (engine/src/main.cpp:6-8).
enum ExitCode { kExitOk = 0, kExitConfig = 1, kExitArgs = 2, kExitOther = 3, kExitBatch = 5 };

struct ConfigError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct CliError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// CellType (engine/src/core/Types.hpp:13-19).
enum : uint8_t { kAir = 0, kRock = 1, kLava = 2, kBasalt = 3, kVoid = 255 };

struct Dims {
    int nx = 1, ny = 1, nz = 1;
    uint64_t cells() const { return (uint64_t)nx * ny * nz; }
    int active_axes() const { return (nx > 1) + (ny > 1) + (nz > 1); }
    bool is2d() const { return active_axes() == 2; }
    bool operator==(const Dims& o) const { return nx == o.nx && ny == o.ny && nz == o.nz; }
    bool operator!=(const Dims& o) const { return !(*this == o); }
};

// Microstructure: unframed SoA planes, index x + nx*(y + ny*z) (engine/src/core/Types.hpp:105-134).
struct Microstructure {
    Dims dims;
    std::vector<uint8_t> type;
    std::vector<int32_t> flow;
    std::vector<float> temp;
    std::vector<uint16_t> solid;
    std::vector<uint16_t> arrival;
    void resize(const Dims& d) {
        dims = d;
        const size_t n = (size_t)d.cells();
        type.assign(n, kAir);
        flow.assign(n, 0);
        temp.assign(n, 0.0f);
        solid.assign(n, 0);
        arrival.assign(n, 0);
    }
};

struct CrystalMap {
    Dims dims;
    std::vector<int32_t> crystal;
};

// Heightmap: ROCK cells per column (engine/src/terrain/TerrainGenerator.hpp:19-29).
struct Heightmap {
    int nx = 0, ny = 0;
    std::vector<int32_t> height;
    int at(int x, int y) const { return height[(size_t)x + (size_t)nx * y]; }
    bool empty() const { return height.empty(); }
};

struct Vent {
    int x, y, z;
    int32_t flow_id;
};

enum class Nb { VonNeumann, Moore, Pentagonal, Hexagonal };
enum class Bc { Absorbing, Periodic };
enum class Mode { Lava, Classic };
enum class TerrainType { Cone, File };
enum class Placement { Crater, Random, Positions };
enum class OutputFormat { Txt, Bin, Both, None };

struct Config {
    Dims space;
    std::string grid;  // "vector" / "matrix": accepted, both give the same results
    Bc boundary = Bc::Absorbing;
    Nb neighborhood = Nb::Moore;
    uint64_t seed = 42;
    struct {
        TerrainType type = TerrainType::Cone;
        double peak = 70, base_radius = 90, crater_radius = 6, crater_depth = 4, noise = 0.05;
        std::string file;
    } terrain;
    struct {
        int count = 1;
        Placement placement = Placement::Crater;
        int eruption_steps = 300;
        double erupt_temp = 1200;
    } vents;
    struct {
        Mode mode = Mode::Lava;
        int max_steps = 5000;
        double cool_ambient = 0.3, cool_lateral = 1.5, cool_fall = 0.1, solidus = 800;
        bool ponding = true;
        bool front = true;
    } ca;
    struct {
        bool enabled = false;
        bool full = false;  // mc.domain
        int Q = 50, mcs = 100;
        double J = 1.0, kT = 0.0;
        bool mobility_from_cooling = true;
        double mobility_min = 0.05;
        int stats_every = 10, snapshots_every = 0;
        bool checkerboard = false;
        bool full_only() const { return enabled && full; }
    } mc;
    struct {
        OutputFormat format = OutputFormat::Txt;
        int snapshots_every = 0;
    } output;
    int threads = 1;
    std::string schedule = "static";
    int chunk = 0;
    std::string affinity = "none";

    Json effective;                // merged JSON (config_used.json)
    std::string source_path;       // the --config file
    bool space_from_user = false;
    std::vector<std::string> warnings;

    static Json defaults_json();
    static Config load(const std::string& path, const std::vector<std::string>& overrides);
    // the same merge and validation for a config object already in memory (the job server's requests);
    // source_path resolves a relative terrain.file
    static Config load_object(const Json& file, const std::string& source_path, const std::vector<std::string>& overrides);
    static Config from_json(const Json& j);
    std::vector<std::pair<int, int>> vent_columns() const;
};

const char* nb_name(Nb n);
const char* bc_name(Bc b);
const char* mode_name(Mode m);

// terrain.cpp
double distance_from_center(const Dims& d, int x, int y);
Heightmap cone_terrain(const Config& c);
Heightmap load_heightmap_csv(const std::string& path, const Dims& d);
std::vector<Vent> place_vents(const Config& c, const Heightmap& hm);
std::vector<Vent> place_at(const std::vector<std::pair<int, int>>& cols, const Dims& d, const Heightmap& hm);
std::vector<Vent> place_seeds(int count, const Dims& d, uint64_t seed);

// results.cpp
std::string format_temp(float v);
void write_ca_bin(const std::string& path, const Microstructure& m);
void write_ca_txt(const std::string& path, const Microstructure& m);
void write_crystal_bin(const std::string& path, const CrystalMap& m);
void write_crystal_txt(const std::string& path, const CrystalMap& m);
void write_json(const std::string& path, const Json& j);
struct ResultSource {
    std::string path, format;
    uint32_t version = 0;
    bool has_solid = false, has_arrival = false;
};
Microstructure read_ca_folder(const std::string& folder, ResultSource* src);

}  // namespace eng

// main.cpp -- the `engine` command line over libvca.so, with the reference engine's surface
// (engine/src/main.cpp, engine/src/app/Cli.cpp, Simulation.cpp, McStage.cpp, Batch.cpp,
// ConfigCheck.cpp): the same options, config keys, result files and exit codes.  The lava CA and
// the Potts MC run on the GPU through the C ABI (include/vca.h); terrain, vents, statistics,
// result files and the batch runner are host code.
#include <fcntl.h>
#include <spawn.h>
#include <sys/wait.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <limits>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "job.hpp"
#include "model.hpp"
#include "vca.h"

extern char** environ;

namespace eng {

namespace fs = std::filesystem;


void vcheck(vca_status s, const char* what) {
    if (s != VCA_OK) {
        if (s == VCA_ERR_ARG) throw ConfigError(std::string(what) + ": " + vca_last_error());
        throw std::runtime_error(std::string(what) + ": " + vca_last_error());
    }
}

std::string fixed(double v, int decimals) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%.*f", decimals, v);
    return buf;
}

// StopReason texts as the reference writes them into stats.json / times.json
// (describe(), engine/src/ca/CaRules.hpp:110-119).
const char* stop_text(int s) {
    switch (s) {
        case VCA_STOP_RUNNING: return "trwa";
        case VCA_STOP_NO_LAVA: return "brak płynnej lawy";
        case VCA_STOP_NO_AIR: return "brak wolnych komórek (AIR)";
        case VCA_STOP_NO_CHANGE: return "brak zmian w kroku";
        case VCA_STOP_MAX_STEPS: return "osiągnięto ca.maxSteps";
    }
    return "?";
}



struct CliOptions {
    std::string config, out, mc_from, batch;
    std::vector<std::string> overrides;
    bool help = false, print_defaults = false, validate = false, progress = false, timing_detail = false,
         thread_stats = false, benchmark = false;
    // the job server (no counterpart in the reference's command line)
    bool serve = false, serve_batch = true;
    int slots = 16;
    double budget_gb = 120.0;
};

// Cli::parse (engine/src/app/Cli.cpp:36-131).
CliOptions parse_cli(int argc, char** argv) {
    CliOptions o;
    auto need = [&](int& i, const std::string& opt) -> std::string {
        if (i + 1 >= argc) throw CliError("opcja " + opt + " wymaga wartości");
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--help" || a == "-h") o.help = true;
        else if (a == "--config") o.config = need(i, a);
        else if (a == "--out") o.out = need(i, a);
        else if (a == "--mc-from") o.mc_from = need(i, a);
        else if (a == "--batch") o.batch = need(i, a);
        else if (a == "--set") {
            const std::string kv = need(i, a);
            if (kv.find('=') == std::string::npos || kv.front() == '=')
                throw CliError("--set wymaga postaci klucz=wartość (np. space.nx=100), podano: " + kv);
            o.overrides.push_back(kv);
        } else if (a == "--grid") o.overrides.push_back("grid=" + need(i, a));
        else if (a == "--threads") {
            const std::string n = need(i, a);
            if (n.empty() || n.find_first_not_of("0123456789") != std::string::npos)
                throw CliError("opcja --threads wymaga liczby całkowitej >= 0 (0 = wszystkie wątki OpenMP), podano: " + n);
            o.overrides.push_back("parallel.threads=" + n);
        } else if (a == "--thread-stats") o.thread_stats = true;
        else if (a == "--high-priority") o.overrides.push_back("parallel.priority=high");
        else if (a == "--benchmark") o.benchmark = true;
        else if (a == "--timing-detail") o.timing_detail = true;
        else if (a == "--print-defaults") o.print_defaults = true;
        else if (a == "--validate") o.validate = true;
        else if (a == "--progress") o.progress = true;
        else if (a == "--serve") o.serve = true;
        else if (a == "--no-batch") o.serve_batch = false;
        else if (a == "--slots") {
            const std::string n = need(i, a);
            if (n.empty() || n.find_first_not_of("0123456789") != std::string::npos || std::atoi(n.c_str()) < 1)
                throw CliError("opcja --slots wymaga liczby całkowitej >= 1, podano: " + n);
            o.slots = std::atoi(n.c_str());
        } else if (a == "--budget-gb") {
            const std::string n = need(i, a);
            char* end = nullptr;
            o.budget_gb = std::strtod(n.c_str(), &end);
            if (n.empty() || *end != '\0' || !(o.budget_gb > 0.0))
                throw CliError("opcja --budget-gb wymaga liczby > 0, podano: " + n);
        } else throw CliError("nieznany argument: " + a + " (zobacz --help)");
    }
    if (o.serve && (o.print_defaults || o.validate || o.benchmark || !o.config.empty() || !o.out.empty() ||
                    !o.mc_from.empty() || !o.batch.empty() || !o.overrides.empty()))
        throw CliError("--serve czyta zadania ze standardowego wejścia i przyjmuje tylko --slots, --budget-gb i --no-batch");
    if (!o.serve && (o.slots != 16 || o.budget_gb != 120.0 || !o.serve_batch))
        throw CliError("--slots, --budget-gb i --no-batch dotyczą tylko --serve");
    if (o.print_defaults && (o.validate || o.benchmark || o.progress || o.timing_detail || o.thread_stats ||
                             !o.config.empty() || !o.out.empty() || !o.mc_from.empty() || !o.batch.empty() ||
                             !o.overrides.empty()))
        throw CliError("--print-defaults nie przyjmuje innych opcji");
    if (!o.batch.empty() && (!o.config.empty() || !o.mc_from.empty() || o.benchmark || o.validate))
        throw CliError("--batch uruchamia wszystkie configi z folderu i nie łączy się z --config, --mc-from, "
                       "--benchmark ani --validate (dozwolone: --out, --set, --grid, --threads, --timing-detail, "
                       "--thread-stats, --progress)");
    if (o.validate && (o.benchmark || o.progress || o.timing_detail || o.thread_stats))
        throw CliError("--validate tylko sprawdza config (--config, --set, --mc-from) i nie łączy się z "
                       "--benchmark, --progress, --timing-detail ani --thread-stats");
    if (o.benchmark)
        throw CliError("--benchmark porównuje układy siatki CPU (vector i matrix); ten silnik ma jeden układ na GPU "
                       "i nie wykonuje tego porównania");
    return o;
}

std::string usage() {
    return "engine: volcano eruption simulation (lava flow cellular automaton and Monte Carlo crystallisation of\n"
           "the solidified lava) on an NVIDIA B200\n"
           "\n"
           "Usage:\n"
           "  engine --config <file.json> --out <folder> [--set key=value]... [--grid vector|matrix]\n"
           "         [--threads N] [--high-priority] [--timing-detail] [--thread-stats] [--progress]\n"
           "  engine --mc-from <ca_result_folder> --config <mc.json> --out <folder> [--set key=value]... [--progress]\n"
           "  engine --batch <config_folder> --out <results_folder> [--set key=value]... [--progress]\n"
           "  engine --validate [--config <file.json>] [--set key=value]... [--mc-from <folder>]\n"
           "  engine --serve [--slots N] [--budget-gb G] [--no-batch]   (jobs as JSON lines on stdin)\n"
           "  engine --print-defaults\n"
           "  engine --help\n"
           "\n"
           "Results in --out: config_used.json, ca_result.txt and/or ca_result.bin, times.json, stats.json;\n"
           "with mc.enabled = true also mc_result.txt and/or mc_result.bin and mc_stats.csv.\n"
           "Monte Carlo runs with mc.update = \"checkerboard\" (the random-order update is sequential).\n"
           "Exit codes: 0 ok, 1 config error, 2 argument error, 3 other error, 5 batch with failures.\n"
           "GPU: VCA_DEVICE=<ordinal> selects the CUDA device (default 0).\n";
}

int device_ordinal() {
    const char* d = std::getenv("VCA_DEVICE");
    return d ? std::atoi(d) : 0;
}

// ---------------------------------------------------------------------------------------------
// CA stage (Simulation::runWith, engine/src/app/Simulation.cpp:158-292)
// ---------------------------------------------------------------------------------------------

std::string resolve_terrain_file(const Config& c) {
    const fs::path p(c.terrain.file);
    if (p.is_absolute() || fs::exists(p) || c.source_path.empty()) return p.string();
    const fs::path next = fs::path(c.source_path).parent_path() / p;
    return fs::exists(next) ? next.string() : p.string();
}

Heightmap build_terrain(const Config& c) {
    if (c.ca.mode == Mode::Classic) return Heightmap{};
    if (c.terrain.type == TerrainType::File) return load_heightmap_csv(resolve_terrain_file(c), c.space);
    return cone_terrain(c);
}

std::vector<Vent> build_vents(const Config& c, const Heightmap& hm) {
    if (c.ca.mode == Mode::Classic) return place_seeds(c.vents.count, c.space, c.seed);
    if (c.vents.placement == Placement::Positions) return place_at(c.vent_columns(), c.space, hm);
    return place_vents(c, hm);
}

// The launch shape tuned for a grid's class (volcano_ca_mc_b200/tuner.py writes the table
// volcano_ca_mc_b200/tuning.json, found beside bin/ or named by VCA_TUNING): tile 64 x tile_y x
// tile_z and resident rules blocks per SM.  The results do not depend on it.  The job server keeps
// the default tiles (its batch steps them).
bool g_use_tuning = true;

const Json& tuning_table() {
    static const Json table = [] {
        std::string path;
        if (const char* e = std::getenv("VCA_TUNING")) {
            path = e;
        } else {
            std::error_code ec;
            const fs::path exe = fs::read_symlink("/proc/self/exe", ec);
            if (!ec) path = (exe.parent_path().parent_path() / "tuning.json").string();
        }
        std::ifstream in(path);
        if (!in) return Json::object();
        std::stringstream ss;
        ss << in.rdbuf();
        try {
            return Json::parse(ss.str(), false);
        } catch (const std::exception&) {
            return Json::object();
        }
    }();
    return table;
}

void apply_tuning(vca_ca_desc& d, const Config& c) {
    if (!g_use_tuning || c.space.ny == 1 || c.space.nz == 1) return;  // the 2D tiles have one shape
    const Json* classes = tuning_table().find("classes");
    if (!classes || !classes->is_object()) return;
    const std::string prefix = std::string("3d-") + nb_name(c.neighborhood) + "-";
    const long lg = std::lround(std::log2((double)c.space.cells()));
    const Json* best = nullptr;
    long best_gap = 1L << 30;
    for (const auto& kv : classes->members()) {
        if (kv.first.rfind(prefix, 0) != 0) continue;
        const long gap = std::labs(std::atol(kv.first.c_str() + prefix.size()) - lg);
        if (gap < best_gap) {
            best_gap = gap;
            best = &kv.second;
        }
    }
    if (!best) return;
    const Json* tile = best->find("tile");
    const Json* blocks = best->find("rules_blocks_per_sm");
    if (tile && tile->is_array() && tile->size() == 2 && blocks) {
        d.tile_y = (int)(*tile)[0].as_i64();
        d.tile_z = (int)(*tile)[1].as_i64();
        d.rules_blocks_per_sm = (int)blocks->as_i64();
    }
}

vca_ca_desc ca_desc(const Config& c) {
    vca_ca_desc d{};
    d.nx = c.space.nx;
    d.ny = c.space.ny;
    d.nz = c.space.nz;
    d.neighborhood = (int)c.neighborhood;
    d.boundary = c.boundary == Bc::Periodic ? VCA_BC_PERIODIC : VCA_BC_ABSORBING;
    d.mode = c.ca.mode == Mode::Classic ? VCA_MODE_CLASSIC : VCA_MODE_LAVA;
    d.seed = c.seed;
    d.max_steps = c.ca.max_steps;
    d.eruption_steps = c.vents.eruption_steps;
    // Simulation::caParams (Simulation.cpp:122-136): the config's doubles cast to float
    d.erupt_temp = (float)c.vents.erupt_temp;
    d.solidus_temp = (float)c.ca.solidus;
    d.cooling_ambient = (float)c.ca.cool_ambient;
    d.cooling_lateral = (float)c.ca.cool_lateral;
    d.cooling_fall = (float)c.ca.cool_fall;
    d.ponding = c.ca.ponding ? 1 : 0;
    d.sweep = c.ca.front ? VCA_SWEEP_ACTIVE : VCA_SWEEP_DENSE;
    d.device = device_ordinal();
    apply_tuning(d, c);
    return d;
}

Microstructure download(vca_ca* ca, const Dims& d) {
    Microstructure m;
    m.resize(d);
    vcheck(vca_ca_download(ca, m.type.data(), m.flow.data(), m.temp.data(), m.solid.data(), m.arrival.data()),
           "vca_ca_download");
    return m;
}

struct CaHandle {
    vca_ca* h = nullptr;
    bool owned = true;  // a resident handle of the job server belongs to the server
    ~CaHandle() {
        if (owned) vca_ca_destroy(h);
    }
};

RunSummary run_ca(const Config& cfg, const std::string& out_dir, Timing& timing, Progress& progress, CaHandle& ca,
                  const RunHandles& res) {
    RunSummary s;
    auto t = Clock::now();
    const vca_ca_desc d = ca_desc(cfg);
    if (res.ca) {  // a resident handle takes this job's space and parameters without allocating
        ca.h = res.ca;
        ca.owned = false;
        vcheck(vca_ca_reconfigure(ca.h, &d), "vca_ca_reconfigure");
    } else {
        vcheck(vca_ca_create(&d, &ca.h), "vca_ca_create");
    }
    timing.add("allocate", ms_since(t));

    t = Clock::now();
    const Heightmap hm = build_terrain(cfg);
    if (!hm.empty()) vcheck(vca_ca_apply_terrain(ca.h, hm.height.data()), "vca_ca_apply_terrain");
    timing.add("terrain", ms_since(t));

    t = Clock::now();
    s.vents = build_vents(cfg, hm);
    std::vector<vca_vent> vv;
    for (const Vent& v : s.vents) vv.push_back(vca_vent{v.x, v.y, v.z, v.flow_id});
    vcheck(vca_ca_place_seeds(ca.h, vv.data(), (int)vv.size()), "vca_ca_place_seeds");
    timing.add("vents", ms_since(t));

    const int every = cfg.output.snapshots_every;
    vca_ca_info info{};
    if (every <= 0 && !progress.on) {
        t = Clock::now();
        if (res.ca_run)
            res.ca_run(ca.h);
        else
            vcheck(vca_ca_run(ca.h), "vca_ca_run");
        timing.add("caSim", ms_since(t));
    } else {
        // step by step: snapshots step_<k>.bin (Simulation.cpp:212-243) and/or progress lines
        const fs::path snap_dir = fs::path(out_dir) / "snapshots";
        double ca_ms = 0.0, snap_ms = 0.0;
        auto snapshot = [&](int k) {
            const auto ts = Clock::now();
            char name[32];
            std::snprintf(name, sizeof(name), "step_%06d.bin", k);
            write_ca_bin((snap_dir / name).string(), download(ca.h, cfg.space));
            snap_ms += ms_since(ts);
        };
        if (every > 0) {
            fs::create_directories(snap_dir);
            snapshot(0);
        }
        vcheck(vca_ca_get_info(ca.h, &info), "vca_ca_get_info");
        progress.report("ca", info.steps, cfg.ca.max_steps, true, "active", 0);
        int running = info.stop_reason == VCA_STOP_RUNNING;
        while (running) {
            const auto ts = Clock::now();
            vcheck(vca_ca_step(ca.h, &running), "vca_ca_step");
            ca_ms += ms_since(ts);
            vcheck(vca_ca_get_info(ca.h, &info), "vca_ca_get_info");
            progress.report("ca", info.steps, cfg.ca.max_steps, !running, "active", info.lava_cells);
            if (every > 0 && (info.steps % every == 0 || !running)) snapshot(info.steps);
        }
        timing.add("caSim", ca_ms);
        if (every > 0) {
            timing.add("snapshots", snap_ms);
            timing.add_file(snap_dir.string(), snap_ms);
        }
    }
    vcheck(vca_ca_get_info(ca.h, &info), "vca_ca_get_info");
    double dev_ms = 0.0, rules_ms = 0.0;
    uint64_t rules_n = 0;
    vca_ca_timing(ca.h, &dev_ms, &rules_ms, &rules_n);
    timing.add_detail("caDevice", dev_ms);

    if (progress.on) progress.report("save", 0, 1, true);
    t = Clock::now();
    s.steps = info.steps;
    s.stop = info.stop_reason;
    s.active.assign((size_t)std::max(1, s.steps), 0);
    s.changed.assign((size_t)std::max(1, s.steps), 0);
    int cnt = 0;
    vcheck(vca_ca_history(ca.h, s.active.data(), s.changed.data(), s.steps, &cnt), "vca_ca_history");
    s.active.resize((size_t)s.steps);
    s.changed.resize((size_t)s.steps);
    s.result = download(ca.h, cfg.space);
    const fs::path out(out_dir);
    if (out_dir.empty()) {  // job server without an output folder: the results leave as digests
        timing.add("save", ms_since(t));
        return s;
    }
    if (cfg.output.format == OutputFormat::Txt || cfg.output.format == OutputFormat::Both) {
        const auto tf = Clock::now();
        write_ca_txt((out / "ca_result.txt").string(), s.result);
        timing.add_file((out / "ca_result.txt").string(), ms_since(tf));
    }
    if (cfg.output.format == OutputFormat::Bin || cfg.output.format == OutputFormat::Both) {
        const auto tf = Clock::now();
        write_ca_bin((out / "ca_result.bin").string(), s.result);
        timing.add_file((out / "ca_result.bin").string(), ms_since(tf));
    }
    timing.add("save", ms_since(t));
    return s;
}

// Simulation::flowSums / statsFromSums (Simulation.cpp:404-524).  The sums come from the device
// (vca_ca_flow_stats).  The reference's reach is the largest hypot(x - vx, y - vy) over a flow's
// cells and is written rounded to 0.01; the device gives the largest squared distance D, and
// sqrt(D) rounds to the same 0.01 step: hypot and sqrt(D) differ by at most one ulp, while
// 100 sqrt(D) of an integer D never lies within 1e-8 of a rounding boundary k + 0.5.
Json ca_stats(const Config& c, const RunSummary& s, vca_ca* ca) {
    const size_t flows = s.vents.size();
    std::vector<uint64_t> lava(flows + 1, 0), basalt(flows + 1, 0), reach2(flows + 1, 0);
    vcheck(vca_ca_flow_stats(ca, (int)flows, lava.data(), basalt.data(), reach2.data()), "vca_ca_flow_stats");
    std::vector<double> reach(flows + 1, 0.0);
    for (size_t f = 1; f <= flows; ++f) reach[f] = std::sqrt((double)reach2[f]);
    Json j = Json::object();
    j["mode"] = mode_name(c.ca.mode);
    j["steps"] = s.steps;
    j["stopReason"] = stop_text(s.stop);
    uint64_t total = 0, total_lava = 0, min_size = std::numeric_limits<uint64_t>::max(), max_size = 0;
    double max_reach = 0.0;
    Json list = Json::array();
    for (size_t f = 1; f <= flows; ++f) {
        const uint64_t cells = lava[f] + basalt[f];
        total += cells;
        total_lava += lava[f];
        max_reach = std::max(max_reach, reach[f]);
        min_size = std::min(min_size, cells);
        max_size = std::max(max_size, cells);
        if (f <= 10000) {
            const Vent& v = s.vents[f - 1];
            Json e = Json::object();
            e["flowId"] = (unsigned long long)f;
            Json vent = Json::array();
            vent.push_back(v.x);
            vent.push_back(v.y);
            vent.push_back(v.z);
            e["vent"] = vent;
            e["cells"] = (unsigned long long)cells;
            if (c.ca.mode == Mode::Lava) {
                e["lava"] = (unsigned long long)lava[f];
                e["basalt"] = (unsigned long long)basalt[f];
                e["maxReach"] = std::round(reach[f] * 100.0) / 100.0;
            }
            list.push_back(e);
        }
    }
    if (c.ca.mode == Mode::Lava) {
        j["totalLavaVolume"] = (unsigned long long)total;
        j["liquidLava"] = (unsigned long long)total_lava;
        j["maxReach"] = std::round(max_reach * 100.0) / 100.0;
    } else {
        j["grains"] = (unsigned long long)flows;
        j["meanGrainSize"] = flows ? double(total) / double(flows) : 0.0;
        j["minGrainSize"] = (unsigned long long)(flows ? min_size : 0);
        j["maxGrainSize"] = (unsigned long long)max_size;
    }
    j["flows"] = list;
    if (flows > 10000) j["flowsTruncated"] = true;
    j["activeCells"] = Json::array_of(s.active);
    j["changedCells"] = Json::array_of(s.changed);
    return j;
}

Json parallel_json(const Config& c) {
    Json j = Json::object();
    j["threads"] = c.threads;
    j["schedule"] = c.schedule;
    j["chunk"] = c.chunk;
    j["affinity"] = c.affinity;
    return j;
}

// ---------------------------------------------------------------------------------------------
// MC stage (McStage::run / save / statsJson, engine/src/app/McStage.cpp:93-383)
// ---------------------------------------------------------------------------------------------
enum class Cooling { None, SolidOnly, Full };



struct ClassGrains {
    uint64_t grains = 0, cells = 0, largest = 0;
    double mean() const { return grains ? double(cells) / double(grains) : 0.0; }
};

constexpr double kMobilityThreshold = 0.5;  // McStage::kMobilityThreshold (McStage.hpp:61)

// The majority classes of McStage (McStage.cpp:47-66) as vca_mc_grains computes them on the device.
void classes(const vca_mc_grain_stats& g, ClassGrains& hi, ClassGrains& lo) {
    hi.grains = g.high_grains;
    hi.cells = g.high_grain_cells;
    hi.largest = g.high_largest;
    lo.grains = g.low_grains;
    lo.cells = g.low_grain_cells;
    lo.largest = g.low_largest;
}

Json class_json(uint64_t cells, const ClassGrains& a, const ClassGrains& b) {
    Json j = Json::object();
    j["cells"] = (unsigned long long)cells;
    j["grainsStart"] = (unsigned long long)a.grains;
    j["grainsEnd"] = (unsigned long long)b.grains;
    j["meanGrainSizeStart"] = round_to(a.mean(), 3);
    j["meanGrainSizeEnd"] = round_to(b.mean(), 3);
    j["largestGrainEnd"] = (unsigned long long)b.largest;
    return j;
}

// CoolingMobility on the host, for CA results read from a file (engine/src/mc/CoolingMobility.cpp).
std::vector<float> mobility_host(const Microstructure& m, const std::vector<uint8_t>& dom, double mobility_min) {
    uint32_t end = 0;
    for (size_t i = 0; i < dom.size(); ++i)
        if (dom[i]) end = std::max<uint32_t>(end, std::max(m.solid[i], m.arrival[i]));
    std::vector<uint32_t> time(dom.size(), 0);
    uint32_t tmin = std::numeric_limits<uint32_t>::max(), tmax = 0;
    for (size_t i = 0; i < dom.size(); ++i) {
        if (!dom[i]) continue;
        const uint32_t solid = m.type[i] == kBasalt ? m.solid[i] : end;
        const uint32_t arrival = m.arrival[i];
        time[i] = solid > arrival ? solid - arrival : 0;
        tmin = std::min(tmin, time[i]);
        tmax = std::max(tmax, time[i]);
    }
    std::vector<float> mob(dom.size(), 0.0f);
    for (size_t i = 0; i < dom.size(); ++i) {
        if (!dom[i]) continue;
        if (tmax == tmin) {
            mob[i] = 1.0f;
            continue;
        }
        const double norm = double(time[i] - tmin) / double(tmax - tmin);
        mob[i] = (float)(mobility_min + (1.0 - mobility_min) * norm);
    }
    return mob;
}

struct McHandle {
    vca_mc* h = nullptr;
    bool owned = true;
    ~McHandle() {
        if (owned) vca_mc_destroy(h);
    }
};

// ca: the CA handle of an in-memory run (domain and mobility built on the device) or null;
// file: the CA result read for --mc-from, or null; resident: the job server's MC handle, or null.
McSummary run_mc(const Config& cfg, vca_ca* ca, const Microstructure* file, Cooling cooling, Timing& timing,
                 Progress& progress, const std::string& out_dir, vca_mc* resident) {
    McSummary s;
    const bool full = ca == nullptr && file == nullptr;
    s.full = full;
    s.mcs = cfg.mc.mcs;
    s.Q = cfg.mc.Q;
    auto t = Clock::now();
    const Dims dims = full ? cfg.space : (file ? file->dims : cfg.space);
    vca_mc_desc d{};
    d.nx = dims.nx;
    d.ny = dims.ny;
    d.nz = dims.nz;
    d.neighborhood = (int)cfg.neighborhood;
    d.boundary = cfg.boundary == Bc::Periodic ? VCA_BC_PERIODIC : VCA_BC_ABSORBING;
    d.domain_full = full ? 1 : 0;
    d.seed = cfg.seed;
    d.Q = cfg.mc.Q;
    d.J = cfg.mc.J;
    d.kT = cfg.mc.kT;
    d.device = device_ordinal();
    McHandle mc;
    if (resident) {
        mc.h = resident;
        mc.owned = false;
        vcheck(vca_mc_reconfigure(mc.h, &d), "vca_mc_reconfigure");
    } else {
        vcheck(vca_mc_create(&d, &mc.h), "vca_mc_create");
    }
    timing.add_detail("mcCreate", ms_since(t));
    auto td = Clock::now();
    bool have_mobility = false;  // mobility values held by the handle: the byMobility classes exist
    if (full) {
        vcheck(vca_mc_set_domain(mc.h, nullptr), "vca_mc_set_domain");
    } else if (ca) {
        vcheck(vca_mc_set_domain_from_ca(mc.h, ca), "vca_mc_set_domain_from_ca");
        vcheck(vca_mc_set_mobility_from_ca(mc.h, ca, cfg.mc.mobility_min, cfg.mc.mobility_from_cooling ? 1 : 0),
               "vca_mc_set_mobility_from_ca");
        have_mobility = true;
        s.mobility_used = cfg.mc.mobility_from_cooling;
    } else {
        std::vector<uint8_t> dom((size_t)dims.cells());
        for (size_t i = 0; i < dom.size(); ++i) dom[i] = (file->type[i] == kBasalt || file->type[i] == kLava) ? 1 : 0;
        vcheck(vca_mc_set_domain(mc.h, dom.data()), "vca_mc_set_domain");
        if (cooling != Cooling::None) {
            const std::vector<float> cell_mob = mobility_host(*file, dom, cfg.mc.mobility_min);
            vcheck(vca_mc_set_mobility_values(mc.h, cell_mob.data(), cfg.mc.mobility_from_cooling ? 1 : 0),
                   "vca_mc_set_mobility_values");
            have_mobility = true;
            s.mobility_used = cfg.mc.mobility_from_cooling;
        }
        if (cooling == Cooling::None && cfg.mc.mobility_from_cooling)
            s.warnings.push_back("wynik CA bez solidStep/arrivalStep (plik txt): mobilność ze stygnięcia "
                                 "wyłączona, MC jak dla mobilityFromCooling = false");
        if (cooling == Cooling::SolidOnly)
            s.warnings.push_back("ca_result.bin w wersji 1 nie zawiera arrivalStep, czas w stanie płynnym "
                                 "liczony od kroku 0 (= solidStep)");
    }
    timing.add_detail("mcDomainMobility", ms_since(td));
    td = Clock::now();
    vcheck(vca_mc_initialize(mc.h), "vca_mc_initialize");
    timing.add_detail("mcInitialize", ms_since(td));
    vca_mc_info info{};
    vcheck(vca_mc_get_info(mc.h, &info), "vca_mc_get_info");
    s.domain_cells = info.domain_cells;
    if (s.domain_cells == 0)
        s.warnings.push_back(full ? "domena MC jest pusta" : "domena MC jest pusta: wynik CA nie zawiera bazaltu");
    timing.add("mcInit", ms_since(t));

    const bool moore = cfg.neighborhood != Nb::VonNeumann;
    double grains_ms = 0.0;
    auto measure = [&](vca_mc_grain_stats* keep) {
        const auto tm = Clock::now();
        vca_mc_grain_stats g{};
        vcheck(vca_mc_grains(mc.h, moore ? 1 : 0, kMobilityThreshold, &g), "vca_mc_grains");
        grains_ms += ms_since(tm);
        McStats st;
        vca_mc_info mi{};
        vcheck(vca_mc_get_info(mc.h, &mi), "vca_mc_get_info");
        st.mcs = mi.sweeps;
        st.grains = g.grains;
        st.mean = g.grains ? double(g.cells) / double(g.grains) : 0.0;
        vcheck(vca_mc_energy(mc.h, &st.energy), "vca_mc_energy");
        if (keep) *keep = g;
        return st;
    };
    const int snap_every = out_dir.empty() ? 0 : cfg.mc.snapshots_every;
    const fs::path snap_dir = fs::path(out_dir) / "mc_snapshots";
    double snap_ms = 0.0;
    auto snapshot = [&](int k) {
        const auto ts = Clock::now();
        char name[32];
        std::snprintf(name, sizeof(name), "mcs_%06d.bin", k);
        CrystalMap m;
        m.dims = dims;
        m.crystal.resize((size_t)dims.cells());
        vcheck(vca_mc_crystals(mc.h, m.crystal.data()), "vca_mc_crystals");
        write_crystal_bin((snap_dir / name).string(), m);
        snap_ms += ms_since(ts);
    };
    if (snap_every > 0) {
        fs::create_directories(snap_dir);
        snapshot(0);
    }
    double sim_ms = 0.0, stats_ms = 0.0;
    vca_mc_grain_stats start_labels{}, end_labels{};
    t = Clock::now();
    s.history.push_back(measure(&start_labels));
    stats_ms += ms_since(t);
    progress.report("mc", 0, cfg.mc.mcs, true);
    uint64_t att_before = 0, acc_before = 0;
    int k = 0;
    while (k < cfg.mc.mcs) {
        // sweeps up to the next measurement, snapshot or progress point
        int next = std::min(cfg.mc.mcs, (k / cfg.mc.stats_every + 1) * cfg.mc.stats_every);
        if (snap_every > 0) next = std::min(next, (k / snap_every + 1) * snap_every);
        if (progress.on) next = std::min(next, k + 1);
        const auto ts = Clock::now();
        vcheck(vca_mc_sweep(mc.h, next - k, nullptr), "vca_mc_sweep");
        sim_ms += ms_since(ts);
        k = next;
        if (k % cfg.mc.stats_every == 0 || k == cfg.mc.mcs) {
            const auto tm = Clock::now();
            McStats st = measure(k == cfg.mc.mcs ? &end_labels : nullptr);
            vca_mc_info mi{};
            vcheck(vca_mc_get_info(mc.h, &mi), "vca_mc_get_info");
            const uint64_t att = mi.attempts - att_before, acc = mi.accepted - acc_before;
            st.accept_rate = att > 0 ? double(acc) / double(att) : 0.0;
            att_before = mi.attempts;
            acc_before = mi.accepted;
            s.history.push_back(st);
            stats_ms += ms_since(tm);
        }
        if (snap_every > 0 && (k % snap_every == 0 || k == cfg.mc.mcs)) snapshot(k);
        progress.report("mc", k, cfg.mc.mcs, k == cfg.mc.mcs);
    }
    if (cfg.mc.mcs == 0) end_labels = start_labels;
    timing.add("mcSim", sim_ms);
    if (snap_every > 0) {
        timing.add("mcSnapshots", snap_ms);
        timing.add_file(snap_dir.string(), snap_ms);
    }
    double dev_ms = 0.0, color_ms = 0.0;
    uint64_t color_n = 0;
    vca_mc_timing(mc.h, &dev_ms, &color_ms, &color_n);
    timing.add_detail("mcDevice", dev_ms);
    timing.add_detail("mcStatsGrains", grains_ms);

    // stats.json "mc" (McStage::statsJson, McStage.cpp:326-383)
    t = Clock::now();
    vcheck(vca_mc_get_info(mc.h, &info), "vca_mc_get_info");
    const McStats& first = s.history.front();
    const McStats& last = s.history.back();
    Json j = Json::object();
    j["domain"] = full ? "full" : "basalt";
    j["domainCells"] = (unsigned long long)s.domain_cells;
    Json sp = Json::array();
    sp.push_back(dims.nx);
    sp.push_back(dims.ny);
    sp.push_back(dims.nz);
    j["space"] = sp;
    j["Q"] = cfg.mc.Q;
    j["mcs"] = cfg.mc.mcs;
    j["J"] = cfg.mc.J;
    j["kT"] = cfg.mc.kT;
    j["update"] = "checkerboard";
    j["colors"] = info.colors;
    j["neighborhood"] = nb_name(cfg.neighborhood);
    j["boundary"] = bc_name(cfg.boundary);
    j["grainConnectivity"] = moore ? "moore" : "von_neumann";
    j["mobility"] = s.mobility_used ? "cooling" : "off";
    if (s.mobility_used) j["mobilityMin"] = cfg.mc.mobility_min;
    j["grainsStart"] = (unsigned long long)first.grains;
    j["grainsEnd"] = (unsigned long long)last.grains;
    j["meanGrainSizeStart"] = round_to(first.mean, 3);
    j["meanGrainSizeEnd"] = round_to(last.mean, 3);
    j["largestGrainEnd"] = (unsigned long long)end_labels.largest;
    j["energyStart"] = first.energy;
    j["energyEnd"] = last.energy;
    j["attempts"] = (unsigned long long)info.attempts;
    j["accepted"] = (unsigned long long)info.accepted;
    j["acceptedUphill"] = (unsigned long long)info.uphill;
    if (have_mobility) {
        ClassGrains hs, ls, he, le;
        classes(start_labels, hs, ls);
        classes(end_labels, he, le);
        const uint64_t hi_cells = start_labels.high_cells;
        Json bm = Json::object();
        bm["threshold"] = kMobilityThreshold;
        bm["mobilityMin"] = cfg.mc.mobility_min;
        bm["rule"] = "ziarno należy do klasy, w której jest większość jego komórek";
        bm["high"] = class_json(hi_cells, hs, he);
        bm["low"] = class_json(s.domain_cells - hi_cells, ls, le);
        j["byMobility"] = bm;
    }
    s.stats = j;
    s.crystals.dims = dims;
    s.crystals.crystal.resize((size_t)dims.cells());
    vcheck(vca_mc_crystals(mc.h, s.crystals.crystal.data()), "vca_mc_crystals");
    timing.add("mcStats", stats_ms + ms_since(t));
    return s;
}

// McStage::save (McStage.cpp:303-324).
void save_mc(const Config& cfg, const McSummary& s, const std::string& out_dir, Timing& timing) {
    const auto t = Clock::now();
    const fs::path out(out_dir);
    if (cfg.output.format == OutputFormat::Txt || cfg.output.format == OutputFormat::Both) {
        const auto tf = Clock::now();
        write_crystal_txt((out / "mc_result.txt").string(), s.crystals);
        timing.add_file((out / "mc_result.txt").string(), ms_since(tf));
    }
    if (cfg.output.format == OutputFormat::Bin || cfg.output.format == OutputFormat::Both) {
        const auto tf = Clock::now();
        write_crystal_bin((out / "mc_result.bin").string(), s.crystals);
        timing.add_file((out / "mc_result.bin").string(), ms_since(tf));
    }
    const auto tf = Clock::now();
    const std::string csv = (out / "mc_stats.csv").string();
    std::ofstream f(csv);
    if (!f) throw std::runtime_error("Nie można utworzyć pliku: " + csv);
    f << "mcs,grains,meanGrainSize,energy,acceptRate\n";
    char line[160];
    for (const McStats& st : s.history) {
        std::snprintf(line, sizeof(line), "%d,%llu,%.4f,%.3f,%.6f\n", st.mcs, (unsigned long long)st.grains, st.mean,
                      st.energy, st.accept_rate);
        f << line;
    }
    if (!f) throw std::runtime_error("Błąd zapisu pliku: " + csv);
    f.close();
    timing.add_file(csv, ms_since(tf));
    timing.add("mcSave", ms_since(t));
}

// ---------------------------------------------------------------------------------------------
// A run: engine --config F --out D (Simulation::runFromCli, Simulation.cpp:526-683) and --mc-from.
// ---------------------------------------------------------------------------------------------
void env_info(Timing& timing) {
    std::ifstream in("/proc/cpuinfo");
    std::string line, cpu = "unknown";
    while (std::getline(in, line))
        if (line.rfind("model name", 0) == 0) {
            const auto c = line.find(':');
            if (c != std::string::npos) cpu = line.substr(c + 2);
            break;
        }
    timing.set("cpu", cpu);
    timing.set("compiler", std::string("GCC ") + __VERSION__);
    timing.set("build", "Release");
    timing.set("gpuLibrary", vca_version());
}

Rss read_rss() {
    Rss r;
    std::ifstream in("/proc/self/status");
    std::string line;
    while (std::getline(in, line)) {
        const bool cur = line.rfind("VmRSS:", 0) == 0, hwm = line.rfind("VmHWM:", 0) == 0;
        if (!cur && !hwm) continue;
        const uint64_t kb = std::strtoull(line.c_str() + 6, nullptr, 10);
        (cur ? r.current : r.peak) = kb * 1024;
        r.ok = true;
    }
    return r;
}

// times.json "memory" (TimingReport::recordMemory, engine/src/io/TimingReport.cpp:104-138): the host
// process; the grid itself lives in device memory.
void memory_info(Timing& timing, const Rss& start) {
    const Rss now = read_rss();
    Json m = Json::object();
    m["method"] = "procfs";
    if (now.ok) {
        m["startRssBytes"] = (unsigned long long)start.current;
        m["endRssBytes"] = (unsigned long long)now.current;
        m["peakRssBytes"] = (unsigned long long)now.peak;
    }
    timing.set("memory", m);
}

// The CA stage, its statistics, the MC stage and every result file of one job (the run of
// Simulation::runFromCli, Simulation.cpp:526-683, after the config is read).  With an empty out_dir
// nothing is written: the job server hands the results on as digests.
JobOutcome run_job(const Config& cfg, const std::string& out_dir, Timing& timing, Progress& progress,
                   const RunHandles& res, Clock::time_point start, const Rss& rss_start) {
    JobOutcome job;
    const bool files = !out_dir.empty();
    const fs::path out(out_dir);
    auto t = Clock::now();
    if (files) {
        write_json((out / "config_used.json").string(), cfg.effective);
        timing.add_file((out / "config_used.json").string(), ms_since(t));
    }
    RunSummary& s = job.ca;
    s.ca_ran = !cfg.mc.full_only();
    CaHandle ca;
    Json stats = Json::object();
    if (s.ca_ran) {
        s = run_ca(cfg, out_dir, timing, progress, ca, res);
        s.ca_ran = true;
        t = Clock::now();
        stats = ca_stats(cfg, s, ca.h);
        timing.add("caStats", ms_since(t));
        if (res.ca_done) res.ca_done();
    }
    stats["parallel"] = parallel_json(cfg);
    McSummary& mc = job.mc;
    job.mc_ran = cfg.mc.enabled;
    if (job.mc_ran) {
        mc = run_mc(cfg, s.ca_ran ? ca.h : nullptr, nullptr, Cooling::Full, timing, progress, out_dir, res.mc);
        progress.report("save", 0, 1, true);
        if (files) save_mc(cfg, mc, out_dir, timing);
        stats["mc"] = mc.stats;
    }
    job.stats = stats;
    t = Clock::now();
    if (files) {
        write_json((out / "stats.json").string(), stats);
        timing.add_file((out / "stats.json").string(), ms_since(t));
    }
    timing.add(job.mc_ran ? "mcSave" : "save", ms_since(t));
    timing.add("total", ms_since(start));
    timing.set("cells", (unsigned long long)cfg.space.cells());
    Json sp = Json::array();
    sp.push_back(cfg.space.nx);
    sp.push_back(cfg.space.ny);
    sp.push_back(cfg.space.nz);
    timing.set("space", sp);
    timing.set("neighborhood", nb_name(cfg.neighborhood));
    timing.set("boundary", bc_name(cfg.boundary));
    if (s.ca_ran) {
        timing.set("steps", s.steps);
        timing.set("grid", cfg.grid);
        timing.set("mode", mode_name(cfg.ca.mode));
        timing.set("stopReason", stop_text(s.stop));
    } else {
        timing.set("mode", "mc_full");
    }
    if (job.mc_ran) {
        timing.set("mcDomain", mc.full ? "full" : "basalt");
        timing.set("mcs", mc.mcs);
        timing.set("domainCells", (unsigned long long)mc.domain_cells);
        timing.set("Q", mc.Q);
        timing.set("mcMobility", mc.mobility_used);
    }
    env_info(timing);
    memory_info(timing, rss_start);
    timing.record_files();
    if (files) write_json((out / "times.json").string(), timing.to_json());
    return job;
}

int run_from_cli(const CliOptions& opt, Clock::time_point start) {
    const Rss rss_start = read_rss();
    Timing timing;
    timing.detail = opt.timing_detail;
    Progress progress;
    progress.on = opt.progress;
    auto t = Clock::now();
    Config cfg = Config::load(opt.config, opt.overrides);
    timing.add("readConfig", ms_since(t));
    timing.set("threads", cfg.threads);
    timing.set("schedule", cfg.schedule);
    timing.set("chunk", cfg.chunk);
    timing.set("affinity", cfg.affinity);
    for (const std::string& w : cfg.warnings) std::cerr << "Ostrzeżenie: " << w << '\n';
    std::string out_dir = opt.out;
    if (out_dir.empty()) {
        const std::string stem = opt.config.empty() ? "default" : fs::path(opt.config).stem().string();
        out_dir = (fs::path("results") / stem).string();
    }
    fs::create_directories(out_dir);
    const fs::path out(out_dir);
    auto common = [&](const Config& c, const Dims& d) {
        timing.set("cells", (unsigned long long)d.cells());
        Json sp = Json::array();
        sp.push_back(d.nx);
        sp.push_back(d.ny);
        sp.push_back(d.nz);
        timing.set("space", sp);
        timing.set("neighborhood", nb_name(c.neighborhood));
        timing.set("boundary", bc_name(c.boundary));
    };
    auto mc_info = [&](const McSummary& mc) {
        timing.set("mcDomain", mc.full ? "full" : "basalt");
        timing.set("mcs", mc.mcs);
        timing.set("domainCells", (unsigned long long)mc.domain_cells);
        timing.set("Q", mc.Q);
        timing.set("mcMobility", mc.mobility_used);
    };

    if (!opt.mc_from.empty()) {
        // Simulation::runMcFrom (Simulation.cpp:334-402)
        if (cfg.mc.full)
            throw ConfigError("--mc-from krystalizuje wynik CA z pliku, więc wymaga mc.domain = \"basalt\" (podano \"" +
                              std::string(cfg.mc.full ? "full" : "basalt") + "\")");
        std::vector<std::string> warnings;
        if (!cfg.mc.enabled) {
            warnings.push_back("mc.enabled = false, a w trybie --mc-from Monte Carlo jest uruchamiane zawsze");
            cfg.mc.enabled = true;
        }
        t = Clock::now();
        ResultSource src;
        const Microstructure ca = read_ca_folder(opt.mc_from, &src);
        timing.add("readInput", ms_since(t));
        if (ca.dims != cfg.space && cfg.space_from_user)
            warnings.push_back("wymiary z pliku " + std::to_string(ca.dims.nx) + " x " + std::to_string(ca.dims.ny) +
                               " x " + std::to_string(ca.dims.nz) + " różnią się od space z configu (" +
                               std::to_string(cfg.space.nx) + " x " + std::to_string(cfg.space.ny) + " x " +
                               std::to_string(cfg.space.nz) + "); obowiązują wymiary z pliku");
        cfg.space = ca.dims;
        if (cfg.neighborhood == Nb::Hexagonal && !cfg.space.is2d())
            throw ConfigError("Sąsiedztwo „hexagonal” jest zdefiniowane tylko w 2D, a wynik CA z pliku jest 3D");
        Json space = Json::object();
        space["nx"] = ca.dims.nx;
        space["ny"] = ca.dims.ny;
        space["nz"] = ca.dims.nz;
        cfg.effective["space"] = space;
        cfg.effective["mc"]["enabled"] = true;
        cfg.effective["_mcFrom"] = fs::absolute(fs::path(opt.mc_from)).lexically_normal().string();
        t = Clock::now();
        write_json((out / "config_used.json").string(), cfg.effective);
        timing.add_file((out / "config_used.json").string(), ms_since(t));
        const Cooling cooling = src.has_arrival ? Cooling::Full : src.has_solid ? Cooling::SolidOnly : Cooling::None;
        McSummary mc = run_mc(cfg, nullptr, &ca, cooling, timing, progress, out_dir, nullptr);
        mc.warnings.insert(mc.warnings.begin(), warnings.begin(), warnings.end());
        progress.report("save", 0, 1, true);
        save_mc(cfg, mc, out_dir, timing);
        t = Clock::now();
        Json stats = Json::object();
        Json source = Json::object();
        source["folder"] = cfg.effective.get("_mcFrom");
        source["file"] = src.path;
        source["format"] = src.format;
        source["version"] = (unsigned long long)src.version;
        source["coolingData"] = cooling == Cooling::Full ? "solidStep+arrivalStep" : cooling == Cooling::SolidOnly ? "solidStep" : "brak";
        stats["source"] = source;
        stats["parallel"] = parallel_json(cfg);
        stats["mc"] = mc.stats;
        write_json((out / "stats.json").string(), stats);
        timing.add_file((out / "stats.json").string(), ms_since(t));
        timing.add("mcSave", ms_since(t));
        timing.add("total", ms_since(start));
        common(cfg, mc.crystals.dims);
        timing.set("mode", "mc_from");
        timing.set("mcFrom", opt.mc_from);
        mc_info(mc);
        env_info(timing);
        memory_info(timing, rss_start);
        timing.record_files();
        write_json((out / "times.json").string(), timing.to_json());
        for (const std::string& w : mc.warnings) std::cerr << "Ostrzeżenie: " << w << '\n';
        std::cout << "=== Monte Carlo on a CA result from a file done ===\nInput          " << opt.mc_from << "\n"
                  << "Space          " << cfg.space.nx << " x " << cfg.space.ny << " x " << cfg.space.nz << "\n"
                  << "Grains (MC)    " << mc.history.front().grains << " -> " << mc.history.back().grains << "\n"
                  << "Results        " << out_dir << '\n';
        return kExitOk;
    }

    JobOutcome job = run_job(cfg, out_dir, timing, progress, RunHandles{}, start, rss_start);
    for (const std::string& w : job.mc.warnings) std::cerr << "Ostrzeżenie: " << w << '\n';
    const RunSummary& s = job.ca;
    const McSummary& mc = job.mc;
    const bool mc_ran = job.mc_ran;

    std::ostringstream os;
    os << "=== Simulation done ===\n";
    os << "Space          " << cfg.space.nx << " x " << cfg.space.ny << " x " << cfg.space.nz << " ("
       << (cfg.space.is2d() ? "2D" : "3D") << ", " << cfg.space.cells() << " cells)\n";
    if (s.ca_ran) {
        os << "Mode           " << mode_name(cfg.ca.mode) << (mc_ran ? " + MC" : "") << "\n";
        os << "Steps          " << s.steps << " (stop: " << stop_text(s.stop) << ")\n";
    } else {
        os << "Mode           Monte Carlo on the whole space (no terrain, no CA)\n";
    }
    if (mc_ran)
        os << "Grains (MC)    " << mc.history.front().grains << " -> " << mc.history.back().grains << ", energy "
           << fixed(mc.history.front().energy, 0) << " -> " << fixed(mc.history.back().energy, 0) << "\n";
    os << "Times [ms]     ";
    const char* sep = "";
    for (const auto& sct : timing.sections) {
        os << sep << sct.first << ' ' << fixed(sct.second, 2);
        sep = " | ";
    }
    os << "\nResults        " << out_dir << '\n';
    std::cout << os.str();
    return kExitOk;
}

// --validate (ConfigCheck::validate, engine/src/app/ConfigCheck.cpp:46-62).
int validate(const CliOptions& opt) {
    Json r = Json::object();
    Json errors = Json::array(), warnings = Json::array();
    try {
        const Config cfg = Config::load(opt.config, opt.overrides);
        for (const auto& w : cfg.warnings) warnings.push_back(w);
        if (!opt.mc_from.empty()) {
            if (cfg.mc.full)
                errors.push_back(std::string("--mc-from krystalizuje wynik CA z pliku, więc wymaga mc.domain = \"basalt\" ") +
                                 "(podano \"full\")");
            if (!cfg.mc.enabled)
                warnings.push_back("mc.enabled = false, a w trybie --mc-from Monte Carlo jest uruchamiane zawsze");
            const fs::path dir(opt.mc_from);
            if (!fs::is_directory(dir)) errors.push_back("Folder wyniku CA (--mc-from) nie istnieje: " + opt.mc_from);
            else if (!fs::exists(dir / "ca_result.bin") && !fs::exists(dir / "ca_result.txt"))
                errors.push_back("W folderze " + opt.mc_from + " nie ma ca_result.bin ani ca_result.txt");
        } else if (!cfg.mc.full_only() && cfg.ca.mode == Mode::Lava && cfg.terrain.type == TerrainType::File) {
            (void)build_terrain(cfg);
        }
    } catch (const std::exception& e) {
        errors.push_back(e.what());
    }
    r["ok"] = errors.size() == 0;
    r["errors"] = errors;
    r["warnings"] = warnings;
    std::cout << r.dump(2) << '\n';
    return errors.size() == 0 ? kExitOk : kExitConfig;
}

// ---------------------------------------------------------------------------------------------
// --batch (BatchRunner, engine/src/app/Batch.cpp:147-418): every *.json of a folder (name order,
// skipping _*.json and series.json) in its own child process, output in <out>/<name>/ with
// engine.log, a batch_summary.csv after every run, exit code 5 when any run failed.
// ---------------------------------------------------------------------------------------------
std::string csv_cell(const std::string& s) {
    if (s.find_first_of(",\"\n\r") == std::string::npos) return s;
    std::string out = "\"";
    for (char c : s) {
        if (c == '"') out += '"';
        out += c;
    }
    return out + '"';
}

Json read_json_file(const fs::path& p) {
    std::ifstream in(p);
    if (!in) return Json();
    std::stringstream ss;
    ss << in.rdbuf();
    try {
        return Json::parse(ss.str(), true);
    } catch (...) {
        return Json();
    }
}

std::string jfield(const Json& j, const std::string& key) {
    if (!j.is_object() || !j.contains(key)) return "";
    const Json& v = j.get(key);
    if (v.is_string()) return v.as_string();
    if (v.is_number() || v.is_bool()) return v.dump();
    return "";
}

int run_child(const std::string& exe, const std::vector<std::string>& args, const fs::path& log) {
    std::vector<char*> argv;
    argv.push_back(const_cast<char*>(exe.c_str()));
    for (const std::string& a : args) argv.push_back(const_cast<char*>(a.c_str()));
    argv.push_back(nullptr);
    posix_spawn_file_actions_t fa;
    posix_spawn_file_actions_init(&fa);
    posix_spawn_file_actions_addopen(&fa, 1, log.c_str(), O_WRONLY | O_CREAT | O_APPEND, 0644);
    posix_spawn_file_actions_adddup2(&fa, 1, 2);
    pid_t pid = 0;
    const int rc = posix_spawn(&pid, exe.c_str(), &fa, nullptr, argv.data(), environ);
    posix_spawn_file_actions_destroy(&fa);
    if (rc != 0) return -1;
    int status = 0;
    if (waitpid(pid, &status, 0) < 0) return -1;
    if (WIFEXITED(status)) return WEXITSTATUS(status);
    return 128 + (WIFSIGNALED(status) ? WTERMSIG(status) : 0);
}

std::string self_exe() {
    char buf[4096];
    const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
    if (n <= 0) return "engine";
    buf[n] = 0;
    return buf;
}

int run_batch(const CliOptions& opt) {
    fs::path folder(opt.batch);
    if (!fs::is_directory(folder)) throw CliError("--batch: folder z configami nie istnieje: " + opt.batch);
    if (folder.filename().empty()) folder = folder.parent_path();
    const fs::path out = opt.out.empty() ? fs::path("results") / folder.filename() : fs::path(opt.out);
    struct Item {
        std::string name;
        fs::path config, out;
    };
    std::vector<Item> items;
    for (const auto& e : fs::directory_iterator(folder)) {
        if (!e.is_regular_file()) continue;
        const fs::path& p = e.path();
        std::string ext = p.extension().string();
        std::transform(ext.begin(), ext.end(), ext.begin(), [](unsigned char c) { return (char)std::tolower(c); });
        const std::string stem = p.stem().string();
        if (ext != ".json" || stem.empty() || stem[0] == '_' || p.filename() == "series.json") continue;
        items.push_back(Item{stem, p, out / stem});
    }
    std::sort(items.begin(), items.end(), [](const Item& a, const Item& b) { return a.name < b.name; });
    if (items.empty())
        throw ConfigError("W folderze " + opt.batch + " nie ma plików konfiguracyjnych *.json "
                          "(series.json i pliki _*.json są pomijane)");
    fs::create_directories(out);
    std::vector<std::string> extra;
    for (const std::string& o : opt.overrides) {
        extra.push_back("--set");
        extra.push_back(o);
    }
    if (opt.timing_detail) extra.push_back("--timing-detail");
    if (opt.thread_stats) extra.push_back("--thread-stats");
    const std::string exe = self_exe();
    const char* const sections[] = {"readConfig", "readInput", "allocate", "terrain", "vents", "caSim", "snapshots",
                                    "save", "mcInit", "mcSim", "mcStats", "mcSave", "total"};
    std::vector<std::string> cols = {"name", "status", "exitCode", "error", "mode", "nx", "ny", "nz", "cells", "grid",
                                     "neighborhood", "boundary", "seeds", "steps", "stopReason", "mcs", "Q", "domainCells"};
    for (const char* s : sections) cols.emplace_back(s);
    for (const char* c : {"wallMs", "caResultTxtBytes", "caResultBinBytes", "mcResultTxtBytes", "mcResultBinBytes",
                          "outputBytes", "compiler", "build", "config", "outDir"})
        cols.emplace_back(c);
    std::vector<std::vector<std::string>> rows;
    Progress progress;
    progress.on = opt.progress;
    progress.report("batch", 0, (long long)items.size(), true);
    bool any_failed = false;
    for (size_t i = 0; i < items.size(); ++i) {
        const Item& it = items[i];
        fs::create_directories(it.out);
        const fs::path log = it.out / "engine.log";
        {
            std::ofstream head(log, std::ios::trunc);
            head << "# engine --batch: " << it.name << "\n# command: " << exe << " --config " << it.config.string()
                 << " --out " << it.out.string();
            for (const std::string& a : extra) head << ' ' << a;
            head << '\n';
        }
        std::vector<std::string> args = {"--config", it.config.string(), "--out", it.out.string()};
        args.insert(args.end(), extra.begin(), extra.end());
        const auto t = Clock::now();
        const int code = run_child(exe, args, log);
        const double wall = ms_since(t);
        std::string error;
        if (code < 0) {
            error = "the run did not start";
        } else if (code != 0) {
            std::ifstream in(log);
            std::string line;
            while (std::getline(in, line))
                if (line.rfind("Błąd", 0) == 0) error = line;  // the stderr prefix of every error
            if (error.empty()) error = "the engine exited with code " + std::to_string(code);
        }
        {
            std::ofstream tail(log, std::ios::app);
            tail << "# end: exit code " << code << ", time " << fixed(wall / 1000.0, 2) << " s\n";
        }
        const bool ok = error.empty();
        any_failed = any_failed || !ok;
        const Json times = ok ? read_json_file(it.out / "times.json") : Json();
        const Json cfgj = ok ? read_json_file(it.out / "config_used.json") : Json();
        const std::string mode = jfield(times, "mode");
        std::vector<std::string> row = {it.name, ok ? "ok" : "error", std::to_string(code), error, mode};
        for (int a = 0; a < 3; ++a) {
            const Json* sp = times.is_object() ? times.find("space") : nullptr;
            row.push_back(sp && sp->is_array() && sp->size() == 3 ? (*sp)[(size_t)a].dump() : "");
        }
        for (const char* k : {"cells", "grid", "neighborhood", "boundary"}) row.push_back(jfield(times, k));
        const bool ca_ran = mode == "lava" || mode == "classic";
        row.push_back(ca_ran && cfgj.is_object() && cfgj.contains("vents") ? jfield(cfgj.get("vents"), "count") : "");
        for (const char* k : {"steps", "stopReason", "mcs", "Q", "domainCells"}) row.push_back(jfield(times, k));
        for (const char* s : sections) row.push_back(jfield(times, s));
        row.push_back(fixed(wall, 3));
        uint64_t total_bytes = 0;
        const Json* files = times.is_object() ? times.find("files") : nullptr;
        for (const char* f : {"ca_result.txt", "ca_result.bin", "mc_result.txt", "mc_result.bin"})
            row.push_back(files && files->contains(f) ? jfield(files->get(f), "bytes") : "");
        if (files)
            for (const auto& kv : files->members())
                if (kv.second.contains("bytes")) total_bytes += kv.second.get("bytes").as_u64();
        row.push_back(files ? std::to_string(total_bytes) : "");
        row.push_back(jfield(times, "compiler"));
        row.push_back(jfield(times, "build"));
        row.push_back(it.config.generic_string());
        row.push_back(it.out.generic_string());
        rows.push_back(row);
        {
            std::ofstream f(out / "batch_summary.csv", std::ios::trunc);
            if (!f) throw std::runtime_error("Nie można zapisać podsumowania serii: " + (out / "batch_summary.csv").string());
            for (size_t c = 0; c < cols.size(); ++c) f << (c ? "," : "") << cols[c];
            f << '\n';
            for (const auto& r : rows) {
                for (size_t c = 0; c < r.size(); ++c) f << (c ? "," : "") << csv_cell(r[c]);
                f << '\n';
            }
        }
        std::cout << '[' << (i + 1) << '/' << items.size() << "] " << it.name << ' '
                  << (ok ? "ok (" + fixed(wall / 1000.0, 2) + " s)" : "ERROR " + error) << '\n'
                  << std::flush;
        progress.report("batch", (long long)(i + 1), (long long)items.size(), true);
    }
    return any_failed ? kExitBatch : kExitOk;
}

}  // namespace eng

int main(int argc, char** argv) {
    using namespace eng;
    const auto start = Clock::now();
    try {
        const CliOptions opt = parse_cli(argc, argv);
        if (opt.help) {
            std::cout << usage();
            return kExitOk;
        }
        if (opt.print_defaults) {
            std::cout << Config::defaults_json().dump(2) << '\n';
            return kExitOk;
        }
        if (opt.validate) return validate(opt);
        if (!opt.batch.empty()) return run_batch(opt);
        if (opt.serve) return run_server(opt.slots, opt.budget_gb, opt.serve_batch);
        return run_from_cli(opt, start);
    } catch (const CliError& e) {
        std::cerr << "Błąd argumentów: " << e.what() << "\n\n" << usage();
        return kExitArgs;
    } catch (const ConfigError& e) {
        std::cerr << "Błąd konfiguracji: " << e.what() << '\n';
        return kExitConfig;
    } catch (const std::exception& e) {
        std::cerr << "Błąd: " << e.what() << '\n';
        return kExitOther;
    }
}

// job.hpp -- what one engine job is made of, shared by the single run, the batch runner and the
// job server (engine --serve): timing sections, progress lines, the CA and MC summaries, and
// run_job, which runs a configured job on given or new device handles.
#pragma once

#include <chrono>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <functional>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

#include "model.hpp"
#include "vca.h"

namespace eng {

namespace fs = std::filesystem;
using Clock = std::chrono::steady_clock;
inline double ms_since(Clock::time_point t) { return std::chrono::duration<double, std::milli>(Clock::now() - t).count(); }

inline double round_to(double v, int decimals) {
    const double f = std::pow(10.0, decimals);
    return std::round(v * f) / f;
}

// ---------------------------------------------------------------------------------------------
// times.json (engine/src/io/TimingReport.cpp:140-157): sections in ms (summed), then info.
// ---------------------------------------------------------------------------------------------
struct Timing {
    std::vector<std::pair<std::string, double>> sections;
    Json info = Json::object();
    std::vector<std::pair<std::string, double>> files;
    std::vector<std::pair<std::string, double>> details;
    bool detail = false;
    void add(const std::string& name, double ms) {
        for (auto& s : sections)
            if (s.first == name) {
                s.second += ms;
                return;
            }
        sections.emplace_back(name, ms);
    }
    void add_detail(const std::string& name, double ms) { details.emplace_back(name, ms); }
    void add_file(const std::string& path, double ms) { files.emplace_back(path, ms); }
    void set(const std::string& k, Json v) { info[k] = std::move(v); }
    Json to_json() const {
        Json j = Json::object();
        j["unit"] = "ms";
        for (const auto& s : sections) j[s.first] = round_to(s.second, 3);
        for (const auto& kv : info.members()) j[kv.first] = kv.second;
        if (detail) {
            Json d = Json::object();
            d["unit"] = "ms";
            for (const auto& x : details) d[x.first] = round_to(x.second, 3);
            j["detail"] = d;
        }
        return j;
    }
    void record_files() {
        Json f = Json::object();
        for (const auto& r : files) {
            std::error_code ec;
            const uint64_t bytes = fs::is_regular_file(r.first, ec) ? (uint64_t)fs::file_size(r.first, ec) : 0;
            Json e = Json::object();
            e["bytes"] = (unsigned long long)bytes;
            e["writeMs"] = round_to(r.second, 3);
            f[fs::path(r.first).filename().string()] = e;
        }
        set("files", f);
    }
};

// PROGRESS lines for a parent process (engine/src/app/Progress.hpp:20-54).
struct Progress {
    bool on = false;
    Clock::time_point last = Clock::now() - std::chrono::hours(1);
    void report(const char* stage, long long done, long long total, bool force = false, const char* key = nullptr,
                uint64_t value = 0) {
        if (!on || (!force && ms_since(last) < 500.0)) return;
        std::cout << "PROGRESS " << stage << ' ' << done << '/' << total;
        if (key) std::cout << ' ' << key << '=' << value;
        std::cout << '\n' << std::flush;
        last = Clock::now();
    }
};

// CA stage (Simulation::runWith, engine/src/app/Simulation.cpp:158-292)
struct RunSummary {
    bool ca_ran = true;
    int steps = 0;
    int stop = 0;
    std::vector<uint64_t> active, changed;
    Microstructure result;
    std::vector<Vent> vents;
};

// MC stage (McStage::run, engine/src/app/McStage.cpp:93-383)
struct McStats {
    int mcs = 0;
    uint64_t grains = 0;
    double mean = 0.0, energy = 0.0, accept_rate = 0.0;
};

struct McSummary {
    bool full = false;
    int mcs = 0, Q = 0;
    uint64_t domain_cells = 0;
    bool mobility_used = false;
    std::vector<std::string> warnings;
    std::vector<McStats> history;
    Json stats;
    CrystalMap crystals;
};

// Resident set of this process from /proc/self/status (VmRSS, VmHWM), bytes.
struct Rss {
    uint64_t current = 0, peak = 0;
    bool ok = false;
};
Rss read_rss();

// Device handles and hooks of a run: the job server passes its resident handles (reconfigured for
// each job, no allocation), a CA runner that steps the grid inside the shared batch, and a hook
// called once the CA stage is done; the single run leaves them empty (new handles, vca_ca_run).
struct RunHandles {
    vca_ca* ca = nullptr;
    vca_mc* mc = nullptr;
    std::function<void(vca_ca*)> ca_run;
    std::function<void()> ca_done;
};

struct JobOutcome {
    RunSummary ca;
    McSummary mc;
    bool mc_ran = false;
    Json stats;
};

JobOutcome run_job(const Config& cfg, const std::string& out_dir, Timing& timing, Progress& progress,
                   const RunHandles& res, Clock::time_point start, const Rss& rss_start);
vca_ca_desc ca_desc(const Config& c);
const char* stop_text(int s);
int run_server(int slots, double budget_gb, bool batched);
extern bool g_use_tuning;  // launch shapes from the tuned table (single runs)

}  // namespace eng

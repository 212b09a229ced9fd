// serve.cpp -- engine --serve: a job server for engine configs that arrive over time.
//
// The reference runs one engine process per job: its batch runner goes through a folder one config
// after another (engine/src/app/Batch.cpp:147-246) and its GUI queue starts one job when the
// previous one ends (gui/jobs.py).  Here one process keeps the GPU busy with many jobs at once:
//
//  * requests are JSON lines on stdin, {"id": ..., "config": "<file.json>" | "json": {...},
//    "set": ["key=value", ...], "out": "<folder>"}, read by the same config parser as a single run
//    (defaults <- file <- --set overrides, the same validation and messages);
//  * a job is admitted when a worker is free and device memory for it fits the budget: jobs run on
//    resident handles (CA + MC) of a capacity class (each axis rounded up to 2^k or 3 * 2^(k-1)); a
//    job reuses an idle handle of its class or larger, a new handle is allocated only while the
//    allocated bytes stay within the budget, and idle handles are freed to make room;
//  * the CA stage of every admitted job joins one shared batch (vca_ca_batch): all running grids
//    step together, three launches per step for all of them, and a job leaves the batch when its stop
//    rule holds; terrain, statistics, the MC stage and the results run on the worker's own streams,
//    overlapping with the batch;
//  * each finished job writes the reference's result files into its "out" folder (none without one)
//    and answers with one JSON line on stdout: its times relative to the server start, its step count
//    and digests of its ca_result.bin and mc_result.bin bytes.
//
// Every job's results are those of a single run of the same config: the batch steps each grid
// exactly as vca_ca_run does.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>

#include "job.hpp"

namespace eng {

namespace {

// A 64-bit digest of a byte string for equality checks (four lanes of multiply-rotate mixing over
// 32-byte blocks, then the tail and the length; not a cryptographic hash).
class Digest {
public:
    void update(const void* data, size_t n) {
        const unsigned char* p = static_cast<const unsigned char*>(data);
        total_ += n;
        if (fill_ > 0) {  // complete the staged block first
            const size_t take = std::min(n, sizeof(buf_) - fill_);
            std::memcpy(buf_ + fill_, p, take);
            fill_ += take;
            p += take;
            n -= take;
            if (fill_ < sizeof(buf_)) return;
            block(buf_);
            fill_ = 0;
        }
        // whole blocks straight from the input; the tail is staged
        for (; n >= sizeof(buf_); p += sizeof(buf_), n -= sizeof(buf_)) block(p);
        std::memcpy(buf_, p, n);
        fill_ = n;
    }
    std::string hex() const {
        uint64_t h = (lane_[0] * 3) ^ (lane_[1] * 5) ^ (lane_[2] * 7) ^ (lane_[3] * 11);
        for (size_t i = 0; i < fill_; ++i) h = (h ^ buf_[i]) * 0x100000001B3ULL;
        h ^= total_;
        h = mix(h);
        char s[17];
        std::snprintf(s, sizeof(s), "%016llx", (unsigned long long)h);
        return s;
    }

private:
    static uint64_t rotl(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }
    static uint64_t mix(uint64_t x) {
        x ^= x >> 33;
        x *= 0xFF51AFD7ED558CCDULL;
        x ^= x >> 33;
        x *= 0xC4CEB9FE1A85EC53ULL;
        return x ^ (x >> 33);
    }
    void block(const unsigned char* b) {
        for (int i = 0; i < 4; ++i) {
            uint64_t w;
            std::memcpy(&w, b + 8 * i, 8);
            lane_[i] = rotl(lane_[i] ^ (w * 0x9E3779B97F4A7C15ULL), 31) * 0xC2B2AE3D27D4EB4FULL;
        }
    }
    uint64_t lane_[4] = {0x243F6A8885A308D3ULL, 0x13198A2E03707344ULL, 0xA4093822299F31D0ULL, 0x082EFA98EC4E6C89ULL};
    unsigned char buf_[32] = {};
    size_t fill_ = 0;
    uint64_t total_ = 0;
};

// The bytes of ca_result.bin / mc_result.bin (ResultWriter.cpp:155-167, 204-213) as digests.
std::string ca_digest(const Microstructure& m) {
    Digest d;
    const char magic[4] = {'V', 'O', 'L', 'C'};
    const uint32_t version = 2;
    const int32_t dims[3] = {m.dims.nx, m.dims.ny, m.dims.nz};
    d.update(magic, 4);
    d.update(&version, 4);
    d.update(dims, 12);
    d.update(m.type.data(), m.type.size());
    d.update(m.flow.data(), 4 * m.flow.size());
    d.update(m.temp.data(), 4 * m.temp.size());
    d.update(m.solid.data(), 2 * m.solid.size());
    d.update(m.arrival.data(), 2 * m.arrival.size());
    return d.hex();
}
std::string mc_digest(const CrystalMap& c) {
    Digest d;
    const char magic[4] = {'V', 'M', 'C', '1'};
    const int32_t dims[3] = {c.dims.nx, c.dims.ny, c.dims.nz};
    d.update(magic, 4);
    d.update(dims, 12);
    d.update(c.crystal.data(), 4 * c.crystal.size());
    return d.hex();
}

struct Request {
    std::string id;
    std::string error;  // set when the request or its config was refused
    Config cfg;
    std::string out;
    double arrival_ms = 0.0;
};

// Capacity class of an axis: the next of 2^k or 3 * 2^(k-1) at or above n.
int class_side(int n, int floor_) {
    int c = floor_;
    while (c < n) {
        const int up = (c & (c - 1)) == 0 ? c + c / 2 : (c / 3) * 4;  // 2^k -> 3*2^(k-1) -> 2^(k+1)
        c = std::max(up, c + 1);
    }
    return c;
}

struct Slot {
    vca_ca* ca = nullptr;
    vca_mc* mc = nullptr;
    Dims cap;
    bool lava = true;
    uint64_t bytes = 0;
    bool busy = false;
    uint64_t used = 0;  // admission counter when it was last taken
};

class Server {
public:
    Server(int workers, uint64_t budget, bool batched) : workers_(workers), budget_(budget), batched_(batched) {}

    int run() {
        start_ = Clock::now();
        rss_ = read_rss();
        if (batched_) {
            vcheck_(vca_ca_batch_create(device_ordinal_(), 256, &batch_), "vca_ca_batch_create");
            batch_thread_ = std::thread([this] { batch_loop(); });
        }
        std::vector<std::thread> pool;
        for (int i = 0; i < workers_; ++i) pool.emplace_back([this] { worker(); });
        std::string line;
        uint64_t seq = 0;
        while (std::getline(std::cin, line)) {
            if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
            auto r = std::make_shared<Request>();
            r->arrival_ms = ms_since(start_);
            parse_request(line, seq++, *r);
            {
                std::lock_guard<std::mutex> lk(qm_);
                queue_.push_back(r);
            }
            qcv_.notify_one();
        }
        {
            std::lock_guard<std::mutex> lk(qm_);
            eof_ = true;
        }
        qcv_.notify_all();
        for (auto& t : pool) t.join();
        if (batched_) {
            {
                std::lock_guard<std::mutex> lk(bm_);
                stopping_ = true;
            }
            bcv_.notify_all();
            batch_thread_.join();
        }
        Json sum = Json::object();
        sum["jobs"] = (unsigned long long)done_;
        sum["failed"] = (unsigned long long)failed_;
        sum["makespan_ms"] = round_to(last_done_ms_, 3);
        sum["workers"] = workers_;
        sum["batched"] = batched_;
        sum["budget_bytes"] = (unsigned long long)budget_;
        sum["peak_allocated_bytes"] = (unsigned long long)peak_alloc_;
        sum["handles_allocated"] = (unsigned long long)allocs_;
        sum["handles_freed"] = (unsigned long long)frees_;
        if (batch_) {
            uint64_t graphs = 0, launches = 0;
            int members = 0;
            vca_ca_batch_info(batch_, &graphs, &launches, &members);
            sum["batch_graphs"] = (unsigned long long)graphs;
            sum["batch_launches"] = (unsigned long long)launches;
        }
        Json top = Json::object();
        top["summary"] = sum;
        emit(top);
        for (Slot* s : slots_) free_slot(s);
        vca_ca_batch_destroy(batch_);
        return failed_ ? kExitBatch : kExitOk;
    }

private:
    static int device_ordinal_() {
        const char* d = std::getenv("VCA_DEVICE");
        return d ? std::atoi(d) : 0;
    }
    static void vcheck_(vca_status s, const char* what) {
        if (s != VCA_OK) throw std::runtime_error(std::string(what) + ": " + vca_last_error());
    }

    void parse_request(const std::string& line, uint64_t seq, Request& r) {
        r.id = std::to_string(seq);
        try {
            Json j = Json::parse(line, false);
            if (!j.is_object()) throw ConfigError("a request is a JSON object {\"config\" | \"json\", \"set\", \"out\", \"id\"}");
            if (const Json* id = j.find("id")) r.id = id->is_string() ? id->as_string() : id->dump();
            std::vector<std::string> sets;
            if (const Json* s = j.find("set")) {
                if (!s->is_array()) throw ConfigError("\"set\" must be a list of \"key=value\" texts");
                for (size_t i = 0; i < s->size(); ++i) {
                    const Json& kv = (*s)[i];
                    if (!kv.is_string() || kv.as_string().find('=') == std::string::npos || kv.as_string()[0] == '=')
                        throw ConfigError("Nadpisanie musi mieć postać klucz=wartość, podano: " + kv.dump());
                    sets.push_back(kv.as_string());
                }
            }
            if (const Json* o = j.find("out")) r.out = o->as_string();
            const Json* path = j.find("config");
            const Json* inl = j.find("json");
            if (path && inl) throw ConfigError("a request gives \"config\" (a file) or \"json\" (an object), not both");
            if (inl)
                r.cfg = Config::load_object(*inl, "", sets);
            else
                r.cfg = Config::load(path ? path->as_string() : std::string(), sets);
        } catch (const ConfigError& e) {
            r.error = std::string("Błąd konfiguracji: ") + e.what();
        } catch (const std::exception& e) {
            r.error = std::string("Błąd: ") + e.what();
        }
    }

    std::shared_ptr<Request> pop() {
        std::unique_lock<std::mutex> lk(qm_);
        qcv_.wait(lk, [&] { return !queue_.empty() || eof_; });
        if (queue_.empty()) return nullptr;
        auto r = queue_.front();
        queue_.pop_front();
        return r;
    }

    // The capacity class of a job and its device bytes (CA + MC handles).
    void capacity(const Config& c, Dims& cap, uint64_t& bytes) {
        const bool y = c.space.ny > 1, z = c.space.nz > 1;
        cap.nx = class_side(c.space.nx, 64);
        cap.ny = y ? class_side(c.space.ny, 16) : 1;
        cap.nz = z ? class_side(c.space.nz, 16) : 1;
        vca_ca_desc d = ca_desc(c);
        d.nx = cap.nx;
        d.ny = cap.ny;
        d.nz = cap.nz;
        d.neighborhood = VCA_NB_MOORE;
        d.max_steps = 65535;
        d.tile_y = d.tile_z = 0;
        uint64_t ca_b = 0, mc_b = 0;
        vcheck_(vca_ca_footprint(&d, &ca_b), "vca_ca_footprint");
        vca_mc_desc m{};
        m.nx = cap.nx;
        m.ny = cap.ny;
        m.nz = cap.nz;
        m.neighborhood = VCA_NB_MOORE;
        m.Q = 2;
        m.J = 1.0;
        m.device = d.device;
        vcheck_(vca_mc_footprint(&m, &mc_b), "vca_mc_footprint");
        bytes = ca_b + mc_b;
    }

    Slot* new_slot(const Config& c, const Dims& cap, uint64_t bytes) {
        auto* s = new Slot();
        s->cap = cap;
        s->bytes = bytes;
        s->lava = c.ca.mode == Mode::Lava;
        vca_ca_desc d = ca_desc(c);
        d.nx = cap.nx;
        d.ny = cap.ny;
        d.nz = cap.nz;
        d.neighborhood = VCA_NB_MOORE;
        d.max_steps = 65535;
        d.tile_y = d.tile_z = 0;
        vca_mc_desc m{};
        m.nx = cap.nx;
        m.ny = cap.ny;
        m.nz = cap.nz;
        m.neighborhood = VCA_NB_MOORE;
        m.Q = 2;
        m.J = 1.0;
        m.device = d.device;
        if (vca_ca_create(&d, &s->ca) != VCA_OK || vca_mc_create(&m, &s->mc) != VCA_OK) {
            const std::string err = vca_last_error();
            free_slot(s);
            throw std::runtime_error("allocating a resident handle: " + err);
        }
        return s;
    }
    void free_slot(Slot* s) {
        vca_mc_destroy(s->mc);
        vca_ca_destroy(s->ca);
        delete s;
    }

    // A resident handle for the job: an idle one that holds it, else a new one within the budget
    // (freeing idle ones to make room), else wait until a job ends.
    Slot* acquire(const Request& r) {
        Dims cap;
        uint64_t bytes = 0;
        capacity(r.cfg, cap, bytes);
        if (bytes > budget_)
            throw std::runtime_error("the job needs " + std::to_string(bytes) + " device bytes, above the budget of " +
                                     std::to_string(budget_));
        const bool lava = r.cfg.ca.mode == Mode::Lava;
        std::unique_lock<std::mutex> lk(sm_);
        for (;;) {
            Slot* best = nullptr;
            for (Slot* s : slots_)
                if (!s->busy && s->lava == lava && (s->cap.ny > 1) == (cap.ny > 1) && (s->cap.nz > 1) == (cap.nz > 1) &&
                    s->cap.nx >= r.cfg.space.nx && s->cap.ny >= r.cfg.space.ny && s->cap.nz >= r.cfg.space.nz &&
                    (!best || s->bytes < best->bytes))
                    best = s;
            if (best) {
                best->busy = true;
                best->used = ++admissions_;
                return best;
            }
            if (allocated_ + bytes <= budget_) {
                allocated_ += bytes;
                peak_alloc_ = std::max(peak_alloc_, allocated_);
                ++allocs_;
                lk.unlock();
                Slot* s = nullptr;
                try {
                    s = new_slot(r.cfg, cap, bytes);
                } catch (...) {
                    lk.lock();
                    allocated_ -= bytes;
                    throw;
                }
                lk.lock();
                s->busy = true;
                s->used = ++admissions_;
                slots_.push_back(s);
                return s;
            }
            // free the least recently used idle handle, if any, and try again
            Slot* idle = nullptr;
            for (Slot* s : slots_)
                if (!s->busy && (!idle || s->used < idle->used)) idle = s;
            if (idle) {
                slots_.erase(std::find(slots_.begin(), slots_.end(), idle));
                allocated_ -= idle->bytes;
                ++frees_;
                lk.unlock();
                free_slot(idle);
                lk.lock();
                continue;
            }
            scv_.wait(lk);
        }
    }
    void release(Slot* s) {
        {
            std::lock_guard<std::mutex> lk(sm_);
            s->busy = false;
        }
        scv_.notify_all();
    }

    // The CA stage inside the shared batch: join, then wait until the batch reports the stop.
    void batch_run(vca_ca* h) {
        std::unique_lock<std::mutex> lk(bm_);
        vcheck_(vca_ca_batch_add(batch_, h), "vca_ca_batch_add");
        finished_[h] = false;
        ++members_;
        bcv_.notify_all();
        bcv_.wait(lk, [&] { return finished_[h] || batch_failed_; });
        finished_.erase(h);
        if (batch_failed_) throw std::runtime_error("the batch stopped: " + batch_error_);
    }
    void batch_loop() {
        std::vector<vca_ca*> done(256);
        std::unique_lock<std::mutex> lk(bm_);
        for (;;) {
            bcv_.wait(lk, [&] { return members_ > 0 || stopping_; });
            if (members_ == 0 && stopping_) return;
            int n = 0, running = 0;
            const vca_status st = vca_ca_batch_advance(batch_, 1, done.data(), (int)done.size(), &n, &running);
            if (st != VCA_OK) {
                batch_failed_ = true;
                batch_error_ = vca_last_error();
                bcv_.notify_all();
                return;
            }
            for (int i = 0; i < n; ++i) finished_[done[(size_t)i]] = true;
            members_ = running;
            if (n) bcv_.notify_all();
        }
    }

    void worker() {
        for (;;) {
            std::shared_ptr<Request> r = pop();
            if (!r) return;
            Json resp = Json::object();
            resp["id"] = r->id;
            resp["arrival_ms"] = round_to(r->arrival_ms, 3);
            if (!r->error.empty()) {
                respond_error(resp, r->error);
                continue;
            }
            Slot* slot = nullptr;
            try {
                slot = acquire(*r);
                const double admitted = ms_since(start_);
                double ca_done = 0.0;
                if (!r->out.empty()) fs::create_directories(r->out);
                Timing timing;
                timing.detail = true;
                Progress progress;
                RunHandles res;
                res.ca = slot->ca;
                res.mc = slot->mc;
                if (batched_ && r->cfg.ca.mode == Mode::Lava) res.ca_run = [this](vca_ca* h) { batch_run(h); };
                res.ca_done = [&] { ca_done = ms_since(start_); };
                timing.add("readConfig", 0.0);
                const JobOutcome job = run_job(r->cfg, r->out, timing, progress, res, Clock::now(), rss_);
                release(slot);
                slot = nullptr;
                const double end = ms_since(start_);
                resp["status"] = "ok";
                resp["admitted_ms"] = round_to(admitted, 3);
                resp["ca_done_ms"] = round_to(ca_done, 3);
                resp["done_ms"] = round_to(end, 3);
                resp["latency_ms"] = round_to(end - r->arrival_ms, 3);
                resp["cells"] = (unsigned long long)r->cfg.space.cells();
                resp["steps"] = job.ca.steps;
                resp["stop"] = stop_text(job.ca.stop);
                resp["cell_updates"] = (unsigned long long)r->cfg.space.cells() * (unsigned long long)job.ca.steps;
                const auto td = Clock::now();
                Json dg = Json::object();
                if (job.ca.ca_ran) dg["ca_result.bin"] = ca_digest(job.ca.result);
                if (job.mc_ran) {
                    dg["mc_result.bin"] = mc_digest(job.mc.crystals);
                    resp["mcs"] = job.mc.mcs;
                    resp["energyEnd"] = job.mc.history.back().energy;
                }
                resp["digest"] = dg;
                // where the job's time went: the sections of its times.json, the MC set-up details and
                // the digests (caDevice / mcDevice are running totals of the resident handles: left out)
                Json tm = Json::object();
                for (const auto& sec : timing.sections) tm[sec.first] = round_to(sec.second, 3);
                for (const auto& det : timing.details)
                    if (det.first != "caDevice" && det.first != "mcDevice") tm[det.first] = round_to(det.second, 3);
                tm["digest"] = round_to(ms_since(td), 3);
                resp["times_ms"] = tm;
                if (!r->out.empty()) resp["out"] = r->out;
                {
                    std::lock_guard<std::mutex> lk(om_);
                    ++done_;
                    last_done_ms_ = std::max(last_done_ms_, end);
                }
                emit(resp);
            } catch (const ConfigError& e) {
                if (slot) release(slot);
                respond_error(resp, std::string("Błąd konfiguracji: ") + e.what());
            } catch (const std::exception& e) {
                if (slot) release(slot);
                respond_error(resp, std::string("Błąd: ") + e.what());
            }
        }
    }

    void respond_error(Json& resp, const std::string& msg) {
        resp["status"] = "error";
        resp["error"] = msg;
        resp["done_ms"] = round_to(ms_since(start_), 3);
        {
            std::lock_guard<std::mutex> lk(om_);
            ++failed_;
        }
        emit(resp);
    }
    void emit(const Json& j) {
        std::lock_guard<std::mutex> lk(om_);
        std::cout << j.dump() << '\n' << std::flush;
    }

    const int workers_;
    const uint64_t budget_;
    const bool batched_;
    Clock::time_point start_;
    Rss rss_;
    // requests
    std::mutex qm_;
    std::condition_variable qcv_;
    std::deque<std::shared_ptr<Request>> queue_;
    bool eof_ = false;
    // resident handles
    std::mutex sm_;
    std::condition_variable scv_;
    std::vector<Slot*> slots_;
    uint64_t allocated_ = 0, peak_alloc_ = 0, allocs_ = 0, frees_ = 0, admissions_ = 0;
    // the shared batch
    vca_ca_batch* batch_ = nullptr;
    std::thread batch_thread_;
    std::mutex bm_;
    std::condition_variable bcv_;
    std::map<vca_ca*, bool> finished_;
    int members_ = 0;
    bool stopping_ = false, batch_failed_ = false;
    std::string batch_error_;
    // output
    std::mutex om_;
    uint64_t done_ = 0, failed_ = 0;
    double last_done_ms_ = 0.0;
};

}  // namespace

int run_server(int workers, double budget_gb, bool batched) {
    g_use_tuning = false;  // batch members keep the default tiles
    Server s(std::max(1, workers), (uint64_t)(budget_gb * 1024.0 * 1024.0 * 1024.0), batched);
    return s.run();
}

}  // namespace eng

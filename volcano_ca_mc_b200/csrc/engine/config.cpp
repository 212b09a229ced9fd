// config.cpp -- configuration with the reference engine's keys, defaults and validation
// (engine/src/io/Config.cpp): defaults <- JSON file <- --set overrides, unknown keys rejected,
// '_'-prefixed keys treated as comments, the merged JSON kept for config_used.json.  The messages
// are the reference's own Polish texts (the batch runner's batch_summary.csv and the GUI show them
// verbatim), so a bad config reads the same through either engine.
#include <cmath>
#include <fstream>
#include <limits>
#include <sstream>

#include "model.hpp"

namespace eng {

namespace {

std::string q(const std::string& path) { return "„" + path + "”"; }  // „path”

std::vector<std::string> split_path(const std::string& path) {
    std::vector<std::string> parts;
    std::stringstream ss(path);
    std::string part;
    while (std::getline(ss, part, '.')) parts.push_back(part);
    return parts;
}

const Json& field(const Json& j, const std::string& path) {
    const Json* cur = &j;
    for (const std::string& part : split_path(path)) {
        if (!cur->is_object() || !cur->contains(part)) throw ConfigError("Brak parametru " + q(path));
        cur = cur->find(part);
    }
    return *cur;
}

// Config.cpp:43-59
long long get_integer(const Json& j, const std::string& path, long long lo, long long hi) {
    const Json& v = field(j, path);
    if (!v.is_integer() || (v.is_unsigned() && v.as_u64() > (uint64_t)hi)) {
        if (v.is_unsigned())
            throw ConfigError("Parametr " + q(path) + " jest za duży (maks. " + std::to_string(hi) + "), podano: " + v.dump());
        throw ConfigError("Parametr " + q(path) + " musi być liczbą całkowitą, podano: " + v.dump());
    }
    const long long x = v.as_i64();
    if (x < lo || x > hi)
        throw ConfigError("Parametr " + q(path) + " musi być z zakresu " + std::to_string(lo) + ".." +
                          std::to_string(hi) + ", podano: " + std::to_string(x));
    return x;
}
int get_int(const Json& j, const std::string& path, int lo, int hi) { return (int)get_integer(j, path, lo, hi); }

// Config.cpp:66-78
double get_number(const Json& j, const std::string& path, double lo, double hi) {
    const Json& v = field(j, path);
    if (!v.is_number()) throw ConfigError("Parametr " + q(path) + " musi być liczbą, podano: " + v.dump());
    const double x = v.as_double();
    if (!std::isfinite(x) || x < lo || x > hi) {
        std::ostringstream os;
        os << "Parametr " << q(path) << " musi być z zakresu " << lo << ".." << hi << ", podano: " << x;
        throw ConfigError(os.str());
    }
    return x;
}

bool get_bool(const Json& j, const std::string& path) {
    const Json& v = field(j, path);
    if (!v.is_bool())
        throw ConfigError("Parametr " + q(path) + " musi mieć wartość true lub false, podano: " + v.dump());
    return v.as_bool();
}

template <class E>
E get_enum(const Json& j, const std::string& path, std::initializer_list<std::pair<const char*, E>> options) {
    const Json& v = field(j, path);
    std::string allowed;
    for (const auto& o : options) allowed += (allowed.empty() ? "" : ", ") + std::string(o.first);
    if (v.is_string())
        for (const auto& o : options)
            if (v.as_string() == o.first) return o.second;
    throw ConfigError("Parametr " + q(path) + " ma nieprawidłową wartość " + v.dump() +
                      "; dozwolone: " + allowed);
}

// vents.positions (Config.cpp:111-147): pairs of integers inside the grid, no repeated column.
std::vector<std::pair<int, int>> get_columns(const Json& j, const std::string& path, const Dims& d) {
    const Json& list = field(j, path);
    if (!list.is_array())
        throw ConfigError("Parametr " + q(path) + " musi być listą par [x, y], np. [[80, 75], [82, 70]], podano: " +
                          list.dump());
    std::vector<std::pair<int, int>> out;
    for (size_t i = 0; i < list.size(); ++i) {
        const Json& p = list[i];
        const std::string where = path + "[" + std::to_string(i) + "]";
        auto is_int = [](const Json& v) { return v.is_integer() && (!v.is_unsigned() || v.as_u64() <= 100000ULL); };
        if (!p.is_array() || p.size() != 2 || !is_int(p[0]) || !is_int(p[1]))
            throw ConfigError("Parametr " + q(where) + " musi być parą liczb całkowitych [x, y], podano: " + p.dump());
        const long long x = p[0].as_i64(), y = p[1].as_i64();
        if (x < 0 || x >= d.nx || y < 0 || y >= d.ny)
            throw ConfigError("Parametr " + q(where) + " = " + p.dump() + " leży poza siatką: x musi być z zakresu 0.." +
                              std::to_string(d.nx - 1) + ", y z zakresu 0.." + std::to_string(d.ny - 1) +
                              " (space.nx = " + std::to_string(d.nx) + ", space.ny = " + std::to_string(d.ny) + ")");
        for (const auto& c : out)
            if (c.first == (int)x && c.second == (int)y)
                throw ConfigError("Parametr " + q(where) + " = " + p.dump() +
                                  " powtarza kolumnę z wcześniejszego elementu listy; w jednej kolumnie może być "
                                  "najwyżej jeden krater");
        out.emplace_back((int)x, (int)y);
    }
    return out;
}

void merge(Json& base, const Json& patch, const std::string& prefix) {
    for (const auto& kv : patch.members()) {
        const std::string& key = kv.first;
        if (!key.empty() && key[0] == '_') continue;  // comment key
        const std::string path = prefix.empty() ? key : prefix + "." + key;
        Json* target = base.find(key);
        if (!target) {
            std::string allowed;
            for (const auto& b : base.members()) allowed += (allowed.empty() ? "" : ", ") + b.first;
            throw ConfigError("Nieznany parametr " + q(path) + "; dozwolone w tej sekcji: " + allowed);
        }
        if (target->is_object()) {
            if (!kv.second.is_object())
                throw ConfigError("Parametr " + q(path) + " jest sekcją: oczekiwano obiektu { ... }, podano: " +
                                  kv.second.dump());
            merge(*target, kv.second, path);
        } else {
            *target = kv.second;
        }
    }
}

// --set a.b=value: JSON when it parses, else a plain string (Config.cpp:205-235).
void apply_override(Json& j, const std::string& kv) {
    const size_t eq = kv.find('=');
    if (eq == std::string::npos || eq == 0) throw ConfigError("Nadpisanie musi mieć postać klucz=wartość, podano: " + kv);
    const std::string key = kv.substr(0, eq), text = kv.substr(eq + 1);
    Json value;
    try {
        value = Json::parse(text, false);
    } catch (const JsonError&) {
        value = Json(text);
    }
    const std::vector<std::string> parts = split_path(key);
    for (const std::string& p : parts)
        if (p.empty()) throw ConfigError("Nieprawidłowa ścieżka parametru w nadpisaniu: " + key);
    Json patch = value;
    for (auto it = parts.rbegin(); it != parts.rend(); ++it) {
        Json obj = Json::object();
        obj[*it] = patch;
        patch = obj;
    }
    merge(j, patch, "");
}

}  // namespace

const char* nb_name(Nb n) {
    switch (n) {
        case Nb::VonNeumann: return "von_neumann";
        case Nb::Moore: return "moore";
        case Nb::Pentagonal: return "pentagonal";
        case Nb::Hexagonal: return "hexagonal";
    }
    return "?";
}
const char* bc_name(Bc b) { return b == Bc::Periodic ? "periodic" : "absorbing"; }
const char* mode_name(Mode m) { return m == Mode::Classic ? "classic" : "lava"; }

// Defaults: the same keys and values as Config::defaultsJson (engine/src/io/Config.cpp:153-176).
Json Config::defaults_json() {
    return Json::parse(R"({
      "space":        { "nx": 200, "ny": 1, "nz": 100 },
      "grid":         "vector",
      "boundary":     "absorbing",
      "neighborhood": "moore",
      "rngSeed":      42,
      "terrain": { "type": "cone", "peakHeight": 70, "baseRadius": 90,
                   "craterRadius": 6, "craterDepth": 4, "noise": 0.05, "file": null },
      "vents":   { "count": 1, "placement": "crater", "positions": [], "eruptionSteps": 300,
                   "eruptTemp": 1200 },
      "ca":      { "mode": "lava", "maxSteps": 5000, "coolingAmbient": 0.3,
                   "coolingLateral": 1.5, "coolingFall": 0.1, "solidusTemp": 800,
                   "ponding": true, "sweep": "front" },
      "mc":      { "enabled": false, "domain": "basalt", "Q": 50, "mcs": 100, "J": 1.0, "kT": 0.0,
                   "mobilityFromCooling": true, "mobilityMin": 0.05, "statsEvery": 10,
                   "snapshotsEvery": 0, "update": "random" },
      "output":  { "format": "txt", "snapshotsEvery": 0 },
      "parallel": { "threads": 1, "schedule": "static", "chunk": 0, "affinity": "none", "priority": "normal" },
      "mpi":     { "exchange": "always", "pack": "manual", "bcast": "json", "io": "gather" }
    })");
}

Config Config::load(const std::string& path, const std::vector<std::string>& overrides) {
    Json j = defaults_json();
    bool space_given = false;
    if (!path.empty()) {
        std::ifstream in(path, std::ios::binary);
        if (!in) throw ConfigError("Nie można otworzyć pliku konfiguracyjnego: " + path);
        std::stringstream ss;
        ss << in.rdbuf();
        Json file;
        try {
            file = Json::parse(ss.str(), true);
        } catch (const JsonError& e) {
            throw ConfigError("Błąd składni JSON w pliku " + path + ": " + e.what());
        }
        if (!file.is_object()) throw ConfigError("Plik konfiguracyjny " + path + " musi zawierać obiekt JSON { ... }");
        merge(j, file, "");
        space_given = file.contains("space");
    }
    for (const std::string& o : overrides) {
        apply_override(j, o);
        space_given = space_given || o.rfind("space", 0) == 0;
    }
    Config c = from_json(j);
    c.source_path = path;
    c.space_from_user = space_given;
    return c;
}

Config Config::load_object(const Json& file, const std::string& source_path, const std::vector<std::string>& overrides) {
    Json j = defaults_json();
    if (!file.is_object()) throw ConfigError("Plik konfiguracyjny " + source_path + " musi zawierać obiekt JSON { ... }");
    merge(j, file, "");
    bool space_given = file.contains("space");
    for (const std::string& o : overrides) {
        apply_override(j, o);
        space_given = space_given || o.rfind("space", 0) == 0;
    }
    Config c = from_json(j);
    c.source_path = source_path;
    c.space_from_user = space_given;
    return c;
}

// Validation in the order of Config::fromJson (engine/src/io/Config.cpp:268-437).
Config Config::from_json(const Json& j) {
    Config c;
    c.space.nx = get_int(j, "space.nx", 1, 100000);
    c.space.ny = get_int(j, "space.ny", 1, 100000);
    c.space.nz = get_int(j, "space.nz", 1, 100000);
    if (c.space.active_axes() < 2)
        throw ConfigError("Przestrzeń musi być 2D (dokładnie jeden wymiar równy 1) lub 3D; podano " +
                          std::to_string(c.space.nx) + " x " + std::to_string(c.space.ny) + " x " + std::to_string(c.space.nz));
    if (c.space.cells() > 2000000000ULL)
        throw ConfigError("Przestrzeń ma za dużo komórek (" + std::to_string(c.space.cells()) +
                          "); maksimum to 2 000 000 000");
    c.grid = get_enum<std::string>(j, "grid", {{"vector", std::string("vector")}, {"matrix", std::string("matrix")}});
    c.boundary = get_enum<Bc>(j, "boundary", {{"absorbing", Bc::Absorbing}, {"periodic", Bc::Periodic}});
    c.neighborhood = get_enum<Nb>(j, "neighborhood", {{"von_neumann", Nb::VonNeumann}, {"moore", Nb::Moore},
                                                      {"pentagonal", Nb::Pentagonal}, {"hexagonal", Nb::Hexagonal}});
    c.seed = (uint64_t)get_integer(j, "rngSeed", 0, std::numeric_limits<long long>::max());

    c.mc.enabled = get_bool(j, "mc.enabled");
    c.mc.full = get_enum<bool>(j, "mc.domain", {{"basalt", false}, {"full", true}});
    c.mc.Q = get_int(j, "mc.Q", 2, 1000000000);
    c.mc.mcs = get_int(j, "mc.mcs", 0, 10000000);
    c.mc.J = get_number(j, "mc.J", 0.0, 1e6);
    if (c.mc.J <= 0.0)
        throw ConfigError("Parametr " + q("mc.J") + " (energia granicy ziarna) musi być większy od 0, podano: " +
                          field(j, "mc.J").dump());
    c.mc.kT = get_number(j, "mc.kT", 0.0, 1e6);
    c.mc.mobility_from_cooling = get_bool(j, "mc.mobilityFromCooling");
    c.mc.mobility_min = get_number(j, "mc.mobilityMin", 0.0, 1.0);
    c.mc.stats_every = get_int(j, "mc.statsEvery", 1, 1000000000);
    c.mc.snapshots_every = get_int(j, "mc.snapshotsEvery", 0, 1000000000);
    c.mc.checkerboard = get_enum<bool>(j, "mc.update", {{"random", false}, {"checkerboard", true}});
    const bool runs_ca = !c.mc.full_only();

    c.ca.mode = get_enum<Mode>(j, "ca.mode", {{"lava", Mode::Lava}, {"classic", Mode::Classic}});
    c.ca.max_steps = get_int(j, "ca.maxSteps", 0, 65535);
    c.ca.cool_ambient = get_number(j, "ca.coolingAmbient", 0.0, 1e6);
    c.ca.cool_lateral = get_number(j, "ca.coolingLateral", 0.0, 1e6);
    c.ca.cool_fall = get_number(j, "ca.coolingFall", 0.0, 1e6);
    c.ca.solidus = get_number(j, "ca.solidusTemp", -1e6, 1e6);
    c.ca.ponding = get_bool(j, "ca.ponding");
    c.ca.front = get_enum<bool>(j, "ca.sweep", {{"front", true}, {"full", false}});

    if (runs_ca && c.ca.mode == Mode::Lava && c.space.is2d() && c.space.ny != 1)
        throw ConfigError("W trybie lava przestrzeń 2D to przekrój pionowy x–z: wymagane ny = 1 (podano nx = " +
                          std::to_string(c.space.nx) + ", ny = " + std::to_string(c.space.ny) + ", nz = " +
                          std::to_string(c.space.nz) + ")");
    if (c.neighborhood == Nb::Hexagonal && !c.space.is2d())
        throw ConfigError("Sąsiedztwo " + q("hexagonal") + " jest zdefiniowane tylko w 2D; dla przestrzeni 3D "
                          "wybierz von_neumann, moore lub pentagonal");

    c.terrain.type = get_enum<TerrainType>(j, "terrain.type", {{"cone", TerrainType::Cone}, {"file", TerrainType::File}});
    c.terrain.peak = get_number(j, "terrain.peakHeight", 0.0, 1e6);
    c.terrain.base_radius = get_number(j, "terrain.baseRadius", 1e-9, 1e6);
    c.terrain.crater_radius = get_number(j, "terrain.craterRadius", 0.0, 1e6);
    c.terrain.crater_depth = get_number(j, "terrain.craterDepth", 0.0, 1e6);
    c.terrain.noise = get_number(j, "terrain.noise", 0.0, 1.0);
    const Json file = field(j, "terrain.file");
    if (!file.is_null() && !file.is_string())
        throw ConfigError("Parametr " + q("terrain.file") + " musi być ścieżką (tekst) albo null, podano: " + file.dump());
    c.terrain.file = file.is_string() ? file.as_string() : std::string();
    if (runs_ca && c.ca.mode == Mode::Lava && c.terrain.type == TerrainType::File && c.terrain.file.empty())
        throw ConfigError("Dla terrain.type = \"file\" trzeba podać ścieżkę w " + q("terrain.file"));

    c.vents.count = get_int(j, "vents.count", 1, 100000000);
    c.vents.placement = get_enum<Placement>(j, "vents.placement", {{"crater", Placement::Crater}, {"random", Placement::Random},
                                                                  {"positions", Placement::Positions}});
    const size_t listed = get_columns(j, "vents.positions", c.space).size();
    const bool lava_ca = runs_ca && c.ca.mode == Mode::Lava;
    if (lava_ca && c.vents.placement == Placement::Positions) {
        if (listed == 0)
            throw ConfigError("vents.placement = \"positions\" wymaga listy kraterów w " + q("vents.positions") +
                              ", np. [[80, 75]] (w GUI: kliknięcie na mapie wysokości)");
        if ((size_t)c.vents.count != listed)
            throw ConfigError("vents.count (" + std::to_string(c.vents.count) + ") musi być równe liczbie kraterów w " +
                              q("vents.positions") + " (" + std::to_string(listed) +
                              "), bo przy placement = \"positions\" każdy krater ma podane położenie");
    } else if (lava_ca && listed > 0) {
        c.warnings.push_back(std::string("vents.positions jest ignorowane, bo vents.placement = \"") +
                             (c.vents.placement == Placement::Crater ? "crater" : "random") +
                             "\" (położenia losowane); kratery w zadanych miejscach: placement = \"positions\"");
    } else if (runs_ca && c.ca.mode == Mode::Classic && c.vents.placement == Placement::Positions) {
        c.warnings.push_back("w trybie classic zarodki są losowane w całej przestrzeni, więc vents.placement = "
                             "\"positions\" i vents.positions są ignorowane");
    }
    c.vents.eruption_steps = get_int(j, "vents.eruptionSteps", 0, 65535);
    c.vents.erupt_temp = get_number(j, "vents.eruptTemp", -1e6, 1e6);
    if (runs_ca && c.ca.mode == Mode::Lava && c.vents.erupt_temp < c.ca.solidus)
        throw ConfigError("vents.eruptTemp musi być nie mniejsze niż ca.solidusTemp, inaczej lawa "
                          "zastygłaby od razu w kraterze");
    if (runs_ca && c.ca.mode == Mode::Classic && (uint64_t)c.vents.count > c.space.cells())
        throw ConfigError("vents.count (" + std::to_string(c.vents.count) + ") nie może przekraczać liczby komórek (" +
                          std::to_string(c.space.cells()) + ")");

    if (c.mc.enabled && !c.mc.full && c.ca.mode == Mode::Classic)
        throw ConfigError("mc.domain = \"basalt\" wymaga ca.mode = \"lava\" (w trybie classic nie ma bazaltu); "
                          "klasyczny rozrost ziaren MC to mc.domain = \"full\"");
    if (c.mc.full_only() && c.mc.mobility_from_cooling)
        c.warnings.push_back("mc.mobilityFromCooling dotyczy tylko mc.domain = \"basalt\" (czas stygnięcia lawy z CA); "
                             "w trybie full jest ignorowane");

    c.output.format = get_enum<OutputFormat>(j, "output.format", {{"txt", OutputFormat::Txt}, {"bin", OutputFormat::Bin},
                                                                  {"both", OutputFormat::Both}, {"none", OutputFormat::None}});
    c.output.snapshots_every = get_int(j, "output.snapshotsEvery", 0, 65535);

    c.threads = get_int(j, "parallel.threads", 0, 256);
    c.schedule = get_enum<std::string>(j, "parallel.schedule", {{"static", std::string("static")},
                                                                {"dynamic", std::string("dynamic")},
                                                                {"guided", std::string("guided")}});
    c.chunk = get_int(j, "parallel.chunk", 0, 1000000);
    c.affinity = get_enum<std::string>(j, "parallel.affinity", {{"none", std::string("none")}, {"pcores", std::string("pcores")}});
    get_enum<bool>(j, "parallel.priority", {{"normal", false}, {"high", true}});
    get_enum<bool>(j, "mpi.exchange", {{"always", false}, {"changed", true}});
    get_enum<bool>(j, "mpi.pack", {{"manual", false}, {"datatype", true}});
    get_enum<bool>(j, "mpi.bcast", {{"json", false}, {"struct", true}});
    get_enum<bool>(j, "mpi.io", {{"gather", false}, {"mpiio", true}});
    if (c.mc.enabled && !c.mc.checkerboard)
        throw ConfigError("mc.update = \"random\" jest z natury sekwencyjne (każda próba widzi wynik poprzednich), "
                          "więc silnik GPU go nie oferuje; równoległe MC: mc.update = \"checkerboard\"");
    c.effective = j;
    return c;
}

std::vector<std::pair<int, int>> Config::vent_columns() const { return get_columns(effective, "vents.positions", space); }

}  // namespace eng

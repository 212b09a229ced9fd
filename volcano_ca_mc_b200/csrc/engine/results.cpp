// results.cpp -- result files in the reference's formats (engine/src/io/ResultWriter.hpp:4-32):
// ca_result.bin (VOLC v2), ca_result.txt, mc_result.bin (VMC1), mc_result.txt, JSON files, and the
// reader of a CA result folder for --mc-from (engine/src/io/ResultReader.cpp:119-160).
#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>

#include "model.hpp"

namespace eng {

namespace {

std::ofstream open_out(const std::string& path, bool binary) {
    std::ofstream out(path, binary ? std::ios::binary : std::ios::out);
    if (!out) throw std::runtime_error("Nie można utworzyć pliku: " + path);
    return out;
}

template <class T>
void write_array(std::ofstream& out, const std::vector<T>& v) {
    out.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

template <class T>
void read_array(std::ifstream& in, std::vector<T>& v, const std::string& path) {
    in.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
    if (!in) throw std::runtime_error("Plik " + path + " jest obcięty (za mało danych)");
}

// Buffered text writer: rows appended to a ~1 MB buffer, flushed when full.
class TextOut {
public:
    explicit TextOut(const std::string& path) : out_(open_out(path, true)) { buf_.reserve((1 << 20) + 256); }
    void put(const char* s, size_t n) { buf_.append(s, n); }
    void put(const std::string& s) { buf_ += s; }
    void put_int(long long v) {
        char b[24];
        auto r = std::to_chars(b, b + sizeof(b), v);
        buf_.append(b, r.ptr);
    }
    void eol() {
        buf_ += '\n';
        if (buf_.size() >= (1u << 20)) flush();
    }
    void flush() {
        out_.write(buf_.data(), (std::streamsize)buf_.size());
        buf_.clear();
    }
    void close(const std::string& path) {
        flush();
        if (!out_) throw std::runtime_error("Błąd zapisu pliku: " + path);
    }

private:
    std::ofstream out_;
    std::string buf_;
};

}  // namespace

// ResultWriter::formatTemp (ResultWriter.cpp:105-124): the characters printf("%.1f", v) gives.
// v * 10 is exact in double (24-bit mantissa times 10), so rounding it to the nearest integer with
// ties to even reproduces printf's correctly rounded decimal digit.
std::string format_temp(float v) {
    const double t = (double)v * 10.0;
    if (!(std::fabs(t) < 1e15)) {
        char b[64];
        std::snprintf(b, sizeof(b), "%.1f", (double)v);
        return b;
    }
    std::string out;
    if (std::signbit(v)) out += '-';
    const unsigned long long n = (unsigned long long)std::fabs(std::nearbyint(t));
    out += std::to_string(n / 10);
    out += '.';
    out += (char)('0' + n % 10);
    return out;
}

void write_ca_bin(const std::string& path, const Microstructure& m) {
    std::ofstream out = open_out(path, true);
    const char magic[4] = {'V', 'O', 'L', 'C'};
    const uint32_t version = 2;
    const int32_t dims[3] = {m.dims.nx, m.dims.ny, m.dims.nz};
    out.write(magic, 4);
    out.write(reinterpret_cast<const char*>(&version), 4);
    out.write(reinterpret_cast<const char*>(dims), 12);
    write_array(out, m.type);
    write_array(out, m.flow);
    write_array(out, m.temp);
    write_array(out, m.solid);
    write_array(out, m.arrival);
    if (!out) throw std::runtime_error("Błąd zapisu pliku: " + path);
}

void write_ca_txt(const std::string& path, const Microstructure& m) {
    TextOut t(path);
    const Dims& d = m.dims;
    t.put(std::to_string(d.nx) + " " + std::to_string(d.ny) + " " + std::to_string(d.nz));
    t.eol();
    t.put(std::string("x y z type flowId temp"));
    t.eol();
    size_t i = 0;
    for (int z = 0; z < d.nz; ++z)
        for (int y = 0; y < d.ny; ++y) {
            const std::string yz = " " + std::to_string(y) + " " + std::to_string(z) + " ";
            for (int x = 0; x < d.nx; ++x, ++i) {
                t.put_int(x);
                t.put(yz);
                t.put_int(m.type[i]);
                t.put(" ", 1);
                t.put_int(m.flow[i]);
                t.put(" ", 1);
                t.put(format_temp(m.temp[i]));
                t.eol();
            }
        }
    t.close(path);
}

void write_crystal_bin(const std::string& path, const CrystalMap& m) {
    std::ofstream out = open_out(path, true);
    const char magic[4] = {'V', 'M', 'C', '1'};
    const int32_t dims[3] = {m.dims.nx, m.dims.ny, m.dims.nz};
    out.write(magic, 4);
    out.write(reinterpret_cast<const char*>(dims), 12);
    write_array(out, m.crystal);
    if (!out) throw std::runtime_error("Błąd zapisu pliku: " + path);
}

void write_crystal_txt(const std::string& path, const CrystalMap& m) {
    TextOut t(path);
    const Dims& d = m.dims;
    t.put(std::to_string(d.nx) + " " + std::to_string(d.ny) + " " + std::to_string(d.nz));
    t.eol();
    t.put(std::string("x y z crystal"));
    t.eol();
    size_t i = 0;
    for (int z = 0; z < d.nz; ++z)
        for (int y = 0; y < d.ny; ++y) {
            const std::string yz = " " + std::to_string(y) + " " + std::to_string(z) + " ";
            for (int x = 0; x < d.nx; ++x, ++i) {
                t.put_int(x);
                t.put(yz);
                t.put_int(m.crystal[i]);
                t.eol();
            }
        }
    t.close(path);
}

void write_json(const std::string& path, const Json& j) {
    std::ofstream out = open_out(path, false);
    out << j.dump(2) << '\n';
    if (!out) throw std::runtime_error("Błąd zapisu pliku: " + path);
}

namespace {

Dims read_txt_header(std::ifstream& in, const std::string& path) {
    if (!in) throw std::runtime_error("Nie można otworzyć pliku: " + path);
    Dims d;
    if (!(in >> d.nx >> d.ny >> d.nz) || d.nx < 1 || d.ny < 1 || d.nz < 1)
        throw std::runtime_error("Plik " + path + ": nieprawidłowy nagłówek wymiarów");
    std::string line;
    std::getline(in, line);
    std::getline(in, line);
    return d;
}

Microstructure read_txt(const std::string& path) {
    std::ifstream in(path);
    const Dims d = read_txt_header(in, path);
    Microstructure m;
    m.resize(d);
    for (uint64_t n = 0; n < d.cells(); ++n) {
        int x = 0, y = 0, z = 0, type = 0;
        int32_t flow = 0;
        float temp = 0.0f;
        if (!(in >> x >> y >> z >> type >> flow >> temp))
            throw std::runtime_error("Plik " + path + ": za mało wierszy danych (wczytano " + std::to_string(n) + " z " +
                                     std::to_string(d.cells()) + ")");
        if (x < 0 || x >= d.nx || y < 0 || y >= d.ny || z < 0 || z >= d.nz)
            throw std::runtime_error("Plik " + path + ": współrzędne poza przestrzenią w wierszu " + std::to_string(n + 3));
        const size_t i = (size_t)x + (size_t)d.nx * ((size_t)y + (size_t)d.ny * z);
        m.type[i] = (uint8_t)type;
        m.flow[i] = flow;
        m.temp[i] = temp;
    }
    return m;
}

Microstructure read_bin(const std::string& path, uint32_t* version_out) {
    std::ifstream in(path, std::ios::binary);
    if (!in) throw std::runtime_error("Nie można otworzyć pliku: " + path);
    char magic[4] = {};
    uint32_t version = 0;
    int32_t dims[3] = {};
    in.read(magic, 4);
    in.read(reinterpret_cast<char*>(&version), 4);
    in.read(reinterpret_cast<char*>(dims), 12);
    if (!in || std::memcmp(magic, "VOLC", 4) != 0) throw std::runtime_error("Plik " + path + " nie jest plikiem wyników VOLC");
    if (version < 1 || version > 2) throw std::runtime_error("Plik " + path + ": nieobsługiwana wersja formatu " + std::to_string(version));
    if (dims[0] < 1 || dims[1] < 1 || dims[2] < 1) throw std::runtime_error("Plik " + path + ": nieprawidłowe wymiary");
    Microstructure m;
    m.resize(Dims{dims[0], dims[1], dims[2]});
    read_array(in, m.type, path);
    read_array(in, m.flow, path);
    read_array(in, m.temp, path);
    read_array(in, m.solid, path);
    if (version >= 2) read_array(in, m.arrival, path);
    *version_out = version;
    return m;
}

}  // namespace

Microstructure read_ca_folder(const std::string& folder, ResultSource* src) {
    const std::filesystem::path dir(folder);
    ResultSource info;
    Microstructure m;
    if (std::filesystem::exists(dir / "ca_result.bin")) {
        info.path = (dir / "ca_result.bin").string();
        info.format = "bin";
        m = read_bin(info.path, &info.version);
        info.has_solid = true;
        info.has_arrival = info.version >= 2;
    } else {
        info.path = (dir / "ca_result.txt").string();
        info.format = "txt";
        m = read_txt(info.path);
    }
    if (src) *src = info;
    return m;
}

}  // namespace eng

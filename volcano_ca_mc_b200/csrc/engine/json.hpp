// json.hpp -- a small ordered JSON value for the engine's configs and result files.
//
// Objects keep insertion order (config_used.json, stats.json and times.json list keys in the
// order they were set, like the reference's ordered_json output).  Numbers keep the distinction
// the config validation needs: unsigned / signed integer / floating.  The parser accepts // and
// /* */ comments (the reference parses configs with comments allowed, engine/src/io/Config.cpp:248).
// dump() indents like the reference's writer (engine/src/io/ResultWriter.cpp:238-244): two spaces,
// one element per line, "key": value, and floating numbers in shortest round-trip digits with
// a trailing ".0" for integral values and exponents written e+XX / e-XX outside 1e-4 .. 1e15.
#pragma once

#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace eng {

class Json {
public:
    enum class Kind { Null, Bool, Unsigned, Integer, Float, String, Array, Object };

    Json() = default;
    Json(std::nullptr_t) {}
    Json(bool b) : kind_(Kind::Bool), b_(b) {}
    Json(int v) { set_int(v); }
    Json(long v) { set_int(v); }
    Json(long long v) { set_int(v); }
    Json(unsigned v) : kind_(Kind::Unsigned), u_(v) {}
    Json(unsigned long v) : kind_(Kind::Unsigned), u_(v) {}
    Json(unsigned long long v) : kind_(Kind::Unsigned), u_(v) {}
    Json(double d) : kind_(Kind::Float), d_(d) {}
    Json(const char* s) : kind_(Kind::String), s_(s) {}
    Json(std::string s) : kind_(Kind::String), s_(std::move(s)) {}

    static Json array() {
        Json j;
        j.kind_ = Kind::Array;
        return j;
    }
    static Json object() {
        Json j;
        j.kind_ = Kind::Object;
        return j;
    }
    template <class T>
    static Json array_of(const std::vector<T>& v) {
        Json j = array();
        for (const T& e : v) j.push_back(Json(e));
        return j;
    }

    Kind kind() const { return kind_; }
    bool is_null() const { return kind_ == Kind::Null; }
    bool is_bool() const { return kind_ == Kind::Bool; }
    bool is_number() const { return kind_ == Kind::Unsigned || kind_ == Kind::Integer || kind_ == Kind::Float; }
    bool is_integer() const { return kind_ == Kind::Unsigned || kind_ == Kind::Integer; }
    bool is_unsigned() const { return kind_ == Kind::Unsigned; }
    bool is_float() const { return kind_ == Kind::Float; }
    bool is_string() const { return kind_ == Kind::String; }
    bool is_array() const { return kind_ == Kind::Array; }
    bool is_object() const { return kind_ == Kind::Object; }

    bool as_bool() const { return b_; }
    uint64_t as_u64() const { return kind_ == Kind::Unsigned ? u_ : (uint64_t)i_; }
    int64_t as_i64() const { return kind_ == Kind::Unsigned ? (int64_t)u_ : (kind_ == Kind::Integer ? i_ : (int64_t)d_); }
    double as_double() const {
        return kind_ == Kind::Float ? d_ : (kind_ == Kind::Unsigned ? (double)u_ : (double)i_);
    }
    const std::string& as_string() const { return s_; }

    // arrays
    size_t size() const { return kind_ == Kind::Array ? arr_.size() : (kind_ == Kind::Object ? obj_.size() : 0); }
    void push_back(Json v) {
        if (kind_ == Kind::Null) kind_ = Kind::Array;
        arr_.push_back(std::move(v));
    }
    const Json& operator[](size_t i) const { return arr_.at(i); }
    Json& at(size_t i) { return arr_.at(i); }
    const std::vector<Json>& items() const { return arr_; }

    // objects (insertion order)
    bool contains(const std::string& k) const { return find(k) != nullptr; }
    const Json* find(const std::string& k) const {
        for (const auto& kv : obj_)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    Json* find(const std::string& k) {
        for (auto& kv : obj_)
            if (kv.first == k) return &kv.second;
        return nullptr;
    }
    Json& operator[](const std::string& k) {
        if (kind_ == Kind::Null) kind_ = Kind::Object;
        if (Json* v = find(k)) return *v;
        obj_.emplace_back(k, Json());
        return obj_.back().second;
    }
    const Json& get(const std::string& k) const {
        const Json* v = find(k);
        if (!v) throw std::out_of_range("missing key " + k);
        return *v;
    }
    const std::vector<std::pair<std::string, Json>>& members() const { return obj_; }
    std::vector<std::pair<std::string, Json>>& members() { return obj_; }

    static Json parse(const std::string& text, bool allow_comments = true);  // throws JsonError
    std::string dump(int indent = -1) const;

private:
    void set_int(long long v) {
        if (v >= 0) {
            kind_ = Kind::Unsigned;
            u_ = (uint64_t)v;
        } else {
            kind_ = Kind::Integer;
            i_ = v;
        }
    }
    void dump_to(std::string& out, int indent, int level) const;

    Kind kind_ = Kind::Null;
    bool b_ = false;
    uint64_t u_ = 0;
    int64_t i_ = 0;
    double d_ = 0.0;
    std::string s_;
    std::vector<Json> arr_;
    std::vector<std::pair<std::string, Json>> obj_;
};

struct JsonError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// A number literal whose value is beyond the range of a double.  Not a JsonError: the reference's
// JSON library reports it as a range error, which its config loader does not turn into a syntax
// message or a plain-string override, so it leaves the loader as it is (engine/src/io/Config.cpp
// catches parse errors only).
struct JsonRangeError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// Shortest round-trip text of a double in the writer's format.
std::string format_double(double d);

}  // namespace eng

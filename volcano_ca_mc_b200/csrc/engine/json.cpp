// json.cpp -- parser and writer of eng::Json.
#include "json.hpp"

#include <charconv>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace eng {

namespace {

struct Parser {
    const std::string& s;
    size_t i = 0;
    bool comments;

    [[noreturn]] void fail(const std::string& what) const {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < i && k < s.size(); ++k) {
            if (s[k] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
        }
        throw JsonError("syntax error at line " + std::to_string(line) + ", column " + std::to_string(col) + ": " + what);
    }

    void skip_ws() {
        for (;;) {
            while (i < s.size() && (s[i] == ' ' || s[i] == '\t' || s[i] == '\n' || s[i] == '\r')) ++i;
            if (comments && i + 1 < s.size() && s[i] == '/' && s[i + 1] == '/') {
                while (i < s.size() && s[i] != '\n') ++i;
                continue;
            }
            if (comments && i + 1 < s.size() && s[i] == '/' && s[i + 1] == '*') {
                const size_t end = s.find("*/", i + 2);
                if (end == std::string::npos) fail("unterminated comment");
                i = end + 2;
                continue;
            }
            break;
        }
    }

    Json value() {
        skip_ws();
        if (i >= s.size()) fail("unexpected end of input");
        const char c = s[i];
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') return Json(string());
        if (c == 't' || c == 'f' || c == 'n') return literal();
        if (c == '-' || (c >= '0' && c <= '9')) return number();
        fail(std::string("unexpected character '") + c + "'");
    }

    Json literal() {
        if (s.compare(i, 4, "true") == 0) {
            i += 4;
            return Json(true);
        }
        if (s.compare(i, 5, "false") == 0) {
            i += 5;
            return Json(false);
        }
        if (s.compare(i, 4, "null") == 0) {
            i += 4;
            return Json();
        }
        fail("invalid literal");
    }

    Json number() {
        const size_t start = i;
        if (s[i] == '-') ++i;
        if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("invalid number");
        if (s[i] == '0') {
            ++i;
        } else {
            while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
        }
        bool is_float = false;
        if (i < s.size() && s[i] == '.') {
            is_float = true;
            ++i;
            if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("invalid number");
            while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
        }
        if (i < s.size() && (s[i] == 'e' || s[i] == 'E')) {
            is_float = true;
            ++i;
            if (i < s.size() && (s[i] == '+' || s[i] == '-')) ++i;
            if (i >= s.size() || !(s[i] >= '0' && s[i] <= '9')) fail("invalid number");
            while (i < s.size() && s[i] >= '0' && s[i] <= '9') ++i;
        }
        const char* b = s.data() + start;
        const char* e = s.data() + i;
        if (!is_float) {
            if (*b == '-') {
                long long v = 0;
                auto r = std::from_chars(b, e, v);
                if (r.ec == std::errc() && r.ptr == e) return Json(v);
            } else {
                unsigned long long v = 0;
                auto r = std::from_chars(b, e, v);
                if (r.ec == std::errc() && r.ptr == e) return Json(v);
            }
            // out of the integer range: keep it as a floating number
        }
        double d = 0.0;
        auto r = std::from_chars(b, e, d);
        if (r.ec == std::errc::result_out_of_range && r.ptr == e) {
            // beyond the double range: an underflow is the nearest value (0 or a subnormal), as
            // strtod gives it; an overflow is an error that names the literal, in the text of the
            // reference's JSON library (its out_of_range error 406)
            const std::string lit(b, e);
            d = std::strtod(lit.c_str(), nullptr);
            if (!std::isfinite(d))
                throw JsonRangeError("[json.exception.out_of_range.406] number overflow parsing '" + lit + "'");
            return Json(d);
        }
        if (r.ec != std::errc() || r.ptr != e) fail("invalid number");
        return Json(d);
    }

    static void put_utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += (char)cp;
        } else if (cp < 0x800) {
            out += (char)(0xC0 | (cp >> 6));
            out += (char)(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18));
            out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F));
            out += (char)(0x80 | (cp & 0x3F));
        }
    }

    uint32_t hex4() {
        if (i + 4 > s.size()) fail("invalid \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = s[i++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (uint32_t)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (uint32_t)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (uint32_t)(c - 'A' + 10);
            else fail("invalid \\u escape");
        }
        return v;
    }

    std::string string() {
        ++i;  // opening quote
        std::string out;
        while (true) {
            if (i >= s.size()) fail("unterminated string");
            const char c = s[i++];
            if (c == '"') break;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i >= s.size()) fail("unterminated string");
            const char e = s[i++];
            switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp <= 0xDBFF && i + 1 < s.size() && s[i] == '\\' && s[i + 1] == 'u') {
                        i += 2;
                        const uint32_t lo = hex4();
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    put_utf8(out, cp);
                    break;
                }
                default: fail("invalid escape");
            }
        }
        return out;
    }

    Json array() {
        ++i;
        Json a = Json::array();
        skip_ws();
        if (i < s.size() && s[i] == ']') {
            ++i;
            return a;
        }
        while (true) {
            a.push_back(value());
            skip_ws();
            if (i >= s.size()) fail("unterminated array");
            if (s[i] == ',') {
                ++i;
                continue;
            }
            if (s[i] == ']') {
                ++i;
                return a;
            }
            fail("expected ',' or ']'");
        }
    }

    Json object() {
        ++i;
        Json o = Json::object();
        skip_ws();
        if (i < s.size() && s[i] == '}') {
            ++i;
            return o;
        }
        while (true) {
            skip_ws();
            if (i >= s.size() || s[i] != '"') fail("expected a key");
            const std::string key = string();
            skip_ws();
            if (i >= s.size() || s[i] != ':') fail("expected ':'");
            ++i;
            o[key] = value();
            skip_ws();
            if (i >= s.size()) fail("unterminated object");
            if (s[i] == ',') {
                ++i;
                continue;
            }
            if (s[i] == '}') {
                ++i;
                return o;
            }
            fail("expected ',' or '}'");
        }
    }
};

void escape_to(std::string& out, const std::string& s) {
    out += '"';
    for (const char ch : s) {
        const unsigned char c = (unsigned char)ch;
        switch (c) {
            case '"': out += "\\\""; break;
            case '\\': out += "\\\\"; break;
            case '\b': out += "\\b"; break;
            case '\f': out += "\\f"; break;
            case '\n': out += "\\n"; break;
            case '\r': out += "\\r"; break;
            case '\t': out += "\\t"; break;
            default:
                if (c < 0x20) {
                    char buf[8];
                    std::snprintf(buf, sizeof(buf), "\\u%04x", c);
                    out += buf;
                } else {
                    out += ch;
                }
        }
    }
    out += '"';
}

}  // namespace

std::string format_double(double d) {
    if (!std::isfinite(d)) return "null";
    if (d == 0.0) return std::signbit(d) ? "-0.0" : "0.0";
    // shortest round-trip digits and decimal exponent
    char buf[64];
    auto r = std::to_chars(buf, buf + sizeof(buf), d, std::chars_format::scientific);
    std::string sci(buf, r.ptr);
    std::string out;
    size_t pos = 0;
    if (sci[0] == '-') {
        out += '-';
        pos = 1;
    }
    const size_t epos = sci.find('e');
    std::string digits;
    for (size_t k = pos; k < epos; ++k)
        if (sci[k] != '.') digits += sci[k];
    const int exp10 = std::stoi(sci.substr(epos + 1));
    const int k = (int)digits.size();
    const int n = exp10 + 1;  // position of the decimal point after the first n digits
    if (k <= n && n <= 15) {
        out += digits + std::string((size_t)(n - k), '0') + ".0";
    } else if (0 < n && n <= 15) {
        out += digits.substr(0, (size_t)n) + "." + digits.substr((size_t)n);
    } else if (-4 < n && n <= 0) {
        out += "0." + std::string((size_t)(-n), '0') + digits;
    } else {
        out += digits.substr(0, 1);
        if (k > 1) out += "." + digits.substr(1);
        const int e = n - 1;
        char eb[16];
        std::snprintf(eb, sizeof(eb), "e%c%02d", e < 0 ? '-' : '+', e < 0 ? -e : e);
        out += eb;
    }
    return out;
}

Json Json::parse(const std::string& text, bool allow_comments) {
    Parser p{text, 0, allow_comments};
    Json v = p.value();
    p.skip_ws();
    if (p.i != text.size()) p.fail("unexpected trailing characters");
    return v;
}

void Json::dump_to(std::string& out, int indent, int level) const {
    const bool pretty = indent >= 0;
    auto newline = [&](int lv) {
        if (!pretty) return;
        out += '\n';
        out.append((size_t)(indent * lv), ' ');
    };
    switch (kind_) {
        case Kind::Null: out += "null"; break;
        case Kind::Bool: out += b_ ? "true" : "false"; break;
        case Kind::Unsigned: out += std::to_string(u_); break;
        case Kind::Integer: out += std::to_string(i_); break;
        case Kind::Float: out += format_double(d_); break;
        case Kind::String: escape_to(out, s_); break;
        case Kind::Array:
            if (arr_.empty()) {
                out += "[]";
                break;
            }
            out += '[';
            for (size_t k = 0; k < arr_.size(); ++k) {
                if (k) out += ',';
                newline(level + 1);
                arr_[k].dump_to(out, indent, level + 1);
            }
            newline(level);
            out += ']';
            break;
        case Kind::Object:
            if (obj_.empty()) {
                out += "{}";
                break;
            }
            out += '{';
            for (size_t k = 0; k < obj_.size(); ++k) {
                if (k) out += ',';
                newline(level + 1);
                escape_to(out, obj_[k].first);
                out += pretty ? ": " : ":";
                obj_[k].second.dump_to(out, indent, level + 1);
            }
            newline(level);
            out += '}';
            break;
    }
}

std::string Json::dump(int indent) const {
    std::string out;
    dump_to(out, indent, 0);
    return out;
}

}  // namespace eng

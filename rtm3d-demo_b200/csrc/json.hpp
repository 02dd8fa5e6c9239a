// json.hpp -- a small JSON reader for input.json.  It keeps the number kinds the reference's
// parameter validation distinguishes (RTMParam::validateParameters, src/param/RTMParam.cpp:59-96):
// an unsigned integer, a signed (negative) integer and a float (written with '.', 'e' or 'E').
#pragma once
#include <cctype>
#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace rtmbjson {

enum class Kind { Null, Bool, Unsigned, Integer, Float, String, Array, Object };

struct Value {
    Kind kind = Kind::Null;
    bool b = false;
    double num = 0.0;
    unsigned long long u = 0;
    long long i = 0;
    std::string s;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;
};

inline const char *kind_name(Kind k) {
    switch (k) {
    case Kind::Null: return "Null";
    case Kind::Bool: return "Boolean";
    case Kind::Unsigned: return "Unsigned_Integer";
    case Kind::Integer: return "Signed_Integer";
    case Kind::Float: return "Float";
    case Kind::String: return "String";
    case Kind::Array: return "Array";
    case Kind::Object: return "Object";
    }
    return "?";
}

class Parser {
  public:
    explicit Parser(const std::string &text) : t_(text) {}

    Value parse() {
        Value v = value();
        ws();
        if (p_ != t_.size()) fail("trailing characters");
        return v;
    }

  private:
    const std::string &t_;
    size_t p_ = 0;

    [[noreturn]] void fail(const char *what) {
        throw std::runtime_error(std::string("JSON parse error at offset ") + std::to_string(p_) + ": " + what);
    }
    void ws() {
        while (p_ < t_.size() && std::isspace(static_cast<unsigned char>(t_[p_]))) ++p_;
    }
    bool eat(char c) {
        ws();
        if (p_ < t_.size() && t_[p_] == c) { ++p_; return true; }
        return false;
    }
    void expect(char c) {
        if (!eat(c)) fail("unexpected character");
    }
    std::string str() {
        expect('"');
        std::string out;
        while (p_ < t_.size() && t_[p_] != '"') {
            char c = t_[p_++];
            if (c == '\\') {
                if (p_ >= t_.size()) fail("bad escape");
                char e = t_[p_++];
                switch (e) {
                case 'n': out += '\n'; break;
                case 't': out += '\t'; break;
                case 'r': out += '\r'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'u': {  // basic multilingual plane only, UTF-8 encoded
                    if (p_ + 4 > t_.size()) fail("bad \\u escape");
                    unsigned cp = std::strtoul(t_.substr(p_, 4).c_str(), nullptr, 16);
                    p_ += 4;
                    if (cp < 0x80) out += char(cp);
                    else if (cp < 0x800) { out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F)); }
                    else { out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F)); }
                    break;
                }
                default: out += e;
                }
            } else {
                out += c;
            }
        }
        if (p_ >= t_.size()) fail("unterminated string");
        ++p_;
        return out;
    }
    Value value() {
        ws();
        if (p_ >= t_.size()) fail("unexpected end");
        Value v;
        char c = t_[p_];
        if (c == '{') {
            ++p_;
            v.kind = Kind::Object;
            if (eat('}')) return v;
            do {
                ws();
                std::string k = str();
                expect(':');
                v.obj[k] = value();
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            ++p_;
            v.kind = Kind::Array;
            if (eat(']')) return v;
            do v.arr.push_back(value());
            while (eat(','));
            expect(']');
        } else if (c == '"') {
            v.kind = Kind::String;
            v.s = str();
        } else if (t_.compare(p_, 4, "true") == 0) {
            p_ += 4; v.kind = Kind::Bool; v.b = true;
        } else if (t_.compare(p_, 5, "false") == 0) {
            p_ += 5; v.kind = Kind::Bool; v.b = false;
        } else if (t_.compare(p_, 4, "null") == 0) {
            p_ += 4;
        } else if (c == '-' || std::isdigit(static_cast<unsigned char>(c))) {
            size_t st = p_;
            bool is_float = false;
            if (t_[p_] == '-') ++p_;
            while (p_ < t_.size()) {
                char d = t_[p_];
                if (std::isdigit(static_cast<unsigned char>(d))) { ++p_; continue; }
                if (d == '.' || d == 'e' || d == 'E' || d == '+' || (d == '-' && p_ > st)) { is_float = true; ++p_; continue; }
                break;
            }
            std::string num = t_.substr(st, p_ - st);
            v.num = std::strtod(num.c_str(), nullptr);
            if (is_float) {
                v.kind = Kind::Float;
            } else if (num[0] == '-') {
                v.kind = Kind::Integer;
                v.i = std::strtoll(num.c_str(), nullptr, 10);
            } else {
                v.kind = Kind::Unsigned;
                v.u = std::strtoull(num.c_str(), nullptr, 10);
            }
        } else {
            fail("unexpected token");
        }
        return v;
    }
};

}  // namespace rtmbjson

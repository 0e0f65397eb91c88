/*
 * Minimal JSON reader/writer for scene files and frame output.
 *
 * Supports the full JSON grammar (objects, arrays, strings with escapes,
 * numbers, true/false/null). Numbers are kept as double, which represents
 * every float32 value written by scene generators exactly. Objects keep key
 * order. Errors throw JsonError with a byte offset; callers at the C ABI
 * catch them and return SPH_ERR_IO.
 */
#ifndef SPH2O_JSON_LITE_H
#define SPH2O_JSON_LITE_H

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace sphjson {

struct JsonError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

class Value {
public:
    enum Kind { Null, Bool, Number, String, Array, Object };

    Value() = default;
    static Value number(double d) { Value v; v.kind_ = Number; v.num_ = d; return v; }

    Kind kind() const { return kind_; }
    bool is_null() const { return kind_ == Null; }
    bool is_array() const { return kind_ == Array; }
    bool is_object() const { return kind_ == Object; }
    bool is_number() const { return kind_ == Number; }

    double as_number(const char* what = "value") const
    {
        if (kind_ == Number) return num_;
        if (kind_ == Bool) return b_ ? 1.0 : 0.0;
        throw JsonError(std::string("expected a number for ") + what);
    }
    bool as_bool(const char* what = "value") const
    {
        if (kind_ == Bool) return b_;
        if (kind_ == Number) return num_ != 0.0;
        throw JsonError(std::string("expected true or false for ") + what);
    }
    const std::string& as_string(const char* what = "value") const
    {
        if (kind_ != String) throw JsonError(std::string("expected a string for ") + what);
        return str_;
    }
    size_t size() const { return kind_ == Array ? arr_.size() : kind_ == Object ? obj_.size() : 0; }
    const Value& at(size_t i) const
    {
        if (kind_ != Array || i >= arr_.size()) throw JsonError("array index out of range");
        return arr_[i];
    }
    const Value* find(const std::string& key) const
    {
        if (kind_ != Object) return nullptr;
        for (const auto& kv : obj_)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    const Value& get(const std::string& key) const
    {
        const Value* v = find(key);
        if (!v) throw JsonError("missing key \"" + key + "\"");
        return *v;
    }
    const std::vector<std::pair<std::string, Value>>& items() const { return obj_; }

    friend class Parser;

private:
    Kind kind_ = Null;
    bool b_ = false;
    double num_ = 0.0;
    std::string str_;
    std::vector<Value> arr_;
    std::vector<std::pair<std::string, Value>> obj_;
};

class Parser {
public:
    explicit Parser(const std::string& text) : s_(text) {}

    Value parse()
    {
        Value v = value(0);
        ws();
        if (p_ != s_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& s_;
    size_t p_ = 0;

    [[noreturn]] void fail(const char* msg) const
    {
        throw JsonError(std::string("JSON parse error at byte ") + std::to_string(p_) + ": " + msg);
    }
    void ws()
    {
        while (p_ < s_.size() && (s_[p_] == ' ' || s_[p_] == '\t' || s_[p_] == '\n' || s_[p_] == '\r')) ++p_;
    }
    bool eat(char c)
    {
        ws();
        if (p_ < s_.size() && s_[p_] == c) { ++p_; return true; }
        return false;
    }
    void expect(char c)
    {
        if (!eat(c)) { char m[32]; snprintf(m, sizeof m, "expected '%c'", c); fail(m); }
    }
    bool lit(const char* w)
    {
        const size_t n = strlen(w);
        if (s_.compare(p_, n, w) == 0) { p_ += n; return true; }
        return false;
    }

    Value value(int depth)
    {
        if (depth > 256) fail("nesting too deep");
        ws();
        if (p_ >= s_.size()) fail("unexpected end of input");
        Value v;
        const char c = s_[p_];
        if (c == '{') {
            ++p_;
            v.kind_ = Value::Object;
            if (eat('}')) return v;
            do {
                ws();
                std::string k = string();
                expect(':');
                v.obj_.emplace_back(std::move(k), value(depth + 1));
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            ++p_;
            v.kind_ = Value::Array;
            if (eat(']')) return v;
            do { v.arr_.push_back(value(depth + 1)); } while (eat(','));
            expect(']');
        } else if (c == '"') {
            v.kind_ = Value::String;
            v.str_ = string();
        } else if (lit("true")) {
            v.kind_ = Value::Bool; v.b_ = true;
        } else if (lit("false")) {
            v.kind_ = Value::Bool; v.b_ = false;
        } else if (lit("null")) {
            v.kind_ = Value::Null;
        } else {
            v.kind_ = Value::Number;
            v.num_ = number();
        }
        return v;
    }

    double number()
    {
        const size_t start = p_;
        if (p_ < s_.size() && (s_[p_] == '-' || s_[p_] == '+')) ++p_;
        while (p_ < s_.size() && (isdigit((unsigned char)s_[p_]) || s_[p_] == '.' || s_[p_] == 'e' ||
                                  s_[p_] == 'E' || s_[p_] == '-' || s_[p_] == '+')) ++p_;
        if (p_ == start) fail("invalid value");
        const std::string tok = s_.substr(start, p_ - start);
        char* end = nullptr;
        const double d = strtod(tok.c_str(), &end);
        if (!end || *end != '\0') fail("invalid number");
        return d;
    }

    static void utf8(std::string& out, unsigned cp)
    {
        if (cp < 0x80) out += (char)cp;
        else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
        else if (cp < 0x10000) {
            out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
        } else {
            out += (char)(0xF0 | (cp >> 18)); out += (char)(0x80 | ((cp >> 12) & 0x3F));
            out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F));
        }
    }
    unsigned hex4()
    {
        if (p_ + 4 > s_.size()) fail("bad \\u escape");
        unsigned v = 0;
        for (int i = 0; i < 4; ++i) {
            const char h = s_[p_++];
            v <<= 4;
            if (h >= '0' && h <= '9') v |= (unsigned)(h - '0');
            else if (h >= 'a' && h <= 'f') v |= (unsigned)(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= (unsigned)(h - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string string()
    {
        if (p_ >= s_.size() || s_[p_] != '"') fail("expected string");
        ++p_;
        std::string out;
        while (true) {
            if (p_ >= s_.size()) fail("unterminated string");
            const char c = s_[p_++];
            if (c == '"') break;
            if (c != '\\') { out += c; continue; }
            if (p_ >= s_.size()) fail("bad escape");
            const char e = s_[p_++];
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
                unsigned cp = hex4();
                if (cp >= 0xD800 && cp < 0xDC00 && p_ + 6 <= s_.size() && s_[p_] == '\\' && s_[p_ + 1] == 'u') {
                    p_ += 2;
                    const unsigned lo = hex4();
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                utf8(out, cp);
                break;
            }
            default: fail("bad escape");
            }
        }
        return out;
    }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

/* Shortest decimal text that reads back as the same float (frame output). */
inline std::string format_float(float f)
{
    char buf[48];
    for (int prec = 6; prec <= 9; ++prec) {
        snprintf(buf, sizeof buf, "%.*g", prec, (double)f);
        if (strtof(buf, nullptr) == f) break;
    }
    return buf;
}

inline std::string format_double(double d)
{
    char buf[48];
    for (int prec = 15; prec <= 17; ++prec) {
        snprintf(buf, sizeof buf, "%.*g", prec, d);
        if (strtod(buf, nullptr) == d) break;
    }
    return buf;
}

} // namespace sphjson

#endif

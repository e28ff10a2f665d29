// Minimal JSON reader for simulation input files: objects, arrays, strings,
// numbers, true/false/null. Values are read with at(key) / at(index) and
// get_*() accessors that throw std::runtime_error naming the missing key or
// the wrong type, the way the reference's loadFromJSON reports bad input
// (src/simulation.cpp:118-208 reads its file with nlohmann::json `at()`).
#pragma once

#include <cstdlib>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace slab {
namespace json {

class Value {
  public:
    enum Kind { Null, Bool, Number, String, Array, Object };

    Kind kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Value> arr;
    std::map<std::string, Value> obj;
    std::string path = "$";  // where the value sits in the document, for messages

    bool contains(const std::string& key) const { return kind == Object && obj.count(key) != 0; }

    const Value& at(const std::string& key) const {
        if (kind != Object) throw std::runtime_error("JSON: " + path + " is not an object");
        auto it = obj.find(key);
        if (it == obj.end()) throw std::runtime_error("JSON: key '" + key + "' not found in " + path);
        return it->second;
    }
    const Value& operator[](size_t i) const {
        if (kind != Array) throw std::runtime_error("JSON: " + path + " is not an array");
        if (i >= arr.size()) throw std::runtime_error("JSON: index " + std::to_string(i) + " out of range in " + path);
        return arr[i];
    }
    double get_double() const {
        if (kind != Number) throw std::runtime_error("JSON: " + path + " is not a number");
        return num;
    }
    int get_int() const { return (int)get_double(); }
    bool get_bool() const {
        if (kind != Bool) throw std::runtime_error("JSON: " + path + " is not a boolean");
        return b;
    }
    const std::string& get_string() const {
        if (kind != String) throw std::runtime_error("JSON: " + path + " is not a string");
        return str;
    }
    size_t size() const { return kind == Array ? arr.size() : kind == Object ? obj.size() : 0; }
};

class Parser {
  public:
    explicit Parser(const std::string& text) : s_(text) {}

    Value parse() {
        Value v = value("$");
        ws();
        if (i_ != s_.size()) fail("trailing characters");
        return v;
    }

  private:
    const std::string& s_;
    size_t i_ = 0;

    [[noreturn]] void fail(const std::string& what) const {
        size_t line = 1, col = 1;
        for (size_t k = 0; k < i_ && k < s_.size(); ++k) {
            if (s_[k] == '\n') {
                ++line;
                col = 1;
            } else {
                ++col;
            }
        }
        throw std::runtime_error("JSON parse error at line " + std::to_string(line) + ", column " + std::to_string(col) + ": " + what);
    }

    void ws() {
        while (i_ < s_.size() && (s_[i_] == ' ' || s_[i_] == '\t' || s_[i_] == '\n' || s_[i_] == '\r')) ++i_;
    }

    bool eat(char c) {
        ws();
        if (i_ < s_.size() && s_[i_] == c) {
            ++i_;
            return true;
        }
        return false;
    }

    void expect(char c) {
        if (!eat(c)) fail(std::string("expected '") + c + "'");
    }

    bool word(const char* w) {
        size_t n = 0;
        while (w[n]) ++n;
        if (s_.compare(i_, n, w) == 0) {
            i_ += n;
            return true;
        }
        return false;
    }

    static void put_utf8(std::string& out, unsigned cp) {
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

    unsigned hex4() {
        if (i_ + 4 > s_.size()) fail("short \\u escape");
        unsigned v = 0;
        for (int k = 0; k < 4; ++k) {
            const char c = s_[i_++];
            v <<= 4;
            if (c >= '0' && c <= '9') v |= (unsigned)(c - '0');
            else if (c >= 'a' && c <= 'f') v |= (unsigned)(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= (unsigned)(c - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }

    std::string string_body() {
        std::string out;
        for (;;) {
            if (i_ >= s_.size()) fail("unterminated string");
            const char c = s_[i_++];
            if (c == '"') return out;
            if ((unsigned char)c < 0x20) fail("control character in string");
            if (c != '\\') {
                out += c;
                continue;
            }
            if (i_ >= s_.size()) fail("unterminated escape");
            const char e = s_[i_++];
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
                    if (cp >= 0xD800 && cp < 0xDC00) {  // surrogate pair
                        if (!(word("\\u"))) fail("lone high surrogate");
                        const unsigned lo = hex4();
                        if (lo < 0xDC00 || lo >= 0xE000) fail("bad low surrogate");
                        cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                    }
                    put_utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
    }

    Value value(const std::string& path) {
        ws();
        if (i_ >= s_.size()) fail("unexpected end of input");
        Value v;
        v.path = path;
        const char c = s_[i_];
        if (c == '{') {
            ++i_;
            v.kind = Value::Object;
            if (eat('}')) return v;
            do {
                ws();
                if (i_ >= s_.size() || s_[i_] != '"') fail("expected a key string");
                ++i_;
                std::string key = string_body();
                expect(':');
                Value item = value(path + "." + key);
                v.obj[key] = std::move(item);
            } while (eat(','));
            expect('}');
        } else if (c == '[') {
            ++i_;
            v.kind = Value::Array;
            if (eat(']')) return v;
            do {
                v.arr.push_back(value(path + "[" + std::to_string(v.arr.size()) + "]"));
            } while (eat(','));
            expect(']');
        } else if (c == '"') {
            ++i_;
            v.kind = Value::String;
            v.str = string_body();
        } else if (word("true")) {
            v.kind = Value::Bool;
            v.b = true;
        } else if (word("false")) {
            v.kind = Value::Bool;
            v.b = false;
        } else if (word("null")) {
            v.kind = Value::Null;
        } else if (c == '-' || (c >= '0' && c <= '9')) {
            const char* begin = s_.c_str() + i_;
            char* end = nullptr;
            v.kind = Value::Number;
            v.num = std::strtod(begin, &end);
            if (end == begin) fail("bad number");
            i_ += (size_t)(end - begin);
        } else {
            fail(std::string("unexpected character '") + c + "'");
        }
        return v;
    }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace json
}  // namespace slab

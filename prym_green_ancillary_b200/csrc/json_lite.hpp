// Minimal JSON reader for the instance and dense-block files (DOM, integers
// kept exact as int64 plus their source text).
#pragma once

#include <cctype>
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace bw {
namespace json {

struct Value {
    enum Kind { Null, Bool, Number, String, Array, Object } kind = Null;
    bool b = false;
    bool is_int = false;
    bool is_u64 = false;        // nonnegative integer above INT64_MAX (held in u)
    int64_t i = 0;
    uint64_t u = 0;
    double d = 0;
    std::string s;
    std::vector<Value> arr;
    std::vector<std::pair<std::string, Value>> obj;

    const Value* find(const std::string& key) const {
        if (kind != Object) return nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    const Value& at(const std::string& key) const {
        const Value* v = find(key);
        if (!v) throw std::runtime_error("missing JSON key '" + key + "'");
        return *v;
    }
    int64_t as_int(const std::string& label) const {
        if (kind != Number || !is_int) throw std::runtime_error("expected an integer for " + label);
        return i;
    }
    uint64_t as_u64(const std::string& label) const {
        if (kind == Number && is_u64) return u;
        int64_t v = as_int(label);
        if (v < 0) throw std::runtime_error("expected a nonnegative integer for " + label);
        return static_cast<uint64_t>(v);
    }
    // All integers of a (possibly nested) array, depth first.
    void flatten_ints(std::vector<int64_t>& out, const std::string& label) const {
        if (kind == Array) {
            for (const auto& e : arr) e.flatten_ints(out, label);
        } else {
            out.push_back(as_int(label));
        }
    }
    std::vector<int64_t> ints(const std::string& label) const {
        if (kind != Array) throw std::runtime_error("JSON key '" + label + "' is not an array");
        std::vector<int64_t> out;
        flatten_ints(out, label);
        return out;
    }
};

class Parser {
public:
    explicit Parser(const std::string& text) : t_(text) {}

    Value parse() {
        Value v = value();
        ws();
        if (p_ != t_.size()) fail("trailing characters");
        return v;
    }

private:
    const std::string& t_;
    size_t p_ = 0;

    [[noreturn]] void fail(const std::string& what) {
        throw std::runtime_error("JSON parse error at offset " + std::to_string(p_) + ": " + what);
    }
    void ws() {
        while (p_ < t_.size() && std::isspace(static_cast<unsigned char>(t_[p_]))) ++p_;
    }
    char peek() {
        ws();
        if (p_ >= t_.size()) fail("unexpected end");
        return t_[p_];
    }
    void expect(char c) {
        if (peek() != c) fail(std::string("expected '") + c + "'");
        ++p_;
    }
    Value value() {
        char c = peek();
        if (c == '{') return object();
        if (c == '[') return array();
        if (c == '"') {
            Value v;
            v.kind = Value::String;
            v.s = string();
            return v;
        }
        if (c == '-' || std::isdigit(static_cast<unsigned char>(c))) return number();
        if (t_.compare(p_, 4, "true") == 0) {
            p_ += 4;
            Value v;
            v.kind = Value::Bool;
            v.b = true;
            return v;
        }
        if (t_.compare(p_, 5, "false") == 0) {
            p_ += 5;
            Value v;
            v.kind = Value::Bool;
            return v;
        }
        if (t_.compare(p_, 4, "null") == 0) {
            p_ += 4;
            return Value{};
        }
        fail("unexpected character");
    }
    Value object() {
        Value v;
        v.kind = Value::Object;
        expect('{');
        if (peek() == '}') {
            ++p_;
            return v;
        }
        while (true) {
            if (peek() != '"') fail("expected a key");
            std::string key = string();
            expect(':');
            v.obj.emplace_back(std::move(key), value());
            char c = peek();
            ++p_;
            if (c == '}') break;
            if (c != ',') fail("expected ',' or '}'");
        }
        return v;
    }
    Value array() {
        Value v;
        v.kind = Value::Array;
        expect('[');
        if (peek() == ']') {
            ++p_;
            return v;
        }
        while (true) {
            v.arr.push_back(value());
            char c = peek();
            ++p_;
            if (c == ']') break;
            if (c != ',') fail("expected ',' or ']'");
        }
        return v;
    }
    std::string string() {
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
                    case 'u': {
                        if (p_ + 4 > t_.size()) fail("bad unicode escape");
                        unsigned cp = std::stoul(t_.substr(p_, 4), nullptr, 16);
                        p_ += 4;
                        if (cp < 0x80) out += static_cast<char>(cp);
                        else if (cp < 0x800) {
                            out += static_cast<char>(0xC0 | (cp >> 6));
                            out += static_cast<char>(0x80 | (cp & 0x3F));
                        } else {
                            out += static_cast<char>(0xE0 | (cp >> 12));
                            out += static_cast<char>(0x80 | ((cp >> 6) & 0x3F));
                            out += static_cast<char>(0x80 | (cp & 0x3F));
                        }
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
    Value number() {
        size_t start = p_;
        if (t_[p_] == '-') ++p_;
        while (p_ < t_.size() && std::isdigit(static_cast<unsigned char>(t_[p_]))) ++p_;
        bool integer = true;
        if (p_ < t_.size() && (t_[p_] == '.' || t_[p_] == 'e' || t_[p_] == 'E')) {
            integer = false;
            while (p_ < t_.size() && (std::isdigit(static_cast<unsigned char>(t_[p_])) || t_[p_] == '.' ||
                                      t_[p_] == 'e' || t_[p_] == 'E' || t_[p_] == '+' || t_[p_] == '-'))
                ++p_;
        }
        Value v;
        v.kind = Value::Number;
        std::string text = t_.substr(start, p_ - start);
        if (integer) {
            try {
                v.i = std::stoll(text);
                v.is_int = true;
                v.d = static_cast<double>(v.i);
            } catch (const std::exception&) {
                if (text[0] == '-') fail("integer out of range");
                try {
                    v.u = std::stoull(text);
                    v.is_u64 = true;
                    v.d = static_cast<double>(v.u);
                } catch (const std::exception&) {
                    fail("integer out of range");
                }
            }
        } else {
            v.d = std::stod(text);
        }
        return v;
    }
};

inline Value parse(const std::string& text) { return Parser(text).parse(); }

}  // namespace json
}  // namespace bw

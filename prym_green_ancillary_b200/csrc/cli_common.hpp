// Small command-line parser for the drop-in executables: accepts the options
// of the reference's CLI11 command lines (positional arguments, "--opt value",
// "--opt=value", short aliases and flags).
#pragma once

#include "../../include/bw_engine.h"

#include <cstdint>
#include <cstdlib>
#include <iostream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace bwcli {

struct Option {
    std::vector<std::string> names;
    std::string help;
    bool flag = false;
    bool required = false;
    std::string value;
    bool seen = false;
};

class Parser {
public:
    explicit Parser(std::string description) : desc_(std::move(description)) {}

    void positional(const std::string& name, const std::string& help) { pos_.push_back({{name}, help, false, true}); }
    void option(const std::vector<std::string>& names, const std::string& help, const std::string& def = "",
                bool required = false) {
        opts_.push_back({names, help, false, required, def});
    }
    void flag(const std::vector<std::string>& names, const std::string& help) {
        opts_.push_back({names, help, true, false, "0"});
    }

    // Returns false (after printing) for --help; throws on errors.
    bool parse(int argc, char** argv) {
        size_t next_pos = 0;
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help") {
                usage(argv[0]);
                return false;
            }
            if (a.size() > 1 && a[0] == '-' && !is_number(a)) {
                std::string name = a, val;
                const size_t eq = a.find('=');
                if (eq != std::string::npos) {
                    name = a.substr(0, eq);
                    val = a.substr(eq + 1);
                }
                Option* o = find(name);
                if (!o) throw std::runtime_error("The following argument was not expected: " + a);
                o->seen = true;
                if (o->flag) {
                    o->value = "1";
                } else if (eq != std::string::npos) {
                    o->value = val;
                } else {
                    if (i + 1 >= argc) throw std::runtime_error(name + " requires an argument");
                    o->value = argv[++i];
                }
            } else {
                if (next_pos >= pos_.size()) throw std::runtime_error("The following argument was not expected: " + a);
                pos_[next_pos].value = a;
                pos_[next_pos++].seen = true;
            }
        }
        for (auto& p : pos_)
            if (!p.seen) throw std::runtime_error(p.names[0] + " is required");
        for (auto& o : opts_)
            if (o.required && !o.seen) throw std::runtime_error(o.names.back() + " is required");
        return true;
    }

    std::string str(const std::string& name) const { return get(name).value; }
    bool has(const std::string& name) const { return get(name).seen; }
    bool on(const std::string& name) const { return get(name).value == "1"; }
    long long integer(const std::string& name) const {
        const std::string& v = get(name).value;
        char* end = nullptr;
        long long x = std::strtoll(v.c_str(), &end, 10);
        if (v.empty() || *end) throw std::runtime_error("Value " + v + " for " + name + " is not an integer");
        return x;
    }
    unsigned long long unsigned_integer(const std::string& name) const {
        const std::string& v = get(name).value;
        char* end = nullptr;
        if (!v.empty() && v[0] == '-') throw std::runtime_error("Value " + v + " for " + name + " must be nonnegative");
        unsigned long long x = std::strtoull(v.c_str(), &end, 10);
        if (v.empty() || *end) throw std::runtime_error("Value " + v + " for " + name + " is not an integer");
        return x;
    }

private:
    static bool is_number(const std::string& s) {
        if (s.size() < 2 || s[0] != '-') return false;
        for (size_t i = 1; i < s.size(); ++i)
            if (s[i] < '0' || s[i] > '9') return false;
        return true;
    }
    Option* find(const std::string& name) {
        for (auto& o : opts_)
            for (auto& n : o.names)
                if (n == name) return &o;
        return nullptr;
    }
    const Option& get(const std::string& name) const {
        for (auto& o : opts_)
            for (auto& n : o.names)
                if (n == name) return o;
        for (auto& p : pos_)
            if (p.names[0] == name) return p;
        throw std::logic_error("unknown option " + name);
    }
    void usage(const char* prog) const {
        std::cout << desc_ << "\nUsage: " << prog;
        for (auto& p : pos_) std::cout << " " << p.names[0];
        std::cout << " [OPTIONS]\n\nOptions:\n";
        for (auto& o : opts_) {
            std::cout << "  ";
            for (size_t i = 0; i < o.names.size(); ++i) std::cout << (i ? "," : "") << o.names[i];
            std::cout << (o.flag ? "" : " VALUE") << "\t" << o.help << "\n";
        }
    }
    std::string desc_;
    std::vector<Option> pos_, opts_;
};

inline void check(int status) {
    if (status != 0) throw std::runtime_error(bw_last_error());
}

}  // namespace bwcli

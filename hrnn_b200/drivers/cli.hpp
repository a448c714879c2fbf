// Command-line options, binary inputs and recall for the drivers.
//
// Options: the flag names, defaults and "--name value" / "--name=value" syntax of
// the reference drivers' program_options tables (src/hrnn_build.cpp:12-36,
// src/hrnn_search.cpp:51-82, src/hrnn_dynamic_test.cpp:102-157), parsed without
// Boost.  Inputs: the fbin and ground-truth layouts of include/utils.h.
#pragma once

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <functional>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <unordered_set>
#include <vector>

namespace cli {

class Options {
    struct Opt {
        std::string help, def;
        bool required = false, seen = false, is_flag = false;
        std::function<void(const std::string&)> set;
    };
    std::string title_;
    std::vector<std::string> order_;
    std::map<std::string, Opt> opts_;
    std::map<std::string, std::string> alias_;

    template <class T>
    static T parse(const std::string& s) {
        std::istringstream is(s);
        T v{};
        is >> v;
        if (is.fail() || !is.eof()) throw std::runtime_error("bad value '" + s + "'");
        return v;
    }

public:
    explicit Options(std::string title) : title_(std::move(title)) {}

    // name may be "long" or "long,s" (a one-letter alias)
    template <class T>
    Options& add(const std::string& name, T* target, const std::string& help, bool required = false,
                 const T& def = T()) {
        std::string lng = name, sh;
        if (auto c = name.find(','); c != std::string::npos) {
            lng = name.substr(0, c);
            sh = name.substr(c + 1);
            alias_[sh] = lng;
        }
        Opt o;
        o.help = help;
        o.required = required;
        if (!required) {
            *target = def;
            std::ostringstream os;
            os << def;
            o.def = os.str();
        }
        o.set = [target](const std::string& v) {
            if constexpr (std::is_same_v<T, std::string>) *target = v;
            else *target = parse<T>(v);
        };
        order_.push_back(lng);
        opts_[lng] = std::move(o);
        return *this;
    }

    void usage(std::ostream& os) const {
        os << title_ << ":\n  -h [ --help ]            Show help\n";
        for (const auto& n : order_) {
            const Opt& o = opts_.at(n);
            os << "  --" << n << " arg";
            if (!o.required) os << " (=" << o.def << ")";
            os << "    " << o.help << "\n";
        }
    }

    // Returns false after printing the usage for -h / --help.
    bool parse(int argc, char** argv) {
        for (int i = 1; i < argc; ++i) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help") {
                usage(std::cout);
                return false;
            }
            std::string name, val;
            bool has_val = false;
            if (a.rfind("--", 0) == 0) {
                name = a.substr(2);
            } else if (a.size() >= 2 && a[0] == '-') {
                name = a.substr(1);
                if (name.size() > 1 && alias_.count(name.substr(0, 1))) {  // -t1
                    val = name.substr(1);
                    name = name.substr(0, 1);
                    has_val = true;
                }
            } else {
                throw std::runtime_error("unexpected argument '" + a + "'");
            }
            if (auto e = name.find('='); e != std::string::npos) {
                val = name.substr(e + 1);
                name = name.substr(0, e);
                has_val = true;
            }
            if (alias_.count(name)) name = alias_[name];
            auto it = opts_.find(name);
            if (it == opts_.end()) throw std::runtime_error("unrecognised option '--" + name + "'");
            if (!has_val) {
                if (i + 1 >= argc) throw std::runtime_error("the option '--" + name + "' requires an argument");
                val = argv[++i];
            }
            it->second.set(val);
            it->second.seen = true;
        }
        for (const auto& n : order_)
            if (opts_.at(n).required && !opts_.at(n).seen)
                throw std::runtime_error("the option '--" + n + "' is required but missing");
        return true;
    }
};

// fbin: [n: u32][d: u32][n*d f32]
struct Fbin {
    uint32_t n = 0, d = 0;
    std::vector<float> data;
};

inline Fbin load_fbin(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Cannot open: " + path);
    Fbin b;
    f.read(reinterpret_cast<char*>(&b.n), 4);
    f.read(reinterpret_cast<char*>(&b.d), 4);
    b.data.resize((size_t)b.n * b.d);
    f.read(reinterpret_cast<char*>(b.data.data()), (std::streamsize)(b.data.size() * 4));
    if (!f) throw std::runtime_error("Read error: " + path);
    return b;
}

// RkNN ground truth: [nq: u32][(nq+1) u32 offsets][total u32 ids][total f32 dists]
struct RknnGt {
    uint32_t nq = 0;
    std::vector<uint32_t> off, ids;
    std::vector<float> dists;
    size_t count(size_t q) const { return off[q + 1] - off[q]; }
};

inline RknnGt load_rknn_gt(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("Cannot open: " + path);
    RknnGt g;
    f.read(reinterpret_cast<char*>(&g.nq), 4);
    g.off.resize((size_t)g.nq + 1);
    f.read(reinterpret_cast<char*>(g.off.data()), (std::streamsize)(g.off.size() * 4));
    const size_t tot = g.off.back();
    g.ids.resize(tot);
    g.dists.resize(tot);
    f.read(reinterpret_cast<char*>(g.ids.data()), (std::streamsize)(tot * 4));
    f.read(reinterpret_cast<char*>(g.dists.data()), (std::streamsize)(tot * 4));
    if (!f) throw std::runtime_error("Read error: " + path);
    return g;
}

struct Recall {
    double macro = 0, micro = 0, avg_results = 0;
};

// Macro recall: mean over queries with a non-empty ground truth of |R n G| / |G|;
// micro: sum |R n G| / sum |G| (include/utils.h:135-157, src/hrnn_search.cpp).
template <class Results>
Recall recall(const RknnGt& gt, const Results& res, size_t nq) {
    Recall r;
    double sum = 0;
    size_t counted = 0, found_all = 0, gt_all = 0;
    for (size_t q = 0; q < nq; ++q) {
        r.avg_results += (double)res[q].size();
        const size_t c = gt.count(q);
        if (c == 0) continue;
        std::unordered_set<uint32_t> s(gt.ids.begin() + gt.off[q], gt.ids.begin() + gt.off[q + 1]);
        size_t found = 0;
        for (auto l : res[q]) found += s.count((uint32_t)l);
        sum += (double)found / (double)c;
        counted++;
        found_all += found;
        gt_all += c;
    }
    r.macro = counted ? sum / (double)counted : 0.0;
    r.micro = gt_all ? (double)found_all / (double)gt_all : 0.0;
    r.avg_results = nq ? r.avg_results / (double)nq : 0.0;
    return r;
}

using Clock = std::chrono::steady_clock;
inline double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

inline std::vector<std::string> split(const std::string& s, char sep = ',') {
    std::vector<std::string> out;
    std::stringstream ss(s);
    std::string item;
    while (std::getline(ss, item, sep))
        if (!item.empty()) out.push_back(item);
    return out;
}

}  // namespace cli

// tuning.cpp -- the autotuned shape table (see ltl_kernels.h: tuning_lookup).
//
// The reference picks its tile counts by hand-run sweeps (NREGIONS_H/V in the
// README's GPU project, scripts/exploreRegionSizesLandscape.py:21-39).  Here the
// sweep is cat_cpu_b200/autotune.py; its winners are read back from a small text
// table, once per process.
#include <dlfcn.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "ltl_kernels.h"

namespace ltl {

namespace {

struct Entry {
    std::string variant;
    int radius = -1;  // -1: any
    long long nmin = 0, nmax = (1ll << 62);
    std::vector<std::pair<std::string, long long>> params;
};

std::vector<Entry> g_entries;
std::once_flag g_once;

std::string table_path() {
    if (const char* e = std::getenv("LTL_TUNING_FILE")) return e;
    Dl_info info;
    if (dladdr((void*)&tuning_lookup, &info) && info.dli_fname) {
        std::string so = info.dli_fname;
        size_t slash = so.rfind('/');
        std::string dir = slash == std::string::npos ? "." : so.substr(0, slash);
        return dir + "/tuning/ltl_tuning.txt";
    }
    return "";
}

void load() {
    const std::string path = table_path();
    if (path.empty()) return;
    FILE* f = std::fopen(path.c_str(), "r");
    if (!f) return;
    char line[1024];
    while (std::fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        Entry e;
        char* save = nullptr;
        for (char* tok = strtok_r(line, " \t\r\n", &save); tok; tok = strtok_r(nullptr, " \t\r\n", &save)) {
            char* eq = std::strchr(tok, '=');
            if (!eq) continue;
            *eq = '\0';
            const std::string k = tok, v = eq + 1;
            if (k == "variant") e.variant = v;
            else if (k == "radius") e.radius = (v == "*") ? -1 : std::atoi(v.c_str());
            else if (k == "nmin") e.nmin = std::atoll(v.c_str());
            else if (k == "nmax") e.nmax = std::atoll(v.c_str());
            else e.params.emplace_back(k, std::atoll(v.c_str()));
        }
        if (!e.variant.empty()) g_entries.push_back(e);
    }
    std::fclose(f);
}

}  // namespace

long long tuning_lookup(const char* variant, int radius, long long n, const char* param, long long fallback) {
    std::call_once(g_once, load);
    for (const Entry& e : g_entries) {
        if (e.variant != variant) continue;
        if (e.radius >= 0 && e.radius != radius) continue;
        if (n < e.nmin || n > e.nmax) continue;
        for (const auto& kv : e.params)
            if (kv.first == param) return kv.second;
    }
    return fallback;
}

}  // namespace ltl

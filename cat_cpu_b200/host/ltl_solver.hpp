// ltl_solver.hpp -- native C++ host mirror of the reference's solver interface
// over the C ABI (include/ltl.h), for programs that do not build against the
// reference tree.  Method names and argument meanings follow CASolver
// (kezada94/CAT_cpu src/CellularAutomata/Solvers/CASolver.h:7-28) and
// CPUBenchmark (src/CPUBenchmark.cpp:21-32); radius and rule are run-time values.
#pragma once

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>
#include <vector>

#include "ltl.h"

namespace ltl {

struct LtlError : std::runtime_error {
    int code;
    LtlError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

inline void check(int rc, const char* what) {
    if (rc != LTL_OK) throw LtlError(rc, std::string(what) + ": " + ltl_last_error());
}

class GpuSolver {
   public:
    GpuSolver(int deviceId, int n, int radius, int smin, int smax, int bmin, int bmax, int variant, int threads = 1)
        : n_(n), threads_(threads) {
        check(ltl_create(&ctx_, deviceId, n, radius, smin, smax, bmin, bmax, variant), "ltl_create");
    }
    ~GpuSolver() {
        if (ctx_) ltl_destroy(ctx_);
    }
    GpuSolver(const GpuSolver&) = delete;
    GpuSolver& operator=(const GpuSolver&) = delete;

    // CASolver::resetState(seed, density): CAStateGenerator with state seed `seed`.
    void resetState(int seed, float density) {
        std::vector<uint8_t> g((size_t)n_ * n_);
        check(ltl_generate_state(g.data(), (size_t)n_, n_, seed, density, threads_), "ltl_generate_state");
        setState(g.data());
    }
    void setState(const uint8_t* cells) { check(ltl_upload(ctx_, cells, (size_t)n_), "ltl_upload"); }
    void doStep() { doSteps(1); }
    void doSteps(int steps) { check(ltl_step(ctx_, steps), "ltl_step"); }
    void synchronize() { check(ltl_synchronize(ctx_), "ltl_synchronize"); }
    std::vector<uint8_t> getCurrentState() {
        std::vector<uint8_t> g((size_t)n_ * n_);
        check(ltl_download(ctx_, g.data(), (size_t)n_), "ltl_download");
        return g;
    }
    // The grid in the PACK coding: n rows of ceil(n / 64) uint64 words, cell
    // (i, j) = bit j % 64 of word j / 64 (ltl_upload_packed / ltl_download_packed).
    void setStatePacked(const uint64_t* words) {
        check(ltl_upload_packed(ctx_, words, 8 * (size_t)((n_ + 63) / 64)), "ltl_upload_packed");
    }
    std::vector<uint64_t> getCurrentStatePacked() {
        std::vector<uint64_t> w((size_t)n_ * ((n_ + 63) / 64));
        check(ltl_download_packed(ctx_, w.data(), 8 * (size_t)((n_ + 63) / 64)), "ltl_download_packed");
        return w;
    }
    void printCurrentState() {
        auto g = getCurrentState();
        for (int i = 0; i < n_; ++i) {
            for (int j = 0; j < n_; ++j) std::printf("%s ", g[(size_t)i * n_ + j] ? "1" : "-");
            std::printf("\n");
        }
    }
    // Shape parameters (ltl_set_param): "band_rows", "depth", ...
    void setParam(const char* name, long long value) { check(ltl_set_param(ctx_, name, value), "ltl_set_param"); }
    ltl_info info() const {
        ltl_info i{};
        check(ltl_get_info(ctx_, &i), "ltl_get_info");
        return i;
    }
    ltl_ctx* handle() { return ctx_; }
    int n() const { return n_; }

   private:
    ltl_ctx* ctx_ = nullptr;
    int n_ = 0;
    int threads_ = 1;
};

}  // namespace ltl

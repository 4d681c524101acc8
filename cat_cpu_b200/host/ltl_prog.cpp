// ltl_prog.cpp -- native CLI with the reference's shape for the GPU solvers.
//
//   ltl_prog n solver steps [-g deviceId] -d density [--seed S] [--threads T]
//            [--doVerify] [--radius R] [--rule SMIN SMAX BMIN BMAX] [--depth D]
//
// Mirrors kezada94/CAT_cpu src/main.cpp:31-130 with solver codes 7 (plain
// CUDA-core), 8 (tcgen05 tensor core), 9 (bit-packed).  The start grid is the
// reference benchmark's (CPUBenchmark.cpp:21-32), the timed region is
// doSteps(steps) plus device completion (CPUBenchmark.cpp:63-85), and stdout is
// the mean ms per step (StatsCollector.cpp:65-68).  --doVerify repeats the run on
// the plain GPU solver, one generation per pass, and compares every cell
// (main.cpp:64-90).  --depth sets solver 7's generations per pass (0: default).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "ltl_solver.hpp"

struct Args {
    int n = 0, solver = -1, steps = 0, device = 0, seed = 0, threads = 1, radius = 1, depth = 0;
    float density = -1.f;
    bool verify = false;
    int rule[4] = {2, 3, 3, 3};
};

static void usage() {
    std::printf(
        "usage: ltl_prog n solver steps [-g deviceId] -d density [--seed S] [--threads T] [--doVerify]\n"
        "                [--radius R] [--rule SMIN SMAX BMIN BMAX] [--depth D]\n"
        "  solver: 7 - GPU plain CUDA-core, 8 - GPU tcgen05 tensor core, 9 - GPU bit-packed\n");
}

static bool parse(int argc, char** argv, Args& a) {
    std::vector<std::string> pos;
    for (int i = 1; i < argc; ++i) {
        std::string s = argv[i];
        auto need = [&](int k) { return i + k < argc; };
        if ((s == "-g" || s == "--deviceId") && need(1)) a.device = std::atoi(argv[++i]);
        else if ((s == "-d" || s == "--density") && need(1)) a.density = std::strtof(argv[++i], nullptr);
        else if (s == "--seed" && need(1)) a.seed = std::atoi(argv[++i]);
        else if (s == "--threads" && need(1)) a.threads = std::atoi(argv[++i]);
        else if (s == "--radius" && need(1)) a.radius = std::atoi(argv[++i]);
        else if (s == "--rule" && need(4)) for (int k = 0; k < 4; ++k) a.rule[k] = std::atoi(argv[++i]);
        else if (s == "--depth" && need(1)) a.depth = std::atoi(argv[++i]);
        else if (s == "--doVerify") a.verify = true;
        else if (s == "-h" || s == "--help") return false;
        else pos.push_back(s);
    }
    if (pos.size() != 3 || a.density < 0.f) return false;
    a.n = std::atoi(pos[0].c_str());
    a.solver = std::atoi(pos[1].c_str());
    a.steps = std::atoi(pos[2].c_str());
    return true;
}

static int variant_for(int code) {
    switch (code) {
        case 7: return LTL_VARIANT_PLAIN;
        case 8: return LTL_VARIANT_TENSOR;
        case 9: return LTL_VARIANT_PACKED;
        default: return -100;
    }
}

int main(int argc, char** argv) {
    Args a;
    if (!parse(argc, argv, a)) {
        usage();
        return 1;
    }
    const int variant = variant_for(a.solver);
    if (variant == -100) {
        std::printf("main(): solver is NULL\n");
        return 1;
    }
    try {
        ltl::GpuSolver s(a.device, a.n, a.radius, a.rule[0], a.rule[1], a.rule[2], a.rule[3], variant, a.threads);
        if (a.depth > 0) s.setParam("depth", a.depth);
        const int state_seed = ltl_benchmark_seed(a.seed);
        s.resetState(state_seed, a.density);
        const int steps = a.steps;
        auto t0 = std::chrono::high_resolution_clock::now();
        s.doSteps(steps);
        s.synchronize();
        auto t1 = std::chrono::high_resolution_clock::now();
        const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count() / (steps > 0 ? steps : 1);
        std::printf("%f\n", ms);
        if (a.verify) {
            std::printf("\n[VERIFY] verifying...\n\n");
            ltl::GpuSolver ref(a.device, a.n, a.radius, a.rule[0], a.rule[1], a.rule[2], a.rule[3],
                               LTL_VARIANT_PLAIN, a.threads);
            ref.setParam("depth", 1);
            ref.resetState(state_seed, a.density);
            ref.doSteps(steps);
            if (s.getCurrentState() != ref.getCurrentState()) {
                std::printf("\n[VERIFY] verification FAILED!.\n\n");
                return 1;
            }
            std::printf("\n[VERIFY] verification successful.\n\n");
        }
    } catch (const ltl::LtlError& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}

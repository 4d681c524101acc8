// ref_dump.cpp -- golden-vector driver for the reference's own CPU solvers.
//
// TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile against the reference
// sources (kezada94/CAT_cpu src/), with the rule fixed by the same compile-time
// macros the reference uses (RADIUS SMIN SMAX BMIN BMAX, Makefile:10-14,27).
// Output goes to oracle/_ref/ only; nothing in the product links it.
//
// It builds a solver through the reference's factory
// (CASolverFactory::createSolver, src/CellularAutomata/CASolverFactory.cpp:6),
// seeds it the way CPUBenchmark::run/reset does (src/CPUBenchmark.cpp:4-32:
// omp_set_num_threads(T); srand(seed); resetState(rand() % 1000000, density)),
// advances it inside one OpenMP team the way CPUBenchmark::doOneRun does
// (src/CPUBenchmark.cpp:63-85), and dumps the inner n*n cells read back with
// getCurrentState() (src/CellularAutomata/Solvers/CASolver.cpp:9-13) after
// every requested checkpoint.
//
// usage: ref_dump <solver> <n> <seed> <density> <gen_threads> <run_threads> <out_prefix> <step>...
//   writes <out_prefix>_<step>.u8 (n*n bytes, row-major, values 0/1) for step 0
//   (the start grid) and for every listed cumulative step count.  The start grid
//   depends on the OpenMP thread count at resetState (one std::mt19937 per
//   thread, CAStateGenerator.h:14-26), so generation and stepping take separate
//   thread counts; the reference CLI uses --threads for both.
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <string>
#include <omp.h>

#include "CellularAutomata/CASolverFactory.h"

static int dump(CASolver* solver, int n, const std::string& prefix, int step) {
    CADataDomain<int>* d = solver->getCurrentState();
    std::vector<unsigned char> buf((size_t)n * n);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            buf[(size_t)i * n + j] = (unsigned char)d->getInnerElementAt(i, j);
    std::string path = prefix + "_" + std::to_string(step) + ".u8";
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return 1;
    size_t w = std::fwrite(buf.data(), 1, buf.size(), f);
    std::fclose(f);
    return w == buf.size() ? 0 : 1;
}

int main(int argc, char** argv) {
    if (argc < 8) {
        std::fprintf(stderr, "usage: %s solver n seed density gen_threads run_threads out_prefix [step...]\n",
                     argv[0]);
        return 2;
    }
    int code = std::atoi(argv[1]);
    int n = std::atoi(argv[2]);
    int seed = std::atoi(argv[3]);
    float density = std::stof(argv[4]);
    int gen_threads = std::atoi(argv[5]);
    int run_threads = std::atoi(argv[6]);
    std::string prefix = argv[7];

    CASolver* solver = CASolverFactory::createSolver(code, 0, n, RADIUS, run_threads);
    if (!solver) {
        std::fprintf(stderr, "solver %d not available\n", code);
        return 1;
    }
    omp_set_num_threads(gen_threads);
    std::srand(seed);
    int s = std::rand() % 1000000;
    solver->resetState(s, density);
    if (dump(solver, n, prefix, 0)) return 1;
    omp_set_num_threads(run_threads);

    int done = 0;
    for (int a = 8; a < argc; ++a) {
        int target = std::atoi(argv[a]);
        int k = target - done;
        if (k <= 0) continue;
#pragma omp parallel
        {
            solver->doSteps(k);
#pragma omp barrier
        }
        done = target;
        if (dump(solver, n, prefix, done)) return 1;
    }
    return 0;
}

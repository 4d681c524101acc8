// generator.cpp -- the reference's start grid, on the host (ltl_generate_state).
//
// Restates, for the GPU solvers' resetState, what the reference does before its
// timed run (kezada94/CAT_cpu):
//   ltl_benchmark_seed = CPUBenchmark::run/reset (src/CPUBenchmark.cpp:21-32):
//       srand(seed); s = rand() % 1000000; then solver->resetState(s, density)
//   ltl_generate_state = CAStateGenerator::generateRandomState
//       (src/Memory/CAStateGenerator.h:11-37), called by CASolver::resetState:
//       the n*n inner cells, row-major, split into `threads` contiguous chunks
//       of ceil(n*n/threads); chunk t drawn from std::mt19937(s + t), cell =
//       (double)(draw - min) / (max - min + 1) < density  (randomVal, :45-47).
// The start grid therefore depends on glibc rand(), on std::mt19937 and on the
// thread count, exactly as in the reference.  Chunks are independent, so they
// are generated concurrently here (one std::thread per chunk, in batches).
#include <cstdint>
#include <cstdlib>
#include <random>
#include <thread>
#include <vector>

#include "../../include/ltl.h"

void ltl_set_error(const char* fmt, ...);

extern "C" int ltl_benchmark_seed(int seed) {
    std::srand((unsigned)seed);
    return std::rand() % 1000000;
}

extern "C" int ltl_generate_state(uint8_t* out, size_t pitch, int n, int seed, float density, int threads) {
    if (!out || n < 1 || pitch < (size_t)n || threads < 1) {
        ltl_set_error("ltl_generate_state: bad arguments (n=%d, pitch=%zu, threads=%d)", n, pitch, threads);
        return LTL_EINVAL;
    }
    const int s = seed;
    const size_t total = (size_t)n * (size_t)n;
    const size_t chunk = (total + (size_t)threads - 1) / (size_t)threads;
    const double prob = (double)density;
    auto fill = [&](int t) {
        std::mt19937 rng((unsigned)(s + t));
        const double span = (double)(rng.max() - rng.min()) + 1.0;
        const size_t start = (size_t)t * chunk;
        for (size_t i = start; i < total && i < start + chunk; ++i) {
            const double u = (double)(rng() - rng.min()) / span;
            out[(i / (size_t)n) * pitch + (i % (size_t)n)] = (uint8_t)(u < prob);
        }
    };
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    for (int base = 0; base < threads; base += (int)hw) {
        std::vector<std::thread> pool;
        const int end = std::min(threads, base + (int)hw);
        for (int t = base + 1; t < end; ++t) pool.emplace_back(fill, t);
        fill(base);
        for (auto& th : pool) th.join();
    }
    return LTL_OK;
}

/*
 * ltl_oracle.c -- CPU restatement of the reference's Larger-than-Life step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA kernels in
 * cat_cpu_b200/csrc are compared against.  It is loaded by tests/, by
 * __graft_entry__.smoke() and by the cpu_baseline leg of bench.py, and by
 * nothing else: the product path never calls into it.
 *
 * What it restates (paths are relative to the reference project, kezada94/CAT_cpu):
 *   - the start grid of CPUBenchmark::run/reset        src/CPUBenchmark.cpp:21-32
 *     and CAStateGenerator::generateRandomState          src/Memory/CAStateGenerator.h:11-37,45-47
 *   - HostSolver<int>::CAStepAlgorithm                  src/CellularAutomata/Solvers/HostSolver.tpp:58-73
 *   - HostSolver<int>::countAliveNeighbors (centre excluded)             HostSolver.tpp:75-91
 *   - HostSolver<int>::transitionFunction ([a <= k <= b])                HostSolver.tpp:47-51
 *   - the torus halo fill (fillHorizontal/VerticalBoundaryConditions)    HostSolver.tpp:93-140
 * with radius and rule as run-time arguments instead of the reference's
 * compile-time RADIUS/SMIN/SMAX/BMIN/BMAX macros (Makefile:10-14,27).
 *
 * Halo semantics.  The reference keeps a halo of width RADIUS and refreshes it
 * before every step by copying inner rows/columns across the torus; for
 * n >= RADIUS this makes inner cell (i+dy, j+dx) read grid[(i+dy) mod n][(j+dx) mod n].
 * The restatement indexes modulo n directly, which is the same function.
 *
 * Pinning: tests/test_oracle_golden.py checks this file against grids dumped
 * by the reference's own HostSolver / AMXSolver16 (tests/golden/, made by
 * tests/golden/make_golden.py from binaries built by oracle/Makefile).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* MT19937, restated from Matsumoto & Nishimura (1998), "Mersenne Twister: a  */
/* 623-dimensionally equidistributed uniform pseudo-random number generator". */
/* Same output sequence as C++ std::mt19937 (default 32-bit parameters), which */
/* is what CAStateGenerator.h:17-18 instantiates.                             */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint32_t s[624];
    int idx;
} mt_state;

static void mt_seed(mt_state* m, uint32_t seed) {
    m->s[0] = seed;
    for (int i = 1; i < 624; ++i) {
        uint32_t p = m->s[i - 1];
        m->s[i] = 1812433253u * (p ^ (p >> 30)) + (uint32_t)i;
    }
    m->idx = 624;
}

static void mt_twist(mt_state* m) {
    for (int i = 0; i < 624; ++i) {
        uint32_t y = (m->s[i] & 0x80000000u) | (m->s[(i + 1) % 624] & 0x7fffffffu);
        uint32_t v = m->s[(i + 397) % 624] ^ (y >> 1);
        if (y & 1u) v ^= 0x9908b0dfu;
        m->s[i] = v;
    }
    m->idx = 0;
}

static uint32_t mt_next(mt_state* m) {
    if (m->idx >= 624) mt_twist(m);
    uint32_t y = m->s[m->idx++];
    y ^= y >> 11;
    y ^= (y << 7) & 0x9d2c5680u;
    y ^= (y << 15) & 0xefc60000u;
    y ^= y >> 18;
    return y;
}

/* First 32-bit output of std::mt19937(seed) after `skip` draws (used by tests
 * to check the generator against the C++ standard library). */
uint32_t oracle_mt19937_draw(uint32_t seed, uint32_t skip) {
    mt_state m;
    mt_seed(&m, seed);
    for (uint32_t i = 0; i < skip; ++i) mt_next(&m);
    return mt_next(&m);
}

/* CPUBenchmark::run: srand(seed); reset(): s = rand() % 1000000   (CPUBenchmark.cpp:21-32). */
int oracle_state_seed(int user_seed) {
    srand((unsigned)user_seed);
    return rand() % 1000000;
}

/*
 * CAStateGenerator::generateRandomState (CAStateGenerator.h:11-37): the n*n
 * inner cells in row-major order are split into `threads` contiguous chunks of
 * ceil(n*n/threads); chunk t is filled from std::mt19937(seed + t), one draw per
 * cell, cell = (double)draw / 2^32 < density  (randomVal, :45-47).
 * `density` is the float the CLI parsed (main.cpp:112-114); it is widened to
 * double for the comparison exactly as in the reference.
 * `out` is n*n bytes, row-major, no halo.
 */
void oracle_generate_from_state_seed(uint8_t* out, int n, int state_seed, float density, int threads) {
    size_t total = (size_t)n * (size_t)n;
    if (threads < 1) threads = 1;
    size_t chunk = (total + (size_t)threads - 1) / (size_t)threads;
    double prob = (double)density;
    for (int t = 0; t < threads; ++t) {
        mt_state m;
        mt_seed(&m, (uint32_t)(state_seed + t));
        size_t start = (size_t)t * chunk;
        for (size_t i = start; i < total && i < start + chunk; ++i) {
            double u = (double)mt_next(&m) / 4294967296.0;
            out[i] = (uint8_t)(u < prob);
        }
    }
}

/* Full start grid as CPUBenchmark::run builds it for a given --seed. */
void oracle_generate(uint8_t* out, int n, int user_seed, float density, int threads) {
    oracle_generate_from_state_seed(out, n, oracle_state_seed(user_seed), density, threads);
}

static inline int in_interval(int k, int a, int b) {
    /* transitionFunction(k,a,b) = [a <= k <= b]   (HostSolver.tpp:47-51) */
    return (k >= a) & (k <= b);
}

static inline int wrap(long v, int n) {
    long r = v % n;
    return (int)(r < 0 ? r + n : r);
}

/*
 * One step, direct O(R^2) neighbour sum exactly as countAliveNeighbors walks it
 * (HostSolver.tpp:75-91).  Used to pin the separable version below.
 */
void oracle_step_direct(const uint8_t* cur, uint8_t* next, int n, int radius,
                        int smin, int smax, int bmin, int bmax) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j < n; ++j) {
            int k = 0;
            for (int dy = -radius; dy <= radius; ++dy)
                for (int dx = -radius; dx <= radius; ++dx) {
                    if (dy == 0 && dx == 0) continue;
                    k += cur[(size_t)wrap(i + dy, n) * n + wrap(j + dx, n)];
                }
            int s = cur[(size_t)i * n + j];
            next[(size_t)i * n + j] =
                (uint8_t)(s * in_interval(k, smin, smax) + (1 - s) * in_interval(k, bmin, bmax));
        }
    }
}

/*
 * One step with separable sliding sums: column sums over the 2R+1 rows, then a
 * sliding window of 2R+1 column sums along each row; k = box - centre.  Same
 * function as oracle_step_direct for every n >= 1 (the windows are multisets of
 * torus rows/columns, so n < 2R+1 simply counts wrapped cells more than once,
 * which is what the reference's halo copies do for n >= RADIUS).
 */
void oracle_step(const uint8_t* cur, uint8_t* next, int n, int radius,
                 int smin, int smax, int bmin, int bmax) {
#pragma omp parallel
    {
        int* col = (int*)malloc(sizeof(int) * (size_t)n);
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) col[j] = 0;
            for (int dy = -radius; dy <= radius; ++dy) {
                const uint8_t* row = cur + (size_t)wrap(i + dy, n) * n;
                for (int j = 0; j < n; ++j) col[j] += row[j];
            }
            int box = 0;
            for (int dx = -radius; dx <= radius; ++dx) box += col[wrap(dx, n)];
            for (int j = 0; j < n; ++j) {
                int s = cur[(size_t)i * n + j];
                int k = box - s;
                next[(size_t)i * n + j] =
                    (uint8_t)(s * in_interval(k, smin, smax) + (1 - s) * in_interval(k, bmin, bmax));
                box += col[wrap(j + radius + 1, n)] - col[wrap(j - radius, n)];
            }
        }
        free(col);
    }
}

/* `steps` generations in place on `grid` (n*n bytes); `scratch` is n*n bytes.
 * Mirrors CASolver::doSteps (CASolver.cpp:15-31): fill halo, step, swap. */
void oracle_run(uint8_t* grid, uint8_t* scratch, int n, int radius,
                int smin, int smax, int bmin, int bmax, int steps) {
    uint8_t* a = grid;
    uint8_t* b = scratch;
    for (int s = 0; s < steps; ++s) {
        oracle_step(a, b, n, radius, smin, smax, bmin, bmax);
        uint8_t* t = a; a = b; b = t;
    }
    if (a != grid) memcpy(grid, a, (size_t)n * (size_t)n);
}

/* Neighbour counts (centre excluded) for every cell: the integer quantity the
 * tensor-core path must reproduce exactly before the rule is applied. */
void oracle_counts(const uint8_t* cur, int32_t* counts, int n, int radius) {
#pragma omp parallel
    {
        int* col = (int*)malloc(sizeof(int) * (size_t)n);
#pragma omp for schedule(static)
        for (int i = 0; i < n; ++i) {
            for (int j = 0; j < n; ++j) col[j] = 0;
            for (int dy = -radius; dy <= radius; ++dy) {
                const uint8_t* row = cur + (size_t)wrap(i + dy, n) * n;
                for (int j = 0; j < n; ++j) col[j] += row[j];
            }
            int box = 0;
            for (int dx = -radius; dx <= radius; ++dx) box += col[wrap(dx, n)];
            for (int j = 0; j < n; ++j) {
                counts[(size_t)i * n + j] = box - cur[(size_t)i * n + j];
                box += col[wrap(j + radius + 1, n)] - col[wrap(j - radius, n)];
            }
        }
        free(col);
    }
}

uint64_t oracle_population(const uint8_t* grid, size_t cells) {
    uint64_t p = 0;
    for (size_t i = 0; i < cells; ++i) p += grid[i];
    return p;
}

void oracle_set_threads(int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
}

"""Python handle on the CPU restatement oracle (oracle/ltl_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py to check or time the CUDA path.  The product
(cat_cpu_b200) never imports this module.

Every function mirrors a reference function (paths inside kezada94/CAT_cpu):
  generate      -> CPUBenchmark::run/reset (src/CPUBenchmark.cpp:21-32) +
                   CAStateGenerator::generateRandomState (src/Memory/CAStateGenerator.h:11-37)
  step / run    -> HostSolver<int>::CAStepAlgorithm + halo fill, CASolver::doSteps
                   (src/CellularAutomata/Solvers/HostSolver.tpp:58-140, CASolver.cpp:15-31)
  counts        -> HostSolver<int>::countAliveNeighbors (HostSolver.tpp:75-91)
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    """Compile liboracle.so with the system gcc (see oracle/Makefile)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        i32p = ctypes.POINTER(ctypes.c_int32)
        L.oracle_generate.argtypes = [u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_int]
        L.oracle_generate_from_state_seed.argtypes = [u8p, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                                      ctypes.c_int]
        L.oracle_state_seed.argtypes = [ctypes.c_int]
        L.oracle_state_seed.restype = ctypes.c_int
        L.oracle_mt19937_draw.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_mt19937_draw.restype = ctypes.c_uint32
        for name in ("oracle_step", "oracle_step_direct"):
            getattr(L, name).argtypes = [u8p, u8p] + [ctypes.c_int] * 6
        L.oracle_run.argtypes = [u8p, u8p] + [ctypes.c_int] * 7
        L.oracle_counts.argtypes = [u8p, i32p, ctypes.c_int, ctypes.c_int]
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _u8(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))


def set_threads(t):
    lib().oracle_set_threads(int(t))


def state_seed(user_seed):
    return lib().oracle_state_seed(int(user_seed))


def mt19937_draw(seed, skip=0):
    return lib().oracle_mt19937_draw(seed, skip)


def generate(n, seed, density, threads=1):
    """Start grid (n x n uint8) exactly as the reference builds it for `--seed seed
    -d density --threads threads` (glibc rand() for the state seed, one
    std::mt19937 per generator thread)."""
    out = np.empty((n, n), dtype=np.uint8)
    lib().oracle_generate(_u8(out), n, int(seed), float(density), int(threads))
    return out


def step(grid, radius, rule, direct=False):
    smin, smax, bmin, bmax = rule
    g = np.ascontiguousarray(grid, dtype=np.uint8)
    n = g.shape[0]
    out = np.empty_like(g)
    f = lib().oracle_step_direct if direct else lib().oracle_step
    f(_u8(g), _u8(out), n, radius, smin, smax, bmin, bmax)
    return out


def run(grid, radius, rule, steps):
    smin, smax, bmin, bmax = rule
    g = np.array(grid, dtype=np.uint8, copy=True, order="C")
    scratch = np.empty_like(g)
    lib().oracle_run(_u8(g), _u8(scratch), g.shape[0], radius, smin, smax, bmin, bmax, int(steps))
    return g


def counts(grid, radius):
    g = np.ascontiguousarray(grid, dtype=np.uint8)
    out = np.empty(g.shape, dtype=np.int32)
    lib().oracle_counts(_u8(g), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), g.shape[0], radius)
    return out


# ---------------------------------------------------------------------------
# Rules.  The reference's k excludes the centre (HostSolver.tpp:84-85), so a
# rule quoted with the centre counted maps to survival bounds - 1, birth as is.
# ---------------------------------------------------------------------------
BOSCO_R5 = (32, 56, 34, 45)   # Bosco S33-57 / B34-45 (centre counted), R=5
CONWAY = (2, 3, 3, 3)         # the reference Makefile defaults (Makefile:10-14)

# Per-radius rule table of the reference's sweep scripts (scripts/RunBenchmark.py:21-26),
# already in the reference's centre-excluded convention; index = radius - 1.
SWEEP_SMIN = [2, 7, 15, 40, 35, 49, 101, 163, 108, 122, 156, 170, 213, 245, 170, 170]
SWEEP_SMAX = [3, 12, 23, 80, 59, 81, 201, 223, 181, 211, 265, 296, 364, 420, 296, 296]
SWEEP_BMIN = [3, 8, 14, 41, 34, 46, 75, 74, 100, 123, 147, 170, 203, 234, 170, 170]
SWEEP_BMAX = [3, 11, 17, 80, 45, 65, 170, 252, 140, 170, 205, 240, 283, 326, 240, 300]
SWEEP_DENSITY = [0.07, 0.15, 0.25, 0.50, 0.21, 0.22, 0.29, 0.23, 0.24, 0.25, 0.24, 0.25, 0.25, 0.25,
                 0.28, 0.26]


def sweep_rule(radius):
    i = radius - 1
    return (SWEEP_SMIN[i], SWEEP_SMAX[i], SWEEP_BMIN[i], SWEEP_BMAX[i])


def scaled_rule(radius):
    """Interval rule scaled to N=(2R+1)^2 with the centre counted: birth
    [ceil(0.34N), floor(0.45N)], survival [ceil(0.33N), floor(0.57N)]; returned in
    the reference's centre-excluded convention (survival bounds - 1).  Integer
    arithmetic, so no floating-point rounding enters the thresholds."""
    N = (2 * radius + 1) ** 2
    ceil_div = lambda a, b: -((-a) // b)
    bmin, bmax = ceil_div(34 * N, 100), (45 * N) // 100
    smin, smax = ceil_div(33 * N, 100) - 1, (57 * N) // 100 - 1
    return (smin, smax, bmin, bmax)

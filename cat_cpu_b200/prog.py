"""Command-line driver with the reference's CLI shape, for the GPU solvers.

    python -m cat_cpu_b200.prog n solver steps [-g deviceId] [-d density] [--seed S]
                                [--threads T] [--doVerify] [--radius R]
                                [--rule SMIN SMAX BMIN BMAX] [--depth D]

Mirrors the reference's main.cpp (kezada94/CAT_cpu src/main.cpp:31-130):
`solver` selects the GPU solver (7 = plain CUDA-core, 8 = tcgen05 tensor core,
9 = bit-packed; the reference's 0-6 are its CPU solvers), the start grid is the
reference benchmark's (srand(seed); resetState(rand() % 1000000, density) with
`threads` generator threads, CPUBenchmark.cpp:21-32), and stdout is the mean
milliseconds per step (StatsCollector::printShortStats, StatsCollector.cpp:65-68).
Radius and rule default to the reference's compile-time defaults (Makefile:10-14:
R=1, S2-3, B3-3) and are run-time options here.

--depth sets solver 7's generations per kernel pass (temporal blocking; 0 keeps
the tuned default).  --doVerify re-runs the same start grid on the plain GPU
solver (code 7, one generation per pass) and compares every cell, printing the reference's "[VERIFY] ..." lines; exit 1 on a
mismatch (main.cpp:64-90).
"""
import argparse
import sys

import numpy as np


def parse(argv):
    ap = argparse.ArgumentParser(prog="cat_cpu_b200.prog", description="LtL on B200 (GPU solvers 7/8/9)")
    ap.add_argument("n", type=int)
    ap.add_argument("solver", type=int, help="7 plain, 8 tensor core, 9 bit-packed")
    ap.add_argument("steps", type=int)
    ap.add_argument("-g", "--deviceId", type=int, default=0)
    ap.add_argument("-d", "--density", type=float, required=True)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--threads", type=int, default=1)
    ap.add_argument("--doVerify", action="store_true")
    ap.add_argument("--radius", type=int, default=1)
    ap.add_argument("--rule", type=int, nargs=4, default=[2, 3, 3, 3], metavar=("SMIN", "SMAX", "BMIN", "BMAX"))
    ap.add_argument("--depth", type=int, default=0,
                    help="solver 7: generations per kernel pass (0 = the tuned default)")
    return ap.parse_args(argv)


def run(args):
    import torch
    import cat_cpu_b200 as C

    torch.cuda.set_device(args.deviceId)
    solver = C.CASolverFactory.createSolver(args.solver, args.deviceId, args.n, args.radius, args.threads,
                                            tuple(args.rule))
    if solver is None:
        print("main(): solver is NULL")
        return 1, None, None
    if args.depth:
        solver.set_param("depth", args.depth)
    start = C.start_grid(args.n, args.seed, args.density, args.threads)
    solver.setState(start)
    stream = torch.cuda.Stream()
    solver.set_stream(stream.cuda_stream)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    steps = args.steps
    a.record(stream)
    solver.doSteps(steps)
    b.record(stream)
    solver.synchronize()
    ms = a.elapsed_time(b) / max(steps, 1)
    return 0, solver, (start, steps, ms)


def main(argv=None):
    args = parse(sys.argv[1:] if argv is None else argv)
    rc, solver, res = run(args)
    if rc:
        return rc
    start, steps, ms = res
    print(f"{ms:f}")
    if args.doVerify:
        import cat_cpu_b200 as C
        print("\n[VERIFY] verifying...\n")
        ref = C.CASolverFactory.createSolver(7, args.deviceId, args.n, args.radius, args.threads,
                                             tuple(args.rule))
        if ref.radius <= 5:
            ref.set_param("depth", 1)  # one generation per pass: independent of the temporally blocked kernel
        ref.setState(start)
        ref.doSteps(steps)
        if not np.array_equal(solver.getCurrentState(), ref.getCurrentState()):
            print("\n[VERIFY] verification FAILED!.\n")
            return 1
        print("\n[VERIFY] verification successful.\n")
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""Generate tests/golden/golden.json from the reference's own CPU solvers.

Run where the reference sources (kezada94/CAT_cpu) are present, with
$LTL_REFERENCE naming their directory (the script's built-in default is the
directory they were mounted at when the fixtures were made):

    python tests/golden/make_golden.py [--jobs 8] [--only NAME_SUBSTRING]

For every case it builds the reference for the case's rule (oracle/Makefile,
target `ref`, into oracle/_ref/), runs oracle/ref_dump.cpp -- which drives the
reference's CASolverFactory / resetState / doSteps exactly as its CPUBenchmark
does -- and records, for the start grid and every checkpoint, the SHA-256 and
population of the inner n*n cells (uint8, row-major).  Grids with n <= 128 are
also stored whole (np.packbits, base64) so that a failing test can show cells.

The reference is not needed at test time: tests read golden.json only.
"""
import argparse
import base64
import concurrent.futures as cf
import hashlib
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.abspath(os.path.join(HERE, "..", ".."))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

REF = os.environ.get("LTL_REFERENCE", "/root/reference")


def cases():
    out = []
    bosco = O.BOSCO_R5
    # Config 1 of the benchmark plan: 1024^2, seed 0, d=0.5, R=5 Bosco, 100 steps.
    out.append(dict(name="config1_bosco_r5_n1024", solver=0, radius=5, rule=bosco, n=1024, seed=0,
                    density=0.5, gen_threads=1, run_threads=8, steps=[1, 10, 100]))
    # Same, but generated with 8 threads: pins the per-thread mt19937 chunking.
    out.append(dict(name="config1_gen8threads", solver=0, radius=5, rule=bosco, n=1024, seed=0,
                    density=0.5, gen_threads=8, run_threads=8, steps=[1, 10]))
    # Config 2: 16384^2, seed 1.  Solver 0 at steps 1 and 10; AMX16 (solver 2,
    # bit-identical to solver 0 for R <= 16, n % 16 == 0) out to 1000 steps.
    out.append(dict(name="config2_bosco_r5_n16384_solver0", solver=0, radius=5, rule=bosco, n=16384,
                    seed=1, density=0.5, gen_threads=1, run_threads=8, steps=[1, 10]))
    out.append(dict(name="config2_bosco_r5_n16384_amx16", solver=2, radius=5, rule=bosco, n=16384,
                    seed=1, density=0.5, gen_threads=1, run_threads=8, steps=[1, 10, 100, 1000]))
    # The reference sweep table (scripts/RunBenchmark.py:21-26), R = 1..16, on an
    # odd size and a multiple of 16.
    for r in range(1, 17):
        rule = O.sweep_rule(r)
        d = O.SWEEP_DENSITY[r - 1]
        out.append(dict(name=f"sweep_r{r}_n97", solver=0, radius=r, rule=rule, n=97, seed=r, density=d,
                        gen_threads=1, run_threads=8, steps=[1, 5, 20]))
        out.append(dict(name=f"sweep_r{r}_n128", solver=0, radius=r, rule=rule, n=128, seed=100 + r,
                        density=d, gen_threads=1, run_threads=8, steps=[1, 5, 20]))
    # Config 3 radii with the scaled interval rule, as 1024^2 crop runs (seed 2).
    for r in (1, 2, 4, 8, 16, 32):
        out.append(dict(name=f"scaled_r{r}_n1024", solver=0, radius=r, rule=O.scaled_rule(r), n=1024,
                        seed=2, density=0.5, gen_threads=1, run_threads=8, steps=[1, 10, 20]))
    # Config 4 radii at small n (seed 3, d=0.3); n = 2R+1 is the smallest torus
    # whose window does not overlap itself.
    for r in (64, 128):
        out.append(dict(name=f"scaled_r{r}_n300", solver=0, radius=r, rule=O.scaled_rule(r), n=300,
                        seed=3, density=0.3, gen_threads=1, run_threads=8, steps=[1, 3, 6]))
    out.append(dict(name="scaled_r64_n129", solver=0, radius=64, rule=O.scaled_rule(64), n=129, seed=3,
                    density=0.3, gen_threads=1, run_threads=8, steps=[1, 4]))
    out.append(dict(name="scaled_r17_n100", solver=0, radius=17, rule=O.scaled_rule(17), n=100, seed=7,
                    density=0.4, gen_threads=1, run_threads=8, steps=[1, 5, 10]))
    out.append(dict(name="scaled_r5_n333", solver=0, radius=5, rule=O.scaled_rule(5), n=333, seed=11,
                    density=0.45, gen_threads=1, run_threads=8, steps=[1, 10, 30]))
    # The scaled rule flips a uniform grid to all-alive / all-dead within a step
    # or two unless the density sits near an interval edge; these densities keep
    # the checked steps mixed, so the counts near every threshold are exercised.
    out.append(dict(name="mixed_r128_n400_d448", solver=0, radius=128, rule=O.scaled_rule(128), n=400, seed=3,
                    density=0.448, gen_threads=1, run_threads=8, steps=[1, 2, 3]))
    out.append(dict(name="mixed_r64_n300_d45", solver=0, radius=64, rule=O.scaled_rule(64), n=300, seed=3,
                    density=0.45, gen_threads=1, run_threads=8, steps=[1, 2, 3, 6]))
    for r in (8, 16, 32):
        out.append(dict(name=f"mixed_r{r}_n1024_d46", solver=0, radius=r, rule=O.scaled_rule(r), n=1024,
                        seed=3, density=0.46, gen_threads=1, run_threads=8, steps=[1, 2, 6]))
    out.append(dict(name="edge_bosco_r5_n7_d25", solver=0, radius=5, rule=bosco, n=7, seed=6, density=0.25,
                    gen_threads=1, run_threads=1, steps=[1, 2, 10]))
    out.append(dict(name="edge_conway_n4", solver=0, radius=1, rule=O.CONWAY, n=4, seed=13, density=0.4,
                    gen_threads=1, run_threads=1, steps=[1, 2, 5]))
    # Edge sizes: n = 2R+1, R < n < 2R+1 (window wraps onto itself), tiny grids.
    out.append(dict(name="edge_bosco_r5_n11", solver=0, radius=5, rule=bosco, n=11, seed=5, density=0.5,
                    gen_threads=1, run_threads=1, steps=[1, 2, 10]))
    out.append(dict(name="edge_bosco_r5_n7", solver=0, radius=5, rule=bosco, n=7, seed=6, density=0.5,
                    gen_threads=1, run_threads=1, steps=[1, 2, 10]))
    out.append(dict(name="edge_conway_n3", solver=0, radius=1, rule=O.CONWAY, n=3, seed=8, density=0.5,
                    gen_threads=1, run_threads=1, steps=[1, 2, 5]))
    out.append(dict(name="edge_conway_n64", solver=0, radius=1, rule=O.CONWAY, n=64, seed=9, density=0.35,
                    gen_threads=1, run_threads=1, steps=[1, 10, 50]))
    out.append(dict(name="edge_sweep_r8_n17", solver=0, radius=8, rule=O.sweep_rule(8), n=17, seed=10,
                    density=0.23, gen_threads=1, run_threads=1, steps=[1, 3, 9]))
    # Non-multiple-of-16 mid size with Bosco, for the tiled kernels' ragged edges.
    out.append(dict(name="ragged_bosco_r5_n1000", solver=0, radius=5, rule=bosco, n=1000, seed=12,
                    density=0.5, gen_threads=1, run_threads=8, steps=[1, 10, 50]))
    return out


def rule_tag(radius, rule):
    smin, smax, bmin, bmax = rule
    return f"R{radius}_S{smin}-{smax}_B{bmin}-{bmax}_portable"


def build(radius, rule, jobs):
    smin, smax, bmin, bmax = rule
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), f"-j{jobs}", "ref", f"REF={REF}",
                    f"R={radius}", f"SMIN={smin}", f"SMAX={smax}", f"BMIN={bmin}", f"BMAX={bmax}"],
                   check=True, stdout=subprocess.DEVNULL)
    return os.path.join(ROOT, "oracle", "_ref", rule_tag(radius, rule), "ref_dump")


def run_case(case, exe):
    with tempfile.TemporaryDirectory() as td:
        prefix = os.path.join(td, "g")
        t0 = time.time()
        cmd = [exe, str(case["solver"]), str(case["n"]), str(case["seed"]), repr(case["density"]),
               str(case["gen_threads"]), str(case["run_threads"]), prefix] + [str(s) for s in case["steps"]]
        subprocess.run(cmd, check=True, cwd=td, stdout=subprocess.DEVNULL)
        n = case["n"]
        cps = []
        for s in [0] + case["steps"]:
            g = np.fromfile(f"{prefix}_{s}.u8", dtype=np.uint8)
            assert g.size == n * n
            cp = dict(step=s, sha256=hashlib.sha256(g.tobytes()).hexdigest(), population=int(g.sum()))
            if n <= 128:
                cp["bits_b64"] = base64.b64encode(np.packbits(g).tobytes()).decode()
            cps.append(cp)
        rec = {k: case[k] for k in ("name", "solver", "radius", "n", "seed", "density", "gen_threads")}
        rec["rule"] = list(case["rule"])
        rec["checkpoints"] = cps
        rec["ref_seconds"] = round(time.time() - t0, 2)
        return rec


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--only", default=None)
    ap.add_argument("--out", default=os.path.join(HERE, "golden.json"))
    args = ap.parse_args()
    todo = [c for c in cases() if args.only is None or args.only in c["name"]]
    exes = {}
    for c in todo:
        key = (c["radius"], tuple(c["rule"]))
        if key not in exes:
            exes[key] = build(c["radius"], c["rule"], args.jobs)
    old = {}
    if os.path.exists(args.out):
        old = {c["name"]: c for c in json.load(open(args.out))["cases"]}
    for c in todo:
        print(f"[golden] {c['name']} ...", flush=True)
        rec = run_case(c, exes[(c["radius"], tuple(c["rule"]))])
        print(f"[golden] {c['name']} done in {rec['ref_seconds']} s", flush=True)
        old[c["name"]] = rec
    order = [c["name"] for c in cases()]
    recs = [old[k] for k in order if k in old]
    doc = {
        "reference": "kezada94/CAT_cpu (solver 0 = HostSolver<int>, solver 2 = AMXSolver16)",
        "made_by": "tests/golden/make_golden.py via oracle/ref_dump.cpp",
        "grid": "inner n*n cells, uint8 0/1, row-major; sha256 over those bytes",
        "cases": recs,
    }
    with open(args.out, "w") as f:
        json.dump(doc, f, indent=1)
    print(f"wrote {args.out} ({len(recs)} cases)")


if __name__ == "__main__":
    main()

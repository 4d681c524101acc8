"""Build libltl_b200.so (the C-ABI library) in-tree with nvcc for sm_100a.

    python -m cat_cpu_b200.build [--force] [--jobs N] [--verbose]

Every .cu / .cpp under cat_cpu_b200/csrc is compiled separately (objects in
cat_cpu_b200/_build/) and linked into cat_cpu_b200/libltl_b200.so.  Objects are
rebuilt when their source or any header under csrc/ or include/ is newer.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libltl_b200.so")
PROG = os.path.join(PKG, "ltl_prog")
HOST = os.path.join(PKG, "host")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-ccbin", "g++", "-Xcompiler", "-fPIC,-O3",
          "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def sources():
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    return srcs


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(ROOT, "include", "*.h")))


def _compile(src, force, verbose, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in headers()])
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    cmd = [NVCC] + ARCH + COMMON + extra + ["-c", src, "-o", obj]
    if src.endswith(".cpp"):
        cmd = [NVCC] + COMMON + ["-x", "c++", "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, f"compile failed: {src}\n{r.stdout}\n{r.stderr}"
    if verbose and r.stderr.strip():
        print(r.stderr, flush=True)
    return obj, None


def build(force=False, jobs=None, verbose=False, ptxas_verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    srcs = sources()
    jobs = jobs or min(len(srcs), os.cpu_count() or 4)
    objs, errors = [], []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, err in ex.map(lambda s: _compile(s, force, verbose or ptxas_verbose, extra), srcs):
            objs.append(obj)
            if err:
                errors.append(err)
    if errors:
        raise RuntimeError("\n".join(errors))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        # shared CUDA runtime: one runtime instance per process, shared with torch
        cmd = [NVCC] + ARCH + ["-shared", "-ccbin", "g++", "-cudart", "shared", "-o", LIB] + objs + \
            ["-lpthread", "-ldl", "-lrt"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed\n{r.stdout}\n{r.stderr}")
    src = os.path.join(HOST, "ltl_prog.cpp")
    deps = [src, os.path.join(HOST, "ltl_solver.hpp"), os.path.join(ROOT, "include", "ltl.h"), LIB]
    if force or not os.path.exists(PROG) or os.path.getmtime(PROG) < max(os.path.getmtime(d) for d in deps):
        cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), "-I", HOST, src, "-o", PROG,
               "-L", PKG, "-lltl_b200", "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"ltl_prog build failed\n{r.stdout}\n{r.stderr}")
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    try:
        print(build(a.force, a.jobs, a.verbose, a.ptxas_verbose))
    except RuntimeError as e:
        print(e, file=sys.stderr)
        sys.exit(1)


if __name__ == "__main__":
    main()

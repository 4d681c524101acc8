"""The GPU solvers inside the reference's own harness, and the native CLI.

prog_gpu is the reference's main.cpp / CPUBenchmark / CADataDomainComparator
built from its sources with cat_cpu_b200/integration dropped in (oracle/Makefile
target `dropin`); --doVerify makes the reference itself compare the GPU solver
against its solver 0 (HostSolver<int>) cell by cell.  Marked `gpu`.
"""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROG_GPU = os.path.join(ROOT, "oracle", "_ref", "R5_S32-56_B34-45_portable", "prog_gpu")
LTL_PROG = os.path.join(ROOT, "cat_cpu_b200", "ltl_prog")


@pytest.mark.parametrize("code", [7, 8, 9])
def test_reference_harness_verifies_gpu_solver(code):
    if not os.path.exists(PROG_GPU):
        pytest.skip("prog_gpu not built (needs the reference sources at build time)")
    threads = str(min(16, os.cpu_count() or 1))
    r = subprocess.run([PROG_GPU, "1024", str(code), "100", "-d", "0.5", "--seed", "0", "--threads", threads,
                        "--doVerify"], capture_output=True, text=True, timeout=600, cwd="/tmp")
    assert r.returncode == 0, r.stdout + r.stderr
    assert "[VERIFY] verification successful." in r.stdout, r.stdout
    float(r.stdout.strip().splitlines()[0])  # the reference's ms/step line


@pytest.mark.parametrize("code", [7, 8, 9])
def test_native_cli_verify(code):
    r = subprocess.run([LTL_PROG, "2000", str(code), "50", "-d", "0.5", "--seed", "3", "--radius", "5", "--rule",
                        "32", "56", "34", "45", "--doVerify"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "[VERIFY] verification successful." in r.stdout


def test_native_cli_unknown_solver():
    r = subprocess.run([LTL_PROG, "64", "3", "1", "-d", "0.5"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "solver is NULL" in r.stdout

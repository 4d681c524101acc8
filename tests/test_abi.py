"""C-ABI checks that need no GPU: the library loads, exports every entry point
include/ltl.h declares, its host-side generator reproduces the reference's
start grids, and argument errors come back as status codes."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from tests.goldutil import sha

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "ltl.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ltl_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_header_symbol():
    import cat_cpu_b200 as C
    L = C.lib()
    names = header_functions()
    assert len(names) >= 25
    for name in names:
        assert hasattr(L, name), f"{name} declared in include/ltl.h but not exported"
    assert set(names) == set(C.ltl.ABI_SYMBOLS)


def test_version_and_error_string():
    import cat_cpu_b200 as C
    assert b"sm_100a" in C.lib().ltl_version()
    assert isinstance(C.lib().ltl_last_error(), bytes)


def test_generator_matches_oracle_and_golden(golden):
    import cat_cpu_b200 as C
    for name in ("config1_bosco_r5_n1024", "config1_gen8threads", "ragged_bosco_r5_n1000", "sweep_r7_n97",
                 "edge_conway_n3"):
        c = golden[name]
        g = C.start_grid(c["n"], c["seed"], c["density"], c["gen_threads"])
        assert sha(g) == c["checkpoints"][0]["sha256"], name
        assert np.array_equal(g, O.generate(c["n"], c["seed"], c["density"], c["gen_threads"]))


def test_generator_pitch_and_threads():
    import cat_cpu_b200 as C
    L = C.lib()
    n, pitch = 37, 64
    buf = np.full((n, pitch), 7, dtype=np.uint8)
    assert L.ltl_generate_state(ctypes.c_void_p(buf.ctypes.data), pitch, n, 1234, 0.3, 3) == 0
    assert np.all(buf[:, n:] == 7)
    want = np.empty((n, n), dtype=np.uint8)
    O.lib().oracle_generate_from_state_seed(want.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n, 1234,
                                            ctypes.c_float(0.3), 3)
    assert np.array_equal(buf[:, :n], want)


def test_argument_errors_without_device():
    import cat_cpu_b200 as C
    L = C.lib()
    h = ctypes.c_void_p()
    assert L.ltl_create(None, 0, 64, 5, 32, 56, 34, 45, 0) == C.ltl.EINVAL
    assert L.ltl_create(ctypes.byref(h), 0, 4, 5, 32, 56, 34, 45, 0) == C.ltl.EINVAL  # n < radius
    assert L.ltl_create(ctypes.byref(h), 0, 64, 0, 0, 0, 0, 0, 0) == C.ltl.EINVAL
    assert L.ltl_create(ctypes.byref(h), 0, 64, 5, 32, 56, 34, 45, 17) == C.ltl.EINVAL  # unknown variant
    assert L.ltl_generate_state(None, 8, 8, 1, 0.5, 1) == C.ltl.EINVAL
    assert L.ltl_step(None, 1) == C.ltl.EINVAL
    assert L.ltl_download(None, None, 0) == C.ltl.EINVAL
    assert L.ltl_pack_device(None, 0, 1, 1, None, 8, None) == C.ltl.EINVAL
    assert L.ltl_destroy(None) == 0


def test_no_device_is_a_cuda_error_not_a_fallback():
    from tests.conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is present")
    import cat_cpu_b200 as C
    with pytest.raises(C.LtlError) as e:
        C.CUDASolver(64, 5, O.BOSCO_R5)
    assert e.value.code == C.ltl.ECUDA


def test_factory_unknown_code_returns_none():
    import cat_cpu_b200 as C
    assert C.CASolverFactory.createSolver(0, 0, 64, 5, 1, O.BOSCO_R5) is None
    assert C.CASolverFactory.createSolver(42, 0, 64, 5, 1, O.BOSCO_R5) is None


def test_pack_coding_helpers():
    """pack_grid / unpack_grid (the host side of ltl_upload_packed and
    ltl_download_packed) against the PACK coding written out cell by cell:
    cell (i, j) = bit j % 64 of uint64 word j / 64, bits past the row's end 0."""
    import cat_cpu_b200 as C
    rng = np.random.default_rng(8)
    for rows, n in ((3, 1), (4, 63), (5, 64), (2, 65), (7, 200), (1, 128)):
        g = (rng.random((rows, n)) < 0.5).astype(np.uint8)
        w = C.pack_grid(g)
        assert w.dtype == np.uint64 and w.shape == (rows, (n + 63) // 64)
        want = np.zeros_like(w)
        for i in range(rows):
            for j in range(n):
                if g[i, j]:
                    want[i, j // 64] |= np.uint64(1) << np.uint64(j % 64)
        assert np.array_equal(w, want)
        assert np.array_equal(C.unpack_grid(w, n), g)


def test_packed_io_argument_errors_without_device():
    import cat_cpu_b200 as C
    L = C.lib()
    buf = (ctypes.c_uint64 * 4)()
    assert L.ltl_upload_packed(None, buf, 32) == C.ltl.EINVAL
    assert L.ltl_download_packed(None, buf, 32) == C.ltl.EINVAL

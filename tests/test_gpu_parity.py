"""GPU parity: every variant of libltl_b200, called through its C ABI, against
the reference's golden vectors and the CPU restatement oracle.  Bit-exact.

Marked `gpu`: needs a CUDA device and the built cat_cpu_b200/libltl_b200.so.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from tests.goldutil import sha, describe_mismatch

pytestmark = pytest.mark.gpu

C = None


def setup_module(module):
    global C
    import cat_cpu_b200 as _C
    C = _C
    O.set_threads(os.cpu_count() or 8)


VARIANTS = ["plain", "packed", "tensor"]
VCODE = {"plain": 0, "tensor": 1, "packed": 2}


def supported(variant, n, r):
    if variant == "packed":
        return r <= 32 and n >= r
    if variant == "tensor":
        return r <= 128 and n >= r
    return n >= r


def make(variant, n, r, rule):
    return C.CUDASolver(n, r, rule, variant=VCODE[variant])


def run_golden_case(variant, c, max_step=None):
    n, r, rule = c["n"], c["radius"], tuple(c["rule"])
    g0 = C.start_grid(n, c["seed"], c["density"], c["gen_threads"])
    assert sha(g0) == c["checkpoints"][0]["sha256"]
    s = make(variant, n, r, rule)
    try:
        s.setState(g0)
        done = 0
        for cp in c["checkpoints"][1:]:
            if max_step is not None and cp["step"] > max_step:
                break
            s.doSteps(cp["step"] - done)
            done = cp["step"]
            got = s.getCurrentState()
            if sha(got) != cp["sha256"]:
                want = O.run(g0, r, rule, done) if n * n <= 4096 * 4096 else None
                msg = describe_mismatch(got, want) if want is not None else "sha differs"
                pytest.fail(f"{variant} {c['name']} step {done}: {msg}")
            assert s.population() == cp["population"]
    finally:
        s.close()


SMALL_CASES = None


def small_case_names(golden):
    return sorted(k for k, c in golden.items() if c["n"] <= 1100)


@pytest.mark.parametrize("variant", VARIANTS)
def test_golden_small(golden, variant):
    ran = 0
    for name in small_case_names(golden):
        c = golden[name]
        if not supported(variant, c["n"], c["radius"]):
            continue
        run_golden_case(variant, c)
        ran += 1
    assert ran >= 20


@pytest.mark.parametrize("variant", VARIANTS)
def test_golden_config2_16384(golden, variant):
    """16384^2, seed 1, R=5 Bosco: steps 1, 10, 100, 1000 against the reference."""
    run_golden_case(variant, golden["config2_bosco_r5_n16384_amx16"])


@pytest.mark.parametrize("variant", VARIANTS)
def test_random_vs_oracle_every_step(variant):
    rng = np.random.default_rng(11 + VCODE[variant])
    for trial in range(24):
        r = int(rng.choice([1, 2, 3, 4, 5, 6, 7, 8, 11, 16, 17, 24, 32, 40, 64, 91, 113, 128]))
        if not supported(variant, 10 ** 6, r):
            continue
        n = int(rng.integers(max(r, 1), max(r + 2, 4 * r + 70)))
        N = (2 * r + 1) ** 2
        d = float(rng.uniform(0.2, 0.6))
        lo = int(rng.integers(0, N // 2))
        rule = (lo, lo + int(rng.integers(0, N // 2)), int(rng.integers(0, N // 2)), int(rng.integers(N // 3, N)))
        g = (rng.random((n, n)) < d).astype(np.uint8)
        s = make(variant, n, r, rule)
        try:
            s.setState(g)
            for step in range(4):
                g = O.step(g, r, rule)
                s.doStep()
                got = s.getCurrentState()
                assert np.array_equal(got, g), f"{variant} n={n} r={r} rule={rule} step {step + 1}: " + \
                    describe_mismatch(got, g)
        finally:
            s.close()


def test_plain_temporal_depths_vs_oracle():
    """The temporally blocked plain kernel (2 or 3 generations per pass) against
    the oracle: every R it supports, ragged and tiny sides, several band heights
    (bands that end inside the grid and bands longer than the grid), and step
    counts that leave a shorter last pass."""
    rng = np.random.default_rng(29)
    for r in (1, 2, 3, 4, 5):
        for depth in (2, 3):
            if depth * r > 16:
                continue
            for trial in range(3):
                n = int(rng.choice([r, r + 1, 17, 97, 130, 263, 600]))
                band = int(rng.choice([16, 23, 64, 128, 700]))
                steps = int(rng.integers(1, 8))
                N = (2 * r + 1) ** 2
                lo = int(rng.integers(0, N // 3))
                rule = (lo, lo + int(rng.integers(1, N // 2)), int(rng.integers(0, N // 3)), int(rng.integers(N // 3, N)))
                g = (rng.random((n, n)) < rng.uniform(0.25, 0.6)).astype(np.uint8)
                s = make("plain", n, r, rule)
                try:
                    s.set_param("depth", depth)
                    s.set_param("band_rows", band)
                    assert s.info.temporal_depth == depth
                    s.setState(g)
                    s.doSteps(steps)
                    want = O.run(g, r, rule, steps)
                    got = s.getCurrentState()
                    assert np.array_equal(got, want), \
                        f"R={r} depth={depth} n={n} band={band} steps={steps} rule={rule}: " + describe_mismatch(got, want)
                finally:
                    s.close()


def test_packed_band_rows_and_strip_edges_vs_oracle():
    """Bit-packed step with the built-in band choice (0) and explicit bands, on
    sides whose word count is a multiple of 32 (the last strip ends at the last
    inner word, whose right neighbour is the halo word) and sides that leave a
    partial last word or a lone halo lane in the last strip."""
    rng = np.random.default_rng(31)
    for n in (1024, 1000, 1056, 2048 + 32, 97):
        for band in (0, 16, 37, 4096):
            r = int(rng.choice([1, 3, 5, 8, 13]))
            N = (2 * r + 1) ** 2
            lo = int(rng.integers(0, N // 3))
            rule = (lo, lo + int(rng.integers(1, N // 2)), int(rng.integers(0, N // 3)), int(rng.integers(N // 3, N)))
            g = (rng.random((n, n)) < rng.uniform(0.25, 0.6)).astype(np.uint8)
            s = make("packed", n, r, rule)
            try:
                s.set_param("band_rows", band)
                s.setState(g)
                s.doSteps(3)
                want = O.run(g, r, rule, 3)
                got = s.getCurrentState()
                assert np.array_equal(got, want), f"n={n} R={r} band={band}: " + describe_mismatch(got, want)
            finally:
                s.close()


def test_plain_default_depth_and_limits():
    s = make("plain", 1024, 5, O.BOSCO_R5)
    try:
        assert s.info.temporal_depth in (1, 2, 3)
        with pytest.raises(C.LtlError):
            s.set_param("depth", 4)        # 4 * 5 > 16
        s.set_param("depth", 1)
        assert s.info.temporal_depth == 1
    finally:
        s.close()
    s = make("plain", 300, 8, O.sweep_rule(8))
    try:
        with pytest.raises(C.LtlError):
            s.set_param("depth", 2)        # R > 5 runs the generic kernel only
    finally:
        s.close()


@pytest.mark.parametrize("variant", VARIANTS)
def test_counts_near_thresholds_r5(variant):
    """Every count value 0..120 sits on a threshold at least once: sweep rules over
    a dense random grid so that an off-by-one anywhere in the count flips cells."""
    n, r = 509, 5
    g = (np.random.default_rng(3).random((n, n)) < 0.5).astype(np.uint8)
    for t in range(0, 121, 7):
        rule = (t, t + 3, t + 1, t + 2)
        s = make(variant, n, r, rule)
        try:
            s.setState(g)
            s.doStep()
            want = O.step(g, r, rule)
            got = s.getCurrentState()
            assert np.array_equal(got, want), f"{variant} rule {rule}: " + describe_mismatch(got, want)
        finally:
            s.close()


def test_population_and_compare_device():
    import torch
    n = 777
    g = C.start_grid(n, 5, 0.4, 1)
    s = make("plain", n, 5, O.BOSCO_R5)
    try:
        s.setState(g)
        assert s.population() == int(g.sum())
        dev = torch.from_numpy(g).cuda()
        mm, first = s.compare_device(dev.data_ptr(), n)
        assert (mm, first) == (0, -1)
        g2 = g.copy()
        g2[3, 4] ^= 1
        g2[100, 200] ^= 1
        dev2 = torch.from_numpy(g2).cuda()
        torch.cuda.synchronize()
        mm, first = s.compare_device(dev2.data_ptr(), n)
        assert mm == 2 and first == 3 * n + 4
        out = torch.zeros((n, n), dtype=torch.uint8, device="cuda")
        s.download_device(out.data_ptr(), n)
        s.synchronize()
        assert np.array_equal(out.cpu().numpy(), g)
    finally:
        s.close()


def test_upload_device_and_streams():
    import torch
    n = 300
    g = C.start_grid(n, 9, 0.5, 1)
    dev = torch.from_numpy(g).cuda()
    st = torch.cuda.Stream()
    for variant in VARIANTS:
        s = make(variant, n, 5, O.BOSCO_R5)
        try:
            s.set_stream(st.cuda_stream)
            s.upload_device(dev.data_ptr(), n)
            s.doSteps(20)
            s.synchronize()
            assert np.array_equal(s.getCurrentState(), O.run(g, 5, O.BOSCO_R5, 20)), variant
        finally:
            s.close()


def test_pack_codec_roundtrip():
    import torch
    import ctypes
    L = C.lib()
    rng = np.random.default_rng(2)
    for rows, cols in [(1, 1), (3, 63), (5, 64), (7, 65), (64, 1000), (129, 4096)]:
        cells = (rng.random((rows, cols)) < 0.5).astype(np.uint8)
        d_cells = torch.from_numpy(cells).cuda()
        nw = (cols + 63) // 64
        d_words = torch.zeros((rows, nw), dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()
        C.ltl.check(L.ltl_pack_device(ctypes.c_void_p(d_cells.data_ptr()), cols, rows, cols,
                                      ctypes.c_void_p(d_words.data_ptr()), nw * 8, None))
        torch.cuda.synchronize()
        words = d_words.cpu().numpy().view(np.uint64)
        want = np.zeros((rows, nw), dtype=np.uint64)
        for j in range(cols):
            want[:, j // 64] |= cells[:, j].astype(np.uint64) << np.uint64(j % 64)
        assert np.array_equal(words, want), (rows, cols)
        back = torch.zeros((rows, cols), dtype=torch.uint8, device="cuda")
        C.ltl.check(L.ltl_unpack_device(ctypes.c_void_p(d_words.data_ptr()), nw * 8, rows, cols,
                                        ctypes.c_void_p(back.data_ptr()), cols, None))
        torch.cuda.synchronize()
        assert np.array_equal(back.cpu().numpy(), cells)


@pytest.mark.parametrize("variant", VARIANTS)
def test_packed_host_io_vs_oracle(variant):
    """ltl_upload_packed / ltl_download_packed (PACK-coded host grids) against the
    uint8 transfers and the oracle: ragged and multiple-of-32/64 widths, uploads
    in either form followed by downloads in either form, and steps in between."""
    rng = np.random.default_rng(21 + VCODE[variant])
    for n, r, rule in ((97, 3, O.sweep_rule(3)), (128, 5, O.BOSCO_R5), (200, 8, O.scaled_rule(8)),
                       (64, 1, O.CONWAY), (300, 2, O.sweep_rule(2))):
        g = (rng.random((n, n)) < 0.45).astype(np.uint8)
        w = C.pack_grid(g)
        s = make(variant, n, r, rule)
        try:
            s.setStatePacked(w)
            assert np.array_equal(s.getCurrentState(), g)
            assert np.array_equal(s.getCurrentStatePacked(), w)
            s.doSteps(3)
            g3 = O.run(g, r, rule, 3)
            assert np.array_equal(s.getCurrentStatePacked(), C.pack_grid(g3)), (variant, n, r)
            s.setState(g)                      # uint8 in, packed out
            assert np.array_equal(s.getCurrentStatePacked(), w)
            s.setStatePacked(C.pack_grid(g3))  # packed in, step, uint8 out
            s.doStep()
            assert np.array_equal(s.getCurrentState(), O.step(g3, r, rule))
        finally:
            s.close()
    if variant == "packed":
        rows, n = 77, 160
        g = (rng.random((rows, n)) < 0.5).astype(np.uint8)
        s = C.CUDASolver(n, 4, O.sweep_rule(4), variant=C.VARIANT_PACKED, rows=rows)
        try:
            s.setStatePacked(C.pack_grid(g))
            assert np.array_equal(s.getCurrentState(), g)
        finally:
            s.close()


def test_errors_on_device():
    with pytest.raises(C.LtlError) as e:
        C.CUDASolver(64, 40, (1, 2, 3, 4), variant=VCODE["packed"])
    assert e.value.code == C.ltl.EUNSUPPORTED
    with pytest.raises(C.LtlError) as e:
        C.CUDASolver(64, 5, O.BOSCO_R5, device=99)
    assert e.value.code == C.ltl.ECUDA


def test_tensor_bounded_wait_reports_timeout_and_recovers():
    """Failure detection without a fault: a withheld completion signal makes the
    tensor kernel's bounded waits run out; the host sees LTL_ETIMEOUT, and the
    same context computes correctly after a fresh upload."""
    n, r = 300, 5
    g = C.start_grid(n, 8, 0.5, 1)
    s = make("tensor", n, r, O.BOSCO_R5)
    try:
        s.set_param("wait_limit_ns", 20_000_000)
        s.set_param("inject_missing_commit", 1)
        s.setState(g)
        s.doStep()
        with pytest.raises(C.LtlError) as e:
            s.synchronize()
        assert e.value.code == C.ltl.ETIMEOUT
        s.set_param("inject_missing_commit", 0)
        s.setState(g)
        s.doSteps(3)
        s.synchronize()
        assert np.array_equal(s.getCurrentState(), O.run(g, r, O.BOSCO_R5, 3))
    finally:
        s.close()

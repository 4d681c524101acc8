"""ltl_step_noalloc: the plain step for callers that may not allocate device
memory (a framework owning all device memory through its own pool, a service
that forbids allocation after start-up, a plug-in given only buffers and a
stream).  Its scratch is a fixed array inside the library; these tests check,
through the C ABI, that two calls in a row give exactly what the regular
allocating entry point gives, that no device memory is allocated by the calls,
and that oversized grids are refused.  Collected last on purpose.  Marked gpu.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _regular(C, L, dev_in, n, radius, rule, steps, torch):
    """The existing allocating path (ltl_create / upload / step / download), plain variant."""
    s = C.CUDASolver(n, radius, rule, variant=C.VARIANT_PLAIN)
    try:
        out = torch.empty((n, n), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        s.upload_device(dev_in.data_ptr(), n)
        s.doSteps(steps)
        s.download_device(out.data_ptr(), n)
        s.synchronize()
        return out.cpu().numpy()
    finally:
        s.close()


def _noalloc(C, L, dev_in, dev_out, n, radius, rule, steps):
    smin, smax, bmin, bmax = rule
    rc = L.ltl_step_noalloc(ctypes.c_void_p(dev_in.data_ptr()), n, ctypes.c_void_p(dev_out.data_ptr()), n, n,
                            radius, smin, smax, bmin, bmax, steps, None)
    return rc


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    import cat_cpu_b200 as C
    L = C.lib()
    cases = [(1000, 5, (32, 56, 34, 45), 7, 1), (777, 3, (15, 23, 14, 17), 4, 2), (300, 8, (95, 163, 99, 130), 3, 3)]
    for k, (n, radius, rule, steps, seed) in enumerate(cases):
        g = C.start_grid(n, seed, 0.45, 1)
        dev_in = torch.from_numpy(g).cuda()
        want = _regular(C, L, dev_in, n, radius, rule, steps, torch)
        outs = []
        for call in range(2):  # two calls in a row on the shared scratch
            dev_out = torch.zeros((n, n), dtype=torch.uint8, device="cuda")
            torch.cuda.synchronize()
            free_before = torch.cuda.mem_get_info()[0]
            assert _noalloc(C, L, dev_in, dev_out, n, radius, rule, steps) == 0, L.ltl_last_error()
            torch.cuda.synchronize()
            if call == 1:  # (the first call may load kernels lazily; the second must change nothing)
                assert torch.cuda.mem_get_info()[0] == free_before, "ltl_step_noalloc allocated device memory"
            outs.append(dev_out.cpu().numpy())
        for call, got in enumerate(outs):
            assert np.array_equal(got, want), f"case {k} call {call}: {int((got != want).sum())} cells differ"


def test_noalloc_in_place_and_stream():
    import torch
    import cat_cpu_b200 as C
    L = C.lib()
    n, radius, rule, steps = 512, 5, (32, 56, 34, 45), 10
    g = C.start_grid(n, 4, 0.5, 1)
    buf = torch.from_numpy(g).cuda()
    want = _regular(C, L, buf, n, radius, rule, steps, torch)
    st = torch.cuda.Stream()
    smin, smax, bmin, bmax = rule
    torch.cuda.synchronize()
    rc = L.ltl_step_noalloc(ctypes.c_void_p(buf.data_ptr()), n, ctypes.c_void_p(buf.data_ptr()), n, n, radius, smin,
                            smax, bmin, bmax, steps, ctypes.c_void_p(st.cuda_stream))
    assert rc == 0, L.ltl_last_error()
    st.synchronize()
    assert np.array_equal(buf.cpu().numpy(), want)


def test_noalloc_size_limit_is_the_documented_bound():
    """n = 4048 at R = 5 fits the two halo'd grids of the 32 MiB scratch; 4049 does not."""
    import torch
    import cat_cpu_b200 as C
    L = C.lib()
    for n, want in ((4048, 0), (4049, C.ltl.EINVAL)):
        dev = torch.zeros((n, n), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        rc = L.ltl_step_noalloc(ctypes.c_void_p(dev.data_ptr()), n, ctypes.c_void_p(dev.data_ptr()), n, n, 5, 32,
                                56, 34, 45, 1, None)
        torch.cuda.synchronize()
        assert rc == want, (n, L.ltl_last_error())
        del dev


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch
    import cat_cpu_b200 as C
    L = C.lib()
    n = 6000
    dev = torch.zeros((n, n), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    rc = L.ltl_step_noalloc(ctypes.c_void_p(dev.data_ptr()), n, ctypes.c_void_p(dev.data_ptr()), n, n, 5, 32, 56, 34,
                            45, 1, None)
    assert rc == C.ltl.EINVAL
    assert b"scratch" in L.ltl_last_error()

"""Rectangular plain contexts (ltl_create_rect) and the row-strip split on the
GPU: several strips of one grid in one process on one device, exchanged by
device copies (the transport a multi-GPU run replaces with NCCL).  Marked gpu."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tests.stripsutil import step_rect

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rows,cols,r,steps", [(100, 256, 5, 7), (37, 500, 3, 5), (70, 200, 8, 4), (16, 64, 1, 6),
                                               (300, 96, 5, 3)])
def test_rect_context_matches_numpy_torus(rows, cols, r, steps):
    import cat_cpu_b200 as C
    rng = np.random.default_rng(rows + cols)
    rule = O.BOSCO_R5 if r == 5 else O.sweep_rule(r)
    g = (rng.random((rows, cols)) < 0.45).astype(np.uint8)
    s = C.CUDASolver(cols, r, rule, variant=C.VARIANT_PLAIN, rows=rows)
    try:
        assert s.get_info().rows == rows
        s.setState(g)
        s.doSteps(steps)
        want = g
        for _ in range(steps):
            want = step_rect(want, r, rule)
        got = s.getCurrentState()
        assert np.array_equal(got, want), f"{int((got != want).sum())} cells differ"
        # row transfers
        buf = torch.empty((5, cols), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        s.download_rows_device(rows - 5, 5, buf.data_ptr(), cols)
        s.synchronize()
        assert np.array_equal(buf.cpu().numpy(), want[rows - 5:])
    finally:
        s.close()


def test_rect_refuses_other_variants_and_bad_rows():
    import cat_cpu_b200 as C
    with pytest.raises(C.LtlError):
        C.CUDASolver(64, 5, O.BOSCO_R5, rows=3)   # rows < radius
    s = C.CUDASolver(64, 2, O.sweep_rule(2), rows=40)
    try:
        buf = torch.empty((4, 64), dtype=torch.uint8, device="cuda")
        with pytest.raises(C.LtlError):
            s.download_rows_device(38, 4, buf.data_ptr(), 64)
    finally:
        s.close()


@pytest.mark.parametrize("n,r,parts,k,gens", [(512, 5, 3, 4, 11), (300, 8, 2, 3, 7), (256, 1, 4, 5, 12)])
def test_gpu_strips_match_full_grid(n, r, parts, k, gens):
    import cat_cpu_b200 as C
    from cat_cpu_b200 import strips as S
    rule = O.BOSCO_R5 if r == 5 else O.sweep_rule(r)
    g0 = C.start_grid(n, 3, 0.45, 1)
    ls = S.LocalStrips(n, r, parts, k, lambda rows, nn: S.GpuStepper(rows, nn, r, rule), device="cuda")
    try:
        ls.set_state(g0)
        ls.step(gens)
        got = ls.get_state().cpu().numpy()
    finally:
        for s in ls.strips:
            s.st.close()
    want = O.run(g0, r, rule, gens)
    assert np.array_equal(got, want), f"{int((got != want).sum())} cells differ"

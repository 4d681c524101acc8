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
    with pytest.raises(C.LtlError) as e:
        C.CUDASolver(64, 2, O.sweep_rule(2), variant=C.VARIANT_TENSOR, rows=40)
    assert e.value.code == C.ltl.EUNSUPPORTED
    s = C.CUDASolver(64, 2, O.sweep_rule(2), rows=40)
    try:
        buf = torch.empty((4, 64), dtype=torch.uint8, device="cuda")
        with pytest.raises(C.LtlError):
            s.download_rows_device(38, 4, buf.data_ptr(), 64)
    finally:
        s.close()


@pytest.mark.parametrize("variant", ["plain", "packed"])
@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("n,r,parts,k,gens", [(512, 5, 3, 4, 11), (300, 8, 2, 3, 7), (256, 1, 4, 5, 12),
                                              (1000, 3, 3, 2, 9)])
def test_gpu_strips_match_full_grid(n, r, parts, k, gens, overlap, variant):
    """Several strips of one grid on one GPU, plain or bit-packed strips, the
    exchange overlapped (edge tori) or not; ragged and multiple-of-32 widths."""
    import cat_cpu_b200 as C
    from cat_cpu_b200 import strips as S
    rule = O.BOSCO_R5 if r == 5 else O.sweep_rule(r)
    code = {"plain": C.VARIANT_PLAIN, "packed": C.VARIANT_PACKED}[variant]
    g0 = C.start_grid(n, 3, 0.45, 1)
    ls = S.LocalStrips(n, r, parts, k, lambda rows, nn: S.GpuStepper(rows, nn, r, rule, variant=code),
                       device="cuda", overlap=overlap)
    try:
        ls.set_state(g0)
        ls.step(gens)
        got = ls.get_state().cpu().numpy()
    finally:
        ls.close()
    want = O.run(g0, r, rule, gens)
    assert np.array_equal(got, want), f"{int((got != want).sum())} cells differ"


def test_packed_rect_rows_roundtrip_and_step():
    """A rectangular bit-packed torus: row-range transfers touch only their rows,
    and a step matches the oracle's rows x n torus."""
    import cat_cpu_b200 as C
    from tests.stripsutil import step_rect
    rows, n, r, rule = 75, 160, 4, O.sweep_rule(4)
    rng = np.random.default_rng(3)
    g = (rng.random((rows, n)) < 0.45).astype(np.uint8)
    s = C.CUDASolver(n, r, rule, variant=C.VARIANT_PACKED, rows=rows)
    try:
        s.setState(g)
        patch = torch.from_numpy((rng.random((7, n)) < 0.5).astype(np.uint8)).cuda()
        s.upload_rows_device(30, 7, patch.data_ptr(), n)
        g[30:37] = patch.cpu().numpy()
        back = torch.empty((9, n), dtype=torch.uint8, device="cuda")
        s.download_rows_device(29, 9, back.data_ptr(), n)
        torch.cuda.synchronize()
        assert np.array_equal(back.cpu().numpy(), g[29:38])
        assert np.array_equal(s.getCurrentState(), g)
        for _ in range(3):
            s.doStep()
            g = step_rect(g, r, rule)
            assert np.array_equal(s.getCurrentState(), g)
    finally:
        s.close()

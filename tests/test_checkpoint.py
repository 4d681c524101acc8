"""Grid checkpoints (cat_cpu_b200/checkpoint.py): the file format on the host,
and save -> load -> continue on the GPU against an uninterrupted run."""
import os

import numpy as np
import pytest

from cat_cpu_b200 import checkpoint as ck


def test_pack_coding_bit_order():
    n = 70
    g = np.zeros((2, n), dtype=np.uint8)
    g[0, 0] = 1      # word 0 bit 0
    g[0, 63] = 1     # word 0 bit 63
    g[1, 64] = 1     # row 1, word 1 bit 0
    g[1, 69] = 1     # word 1 bit 5
    w = ck.pack_host(g)
    assert w.shape == (2, 2)
    assert int(w[0, 0]) == (1 | (1 << 63)) and int(w[0, 1]) == 0
    assert int(w[1, 0]) == 0 and int(w[1, 1]) == (1 | (1 << 5))
    assert np.array_equal(ck.unpack_host(w, n), g)


@pytest.mark.parametrize("n", [1, 63, 64, 65, 200])
def test_host_roundtrip_and_file(tmp_path, n):
    rng = np.random.default_rng(n)
    g = (rng.random((n, n)) < 0.4).astype(np.uint8)
    p = os.path.join(tmp_path, "g.ckpt")
    ck.write(p, ck.pack_host(g), n, 5, (32, 56, 34, 45), generation=17, meta={"seed": 3})
    head, words = ck.read(p)
    assert head["n"] == n and head["generation"] == 17 and head["rule"] == [32, 56, 34, 45]
    assert head["meta"] == {"seed": 3}
    assert np.array_equal(ck.unpack_host(words, n), g)


def test_corrupt_file_is_rejected(tmp_path):
    g = np.eye(64, dtype=np.uint8)
    p = os.path.join(tmp_path, "g.ckpt")
    ck.write(p, ck.pack_host(g), 64, 1, (2, 3, 3, 3))
    raw = bytearray(open(p, "rb").read())
    raw[-1] ^= 1
    open(p, "wb").write(bytes(raw))
    with pytest.raises(ValueError, match="checksum"):
        ck.read(p)
    open(p, "wb").write(bytes(raw[:-8]))
    with pytest.raises(ValueError, match="truncated"):
        ck.read(p)
    open(p, "wb").write(b"not a checkpoint")
    with pytest.raises(ValueError, match="not a grid checkpoint"):
        ck.read(p)


def test_rectangular_grid_roundtrip(tmp_path):
    rows, n = 37, 130
    rng = np.random.default_rng(5)
    g = (rng.random((rows, n)) < 0.5).astype(np.uint8)
    p = os.path.join(tmp_path, "strip.ckpt")
    ck.write(p, ck.pack_host(g), n, 3, (2, 3, 3, 3), rows=rows)
    head, words = ck.read(p)
    assert (head["n"], head["rows"]) == (n, rows) and words.shape == (rows, 3)
    assert np.array_equal(ck.unpack_host(words, n), g)
    with pytest.raises(ValueError, match="rows x n"):
        ck.write(p, ck.pack_host(g), n, 3, (2, 3, 3, 3))  # rows defaults to n: sizes disagree


def test_header_without_rows_means_square(tmp_path):
    import json
    import struct
    n = 40
    g = np.eye(n, dtype=np.uint8)
    p = os.path.join(tmp_path, "old.ckpt")
    ck.write(p, ck.pack_host(g), n, 2, (1, 2, 3, 4))
    raw = open(p, "rb").read()
    (hl,) = struct.unpack("<I", raw[8:12])
    head = json.loads(raw[12:12 + hl])
    del head["rows"]
    h2 = json.dumps(head, sort_keys=True).encode()
    open(p, "wb").write(raw[:8] + struct.pack("<I", len(h2)) + h2 + raw[12 + hl:])
    head, words = ck.read(p)
    assert head["rows"] == n and np.array_equal(ck.unpack_host(words, n), g)


class _FakeSolver:
    def __init__(self, n, rows, radius, rule):
        self.n, self.rows, self.radius, self.rule = n, rows, radius, rule


@pytest.mark.parametrize("field,fake", [
    ("n", _FakeSolver(65, 64, 5, (32, 56, 34, 45))),
    ("rows", _FakeSolver(64, 80, 5, (32, 56, 34, 45))),
    ("radius", _FakeSolver(64, 64, 4, (32, 56, 34, 45))),
    ("rule", _FakeSolver(64, 64, 5, (32, 57, 34, 45))),
])
def test_load_refuses_incompatible_solver(tmp_path, field, fake):
    """load() checks the header against an existing solver before touching the
    device: a grid restored under another radius or rule would be stepped wrongly."""
    g = np.zeros((64, 64), dtype=np.uint8)
    p = os.path.join(tmp_path, "g.ckpt")
    ck.write(p, ck.pack_host(g), 64, 5, (32, 56, 34, 45))
    with pytest.raises(ValueError, match=field):
        ck.load(p, solver=fake)


@pytest.mark.gpu
def test_rect_solver_save_load(tmp_path):
    import cat_cpu_b200 as C
    rows, n, r, rule = 90, 200, 3, (7, 14, 8, 12)
    g0 = (np.random.default_rng(2).random((rows, n)) < 0.5).astype(np.uint8)
    a = C.CUDASolver(n, r, rule, variant=C.VARIANT_PLAIN, rows=rows)
    p = os.path.join(tmp_path, "strip.ckpt")
    try:
        a.setState(g0)
        a.doSteps(3)
        want = a.getCurrentState()
        ck.save(p, a, generation=3)
    finally:
        a.close()
    head, words = ck.read(p)
    assert head["rows"] == rows and np.array_equal(ck.unpack_host(words, n), want)
    b, head = ck.load(p)
    try:
        assert (b.rows, b.n) == (rows, n)
        assert np.array_equal(b.getCurrentState(), want)
    finally:
        b.close()


@pytest.mark.gpu
def test_save_load_continue_matches_uninterrupted(tmp_path):
    import cat_cpu_b200 as C
    n, r, rule = 1000, 5, (32, 56, 34, 45)
    g0 = C.start_grid(n, 7, 0.5, 1)
    ref = C.CUDASolver(n, r, rule, variant=C.VARIANT_PLAIN)
    try:
        ref.setState(g0)
        ref.doSteps(9)
        want = ref.getCurrentState()
    finally:
        ref.close()
    p = os.path.join(tmp_path, "mid.ckpt")
    a = C.CUDASolver(n, r, rule, variant=C.VARIANT_PACKED)
    try:
        a.setState(g0)
        a.doSteps(4)
        ck.save(p, a, generation=4)
        mid = a.getCurrentState()
    finally:
        a.close()
    head, words = ck.read(p)
    assert head["generation"] == 4 and np.array_equal(ck.unpack_host(words, n), mid)
    b, head = ck.load(p, variant=C.VARIANT_TENSOR)
    try:
        b.doSteps(5)
        assert np.array_equal(b.getCurrentState(), want)
    finally:
        b.close()

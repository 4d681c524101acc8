"""Helpers shared by the golden-vector tests."""
import base64
import hashlib

import numpy as np


def sha(grid):
    return hashlib.sha256(np.ascontiguousarray(grid, dtype=np.uint8).tobytes()).hexdigest()


def grid_from_bits(cp, n):
    bits = np.frombuffer(base64.b64decode(cp["bits_b64"]), dtype=np.uint8)
    return np.unpackbits(bits)[: n * n].reshape(n, n)


def describe_mismatch(got, want):
    d = np.argwhere(got != want)
    if d.size == 0:
        return "no mismatch"
    i, j = d[0]
    return f"{len(d)} cells differ; first at ({i},{j}) got {got[i, j]} want {want[i, j]}"

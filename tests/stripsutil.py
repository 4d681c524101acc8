"""Test helpers for the row-strip split: a numpy stepper for a rows x n torus
(the CPU stand-in for a rectangular GPU context)."""
import numpy as np
import torch


def step_rect(g, radius, rule):
    """One LtL generation of a rows x n torus (centre excluded in k)."""
    smin, smax, bmin, bmax = rule
    R = radius
    p = np.pad(g.astype(np.int64), R, mode="wrap")
    c = p.cumsum(0).cumsum(1)
    c = np.pad(c, ((1, 0), (1, 0)))
    rows, n = g.shape
    w = 2 * R + 1
    B = c[w:w + rows, w:w + n] - c[0:rows, w:w + n] - c[w:w + rows, 0:n] + c[0:rows, 0:n]
    k = B - g
    alive = (k >= smin) & (k <= smax)
    born = (k >= bmin) & (k <= bmax)
    return np.where(g == 1, alive, born).astype(np.uint8)


class NumpyStepper:
    def __init__(self, rows, n, radius, rule):
        self.rows, self.n, self.radius, self.rule = rows, n, radius, rule
        self.g = np.zeros((rows, n), dtype=np.uint8)

    def read_rows(self, row0, nrows, out):
        out.copy_(torch.from_numpy(self.g[row0:row0 + nrows].copy()))

    def write_rows(self, row0, src):
        self.g[row0:row0 + src.shape[0]] = src.cpu().numpy()

    def step(self, gens):
        for _ in range(gens):
            self.g = step_rect(self.g, self.radius, self.rule)

"""The work split of the persistent batch kernel (persist_grid in
cat_cpu_b200/csrc/k_batch.cu), restated in Python and checked on the CPU: for
every grid side and radius the (segment, strip, band) items a CTA's warps walk
cover every output (row, word) of the grid exactly once, every band is at least
one row, and a warp's segments all run the same number of iterations."""
import pytest

WARPS = 8  # kPersistWarps


def plan(n, R):
    nw = (n + 31) // 32
    seg = 32 if nw >= 32 else (1 if nw <= 1 else 1 << (nw - 1).bit_length())
    ns = 32 // seg
    strips = (nw + seg - 1) // seg
    want = max(1, WARPS * ns // strips)
    band_rows = min(n, max((n + want - 1) // want, 4 * R + 2))
    bands = (n + band_rows - 1) // band_rows
    return nw, seg, ns, strips, band_rows, bands


@pytest.mark.parametrize("R", [1, 2, 5, 8, 12, 16])
def test_items_cover_each_output_once(R):
    for n in list(range(max(R, 1), 140)) + [200, 255, 256, 257, 511, 512, 700, 1023, 1024, 1025, 1500, 2048]:
        if n < R:
            continue
        nw, seg, ns, strips, band_rows, bands = plan(n, R)
        assert seg & (seg - 1) == 0 and seg >= min(nw, 32)
        items = strips * bands
        seen = {}
        for wid in range(WARPS):
            base = wid * ns
            while base < items:  # the warp-uniform loop of the kernel
                for lane in range(32):
                    wl, sidx = lane & (seg - 1), lane // seg
                    item = base + sidx
                    if item >= items:
                        continue
                    strip, band = item % strips, item // strips
                    r0, r1 = band * band_rows, min(band * band_rows + band_rows, n)
                    assert r1 > r0 and r1 - r0 <= band_rows  # the uniform loop covers the band
                    w = strip * seg + wl
                    if w >= nw:
                        continue
                    for r in range(r0, r1):
                        seen[(r, w)] = seen.get((r, w), 0) + 1
                base += WARPS * ns
        assert len(seen) == n * nw and set(seen.values()) == {1}, (n, R)

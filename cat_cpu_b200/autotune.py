"""Shape autotuner: sweeps the kernels' work-item shapes on the device and writes
the winners to cat_cpu_b200/tuning/ltl_tuning.txt, which libltl_b200 reads at
ltl_create / ltl_batch_create.

    python -m cat_cpu_b200.autotune [--quick] [--out DIR]

This is the analogue of the reference project's region-count landscape search
(NREGIONS_H/V over 1..30 x 1..30, scripts/exploreRegionSizesLandscape.py:21-39,
scripts/extractBestRegionSize.py): here the swept shapes are
  plain / packed   band_rows: rows a warp walks down per work item (the vertical
                   window is restarted once per band, so longer bands re-read less
                   but leave fewer items to balance over 148 SMs);
  plain            depth: generations per pass of the temporally blocked kernel
                   (1, 2 or 3), swept jointly with band_rows;
  batch            persistent: one launch per call that runs every generation of
                   every grid (1), or per-generation launches (0), and for the
                   latter stream_band_rows of the streamed per-step kernels and
                   resident_max_bytes: which grids are kept in shared memory for
                   a whole multi-step launch and which are streamed each step.
The full landscape (every candidate's time) is written next to the table.
"""
import argparse
import concurrent.futures as cf
import os
import time

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))


def _time_steps(torch, solver, stream, steps, reps=3):
    best = None
    for _ in range(reps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.doSteps(steps)
        b.record(stream)
        stream.synchronize()
        ms = a.elapsed_time(b) / steps
        best = ms if best is None else min(best, ms)
    return best


def size_class(n):
    """Grid-side class a tuned value applies to: [1, 8191], [8192, 24575], [24576, 2^30]."""
    if n < 8192:
        return 1, 8191
    if n < 24576:
        return 8192, 24575
    return 24576, 1 << 30


def tune_single(torch, C, variant, n, radius, rule, candidates, steps, depths=(1,)):
    """Times every (depth, band_rows) pair; `steps` should be a multiple of every depth."""
    vcode = {"plain": C.VARIANT_PLAIN, "packed": C.VARIANT_PACKED}[variant]
    g = C.generate_state(n, 12345, 0.5, 1)
    stream = torch.cuda.Stream()
    s = C.CUDASolver(n, radius, rule, variant=vcode)
    s.set_stream(stream.cuda_stream)
    rows = []
    try:
        for d in depths:
            if variant == "plain":
                s.set_param("depth", d)
            for br in candidates:
                s.set_param("band_rows", br)
                s.setState(g)
                s.doSteps(12)
                ms = _time_steps(torch, s, stream, steps)
                rows.append(((d, br), ms))
    finally:
        s.close()
    best = min(rows, key=lambda x: x[1])
    return best, rows


def tune_batch(torch, C, band_candidates, resident_candidates, steps):
    from cat_cpu_b200.workloads import batch_config
    cfg = batch_config()
    with cf.ThreadPoolExecutor(os.cpu_count() or 8) as ex:
        grids = list(ex.map(lambda c: C.generate_state(c[0], c[4], c[3], 1), cfg))
    flat = np.concatenate([g.ravel() for g in grids])
    stream = torch.cuda.Stream()
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg])
    rows = []
    try:
        b.set_stream(stream.cuda_stream)
        # (persistent, stream_band_rows, resident_max_bytes); the last two only
        # matter for per-generation launches
        cands = [(1, band_candidates[0], resident_candidates[0])] + \
            [(0, br, rm) for rm in resident_candidates for br in band_candidates]
        for pers, br, rm in cands:
            b.set_param("persistent", pers)
            b.set_param("resident_max_bytes", rm)
            b.set_param("stream_band_rows", br)
            b.upload_all(flat)
            b.step(steps)          # builds and warms the graph
            b.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            b.step(steps)
            e.record(stream)
            stream.synchronize()
            rows.append(((pers, br, rm), a.elapsed_time(e)))
    finally:
        b.close()
    best = min(rows, key=lambda x: x[1])
    return best, rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick", action="store_true", help="fewer candidates")
    ap.add_argument("--out", default=os.path.join(PKG, "tuning"))
    args = ap.parse_args()
    import torch
    import cat_cpu_b200 as C
    from cat_cpu_b200.workloads import scaled_rule, BOSCO_R5

    os.makedirs(args.out, exist_ok=True)
    dev = torch.cuda.get_device_name(0)
    table = [f"# autotuned on {dev} by cat_cpu_b200/autotune.py, {time.strftime('%Y-%m-%d %H:%M:%S')}"]
    land = [f"# landscape ({dev}): candidate -> ms per step (single grids) or per 256-step batch run"]
    plain_c = [64, 128, 256, 512] if args.quick else [64, 96, 128, 192, 256, 384, 512]
    packed_c = [0, 32, 64, 128] if args.quick else [0, 32, 48, 64, 96, 128, 192, 256]  # 0: built-in choice
    jobs = [("plain", 16384, 5, BOSCO_R5, plain_c), ("plain", 4096, 5, BOSCO_R5, plain_c),
            ("packed", 16384, 5, BOSCO_R5, packed_c), ("packed", 32768, 5, BOSCO_R5, packed_c)]
    for r in (1, 2, 4, 8, 16, 32):
        if not args.quick or r in (1, 8):
            jobs.append(("packed", 32768, r, scaled_rule(r), packed_c))
    for variant, n, r, rule, cands in jobs:
        depths = [d for d in (1, 2, 3) if d == 1 or (r <= 5 and d * r <= 16)] if variant == "plain" else [1]
        ((d, br), ms), rows = tune_single(torch, C, variant, n, r, rule, cands, 24, depths)
        lo, hi = size_class(n)
        extra = f" depth={d}" if variant == "plain" else ""
        table.append(f"variant={variant} radius={r} nmin={lo} nmax={hi} band_rows={br}{extra}")
        land.append(f"{variant} n={n} R={r} (depth, band_rows): " + ", ".join(f"{c}:{t:.4f}" for c, t in rows) +
                    f"  -> {(d, br)}")
        print(land[-1], flush=True)
    band_c = [32, 64, 128] if args.quick else [32, 48, 64, 96, 128]
    res_c = [0, 225280] if args.quick else [0, 65536, 131072, 225280]
    ((pers, br, rm), ms), rows = tune_batch(torch, C, band_c, res_c, 256)
    table.append(f"variant=batch radius=* persistent={pers} stream_band_rows={br} resident_max_bytes={rm}")
    land.append("batch (persistent, stream_band_rows, resident_max_bytes): " +
                ", ".join(f"{c}:{t:.2f}" for c, t in rows) + f"  -> {(pers, br, rm)}")
    print(land[-1], flush=True)
    with open(os.path.join(args.out, "ltl_tuning.txt"), "w") as f:
        f.write("\n".join(table) + "\n")
    with open(os.path.join(args.out, "landscape.txt"), "w") as f:
        f.write("\n".join(land) + "\n")
    print("wrote", os.path.join(args.out, "ltl_tuning.txt"))


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""LtL stepping throughput on B200: GCUPS of every exact GPU variant.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one generation of the whole grid): a 16384 x 16384
torus, R = 5, Bosco's rule (S33-57 / B34-45 with the centre counted, i.e. the
reference's S32-56 / B34-45), start grid = the reference generator's grid for
--seed 1 -d 0.5 (host-generated, uploaded once).  Each variant (plain CUDA-core
SWAR stencil, bit-packed, tcgen05 tensor core when built) is first checked
bit-exact against the reference's own step-100 grid (tests/golden/golden.json),
then timed: K steps, each preceded by an untimed 256 MiB L2 flush, each bracketed
by CUDA events on the solver's stream.  `value` is the fastest variant's
whole-job GCUPS (cells * steps / max-over-ranks time; every rank runs its own
replica grid, so scaling is weak).

With --impl reference the reference's own CPU solver (built from its sources
into oracle/_ref/, AMX16 when the host has AMX-INT8, else AVX2) is timed on the
host cores for the same workload.
"""
import argparse
import glob
import hashlib
import json
import os
import shutil
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N = 16384
RADIUS = 5
RULE = (32, 56, 34, 45)
SEED = 1
DENSITY = 0.5
WORKLOAD = ("16384x16384 torus, R=5 Moore, Bosco S33-57/B34-45 (centre counted; reference S32-56/B34-45), "
            "start grid = reference generator --seed 1 -d 0.5 --threads 1")
METRIC = "GCUPS (cell updates / s / 1e9) of generations of a 16384^2 LtL torus, R=5, bit-exact"
# algorithmic HBM bytes per cell-update: one read and one write of the state
# (uint8 cells for plain; bit-packed cells for packed and tensor, whose grids
# live in the packed frame between generations)
BYTES_PER_UPDATE = {"plain": 2.0, "tensor": 0.25, "packed": 0.25}
DTYPE = {"plain": "u8", "tensor": "b1 state, u8 x u8 -> s32 operands (tcgen05 kind::i8)",
         "packed": "b1 (32 cells per u32)"}
REF_RULE_TAG = "R5_S32-56_B34-45"
# What bounds each step kernel, from the committed ncu captures of the 16384^2 R=5
# workload (the bit-packed kernels are bound by logic operations on the ALU pipe,
# the tensor kernel by hand-offs between its warp roles, not by HBM).
LIMITER = {
    "plain": {"pipe": "alu", "ncu_pct_of_peak": 72.0, "source": "profiles/k_plain_swar8_tb_n16384_r5.md"},
    "packed": {"pipe": "alu", "ncu_pct_of_peak": 70.7, "source": "profiles/k_packed_step_n16384_r5.md"},
    "tensor": {"pipe": "tensor", "ncu_pct_of_peak": 32.8, "issue_active_pct": 59.9,
               "source": "profiles/k_tensor_step_n16384_r5.md"},
}


def env_int(name, default):
    try:
        return int(os.environ.get(name, default))
    except ValueError:
        return default


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_table():
    """Per-launch DRAM bytes from the committed ncu summary, keyed by variant."""
    out = {}
    p = os.path.join(ROOT, "profiles", "traffic_n16384_r5.txt")
    if os.path.exists(p):
        for line in open(p):
            line = line.strip()
            if not line or line.startswith("#"):
                continue
            kv = dict(x.split("=", 1) for x in line.split())
            if "variant" in kv and "dram_bytes_per_launch" in kv:
                out[kv["variant"]] = float(kv["dram_bytes_per_launch"])
    return out


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 20 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"ltl_clocks_{os.getpid()}.csv")

    def start(self):
        if shutil.which("nvidia-smi") is None:
            return
        self.fh = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits", "-lms", "20"], stdout=self.fh,
                                     stderr=subprocess.DEVNULL)
        # the timed region starts only once the sampler is producing samples
        t0 = time.time()
        while time.time() - t0 < 5.0:
            self.fh.flush()
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def dist_setup(args):
    world = env_int("WORLD_SIZE", 1)
    rank = env_int("RANK", 0)
    local = env_int("LOCAL_RANK", 0)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch
        import torch.distributed as dist
        dist.barrier()
        torch.cuda.synchronize()


def max_over_ranks(v, world):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def golden_step100():
    p = os.path.join(ROOT, "tests", "golden", "golden.json")
    for c in json.load(open(p))["cases"]:
        if c["name"] == "config2_bosco_r5_n16384_amx16":
            for cp in c["checkpoints"]:
                if cp["step"] == 100:
                    return cp["sha256"]
    return None


def run_variant(C, torch, name, start, args, flush, sampler=None):
    vcode = {"plain": C.VARIANT_PLAIN, "tensor": C.VARIANT_TENSOR, "packed": C.VARIANT_PACKED}[name]
    stream = torch.cuda.Stream()
    s = C.CUDASolver(N, RADIUS, RULE, variant=vcode, device=torch.cuda.current_device())
    try:
        s.set_stream(stream.cuda_stream)
        depth = s.info.temporal_depth
        # bit-exactness against the reference's own grid after 100 generations
        s.setState(start)
        s.doSteps(100)
        got = s.getCurrentState()
        want = golden_step100()
        bit_exact = want is not None and hashlib.sha256(got.tobytes()).hexdigest() == want
        # warm-up from the start grid
        s.setState(start)
        s.doSteps(args.warmup * depth)
        s.synchronize()
        passes = max(1, args.steps // depth)
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(passes)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(passes)]
        if sampler:
            # nvidia-smi samples every 20 ms, longer than the timed passes below
            # (K passes of ~0.1 ms each): the sampler also covers a sustained,
            # untimed run of the same passes (L2 flush included) right before them
            sampler.start()
            t_end = time.time() + 0.6
            with torch.cuda.stream(stream):
                while time.time() < t_end:
                    for _ in range(20):
                        flush.zero_()
                        s.doSteps(depth)
                    stream.synchronize()
        s.set_timing(True)
        barrier(args.world)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for p in range(passes):
                flush.zero_()
                starts[p].record(stream)
                s.doSteps(depth)
                ends[p].record(stream)
        stream.synchronize()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier(args.world)
        ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
        kernel_ms, kernel_launches, all_launches = s.get_timing()
        s.set_timing(False)
        gens = passes * depth
        return dict(ms_total=ms, generations=gens, kernel_ms=kernel_ms, kernel_launches=kernel_launches,
                    all_launches=all_launches, depth=depth, bit_exact_step100=bool(bit_exact), clocks=clocks,
                    operand_bits=s.info.operand_bits)
    finally:
        s.close()


def e2e_run(C, torch, name, start, steps, packed_io=None):
    """Through the public API with host buffers: upload the start grid from pinned
    memory, advance `steps` generations, download the grid -- timed together.
    The bit-packed variants move the grid in the PACK coding (ltl_upload_packed /
    ltl_download_packed: 1 bit per cell), the plain one as uint8 cells
    (ltl_upload / ltl_download); packed_io=False forces uint8 for any variant.
    The downloaded grid is checked against the context's own uint8 download."""
    import ctypes
    import numpy as np
    vcode = {"plain": C.VARIANT_PLAIN, "tensor": C.VARIANT_TENSOR, "packed": C.VARIANT_PACKED}[name]
    if packed_io is None:
        packed_io = name in ("packed", "tensor")
    stream = torch.cuda.Stream()
    if packed_io:
        host = C.pack_grid(start)
        pinned_in = torch.from_numpy(host.view(np.int64)).pin_memory()
        pitch = host.shape[1] * 8
    else:
        pinned_in = torch.from_numpy(start).pin_memory()
        pitch = N
    pinned_out = torch.empty_like(pinned_in).pin_memory()
    nbytes = pinned_in.numel() * pinned_in.element_size()
    L = C.lib()
    up, down = (L.ltl_upload_packed, L.ltl_download_packed) if packed_io else (L.ltl_upload, L.ltl_download)
    s = C.CUDASolver(N, RADIUS, RULE, variant=vcode, device=torch.cuda.current_device())
    try:
        s.set_stream(stream.cuda_stream)
        depth = s.info.temporal_depth
        steps = max(depth, steps - steps % depth)
        times = []
        for it in range(3):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            C.ltl.check(up(s._h, ctypes.c_void_p(pinned_in.data_ptr()), pitch))
            s.doSteps(steps)
            C.ltl.check(down(s._h, ctypes.c_void_p(pinned_out.data_ptr()), pitch))
            b.record(stream)
            stream.synchronize()
            if it > 0:
                times.append(a.elapsed_time(b))
        ms = sum(times) / len(times)
        got = pinned_out.numpy()
        got = C.unpack_grid(got.view(np.uint64), N) if packed_io else got
        same = bool(np.array_equal(got, s.getCurrentState()))
        return dict(ms=ms, steps=steps, gcups=N * N * steps / (ms * 1e-3) / 1e9, h2d=nbytes, d2h=nbytes,
                    io="PACK-coded uint64 rows (1 bit per cell)" if packed_io else "uint8 cells",
                    download_matches=same)
    finally:
        s.close()


SWEEP_POINTS = [(1, 2, 0.5), (2, 2, 0.5), (4, 2, 0.5), (8, 2, 0.5), (16, 2, 0.5), (32, 2, 0.5),
                (64, 3, 0.3), (128, 3, 0.3)]


def radius_sweep(C, torch, args, passes_per_variant, emit=None):
    """The radius-sweep workloads: 32768^2, seed 2, d = 0.5, R in {1,2,4,8,16,32},
    scaled interval rule, and R in {64,128} at d = 0.3 (seed 3).  One record per
    radius with every variant's GCUPS (passes timed with CUDA events on the
    launching stream, L2 flushed before each pass), the step kernel's own GCUPS
    (halo launches excluded) and its HBM roofline at the variant's algorithmic
    bytes per cell-update.  Exactness at these sizes is covered by
    tests/test_gpu_fullsize.py.  `emit(record)` is called per radius."""
    from cat_cpu_b200.workloads import scaled_rule
    n = 32768
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    vcodes = {"plain": C.VARIANT_PLAIN, "packed": C.VARIANT_PACKED, "tensor": C.VARIANT_TENSOR}
    peak, peak_kind = measured_peaks()
    starts = {}
    records = []
    for radius, seed, dens in SWEEP_POINTS:
        rule = scaled_rule(radius)
        if (seed, dens) not in starts:
            starts.clear()
            starts[(seed, dens)] = C.start_grid(n, seed, dens, 1)
        start = starts[(seed, dens)]
        out = {"workload": f"{n}x{n} torus, R={radius}, scaled interval rule, seed {seed}, d={dens}",
               "radius": radius, "unit": "GCUPS", "peak_kind": f"{peak_kind} hbm_gbs", "variants": {}}
        for name in [v for v in args.variants.split(",") if v]:
            try:
                s = C.CUDASolver(n, radius, rule, variant=vcodes[name])
            except C.LtlError as e:
                out["variants"][name] = {"unsupported": str(e)}
                continue
            try:
                stream = torch.cuda.Stream()
                s.set_stream(stream.cuda_stream)
                depth = s.info.temporal_depth
                s.setState(start)
                s.doSteps(3 * depth)
                s.synchronize()
                passes = max(1, passes_per_variant // depth)
                ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                      for _ in range(passes)]
                s.set_timing(True)
                with torch.cuda.stream(stream):
                    for a, b in ev:
                        flush.zero_()
                        a.record(stream)
                        s.doSteps(depth)
                        b.record(stream)
                stream.synchronize()
                ms = sum(a.elapsed_time(b) for a, b in ev)
                kernel_ms, kernel_launches, _ = s.get_timing()
                s.set_timing(False)
                gens = passes * depth
                # roofline of the step kernel alone (halo launches excluded):
                # algorithmic bytes per cell-update x cell-updates / kernel time
                achieved = n * n * gens * BYTES_PER_UPDATE[name] / (kernel_ms * 1e-3) / 1e9
                out["variants"][name] = {"gcups": round(n * n * gens / (ms * 1e-3) / 1e9, 2),
                                         "kernel_gcups": round(n * n * gens / (kernel_ms * 1e-3) / 1e9, 2),
                                         "ms_per_generation": round(ms / gens, 4), "temporal_depth": depth,
                                         "generations": gens, "population": s.population(),
                                         "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                                                      "unit": "GB/s", "frac": round(achieved / peak, 4),
                                                      "bytes_per_update": BYTES_PER_UPDATE[name]}}
                if name == "tensor":
                    # product-2 operand chosen from the exactness bound of the row sums
                    out["variants"][name]["operand"] = "f16" if s.info.operand_bits == 16 else "u8"
            finally:
                s.close()
        v = out["variants"]
        if "gcups" in v.get("tensor", {}) and "gcups" in v.get("plain", {}):
            out["tensor_vs_plain"] = round(v["tensor"]["gcups"] / v["plain"]["gcups"], 3)
        records.append(out)
        if emit:
            emit(out)
    return records


def strips_run(C, torch, args, world, rank, local):
    """The 16384^2 R=5 grid split into `world` row strips (one per rank,
    bit-packed variant), halos exchanged every args.strips generations behind the
    strips' own steps (NCCL between ranks; with one rank the strip exchanges with
    itself).  Strong scaling: the total
    work is fixed.  Times `steps` generations after `warmup` with CUDA events on
    the rank's stream, max over ranks; checks the gathered grid at generation
    100 against the reference's grid."""
    from cat_cpu_b200 import strips as S
    k = args.strips
    dev = torch.device("cuda", local)
    make = lambda rows, n: S.GpuStepper(rows, n, RADIUS, RULE, device=local,  # noqa: E731
                                        variant=C.VARIANT_PACKED)
    if world > 1:
        st = S.DistStrips(N, RADIUS, k, make, dev)
    else:
        st = S.LocalStrips(N, RADIUS, 1, k, make, device=dev)
    start = C.start_grid(N, SEED, DENSITY, 1)
    try:
        st.set_state(start)
        st.step(100)
        got = st.get_state().cpu().numpy()
        bit_exact = hashlib.sha256(got.tobytes()).hexdigest() == golden_step100()
        st.set_state(start)
        st.step(max(args.warmup, 3) * k)
        torch.cuda.synchronize()
        barrier(world)
        stream = st.stream  # the strips' own stream: every kernel and copy of theirs runs on it
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        gens = max(k, args.steps - args.steps % k)
        a.record(stream)
        st.step(gens)
        b.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(a.elapsed_time(b), world)
    finally:
        st.close()
    return dict(ms=ms, generations=gens, bit_exact=bit_exact, halo_rows=st.h)


def batched_run(C, torch, steps, warmup_steps):
    """The batched workload (4096 grids, sides log-uniform in [64, 2048], R in 1..8,
    scaled interval rule, 256 steps per ltl_batch_step call)."""
    import concurrent.futures as cf
    import numpy as np
    from cat_cpu_b200.workloads import batch_config
    cfg = batch_config()
    with cf.ThreadPoolExecutor(os.cpu_count() or 8) as ex:
        grids = list(ex.map(lambda c: C.generate_state(c[0], c[4], c[3], 1), cfg))
    flat = np.concatenate([g.ravel() for g in grids])
    stream = torch.cuda.Stream()
    b = C.Batch([(n, r, rule) for (n, r, rule, d, s) in cfg])
    try:
        b.set_stream(stream.cuda_stream)
        b.upload_all(flat)
        cells, dev_bytes, resident = b.info()
        b.step(warmup_steps)
        b.synchronize()
        a = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        b.step(steps)
        e.record(stream)
        stream.synchronize()
        ms = a.elapsed_time(e)
        return dict(ms=ms, cells=cells, grids=len(cfg), steps=steps, resident_grids=resident)
    finally:
        b.close()


# ---------------------------------------------------------------------------
# Reference CPU solver (built from the reference sources into oracle/_ref/)
# ---------------------------------------------------------------------------
def cpu_flags():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("flags"):
                return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def reference_binary():
    flags = cpu_flags()
    base = os.path.join(ROOT, "oracle", "_ref")
    native = os.path.join(base, REF_RULE_TAG + "_native", "prog")
    portable = os.path.join(base, REF_RULE_TAG + "_portable", "prog")
    need_native = {"avx512f", "avx512bw", "avx512vl", "amx_int8", "amx_tile", "avx512_fp16", "avx512_vnni"}
    if os.path.exists(native) and need_native <= flags:
        return native, "native"
    if os.path.exists(portable) and "avx2" in flags:
        return portable, "portable"
    return None, None


def run_reference(steps, threads, solver):
    exe, build = reference_binary()
    if exe is None:
        return None
    t0 = time.time()
    r = subprocess.run([exe, str(N), str(solver), str(steps), "-d", str(DENSITY), "--seed", str(SEED), "--threads",
                        str(threads)], capture_output=True, text=True, cwd="/tmp", timeout=1800)
    wall = time.time() - t0
    if r.returncode != 0:
        return None
    ms = float(r.stdout.strip().splitlines()[0])
    return dict(ms_per_step=ms, gcups=N * N / (ms * 1e-3) / 1e9, wall_s=wall, build=build, exe=exe)


def reference_solver_choice():
    flags = cpu_flags()
    if {"amx_int8", "amx_tile"} <= flags:
        return 2, "AMX16 (solver 2)"
    return 3, "AVX2 (solver 3)"


def cpu_baseline_sample(threads):
    """~10-30 s of the reference's best CPU solver on this workload."""
    solver, label = reference_solver_choice()
    probe = run_reference(1, threads, solver)
    if probe is None:
        return None
    steps = int(max(1, min(50, 20000.0 / max(probe["ms_per_step"], 1e-3))))
    res = run_reference(steps, threads, solver)
    if res is None:
        return None
    return {"value": round(res["gcups"], 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
            "sample": f"reference {label}, {res['build']} build, {N}x{N} R=5 Bosco, {steps} steps after a "
                      f"1-step probe, its own ms/step ({res['ms_per_step']:.1f} ms)"}


def main_reference(args):
    world, rank, _ = env_int("WORLD_SIZE", 1), env_int("RANK", 0), env_int("LOCAL_RANK", 0)
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    solver, label = reference_solver_choice()
    exe, build = reference_binary()
    if exe is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference binaries not built for this host "
                          "(oracle/_ref missing or CPU lacks AVX2)"}))
        return
    # warm-up sample (page-in, caches), then the timed sample
    run_reference(max(1, min(args.warmup, 2)), threads, solver)
    probe = run_reference(1, threads, solver)
    budget_ms = 150000.0
    steps = int(max(1, min(args.steps, budget_ms / max(probe["ms_per_step"], 1e-3))))
    res = run_reference(steps, threads, solver)
    gcups = res["gcups"]
    line = {
        "impl": "reference", "metric": METRIC, "value": round(gcups, 4), "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": steps, "warmup": args.warmup, "ms_per_step": round(res["ms_per_step"], 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic: reference generator start grid", "config": {"workload": WORKLOAD, "solver": label},
        "cpu_baseline": {"value": round(gcups, 4), "unit": "GCUPS", "cores": threads, "kind": "reference",
                         "sample": f"reference {label} ({build} build), {steps} steps of {N}x{N}, "
                                   f"{threads} OpenMP threads, its own ms/step"},
        "e2e": {"value": round(gcups, 4), "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variants", default="plain,packed,tensor")
    ap.add_argument("--sweep", action="store_true",
                    help="radius sweep at 32768^2 (one JSON line per radius) instead of the headline run")
    ap.add_argument("--sweep-steps", type=int, default=100)
    ap.add_argument("--strips", type=int, default=0, metavar="K",
                    help="one 16384^2 grid split into row strips across the ranks (strong scaling), "
                         "halo exchange every K generations, instead of the per-rank replicas")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sweep", action="store_true",
                    help="skip the short radius sweep (32768^2, R = 1..128) that rank 0 appends to the line")
    ap.add_argument("--e2e-steps", type=int, default=None)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        main_reference(args)
        return

    world, rank, local = dist_setup(args)
    args.world = world
    import torch
    torch.cuda.set_device(local)
    import cat_cpu_b200 as C

    if args.sweep:
        radius_sweep(C, torch, args, min(args.sweep_steps, 200), emit=lambda r: print(json.dumps(r), flush=True))
        return
    if args.strips > 0:
        r = strips_run(C, torch, args, world, rank, local)
        if rank == 0:
            print(json.dumps({
                "metric": METRIC, "value": round(N * N * r["generations"] / (r["ms"] * 1e-3) / 1e9, 3),
                "unit": "GCUPS", "n_gpus": world, "steps": r["generations"], "warmup": args.warmup,
                "ms_per_step": round(r["ms"] / r["generations"], 5), "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": DTYPE["packed"],
                "data": "synthetic: reference generator start grid (seed 1)",
                "config": {"workload": WORKLOAD, "variant": "packed, row strips", "n": N, "radius": RADIUS,
                           "parallelism": f"row strips x{world}, {r['halo_rows']}-row halo exchange every "
                                          f"{args.strips} generations, overlapped with the strips' steps",
                           "l2": "not flushed (continuous run)"},
                "bit_exact_step100": r["bit_exact"]}))
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    start = C.start_grid(N, SEED, DENSITY, 1)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    results = {}
    sampler = ClockSampler(local)
    for name in [v for v in args.variants.split(",") if v]:
        try:
            results[name] = run_variant(C, torch, name, start, args, flush, sampler if rank == 0 else None)
        except C.LtlError as e:
            if e.code == C.ltl.EUNSUPPORTED:
                results[name] = {"unsupported": str(e)}
                continue
            raise
    peak, peak_kind = measured_peaks()
    traffic = traffic_table()
    variants = {}
    best = None
    for name, r in results.items():
        if "unsupported" in r:
            variants[name] = r
            continue
        t_max = max_over_ranks(r["ms_total"], world)
        gcups = world * N * N * r["generations"] / (t_max * 1e-3) / 1e9
        kernel_ms_launch = r["kernel_ms"] / max(r["kernel_launches"], 1)
        # algorithmic bytes per launch = bytes per cell-update x the cell-updates
        # one launch performs (a temporally blocked pass does `depth` of them per
        # cell, so its achieved figure can exceed the HBM peak; its measured DRAM
        # traffic per launch stays near one read and one write of the grid)
        alg = N * N * BYTES_PER_UPDATE[name] * r["depth"]
        achieved = alg / (kernel_ms_launch * 1e-3) / 1e9
        variants[name] = {
            "gcups": round(gcups, 3), "ms_per_step": round(t_max / r["generations"], 5),
            "kernel_ms_per_launch": round(kernel_ms_launch, 5), "temporal_depth": r["depth"],
            "bit_exact_step100": r["bit_exact_step100"], "dtype": DTYPE[name],
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic.get(name),
                         "traffic_source": "profiles/traffic_n16384_r5.txt: dram bytes of one ncu capture of "
                                           "the step kernel (cache control on, the run's L2 flush not applied)"},
            "limiter": LIMITER[name],
            "gpu_launches": r["all_launches"],
        }
        if r["bit_exact_step100"] and (best is None or gcups > variants[best]["gcups"]):
            best = name
    if best is None:
        raise SystemExit("no variant was bit-exact against the reference grid")
    head = variants[best]
    line = {
        "metric": METRIC,
        "value": head["gcups"], "unit": "GCUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": head["dtype"], "data": "synthetic: reference generator start grid (seed 1, d=0.5), one replica "
                                        "per rank",
        "config": {"workload": WORKLOAD, "variant": best, "n": N, "radius": RADIUS, "rule_centre_excluded": RULE,
                   "l2": "flushed before every timed step (256 MiB device write, untimed)",
                   "parallelism": f"replicas x{world}"},
        "variants": variants,
        "roofline": dict(head["roofline"], peak_kind=f"{peak_kind} hbm_gbs"),
        "gpu_launches": head["gpu_launches"],
    }
    if "plain" in variants and "gcups" in variants.get("tensor", {}):
        line["tensor_vs_plain"] = round(variants["tensor"]["gcups"] / variants["plain"]["gcups"], 3)
    if rank == 0 and results[best].get("clocks"):
        line["clocks"] = results[best]["clocks"]
    # batched workload (grids*steps/s), one replica per rank
    br = batched_run(C, torch, 256, 256)
    b_ms = max_over_ranks(br["ms"], world)
    b_gcups = world * br["cells"] * br["steps"] / (b_ms * 1e-3) / 1e9
    line["batched"] = {
        "workload": "4096 grids, sides log-uniform [64,2048], R uniform 1..8, scaled interval rule, density "
                    "U[0.2,0.6] (mt19937_64 seed 4), 256 steps per ltl_batch_step call, bit-packed",
        "grid_steps_per_s": round(world * br["grids"] * br["steps"] / (b_ms * 1e-3), 1),
        "gcups": round(b_gcups, 2), "ms": round(b_ms, 3), "cells": br["cells"],
        "mode": "persistent: one launch per rule class per ltl_batch_step call runs all 256 generations, "
                "each CTA advancing whole grids (largest first) with the grid held in L1/L2",
        "grids_all_steps_in_one_launch": br["resident_grids"],
        "roofline": {"bound": "hbm", "bytes_per_update": 0.25, "achieved": round(b_gcups * 0.25, 1),
                     "peak": peak, "unit": "GB/s", "frac": round(b_gcups * 0.25 / peak, 4),
                     "frac_u8_equivalent": round(b_gcups * 2.0 / peak, 4)},
    }
    # end to end through the public API with host buffers
    e2 = e2e_run(C, torch, best, start, args.e2e_steps or args.steps)
    e2_ms = max_over_ranks(e2["ms"], world)
    line["e2e"] = {"value": round(world * N * N * e2["steps"] / (e2_ms * 1e-3) / 1e9, 3), "unit": "GCUPS",
                   "h2d_bytes_per_step": int(e2["h2d"] / e2["steps"]), "d2h_bytes_per_step": int(e2["d2h"] /
                                                                                                e2["steps"]),
                   "io": e2["io"], "download_matches": e2["download_matches"],
                   "note": f"upload start grid from pinned host memory + {e2['steps']} steps + download, "
                           f"{best} variant"}
    if best in ("packed", "tensor"):
        # the same run with the grid moved as uint8 cells
        e3 = e2e_run(C, torch, best, start, args.e2e_steps or args.steps, packed_io=False)
        e3_ms = max_over_ranks(e3["ms"], world)
        line["e2e"]["uint8_io"] = {"value": round(world * N * N * e3["steps"] / (e3_ms * 1e-3) / 1e9, 3),
                                   "h2d_bytes_per_step": int(e3["h2d"] / e3["steps"]),
                                   "d2h_bytes_per_step": int(e3["d2h"] / e3["steps"])}
    if rank == 0 and not args.no_sweep:
        # the radius-sweep workloads (32768^2, R in {1,2,4,8,16,32} and {64,128}) at
        # 4 timed generations per variant and radius; `bench.py --sweep` runs more
        recs = radius_sweep(C, torch, args, 4)
        line["radius_sweep"] = {
            "workload": "32768x32768 torus, scaled interval rule; seed 2 d=0.5 for R<=32, seed 3 d=0.3 for R=64,128; "
                        "4 generations per variant, L2 flushed before each, CUDA events",
            "unit": "GCUPS",
            "by_radius": {str(r["radius"]): dict(
                {v: ({"gcups": d["gcups"], "kernel_gcups": d["kernel_gcups"], "hbm_frac": d["roofline"]["frac"],
                      **({"operand": d["operand"]} if "operand" in d else {})} if "gcups" in d else
                     {"unsupported": d["unsupported"]})
                 for v, d in r["variants"].items()},
                **({"tensor_vs_plain": r["tensor_vs_plain"]} if "tensor_vs_plain" in r else {}))
                for r in recs}}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_sample(os.cpu_count() or 1)
        if cb is not None:
            line["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

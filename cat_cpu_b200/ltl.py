"""Python host mirror of the reference's solver interface over libltl_b200's C ABI.

The reference (kezada94/CAT_cpu) drives its solvers through
  CASolverFactory::createSolver(code, deviceId, n, halo, nThreads)   src/CellularAutomata/CASolverFactory.cpp:6
  CASolver::resetState(seed, density) / doStep() / doSteps(k) /
  getCurrentState() / printCurrentState()                           src/CellularAutomata/Solvers/CASolver.h:7-28
  CPUBenchmark::run (srand(seed); resetState(rand() % 1000000, d))  src/CPUBenchmark.cpp:21-32
  CADataDomainComparator::compareCurrentStates()                    src/CellularAutomata/CADataDomainComparator.tpp:8-27
This module keeps those names and argument meanings for the GPU solvers.  All
work goes through ctypes calls into cat_cpu_b200/libltl_b200.so; there is no
CPU path: if the library or a CUDA device is missing, calls raise.
"""
import ctypes
import os

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libltl_b200.so")

OK, EINVAL, ECUDA, ETIMEOUT, EUNSUPPORTED, ENOMEM = 0, -1, -2, -3, -4, -5
VARIANT_AUTO, VARIANT_PLAIN, VARIANT_TENSOR, VARIANT_PACKED = -1, 0, 1, 2
VARIANT_NAMES = {VARIANT_PLAIN: "plain", VARIANT_TENSOR: "tensor", VARIANT_PACKED: "packed"}

# GPU solver codes added beside the reference's CPU codes 0-6 (CASolverFactory.cpp:10-119).
SOLVER_CODE_TO_VARIANT = {7: VARIANT_PLAIN, 8: VARIANT_TENSOR, 9: VARIANT_PACKED}

# Every symbol include/ltl.h declares (tests check the library exports them all).
ABI_SYMBOLS = [
    "ltl_create", "ltl_destroy", "ltl_set_stream", "ltl_get_info", "ltl_upload", "ltl_download",
    "ltl_upload_packed", "ltl_download_packed",
    "ltl_upload_device", "ltl_download_device", "ltl_step", "ltl_synchronize", "ltl_population",
    "ltl_compare_device", "ltl_benchmark_seed", "ltl_generate_state", "ltl_pack_device", "ltl_unpack_device",
    "ltl_batch_create", "ltl_batch_destroy", "ltl_batch_set_stream", "ltl_batch_upload", "ltl_batch_download",
    "ltl_batch_upload_all", "ltl_batch_download_all", "ltl_batch_step", "ltl_batch_synchronize",
    "ltl_batch_info", "ltl_batch_set_param", "ltl_set_param", "ltl_set_timing", "ltl_get_timing", "ltl_step_noalloc", "ltl_create_rect", "ltl_create_rect_variant", "ltl_download_rows_device", "ltl_upload_rows_device",
    "ltl_last_error", "ltl_version",
]


class LtlError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libltl_b200 error {code}: {msg}")
        self.code = code


class Info(ctypes.Structure):
    _fields_ = [("variant", ctypes.c_int), ("n", ctypes.c_int), ("radius", ctypes.c_int),
                ("smin", ctypes.c_int), ("smax", ctypes.c_int), ("bmin", ctypes.c_int), ("bmax", ctypes.c_int),
                ("halo", ctypes.c_int), ("pitch", ctypes.c_longlong), ("temporal_depth", ctypes.c_int),
                ("operand_bits", ctypes.c_int), ("device_bytes", ctypes.c_longlong), ("rows", ctypes.c_int)]


class GridDesc(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("radius", ctypes.c_int), ("smin", ctypes.c_int), ("smax", ctypes.c_int),
                ("bmin", ctypes.c_int), ("bmax", ctypes.c_int)]


_lib = None


def lib():
    """Load libltl_b200.so (raises if it was not built: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} not found: build it with `python -m cat_cpu_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, u8p = ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint8)
    sz, i, f = ctypes.c_size_t, ctypes.c_int, ctypes.c_float
    L.ltl_create.argtypes = [ctypes.POINTER(vp), i, i, i, i, i, i, i, i]
    L.ltl_destroy.argtypes = [vp]
    L.ltl_set_stream.argtypes = [vp, vp]
    L.ltl_get_info.argtypes = [vp, ctypes.POINTER(Info)]
    L.ltl_upload.argtypes = [vp, vp, sz]
    L.ltl_upload_packed.argtypes = [vp, vp, sz]
    L.ltl_download_packed.argtypes = [vp, vp, sz]
    L.ltl_download.argtypes = [vp, vp, sz]
    L.ltl_upload_device.argtypes = [vp, vp, sz]
    L.ltl_download_device.argtypes = [vp, vp, sz]
    L.ltl_step.argtypes = [vp, i]
    L.ltl_synchronize.argtypes = [vp]
    L.ltl_population.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64)]
    L.ltl_compare_device.argtypes = [vp, vp, sz, ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int64)]
    L.ltl_benchmark_seed.argtypes = [i]
    L.ltl_generate_state.argtypes = [vp, sz, i, i, f, i]
    L.ltl_pack_device.argtypes = [vp, sz, i, i, vp, sz, vp]
    L.ltl_unpack_device.argtypes = [vp, sz, i, i, vp, sz, vp]
    L.ltl_batch_create.argtypes = [ctypes.POINTER(vp), i, ctypes.POINTER(GridDesc), i, i]
    L.ltl_batch_destroy.argtypes = [vp]
    L.ltl_batch_set_stream.argtypes = [vp, vp]
    L.ltl_batch_upload.argtypes = [vp, i, vp, sz]
    L.ltl_batch_download.argtypes = [vp, i, vp, sz]
    L.ltl_batch_upload_all.argtypes = [vp, vp]
    L.ltl_batch_download_all.argtypes = [vp, vp]
    L.ltl_batch_step.argtypes = [vp, i]
    L.ltl_batch_synchronize.argtypes = [vp]
    L.ltl_batch_info.argtypes = [vp, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_int)]
    L.ltl_set_param.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
    L.ltl_batch_set_param.argtypes = [vp, ctypes.c_char_p, ctypes.c_longlong]
    L.ltl_set_timing.argtypes = [vp, i]
    L.ltl_get_timing.argtypes = [vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_longlong)]
    L.ltl_step_noalloc.argtypes = [vp, sz, vp, sz, i, i, i, i, i, i, i, vp]
    L.ltl_create_rect.argtypes = [ctypes.POINTER(vp), i, i, i, i, i, i, i, i]
    L.ltl_create_rect_variant.argtypes = [ctypes.POINTER(vp), i, i, i, i, i, i, i, i, i]
    L.ltl_download_rows_device.argtypes = [vp, i, i, vp, sz]
    L.ltl_upload_rows_device.argtypes = [vp, i, i, vp, sz]
    L.ltl_last_error.restype = ctypes.c_char_p
    L.ltl_version.restype = ctypes.c_char_p
    _lib = L
    return L


def check(code):
    if code != OK:
        raise LtlError(code, lib().ltl_last_error().decode(errors="replace"))
    return code


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def benchmark_seed(seed):
    """CPUBenchmark::run/reset: srand(seed); rand() % 1000000 (CPUBenchmark.cpp:21-32)."""
    return lib().ltl_benchmark_seed(int(seed))


def generate_state(n, seed, density, threads=1):
    """CAStateGenerator::generateRandomState for state seed `seed` (CAStateGenerator.h:11-37)."""
    out = np.empty((n, n), dtype=np.uint8)
    check(lib().ltl_generate_state(_ptr(out), n, n, int(seed), float(density), int(threads)))
    return out


def start_grid(n, user_seed, density, threads=1):
    """The start grid the reference benchmarks for `--seed user_seed -d density --threads threads`."""
    return generate_state(n, benchmark_seed(user_seed), density, threads)


class CUDASolver:
    """One n x n torus on a GPU.  Method names follow CASolver (CASolver.h:7-28);
    radius and rule (reference centre-excluded convention) are run-time values.
    rows: a rows x n torus instead (plain or packed variant; ltl_create_rect_variant)."""

    def __init__(self, n, radius, rule, variant=VARIANT_AUTO, device=0, threads=1, rows=None):
        smin, smax, bmin, bmax = rule
        h = ctypes.c_void_p()
        if rows is None:
            check(lib().ltl_create(ctypes.byref(h), int(device), int(n), int(radius), int(smin), int(smax),
                                   int(bmin), int(bmax), int(variant)))
        else:
            check(lib().ltl_create_rect_variant(ctypes.byref(h), int(device), int(rows), int(n), int(radius),
                                                int(smin), int(smax), int(bmin), int(bmax), int(variant)))
        self._h = h
        self.n, self.radius, self.rule, self.device, self.threads = n, radius, tuple(rule), device, threads
        self.rows = n if rows is None else int(rows)
        self.info = self.get_info()
        self.variant = self.info.variant

    # --- lifecycle -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().ltl_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def get_info(self):
        info = Info()
        check(lib().ltl_get_info(self._h, ctypes.byref(info)))
        return info

    # --- CASolver interface ----------------------------------------------
    def resetState(self, seed, density):
        """CASolver::resetState (CASolver.cpp:3-7): generate with state seed `seed`
        on the host (as many generator threads as the solver was given), upload."""
        self.setState(generate_state(self.n, seed, density, self.threads))

    def setState(self, grid):
        g = np.ascontiguousarray(grid, dtype=np.uint8)
        assert g.shape == (self.rows, self.n)
        check(lib().ltl_upload(self._h, _ptr(g), self.n))

    def doStep(self):
        self.doSteps(1)

    def doSteps(self, steps):
        check(lib().ltl_step(self._h, int(steps)))

    def synchronize(self):
        check(lib().ltl_synchronize(self._h))

    def setStatePacked(self, words):
        """Upload a grid in the PACK coding: uint64 array (rows, ceil(n / 64)),
        cell (i, j) = bit j % 64 of word j / 64 (see pack_grid)."""
        w = np.ascontiguousarray(words, dtype=np.uint64)
        assert w.shape == (self.rows, (self.n + 63) // 64)
        check(lib().ltl_upload_packed(self._h, _ptr(w), w.shape[1] * 8))

    def getCurrentStatePacked(self):
        """The current grid in the PACK coding (bits past n are 0)."""
        out = np.empty((self.rows, (self.n + 63) // 64), dtype=np.uint64)
        check(lib().ltl_download_packed(self._h, _ptr(out), out.shape[1] * 8))
        return out

    def getCurrentState(self):
        """CASolver::getCurrentState (CASolver.cpp:9-13): inner n x n (rows x n) cells, uint8."""
        out = np.empty((self.rows, self.n), dtype=np.uint8)
        check(lib().ltl_download(self._h, _ptr(out), self.n))
        return out

    def printCurrentState(self):
        """CADataPrinter-style dump without halo ('-' for dead cells)."""
        g = self.getCurrentState()
        for row in g:
            print(" ".join("-" if v == 0 else str(int(v)) for v in row))

    def set_param(self, name, value):
        check(lib().ltl_set_param(self._h, name.encode(), int(value)))
        self.info = self.get_info()

    def set_timing(self, enable):
        check(lib().ltl_set_timing(self._h, int(bool(enable))))

    def get_timing(self):
        """(summed step-kernel milliseconds, step-kernel launches, all library launches)."""
        ms, k, a = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_longlong()
        check(lib().ltl_get_timing(self._h, ctypes.byref(ms), ctypes.byref(k), ctypes.byref(a)))
        return ms.value, k.value, a.value

    def population(self):
        v = ctypes.c_uint64()
        check(lib().ltl_population(self._h, ctypes.byref(v)))
        return v.value

    # --- device-pointer variants (torch tensors or raw CUDA pointers) ------
    def set_stream(self, stream_ptr):
        check(lib().ltl_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    def upload_device(self, dev_ptr, pitch):
        check(lib().ltl_upload_device(self._h, ctypes.c_void_p(dev_ptr), int(pitch)))

    def download_device(self, dev_ptr, pitch):
        check(lib().ltl_download_device(self._h, ctypes.c_void_p(dev_ptr), int(pitch)))

    def download_rows_device(self, row0, nrows, dev_ptr, pitch):
        check(lib().ltl_download_rows_device(self._h, int(row0), int(nrows), ctypes.c_void_p(dev_ptr), int(pitch)))

    def upload_rows_device(self, row0, nrows, dev_ptr, pitch):
        check(lib().ltl_upload_rows_device(self._h, int(row0), int(nrows), ctypes.c_void_p(dev_ptr), int(pitch)))

    def compare_device(self, dev_ptr, pitch):
        mm, first = ctypes.c_uint64(), ctypes.c_int64()
        check(lib().ltl_compare_device(self._h, ctypes.c_void_p(dev_ptr), int(pitch), ctypes.byref(mm),
                                       ctypes.byref(first)))
        return mm.value, first.value


class CASolverFactory:
    """createSolver(code, deviceId, n, radius, nThreads, rule) -> CUDASolver or None
    (the reference returns nullptr for unknown codes, CASolverFactory.cpp:119-120).
    Codes 7/8/9 are the GPU plain / tensor-core / packed solvers."""

    @staticmethod
    def createSolver(code, deviceId, n, radius, nThreads, rule):
        variant = SOLVER_CODE_TO_VARIANT.get(code)
        if variant is None:
            return None
        return CUDASolver(n, radius, rule, variant=variant, device=deviceId, threads=nThreads)


def compareCurrentStates(solver, reference_grid):
    """CADataDomainComparator::compareCurrentStates: True iff every inner cell matches."""
    return bool(np.array_equal(solver.getCurrentState(), np.asarray(reference_grid, dtype=np.uint8)))


class Batch:
    """Many independent tori advanced together (ltl_batch_*)."""

    def __init__(self, grids, device=0, flags=0):
        """grids: list of (n, radius, (smin, smax, bmin, bmax))."""
        arr = (GridDesc * len(grids))()
        for k, (n, r, rule) in enumerate(grids):
            arr[k] = GridDesc(int(n), int(r), *[int(v) for v in rule])
        h = ctypes.c_void_p()
        check(lib().ltl_batch_create(ctypes.byref(h), int(device), arr, len(grids), int(flags)))
        self._h = h
        self.grids = list(grids)
        self.sizes = [int(g[0]) for g in grids]
        self.offsets = np.concatenate([[0], np.cumsum([s * s for s in self.sizes])]).astype(np.int64)

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib().ltl_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        cells, dev, depth = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_int()
        check(lib().ltl_batch_info(self._h, ctypes.byref(cells), ctypes.byref(dev), ctypes.byref(depth)))
        return cells.value, dev.value, depth.value

    def upload(self, k, grid):
        g = np.ascontiguousarray(grid, dtype=np.uint8)
        check(lib().ltl_batch_upload(self._h, int(k), _ptr(g), g.shape[1]))

    def download(self, k):
        n = self.sizes[k]
        out = np.empty((n, n), dtype=np.uint8)
        check(lib().ltl_batch_download(self._h, int(k), _ptr(out), n))
        return out

    def upload_all(self, flat):
        flat = np.ascontiguousarray(flat, dtype=np.uint8)
        assert flat.size == self.offsets[-1]
        check(lib().ltl_batch_upload_all(self._h, _ptr(flat)))

    def download_all(self, out=None):
        if out is None:
            out = np.empty(int(self.offsets[-1]), dtype=np.uint8)
        check(lib().ltl_batch_download_all(self._h, _ptr(out)))
        return out

    def step(self, steps):
        check(lib().ltl_batch_step(self._h, int(steps)))

    def set_param(self, name, value):
        check(lib().ltl_batch_set_param(self._h, name.encode(), int(value)))

    def synchronize(self):
        check(lib().ltl_batch_synchronize(self._h))

    def set_stream(self, stream_ptr):
        check(lib().ltl_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr)))


def pack_grid(grid):
    """A 0/1 uint8 grid (rows, n) in the PACK coding: uint64 (rows, ceil(n / 64)),
    cell (i, j) = bit j % 64 of word j / 64."""
    g = np.asarray(grid, dtype=np.uint8)
    rows, n = g.shape
    nw = (n + 63) // 64
    padded = np.zeros((rows, nw * 64), dtype=np.uint8)
    padded[:, :n] = g != 0
    return np.packbits(padded, axis=1, bitorder="little").view("<u8").reshape(rows, nw)


def unpack_grid(words, n):
    """Inverse of pack_grid: uint8 (rows, n)."""
    w = np.ascontiguousarray(words, dtype="<u8")
    bits = np.unpackbits(w.view(np.uint8), axis=1, bitorder="little")
    return bits[:, :n].copy()

/*
 * ltl.h -- C ABI of the B200 Larger-than-Life stepping engine (libltl_b200.so).
 *
 * Plain C: pointers, sizes and int status codes; no CUDA or torch types.  Every
 * entry point returns LTL_OK (0) or a negative LTL_E* code and never throws;
 * ltl_last_error() gives the calling thread's last message.
 *
 * Cell and rule conventions follow the reference (kezada94/CAT_cpu):
 *   - a grid is a square torus of n x n cells, each 0 or 1 (uint8 on the host);
 *   - k = live cells in the (2R+1)^2 Moore box around a cell, centre EXCLUDED
 *     (HostSolver.tpp:75-91);
 *   - next = s ? [smin <= k <= smax] : [bmin <= k <= bmax]   (HostSolver.tpp:58-73).
 * A rule quoted with the centre counted (e.g. Bosco S33-57/B34-45) maps to
 * smin/smax one lower and bmin/bmax unchanged.
 *
 * Each declaration names the reference interface it replaces (file:line inside
 * the reference project).
 */
#ifndef LTL_H
#define LTL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference has none (it exit(1)s, main.cpp:52-56,81-85). */
#define LTL_OK 0
#define LTL_EINVAL (-1)       /* bad argument: n, radius, pointer, pitch, grid index */
#define LTL_ECUDA (-2)        /* a CUDA runtime/driver call failed */
#define LTL_ETIMEOUT (-3)     /* a bounded device wait gave up (error flag set by a kernel) */
#define LTL_EUNSUPPORTED (-4) /* variant cannot run this (n, radius) exactly */
#define LTL_ENOMEM (-5)       /* device allocation failed */

/* Stepping variants (the GPU analogues of the reference's solver codes,
 * CASolverFactory.cpp:10-119; the reference's own codes 0-6 are CPU solvers). */
#define LTL_VARIANT_AUTO (-1)  /* pick the fastest exact variant for (n, R) */
#define LTL_VARIANT_PLAIN 0    /* CUDA-core SWAR stencil, uint8 cells */
#define LTL_VARIANT_TENSOR 1   /* tcgen05 banded products B_v * X * B_h, bit-packed grid */
#define LTL_VARIANT_PACKED 2   /* bit-packed cells (64 per uint64), CUDA-core bit logic */

typedef struct ltl_ctx ltl_ctx;

typedef struct {
    int variant;          /* variant actually used */
    int n, radius;
    int smin, smax, bmin, bmax;
    int halo;             /* halo width of the device grid (cells) */
    long long pitch;      /* device row pitch (bytes) */
    int temporal_depth;   /* generations advanced per kernel pass */
    int operand_bits;     /* tensor path: 8 (u8 kind::i8) or 16 (f16 kind::f16); 0 otherwise */
    long long device_bytes; /* device memory held by the context */
    int rows;             /* rows of the torus (== n except for ltl_create_rect) */
} ltl_info;

/* Create a solver for one n x n torus on `device` (CUDA ordinal).
 * Replaces CASolverFactory::createSolver (CASolverFactory.cpp:6-121) for the
 * GPU codes; radius and rule are run-time values instead of the RADIUS/SMIN/
 * SMAX/BMIN/BMAX macros (Makefile:10-14).  n >= radius is required (the
 * reference's torus halo is only defined there, HostSolver.tpp:93-140).
 * Radius ranges: plain 1..2038, packed 1..32, tensor 1..128; outside them
 * LTL_EUNSUPPORTED. */
int ltl_create(ltl_ctx** out, int device, int n, int radius, int smin, int smax, int bmin, int bmax,
               int variant);

/* A plain-variant solver for a rows x cols torus (rows may differ from cols).
 * The building block of one grid split into row strips across GPUs: a strip of
 * m rows plus R*k halo rows above and below, stepped as a torus of its own for
 * k generations, leaves its m inner rows exact (the false vertical wrap only
 * reaches R*k rows in).  No counterpart in the reference, whose grids are
 * square and live in one process (CADataDomain.tpp:4-98). */
int ltl_create_rect(ltl_ctx** out, int device, int rows, int cols, int radius, int smin, int smax, int bmin,
                    int bmax);

/* ltl_create_rect for a chosen variant: LTL_VARIANT_PLAIN or LTL_VARIANT_PACKED
 * (the bit-packed step also takes rows != cols; LTL_VARIANT_AUTO means plain,
 * any other variant LTL_EUNSUPPORTED when rows != cols).  Row strips of the
 * packed variant move their halo rows through ltl_download_rows_device /
 * ltl_upload_rows_device, which unpack or pack only the rows asked for.  No
 * counterpart in the reference. */
int ltl_create_rect_variant(ltl_ctx** out, int device, int rows, int cols, int radius, int smin, int smax, int bmin,
                            int bmax, int variant);

/* Release device memory and graphs.  (The reference never frees its domains.) */
int ltl_destroy(ltl_ctx* ctx);

/* Use a caller-owned cudaStream_t (passed as void*) for all later work; NULL
 * restores the context's own stream. */
int ltl_set_stream(ltl_ctx* ctx, void* stream);

int ltl_get_info(const ltl_ctx* ctx, ltl_info* info);

/* Host -> device: `inner` holds n rows of n bytes (0/1), rows `pitch` bytes apart.
 * Replaces copyHostVisibleDataToCurrentState (e.g. AMXSolver16.cpp:209-214),
 * reached from CASolver::resetState (CASolver.cpp:3-7).  Synchronous. */
int ltl_upload(ltl_ctx* ctx, const uint8_t* inner, size_t pitch);

/* Device -> host, same layout.  Replaces copyCurrentStateToHostVisibleData
 * (AMXSolver16.cpp:202-207) reached from CASolver::getCurrentState
 * (CASolver.cpp:9-13).  Synchronous. */
int ltl_download(ltl_ctx* ctx, uint8_t* inner, size_t pitch);

/* The same two transfers with the host grid in the PACK coding: row i holds
 * ceil(cols / 64) uint64 words, cell (i, j) = bit j % 64 of word j / 64 (bits past
 * cols are 0 on download and ignored on upload), rows `word_pitch_bytes` apart
 * (at least 8 ceil(cols / 64)).  Eight times fewer bytes cross PCIe than with the
 * uint8 forms; for the packed and tensor variants the words go straight into the
 * device's packed frames (a little-endian uint64 row is the frames' 32-bit word
 * row).  Synchronous.  The reference keeps uint8 grids only; this is the packed
 * grid I/O of its GPU project's PACK solver, whose source it does not include. */
int ltl_upload_packed(ltl_ctx* ctx, const uint64_t* words, size_t word_pitch_bytes);
int ltl_download_packed(ltl_ctx* ctx, uint64_t* words, size_t word_pitch_bytes);

/* Same as ltl_upload/ltl_download with device-resident inner grids (stream-ordered
 * on the context's stream, not synchronised). */
int ltl_upload_device(ltl_ctx* ctx, const uint8_t* dev_inner, size_t pitch);
int ltl_download_device(ltl_ctx* ctx, uint8_t* dev_inner, size_t pitch);

/* Advance `steps` generations (asynchronous on the context's stream).
 * Replaces CASolver::doSteps/doStep (CASolver.cpp:15-31): halo fill, step, swap. */
int ltl_step(ltl_ctx* ctx, int steps);

/* Wait for all work queued on the context's stream; reports device-side error flags. */
int ltl_synchronize(ltl_ctx* ctx);

/* Live-cell count of the current grid (device reduction; synchronous). */
int ltl_population(ltl_ctx* ctx, uint64_t* live);

/* Compare the current grid with a device-resident n x n grid: number of
 * differing cells and the row-major index of the first one (-1 if none).
 * Replaces CADataDomainComparator::compareCurrentStates
 * (CADataDomainComparator.tpp:8-27), which stops at the first mismatch. */
int ltl_compare_device(ltl_ctx* ctx, const uint8_t* dev_expected, size_t pitch, uint64_t* mismatches,
                       int64_t* first_index);

/* The state seed the reference's benchmark derives from --seed:
 * CPUBenchmark::run/reset (CPUBenchmark.cpp:21-32) do srand(seed) and pass
 * rand() % 1000000 to resetState.  Uses (and reseeds) the process-wide rand(). */
int ltl_benchmark_seed(int seed);

/* The reference's start grid on the host, CAStateGenerator::generateRandomState
 * (CAStateGenerator.h:11-37) as called by CASolver::resetState(seed, density)
 * (CASolver.cpp:3-7) with `threads` OpenMP threads: the n*n cells (row-major) are
 * split into `threads` contiguous chunks of ceil(n*n/threads); chunk t is drawn
 * from std::mt19937(seed + t), cell = draw / 2^32 < density.  Writes n rows of
 * n bytes (0/1), `pitch` bytes apart. */
int ltl_generate_state(uint8_t* out, size_t pitch, int n, int seed, float density, int threads);

/* ---------------- PACK codec (device pointers, stream-ordered) ---------------
 * Bit-packed row layout used by LTL_VARIANT_PACKED: cell (i, j) is bit (j % 64)
 * of uint64 word j / 64 of row i; bits past n in the last word are zero.
 * No reference counterpart in CAT_cpu (its README's PACK solver has no source
 * in that tree); defined here. */
int ltl_pack_device(const uint8_t* dev_cells, size_t cell_pitch, int rows, int cols, uint64_t* dev_words,
                    size_t word_pitch_bytes, void* stream);
int ltl_unpack_device(const uint64_t* dev_words, size_t word_pitch_bytes, int rows, int cols,
                      uint8_t* dev_cells, size_t cell_pitch, void* stream);

/* ---------------- Batched grids --------------------------------------------
 * Many independent tori of uneven size, radius and rule advanced together in
 * one persistent launch per pass.  The reference runs one grid per process
 * (CPUBenchmark.cpp:63-85); this is the batched analogue of CASolver::doSteps. */
typedef struct {
    int n;
    int radius;
    int smin, smax, bmin, bmax;
} ltl_grid_desc;

typedef struct ltl_batch ltl_batch;

/* ltl_batch_create flags */
#define LTL_BATCH_STREAM_ALL 1  /* per-generation launches only: no persistent or shared-memory-resident grids */
#define LTL_BATCH_NO_GRAPH 2    /* launch the step loop directly instead of replaying a CUDA graph */

int ltl_batch_create(ltl_batch** out, int device, const ltl_grid_desc* descs, int count, int flags);
int ltl_batch_destroy(ltl_batch* b);
int ltl_batch_set_stream(ltl_batch* b, void* stream);
int ltl_batch_upload(ltl_batch* b, int grid, const uint8_t* inner, size_t pitch);
int ltl_batch_download(ltl_batch* b, int grid, uint8_t* inner, size_t pitch);
/* One host buffer holding every grid back to back (grid g at offset
 * sum_{h<g} n_h^2, rows of n_g bytes): one copy each way for the whole batch. */
int ltl_batch_upload_all(ltl_batch* b, const uint8_t* cells);
int ltl_batch_download_all(ltl_batch* b, uint8_t* cells);
int ltl_batch_step(ltl_batch* b, int steps);
/* Batch shape parameters (autotuned; also read from the tuning table):
 *   "persistent"          1 (default): one persistent launch per rule class runs
 *                         every generation of an ltl_batch_step, each CTA taking
 *                         whole grids, largest first; 0: per-generation launches
 *                         (the two parameters below apply)
 *   "stream_band_rows"    rows per work item of the streamed per-step kernels
 *   "resident_max_bytes"  shared-memory budget deciding which grids stay resident
 * Setting one rebuilds the work lists before the next step. */
int ltl_batch_set_param(ltl_batch* b, const char* name, long long value);
int ltl_batch_synchronize(ltl_batch* b);
/* Total cells of the batch (sum of n^2) and its device bytes; temporal_depth =
 * the number of grids that run all generations of an ltl_batch_step inside
 * one launch (every grid in persistent mode, the shared-memory-resident ones
 * otherwise). */
int ltl_batch_info(const ltl_batch* b, long long* cells, long long* device_bytes, int* temporal_depth);

/* Shape parameters (what cat_cpu_b200/autotune.py sweeps; the autotuned table
 * tuning/ltl_tuning.txt next to the library sets them at ltl_create):
 *   "band_rows"  rows per work item of the plain and packed step kernels
 *                (0: the built-in choice);
 *   "depth"      generations per pass of the plain variant: 1, or 2..3 with
 *                depth * R <= 16 and R <= 5 (temporal blocking: one read and
 *                one write of the grid per pass).  ltl_step accepts any step
 *                count; a remainder runs as one shorter pass.
 * The analogue of the reference project's NREGIONS_H/V region counts.
 * Failure-path controls of the tensor variant (its kernel waits on mbarriers,
 * every wait bounded):
 *   "wait_limit_ns"          limit of each wait (default 2e9);
 *   "inject_missing_commit"  1 = withhold one completion signal, so the next
 *                            pass's waits run out and ltl_synchronize returns
 *                            LTL_ETIMEOUT (used by the failure-detection test). */
int ltl_set_param(ltl_ctx* ctx, const char* name, long long value);

/* Kernel timing for benchmarks (the reference times whole runs with a
 * host clock, CpuTimer.cpp:7-19 / CPUBenchmark.cpp:71-84).  While enabled,
 * ltl_step launches passes one by one (no CUDA graph) and records CUDA events
 * around the step kernel(s) of every pass on the context's stream;
 * ltl_get_timing synchronises and returns their summed duration and how many
 * step-kernel launches and library kernel launches (step + halo) were made
 * since timing was enabled.  Enabling resets the counters. */
int ltl_set_timing(ltl_ctx* ctx, int enable);
int ltl_get_timing(ltl_ctx* ctx, double* step_kernel_ms, long long* step_kernel_launches,
                   long long* all_launches);

/* One plain CUDA-core run for callers that cannot allocate device memory
 * (a host framework that owns all device memory through its own pool, a
 * real-time service that forbids allocation after start-up, a plug-in that is
 * handed buffers and a stream and nothing else).  No counterpart in the
 * reference: it is an addition of this library.
 *
 * Advances the n x n grid `dev_in` (device memory, rows `in_pitch` bytes
 * apart, cells 0/1) by `steps` generations and writes it to `dev_out` (may be
 * the same buffer), stream-ordered on `stream` (NULL: the default stream) of
 * the current device.  It calls no cudaMalloc/cudaFree: the two halo'd grids it
 * needs live in a fixed 32 MiB array in device memory that every GPU loading
 * the library holds until the process exits.  Grids needing more return
 * LTL_EINVAL with a message: a grid takes round_up((n + 2H + 1) * pitch, 256)
 * bytes, H = 16 for R <= 16 (32 up to R = 32, ...), pitch = round_up(n + 2H + 16,
 * 64), and two must fit, so n <= 4048 for R <= 16 and less for larger R.
 * The first call on a device looks up that array's address and sets the
 * kernels' shared-memory limits; make that first call before any stream
 * capture.  All calls share the one array and it keeps the last call's data:
 * calls that can overlap on the GPU (different streams, or different threads
 * without ordering) race and corrupt each other's results. */
int ltl_step_noalloc(const uint8_t* dev_in, size_t in_pitch, uint8_t* dev_out, size_t out_pitch, int n, int radius,
                     int smin, int smax, int bmin, int bmax, int steps, void* stream);

/* Rows [row0, row0 + nrows) of the current grid to or from device memory
 * (`pitch` bytes between rows, cells 0/1), stream-ordered on the context's
 * stream: the halo exchange of row strips.  No reference counterpart. */
int ltl_download_rows_device(ltl_ctx* ctx, int row0, int nrows, uint8_t* dev, size_t pitch);
int ltl_upload_rows_device(ltl_ctx* ctx, int row0, int nrows, const uint8_t* dev, size_t pitch);

/* Message for the calling thread's last failed call ("" if none). */
const char* ltl_last_error(void);

/* Library version string. */
const char* ltl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* LTL_H */

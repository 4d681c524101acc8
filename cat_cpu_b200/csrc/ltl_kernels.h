// ltl_kernels.h -- host-side launchers of the libltl_b200 kernels (internal).
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "ltl_internal.cuh"

namespace ltl {

// K5: refresh the torus halo of a frame (every halo cell <- its inner source).
cudaError_t launch_halo_fill(const Frame& f, cudaStream_t s);

// K1 fast path: SWAR 8-bit lanes, warp-shuffle row sums; R <= 5.
bool plain_swar8_supported(int radius);
// One-time function attributes (dynamic shared memory) so that launches can be
// captured in CUDA graphs without configuration calls.
cudaError_t plain_prepare(int radius);
cudaError_t packed_prepare(int radius);
// wrap: read every cell from its inner position (torus wrap inside the kernel),
// so the frame halo is neither read nor needed; requires plain_wrap_supported(n).
bool plain_wrap_supported(int n, int rows);
cudaError_t launch_plain_swar8(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows, bool wrap,
                               cudaStream_t s);
int plain_swar8_band_rows(int n, int device);
// Temporally blocked SWAR step: `depth` (2 or 3, depth * R <= 16) generations per
// pass; the frames' halo must be at least depth * R.
bool plain_tb_supported(int radius, int depth);
cudaError_t plain_tb_prepare(int radius);
cudaError_t launch_plain_tb(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows, int depth,
                            bool wrap, cudaStream_t s);

// K1 generic path (R up to 2038): one fused kernel (vertical window sums in
// registers, a prefix scan per row, or per pair of rows, in shared memory, the
// rule); needs a halo of at least R rounded up to plain_wide_cols_per_thread(R).
// band_rows: rows per CTA (0: 64).
bool plain_generic_supported(int radius);
int plain_wide_cols_per_thread(int radius);
cudaError_t launch_plain_generic(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows,
                                 cudaStream_t s);

// K6: population and comparison over the inner n x n cells.  `scratch` holds
// two uint64 (count, first index) in device memory.
cudaError_t launch_population(const Frame& f, unsigned long long* scratch, cudaStream_t s);
cudaError_t launch_compare(const Frame& f, const uint8_t* other, size_t other_pitch,
                           unsigned long long* scratch, cudaStream_t s);

// Copies between a dense n x n grid (pitch bytes per row) and a frame's inner cells.
cudaError_t launch_copy_in(const Frame& f, const uint8_t* src, size_t src_pitch, cudaStream_t s);
cudaError_t launch_copy_out(const Frame& f, uint8_t* dst, size_t dst_pitch, cudaStream_t s);

// K3: bit-packed variant.  Packed frame: 32-bit words, cell (i, j) is bit j % 32
// of word j / 32 (LSB first; two consecutive words are one little-endian uint64
// of the PACK codec).  Inner row i is frame row HR + i, inner word w is frame
// column HW + w; halo bits hold torus copies, like the byte frame.
struct PackedFrame {
    uint32_t* words;
    int n;          // cells per side
    int nw;         // inner words per row = ceil(n / 32)
    int HR;         // halo rows (>= R + 1)
    int HW;         // halo words on each side (1: radius <= 32)
    size_t wpitch;  // words per frame row
    int rows = 0;   // inner rows of a rectangular torus (0: square, n rows)
    __host__ __device__ int nrows() const { return rows ? rows : n; }
};
bool packed_supported(int n, int radius);
// band_rows <= 0: built-in heuristic; > 0: rows per work item (tuning table / ltl_set_param)
cudaError_t launch_packed_step(const PackedFrame& cur, const PackedFrame& nxt, const Rule& rule, int band_rows,
                               cudaStream_t s);
cudaError_t launch_packed_halo(const PackedFrame& f, cudaStream_t s);
// true when launch_packed_step also refreshes the output frame's halo
bool packed_fused_halo(const PackedFrame& f, int radius);
cudaError_t launch_pack_frame(const Frame& src, const PackedFrame& dst, cudaStream_t s);
cudaError_t launch_unpack_frame(const PackedFrame& src, const Frame& dst, cudaStream_t s);
// Inner rows [row0, row0 + nrows) of a packed frame to / from a dense byte
// buffer (buffer row i = frame row row0 + i, `pitch` bytes apart, 0/1 cells).
// After packing rows in, the frame's halo is stale: refresh it.
cudaError_t launch_unpack_rows(const PackedFrame& src, int row0, int nrows, uint8_t* dst, size_t pitch, cudaStream_t s);
cudaError_t launch_pack_rows(const uint8_t* src, size_t pitch, const PackedFrame& dst, int row0, int nrows,
                             cudaStream_t s);
// A packed frame's inner words as PACK-coded rows (bits past n cleared).
cudaError_t launch_frame_to_pack64(const PackedFrame& f, uint64_t* dst, size_t dst_pitch_words, cudaStream_t s);
cudaError_t launch_pack(const uint8_t* cells, size_t cell_pitch, int rows, int cols, uint64_t* words,
                        size_t word_pitch_words, cudaStream_t s);
cudaError_t launch_unpack(const uint64_t* words, size_t word_pitch_words, int rows, int cols, uint8_t* cells,
                          size_t cell_pitch, cudaStream_t s);

// K2: tcgen05 banded-product step on packed frames (the tensor variant keeps
// its grid in the packed layout of K3; the kernel wraps rows and words modulo n
// itself, so the packed halo is never read).  The frames need HW >= 1.
struct TensorPlan;
bool tensor_supported(int n, int radius, char* why, size_t why_len);
TensorPlan* tensor_plan_create(const PackedFrame& a, const PackedFrame& b, const Rule& rule, int device, char* why,
                               size_t why_len);
void tensor_plan_destroy(TensorPlan* p);
int tensor_plan_depth(const TensorPlan* p);
int tensor_plan_operand_bits(const TensorPlan* p);
// Advance one pass (tensor_plan_depth generations) from packed frame `src_is_a ? a : b`.
cudaError_t launch_tensor_pass(TensorPlan* p, bool src_is_a, cudaStream_t s);
unsigned int* tensor_plan_error_flag(TensorPlan* p);
// Limit of the kernel's bounded waits, and a test hook that withholds one
// completion signal so that the waits run out (no fault, no hang: the kernel
// returns after the limit with an error bit set).
void tensor_plan_set_wait(TensorPlan* p, unsigned long long ns, int inject_missing_commit);

// Tuning table (written by cat_cpu_b200/autotune.py): the value of `param` for
// (variant name, radius, n), or `fallback` when no line matches.  Lines look like
//   variant=plain radius=5 nmin=8192 nmax=65536 band_rows=128
// radius=* matches every radius.  The file is $LTL_TUNING_FILE, else
// tuning/ltl_tuning.txt next to libltl_b200.so.
long long tuning_lookup(const char* variant, int radius, long long n, const char* param, long long fallback);

}  // namespace ltl

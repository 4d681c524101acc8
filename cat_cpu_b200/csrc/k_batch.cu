// k_batch.cu -- K4: many independent tori of uneven size, radius and rule,
// advanced together (ltl_batch_* in include/ltl.h).
//
// Semantics per grid are the reference's HostSolver<int> step (kezada94/CAT_cpu,
// src/CellularAutomata/Solvers/HostSolver.tpp:58-140); the reference runs one
// grid per process (CPUBenchmark.cpp:63-85).  Design:
//   - every grid is stored bit-packed (packed_core.cuh) in one device arena,
//     two arenas ping-pong;
//   - grids are grouped into rule classes (radius + rule); each class gets its
//     own kernel instantiation, with the rule's bit masks in the constant bank;
//   - "resident" grids (small enough that two packed copies fit in one SM's
//     shared memory) are advanced all requested steps in ONE launch: a CTA loads
//     the grid once, keeps the torus halo in shared memory and writes the grid
//     back after the last step (temporal blocking of the whole run);
//   - larger grids are advanced one generation per launch by a persistent
//     kernel that walks a (grid, row band, word strip) work list, followed by a
//     batched halo refresh; the whole step loop is captured in a CUDA graph, and
//     the resident launches run concurrently on a forked stream.
#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "../../include/ltl.h"
#include "packed_core.cuh"

namespace ltl {

struct BatchGrid {
    long long off;       // word offset of the grid's packed frame in an arena
    long long cell_off;  // byte offset of the grid in the dense staging buffer
    int n, nw, HR, wp;   // cells per side, inner words per row, halo rows, words per frame row
    int R;
    int cls;             // rule class
};

#define LTL_BATCH_RADII(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16)

constexpr int kBatchWarps = 4;
constexpr int kResThreads = 1024;
constexpr int kResSmemLimit = 220 * 1024;

// ---------------------------------------------------------------------------
// Per-step kernel for the streamed grids of one rule class.
// ---------------------------------------------------------------------------
template <int R>
__global__ void __launch_bounds__(kBatchWarps * 32)
k_batch_step(const uint32_t* __restrict__ cur, uint32_t* __restrict__ nxt, const BatchGrid* __restrict__ grids,
             const int4* __restrict__ items, int n_items, const __grid_constant__ PackedRule pr) {
    using Ring = PackedRing<R, kBatchWarps>;
    extern __shared__ uint32_t ring_all[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    uint32_t* ring_lane = ring_all + (size_t)wid * Ring::WARP_WORDS + lane;
    const int gwarp = blockIdx.x * kBatchWarps + wid;
    const int gwarps = gridDim.x * kBatchWarps;
    for (int it = gwarp; it < n_items; it += gwarps) {
        const int4 item = items[it];  // grid, r0, r1, word strip
        const BatchGrid g = grids[item.x];
        const int w = item.w * 32 + lane;
        packed_band<R, Ring::fits>(cur + g.off, nxt + g.off, (size_t)g.wp, g.HR, item.y, item.z, 1 + w, w <= g.nw,
                                   w < g.nw, lane, ring_lane, pr);
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Halo refresh of packed frames (same rules as k_packed.cu's halo kernels):
// bit position p of an inner row holds cell (p - 32) mod n, then the top and
// bottom halo rows are copies of the inner rows they wrap to.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t frame_bit(const uint32_t* row, int cell) {
    const int p = 32 + cell;
    return (row[p >> 5] >> (p & 31)) & 1u;
}

__device__ __forceinline__ uint32_t halo_word_bits(const uint32_t* row, int fw, int n, int nw) {
    // frame word fw (0 = left halo, nw = last inner, nw + 1 = right halo), bit by bit
    if (fw == nw) {
        const int inner_bits = n - 32 * (nw - 1);
        uint32_t v = inner_bits >= 32 ? row[fw] : (row[fw] & ((1u << inner_bits) - 1u));
        for (int b = inner_bits; b < 32; ++b) v |= frame_bit(row, (32 * (nw - 1) + b) % n) << b;
        return v;
    }
    uint32_t v = 0u;
    for (int b = 0; b < 32; ++b) {
        const int cell = 32 * (fw - 1) + b;
        v |= frame_bit(row, ((cell % n) + n) % n) << b;
    }
    return v;
}

__device__ __forceinline__ uint32_t halo_word(const uint32_t* row, int fw, int n, int nw) {
    return packed_halo_word(row, fw, n, nw, [&] { return halo_word_bits(row, fw, n, nw); });
}

// The three column-halo words of one inner frame row: frame word 0 (cells
// n-32 .. n-1), the last inner word's bits past n, and frame word nw + 1 (the
// cells that follow).  For n >= 64 it reads the four inner words they come
// from once (first two, last two); smaller grids take the bit-by-bit path.
__device__ __forceinline__ void halo_cols_row(uint32_t* row, int n, int nw) {
    if (n >= 64) {
        const uint32_t w1 = row[1], w2 = row[2];  // inner words 0 and 1
        const uint32_t wl = row[nw], wp = row[nw - 1];  // inner words nw - 1 and nw - 2
        const int ib = n - 32 * (nw - 1);  // inner bits of the last word, 1..32
        // the last inner word with its bits past n filled from the row's start
        const uint32_t last = ib >= 32 ? wl : ((wl & ((1u << ib) - 1u)) | (w1 << ib));
        // frame word 0: cells n-32 .. n-1 = the 32 bits that end at inner bit ib of the last word
        const uint32_t left = ib >= 32 ? wl : __funnelshift_r(wp, wl, ib);
        // frame word nw + 1: cells 32 nw - n .. (the row's start shifted by the bits past n)
        const int c = 32 * nw - n;
        const uint32_t right = c ? __funnelshift_r(w1, w2, c) : w1;
        row[0] = left;
        row[nw] = last;
        row[nw + 1] = right;
    } else {
        for (int k = 0; k < 3; ++k) {
            const int fw = k == 0 ? 0 : nw + (k - 1);
            row[fw] = halo_word(row, fw, n, nw);
        }
    }
}

// One thread per inner row writes the row's three column-halo words.
__global__ void k_batch_halo_cols(uint32_t* __restrict__ arena, const BatchGrid* __restrict__ grids,
                                  const int* __restrict__ list) {
    const BatchGrid g = grids[list[blockIdx.y]];
    uint32_t* f = arena + g.off;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < g.n; i += gridDim.x * blockDim.x)
        halo_cols_row(f + (size_t)(g.HR + i) * g.wp, g.n, g.nw);
}

__global__ void k_batch_halo_rows(uint32_t* __restrict__ arena, const BatchGrid* __restrict__ grids,
                                  const int* __restrict__ list) {
    const BatchGrid g = grids[list[blockIdx.y]];
    uint32_t* f = arena + g.off;
    const int total = 2 * g.HR * g.wp;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
        const int band = t / g.wp, w = t % g.wp;
        const int r = band < g.HR ? band : g.n + band;
        const int src = g.HR + (((r - g.HR) % g.n) + g.n) % g.n;
        f[(size_t)r * g.wp + w] = f[(size_t)src * g.wp + w];
    }
}

// ---------------------------------------------------------------------------
// Resident kernel: whole grids in shared memory for `steps` generations.
// ---------------------------------------------------------------------------
__device__ void smem_halo(uint32_t* buf, int n, int nw, int HR, int wp) {
    for (int t = threadIdx.x; t < n * 3; t += blockDim.x) {
        const int i = t / 3, k = t % 3;
        const int fw = k == 0 ? 0 : nw + (k - 1);
        uint32_t* row = buf + (size_t)(HR + i) * wp;
        row[fw] = halo_word(row, fw, n, nw);
    }
    __syncthreads();
    for (int t = threadIdx.x; t < 2 * HR * wp; t += blockDim.x) {
        const int band = t / wp, w = t % wp;
        const int r = band < HR ? band : n + band;
        const int src = HR + (((r - HR) % n) + n) % n;
        buf[(size_t)r * wp + w] = buf[(size_t)src * wp + w];
    }
    __syncthreads();
}

template <int R>
__global__ void __launch_bounds__(kResThreads, 1)
k_batch_resident(const uint32_t* __restrict__ src, uint32_t* __restrict__ dst, const BatchGrid* __restrict__ grids,
                 const int* __restrict__ list, int n_list, int steps, const __grid_constant__ PackedRule pr) {
    constexpr int PH = bits_for(2 * R + 1);
    constexpr int PB = bits_for((2 * R + 1) * (2 * R + 1));
    extern __shared__ uint32_t sm[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int li = blockIdx.x; li < n_list; li += gridDim.x) {
        const BatchGrid g = grids[list[li]];
        const int rows = g.n + 2 * g.HR;
        uint32_t* bufA = sm;
        uint32_t* bufB = sm + (size_t)rows * g.wp;
        // inner words in, halos built in shared memory
        for (int t = threadIdx.x; t < g.n * g.nw; t += blockDim.x) {
            const int i = t / g.nw, w = t % g.nw;
            bufA[(size_t)(g.HR + i) * g.wp + 1 + w] = src[g.off + (size_t)(g.HR + i) * g.wp + 1 + w];
        }
        __syncthreads();
        smem_halo(bufA, g.n, g.nw, g.HR, g.wp);
        // work split: every warp owns a band of rows of one 32-word strip
        const int strips = (g.nw + 31) / 32;
        const int warps = blockDim.x >> 5;
        const int bands = max(1, warps / strips);
        const int band_rows = (g.n + bands - 1) / bands;
        for (int s = 0; s < steps; ++s) {
            for (int it = wid; it < strips * bands; it += warps) {
                const int ws = it % strips, band = it / strips;
                const int r0 = band * band_rows, r1 = min(r0 + band_rows, g.n);
                if (r0 >= r1) continue;  // warp-uniform
                const int w = ws * 32 + lane;
                const bool active = w <= g.nw, outputs = w < g.nw;
                const int fw = 1 + w;
                auto rowp = [&](int r) { return bufA + (size_t)(g.HR + r) * g.wp; };
                uint32_t B[PB];
#pragma unroll
                for (int i = 0; i < PB; ++i) B[i] = 0u;
#pragma unroll 1
                for (int dy = -R; dy <= R; ++dy) {
                    uint32_t h[PH];
                    hcount<R, PH, false>(rowp(r0 + dy), fw, active, lane, h);
                    planes_add<PB, PH>(B, h);
                }
#pragma unroll 1
                for (int r = r0; r < r1; ++r) {
                    if (outputs) {
                        const uint32_t sv = rowp(r)[fw];
                        const uint32_t in1 = planes_in<PB>(B, pr.lo[1], pr.hi[1]) & pr.keep[1];
                        const uint32_t in0 = planes_in<PB>(B, pr.lo[0], pr.hi[0]) & pr.keep[0];
                        bufB[(size_t)(g.HR + r) * g.wp + fw] = (sv & in1) | (~sv & in0);
                    }
                    if (r + 1 < r1) {
                        uint32_t h[PH];
                        hcount<R, PH, false>(rowp(r - R), fw, active, lane, h);
                        planes_sub<PB, PH>(B, h);
                        hcount<R, PH, false>(rowp(r + R + 1), fw, active, lane, h);
                        planes_add<PB, PH>(B, h);
                    }
                }
            }
            __syncthreads();
            smem_halo(bufB, g.n, g.nw, g.HR, g.wp);
            uint32_t* t = bufA;
            bufA = bufB;
            bufB = t;
        }
        for (int t = threadIdx.x; t < g.n * g.nw; t += blockDim.x) {
            const int i = t / g.nw, w = t % g.nw;
            dst[g.off + (size_t)(g.HR + i) * g.wp + 1 + w] = bufA[(size_t)(g.HR + i) * g.wp + 1 + w];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Persistent kernel: one launch advances every grid of the batch through all
// the generations of one ltl_batch_step.  A CTA takes whole grids from a device
// counter, the most work first, and runs a grid's generations back to back with
// CTA barriers between them, so the grid stays in this SM's L1 and the L2 for
// the whole run (temporal blocking of the run) and no per-generation launch or
// halo launch is made.  The grid's radius selects the band walk (a switch over
// the compiled radii) and its rule class the comparator masks, which are loaded
// once per grid.  Rows of fewer than 32 words are handled by segments of a warp
// working on different row bands.
// ---------------------------------------------------------------------------
constexpr int kPersistWarps = 8;

// Halo of one frame in global memory, by the whole CTA: the column words of
// every inner row, then the top and bottom halo rows (copies of whole frame
// rows, their column words included).  Plain loads: the CTA reads what it
// wrote before the barrier.
__device__ void frame_halo_cta(uint32_t* f, const BatchGrid& g) {
    for (int i = threadIdx.x; i < g.n; i += blockDim.x) halo_cols_row(f + (size_t)(g.HR + i) * g.wp, g.n, g.nw);
    __syncthreads();
    const int total = 2 * g.HR * g.wp;
    for (int t = threadIdx.x; t < total; t += blockDim.x) {
        const int band = t / g.wp, w = t % g.wp;
        const int r = band < g.HR ? band : g.n + band;
        const int src = g.HR + (((r - g.HR) % g.n) + g.n) % g.n;
        f[(size_t)r * g.wp + w] = f[(size_t)src * g.wp + w];
    }
    __syncthreads();
}

// All generations of one grid by the whole CTA (radius R).
template <int R>
__device__ void persist_grid(const BatchGrid& g, uint32_t* a0, uint32_t* a1, int steps, const PackedRule& rule,
                             uint32_t* ring_all) {
    using Ring = PackedRing<R, kPersistWarps>;
    const PackedRule pr = rule;  // the masks the comparators use, kept in registers
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t* ring_lane = ring_all + (size_t)wid * Ring::WARP_WORDS + lane;
    uint32_t* f0 = a0 + g.off;
    uint32_t* f1 = a1 + g.off;
    frame_halo_cta(f0, g);
    // lanes per segment: the row's words rounded up to a power of two, at most 32
    const int seg = g.nw >= 32 ? 32 : (g.nw <= 1 ? 1 : 1 << (32 - __clz(g.nw - 1)));
    const int ns = 32 / seg;  // segments per warp
    const int strips = (g.nw + seg - 1) / seg;
    // enough bands for every segment of the CTA, none shorter than 2 (2R + 1)
    // rows (a band first counts 2R + 1 rows to start its window)
    const int want = max(1, kPersistWarps * ns / strips);
    const int band_rows = min(g.n, max((g.n + want - 1) / want, 4 * R + 2));
    const int bands = (g.n + band_rows - 1) / band_rows;
    const int items = strips * bands;
    const int wl = lane & (seg - 1), sidx = lane / seg;
    for (int s = 0; s < steps; ++s) {
        const uint32_t* src = (s & 1) ? f1 : f0;
        uint32_t* dst = (s & 1) ? f0 : f1;
        for (int base = wid * ns; base < items; base += kPersistWarps * ns) {  // warp-uniform
            const int item = base + sidx;
            const bool valid = item < items;
            const int strip = valid ? item % strips : 0;
            const int band = valid ? item / strips : 0;
            const int r0 = band * band_rows, r1 = min(r0 + band_rows, g.n);
            const int w = strip * seg + wl;
            const bool active = valid && w < g.nw;
            packed_band_seg<R, Ring::fits>(src, dst, (size_t)g.wp, g.HR, r0, r1, band_rows, 1 + w, active, wl == 0,
                                           wl == seg - 1 || w == g.nw - 1, ring_lane, pr);
        }
        __syncthreads();
        frame_halo_cta(dst, g);
    }
}

__global__ void __launch_bounds__(kPersistWarps * 32)
k_batch_persist(uint32_t* a0, uint32_t* a1, const BatchGrid* __restrict__ grids, const PackedRule* __restrict__ rules,
                const int* __restrict__ order, int n_order, int* next, int steps) {
    extern __shared__ uint32_t ring_all[];
    __shared__ int s_item;
    while (true) {
        if (threadIdx.x == 0) s_item = atomicAdd(next, 1);
        __syncthreads();
        const int li = s_item;
        __syncthreads();  // every thread has read s_item before it is overwritten
        if (li >= n_order) break;
        const BatchGrid g = grids[order[li]];
        switch (g.R) {
#define LTL_C(r) \
    case r: persist_grid<r>(g, a0, a1, steps, rules[g.cls], ring_all); break;
            LTL_BATCH_RADII(LTL_C)
#undef LTL_C
            default: break;
        }
    }
}

// Shared memory of the persistent kernel for a batch whose largest radius is R:
// 8 warps' h rings when they fit (else the walk counts leaving rows again).
template <int R>
static size_t persist_ring_bytes() {
    using Ring = PackedRing<R, kPersistWarps>;
    return Ring::fits ? (size_t)Ring::BYTES : 0;
}

// ---------------------------------------------------------------------------
// Dense staging <-> arena (all grids of a list, or one grid)
// ---------------------------------------------------------------------------
__global__ void k_batch_pack(const uint8_t* __restrict__ cells, uint32_t* __restrict__ arena,
                             const BatchGrid* __restrict__ grids, int first) {
    const BatchGrid g = grids[first + blockIdx.y];
    const uint8_t* c = cells + g.cell_off;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < g.n * g.nw; t += gridDim.x * blockDim.x) {
        const int i = t / g.nw, w = t % g.nw;
        uint32_t v = 0u;
        for (int b = 0; b < 32 && 32 * w + b < g.n; ++b) v |= (uint32_t)(c[(size_t)i * g.n + 32 * w + b] ? 1u : 0u) << b;
        arena[g.off + (size_t)(g.HR + i) * g.wp + 1 + w] = v;
    }
}

__global__ void k_batch_unpack(const uint32_t* __restrict__ arena, uint8_t* __restrict__ cells,
                               const BatchGrid* __restrict__ grids, int first) {
    const BatchGrid g = grids[first + blockIdx.y];
    uint8_t* c = cells + g.cell_off;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < g.n * g.nw; t += gridDim.x * blockDim.x) {
        const int i = t / g.nw, w = t % g.nw;
        const uint32_t v = arena[g.off + (size_t)(g.HR + i) * g.wp + 1 + w];
        for (int b = 0; b < 32 && 32 * w + b < g.n; ++b) c[(size_t)i * g.n + 32 * w + b] = (uint8_t)((v >> b) & 1u);
    }
}

// ---------------------------------------------------------------------------
// Launch helpers per radius (R <= 32 in the packed representation)
// ---------------------------------------------------------------------------
template <int R>
static size_t res_smem_bytes(int n) {
    const int nw = (n + 31) / 32;
    const int wp = (nw + 3 + 3) / 4 * 4;
    return 2ull * (size_t)(n + 2 * (R + 1)) * wp * 4;
}

template <int R>
static cudaError_t launch_batch_step_r(const uint32_t* cur, uint32_t* nxt, const BatchGrid* grids, const int4* items,
                                       int n_items, const PackedRule& pr, int sms, cudaStream_t s) {
    using Ring = PackedRing<R, kBatchWarps>;
    const int smem = Ring::fits ? Ring::BYTES : 0;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_step<R>, kBatchWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    const int ctas = std::max(1, std::min((n_items + kBatchWarps - 1) / kBatchWarps, sms * per_sm));
    k_batch_step<R><<<ctas, kBatchWarps * 32, smem, s>>>(cur, nxt, grids, items, n_items, pr);
    return cudaGetLastError();
}

// Shared-memory limit of the streamed step kernel (its h ring), set once per
// radius outside any stream capture.
template <int R>
static cudaError_t prepare_batch_step_r() {
    using Ring = PackedRing<R, kBatchWarps>;
    if (!Ring::fits || Ring::BYTES <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(k_batch_step<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, Ring::BYTES);
}

template <int R>
static cudaError_t launch_batch_resident_r(const uint32_t* src, uint32_t* dst, const BatchGrid* grids, const int* list,
                                           int n_list, int steps, const PackedRule& pr, size_t smem, int sms,
                                           cudaStream_t s) {
    const int ctas = std::max(1, std::min(n_list, sms));
    k_batch_resident<R><<<ctas, kResThreads, smem, s>>>(src, dst, grids, list, n_list, steps, pr);
    return cudaGetLastError();
}

static cudaError_t batch_step_dispatch(int R, const uint32_t* cur, uint32_t* nxt, const BatchGrid* grids,
                                       const int4* items, int n_items, const PackedRule& pr, int sms, cudaStream_t s) {
    switch (R) {
#define LTL_C(r) \
    case r: return launch_batch_step_r<r>(cur, nxt, grids, items, n_items, pr, sms, s);
        LTL_BATCH_RADII(LTL_C)
#undef LTL_C
        default: return cudaErrorInvalidValue;
    }
}

static cudaError_t batch_resident_dispatch(int R, const uint32_t* src, uint32_t* dst, const BatchGrid* grids,
                                           const int* list, int n_list, int steps, const PackedRule& pr, size_t smem,
                                           int sms, cudaStream_t s) {
    switch (R) {
#define LTL_C(r) \
    case r: return launch_batch_resident_r<r>(src, dst, grids, list, n_list, steps, pr, smem, sms, s);
        LTL_BATCH_RADII(LTL_C)
#undef LTL_C
        default: return cudaErrorInvalidValue;
    }
}

template <int R>
static cudaError_t prepare_resident_r(size_t smem) {
    return cudaFuncSetAttribute(k_batch_resident<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
}

static cudaError_t batch_step_prepare_dispatch(int R) {
    switch (R) {
#define LTL_BSP(r) \
    case r: return prepare_batch_step_r<r>();
        LTL_BATCH_RADII(LTL_BSP)
#undef LTL_BSP
        default: return cudaErrorInvalidValue;
    }
}

static cudaError_t batch_prepare_dispatch(int R, size_t smem) {
    switch (R) {
#define LTL_C(r) \
    case r: return prepare_resident_r<r>(smem);
        LTL_BATCH_RADII(LTL_C)
#undef LTL_C
        default: return cudaErrorInvalidValue;
    }
}

static size_t persist_ring_dispatch(int R) {
    switch (R) {
#define LTL_C(r) \
    case r: return persist_ring_bytes<r>();
        LTL_BATCH_RADII(LTL_C)
#undef LTL_C
        default: return 0;
    }
}

static size_t res_smem_dispatch(int R, int n) {
    switch (R) {
#define LTL_C(r) \
    case r: return res_smem_bytes<r>(n);
        LTL_BATCH_RADII(LTL_C)
#undef LTL_C
        default: return (size_t)-1;
    }
}

}  // namespace ltl

using namespace ltl;

struct BatchClass {
    Rule rule;
    PackedRule pr;
    std::vector<int> resident;   // grid ids kept in shared memory
    std::vector<int> streamed;   // grid ids streamed per step
    int* d_resident = nullptr;
    int4* d_items = nullptr;
    int n_items = 0;
    size_t res_smem = 0;
};

struct ltl_batch {
    int device = 0;
    int sms = 148;
    std::vector<BatchGrid> grids;
    std::vector<ltl_grid_desc> descs;
    std::vector<BatchClass> classes;
    std::vector<int> cls_id;
    int stream_band_rows = 64;
    long long resident_max = 0;
    BatchGrid* d_grids = nullptr;
    int* d_streamed_all = nullptr;
    int n_streamed_all = 0;
    uint32_t* arena[2] = {nullptr, nullptr};
    size_t arena_words = 0;
    uint8_t* staging = nullptr;
    long long total_cells = 0;
    bool cur_is_a = true;
    bool no_graph = false;
    bool persistent = true;
    // persistent mode: every grid, the most work first; the CTAs' grid counter;
    // the rule classes' comparator masks
    int* d_order = nullptr;
    int n_order = 0;
    int* d_next = nullptr;
    PackedRule* d_rules = nullptr;
    int persist_ctas = 0;
    size_t persist_smem = 0;
    cudaStream_t own = nullptr, stream = nullptr, aux = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
    // graph cache: (steps, parity) -> exec
    std::map<std::pair<int, int>, cudaGraphExec_t> graphs;
};

static void batch_release(ltl_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    for (auto& c : b->classes) {
        if (c.d_resident) cudaFree(c.d_resident);
        if (c.d_items) cudaFree(c.d_items);
    }
    if (b->d_next) cudaFree(b->d_next);
    if (b->d_order) cudaFree(b->d_order);
    if (b->d_rules) cudaFree(b->d_rules);
    if (b->d_grids) cudaFree(b->d_grids);
    if (b->d_streamed_all) cudaFree(b->d_streamed_all);
    for (auto& a : b->arena)
        if (a) cudaFree(a);
    if (b->staging) cudaFree(b->staging);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->join) cudaEventDestroy(b->join);
    if (b->aux) cudaStreamDestroy(b->aux);
    if (b->own) cudaStreamDestroy(b->own);
    delete b;
}

#define BATCH_CUDA(call)                                                                           \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            ltl_set_error("%s failed: %s", #call, cudaGetErrorString(e_));                         \
            return e_ == cudaErrorMemoryAllocation ? LTL_ENOMEM : LTL_ECUDA;                       \
        }                                                                                          \
    } while (0)

static uint32_t* cur_arena(ltl_batch* b);
static cudaError_t refresh_streamed_halo(ltl_batch* b, uint32_t* arena, cudaStream_t s);

// Work plan: which grids are resident, and the streamed work lists.  Rebuilt
// when a shape parameter changes (the arenas' layout does not depend on it).
static int batch_plan(ltl_batch* b) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    for (auto& c : b->classes) {
        if (c.d_resident) cudaFree(c.d_resident);
        if (c.d_items) cudaFree(c.d_items);
        c.d_resident = nullptr;
        c.d_items = nullptr;
        c.resident.clear();
        c.streamed.clear();
        c.n_items = 0;
        c.res_smem = 0;
    }
    if (b->d_order) cudaFree(b->d_order);
    b->d_order = nullptr;
    b->n_order = 0;
    if (b->d_streamed_all) cudaFree(b->d_streamed_all);
    b->d_streamed_all = nullptr;
    b->n_streamed_all = 0;
    const int count = (int)b->grids.size();
    if (b->persistent) {
        // one list of every grid, the most work first (cells x a cost that grows
        // with R), which the CTAs of the one launch take in order
        std::vector<int> order(count);
        size_t smem = 0;
        for (int i = 0; i < count; ++i) {
            order[i] = i;
            smem = std::max(smem, persist_ring_dispatch(b->grids[i].R));
        }
        auto cost = [&](int i) { return (double)b->grids[i].n * b->grids[i].n * (4.0 + b->grids[i].R); };
        std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
        // always raised: the kernel's own static shared memory counts against the default 48 KiB too
        BATCH_CUDA(cudaFuncSetAttribute(k_batch_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per_sm = 0;
        BATCH_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_persist, kPersistWarps * 32, smem));
        b->persist_smem = smem;
        b->persist_ctas = std::max(1, std::min(count, b->sms * std::max(per_sm, 1)));
        b->n_order = count;
        BATCH_CUDA(cudaMalloc(&b->d_order, sizeof(int) * count));
        BATCH_CUDA(cudaMemcpy(b->d_order, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice));
        return LTL_OK;
    }
    std::vector<int> streamed_all;
    for (int i = 0; i < count; ++i) {
        BatchClass& c = b->classes[b->cls_id[i]];
        const size_t need = res_smem_dispatch(b->grids[i].R, b->grids[i].n);
        if (need <= (size_t)b->resident_max) {
            c.resident.push_back(i);
            c.res_smem = std::max(c.res_smem, need);
        } else {
            c.streamed.push_back(i);
            streamed_all.push_back(i);
        }
    }
    b->n_streamed_all = (int)streamed_all.size();
    if (!streamed_all.empty()) {
        BATCH_CUDA(cudaMalloc(&b->d_streamed_all, sizeof(int) * streamed_all.size()));
        BATCH_CUDA(cudaMemcpy(b->d_streamed_all, streamed_all.data(), sizeof(int) * streamed_all.size(),
                              cudaMemcpyHostToDevice));
    }
    // one shared-memory limit per kernel instantiation (radius): the largest any class of that radius needs
    std::map<int, size_t> smem_by_radius;
    for (auto& c : b->classes)
        if (!c.resident.empty()) smem_by_radius[c.rule.radius] = std::max(smem_by_radius[c.rule.radius], c.res_smem);
    for (auto& kv : smem_by_radius) BATCH_CUDA(batch_prepare_dispatch(kv.first, kv.second));
    for (auto& c : b->classes)
        if (!c.streamed.empty()) BATCH_CUDA(batch_step_prepare_dispatch(c.rule.radius));
    for (auto& c : b->classes) {
        if (!c.resident.empty()) {
            BATCH_CUDA(cudaMalloc(&c.d_resident, sizeof(int) * c.resident.size()));
            BATCH_CUDA(cudaMemcpy(c.d_resident, c.resident.data(), sizeof(int) * c.resident.size(),
                                  cudaMemcpyHostToDevice));
        }
        std::vector<int4> items;
        for (int gi : c.streamed) {
            const BatchGrid& g = b->grids[gi];
            const int strips = (g.nw + 31) / 32;
            const int band_rows = b->stream_band_rows;
            for (int r0 = 0; r0 < g.n; r0 += band_rows)
                for (int ws = 0; ws < strips; ++ws) items.push_back(make_int4(gi, r0, std::min(g.n, r0 + band_rows), ws));
        }
        c.n_items = (int)items.size();
        if (!items.empty()) {
            BATCH_CUDA(cudaMalloc(&c.d_items, sizeof(int4) * items.size()));
            BATCH_CUDA(cudaMemcpy(c.d_items, items.data(), sizeof(int4) * items.size(), cudaMemcpyHostToDevice));
        }
    }
    // the streamed kernels read halos that an upload made in persistent mode left unset
    if (b->stream && b->arena[0]) {
        BATCH_CUDA(refresh_streamed_halo(b, cur_arena(b), b->stream));
        BATCH_CUDA(cudaStreamSynchronize(b->stream));
    }
    return LTL_OK;
}

static int batch_build(ltl_batch* b, int flags) {
    const int count = (int)b->descs.size();
    // rule classes
    std::map<std::vector<int>, int> cls_of;
    size_t words = 0;
    long long cells = 0;
    b->grids.resize(count);
    b->cls_id.resize(count);
    int rmax = 1;
    for (int i = 0; i < count; ++i) {
        const ltl_grid_desc& d = b->descs[i];
        std::vector<int> key = {d.radius, d.smin, d.smax, d.bmin, d.bmax};
        auto it = cls_of.find(key);
        if (it == cls_of.end()) {
            BatchClass c;
            c.rule = Rule{d.radius, d.smin, d.smax, d.bmin, d.bmax};
            c.pr = make_packed_rule(c.rule);
            it = cls_of.emplace(key, (int)b->classes.size()).first;
            b->classes.push_back(c);
        }
        b->cls_id[i] = it->second;
        BatchGrid g{};
        g.n = d.n;
        g.nw = (d.n + 31) / 32;
        g.HR = d.radius + 1;
        g.wp = (g.nw + 3 + 3) / 4 * 4;
        g.R = d.radius;
        g.off = (long long)words;
        g.cell_off = cells;
        words += (size_t)(g.n + 2 * g.HR) * g.wp;
        words = (words + 31) / 32 * 32;
        cells += (long long)g.n * g.n;
        g.cls = it->second;
        b->grids[i] = g;
        rmax = std::max(rmax, d.radius);
    }
    b->arena_words = words + 64;
    b->total_cells = cells;
    b->stream_band_rows = (int)tuning_lookup("batch", -1, 0, "stream_band_rows", 64);
    b->resident_max = (flags & LTL_BATCH_STREAM_ALL) ? 0
                                                     : tuning_lookup("batch", -1, 0, "resident_max_bytes", kResSmemLimit);
    b->persistent = !(flags & LTL_BATCH_STREAM_ALL) && tuning_lookup("batch", -1, 0, "persistent", 1) != 0;
    BATCH_CUDA(cudaMalloc(&b->d_next, sizeof(int)));
    {
        std::vector<PackedRule> rules;
        for (auto& c : b->classes) rules.push_back(c.pr);
        BATCH_CUDA(cudaMalloc(&b->d_rules, sizeof(PackedRule) * rules.size()));
        BATCH_CUDA(cudaMemcpy(b->d_rules, rules.data(), sizeof(PackedRule) * rules.size(), cudaMemcpyHostToDevice));
    }
    BATCH_CUDA(cudaMalloc(&b->d_grids, sizeof(BatchGrid) * count));
    BATCH_CUDA(cudaMemcpy(b->d_grids, b->grids.data(), sizeof(BatchGrid) * count, cudaMemcpyHostToDevice));
    for (auto& a : b->arena) {
        BATCH_CUDA(cudaMalloc(&a, b->arena_words * sizeof(uint32_t)));
        BATCH_CUDA(cudaMemset(a, 0, b->arena_words * sizeof(uint32_t)));
    }
    BATCH_CUDA(cudaMalloc(&b->staging, (size_t)std::max<long long>(cells, 1)));
    return batch_plan(b);
}

extern "C" int ltl_batch_set_param(ltl_batch* b, const char* name, long long value) {
    if (!b || !name) {
        ltl_set_error("ltl_batch_set_param: bad arguments");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    if (std::strcmp(name, "stream_band_rows") == 0) {
        if (value < 8 || value > 4096) {
            ltl_set_error("ltl_batch_set_param: stream_band_rows must be in [8, 4096]");
            return LTL_EINVAL;
        }
        b->stream_band_rows = (int)value;
    } else if (std::strcmp(name, "persistent") == 0) {
        if (value != 0 && value != 1) {
            ltl_set_error("ltl_batch_set_param: persistent must be 0 or 1");
            return LTL_EINVAL;
        }
        b->persistent = value != 0;
    } else if (std::strcmp(name, "resident_max_bytes") == 0) {
        if (value < 0 || value > kResSmemLimit) {
            ltl_set_error("ltl_batch_set_param: resident_max_bytes must be in [0, %d]", kResSmemLimit);
            return LTL_EINVAL;
        }
        b->resident_max = value;
    } else {
        ltl_set_error("ltl_batch_set_param: unknown parameter '%s'", name);
        return LTL_EINVAL;
    }
    return batch_plan(b);
}

extern "C" int ltl_batch_create(ltl_batch** out, int device, const ltl_grid_desc* descs, int count, int flags) {
    if (!out || !descs || count < 1) {
        ltl_set_error("ltl_batch_create: bad arguments");
        return LTL_EINVAL;
    }
    *out = nullptr;
    for (int i = 0; i < count; ++i) {
        const ltl_grid_desc& d = descs[i];
        if (d.n < 1 || d.radius < 1 || d.n < d.radius) {
            ltl_set_error("ltl_batch_create: grid %d: need n >= radius >= 1 (n=%d, radius=%d)", i, d.n, d.radius);
            return LTL_EINVAL;
        }
        if (d.radius > 16) {
            ltl_set_error("ltl_batch_create: grid %d: batched grids support radius <= 16 (got %d)", i, d.radius);
            return LTL_EUNSUPPORTED;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        ltl_set_error("ltl_batch_create: CUDA device %d not available", device);
        return LTL_ECUDA;
    }
    ltl_batch* b = new (std::nothrow) ltl_batch();
    if (!b) return LTL_ENOMEM;
    b->device = device;
    b->descs.assign(descs, descs + count);
    cudaSetDevice(device);
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    cudaError_t se = cudaStreamCreateWithFlags(&b->own, cudaStreamNonBlocking);
    if (se == cudaSuccess) se = cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking);
    if (se == cudaSuccess) se = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (se == cudaSuccess) se = cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming);
    if (se != cudaSuccess) {
        ltl_set_error("ltl_batch_create: stream/event creation failed: %s", cudaGetErrorString(se));
        batch_release(b);
        return LTL_ECUDA;
    }
    b->stream = b->own;
    b->no_graph = (flags & LTL_BATCH_NO_GRAPH) != 0;
    int rc = batch_build(b, flags);
    if (rc != LTL_OK) {
        batch_release(b);
        return rc;
    }
    *out = b;
    return LTL_OK;
}

extern "C" int ltl_batch_destroy(ltl_batch* b) {
    if (!b) return LTL_OK;
    cudaSetDevice(b->device);
    cudaStreamSynchronize(b->stream);
    batch_release(b);
    return LTL_OK;
}

extern "C" int ltl_batch_set_stream(ltl_batch* b, void* stream) {
    if (!b) {
        ltl_set_error("null batch");
        return LTL_EINVAL;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : b->own;
    if (s != b->stream) {
        for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
        b->graphs.clear();
    }
    b->stream = s;
    return LTL_OK;
}

static uint32_t* cur_arena(ltl_batch* b) { return b->arena[b->cur_is_a ? 0 : 1]; }
static uint32_t* nxt_arena(ltl_batch* b) { return b->arena[b->cur_is_a ? 1 : 0]; }

static cudaError_t refresh_streamed_halo(ltl_batch* b, uint32_t* arena, cudaStream_t s) {
    if (b->n_streamed_all == 0) return cudaSuccess;
    // one block row per grid; launches of at most 65535 grids (the grid-y limit)
    for (int first = 0; first < b->n_streamed_all; first += 65535) {
        dim3 g1(8, (unsigned)std::min(65535, b->n_streamed_all - first));
        k_batch_halo_cols<<<g1, 128, 0, s>>>(arena, b->d_grids, b->d_streamed_all + first);
        k_batch_halo_rows<<<g1, 128, 0, s>>>(arena, b->d_grids, b->d_streamed_all + first);
    }
    return cudaGetLastError();
}

extern "C" int ltl_batch_upload_all(ltl_batch* b, const uint8_t* cells) {
    if (!b || !cells) {
        ltl_set_error("ltl_batch_upload_all: bad arguments");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    BATCH_CUDA(cudaMemcpyAsync(b->staging, cells, (size_t)b->total_cells, cudaMemcpyHostToDevice, b->stream));
    const int count = (int)b->grids.size();
    for (int first = 0; first < count; first += 65535) {
        dim3 g(16, (unsigned)std::min(65535, count - first));
        k_batch_pack<<<g, 256, 0, b->stream>>>(b->staging, cur_arena(b), b->d_grids, first);
    }
    BATCH_CUDA(cudaGetLastError());
    BATCH_CUDA(refresh_streamed_halo(b, cur_arena(b), b->stream));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return LTL_OK;
}

extern "C" int ltl_batch_download_all(ltl_batch* b, uint8_t* cells) {
    if (!b || !cells) {
        ltl_set_error("ltl_batch_download_all: bad arguments");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    const int count = (int)b->grids.size();
    for (int first = 0; first < count; first += 65535) {
        dim3 g(16, (unsigned)std::min(65535, count - first));
        k_batch_unpack<<<g, 256, 0, b->stream>>>(cur_arena(b), b->staging, b->d_grids, first);
    }
    BATCH_CUDA(cudaGetLastError());
    BATCH_CUDA(cudaMemcpyAsync(cells, b->staging, (size_t)b->total_cells, cudaMemcpyDeviceToHost, b->stream));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return LTL_OK;
}

extern "C" int ltl_batch_upload(ltl_batch* b, int grid, const uint8_t* inner, size_t pitch) {
    if (!b || !inner || grid < 0 || grid >= (int)b->grids.size() || pitch < (size_t)b->grids[grid].n) {
        ltl_set_error("ltl_batch_upload: bad arguments");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    const BatchGrid& g = b->grids[grid];
    BATCH_CUDA(cudaMemcpy2DAsync(b->staging + g.cell_off, g.n, inner, pitch, g.n, g.n, cudaMemcpyHostToDevice,
                                 b->stream));
    k_batch_pack<<<dim3(16, 1), 256, 0, b->stream>>>(b->staging, cur_arena(b), b->d_grids, grid);
    BATCH_CUDA(cudaGetLastError());
    BATCH_CUDA(refresh_streamed_halo(b, cur_arena(b), b->stream));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return LTL_OK;
}

extern "C" int ltl_batch_download(ltl_batch* b, int grid, uint8_t* inner, size_t pitch) {
    if (!b || !inner || grid < 0 || grid >= (int)b->grids.size() || pitch < (size_t)b->grids[grid].n) {
        ltl_set_error("ltl_batch_download: bad arguments");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    const BatchGrid& g = b->grids[grid];
    k_batch_unpack<<<dim3(16, 1), 256, 0, b->stream>>>(cur_arena(b), b->staging, b->d_grids, grid);
    BATCH_CUDA(cudaGetLastError());
    BATCH_CUDA(cudaMemcpy2DAsync(inner, pitch, b->staging + g.cell_off, g.n, g.n, g.n, cudaMemcpyDeviceToHost,
                                 b->stream));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return LTL_OK;
}

// Enqueue `steps` generations of every grid (stream-ordered on b->stream).
// On failure, `what` names the call that failed.
static cudaError_t enqueue_steps(ltl_batch* b, int steps, const char** what) {
    cudaError_t e = cudaSuccess;
    uint32_t* a0 = cur_arena(b);
    uint32_t* a1 = nxt_arena(b);
    if (b->persistent) {
        *what = "grid counter reset";
        e = cudaMemsetAsync(b->d_next, 0, sizeof(int), b->stream);
        if (e == cudaSuccess) {
            *what = "persistent kernel launch";
            k_batch_persist<<<b->persist_ctas, kPersistWarps * 32, b->persist_smem, b->stream>>>(
                a0, a1, b->d_grids, b->d_rules, b->d_order, b->n_order, b->d_next, steps);
            e = cudaGetLastError();
        }
        return e;
    }
    bool any_res = false;
    for (auto& c : b->classes) any_res |= !c.resident.empty();
    if (any_res) {
        *what = "fork event record";
        e = cudaEventRecord(b->fork, b->stream);
        if (e == cudaSuccess) {
            *what = "fork stream wait";
            e = cudaStreamWaitEvent(b->aux, b->fork, 0);
        }
        uint32_t* dst = (steps % 2) ? a1 : a0;
        for (auto& c : b->classes) {
            if (c.resident.empty() || e != cudaSuccess) continue;
            *what = "resident kernel launch";
            e = batch_resident_dispatch(c.rule.radius, a0, dst, b->d_grids, c.d_resident, (int)c.resident.size(),
                                        steps, c.pr, c.res_smem, b->sms, b->aux);
        }
        if (e == cudaSuccess) {
            *what = "join event record";
            e = cudaEventRecord(b->join, b->aux);
        }
    }
    for (int s = 0; s < steps && e == cudaSuccess; ++s) {
        const uint32_t* src = (s % 2) ? a1 : a0;
        uint32_t* dst = (s % 2) ? a0 : a1;
        for (auto& c : b->classes) {
            if (c.n_items == 0 || e != cudaSuccess) continue;
            *what = "streamed step kernel launch";
            e = batch_step_dispatch(c.rule.radius, src, dst, b->d_grids, c.d_items, c.n_items, c.pr, b->sms,
                                    b->stream);
        }
        if (e == cudaSuccess) {
            *what = "halo kernel launch";
            e = refresh_streamed_halo(b, dst, b->stream);
        }
    }
    if (any_res && e == cudaSuccess) {
        *what = "join stream wait";
        e = cudaStreamWaitEvent(b->stream, b->join, 0);
    }
    return e;
}

extern "C" int ltl_batch_step(ltl_batch* b, int steps) {
    if (!b || steps < 0) {
        ltl_set_error("ltl_batch_step: bad arguments");
        return LTL_EINVAL;
    }
    if (steps == 0) return LTL_OK;
    BATCH_CUDA(cudaSetDevice(b->device));
    const char* what = "";
    if (b->no_graph) {
        cudaError_t e = enqueue_steps(b, steps, &what);
        if (e != cudaSuccess) {
            ltl_set_error("ltl_batch_step: %s failed: %s", what, cudaGetErrorString(e));
            return LTL_ECUDA;
        }
        if (steps % 2) b->cur_is_a = !b->cur_is_a;
        return LTL_OK;
    }
    const std::pair<int, int> key(steps, b->cur_is_a ? 0 : 1);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        cudaGraph_t g = nullptr;
        BATCH_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = enqueue_steps(b, steps, &what);
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            ltl_set_error("ltl_batch_step: graph capture failed at %s: %s / end capture: %s", what,
                          cudaGetErrorString(e), cudaGetErrorString(e2));
            cudaGetLastError();
            return LTL_ECUDA;
        }
        cudaGraphExec_t ex = nullptr;
        cudaError_t e3 = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e3 != cudaSuccess) {
            ltl_set_error("ltl_batch_step: graph instantiate failed: %s", cudaGetErrorString(e3));
            return LTL_ECUDA;
        }
        it = b->graphs.emplace(key, ex).first;
    }
    BATCH_CUDA(cudaGraphLaunch(it->second, b->stream));
    if (steps % 2) b->cur_is_a = !b->cur_is_a;
    return LTL_OK;
}

extern "C" int ltl_batch_synchronize(ltl_batch* b) {
    if (!b) {
        ltl_set_error("null batch");
        return LTL_EINVAL;
    }
    BATCH_CUDA(cudaSetDevice(b->device));
    BATCH_CUDA(cudaStreamSynchronize(b->stream));
    return LTL_OK;
}

extern "C" int ltl_batch_info(const ltl_batch* b, long long* cells, long long* device_bytes, int* temporal_depth) {
    if (!b) {
        ltl_set_error("null batch");
        return LTL_EINVAL;
    }
    if (cells) *cells = b->total_cells;
    if (device_bytes) *device_bytes = (long long)(2 * b->arena_words * 4 + b->total_cells);
    if (temporal_depth) {
        // grids that run every generation of an ltl_batch_step inside one launch
        int res = 0;
        if (b->persistent) res = (int)b->grids.size();
        else
            for (auto& c : b->classes) res += (int)c.resident.size();
        *temporal_depth = res;
    }
    return LTL_OK;
}

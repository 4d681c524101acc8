// k_packed.cu -- K3: bit-packed LtL step (one bit per cell) and the PACK codec.
//
// Same function as the reference's HostSolver<int> step (kezada94/CAT_cpu,
// src/CellularAutomata/Solvers/HostSolver.tpp:58-91, torus halo :93-140), with
// 32 cells per 32-bit word and the neighbour count kept bit-sliced:
//   h(row) = horizontal (2R+1)-window count of one row, as PH bit planes, by a
//            carry-save (Wallace) reduction of the 2R+1 shifted row words;
//   B      = vertical sliding sum of h over 2R+1 rows, as PB bit planes
//            (B -= h(r-R); B += h(r+R+1) while a thread walks down its band);
//   next   = s ? [smin+1 <= B <= smax+1] : [bmin <= B <= bmax]   (B includes the centre)
// evaluated with bit-sliced comparators.  Every operation acts on 32 cells.
//
// The PACK codec (ltl_pack_device / ltl_unpack_device) stores row i of a grid
// as ceil(cols/64) uint64 words, cell (i, j) = bit j % 64 of word j / 64.
#include <algorithm>

#include "packed_core.cuh"

namespace ltl {

constexpr int kPackedWarps = 4;

// Rows per work item when no tuned value applies: as few bands as fill every
// resident warp once (each band re-counts 2R+1 rows to start its window, so
// fewer, longer bands waste less), split further only where a band would be
// longer than 256 rows.
static int packed_band_rows(int n, int n_wstrips, int resident_warps) {
    const int per_wave = std::max(1, resident_warps / std::max(n_wstrips, 1));
    int bands = per_wave;
    while ((n + bands - 1) / bands > 256) bands += per_wave;
    return std::max(16, (n + bands - 1) / bands);
}

template <int R, bool FUSE>
__global__ void __launch_bounds__(kPackedWarps * 32)
k_packed_step(const uint32_t* __restrict__ cur, uint32_t* __restrict__ nxt, int rows, int nw, int HR, int HW,
              size_t wp, int n_wstrips, int n_items, int band_rows, const __grid_constant__ PackedRule pr) {
    using Ring = PackedRing<R, kPackedWarps>;
    extern __shared__ uint32_t ring_all[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    uint32_t* ring_lane = ring_all + (size_t)wid * Ring::WARP_WORDS + lane;
    const int gwarp = blockIdx.x * kPackedWarps + wid;
    const int gwarps = gridDim.x * kPackedWarps;

    for (int item = gwarp; item < n_items; item += gwarps) {
        const int ws = item % n_wstrips;
        const int band = item / n_wstrips;
        const int r0 = band * band_rows;
        const int r1 = min(r0 + band_rows, rows);
        const int w = ws * 32 + lane;     // inner word
        const bool active = w <= nw;      // w == nw is the right halo word (neighbour of the last word)
        const bool outputs = w < nw;
        packed_band<R, Ring::fits, FUSE>(cur, nxt, wp, HR, r0, r1, HW + w, active, outputs, lane, ring_lane, pr,
                                         rows, nw);
        __syncwarp();
    }
}

bool packed_supported(int n, int radius) { return radius >= 1 && radius <= 32 && n >= radius; }

// The step writes the output frame's halo itself (packed_band's kFuse) where
// every halo word is a whole inner word: n a multiple of 32, one halo word.
bool packed_fused_halo(const PackedFrame& f, int radius) {
    return f.HW == 1 && f.n % 32 == 0 && f.n >= 64 && f.nrows() >= 2 * radius + 2;
}

template <int R>
static cudaError_t launch_packed_r(const PackedFrame& c, const PackedFrame& x, const PackedRule& pr,
                                   int band_override, cudaStream_t s) {
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // strips of 32 words cover the inner words; a lane whose word is the right
    // halo word (w == nw) only feeds its left neighbour, and lane 31 loads the
    // word past its own directly, so no strip is needed for the halo alone
    const int n_wstrips = (c.nw + 31) / 32;
    const int smem = PackedRing<R, kPackedWarps>::fits ? PackedRing<R, kPackedWarps>::BYTES : 0;
    const bool fuse = packed_fused_halo(x, R);
    auto kernel = fuse ? k_packed_step<R, true> : k_packed_step<R, false>;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPackedWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    const int band_rows =
        band_override > 0 ? band_override : packed_band_rows(c.nrows(), n_wstrips, sms * per_sm * kPackedWarps);
    const int bands = (c.nrows() + band_rows - 1) / band_rows;
    const int items = n_wstrips * bands;
    int ctas = std::min((items + kPackedWarps - 1) / kPackedWarps, sms * per_sm);
    kernel<<<ctas, kPackedWarps * 32, smem, s>>>(c.words, x.words, c.nrows(), c.nw, c.HR, c.HW, c.wpitch,
                                                           n_wstrips, items, band_rows, pr);
    return cudaGetLastError();
}

template <int R>
static cudaError_t prepare_packed_r() {
    const int smem = PackedRing<R, kPackedWarps>::fits ? PackedRing<R, kPackedWarps>::BYTES : 0;
    if (smem <= 48 * 1024) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_packed_step<R, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_packed_step<R, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

cudaError_t packed_prepare(int radius) {
    switch (radius) {
#define LTL_PP(r) \
    case r: return prepare_packed_r<r>();
        LTL_PP(1) LTL_PP(2) LTL_PP(3) LTL_PP(4) LTL_PP(5) LTL_PP(6) LTL_PP(7) LTL_PP(8)
        LTL_PP(9) LTL_PP(10) LTL_PP(11) LTL_PP(12) LTL_PP(13) LTL_PP(14) LTL_PP(15) LTL_PP(16)
        LTL_PP(17) LTL_PP(18) LTL_PP(19) LTL_PP(20) LTL_PP(21) LTL_PP(22) LTL_PP(23) LTL_PP(24)
        LTL_PP(25) LTL_PP(26) LTL_PP(27) LTL_PP(28) LTL_PP(29) LTL_PP(30) LTL_PP(31) LTL_PP(32)
#undef LTL_PP
        default: return cudaSuccess;
    }
}

cudaError_t launch_packed_step(const PackedFrame& cur, const PackedFrame& nxt, const Rule& rule, int band_rows,
                               cudaStream_t s) {
    PackedRule pr = make_packed_rule(rule);
    switch (rule.radius) {
#define LTL_PR(r) \
    case r: return launch_packed_r<r>(cur, nxt, pr, band_rows, s);
        LTL_PR(1) LTL_PR(2) LTL_PR(3) LTL_PR(4) LTL_PR(5) LTL_PR(6) LTL_PR(7) LTL_PR(8)
        LTL_PR(9) LTL_PR(10) LTL_PR(11) LTL_PR(12) LTL_PR(13) LTL_PR(14) LTL_PR(15) LTL_PR(16)
        LTL_PR(17) LTL_PR(18) LTL_PR(19) LTL_PR(20) LTL_PR(21) LTL_PR(22) LTL_PR(23) LTL_PR(24)
        LTL_PR(25) LTL_PR(26) LTL_PR(27) LTL_PR(28) LTL_PR(29) LTL_PR(30) LTL_PR(31) LTL_PR(32)
#undef LTL_PR
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// Packed halo: column halo bits of inner rows (bit position p of the frame row
// holds cell (p - 32*HW) mod n), then whole top/bottom rows copied from the
// inner rows they wrap to.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t packed_bit(const uint32_t* row, int HW, int cell) {
    int p = 32 * HW + cell;
    return (row[p >> 5] >> (p & 31)) & 1u;
}

__global__ void k_packed_halo_cols(uint32_t* __restrict__ g, int n, int rows, int nw, int HR, int HW, size_t wp) {
    // per inner row: words [0, HW) and [HW + nw - 1, HW + nw + HW)
    const int per_row = 2 * HW + 1;
    const long long total = (long long)rows * per_row;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / per_row);
        const int k = (int)(t % per_row);
        const int fw = k < HW ? k : HW + nw - 1 + (k - HW);
        uint32_t* row = g + (size_t)(HR + i) * wp;
        auto slow = [&]() -> uint32_t {
            uint32_t v = 0u;
            if (fw == HW + nw - 1) {
                // last inner word: keep its inner bits, rewrite the bits past n
                const int inner_bits = n - 32 * (nw - 1);
                v = inner_bits >= 32 ? row[fw] : (row[fw] & ((1u << inner_bits) - 1u));
                for (int b = inner_bits; b < 32; ++b) {
                    int cell = 32 * (nw - 1) + b;
                    v |= packed_bit(row, HW, cell % n) << b;
                }
            } else {
                for (int b = 0; b < 32; ++b) {
                    int cell = 32 * (fw - HW) + b;
                    int src = ((cell % n) + n) % n;
                    v |= packed_bit(row, HW, src) << b;
                }
            }
            return v;
        };
        const uint32_t v = HW == 1 ? packed_halo_word(row, fw, n, nw, slow) : slow();
        // the halo words only read inner bits (< n), never bits written here
        row[fw] = v;
    }
}

__global__ void k_packed_halo_rows(uint32_t* __restrict__ g, int rows, int HR, size_t wp) {
    const int band = blockIdx.y;  // 0 .. 2HR-1
    const int r = band < HR ? band : rows + band;
    const int src = HR + (((r - HR) % rows) + rows) % rows;
    uint32_t* d = g + (size_t)r * wp;
    const uint32_t* sp = g + (size_t)src * wp;
    for (int w = blockIdx.x * blockDim.x + threadIdx.x; w < (int)wp; w += gridDim.x * blockDim.x) d[w] = sp[w];
}

cudaError_t launch_packed_halo(const PackedFrame& f, cudaStream_t s) {
    const long long total = (long long)f.nrows() * (2 * f.HW + 1);
    int blocks = (int)std::min<long long>((total + 127) / 128, 4096);
    k_packed_halo_cols<<<blocks, 128, 0, s>>>(f.words, f.n, f.nrows(), f.nw, f.HR, f.HW, f.wpitch);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    dim3 g2((unsigned)std::max<size_t>(1, std::min<size_t>((f.wpitch + 127) / 128, 64)), (unsigned)(2 * f.HR));
    k_packed_halo_rows<<<g2, 128, 0, s>>>(f.words, f.nrows(), f.HR, f.wpitch);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Byte frame <-> packed frame (inner cells only; halos are refilled after).
// ---------------------------------------------------------------------------
// Four 0/1 bytes of a word -> 4 bits: the multiply places byte k's bit at bit
// 24 + k with no two partial products overlapping (so no carries), and back:
// the 4 bits of a nibble spread to bit 0 of each byte by copies 7 bits apart.
__device__ __forceinline__ uint32_t bytes4_to_bits(uint32_t w) { return ((w & 0x01010101u) * 0x01020408u) >> 24; }
__device__ __forceinline__ uint32_t bits4_to_bytes(uint32_t nib) { return (nib * 0x00204081u) & 0x01010101u; }

// Inner rows [row0, row0 + nrows) of a packed frame from / to a dense byte
// buffer whose row i (`pitch` bytes apart, `src`/`dst` = its cell (0, 0)) is
// frame row row0 + i.  `vec`: buffer and pitch 16-byte aligned, so whole
// 32-cell words move as two 16-byte vectors.
__global__ void k_pack_rows(const uint8_t* __restrict__ src, size_t pitch, bool vec, int n, int nw, int HR, int HW,
                            size_t wp, int row0, int nrows, uint32_t* __restrict__ dst) {
    const long long total = (long long)nrows * nw;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        const uint8_t* p = src + (size_t)i * pitch + 32 * w;
        uint32_t v = 0u;
        if (vec && 32 * w + 32 <= n) {
            const uint4 a = *(const uint4*)p, b = *(const uint4*)(p + 16);
            const uint32_t q[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
            for (int k = 0; k < 8; ++k) v |= bytes4_to_bits(q[k]) << (4 * k);
        } else {
            for (int b = 0; b < 32 && 32 * w + b < n; ++b) v |= (uint32_t)(p[b] & 1u) << b;
        }
        dst[(size_t)(HR + row0 + i) * wp + HW + w] = v;
    }
}

__global__ void k_unpack_rows(const uint32_t* __restrict__ src, int n, int nw, int HR, int HW, size_t wp, int row0,
                              int nrows, uint8_t* __restrict__ dst, size_t pitch, bool vec) {
    const long long total = (long long)nrows * nw;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        const uint32_t v = src[(size_t)(HR + row0 + i) * wp + HW + w];
        uint8_t* p = dst + (size_t)i * pitch + 32 * w;
        if (vec && 32 * w + 32 <= n) {
            uint32_t q[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) q[k] = bits4_to_bytes((v >> (4 * k)) & 0xFu);
            *(uint4*)p = make_uint4(q[0], q[1], q[2], q[3]);
            *(uint4*)(p + 16) = make_uint4(q[4], q[5], q[6], q[7]);
        } else {
            for (int b = 0; b < 32 && 32 * w + b < n; ++b) p[b] = (uint8_t)((v >> b) & 1u);
        }
    }
}

static bool vec16(const void* p, size_t pitch) { return ((uintptr_t)p % 16 == 0) && (pitch % 16 == 0); }

cudaError_t launch_pack_rows(const uint8_t* src, size_t pitch, const PackedFrame& dst, int row0, int nrows,
                             cudaStream_t s) {
    if (nrows <= 0) return cudaSuccess;
    const long long total = (long long)nrows * dst.nw;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_pack_rows<<<blocks, 256, 0, s>>>(src, pitch, vec16(src, pitch), dst.n, dst.nw, dst.HR, dst.HW, dst.wpitch,
                                       row0, nrows, dst.words);
    return cudaGetLastError();
}

cudaError_t launch_unpack_rows(const PackedFrame& src, int row0, int nrows, uint8_t* dst, size_t pitch,
                               cudaStream_t s) {
    if (nrows <= 0) return cudaSuccess;
    const long long total = (long long)nrows * src.nw;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_unpack_rows<<<blocks, 256, 0, s>>>(src.words, src.n, src.nw, src.HR, src.HW, src.wpitch, row0, nrows, dst,
                                         pitch, vec16(dst, pitch));
    return cudaGetLastError();
}

// byte frame -> packed frame, inner cells only (halos are refilled after)
cudaError_t launch_pack_frame(const Frame& src, const PackedFrame& dst, cudaStream_t s) {
    return launch_pack_rows(src.base + (size_t)src.H * src.pitch + src.H, src.pitch, dst, 0, dst.nrows(), s);
}

cudaError_t launch_unpack_frame(const PackedFrame& src, const Frame& dst, cudaStream_t s) {
    cudaError_t e =
        launch_unpack_rows(src, 0, src.nrows(), dst.base + (size_t)dst.H * dst.pitch + dst.H, dst.pitch, s);
    if (e != cudaSuccess) return e;
    return launch_halo_fill(dst, s);
}

// ---------------------------------------------------------------------------
// PACK codec on dense device buffers.
// ---------------------------------------------------------------------------
__global__ void k_pack64(const uint8_t* __restrict__ cells, size_t cp, int rows, int cols, uint64_t* __restrict__ words,
                         size_t wp) {
    const int nw = (cols + 63) / 64;
    const long long total = (long long)rows * nw;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        const uint8_t* p = cells + (size_t)i * cp + 64 * (size_t)w;
        uint64_t v = 0ull;
        for (int b = 0; b < 64 && 64 * w + b < cols; ++b) v |= (uint64_t)(p[b] ? 1u : 0u) << b;
        words[(size_t)i * wp + w] = v;
    }
}

__global__ void k_unpack64(const uint64_t* __restrict__ words, size_t wp, int rows, int cols, uint8_t* __restrict__ cells,
                           size_t cp) {
    const int nw = (cols + 63) / 64;
    const long long total = (long long)rows * nw;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nw), w = (int)(t % nw);
        const uint64_t v = words[(size_t)i * wp + w];
        uint8_t* p = cells + (size_t)i * cp + 64 * (size_t)w;
        for (int b = 0; b < 64 && 64 * w + b < cols; ++b) p[b] = (uint8_t)((v >> b) & 1ull);
    }
}

// Inner words of a packed frame -> PACK-coded rows (uint64 word k of a row =
// frame words 2k and 2k + 1), bits past n cleared.
__global__ void k_frame_to_pack64(const uint32_t* __restrict__ src, int n, int rows, int nw, int HR, int HW,
                                  size_t wp, uint64_t* __restrict__ dst, size_t dst_wp) {
    const int nw64 = (n + 63) / 64;
    const long long total = (long long)rows * nw64;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(t / nw64), k = (int)(t % nw64);
        const uint32_t* row = src + (size_t)(HR + i) * wp + HW;
        uint32_t lo = row[2 * k];
        uint32_t hi = 2 * k + 1 < nw ? row[2 * k + 1] : 0u;
        uint64_t v = ((uint64_t)hi << 32) | lo;
        const int valid = n - 64 * k;  // cells of this word inside the row
        if (valid < 64) v &= (1ull << valid) - 1ull;
        dst[(size_t)i * dst_wp + k] = v;
    }
}

cudaError_t launch_frame_to_pack64(const PackedFrame& f, uint64_t* dst, size_t dst_pitch_words, cudaStream_t s) {
    const long long total = (long long)f.nrows() * ((f.n + 63) / 64);
    if (total == 0) return cudaSuccess;
    const int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_frame_to_pack64<<<blocks, 256, 0, s>>>(f.words, f.n, f.nrows(), f.nw, f.HR, f.HW, f.wpitch, dst,
                                             dst_pitch_words);
    return cudaGetLastError();
}

cudaError_t launch_pack(const uint8_t* cells, size_t cell_pitch, int rows, int cols, uint64_t* words,
                        size_t word_pitch_words, cudaStream_t s) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    long long total = (long long)rows * ((cols + 63) / 64);
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_pack64<<<blocks, 256, 0, s>>>(cells, cell_pitch, rows, cols, words, word_pitch_words);
    return cudaGetLastError();
}

cudaError_t launch_unpack(const uint64_t* words, size_t word_pitch_words, int rows, int cols, uint8_t* cells,
                          size_t cell_pitch, cudaStream_t s) {
    if (rows == 0 || cols == 0) return cudaSuccess;
    long long total = (long long)rows * ((cols + 63) / 64);
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_unpack64<<<blocks, 256, 0, s>>>(words, word_pitch_words, rows, cols, cells, cell_pitch);
    return cudaGetLastError();
}

}  // namespace ltl

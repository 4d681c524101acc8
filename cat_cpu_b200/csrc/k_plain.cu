// k_plain.cu -- CUDA-core kernels of libltl_b200:
//   K5 torus halo fill, K1 plain LtL step (SWAR fast path for R <= 5 and a
//   generic two-pass path for any R), K6 population / comparison, and the
//   dense <-> frame copies used by upload/download.
//
// Semantics restated from the reference (kezada94/CAT_cpu):
//   step  HostSolver<int>::CAStepAlgorithm, src/CellularAutomata/Solvers/HostSolver.tpp:58-73
//   count HostSolver<int>::countAliveNeighbors (centre excluded), HostSolver.tpp:75-91
//   rule  transitionFunction [a <= k <= b], HostSolver.tpp:47-51
//   halo  fillHorizontal/VerticalBoundaryConditions (torus), HostSolver.tpp:93-140
#include <algorithm>
#include <type_traits>

#include "ltl_kernels.h"

namespace ltl {

// ---------------------------------------------------------------------------
// K5: halo fill.  Frame cell (r, c) <- inner ((r-H) mod n, (c-H) mod n).  All
// sources are inner cells, so no ordering between halo bands is needed.
// Top/bottom bands copy 16-byte chunks whose columns are inner (same column in
// the source row); everything else goes byte by byte.
// ---------------------------------------------------------------------------
__global__ void k_halo_rows(uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch) {
    const int band = blockIdx.y;                       // 0 .. 2H-1
    const int r = band < H ? band : rows + band;       // frame row
    const int src_r = H + wrap_mod(r - H, rows);
    const int W = n + 2 * H;
    const int nchunks = (W + 15) / 16;
    uint8_t* dst_row = g + (size_t)r * pitch;
    const uint8_t* src_row = g + (size_t)src_r * pitch;
    for (int ch = blockIdx.x * blockDim.x + threadIdx.x; ch < nchunks; ch += gridDim.x * blockDim.x) {
        int c0 = ch * 16;
        if (c0 >= H && c0 + 16 <= H + n) {
            *(uint4*)(dst_row + c0) = *(const uint4*)(src_row + c0);
        } else {
            for (int c = c0; c < c0 + 16 && c < W; ++c) dst_row[c] = src_row[H + wrap_mod(c - H, n)];
        }
    }
}

__global__ void k_halo_cols(uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch) {
    // inner rows only; 2H halo bytes per row
    const int per_row = 2 * H;
    const long long total = (long long)rows * per_row;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / per_row);
        int k = (int)(t % per_row);
        int c = k < H ? k : n + k;  // frame column
        uint8_t* row = g + (size_t)(H + i) * pitch;
        row[c] = row[H + wrap_mod(c - H, n)];
    }
}

cudaError_t launch_halo_fill(const Frame& f, cudaStream_t s) {
    const int W = f.n + 2 * f.H;
    const int nchunks = (W + 15) / 16;
    dim3 g1((unsigned)std::min((nchunks + 127) / 128, 64), (unsigned)(2 * f.H));
    k_halo_rows<<<g1, 128, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch);
    long long total = (long long)f.nrows() * 2 * f.H;
    int blocks = (int)std::min<long long>((total + 255) / 256, 4096);
    k_halo_cols<<<blocks, 256, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K1 fast path (R <= 5): SWAR with 8-bit lanes.
//
// A warp owns a 512-column strip: lane L holds the 16-cell chunk at inner
// columns [x, x+16), x = strip*480 - 16 + 16L, as four 32-bit words of byte
// lanes.  It slides a vertical window of 2R+1 rows down its band: V = column
// sums (<= 2R+1 per lane).  Row sums of V come from the lane's own words plus
// the neighbouring lanes' edge words (warp shuffles), so lanes 1..30 produce
// 16 output cells each (480 per warp).  Box counts B <= (2R+1)^2 <= 121 fit a
// byte lane, and the interval rule is evaluated four cells at a time with the
// borrow bit of each lane (rule_swar8).
// ---------------------------------------------------------------------------
constexpr int kStripOut = 480;  // output columns per warp

// Torus wrap of a row or column index that is at most one side outside [0, n).
// With `wrap` set, the SWAR kernels read every cell from its inner position
// (row and column taken modulo n), so the frame's halo is not read and needs
// no refresh.  Column chunks of 16 bytes stay 16-byte aligned only if n is a
// multiple of 16, which the host checks before it sets `wrap`.
__device__ __forceinline__ int wrap1(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }

__device__ __forceinline__ void v_add(uint32_t (&v)[4], uint4 a) {
    v[0] += a.x; v[1] += a.y; v[2] += a.z; v[3] += a.w;
}
__device__ __forceinline__ void v_slide(uint32_t (&v)[4], uint4 in, uint4 out) {
    v[0] += in.x - out.x; v[1] += in.y - out.y; v[2] += in.z - out.z; v[3] += in.w - out.w;
}

// Row box sums for the lane's four output words.  w[0..7] = byte words at
// offsets -8 .. +28 of the lane's chunk (two words of the left lane, the four
// own words, two words of the right lane); byte offset o of the chunk is byte
// o + 8 of w.  The (2R+1)-wide window is split into power-of-two segments
// (e.g. 11 = 8 + 2 + 1), and the segment sums P_k (k consecutive bytes, SWAR)
// are built by doubling: P_2k(y) = P_k(y) + P_k(y + k).
template <int K>
__device__ __forceinline__ void double_seg(const uint32_t (&a)[8], uint32_t (&b)[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if constexpr (K < 4) {
            b[j] = (j + 1 < 8) ? a[j] + __funnelshift_r(a[j], a[j + 1], 8 * K) : 0u;
        } else {
            b[j] = (j + K / 4 < 8) ? a[j] + a[j + K / 4] : 0u;
        }
    }
}

template <int O>
__device__ __forceinline__ uint32_t bytes_at(const uint32_t (&w)[8]) {
    constexpr int idx = O >> 2, sh = O & 3;
    if constexpr (sh == 0) {
        return w[idx];
    } else {
        return __funnelshift_r(w[idx], w[idx + 1], 8 * sh);
    }
}

template <int L, int O>
__device__ __forceinline__ uint32_t window_sum(const uint32_t (&p1)[8], const uint32_t (&p2)[8],
                                               const uint32_t (&p4)[8], const uint32_t (&p8)[8]) {
    // sum of L consecutive bytes starting at w-offset O (L <= 15)
    if constexpr (L == 0) {
        return 0u;
    } else if constexpr (L >= 8) {
        return bytes_at<O>(p8) + window_sum<L - 8, O + 8>(p1, p2, p4, p8);
    } else if constexpr (L >= 4) {
        return bytes_at<O>(p4) + window_sum<L - 4, O + 4>(p1, p2, p4, p8);
    } else if constexpr (L >= 2) {
        return bytes_at<O>(p2) + window_sum<L - 2, O + 2>(p1, p2, p4, p8);
    } else {
        return bytes_at<O>(p1);
    }
}

template <int R>
__device__ __forceinline__ void row_boxes(const uint32_t (&w)[8], uint32_t (&box)[4]) {
    uint32_t p2[8], p4[8], p8[8];
    double_seg<1>(w, p2);
    double_seg<2>(p2, p4);
    double_seg<4>(p4, p8);
    box[0] = window_sum<2 * R + 1, 0 * 4 - R + 8>(w, p2, p4, p8);
    box[1] = window_sum<2 * R + 1, 1 * 4 - R + 8>(w, p2, p4, p8);
    box[2] = window_sum<2 * R + 1, 2 * 4 - R + 8>(w, p2, p4, p8);
    box[3] = window_sum<2 * R + 1, 3 * 4 - R + 8>(w, p2, p4, p8);
}

// Each warp streams its strip's rows through a private shared-memory ring with
// cp.async (16 bytes per lane per row, one commit group per row, kAhead rows in
// flight): every row is read from global memory once per band, and the centre
// and leaving rows come back from shared memory.  A lane only ever reads the
// ring bytes it copied itself, so no intra-warp synchronisation is needed.
constexpr int kRingRows = 32;  // power of two >= 2R + 2 + kAhead
constexpr int kAhead = 8;
constexpr int kPlainWarps = 4;

// Store the first `count` (< 16) bytes of v; compile-time lane indices only, so
// v stays in registers.
__device__ __forceinline__ void store_partial16(uint8_t* dst, uint4 v, int count) {
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int j = 0; j < 16; ++j)
        if (j < count) dst[j] = (uint8_t)(w[j >> 2] >> (8 * (j & 3)));
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem)),
                 "l"(gmem)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

template <int R>
__global__ void __launch_bounds__(kPlainWarps * 32)
k_plain_swar8(const uint8_t* __restrict__ cur, uint8_t* __restrict__ nxt, int n, int rows, int H, size_t pitch,
              int band_rows, int n_strips, int n_items, RuleSwar8 q, int wrap) {
    static_assert(2 * R + 2 + kAhead <= kRingRows, "ring too small");
    extern __shared__ uint4 ring_all[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    uint4* ring = ring_all + (size_t)wid * kRingRows * 32 + lane;
    const int gwarp = blockIdx.x * kPlainWarps + wid;
    const int gwarps = gridDim.x * kPlainWarps;

    for (int item = gwarp; item < n_items; item += gwarps) {
        const int strip = item % n_strips;
        const int band = item / n_strips;
        const int r0 = band * band_rows;
        const int r1 = min(r0 + band_rows, rows);
        const int x = strip * kStripOut - 16 + 16 * lane;      // inner column of this lane's chunk
        const bool loads = x < n + 16;                          // chunks past that feed no output
        const bool outputs = lane >= 1 && lane <= 30 && x < n;
        const uint8_t* col = cur + (size_t)H + (loads ? (wrap ? wrap1(x, n) : x) : 0);
        const int rlast = min(r1 - 1 + R, rows - 1 + R);        // last row any window of the band needs
        auto slot = [&](int r) { return ring + (r & (kRingRows - 1)) * 32; };
        auto issue = [&](int r) {
            if (loads && r <= rlast) cp_async16(slot(r), col + (size_t)(H + (wrap ? wrap1(r, rows) : r)) * pitch);
            cp_async_commit();
        };
        // rows r0-R .. r0+R start the window; kAhead more go in flight behind them
        for (int r = r0 - R; r <= r0 + R + kAhead; ++r) issue(r);
        cp_async_wait<kAhead>();
        uint32_t V[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy) v_add(V, *slot(r0 + dy));

#pragma unroll 1
        for (int rr = r0; rr < r1; ++rr) {
            uint32_t w[8];
            w[0] = __shfl_up_sync(0xffffffffu, V[2], 1);
            w[1] = __shfl_up_sync(0xffffffffu, V[3], 1);
            w[2] = V[0]; w[3] = V[1]; w[4] = V[2]; w[5] = V[3];
            w[6] = __shfl_down_sync(0xffffffffu, V[0], 1);
            w[7] = __shfl_down_sync(0xffffffffu, V[1], 1);
            if (outputs) {
                const uint4 c = *slot(rr);
                uint32_t box[4];
                row_boxes<R>(w, box);
                uint4 o;
                o.x = rule_swar8(box[0], c.x, q);
                o.y = rule_swar8(box[1], c.y, q);
                o.z = rule_swar8(box[2], c.z, q);
                o.w = rule_swar8(box[3], c.w, q);
                uint8_t* dst = nxt + (size_t)(H + rr) * pitch + H + x;
                if (x + 16 <= n) {
                    *(uint4*)dst = o;
                } else {
                    store_partial16(dst, o, n - x);
                }
            }
            if (rr + 1 < r1) {
                issue(rr + R + 1 + kAhead);
                cp_async_wait<kAhead>();          // row rr + R + 1 has landed
                v_slide(V, *slot(rr + R + 1), *slot(rr - R));
            }
        }
        cp_async_wait<0>();
    }
}

bool plain_swar8_supported(int radius) { return radius >= 1 && radius <= 5; }

int plain_swar8_band_rows(int n, int device) {
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int strips = (n + kStripOut - 1) / kStripOut;
    // Enough items for ~32 resident warps per SM, but bands of at least 96 rows:
    // every band re-reads 2R+1 rows to start its vertical window.
    long long target_items = (long long)sms * 32;
    int bands = (int)std::max<long long>(1, target_items / std::max(strips, 1));
    int rows = (n + bands - 1) / bands;
    rows = std::max(96, std::min(rows, 512));
    return rows;
}

template <int R>
static cudaError_t launch_swar8_r(const Frame& cur, const Frame& nxt, const RuleSwar8& q, int band_rows, int wrap,
                                  cudaStream_t s) {
    const int n = cur.n, rows = cur.nrows();
    const int strips = (n + kStripOut - 1) / kStripOut;
    const int bands = (rows + band_rows - 1) / band_rows;
    const int items = strips * bands;
    const int smem = kPlainWarps * kRingRows * 32 * (int)sizeof(uint4);
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_plain_swar8<R>, kPlainWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    int ctas = std::min((items + kPlainWarps - 1) / kPlainWarps, sms * per_sm);
    k_plain_swar8<R><<<ctas, kPlainWarps * 32, smem, s>>>(cur.base, nxt.base, n, rows, cur.H, cur.pitch, band_rows,
                                                         strips, items, q, wrap);
    return cudaGetLastError();
}

template <int R>
static cudaError_t prepare_swar8_r() {
    const int smem = kPlainWarps * kRingRows * 32 * (int)sizeof(uint4);
    return cudaFuncSetAttribute(k_plain_swar8<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
}

cudaError_t plain_prepare(int radius) {
    switch (radius) {
        case 1: return prepare_swar8_r<1>();
        case 2: return prepare_swar8_r<2>();
        case 3: return prepare_swar8_r<3>();
        case 4: return prepare_swar8_r<4>();
        case 5: return prepare_swar8_r<5>();
        default: return cudaSuccess;
    }
}

bool plain_wrap_supported(int n, int rows) { return n >= 64 && n % 16 == 0 && rows >= 16; }

cudaError_t launch_plain_swar8(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows, bool wrap,
                               cudaStream_t s) {
    if (wrap && !plain_wrap_supported(cur.n, cur.nrows())) return cudaErrorInvalidValue;
    RuleSwar8 q = make_rule_swar8(rule);
    const int w = wrap ? 1 : 0;
    switch (rule.radius) {
        case 1: return launch_swar8_r<1>(cur, nxt, q, band_rows, w, s);
        case 2: return launch_swar8_r<2>(cur, nxt, q, band_rows, w, s);
        case 3: return launch_swar8_r<3>(cur, nxt, q, band_rows, w, s);
        case 4: return launch_swar8_r<4>(cur, nxt, q, band_rows, w, s);
        case 5: return launch_swar8_r<5>(cur, nxt, q, band_rows, w, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// K1 temporally blocked (R <= 5, D = 2 or 3 generations per pass, D*R <= 16).
//
// The same SWAR row step as k_plain_swar8, stacked D times inside one warp so
// that a pass reads the grid once and writes it once for D generations.  Stage
// 1 slides its vertical window over the input rows (shared-memory ring 0, fed
// by cp.async); stage k > 1 slides over the rows stage k-1 has just produced
// (ring k-1), one row behind per R rows of lag.  All 32 lanes run the inner
// stages: lane 0's bytes [kR, 16) and lane 31's bytes [0, 16 - kR) of stage k
// are exact (the rest read past the strip), and D*R <= 16 keeps every byte
// lanes 1..30 of stage D read inside that exact part.  Rows: stage k
// produces rows [r0 - (D-k)R, r1 - 1 + (D-k)R] of the band, so the inputs are
// rows [r0 - DR, r1 - 1 + DR], inside the frame's halo (H >= D*R).  Stage
// values in halo rows and columns are exact torus values because the halo is
// an exact copy to depth H.
// ---------------------------------------------------------------------------
constexpr int kTbRing = 16;  // rows of the input ring (power of two >= 2R + 2 + ahead)

template <int R>
constexpr int tb_ahead() {
    return (kTbRing - (2 * R + 2)) < 8 ? (kTbRing - (2 * R + 2)) : 8;
}

// The input ring has kTbRing rows; each inner stage's ring has 2R + 2 (the
// rows its successor's window spans plus the one leaving it).
template <int R, int D>
constexpr int tb_ring_rows() {
    return kTbRing + (D - 1) * (2 * R + 2);
}

template <int R, int D>
constexpr int tb_smem_bytes() {
    return kPlainWarps * tb_ring_rows<R, D>() * 32 * (int)sizeof(uint4);
}

// One SWAR row of the interval rule for all lanes: V = the lane's vertical
// window sums, c = the lane's centre cells.  Every lane of the warp must call it.
template <int R>
__device__ __forceinline__ uint4 swar8_row(const uint32_t (&V)[4], uint4 c, const RuleSwar8& q) {
    uint32_t w[8];
    w[0] = __shfl_up_sync(0xffffffffu, V[2], 1);
    w[1] = __shfl_up_sync(0xffffffffu, V[3], 1);
    w[2] = V[0]; w[3] = V[1]; w[4] = V[2]; w[5] = V[3];
    w[6] = __shfl_down_sync(0xffffffffu, V[0], 1);
    w[7] = __shfl_down_sync(0xffffffffu, V[1], 1);
    uint32_t box[4];
    row_boxes<R>(w, box);
    uint4 o;
    o.x = rule_swar8(box[0], c.x, q);
    o.y = rule_swar8(box[1], c.y, q);
    o.z = rule_swar8(box[2], c.z, q);
    o.w = rule_swar8(box[3], c.w, q);
    return o;
}

template <int R, int D>
__global__ void __launch_bounds__(kPlainWarps * 32)
k_plain_swar8_tb(const uint8_t* __restrict__ cur, uint8_t* __restrict__ nxt, int n, int rows, int H, size_t pitch,
                 int band_rows, int n_strips, int n_items, RuleSwar8 q, int wrap) {
    constexpr int kAh = tb_ahead<R>();
    constexpr int kRS = 2 * R + 2;  // rows per inner-stage ring
    static_assert(D >= 2 && D * R <= 16 && kAh >= 1, "unsupported depth");
    extern __shared__ uint4 ring_all[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    uint4* ring0 = ring_all + (size_t)wid * tb_ring_rows<R, D>() * 32 + lane;  // input rows
    auto slot0 = [&](int r) { return ring0 + (r & (kTbRing - 1)) * 32; };
    // ring k >= 1 (rows of stage k), slot s in [0, kRS)
    auto slotk = [&](int k, int sl) { return ring0 + (kTbRing + (k - 1) * kRS + sl) * 32; };
    auto wrap_rs = [](int v) { return v >= kRS ? v - kRS : v; };
    const int gwarp = blockIdx.x * kPlainWarps + wid;
    const int gwarps = gridDim.x * kPlainWarps;

    for (int item = gwarp; item < n_items; item += gwarps) {
        const int strip = item % n_strips;
        const int band = item / n_strips;
        const int r0 = band * band_rows;
        const int r1 = min(r0 + band_rows, rows);
        const int x = strip * kStripOut - 16 + 16 * lane;
        const bool loads = x < n + 16;  // (D*R <= 16: columns >= n + 16 feed no output)
        const bool outputs = lane >= 1 && lane <= 30 && x < n;
        const uint8_t* col = cur + (size_t)H + (loads ? (wrap ? wrap1(x, n) : x) : 0);
        const int rlast = r1 - 1 + D * R;          // last input row of the band
        const int yfirst = r0 - (D - 1) * R;        // first and last stage-1 rows
        const int ylast = r1 - 1 + (D - 1) * R;
        for (int r = yfirst - R; r <= yfirst + R + kAh; ++r) {
            if (loads && r <= rlast) cp_async16(slot0(r), col + (size_t)(H + (wrap ? wrap1(r, rows) : r)) * pitch);
            cp_async_commit();
        }
        // next input row to request (y + R + 1 + kAh at iteration y, never
        // negative), and the output row of stage D once it produces (y - (D-1)R)
        int r_next = yfirst + R + 1 + kAh;
        const uint8_t* src_next = col + (size_t)(H + (wrap ? wrap1(r_next, rows) : r_next)) * pitch;
        uint8_t* dst = nxt + (size_t)(H + r0) * pitch + H + x;
        cp_async_wait<kAh>();
        uint32_t V[D][4];
#pragma unroll
        for (int k = 0; k < D; ++k) V[k][0] = V[k][1] = V[k][2] = V[k][3] = 0u;
#pragma unroll 1
        for (int dy = -R; dy <= R; ++dy) v_add(V[0], *slot0(yfirst + dy));
        // sl[k] = ring-k slot of the row stage k produces in this iteration,
        // y - (k-1)R, modulo kRS (rows may be negative: start from a non-negative
        // representative)
        int sl[D];
#pragma unroll
        for (int k = 1; k < D; ++k) sl[k] = ((yfirst - (k - 1) * R) % kRS + kRS) % kRS;

        // One iteration (stage-1 row y).  Stage k >= 2 absorbs row yin = y - (k-2)R
        // of stage k-1 and, once its window is full, produces row yin - R.  In ring
        // k-1 the leaving row yin - 2R - 1 sits one slot after yin, and row yin - R
        // sits R + 2 after.  kSteady: every stage's window is full and sliding (from
        // y = yfirst + 2R(D-1) + 1 on), so no stage needs its fill checks.
        auto iteration = [&](int y, auto steady) {
            constexpr bool kSteady = decltype(steady)::value;
            uint4 prod = swar8_row<R>(V[0], *slot0(y), q);
            *slotk(1, sl[1]) = prod;
            bool live = true;
#pragma unroll
            for (int k = 2; k <= D; ++k) {
                if (kSteady || live) {
                    const int absorbed = kSteady ? 0 : (y - (k - 2) * R) - (r0 - (D - k + 1) * R) + 1;
                    v_add(V[k - 1], prod);
                    if (kSteady || absorbed > 2 * R + 1) {
                        const uint4 out = *slotk(k - 1, wrap_rs(sl[k - 1] + 1));
                        V[k - 1][0] -= out.x; V[k - 1][1] -= out.y; V[k - 1][2] -= out.z; V[k - 1][3] -= out.w;
                    }
                    if (kSteady || absorbed >= 2 * R + 1) {
                        const uint4 c = *slotk(k - 1, wrap_rs(sl[k - 1] + R + 2));
                        if (k < D) {
                            prod = swar8_row<R>(V[k - 1], c, q);
                            *slotk(k, sl[k]) = prod;
                        } else {
                            const uint4 o = swar8_row<R>(V[k - 1], c, q);
                            if (outputs) {
                                if (x + 16 <= n) {
                                    *(uint4*)dst = o;
                                } else {
                                    store_partial16(dst, o, n - x);
                                }
                            }
                            dst += pitch;
                        }
                    } else {
                        live = false;
                    }
                }
            }
#pragma unroll
            for (int k = 1; k < D; ++k) sl[k] = wrap_rs(sl[k] + 1);
            if (y < ylast) {
                if (loads && r_next <= rlast) cp_async16(slot0(r_next), src_next);
                cp_async_commit();
                ++r_next;
                src_next += pitch;
                if (wrap && r_next == rows) src_next -= (size_t)rows * pitch;  // the next row is inner row 0
                cp_async_wait<kAh>();  // input row y + R + 1 has landed
                v_slide(V[0], *slot0(y + R + 1), *slot0(y - R));
            }
        };
        const int ysteady = yfirst + 2 * R * (D - 1) + 1;
        int y = yfirst;
#pragma unroll 1
        for (; y < ysteady && y <= ylast; ++y) iteration(y, std::false_type{});
#pragma unroll 1
        for (; y <= ylast; ++y) iteration(y, std::true_type{});
        cp_async_wait<0>();
    }
}

bool plain_tb_supported(int radius, int depth) {
    return plain_swar8_supported(radius) && (depth == 2 || depth == 3) && depth * radius <= 16;
}

template <int R, int D>
static cudaError_t launch_tb_rd(const Frame& cur, const Frame& nxt, const RuleSwar8& q, int band_rows, int wrap,
                                cudaStream_t s) {
    const int n = cur.n, rows = cur.nrows();
    const int strips = (n + kStripOut - 1) / kStripOut;
    const int bands = (rows + band_rows - 1) / band_rows;
    const int items = strips * bands;
    constexpr int smem = tb_smem_bytes<R, D>();
    int dev = 0, sms = 148, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_plain_swar8_tb<R, D>, kPlainWarps * 32, smem);
    if (per_sm < 1) per_sm = 1;
    int ctas = std::min((items + kPlainWarps - 1) / kPlainWarps, sms * per_sm);
    k_plain_swar8_tb<R, D><<<ctas, kPlainWarps * 32, smem, s>>>(cur.base, nxt.base, n, rows, cur.H, cur.pitch,
                                                               band_rows, strips, items, q, wrap);
    return cudaGetLastError();
}

template <int R, int D>
static cudaError_t prepare_tb_rd() {
    if constexpr (D * R <= 16) {
        return cudaFuncSetAttribute(k_plain_swar8_tb<R, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    tb_smem_bytes<R, D>());
    } else {
        return cudaSuccess;
    }
}

template <int R>
static cudaError_t launch_tb_r(const Frame& cur, const Frame& nxt, const RuleSwar8& q, int band_rows, int depth,
                               int wrap, cudaStream_t s) {
    if (depth == 2) return launch_tb_rd<R, 2>(cur, nxt, q, band_rows, wrap, s);
    if constexpr (3 * R <= 16) {
        if (depth == 3) return launch_tb_rd<R, 3>(cur, nxt, q, band_rows, wrap, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t plain_tb_prepare(int radius) {
    cudaError_t e = cudaSuccess;
    switch (radius) {
#define LTL_TBP(r) \
    case r: e = prepare_tb_rd<r, 2>(); if (e == cudaSuccess) e = prepare_tb_rd<r, 3>(); break;
        LTL_TBP(1) LTL_TBP(2) LTL_TBP(3) LTL_TBP(4) LTL_TBP(5)
#undef LTL_TBP
        default: break;
    }
    return e;
}

cudaError_t launch_plain_tb(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows, int depth,
                            bool wrap, cudaStream_t s) {
    if (!plain_tb_supported(rule.radius, depth) || cur.H < depth * rule.radius) return cudaErrorInvalidValue;
    if (wrap && !plain_wrap_supported(cur.n, cur.nrows())) return cudaErrorInvalidValue;
    RuleSwar8 q = make_rule_swar8(rule);
    const int w = wrap ? 1 : 0;
    switch (rule.radius) {
        case 1: return launch_tb_r<1>(cur, nxt, q, band_rows, depth, w, s);
        case 2: return launch_tb_r<2>(cur, nxt, q, band_rows, depth, w, s);
        case 3: return launch_tb_r<3>(cur, nxt, q, band_rows, depth, w, s);
        case 4: return launch_tb_r<4>(cur, nxt, q, band_rows, depth, w, s);
        case 5: return launch_tb_r<5>(cur, nxt, q, band_rows, depth, w, s);
        default: return cudaErrorInvalidValue;
    }
}

// ---------------------------------------------------------------------------
// K1 generic path (any R >= 1): one fused kernel, work per cell independent of R.
//
// A CTA of 256 threads owns a tile of T output columns [j0, j0 + T) and a band
// of rows.  Its window columns are [c0, c0 + 1024K), c0 = j0 - R rounded down
// to a multiple of 4; thread t owns the 4K consecutive columns starting at
// c0 + 4Kt and keeps their vertical window sums V (2R+1 rows) in registers as
// 16-bit SWAR lanes, sliding them down one row at a time (V += X(r+R+1) -
// X(r-R)).  For every row the CTA scans V into prefix sums P in shared memory
// (local sums, a warp scan, the warp totals), and each output reads
//   B(j) = P[j - c0 + R + 1] - P[j - c0 - R],   k = B - centre,
// then applies the interval rule.  P is double-buffered, so two barriers per
// row suffice.  This replaces a two-kernel version that wrote V to HBM.
// ---------------------------------------------------------------------------
constexpr int kWideThreads = 256;

template <int K>
__global__ void __launch_bounds__(kWideThreads)
k_plain_wide(const uint8_t* __restrict__ X, uint8_t* __restrict__ Y, int n, int rows, int H, size_t pitch,
             int band_rows, int T, Rule rule) {
    constexpr int L = 1024 * K;  // window columns per CTA
    __shared__ int P[2][L + 1];
    __shared__ int wsum[kWideThreads / 32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int R = rule.radius;
    const int j0 = blockIdx.x * T;
    const int r0 = blockIdx.y * band_rows;
    const int r1 = min(r0 + band_rows, rows);
    const int c0 = (j0 - R) & ~3;                  // floor to a multiple of 4 (two's complement)
    const int cstart = c0 + 4 * K * t;             // inner column of this thread's first window column
    const bool need = cstart <= n - 1 + R;         // later columns feed no output (and may lie past the row)
    const uint8_t* col = X + (size_t)H + cstart;   // 4-byte aligned: H, pitch and cstart are multiples of 4
    auto ldw = [&](int r, int k) { return __ldg((const uint32_t*)(col + (size_t)(H + r) * pitch) + k); };

    uint32_t V[2 * K];  // V[2k]: columns 4k, 4k+1; V[2k+1]: columns 4k+2, 4k+3 (16-bit lanes)
#pragma unroll
    for (int k = 0; k < 2 * K; ++k) V[k] = 0u;
    if (need) {
        for (int dy = -R; dy <= R; ++dy) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint32_t x = ldw(r0 + dy, k);
                V[2 * k] += __byte_perm(x, 0, 0x4140);
                V[2 * k + 1] += __byte_perm(x, 0, 0x4342);
            }
        }
    }
    for (int r = r0; r < r1; ++r) {
        int* Pr = P[r & 1];
        // issue this row's global loads first (the next row's entering and
        // leaving window rows, the first output chunk's centre cells), so that
        // their latency hides behind the scan
        const bool slide = r + 1 < r1 && need;
        uint32_t xa[K], xb[K];
#pragma unroll
        for (int k = 0; k < K; ++k) {
            xa[k] = slide ? ldw(r + R + 1, k) : 0u;
            xb[k] = slide ? ldw(r - R, k) : 0u;
        }
        const int q0 = 4 * t;
        const bool out0 = q0 < T && j0 + q0 < n;
        const uint32_t sw0 = out0 ? __ldg((const uint32_t*)(X + (size_t)(H + r) * pitch + H + j0 + q0)) : 0u;
        // this thread's values and their local sum
        int v[4 * K];
#pragma unroll
        for (int k = 0; k < 2 * K; ++k) {
            v[2 * k] = (int)(V[k] & 0xffffu);
            v[2 * k + 1] = (int)(V[k] >> 16);
        }
        int sum = 0;
#pragma unroll
        for (int i = 0; i < 4 * K; ++i) sum += v[i];
        int incl = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        // exclusive prefix of the 8 warp totals, scanned by each warp's first lanes
        int wt = lane < kWideThreads / 32 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < kWideThreads / 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, wt, o);
            if (lane >= o) wt += y;
        }
        const int wpre = __shfl_sync(0xffffffffu, wt, (wid + 31) & 31);  // inclusive total of warps < wid
        int run = incl - sum + (wid > 0 ? wpre : 0);
#pragma unroll
        for (int i = 0; i < 4 * K; ++i) {
            Pr[4 * K * t + i] = run;
            run += v[i];
        }
        if (t == kWideThreads - 1) Pr[L] = run;
        __syncthreads();
        // outputs: 4 consecutive cells per thread per pass
        for (int q = q0; q < T; q += 4 * kWideThreads) {
            const int j = j0 + q;
            if (j >= n) break;
            const uint32_t sw = q == q0 ? sw0 : __ldg((const uint32_t*)(X + (size_t)(H + r) * pitch + H + j));
            const int base = j - c0;
            uint32_t ow = 0;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int B = Pr[base + u + R + 1] - Pr[base + u - R];
                const int sv = (sw >> (8 * u)) & 1;
                // k in [lo, hi]  <=>  (unsigned)(k - lo) <= (unsigned)(hi - lo); an empty
                // interval (hi < lo) has a negative width that no k passes as unsigned
                const int lo = sv ? rule.smin : rule.bmin;
                const int wdt = sv ? rule.smax - rule.smin : rule.bmax - rule.bmin;
                const uint32_t in = wdt >= 0 && (uint32_t)(B - sv - lo) <= (uint32_t)wdt;
                ow |= in << (8 * u);
            }
            uint8_t* yr = Y + (size_t)(H + r) * pitch + H + j;
            if (j + 4 <= n) {
                *(uint32_t*)yr = ow;
            } else {
                for (int u = 0; u < n - j; ++u) yr[u] = (uint8_t)((ow >> (8 * u)) & 0xffu);
            }
        }
        if (slide) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                V[2 * k] += __byte_perm(xa[k], 0, 0x4140) - __byte_perm(xb[k], 0, 0x4140);
                V[2 * k + 1] += __byte_perm(xa[k], 0, 0x4342) - __byte_perm(xb[k], 0, 0x4342);
            }
        }
    }
}

cudaError_t launch_plain_generic(const Frame& cur, const Frame& nxt, const Rule& rule, cudaStream_t s) {
    const int n = cur.n, rows = cur.nrows(), R = rule.radius;
    if (cur.H < ((R + 3) & ~3) || (cur.H & 3) || (cur.pitch & 3)) return cudaErrorInvalidValue;
    // T: outputs per tile, so that [j0 - R, j0 + T + R] (plus the rounding of c0)
    // fits the window columns; bands long enough to amortise the 2R+1-row start
    // (and short enough that tiles x bands keep about 6 CTAs per SM busy)
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int K = (1024 - 2 * R - 3 >= 256) ? 1 : 2;
    if (2048 - 2 * R - 3 < 256) return cudaErrorInvalidValue;  // R > 893
    const int T = (1024 * K - 2 * R - 3) & ~3;
    const int tiles = (n + T - 1) / T;
    const int want_bands = std::max(1, (6 * sms + tiles - 1) / tiles);
    const int band = std::max(32, std::min({512, 4 * (2 * R + 1), (rows + want_bands - 1) / want_bands}));
    const dim3 grid(tiles, (rows + band - 1) / band), block(kWideThreads);
    if (K == 1)
        k_plain_wide<1><<<grid, block, 0, s>>>(cur.base, nxt.base, n, rows, cur.H, cur.pitch, band, T, rule);
    else
        k_plain_wide<2><<<grid, block, 0, s>>>(cur.base, nxt.base, n, rows, cur.H, cur.pitch, band, T, rule);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// K6: population and comparison over inner cells.
// ---------------------------------------------------------------------------
__global__ void k_population(const uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch,
                             unsigned long long* out) {
    unsigned long long acc = 0;
    const long long total = (long long)rows * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / n), j = (int)(t % n);
        acc += g[(size_t)(H + i) * pitch + H + j];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}

__global__ void k_compare(const uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch,
                          const uint8_t* __restrict__ other, size_t opitch, unsigned long long* out) {
    unsigned long long cnt = 0, first = ~0ull;
    const long long total = (long long)rows * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / n), j = (int)(t % n);
        if (g[(size_t)(H + i) * pitch + H + j] != other[(size_t)i * opitch + j]) {
            ++cnt;
            if ((unsigned long long)t < first) first = (unsigned long long)t;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cnt += __shfl_down_sync(0xffffffffu, cnt, o);
        unsigned long long f2 = __shfl_down_sync(0xffffffffu, first, o);
        first = f2 < first ? f2 : first;
    }
    if ((threadIdx.x & 31) == 0 && cnt) {
        atomicAdd(out, cnt);
        atomicMin(out + 1, first);
    }
}

cudaError_t launch_population(const Frame& f, unsigned long long* scratch, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    long long total = (long long)f.nrows() * f.n;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    k_population<<<blocks, 256, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch, scratch);
    return cudaGetLastError();
}

cudaError_t launch_compare(const Frame& f, const uint8_t* other, size_t other_pitch,
                           unsigned long long* scratch, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(scratch, 0, sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(scratch + 1, 0xff, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    long long total = (long long)f.nrows() * f.n;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 16);
    k_compare<<<blocks, 256, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch, other, other_pitch, scratch);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Dense n x n <-> frame inner copies (device to device).
// ---------------------------------------------------------------------------
__global__ void k_copy_in(uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch,
                          const uint8_t* __restrict__ src, size_t sp) {
    const long long total = (long long)rows * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / n), j = (int)(t % n);
        g[(size_t)(H + i) * pitch + H + j] = src[(size_t)i * sp + j] ? 1 : 0;
    }
}

__global__ void k_copy_out(const uint8_t* __restrict__ g, int n, int rows, int H, size_t pitch,
                           uint8_t* __restrict__ dst, size_t dp) {
    const long long total = (long long)rows * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / n), j = (int)(t % n);
        dst[(size_t)i * dp + j] = g[(size_t)(H + i) * pitch + H + j];
    }
}

cudaError_t launch_copy_in(const Frame& f, const uint8_t* src, size_t src_pitch, cudaStream_t s) {
    long long total = (long long)f.nrows() * f.n;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_copy_in<<<blocks, 256, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch, src, src_pitch);
    return cudaGetLastError();
}

cudaError_t launch_copy_out(const Frame& f, uint8_t* dst, size_t dst_pitch, cudaStream_t s) {
    long long total = (long long)f.nrows() * f.n;
    int blocks = (int)std::min<long long>((total + 255) / 256, 148 * 32);
    k_copy_out<<<blocks, 256, 0, s>>>(f.base, f.n, f.nrows(), f.H, f.pitch, dst, dst_pitch);
    return cudaGetLastError();
}

}  // namespace ltl

// k_plain.cu -- CUDA-core kernels of libltl_b200:
//   K5 torus halo fill, K1 plain LtL step (SWAR fast path for R <= 5 and a
//   fused prefix-sum path for larger R), K6 population / comparison, and the
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
// K1 generic path (any R up to 2038; serves R > 5): one fused kernel, work per
// cell independent of R.
//
// A CTA of NT threads owns a tile of T output columns [j0, j0 + T) and a band
// of rows.  Its window columns are [c0, c0 + NT CPT), c0 = j0 - R rounded down
// to a multiple of CPT; thread t owns the CPT consecutive columns starting at
// c0 + CPT t and slides their vertical window sums V (2R+1 rows) down the band
// in registers, as 16-bit lanes (two columns per word):
//   V(r+1) = V(r) + X(r+R+1) - X(r-R).
// For every row the CTA turns V into prefix sums P over the window columns in
// shared memory (a local scan, a warp scan, the warp totals), and each output
// reads two of them:
//   B(j) = P[j - c0 + R + 1] - P[j - c0 - R],   k = B - centre.
// Row pairs (R <= 90): one 32-bit word carries the vertical sums of two rows
// for one column, row r in the low 16 bits and row r+1 in the high 16 bits.
// Integer adds of such words keep the two lanes apart up to a carry out of the
// low lane, and the window difference of the prefix sums is again a pair of
// box counts B(r) + 65536 B(r+1) as long as B(r) < 65536.  R <= 90 keeps every
// box count below 2^15 (181^2 = 32761), so one scan, one subtraction and a
// 16-bit lane interval test serve two rows.  Above R = 90 each word carries
// one row and the interval test runs on 32-bit lanes.
//
// Interval test on a lane holding B (centre included): with nlo = M - lo and
// hiM = M + hi (M = 2^15 or 2^31, lo/hi clamped to [0, N+1] and [-1, N]),
// B + nlo has the lane's top bit set iff B >= lo and hiM - B has it set iff
// B <= hi; neither overflows the lane.  lo and hi depend on the centre s
// (s ? [smin+1, smax+1] : [bmin, bmax]); one multiply-add of the lane-packed
// centres selects them for both lanes at once.
// ---------------------------------------------------------------------------
constexpr int kWidePairMaxRadius = 90;  // (2R+1)^2 < 2^15
// threads per CTA: 128 up to R = 128 (the window overhead 2R/(128 CPT) stays
// small and a CTA's barrier waits for fewer warps), 256 above, where the wider
// window keeps the overlap of neighbouring tiles down
constexpr int kWideNarrowMaxRadius = 128;
inline int wide_threads(int radius) { return radius <= kWideNarrowMaxRadius ? 128 : 256; }

struct RuleScan {
    int radius;
    uint32_t nlo0, hih0;  // dead centre, replicated to both 16-bit lanes in row-pair mode
    int32_t dnlo, dhih;   // change for a live centre
};

static RuleScan make_rule_scan(const Rule& r, bool pair) {
    const long long N = (2ll * r.radius + 1) * (2ll * r.radius + 1);
    auto clampll = [](long long v, long long a, long long b) { return v < a ? a : (v > b ? b : v); };
    const long long lo0 = clampll(r.bmin, 0, N + 1), hi0 = clampll(r.bmax, -1, N);
    const long long lo1 = clampll((long long)r.smin + 1, 0, N + 1), hi1 = clampll((long long)r.smax + 1, -1, N);
    const long long M = pair ? 0x8000ll : 0x80000000ll;
    RuleScan q;
    q.radius = r.radius;
    q.nlo0 = (uint32_t)(pair ? (M - lo0) * 0x10001ll : M - lo0);
    q.hih0 = (uint32_t)(pair ? (M + hi0) * 0x10001ll : M + hi0);
    q.dnlo = (int32_t)(lo0 - lo1);
    q.dhih = (int32_t)(hi1 - hi0);
    return q;
}

// PTX prmt in its default mode: result byte i is source byte sel[4i+2:4i] of
// {b, a}; when bit 4i+3 of sel is set the byte is replaced by copies of that
// source byte's top bit (zero for a 0/1 cell).
template <uint32_t SEL>
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "n"(SEL));
    return d;
}

// CPT bytes of one frame row at an address aligned to CPT.
template <int CPT>
__device__ __forceinline__ void ld_cells(const uint8_t* p, uint32_t (&w)[CPT / 4]) {
    if constexpr (CPT == 8) {
        const uint2 v = __ldg((const uint2*)p);
        w[0] = v.x; w[1] = v.y;
    } else {
        const uint4 v = __ldg((const uint4*)p);
        w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w;
    }
}

// V += X(entering) - X(leaving) for 4 columns held as two words of 16-bit lanes.
// The byte difference is taken with a +1 bias so that no lane borrows.
__device__ __forceinline__ void slide4(uint32_t& v01, uint32_t& v23, uint32_t xin, uint32_t xout) {
    const uint32_t d = xin + 0x01010101u - xout;  // bytes in [0, 2]
    v01 = v01 + prmt<0x4140>(d, 0u) - 0x00010001u;
    v23 = v23 + prmt<0x4342>(d, 0u) - 0x00010001u;
}

// Inclusive warp-scan step: v += v of lane (lane - O), for lanes >= O (the
// shuffle's own in-range predicate guards the add).
template <int O>
__device__ __forceinline__ uint32_t scan_up(uint32_t v) {
    asm("{\n\t.reg .pred p;\n\t.reg .b32 y;\n\t"
        "shfl.sync.up.b32 y|p, %0, %1, 0, -1;\n\t"
        "@p add.u32 %0, %0, y;\n\t}"
        : "+r"(v)
        : "n"(O));
    return v;
}

// v[u] = p[A + u], u = 0..3, for a 16-byte aligned p.
template <int A>
__device__ __forceinline__ void lds4(const uint32_t* p, uint32_t (&v)[4]) {
    const uint4 a = *(const uint4*)p;
    if constexpr (A == 0) {
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
        const uint4 b = *(const uint4*)(p + 4);
        const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = w[A + u];
    }
}

// PAIR: two rows per iteration in 16-bit lanes (R <= 90); CPT: window columns
// per thread (8 or 16); RM = R mod 4 fixes the alignment of the two prefix
// reads of every output group.
template <bool PAIR, int CPT, int RM, int NT>
__global__ void __launch_bounds__(NT)
k_plain_wide(const uint8_t* __restrict__ X, uint8_t* __restrict__ Y, int n, int rows, int H, size_t pitch,
             int band_rows, int T, RuleScan q) {
    constexpr int kWideThreads = NT;
    static_assert(kWideThreads == 128 || kWideThreads == 256, "warp totals are read as one or two uint4");
    constexpr int L = kWideThreads * CPT;  // window columns per CTA
    constexpr int NW = CPT / 4;            // words of cells per thread and row; output groups per thread
    constexpr int EA = (RM + 1) & 3;       // (j - c0 + R + 1) mod 4
    constexpr int SA = (4 - RM) & 3;       // (j - c0 - R) mod 4
    constexpr int STEP = PAIR ? 2 : 1;     // rows per iteration
    constexpr int PS = L + 4;              // words per P buffer
    __shared__ __align__(16) uint32_t P[2 * PS];
    __shared__ __align__(16) uint32_t wsum[2][kWideThreads / 32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int R = q.radius;
    const uint32_t nlo0 = q.nlo0, hih0 = q.hih0, dnlo = (uint32_t)q.dnlo, dhih = (uint32_t)q.dhih;
    const int j0 = blockIdx.x * T;
    const int r0 = blockIdx.y * band_rows;
    const int r1 = min(r0 + band_rows, rows);
    const int c0 = (j0 - R) & ~(CPT - 1);  // floor to a multiple of CPT (two's complement)
    const int cstart = c0 + CPT * t;       // inner column of this thread's first window column
    // later columns feed no output (and may lie past the row's halo)
    const bool need = cstart <= n - 1 + R;
    const ptrdiff_t pp = (ptrdiff_t)pitch;
    // frame row 0 at this thread's window columns; aligned to CPT (H, pitch, c0
    // are multiples of 16, 64 and CPT)
    const uint8_t* colp = X + (ptrdiff_t)H + cstart;

    // vertical window sums of row r0, 16-bit lanes: V[2k] columns 4k, 4k+1, V[2k+1] columns 4k+2, 4k+3
    uint32_t V[2 * NW];
#pragma unroll
    for (int k = 0; k < 2 * NW; ++k) V[k] = 0u;
    if (need) {
        const uint8_t* p = colp + (ptrdiff_t)(H + r0 - R) * pp;
        if constexpr (PAIR) {
            uint32_t acc[NW];  // byte lanes: 2R+1 <= 181
#pragma unroll
            for (int k = 0; k < NW; ++k) acc[k] = 0u;
#pragma unroll 16
            for (int dy = -R; dy <= R; ++dy, p += pp) {
                uint32_t x[NW];
                ld_cells<CPT>(p, x);
#pragma unroll
                for (int k = 0; k < NW; ++k) acc[k] += x[k];
            }
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                V[2 * k] = prmt<0x4140>(acc[k], 0u);
                V[2 * k + 1] = prmt<0x4342>(acc[k], 0u);
            }
        } else {
            // byte lanes over chunks of at most 255 rows, widened once per chunk
            for (int dy0 = -R; dy0 <= R; dy0 += 255) {
                const int cnt = min(255, R - dy0 + 1);
                uint32_t acc[NW];
#pragma unroll
                for (int k = 0; k < NW; ++k) acc[k] = 0u;
#pragma unroll 8
                for (int i = 0; i < cnt; ++i, p += pp) {
                    uint32_t x[NW];
                    ld_cells<CPT>(p, x);
#pragma unroll
                    for (int k = 0; k < NW; ++k) acc[k] += x[k];
                }
#pragma unroll
                for (int k = 0; k < NW; ++k) {
                    V[2 * k] += prmt<0x4140>(acc[k], 0u);
                    V[2 * k + 1] += prmt<0x4342>(acc[k], 0u);
                }
            }
        }
    }

    // this thread's output groups: columns j0 + 4t + 4 NT g, g < NW (T < NT CPT)
    // Row-pair mode keeps its output phase free of branches: a group past the
    // tile reads P at group 0's offset minus 4t (a valid position) and stores
    // nothing, and a group at the ragged right end of a row stores whole 4-byte
    // words, whose bytes past column n - 1 land in the frame's right halo (which
    // the halo fill after the step rewrites).  The 32-bit-lane mode, measured
    // faster with branches, skips such groups and stores the ragged end bytewise.
    bool has[NW], full[NW];
    int goff[NW];  // P offset of group g from group 0's
#pragma unroll
    for (int g = 0; g < NW; ++g) {
        const int qq = 4 * t + 4 * kWideThreads * g;
        has[g] = qq < T && j0 + qq < n;
        full[g] = j0 + qq + 4 <= n;
        goff[g] = (has[g] || !PAIR) ? 4 * kWideThreads * g : -4 * t;
    }
    const int dj = j0 - c0;  // in [R, R + CPT - 1], a multiple of 4
    const uint32_t* pe_sm = P + 4 * t + dj + R + 1 - EA;  // 16-byte aligned
    const uint32_t* ps_sm = P + 4 * t + dj - R - SA;
    uint32_t* pw_sm = P + CPT * t;

    // Per iteration (rows r, r+1 for pairs): the rows entering and leaving the
    // window on the way to rows r+1 ([0]) and r+2 ([1], pairs only), and the
    // centre cells of the output groups.  Two sets, the current one and the one
    // being loaded for the next iteration, swap roles every iteration.
    uint32_t inA[STEP][NW], outA[STEP][NW], cenA[NW][STEP];
    uint32_t inB[STEP][NW], outB[STEP][NW], cenB[NW][STEP];
    const uint8_t* xc = X + (ptrdiff_t)H * pp + H + j0 + 4 * t;  // centre row 0, group 0
    auto load_rows = [&](int r, const uint8_t* pin, const uint8_t* pout, uint32_t(&in)[STEP][NW],
                         uint32_t(&out)[STEP][NW]) {
#pragma unroll
        for (int h = 0; h < STEP; ++h) {
            if (need && r + 1 + h < r1) {
                ld_cells<CPT>(pin + h * pp, in[h]);
                ld_cells<CPT>(pout + h * pp, out[h]);
            } else {
#pragma unroll
                for (int k = 0; k < NW; ++k) in[h][k] = out[h][k] = 0u;
            }
        }
    };
    auto load_centre = [&](int r, const uint8_t* pc, uint32_t(&c)[NW][STEP]) {
#pragma unroll
        for (int g = 0; g < NW; ++g)
#pragma unroll
            for (int h = 0; h < STEP; ++h)
                c[g][h] = (r < r1 && has[g]) ? __ldg((const uint32_t*)(pc + h * pp + 4 * kWideThreads * g)) : 0u;
    };
    load_rows(r0, colp + (ptrdiff_t)(H + r0 + R + 1) * pp, colp + (ptrdiff_t)(H + r0 - R) * pp, inA, outA);
    load_centre(r0, xc + (ptrdiff_t)r0 * pp, cenA);
    const ptrdiff_t sp = STEP * pp;
    const uint8_t* pin = colp + (ptrdiff_t)(H + r0 + STEP + R + 1) * pp;  // next iteration's rows
    const uint8_t* pout = colp + (ptrdiff_t)(H + r0 + STEP - R) * pp;
    const uint8_t* pc = xc + (ptrdiff_t)(r0 + STEP) * pp;
    uint8_t* py = Y + (ptrdiff_t)(H + r0) * pp + H + j0 + 4 * t;

    auto iteration = [&](const int b, int r, uint32_t(&in)[STEP][NW], uint32_t(&out)[STEP][NW],
                         uint32_t(&cen)[NW][STEP], uint32_t(&nin)[STEP][NW], uint32_t(&nout)[STEP][NW],
                         uint32_t(&ncen)[NW][STEP]) {
        load_rows(r + STEP, pin, pout, nin, nout);
        load_centre(r + STEP, pc, ncen);
        pin += sp;
        pout += sp;
        pc += sp;
        // one word per window column
        uint32_t W[CPT];
        uint32_t V1[2 * NW];
        if constexpr (PAIR) {
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                V1[2 * k] = V[2 * k];
                V1[2 * k + 1] = V[2 * k + 1];
                slide4(V1[2 * k], V1[2 * k + 1], in[0][k], out[0][k]);  // row r+1
                W[4 * k + 0] = prmt<0x5410>(V[2 * k], V1[2 * k]);
                W[4 * k + 1] = prmt<0x7632>(V[2 * k], V1[2 * k]);
                W[4 * k + 2] = prmt<0x5410>(V[2 * k + 1], V1[2 * k + 1]);
                W[4 * k + 3] = prmt<0x7632>(V[2 * k + 1], V1[2 * k + 1]);
            }
        } else {
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                W[4 * k + 0] = prmt<0x4410>(V[2 * k], 0u);
                W[4 * k + 1] = prmt<0x4432>(V[2 * k], 0u);
                W[4 * k + 2] = prmt<0x4410>(V[2 * k + 1], 0u);
                W[4 * k + 3] = prmt<0x4432>(V[2 * k + 1], 0u);
            }
        }
        // prefix sums over the window: local, warp, then the warp totals
#pragma unroll
        for (int i = 1; i < CPT; ++i) W[i] += W[i - 1];
        const uint32_t tot = W[CPT - 1];
        uint32_t incl = tot;
        incl = scan_up<1>(incl);
        incl = scan_up<2>(incl);
        incl = scan_up<4>(incl);
        incl = scan_up<8>(incl);
        incl = scan_up<16>(incl);
        if (lane == 31) wsum[b][wid] = incl;
        __syncthreads();
        // total of the warps before this one (4 or 8 warp totals, read as 16-byte vectors)
        const uint4 w0 = *(const uint4*)wsum[b];
        uint32_t wpre = (wid > 0 ? w0.x : 0u) + (wid > 1 ? w0.y : 0u) + (wid > 2 ? w0.z : 0u);
        if constexpr (kWideThreads == 256) {
            const uint4 w1 = *(const uint4*)(wsum[b] + 4);
            wpre += (wid > 3 ? w0.w : 0u) + (wid > 4 ? w1.x : 0u) + (wid > 5 ? w1.y : 0u) + (wid > 6 ? w1.z : 0u);
        }
        const uint32_t off = incl - tot + wpre;
#pragma unroll
        for (int k = 0; k < NW; ++k) {
            uint4 w;
            w.x = off + (k > 0 ? W[4 * k - 1] : 0u);
            w.y = off + W[4 * k];
            w.z = off + W[4 * k + 1];
            w.w = off + W[4 * k + 2];
            *(uint4*)(pw_sm + b * PS + 4 * k) = w;
        }
        if (t == kWideThreads - 1) P[b * PS + L] = off + tot;
        __syncthreads();

        // outputs: 4 consecutive columns (of row r, and of row r+1 for pairs) per group
        const bool second = r + 1 < r1;
#pragma unroll
        for (int g = 0; g < NW; ++g) {
            if constexpr (!PAIR) {
                if (!has[g]) break;
            }
            uint32_t pe[4], ps[4];
            lds4<EA>(pe_sm + b * PS + goff[g], pe);
            lds4<SA>(ps_sm + b * PS + goff[g], ps);
            uint8_t* yr = py + 4 * kWideThreads * g;
            const uint32_t cr = cen[g][0];
            uint32_t res[4];
            if constexpr (PAIR) {
                const uint32_t cr1 = cen[g][STEP - 1];
                uint32_t sw[4];
                sw[0] = prmt<0x8480>(cr, cr1);  // centre of column u: row r in bit 0, row r+1 in bit 16
                sw[1] = prmt<0x9591>(cr, cr1);
                sw[2] = prmt<0xA6A2>(cr, cr1);
                sw[3] = prmt<0xB7B3>(cr, cr1);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t ge = pe[u] - ps[u] + (sw[u] * dnlo + nlo0);
                    const uint32_t le = (sw[u] * dhih + hih0) - pe[u] + ps[u];
                    res[u] = ge & le & 0x80008000u;
                }
                const uint32_t t01 = prmt<0x7351>(res[0], res[1]);
                const uint32_t t23 = prmt<0x7351>(res[2], res[3]);
                const uint32_t o0 = prmt<0x5410>(t01, t23) >> 7;
                const uint32_t o1 = prmt<0x7632>(t01, t23) >> 7;
                if (has[g]) *(uint32_t*)yr = o0;
                if (has[g] && second) *(uint32_t*)(yr + pp) = o1;
            } else {
                uint32_t sw[4];
                sw[0] = prmt<0x4440>(cr, 0u);
                sw[1] = prmt<0x4441>(cr, 0u);
                sw[2] = prmt<0x4442>(cr, 0u);
                sw[3] = prmt<0x4443>(cr, 0u);
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const uint32_t ge = pe[u] - ps[u] + (sw[u] * dnlo + nlo0);
                    const uint32_t le = (sw[u] * dhih + hih0) - pe[u] + ps[u];
                    res[u] = ge & le & 0x80000000u;
                }
                const uint32_t t01 = prmt<0x7373>(res[0], res[1]);
                const uint32_t t23 = prmt<0x7373>(res[2], res[3]);
                const uint32_t o0 = prmt<0x5410>(t01, t23) >> 7;
                if (full[g]) {
                    *(uint32_t*)yr = o0;
                } else {
                    for (int u = 0; u < n - j0 - 4 * t - 4 * kWideThreads * g; ++u) yr[u] = (uint8_t)(o0 >> (8 * u));
                }
            }
        }
        py += sp;

        // slide to the next iteration's first row
        if constexpr (PAIR) {
#pragma unroll
            for (int k = 0; k < NW; ++k) {
                V[2 * k] = V1[2 * k];
                V[2 * k + 1] = V1[2 * k + 1];
                slide4(V[2 * k], V[2 * k + 1], in[1][k], out[1][k]);  // row r+2
            }
        } else {
#pragma unroll
            for (int k = 0; k < NW; ++k) slide4(V[2 * k], V[2 * k + 1], in[0][k], out[0][k]);
        }
    };

    // two iterations per trip, so that the load sets and the P buffers alternate
    // without copies
    for (int r = r0;;) {
        iteration(0, r, inA, outA, cenA, inB, outB, cenB);
        r += STEP;
        if (r >= r1) break;
        iteration(1, r, inB, outB, cenB, inA, outA, cenA);
        r += STEP;
        if (r >= r1) break;
    }
}

int plain_wide_cols_per_thread(int radius) { return radius <= 1018 ? 8 : 16; }

bool plain_generic_supported(int radius) { return radius >= 1 && radius <= 2038; }

template <bool PAIR, int CPT, int NT>
static cudaError_t launch_wide_rm(const Frame& cur, const Frame& nxt, const RuleScan& q, int band, int T,
                                  dim3 grid, cudaStream_t s) {
    const dim3 block(NT);
    const int n = cur.n, rows = cur.nrows();
    const uint8_t* x = cur.base;
    uint8_t* y = nxt.base;
    switch (q.radius & 3) {
        case 0: k_plain_wide<PAIR, CPT, 0, NT><<<grid, block, 0, s>>>(x, y, n, rows, cur.H, cur.pitch, band, T, q); break;
        case 1: k_plain_wide<PAIR, CPT, 1, NT><<<grid, block, 0, s>>>(x, y, n, rows, cur.H, cur.pitch, band, T, q); break;
        case 2: k_plain_wide<PAIR, CPT, 2, NT><<<grid, block, 0, s>>>(x, y, n, rows, cur.H, cur.pitch, band, T, q); break;
        default: k_plain_wide<PAIR, CPT, 3, NT><<<grid, block, 0, s>>>(x, y, n, rows, cur.H, cur.pitch, band, T, q); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_plain_generic(const Frame& cur, const Frame& nxt, const Rule& rule, int band_rows,
                                 cudaStream_t s) {
    const int n = cur.n, rows = cur.nrows(), R = rule.radius;
    if (!plain_generic_supported(R)) return cudaErrorInvalidValue;
    const bool pair = R <= kWidePairMaxRadius;
    const int cpt = plain_wide_cols_per_thread(R);
    if (cur.H < (int)round_up((size_t)R, (size_t)cpt) || (cur.H & 15) || (cur.pitch & 63))
        return cudaErrorInvalidValue;
    // T: outputs per tile, so that the prefix reads of the last output group,
    // up to P[T - 4 + (R + cpt - 1) + R + 4], stay inside P[0 .. NT cpt]
    const int nt = wide_threads(R);
    const int T = (nt * cpt - 2 * R - cpt + 1) & ~3;
    const int tiles = (n + T - 1) / T;
    // bands of 64 rows unless set: many CTAs per SM over the launch, so that
    // their 2R+1-row starts (independent loads) overlap other CTAs' scans
    // (measured on 16384^2 and 32768^2 for R = 6..200: within a few percent of
    // the best height everywhere)
    int band = band_rows > 0 ? band_rows : 64;
    band = std::max(band, (rows + 65534) / 65535);  // grid y limit
    band = std::min(band + (band & 1), std::max(rows + (rows & 1), 2));  // even: row pairs never straddle bands
    const dim3 grid(tiles, (rows + band - 1) / band);
    const RuleScan q = make_rule_scan(rule, pair);
    // R <= 90: row pairs, cpt 8, 128 threads; R <= 128: 128 threads; R <= 1018: cpt 8
    if (pair) return launch_wide_rm<true, 8, 128>(cur, nxt, q, band, T, grid, s);
    if (nt == 128) return launch_wide_rm<false, 8, 128>(cur, nxt, q, band, T, grid, s);
    return cpt == 8 ? launch_wide_rm<false, 8, 256>(cur, nxt, q, band, T, grid, s)
                    : launch_wide_rm<false, 16, 256>(cur, nxt, q, band, T, grid, s);
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

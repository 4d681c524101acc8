// k_tensor.cu -- K2: the LtL step as two banded 0/1 matrix products on the
// 5th-generation tensor cores (tcgen05, kind::i8, accumulators in TMEM), on a
// bit-packed grid (32 cells per 32-bit word, the PACK coding).
//
// This is the reference's AMX formulation (kezada94/CAT_cpu,
// src/CellularAutomata/Solvers/AMXSolver16.cpp:63-138 band tiles, :254-309 row
// sums X*B, :322-384 column sums + rule) re-designed for sm_100a:
//   - one CTA per SM walks a strided list of output tiles of Tr x Tc cells;
//   - unpack warps read the tile's packed input words (rows and words taken
//     modulo n: the torus wrap happens here, so no halo pass runs between
//     generations) and spread every bit to a byte in shared memory, in the
//     128-byte-swizzled K-major layout the MMA reads (128 rows x 256..512 columns);
//   - product 1:  H = X * B_h   (row sums; M = 128 tile rows, N = Tc, one MMA
//     per 32-column K step of the tile's window; u8 x u8 -> s32 in TMEM);
//   - H (<= 2R+1) is read back with tcgen05.ld, re-quantised to u8 and stored
//     as the MN-major B operand of
//   - product 2:  C = B_v * H   (column sums; M = 128, N = Tc, K = 128 per row
//     block) with B_v[m][k] = [m <= k <= m + 2R], so the reference's transposed
//     scatter between the two products (AMXSolver.cpp:321-325) disappears;
//   - epilogue: C is the box count including the centre; the birth/survival
//     interval rule (HostSolver.tpp:47-73, k = C - centre) runs on four 8-bit
//     (R <= 5), two 16-bit (R <= 90) or one 32-bit lane per register, and the
//     result bits are gathered straight into the output word.
//
// MMA count.  A tcgen05.mma costs the issuing warp a few tens of cycles plus a
// round trip through the barriers per batch, whatever its N, so a tile is done
// in few, wide MMAs: product 1 is one MMA of N = Tc per K step (5 at R <= 16),
// product 2 one per 32 bytes of K (4 per row block with u8 row sums, 8 with
// f16).  The band matrix B_h of a K step is the same matrix shifted by 32
// columns per step, so one Toeplitz matrix W of (KS + nchunks - 1) * 32 rows
// serves every step: the step's B descriptor starts 32 rows further up.  B_v
// is Toeplitz too and is stored the same way (G), which keeps it small enough
// for the f16 operands of R = 128.
//
// Column order.  A packed word w spreads to bytes with (w >> k) & 0x01010101,
// k = 0..7: register k holds cells k, 8+k, 16+k, 24+k.  The shared-memory tile
// keeps that order: within each 32-column group, byte position 4k+j holds the
// group's cell 8j+k (the permutation pi(4k+j) = 8j+k).  Product 1 contracts over
// the positions, so W's K index follows pi, and its N index (the column order
// of H and C within each 32-column chunk) is chosen so that the rule's result
// bits land in the output word's own bit order with one shift per register
// (sigma below).  No byte is moved to undo the permutation.
//
// Operand precision per radius (the exactness bound decides, not a tolerance):
// inputs are 0/1 and product 1 runs in kind::i8 (u8 x u8 -> s32).  The row
// sums H <= 2R+1 go back to the tensor core for product 2 as
//   u8   while 2R+1 <= 255 (R <= 127): kind::i8 again, C in s32;
//   f16  above (R = 128, H up to 257): kind::f16 with f32 accumulation.  H is
//        stored as the f16 of H + 1024, whose bit pattern is 0x6400 + H for
//        0 <= H <= 1024 (one integer add per two values), so C arrives as the
//        f32 of C + 1024 (2R+1) -- every row of B_v holds 2R+1 ones -- exact
//        while that stays below 2^24.  The rule compares raw f32 bit
//        patterns, which order non-negative floats like their values, against
//        thresholds shifted by the same constant.
// Box counts (2R+1)^2 decide the rule lanes: 8 bits while <= 127, 16 bits while
// < 2^15 (R <= 90), 32 bits above.
//
// Every wait on an mbarrier is bounded (globaltimer); on timeout the kernel
// sets a bit in an error word that the host reads (ltl_synchronize), waits
// (bounded) for its own MMAs, frees its TMEM and returns.
#include <algorithm>
#include <cstdio>
#include <cstring>

#include "ltl_kernels.h"
#include "tc_ptx.cuh"

namespace ltl {

using namespace tc;

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
constexpr int kAtomBytes = 128 * 128;  // one 128-row x 128-byte swizzle atom
constexpr int kMaxStages = 4;
constexpr int kTc = 128;     // output columns per tile
constexpr int kChunks = kTc / 32;
constexpr int kN1 = 32;      // one chunk = one output word
constexpr int kUnpackWarps = 4;       // one X row per unpack thread
constexpr int kRqWarps = 2 * 4;       // re-quantisation: two chunks per warp, four lane quarters
constexpr int kRuleChunks = 2;        // rule: two chunks per warp, four lane quarters
constexpr int kRuleWarps = kChunks / kRuleChunks * 4;
static_assert(kRuleChunks == 2, "the rule role handles two chunks per warp");
// warp 0: product-1 MMAs, warp 1: product-2 MMAs, 2..3: packed-word loads,
// 4..7: unpack, 8..15: re-quantisation, 16..23: rule.  A warp runs on
// scheduler warp % 4: each scheduler holds one unpack warp and one of the four
// lighter single roles (the two MMA issuers, the two loaders), so that no
// unpack warp -- all four gate every X stage -- shares its scheduler with more
// work than the others.
constexpr int kLoadWarp0 = 2;
constexpr int kLoadWarps = 2;
constexpr int kUnpackWarp0 = kLoadWarp0 + kLoadWarps;
constexpr int kRqWarp0 = kUnpackWarp0 + kUnpackWarps;
constexpr int kRuleWarp0 = kRqWarp0 + kRqWarps;
constexpr int kThreads = 32 * (kRuleWarp0 + kRuleWarps);
constexpr int kWordDepth = 4;  // packed-word ring of the unpack warps: units in flight
constexpr int kSmemLimit = 227 * 1024;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait
// Back-off between barrier tries: every waiting warp shares its scheduler
// with working ones, so none of them polls without a pause.
constexpr uint32_t kSleepNs = 32;
// TMEM columns: H in two buffers (units alternate), C in two buffers (tiles alternate)
__host__ __device__ constexpr uint32_t h_col(int buf) { return 128u * (uint32_t)buf; }
__host__ __device__ constexpr uint32_t c_col(int buf) { return 256u + 128u * (uint32_t)buf; }
// X in tensor memory (the XT form, NG <= 5): one H buffer (columns 0..127; the
// re-quantisation warps release it as soon as they have loaded it), C at
// columns 128..383, and the X stages of 8 NG columns each from column 384
// (three stages of 40 columns at NG = 5)
constexpr int kXtStages = 3;
__host__ __device__ constexpr uint32_t c_col_xt(int buf) { return 128u + 128u * (uint32_t)buf; }
__host__ __device__ constexpr uint32_t x_col(int stage, int ng) { return 384u + 8u * (uint32_t)(ng * stage); }

struct TcParams {
    const uint32_t* src;  // inner word (0, 0) of the current packed frame
    uint32_t* dst;        // inner word (0, 0) of the next packed frame
    long long wpitch;     // words per frame row
    int n, nw;
    int R, PADC;      // radius, column halo of a tile (16 mod 32)
    int Tr;           // output rows per tile
    int nb;           // 128-row X blocks per tile: product 2 contracts over 128 * nb rows
    int stages;       // X ring stages
    int tiles_x, tiles_y;
    uint32_t nlo0, dlo, hiH0, dhi;  // rule constants (lane-broadcast; d* = live minus dead, mod 2^32)
    unsigned int* err;
    unsigned long long wait_ns;
    int inject_missing_commit;  // test hook: product 1 of the first unit never signals
};

struct SmemLayout {
    int x_off, wr_off, hs_off, w_off, bv_off, bar_off, tmem_off, total;
};

enum Bar {
    X_FULL = 0,
    X_EMPTY = kMaxStages,
    H_FULL = 2 * kMaxStages,  // [2] per H buffer
    H_EMPTY = H_FULL + 2,     // [2]
    HS_FULL = H_EMPTY + 2,    // [2] per shared-memory H buffer
    HS_EMPTY = HS_FULL + 2,   // [2]
    C_FULL = HS_EMPTY + 2,    // [2] per C buffer
    C_EMPTY = C_FULL + 2,     // [2]
    DRAIN = C_EMPTY + 2,      // [2] per MMA-issuing warp
    W_FULL = DRAIN + 2,       // [kWordDepth] packed-word ring slots
    W_EMPTY = W_FULL + kWordDepth,
    NBARS = W_EMPTY + kWordDepth
};

// Rule lanes and product-2 operand type (the template parameter MODE):
enum TcMode {
    kLanes8 = 0,   // four 8-bit rule lanes per register, H as u8
    kLanes16 = 1,  // two 16-bit rule lanes, H as u8
    kLanes32 = 2,  // one 32-bit rule lane (s32 box counts), H as u8
    kF16 = 3       // one 32-bit rule lane on f32 bit patterns, H as f16 (kind::f16)
};
__host__ __device__ constexpr int h_bytes(int mode) { return mode == kF16 ? 2 : 1; }
// K rows of one product-2 MMA (32 bytes of K either way)
__host__ __device__ constexpr int k2_rows(int mode) { return mode == kF16 ? 16 : 32; }
// f16 row sums are stored as H + kF16Offset (see the header)
constexpr int kF16Offset = 1024;

// Words per X row in the packed-word ring: the NG + 1 words a row needs, rounded
// up to whole 16-byte chunks (rows are 16-byte aligned in the ring).
__host__ __device__ constexpr int ring_row_words(int ng) { return (ng + 1 + 3) / 4 * 4; }

// W: (ng + kChunks - 1) * 32 rows (the N index) x 32 bytes (the K index of one step)
__host__ __device__ constexpr int w_rows(int ng) { return 32 * (ng + kChunks - 1); }
__host__ __device__ constexpr int atoms_for(int ng) { return (ng + 3) / 4; }
// G, the Toeplitz store of B_v: 128 + k2 (T - 1) rows x 32 bytes, T = 128 nb / k2
// product-2 K steps per tile; step t reads rows k2 (T - 1 - t) .. + 127.
__host__ __device__ constexpr int g_rows(int nb, int mode) {
    return 128 + k2_rows(mode) * (128 * nb / k2_rows(mode) - 1);
}

__host__ __device__ inline SmemLayout smem_layout(int stages, int ng, int nb, bool fast, int mode, bool xt = false) {
    SmemLayout L{};
    int o = 0;
    L.x_off = o;
    o += xt ? 0 : stages * atoms_for(ng) * kAtomBytes;  // 1024-aligned stages (none when X is in TMEM)
    L.wr_off = o;
    o += fast ? kWordDepth * 128 * ring_row_words(ng) * 4 : 0;  // packed words of the next units
    L.hs_off = o;
    o += 2 * 128 * kTc * h_bytes(mode);        // H (u8 or f16), MN-major, two buffers
    L.w_off = o;
    o += 32 * w_rows(ng);                      // W
    L.bv_off = o;
    o += 32 * g_rows(nb, mode);                // G (B_v)
    o = (o + 7) & ~7;
    L.bar_off = o;
    o += NBARS * 8;
    L.tmem_off = o;
    o += 16;
    L.total = o;
    return L;
}

// Column permutation inside a 32-column group: byte position q holds cell pi(q).
__host__ __device__ constexpr int perm_pi(int q) { return 8 * (q & 3) + (q >> 2); }
// Output cell (within a 32-column chunk) of accumulator column n.
__host__ __device__ constexpr int perm_sigma(int n, int mode) {
    return mode == kLanes8 ? perm_pi(n) : mode == kLanes16 ? 16 * (n & 1) + (n >> 1) : n;
}

__device__ __forceinline__ int wrap_slow(int v, int n) {
    int r = v % n;
    return r < 0 ? r + n : r;
}

// Cells a .. a+31 (modulo n) of one packed row, bit b = cell a+b; 0 <= a < n.
// Bits past n in the row's last word are ignored.
__device__ __forceinline__ uint32_t fetch32(const uint32_t* __restrict__ row, int a, int n) {
    if (n >= 32) {
        const int w0 = a >> 5, s = a & 31;
        // row[w0 + 1] may be the right halo word (w0 = nw - 1): its bits are masked below
        uint32_t v = __funnelshift_r(__ldg(row + w0), __ldg(row + w0 + 1), s);
        const int valid = n - a;
        if (valid < 32) v = (v & ((1u << valid) - 1u)) | (__ldg(row) << valid);
        return v;
    }
    const uint32_t w = __ldg(row);
    uint32_t v = 0u;
    int c = a;
    for (int b = 0; b < 32; ++b) {
        v |= ((w >> c) & 1u) << b;
        if (++c == n) c = 0;
    }
    return v;
}

// Position in this CTA's stream of work, advanced incrementally (no integer
// division in the loops).  Tiles t = blockIdx.x + j * gridDim.x, units (X
// blocks) u = j * nb + b.  The strides live in a Walk shared by the cursors
// of a thread.
struct Walk {
    int step_x, step_y, tiles_x, nb, stages;
    __device__ explicit Walk(const TcParams& p) {
        tiles_x = p.tiles_x;
        nb = p.nb;
        stages = p.stages;
        step_y = (int)gridDim.x / tiles_x;
        step_x = (int)gridDim.x - step_y * tiles_x;
    }
};

struct Cursor {
    int u, b, j;  // unit, row block within the tile, tile count
    int st, sph;  // X ring stage of unit u and its phase parity ((u / stages) & 1)
    int ty, tx;   // tile coordinates

    __device__ void init(const Walk& w) {
        u = b = j = st = sph = 0;
        ty = (int)blockIdx.x / w.tiles_x;
        tx = (int)blockIdx.x - ty * w.tiles_x;
    }
    __device__ void next(const Walk& w) {
        ++u;
        if (++st == w.stages) {
            st = 0;
            sph ^= 1;
        }
        if (++b == w.nb) {
            b = 0;
            ++j;
            tx += w.step_x;
            ty += w.step_y;
            if (tx >= w.tiles_x) {
                tx -= w.tiles_x;
                ++ty;
            }
        }
    }
};

// The work is a stream of units u = tile j * nb + row block b.  Per unit the
// unpack warps fill one X stage, one MMA warp runs product 1 into H buffer
// u % 2, the epilogue re-quantises H to shared-memory buffer u % 2, and
// another MMA warp adds product 2, B_v[:, 128b ..] * H, to C buffer j % 2.
// After a tile's last block the epilogue applies the rule to C.  With two
// buffers at every hand-over and the epilogue re-quantising unit u before it
// applies the rule to unit u - 1, the tensor core has the next unit's product 1
// queued while the epilogue finishes the previous one.
//
// MODE: rule lanes and product-2 operand type (TcMode); FAST: n % 32 == 0 and
// large enough that rows and words wrap with one correction; NG: product-1 K
// steps = X groups of 32 columns per row.
template <int MODE, bool FAST, int NG, bool XT>
__global__ void __launch_bounds__(kThreads, 1) k_tensor_step(const __grid_constant__ TcParams p) {
    static_assert(!XT || (FAST && NG <= 5), "X in tensor memory: FAST tiles with at most 5 K steps");
    constexpr int kHBufs = XT ? 1 : 2;  // H buffers in TMEM (C has two either way)
    constexpr int kCBufs = 2;
    auto ccol = [](int buf) -> uint32_t { return XT ? c_col_xt(buf) : c_col(buf); };
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    constexpr int ATOMS = atoms_for(NG);
    constexpr int HB = h_bytes(MODE);   // bytes per H value in shared memory
    constexpr int K2 = k2_rows(MODE);   // K rows per product-2 MMA
    constexpr int S2 = 128 / K2;        // product-2 MMAs per row block
    const int nb = p.nb, S = p.stages, R = p.R;
    const SmemLayout L = smem_layout(S, NG, nb, FAST, MODE, XT);
    uint8_t* xs = smem + L.x_off;
    uint8_t* hs = smem + L.hs_off;
    uint8_t* wm = smem + L.w_off;
    uint8_t* bv = smem + L.bv_off;
    uint64_t* bars = (uint64_t*)(smem + L.bar_off);
    uint32_t* tmem_slot = (uint32_t*)(smem + L.tmem_off);
    constexpr int kXB = ATOMS * kAtomBytes;  // bytes of one X stage

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ntiles = p.tiles_x * p.tiles_y;
    const int mine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int units = mine * nb;
    constexpr uint32_t kTmemCols = 512;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(&bars[X_FULL + i], kUnpackWarps);
            mbar_init(&bars[X_EMPTY + i], 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(&bars[H_FULL + i], 1);
            mbar_init(&bars[H_EMPTY + i], kRqWarps);
            mbar_init(&bars[HS_FULL + i], kRqWarps);
            mbar_init(&bars[HS_EMPTY + i], 1);
            mbar_init(&bars[C_FULL + i], 1);
            mbar_init(&bars[C_EMPTY + i], kRuleWarps);
            mbar_init(&bars[DRAIN + i], 1);
        }
        for (int i = 0; i < kWordDepth; ++i) {
            mbar_init(&bars[W_FULL + i], 32 * kLoadWarps);  // one cp.async-tracking arrival per loader thread
            mbar_init(&bars[W_EMPTY + i], kUnpackWarps);
        }
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
    // W (B operand of product 1, K-major, no swizzle: [m / 8][k / 16][8][16 bytes],
    // m < w_rows, k < 32).  Row m belongs to chunk offset D = NG - 1 - m / 32 and
    // accumulator column m % 32 of that chunk; byte k is position k of a group (cell
    // pi(k)).  K step s reads rows [32 (NG - 1 - s), + kTc): there, accumulator
    // column n of chunk c = n / 32 meets X group s, D = s - c.
    for (int idx = tid; idx < w_rows(NG) * 32; idx += kThreads) {
        const int m = idx >> 5, k = idx & 31;
        const int D = NG - 1 - (m >> 5);
        const int d = 32 * D + perm_pi(k) - p.PADC - perm_sigma(m & 31, MODE);
        wm[((m >> 3) * 2 + (k >> 4)) * 128 + (m & 7) * 16 + (k & 15)] = (d >= -R && d <= R) ? 1 : 0;
    }
    // G, the A operand of product 2 (K-major, no swizzle: [i / 8][two 16-byte
    // halves][8][16 bytes], like W).  B_v[m][k] = [m <= k <= m + 2R] depends on
    // k - m only, so product-2 K step t (rows K2 t .. K2 t + K2 - 1 of the
    // tile's 128 nb X rows) is the 128-row window of G from row K2 (T2 - 1 - t):
    // G[i][kk] = [0 <= K2 (T2 - 1) + kk - i <= 2R].  Entries are u8 1 or f16 1.0.
    {
        const int T2 = S2 * nb;
        const int grows = g_rows(nb, MODE);
        for (int idx = tid; idx < grows * 2; idx += kThreads) {
            const int i = idx >> 1, half = idx & 1;  // row, 16-byte half of the row's 32 bytes
            uint32_t w[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                uint32_t v = 0;
                if (MODE == kF16) {
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        const int d = K2 * (T2 - 1) + (8 * half + 2 * q + e) - i;
                        v |= (d >= 0 && d <= 2 * R) ? (0x3C00u << (16 * e)) : 0u;
                    }
                } else {
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int d = K2 * (T2 - 1) + (16 * half + 4 * q + e) - i;
                        v |= (uint32_t)(d >= 0 && d <= 2 * R) << (8 * e);
                    }
                }
                w[q] = v;
            }
            *(uint4*)(bv + (((i >> 3) * 2 + half) * 128 + (i & 7) * 16)) = make_uint4(w[0], w[1], w[2], w[3]);
        }
    }
    fence_proxy_async();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp < kLoadWarp0) {
        // --------------------------- MMA issuers ----------------------------
        // Warp 0 issues product 1 of every unit, warp 1 product 2, so that the
        // tensor core queue gets the next unit's product 1 while product 2 waits
        // for the epilogue, and the reverse.  Each warp runs its loop whole
        // (waits and descriptor arithmetic are warp-uniform); its lane 0 alone
        // issues the MMAs and the commits, so that every commit tracks every MMA
        // of that warp before it.  Descriptors are 64-bit bases plus
        // start-address offsets in 16-byte units (within the 14-bit field).
        const bool leader = lane == 0;
        auto wait = [&](uint64_t* bar, uint32_t ph) -> bool {
            return __all_sync(0xffffffffu, mbar_wait(bar, ph, p.wait_ns, kSleepNs));
        };
        const Walk wk(p);
        Cursor c;
        c.init(wk);
        bool ok = true;
        if (warp == 0) {
            // product 1 of unit c: H(u % 2) = X(u) * B_h
            constexpr uint32_t id1 = idesc_u8(kTc, false);
            const uint64_t xd0 = desc_k_sw128(smem_u32(xs));
            const uint64_t wd0 = desc_noswz(smem_u32(wm), 128, 256);
            for (; c.u < units && ok; c.next(wk)) {
                const int hb = c.u % kHBufs;
                ok = wait(&bars[X_FULL + c.st], (uint32_t)c.sph);
                if (ok && c.u >= kHBufs) ok = wait(&bars[H_EMPTY + hb], (uint32_t)(((c.u / kHBufs) - 1) & 1));
                if (!ok) break;
                fence_after();
                if (leader) {
                    const uint64_t xs0 = xd0 + (uint64_t)((c.st * kXB) >> 4);
#pragma unroll
                    for (int s = 0; s < NG; ++s) {
                        // X group s: atom s / 4, byte 32 (s % 4) of its rows; W from row 32 (NG - 1 - s)
                        const uint64_t ad = xs0 + (uint64_t)((s >> 2) * (kAtomBytes >> 4) + (s & 3) * 2);
                        const uint64_t bd = wd0 + (uint64_t)((NG - 1 - s) * 4 * (256 >> 4));
                        if constexpr (XT) {
                            mma_i8_ts(tmem + h_col(hb), tmem + x_col(c.st, NG) + 8u * (uint32_t)s, bd, id1,
                                      s > 0 ? 1u : 0u);
                        } else {
                            mma_i8(tmem + h_col(hb), ad, bd, id1, s > 0 ? 1u : 0u);
                        }
                    }
                    if (!(p.inject_missing_commit && c.u == 0)) mma_commit(&bars[H_FULL + hb]);
                    mma_commit(&bars[X_EMPTY + c.st]);  // the stage is free once product 1 has read it
                }
                __syncwarp();
            }
        } else {
            // product 2 of unit c: C(j % 2) (+)= B_v[:, 128b ..] * H(u), H(u) from
            // shared-memory buffer u % 2
            constexpr uint32_t id2 = MODE == kF16 ? idesc_f16(kTc, true) : idesc_u8(kTc, true);
            const uint64_t gd0 = desc_noswz(smem_u32(bv), 128, 256);
            const uint64_t hsd0 = desc_noswz(smem_u32(hs), 128, 128 * 16);
            const int T2 = S2 * nb;
            for (; c.u < units && ok; c.next(wk)) {
                const int hb = c.u & 1, cb = c.j % kCBufs;
                ok = wait(&bars[HS_FULL + hb], (uint32_t)((c.u >> 1) & 1));
                if (ok && c.b == 0 && c.j >= kCBufs)
                    ok = wait(&bars[C_EMPTY + cb], (uint32_t)(((c.j / kCBufs) - 1) & 1));
                if (!ok) break;
                fence_after();
                if (leader) {
                    const uint64_t hd = hsd0 + (uint64_t)((hb * 128 * kTc * HB) >> 4);
                    // K step t = S2 b + s starts at G row K2 (T2 - 1 - t): 32 K2 bytes per K2 rows
                    const uint64_t gd = gd0 + (uint64_t)(2 * K2 * (T2 - 1 - S2 * c.b));
#pragma unroll
                    for (int s = 0; s < S2; ++s) {
                        const uint64_t ad = gd - (uint64_t)(2 * K2 * s);
                        const uint64_t bd = hd + (uint64_t)((s * K2 * 16) >> 4);
                        const uint32_t acc = (c.b > 0 || s > 0) ? 1u : 0u;
                        if constexpr (MODE == kF16) {
                            mma_f16(tmem + ccol(cb), ad, bd, id2, acc);
                        } else {
                            mma_i8(tmem + ccol(cb), ad, bd, id2, acc);
                        }
                    }
                    mma_commit(&bars[HS_EMPTY + hb]);
                    if (c.b == nb - 1) mma_commit(&bars[C_FULL + cb]);
                }
                __syncwarp();
            }
        }
        if (!ok && leader) atomicOr(p.err, 2u);
        // never leave with an MMA in flight (TMEM is freed below)
        if (leader) mma_commit(&bars[DRAIN + warp]);
        __syncwarp();
        if (!__all_sync(0xffffffffu, mbar_wait(&bars[DRAIN + warp], 0u, p.wait_ns)) && leader) atomicOr(p.err, 32u);
    } else if (warp < kUnpackWarp0) {
        // --------------------------- packed words ---------------------------
        // FAST tiles: the NG + 1 packed words of every X row of a unit (group g =
        // upper half of word g, lower half of word g + 1) go by cp.async into a
        // ring of kWordDepth units, row-major (ring_row_words per row); loader
        // warp lw takes rows 64 lw .. 64 lw + 63.  Where the unit's words start on
        // a 16-byte boundary and do not cross the torus seam (every interior tile
        // when R <= 16) a row is whole 16-byte copies, else one copy per word.
        // The ring slot's barrier tracks the copies themselves
        // (cp.async.mbarrier.arrive), so the unpack warps, whose proxy fences wait
        // for every memory access of their own still in flight, never have a
        // global load outstanding.
        if (FAST) {
            constexpr int NW1 = NG + 1;
            constexpr int RW = ring_row_words(NG);
            uint32_t* ring = (uint32_t*)(smem + L.wr_off);  // [kWordDepth][128][RW]
            const int row_base = 64 * (warp - kLoadWarp0);
            const Walk wk(p);
            Cursor c;
            c.init(wk);
            bool ok = true;
            for (; c.u < units; c.next(wk)) {
                const int slot = c.u & (kWordDepth - 1);
                if (c.u >= kWordDepth) {
                    ok = __all_sync(0xffffffffu, mbar_wait(&bars[W_EMPTY + slot],
                                                           (uint32_t)(((c.u / kWordDepth) - 1) & 1), p.wait_ns,
                                                           kSleepNs));
                    if (!ok) break;
                }
                uint32_t* d = ring + slot * 128 * RW;
                int wi0 = (c.tx * kTc - p.PADC - 16) >> 5;  // word holding X column 0
                if (wi0 < 0) wi0 += p.nw;
                // whole 16-byte chunks: aligned start (rows are 16-byte aligned:
                // wpitch % 4 == 0), no seam inside the needed words, the chunks'
                // extra words still inside the frame row
                const bool vec = ((uintptr_t)(p.src + wi0) & 15) == 0 && (p.wpitch & 3) == 0 &&
                                 wi0 + NW1 <= p.nw && wi0 + RW <= p.wpitch - 1;
                const int gr0 = c.ty * p.Tr - R + 128 * c.b;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const int row = row_base + lane + 32 * i;
                    int gr = gr0 + row;
                    if (gr < 0) gr += p.n;
                    else if (gr >= p.n) gr -= p.n;
                    const uint32_t* rp = p.src + (size_t)gr * (size_t)p.wpitch;
                    uint32_t* dr = d + row * RW;
                    if (vec) {
#pragma unroll
                        for (int k = 0; k < RW; k += 4) cp_async16(dr + k, rp + wi0 + k);
                    } else {
                        int wi = wi0;
#pragma unroll
                        for (int k = 0; k < NW1; ++k) {
                            cp_async4(dr + k, rp + wi);
                            if (++wi == p.nw) wi = 0;
                        }
                    }
                }
                cp_async_mbar_arrive(&bars[W_FULL + slot]);
            }
            cp_async_wait<0>();
            if (!ok && lane == 0) atomicOr(p.err, 64u);
        }
    } else if (warp < kRqWarp0) {
        // ------------------------------ unpack ------------------------------
        // Thread `row` (0..127) fills X row `row` of every stage: NG groups of 32
        // columns of one packed row.
        const int row = tid - 32 * kUnpackWarp0;
        const int sw = row & 7;
        const Walk wk(p);
        Cursor c;  // the unit being stored
        c.init(wk);
        bool ok = true;
        // spreads X row `row` of unit c to the stage: group g from x_of(g)
        auto store = [&](const Cursor& cc, auto x_of) -> bool {
            if (cc.u >= S) {
                bool wt = true;
                if (lane == 0) wt = mbar_wait(&bars[X_EMPTY + cc.st], (uint32_t)(cc.sph ^ 1), p.wait_ns, kSleepNs);
                if (!__shfl_sync(0xffffffffu, wt, 0)) return false;
            }
            if constexpr (XT) {
                // X row `row` is TMEM lane `row` (this warp's lane quarter, warp % 4):
                // group g is 8 columns, four K bytes per column
                fence_after();
                const uint32_t xa = tmem + ((uint32_t)(32 * (warp & 3)) << 16) + x_col(cc.st, NG);
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    const uint32_t x = x_of(g);
                    uint32_t v[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[k] = (x >> k) & 0x01010101u;
                    tmem_st8(xa + 8u * (uint32_t)g, v);
                }
                tmem_wait_st();
                fence_before();
            } else {
                uint8_t* xrow = xs + cc.st * kXB + row * 128;
#pragma unroll
                for (int g = 0; g < NG; ++g) {
                    const uint32_t x = x_of(g);
                    uint32_t v[8];
#pragma unroll
                    for (int k = 0; k < 8; ++k) v[k] = (x >> k) & 0x01010101u;
                    uint8_t* ap = xrow + (g >> 2) * kAtomBytes;
                    const int ch = 2 * (g & 3);
                    *(uint4*)(ap + ((ch ^ sw) << 4)) = make_uint4(v[0], v[1], v[2], v[3]);
                    *(uint4*)(ap + (((ch + 1) ^ sw) << 4)) = make_uint4(v[4], v[5], v[6], v[7]);
                }
                fence_proxy_async();
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars[X_FULL + cc.st]);
            return true;
        };
        if (FAST) {
            // words from the loader warps' ring (see above): this row's, as 16-byte vectors
            constexpr int NW1 = NG + 1;
            constexpr int RW = ring_row_words(NG);
            const uint32_t* ring = (const uint32_t*)(smem + L.wr_off) + row * RW;  // [kWordDepth][128][RW]
            for (; c.u < units; c.next(wk)) {
                const int slot = c.u & (kWordDepth - 1);
                ok = __all_sync(0xffffffffu, mbar_wait(&bars[W_FULL + slot], (uint32_t)((c.u / kWordDepth) & 1),
                                                       p.wait_ns, kSleepNs));
                if (!ok) break;
                const uint4* d = (const uint4*)(ring + slot * 128 * RW);
                uint32_t w[RW];
#pragma unroll
                for (int k = 0; k < RW / 4; ++k) {
                    const uint4 v = d[k];
                    w[4 * k] = v.x;
                    w[4 * k + 1] = v.y;
                    w[4 * k + 2] = v.z;
                    w[4 * k + 3] = v.w;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars[W_EMPTY + slot]);
                ok = store(c, [&](int g) { return prmt(w[g], w[g + 1], 0x5432u); });
                if (!ok) break;
            }
        } else {
            uint32_t w[NG];
            // the NG groups of X row `row` of unit cc, rows and columns taken modulo n
            auto gather = [&](const Cursor& cc) {
                const int gr0 = cc.ty * p.Tr - R + 128 * cc.b + row;
                const uint32_t* rp = p.src + (size_t)wrap_slow(gr0, p.n) * (size_t)p.wpitch;
                int a = wrap_slow(cc.tx * kTc - p.PADC, p.n);
#pragma unroll
                for (int k = 0; k < NG; ++k) {
                    w[k] = fetch32(rp, a, p.n);
                    a += 32;
                    while (a >= p.n) a -= p.n;
                }
            };
            for (; c.u < units; c.next(wk)) {
                gather(c);
                ok = store(c, [&](int g) { return w[g]; });
                if (!ok) break;
            }
        }
        if (!ok && lane == 0) atomicOr(p.err, 4u);
    } else {
        // ---------------------------- epilogue ------------------------------
        // TMEM lane quarter q (= warp % 4, the lanes a warp may access) holds tile
        // rows 32q .. 32q + 31, one per thread.
        const int q = warp & 3;
        const int m = q * 32 + lane;  // tile row (TMEM lane)
        auto wait_all = [&](uint64_t* bar, uint32_t ph) -> bool {
            const bool wt = mbar_wait(bar, ph, p.wait_ns, kSleepNs);
            return __all_sync(0xffffffffu, wt);
        };
        const Walk wk(p);
        Cursor c;
        c.init(wk);
        bool ok = true;
        if (warp < kRuleWarp0) {
            // re-quantisation: H(u) -> u8 in shared-memory buffer u % 2 (MN-major B
            // operand of product 2), chunks 2h and 2h + 1 of this lane quarter
            const int h = (warp - kRqWarp0) >> 2;
            const uint32_t lane_off = ((uint32_t)(q * 32) << 16) + (uint32_t)(2 * kN1 * h);
            for (; c.u < units && ok; c.next(wk)) {
                const int hb = c.u & 1;           // shared-memory H buffer (two)
                const int tb = c.u % kHBufs;      // TMEM H buffer
                ok = wait_all(&bars[H_FULL + tb], (uint32_t)((c.u / kHBufs) & 1));
                if (!ok) break;
                fence_after();
                uint32_t va[16], vb[16];
                tmem_ld32p(tmem + lane_off + h_col(tb), va);
                tmem_ld32p(tmem + lane_off + h_col(tb) + kN1, vb);
                tmem_wait_2x16(va, vb);
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars[H_EMPTY + tb]);
                // product 2 of unit u - 2 has read the buffer
                if (c.u >= 2) ok = wait_all(&bars[HS_EMPTY + hb], (uint32_t)(((c.u >> 1) - 1) & 1));
                if (!ok) break;
                // 16 bytes of one row m per store; consecutive N groups of 16 bytes
                // are 128 rows x 16 bytes apart
                uint8_t* hsb = hs + hb * 128 * kTc * HB + m * 16;
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const uint32_t* v = e ? vb : va;
                    if constexpr (MODE == kF16) {
                        // register r = columns 2r, 2r + 1 as 16-bit halves; + 0x6400 in
                        // each half gives the f16 of H + 1024 (H <= 1024: no carry out)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            uint4 wv;
                            wv.x = v[4 * j + 0] + 0x64006400u;
                            wv.y = v[4 * j + 1] + 0x64006400u;
                            wv.z = v[4 * j + 2] + 0x64006400u;
                            wv.w = v[4 * j + 3] + 0x64006400u;
                            *(uint4*)(hsb + (4 * (2 * h + e) + j) * 128 * 16) = wv;
                        }
                    } else {
#pragma unroll
                        for (int hh = 0; hh < 2; ++hh) {
                            uint4 wv;
                            wv.x = prmt(v[8 * hh + 0], v[8 * hh + 1], 0x6420u);
                            wv.y = prmt(v[8 * hh + 2], v[8 * hh + 3], 0x6420u);
                            wv.z = prmt(v[8 * hh + 4], v[8 * hh + 5], 0x6420u);
                            wv.w = prmt(v[8 * hh + 6], v[8 * hh + 7], 0x6420u);
                            *(uint4*)(hsb + (4 * h + 2 * e + hh) * 128 * 16) = wv;
                        }
                    }
                }
                fence_proxy_async();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars[HS_FULL + hb]);
            }
        } else {
            // rule: chunks grp0 and grp0 + 1 of C(j % 2) for every tile j, bits
            // straight into the output words
            const int grp0 = ((warp - kRuleWarp0) >> 2) * kRuleChunks;
            const uint32_t lane_off = ((uint32_t)(q * 32) << 16) + (uint32_t)(kN1 * grp0);
            const uint32_t nlo0 = p.nlo0, dlo = p.dlo, hiH0 = p.hiH0, dhi = p.dhi;
            // output word e of this thread in the tile of cursor c (offset, or -1)
            auto out_at = [&](const Cursor& cc, int e) -> long long {
                const int gi = cc.ty * p.Tr + m;
                const int wi = cc.tx * kChunks + grp0 + e;
                if (m >= p.Tr || gi >= p.n || wi >= p.nw) return -1;
                return (long long)gi * p.wpitch + wi;
            };
            // one output word from a chunk loaded with .pack::16b (8- and 16-bit lanes)
            auto rule16 = [&](const uint32_t (&v)[16], uint32_t cw) -> uint32_t {
                uint32_t acc = 0u;
                if constexpr (MODE == kLanes8) {
                    // accumulator column 4k+j = output cell 8j+k: four box counts per
                    // register, bit 7 of each byte lane = the rule's result
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const uint32_t B4 = prmt(v[2 * k], v[2 * k + 1], 0x6420u);
                        const uint32_t s4 = (cw >> k) & 0x01010101u;
                        const uint32_t ge = (B4 + nlo0) + s4 * dlo;  // bit 7: B >= lo(s)
                        const uint32_t le = (hiH0 + s4 * dhi) - B4;  // bit 7: B <= hi(s)
                        acc |= (ge & le & 0x80808080u) >> (7 - k);
                    }
                } else {
                    // accumulator column 2r+e = output cell 16e+r: two box counts per
                    // register, bit 15 of each 16-bit lane = the rule's result
#pragma unroll
                    for (int k = 0; k < 16; ++k) {
                        const uint32_t s2 = (cw >> k) & 0x00010001u;
                        const uint32_t ge = (v[k] + nlo0) + s2 * dlo;
                        const uint32_t le = (hiH0 + s2 * dhi) - v[k];
                        acc |= (ge & le & 0x80008000u) >> (15 - k);
                    }
                }
                return acc;
            };
            // one output word from a chunk of 32-bit counts: accumulator column n =
            // output cell n, bit 31 = the rule's result (s32 counts, or the f32 bits
            // of the count plus a constant)
            auto rule32 = [&](const uint32_t (&v0)[16], const uint32_t (&v1)[16], uint32_t cw) -> uint32_t {
                uint32_t acc = 0u;
#pragma unroll
                for (int k = 0; k < 32; ++k) {
                    const uint32_t B = k < 16 ? v0[k] : v1[k - 16];
                    const uint32_t s1 = (cw >> k) & 1u;
                    const uint32_t ge = (B + nlo0) + s1 * dlo;
                    const uint32_t le = (hiH0 + s1 * dhi) - B;
                    acc |= ((ge & le) >> 31) << k;
                }
                return acc;
            };
            // the centre words (the output words' own cells in the current grid) of
            // the next tile are loaded while this one is processed
            long long at0 = mine > 0 ? out_at(c, 0) : -1, at1 = mine > 0 ? out_at(c, 1) : -1;
            uint32_t cw0 = at0 >= 0 ? __ldg(p.src + at0) : 0u, cw1 = at1 >= 0 ? __ldg(p.src + at1) : 0u;
            for (int j = 0; j < mine && ok; ++j) {
                const int cb = j % kCBufs;
                ok = wait_all(&bars[C_FULL + cb], (uint32_t)((j / kCBufs) & 1));
                if (!ok) break;
                fence_after();
                uint32_t acc0, acc1;
                if constexpr (MODE >= kLanes32) {
                    // 64 values do not fit the registers at once: one chunk after the
                    // other, the C buffer released after the second chunk's loads
                    uint32_t v0[16], v1[16];
                    tmem_ld16(tmem + lane_off + ccol(cb), v0);
                    tmem_ld16(tmem + lane_off + ccol(cb) + 16, v1);
                    tmem_wait_2x16(v0, v1);
                    acc0 = rule32(v0, v1, cw0);
                    tmem_ld16(tmem + lane_off + ccol(cb) + kN1, v0);
                    tmem_ld16(tmem + lane_off + ccol(cb) + kN1 + 16, v1);
                    tmem_wait_2x16(v0, v1);
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars[C_EMPTY + cb]);
                    acc1 = rule32(v0, v1, cw1);
                } else {
                    uint32_t va[16], vb[16];
                    tmem_ld32p(tmem + lane_off + ccol(cb), va);
                    tmem_ld32p(tmem + lane_off + ccol(cb) + kN1, vb);
                    tmem_wait_2x16(va, vb);
                    fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&bars[C_EMPTY + cb]);
                    acc0 = rule16(va, cw0);
                    acc1 = rule16(vb, cw1);
                }
                if (at0 >= 0) p.dst[at0] = acc0;
                if (at1 >= 0) p.dst[at1] = acc1;
                for (int b = 0; b < nb; ++b) c.next(wk);
                at0 = j + 1 < mine ? out_at(c, 0) : -1;
                at1 = j + 1 < mine ? out_at(c, 1) : -1;
                cw0 = at0 >= 0 ? __ldg(p.src + at0) : 0u;
                cw1 = at1 >= 0 ? __ldg(p.src + at1) : 0u;
            }
        }
        if (!ok && lane == 0) atomicOr(p.err, 8u);
    }
    fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
using TcKernel = void (*)(TcParams);

struct TensorPlan {
    TcParams prm[2];  // source frame a -> b, b -> a
    TcKernel kernel;
    int smem_bytes;
    int grid;
    int operand_bits;  // product-2 operand: 8 (u8) or 16 (f16)
    unsigned int* err;
};

// The instantiations that exist (R ranges as tensor_geometry lays them out):
//   R <= 5       8-bit lanes,  5 K steps
//   R 6..16      16-bit lanes, 5 K steps
//   R 17..48     16-bit lanes, 7 K steps (row blocks from R = 33)
//   R 49..80     16-bit lanes, 9 K steps
//   R 81..90     16-bit lanes, 11 K steps
//   R 91..112    32-bit lanes, 11 K steps
//   R 113..127   32-bit lanes, 13 K steps
//   R 128        32-bit lanes on f32 counts, f16 product 2, 13 K steps
template <int MODE, int NG>
static TcKernel pick_fast(bool fast) {
    return fast ? k_tensor_step<MODE, true, NG, false> : k_tensor_step<MODE, false, NG, false>;
}
// X in tensor memory: FAST tiles of 8- and 16-bit rule lanes with 5 K steps (R <= 16)
static bool tensor_xt(int mode, bool fast, int ng) { return fast && ng == 5 && mode <= kLanes16; }
static TcKernel pick_kernel(int mode, bool fast, int ng) {
    if (tensor_xt(mode, fast, ng))
        return mode == kLanes8 ? k_tensor_step<kLanes8, true, 5, true> : k_tensor_step<kLanes16, true, 5, true>;
    switch (mode) {
        case kLanes8: return ng == 5 ? pick_fast<kLanes8, 5>(fast) : nullptr;
        case kLanes16:
            switch (ng) {
                case 5: return pick_fast<kLanes16, 5>(fast);
                case 7: return pick_fast<kLanes16, 7>(fast);
                case 9: return pick_fast<kLanes16, 9>(fast);
                case 11: return pick_fast<kLanes16, 11>(fast);
                default: return nullptr;
            }
        case kLanes32:
            switch (ng) {
                case 11: return pick_fast<kLanes32, 11>(fast);
                case 13: return pick_fast<kLanes32, 13>(fast);
                default: return nullptr;
            }
        case kF16: return ng == 13 ? pick_fast<kF16, 13>(fast) : nullptr;
        default: return nullptr;
    }
}

// Largest radius of the tensor step.  Row sums 2R+1 <= 255 travel as u8; R = 128
// (row sums up to 257) as f16.  Above it the X tiles of three or more row blocks
// and the f16 operands no longer fit one SM's shared memory twice over.
constexpr int kTensorMaxRadius = 128;

bool tensor_supported(int n, int radius, char* why, size_t why_len) {
    if (radius < 1 || radius > kTensorMaxRadius) {
        snprintf(why, why_len, "tensor variant supports 1 <= R <= %d (got %d)", kTensorMaxRadius, radius);
        return false;
    }
    if (n < radius) {
        snprintf(why, why_len, "n < R");
        return false;
    }
    return true;
}

// Lane constants of the interval rule on the box count B (centre included):
// a live cell survives iff smin+1 <= B <= smax+1, a dead one is born iff
// bmin <= B <= bmax.  For a lane of `bits` bits whose top bit is the marker,
// nlo = top - lo (B + nlo has the marker set iff B >= lo) and hiH = top + hi
// (hiH - B has it set iff B <= hi); empty intervals become lo = top, hi = 0.
static void lane_consts(int lo, int hi, int bits, int& nlo, int& hiH) {
    const int top = 1 << (bits - 1);
    if (lo < 0) lo = 0;
    if (hi > top - 1) hi = top - 1;
    if (hi < lo || lo > top - 1) {
        lo = top;
        hi = 0;
    }
    nlo = top - lo;
    hiH = top + hi;
}

// The same for one 32-bit lane (marker bit 31).  The lane holds either the
// box count B itself (s32) or, with `fbits`, the bit pattern of the f32 value
// B + off; both are below 2^31 and ordered like B, so the thresholds are
// transformed the same way.  An empty interval gives nlo = 0 (B + 0 never has
// bit 31 set).
static void lane_consts32(int lo, int hi, int maxB, bool fbits, int off, uint32_t& nlo, uint32_t& hiH) {
    if (lo < 0) lo = 0;
    if (hi > maxB) hi = maxB;
    if (hi < lo) {
        nlo = 0u;
        hiH = 0x80000000u;
        return;
    }
    uint32_t l = (uint32_t)lo, h = (uint32_t)hi;
    if (fbits) {
        const float fl = (float)(lo + off), fh = (float)(hi + off);
        memcpy(&l, &fl, 4);
        memcpy(&h, &fh, 4);
    }
    nlo = 0x80000000u - l;
    hiH = 0x80000000u + h;
}

// Tile geometry for radius R (also restated in tests/test_tensor_tiles.py):
//   Tc = 128 output columns per tile (H and C, two buffers each, fill the 512
//          TMEM columns);
//   PADC = 16 + 32a >= R columns of halo on each side of the output columns
//          (16 mod 32, so that every X group straddles two packed words by halves);
//   nb = 1 row block for R <= 32 (Tr = 128 - 2R output rows per tile), else
//          enough 128-row blocks for Tr = 128 rows plus 2R halo rows;
//   ng = ceil((PADC + Tc + R) / 32) product-1 K steps reach every X column
//          that any output column of the tile needs;
//   mode = the rule lanes and product-2 operand (TcMode);
//   fast = the packed words of the next units staged through shared memory,
//          where n allows it and the ring fits beside the deepest X ring.
struct TensorGeometry {
    int PADC, Tr, nb, ng, mode, stages;
    bool fast;
};

static int tensor_mode(int R) {
    if ((2 * R + 1) * (2 * R + 1) <= 127) return kLanes8;
    if ((2 * R + 1) * (2 * R + 1) < (1 << 15)) return kLanes16;
    return 2 * R + 1 <= 255 ? kLanes32 : kF16;
}

static bool tensor_geometry(int R, bool fast_ok, TensorGeometry& G) {
    G.PADC = R <= 16 ? 16 : 16 + 32 * ((R - 16 + 31) / 32);
    G.nb = R <= 32 ? 1 : (128 + 2 * R + 127) / 128;
    G.Tr = G.nb == 1 ? 128 - 2 * R : std::min(128, 128 * G.nb - 2 * R);
    G.ng = (G.PADC + kTc + R + 31) / 32;
    G.mode = tensor_mode(R);
    if (G.Tr < 1 || R > kTensorMaxRadius || 2 * R + 1 + kF16Offset > 2048) return false;
    if (tensor_xt(G.mode, fast_ok, G.ng)) {
        // X in tensor memory: kXtStages stages of TMEM columns, no X in shared memory
        G.stages = kXtStages;
        G.fast = true;
        return smem_layout(G.stages, G.ng, G.nb, true, G.mode, true).total + 1024 <= kSmemLimit;
    }
    // the deepest X ring that fits, with the word ring where possible
    for (int f = fast_ok ? 1 : 0; f >= 0; --f) {
        for (int st = kMaxStages; st >= 2; --st) {
            if (smem_layout(st, G.ng, G.nb, f != 0, G.mode).total + 1024 <= kSmemLimit) {
                G.stages = st;
                G.fast = f != 0;
                return true;
            }
        }
    }
    return false;
}

TensorPlan* tensor_plan_create(const PackedFrame& a, const PackedFrame& b, const Rule& rule, int device, char* why,
                               size_t why_len) {
    if (!tensor_supported(a.n, rule.radius, why, why_len)) return nullptr;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) {
        snprintf(why, why_len, "tcgen05 needs an sm_100 device (compute capability %d.x)", major);
        return nullptr;
    }
    if (a.HW < 1 || b.HW < 1) {
        snprintf(why, why_len, "packed frames need a halo word");
        return nullptr;
    }
    const int R = rule.radius;
    const int nw = a.nw;
    // one correction wraps a row (rows span [-R, n + 128 nb)) and a word index
    // (words span [-4, nw + ng)); groups are word halves
    const int nb_of_r = R <= 32 ? 1 : (128 + 2 * R + 127) / 128;
    const bool fast_ok = a.n % 32 == 0 && nw >= 4 && a.n >= 128 * nb_of_r + R;
    TensorGeometry G{};
    if (!tensor_geometry(R, fast_ok, G)) {
        snprintf(why, why_len, "no tile shape for R=%d", R);
        return nullptr;
    }
    const bool fast = G.fast;
    TensorPlan* P = new TensorPlan();
    P->operand_bits = G.mode == kF16 ? 16 : 8;
    uint32_t nlo_d, hiH_d, nlo_s, hiH_s, bcast = 1u;
    if (G.mode >= kLanes32) {
        const int maxB = (2 * R + 1) * (2 * R + 1);
        const bool fb = G.mode == kF16;
        const int off = fb ? kF16Offset * (2 * R + 1) : 0;
        lane_consts32(rule.bmin, rule.bmax, maxB, fb, off, nlo_d, hiH_d);
        lane_consts32(rule.smin + 1, rule.smax + 1, maxB, fb, off, nlo_s, hiH_s);
    } else {
        const int bits = G.mode == kLanes16 ? 16 : 8;
        bcast = G.mode == kLanes16 ? 0x00010001u : 0x01010101u;
        int a0, b0, a1, b1;
        lane_consts(rule.bmin, rule.bmax, bits, a0, b0);
        lane_consts(rule.smin + 1, rule.smax + 1, bits, a1, b1);
        nlo_d = (uint32_t)a0;
        hiH_d = (uint32_t)b0;
        nlo_s = (uint32_t)a1;
        hiH_s = (uint32_t)b1;
    }
    const PackedFrame* src[2] = {&a, &b};
    const PackedFrame* dst[2] = {&b, &a};
    for (int i = 0; i < 2; ++i) {
        TcParams& q = P->prm[i];
        q.src = src[i]->words + (size_t)src[i]->HR * src[i]->wpitch + src[i]->HW;
        q.dst = dst[i]->words + (size_t)dst[i]->HR * dst[i]->wpitch + dst[i]->HW;
        q.wpitch = (long long)a.wpitch;
        q.n = a.n;
        q.nw = nw;
        q.R = R;
        q.PADC = G.PADC;
        q.Tr = G.Tr;
        q.nb = G.nb;
        q.stages = G.stages;
        q.tiles_x = (a.n + kTc - 1) / kTc;
        q.tiles_y = (a.n + G.Tr - 1) / G.Tr;
        q.nlo0 = nlo_d * bcast;
        q.dlo = nlo_s - nlo_d;
        q.hiH0 = hiH_d * bcast;
        q.dhi = hiH_s - hiH_d;
    }
    if (cudaMalloc(&P->err, sizeof(unsigned int)) != cudaSuccess) {
        snprintf(why, why_len, "error-flag allocation failed");
        delete P;
        return nullptr;
    }
    cudaMemset(P->err, 0, sizeof(unsigned int));
    for (auto& q : P->prm) {
        q.err = P->err;
        q.wait_ns = kWaitLimitNs;
        q.inject_missing_commit = 0;
    }
    P->kernel = pick_kernel(G.mode, fast, G.ng);
    if (!P->kernel) {
        snprintf(why, why_len, "no kernel instantiation for R=%d", R);
        cudaFree(P->err);
        delete P;
        return nullptr;
    }
    P->smem_bytes = smem_layout(G.stages, G.ng, G.nb, fast, G.mode, tensor_xt(G.mode, fast, G.ng)).total + 1024;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    P->grid = std::min(P->prm[0].tiles_x * P->prm[0].tiles_y, sms);
    if (cudaFuncSetAttribute(P->kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_bytes) !=
        cudaSuccess) {
        snprintf(why, why_len, "cannot reserve %d bytes of shared memory", P->smem_bytes);
        cudaFree(P->err);
        delete P;
        return nullptr;
    }
    return P;
}

void tensor_plan_destroy(TensorPlan* p) {
    if (!p) return;
    if (p->err) cudaFree(p->err);
    delete p;
}

int tensor_plan_depth(const TensorPlan*) { return 1; }

void tensor_plan_set_wait(TensorPlan* p, unsigned long long ns, int inject_missing_commit) {
    for (auto& q : p->prm) {
        q.wait_ns = ns;
        q.inject_missing_commit = inject_missing_commit;
    }
}
int tensor_plan_operand_bits(const TensorPlan* p) { return p ? p->operand_bits : 0; }
unsigned int* tensor_plan_error_flag(TensorPlan* p) { return p ? p->err : nullptr; }

cudaError_t launch_tensor_pass(TensorPlan* p, bool src_is_a, cudaStream_t s) {
    const int i = src_is_a ? 0 : 1;
    p->kernel<<<p->grid, kThreads, p->smem_bytes, s>>>(p->prm[i]);
    return cudaGetLastError();
}

}  // namespace ltl

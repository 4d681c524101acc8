// k_tensor.cu -- K2: the LtL step as two banded 0/1 matrix products on the
// 5th-generation tensor cores (tcgen05, kind::i8, accumulators in TMEM).
//
// This is the reference's AMX formulation (kezada94/CAT_cpu,
// src/CellularAutomata/Solvers/AMXSolver16.cpp:63-138 band tiles, :254-309 row
// sums X*B, :322-384 column sums + rule) re-designed for sm_100a:
//   - one CTA owns a tile of Tr x Tc output cells.  TMA brings the halo'd input
//     tile X (128 rows x 256 bytes, two 128-byte swizzle atoms) into shared memory;
//   - product 1:  H = X * B_h   (row sums; M = 128 tile rows, N = 32-column
//     chunks, K = a 64-column window; u8 x u8 -> s32 in TMEM).  B_h is the 0/1
//     band |k - PADC - n| <= R, built once per CTA in shared memory;
//   - H (<= 2R+1) is read back with tcgen05.ld, re-quantised to u8 and stored
//     as the MN-major B operand of
//   - product 2:  C = B_v * H   (column sums; M = 128, N = Tc, K = 128) with the
//     band B_v[m][k] = [m <= k <= m + 2R], so the reference's transposed
//     scatter between the two products (AMXSolver.cpp:321-325) disappears;
//   - epilogue: C is the box count including the centre, the birth/survival
//     interval rule (HostSolver.tpp:47-73, k = C - centre) is applied four
//     cells per register, and the uint8 result goes straight to global memory.
// Exactness: inputs are 0/1, H <= 2R+1 <= 255 fits u8, C <= (2R+1)^2 in s32.
//
// Every wait on an mbarrier is bounded (globaltimer); on timeout the kernel
// sets a bit in an error word that the host reads (ltl_synchronize), finishes
// waiting for its own TMA copy (also bounded), frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "ltl_kernels.h"

namespace ltl {

// ---------------------------------------------------------------------------
// PTX helpers (sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// Bounded wait for `phase` of `bar`: false after `limit_ns` of wall time.  The
// clock is read once per 16 tries, so that a waiting warp spends few issue
// slots per try; `sleep_ns` > 0 backs off between tries (for warps whose wait
// is not on the critical path).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase, uint64_t limit_ns, uint32_t sleep_ns = 0) {
    if (mbar_try(bar, phase)) return true;
    const uint64_t t0 = globaltimer();
    while (true) {
#pragma unroll 4
        for (int i = 0; i < 16; ++i) {
            if (mbar_try(bar, phase)) return true;
            if (sleep_ns) __nanosleep(sleep_ns);
        }
        if (globaltimer() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::
            "r"(smem_u32(dst)),
        "l"((uint64_t)map), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive TMEM columns of this thread's lane, packed in pairs
// (.pack::16b): register k holds the low 16 bits of column 2k in its low half
// and those of column 2k + 1 in its high half.  Every accumulator read here
// fits 16 bits: row sums are <= 2R + 1 and box counts <= (2R + 1)^2 < 2^16 for
// R <= 32.  The registers are defined only after tmem_wait8 on the same array:
// the wait takes them as read-write operands so that the compiler cannot move
// a use of them above it.
__device__ __forceinline__ void tmem_ld16p(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.pack::16b.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// Waits for every tcgen05.ld this thread issued.
__device__ __forceinline__ void tmem_wait8(uint32_t (&v)[8]) {
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(v[0]), "+r"(v[1]), "+r"(v[2]), "+r"(v[3]), "+r"(v[4]), "+r"(v[5]), "+r"(v[6]), "+r"(v[7])
                 :
                 : "memory");
}

// Bytes 0 and 2 of a and of b: the low bytes of the four 16-bit values of two
// packed registers, in column order.
__device__ __forceinline__ uint32_t low_bytes4(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x6420); }

// Walks this warp's 16-column chunks of a TMEM accumulator row, loading chunk
// c + 1 while f(values, column) processes chunk c.  The chunks are the halves
// of 32-column blocks grp, grp + groups, grp + 2*groups, ... below `cols`;
// `max_chunks` bounds the unrolled loop.  Every argument is warp-uniform, as
// tcgen05.ld requires.
template <int max_chunks, class F>
__device__ __forceinline__ void tmem_walk16(uint32_t trow, int grp, int groups, int cols, F&& f) {
    const int blocks = grp * 32 < cols ? (cols / 32 - grp + groups - 1) / groups : 0;
    const int nc = 2 * blocks < max_chunks ? 2 * blocks : max_chunks;
    auto col = [&](int c) { return 32 * (grp + groups * (c >> 1)) + 16 * (c & 1); };
    if (nc == 0) return;
    uint32_t a[8], b[8];
    tmem_ld16p(trow + col(0), a);
    tmem_wait8(a);
#pragma unroll
    for (int c = 0; c < max_chunks; ++c) {
        if (c < nc) {
            const bool more = c + 1 < nc;
            if ((c & 1) == 0) {
                if (more) tmem_ld16p(trow + col(c + 1), b);
                f(a, col(c));
                if (more) tmem_wait8(b);
            } else {
                if (more) tmem_ld16p(trow + col(c + 1), a);
                f(b, col(c));
                if (more) tmem_wait8(a);
            }
        }
    }
}

// Shared-memory matrix descriptors (tcgen05 "version 1" format).
// K-major, 128-byte swizzle: 8-row atoms of 1024 B (SBO), LBO unused.
__device__ __forceinline__ uint64_t desc_k_sw128(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
           ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}
// No swizzle ("interleave"): 8 x 16-byte core matrices stored as 128 contiguous
// bytes; `lbo` / `sbo` are the byte strides between core matrices along the
// leading / strided dimension.
__device__ __forceinline__ uint64_t desc_noswz(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1u << 46);
}

// Instruction descriptor: kind::i8, u8 x u8 -> s32, M = 128.
__host__ __device__ constexpr uint32_t idesc_u8(int N, bool b_mn_major) {
    return (2u << 4)                       // D format s32
           | (0u << 7) | (0u << 10)        // A, B unsigned 8-bit
           | (0u << 15)                    // A K-major
           | ((b_mn_major ? 1u : 0u) << 16)
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// ---------------------------------------------------------------------------
// Tile geometry and the persistent, warp-specialised kernel
//
// One CTA per SM walks a strided list of tiles.  Warp roles:
//   warp 0    TMA producer: X tiles into a kXStages ring (x_full / x_empty);
//   warp 1    MMA issuer, per tile j:  product 2 of tile j-1 (once H(j-1) is in
//             shared memory and C of tile j-2 has been read), then product 1 of
//             tile j (H's TMEM columns are free as soon as H(j-1) was read);
//   warps 2.. epilogue: kEpiGroups groups of 4 warps (one warp per TMEM lane
//             quarter); group g handles the 32-column blocks g, g + kEpiGroups,
//             ... of every tile: re-quantise H(j), then rule + store C(j).
// TMEM holds H (columns [0, Tc)) and C (columns [256, 256 + Tc)) separately, so
// product 1 of the next tile overlaps the rule of the current one and only
// product 2's latency is on the epilogue's critical path.  All waits are bounded.
// ---------------------------------------------------------------------------
constexpr int kAtomBytes = 128 * 128;  // one 128-row x 128-byte swizzle atom
constexpr int kAtoms = 2;              // X tile = 128 rows x 256 columns
constexpr int kXBytes = kAtoms * kAtomBytes;
constexpr int kXCols = 128 * kAtoms;
constexpr int kXStages = 4;
constexpr int kHCol = 0;               // TMEM column of H
constexpr int kCCol = 256;             // TMEM column of C
constexpr int kN1 = 32;                // product-1 column chunk
constexpr int kEpiGroups = 4;          // epilogue warp groups (column blocks round-robin)
// The MMA warp waits for the epilogue most of the time; between its tries it
// sleeps this long, so that it leaves issue slots to the epilogue warps that
// share its scheduler.
constexpr uint32_t kMmaSleepNs = 32;
constexpr int kMaxChunks = 4;          // 16-column chunks per epilogue warp: 2 blocks of 32 (Tc <= 256)
constexpr int kEpiWarps = 4 * kEpiGroups;
constexpr int kThreads = 64 + 32 * kEpiWarps;  // producer + MMA + epilogue warps
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait

struct TensorParams {
    uint8_t* out;      // destination frame base
    int n, H;
    long long pitch;
    int R, PADC;       // radius, column halo of the tile (multiple of 16, >= R)
    int Tr, Tc;        // output rows / columns per tile
    int K1c;           // product-1 K window (multiple of 32)
    int tiles_x, tiles_y;
    RuleSwar8 q;       // rule on the box count (used when (2R+1)^2 <= 127)
    int slo, shi, blo, bhi;  // rule on the box count, scalar form
    unsigned int* err;
    unsigned long long wait_ns;  // limit of every mbarrier wait
    int inject_missing_commit;   // test hook: product 1 of the first tile never signals
};

struct SmemLayout {
    int x_off, hs_off, bh_off, bv_off, bar_off, tmem_off, total;
};

enum Bar { X_FULL = 0, X_EMPTY = kXStages, H_FULL = 2 * kXStages, HS_FULL, C_FULL, C_EMPTY, NBARS };

__host__ __device__ inline SmemLayout smem_layout(int Tc, int K1c) {
    SmemLayout L{};
    int o = 0;
    L.x_off = o;
    o += kXStages * kXBytes;                // 1024-aligned stages
    L.hs_off = o;
    o += 2 * 128 * Tc;                      // H as u8, MN-major, two buffers (tile parity)
    L.bh_off = o;
    o += kN1 * K1c;                         // B_h
    L.bv_off = o;
    o += 128 * 128;                         // B_v
    o = (o + 7) & ~7;
    L.bar_off = o;
    o += NBARS * 8;
    L.tmem_off = o;
    o += 16;
    L.total = o;
    return L;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__global__ void __launch_bounds__(kThreads, 1)
k_tensor_step(const __grid_constant__ CUtensorMap xmap, TensorParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const SmemLayout L = smem_layout(p.Tc, p.K1c);
    uint8_t* xs = smem + L.x_off;
    uint8_t* hs = smem + L.hs_off;
    uint8_t* bh = smem + L.bh_off;
    uint8_t* bv = smem + L.bv_off;
    uint64_t* bars = (uint64_t*)(smem + L.bar_off);
    uint32_t* tmem_slot = (uint32_t*)(smem + L.tmem_off);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = p.R, PADC = p.PADC, Tc = p.Tc, K1c = p.K1c;
    const int ntiles = p.tiles_x * p.tiles_y;
    int mine = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) ++mine;
    constexpr uint32_t kTmemCols = 512;

    if (tid == 0) {
        for (int i = 0; i < kXStages; ++i) {
            mbar_init(&bars[X_FULL + i], 1);
            mbar_init(&bars[X_EMPTY + i], kEpiWarps);
        }
        mbar_init(&bars[H_FULL], 1);
        mbar_init(&bars[HS_FULL], kEpiWarps);
        mbar_init(&bars[C_FULL], 1);
        mbar_init(&bars[C_EMPTY], kEpiWarps);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
    // Band matrices (no-swizzle K-major layouts: [k / 16][row][16 bytes]).
    // B_h[n][k] = [|k - PADC - n| <= R], n < 32, k < K1c
    for (int idx = tid; idx < kN1 * K1c; idx += kThreads) {
        const int k = idx / kN1, n = idx % kN1;
        const int d = k - PADC - n;
        bh[((k >> 4) * kN1 + n) * 16 + (k & 15)] = (d >= -R && d <= R) ? 1 : 0;
    }
    // B_v[m][k] = [m <= k <= m + 2R], m, k < 128 (16 bytes per store)
    for (int idx = tid; idx < 8 * 128; idx += kThreads) {
        const int kc = idx / 128, m = idx % 128;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint32_t v = 0;
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int k = kc * 16 + 4 * q + e;
                v |= (uint32_t)(k >= m && k <= m + 2 * R) << (8 * e);
            }
            w[q] = v;
        }
        *(uint4*)(bv + (kc * 128 + m) * 16) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    fence_proxy_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // ------------------------- TMA producer -----------------------------
        if (lane == 0) {
            int it = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
                const int st = it % kXStages;
                const uint32_t ph = (uint32_t)(it / kXStages) & 1u;
                if (it >= kXStages) ok = mbar_wait(&bars[X_EMPTY + st], ph ^ 1u, p.wait_ns, 128);
                if (!ok) {
                    atomicOr(p.err, 1u);
                    break;
                }
                const int ty = t / p.tiles_x, tx = t % p.tiles_x;
                const int y = p.H + ty * p.Tr - R;
                const int x = p.H + tx * Tc - PADC;
                uint8_t* dst = xs + st * kXBytes;
                mbar_expect_tx(&bars[X_FULL + st], kXBytes);
#pragma unroll
                for (int a = 0; a < kAtoms; ++a) tma_load_2d(dst + a * kAtomBytes, &xmap, &bars[X_FULL + st], x + 128 * a, y);
            }
            // never leave with a copy in flight into this CTA's shared memory
            const int issued = it;
            for (int j = (issued > kXStages ? issued - kXStages : 0); j < issued; ++j) {
                if (!mbar_wait(&bars[X_FULL + j % kXStages], (uint32_t)(j / kXStages) & 1u, p.wait_ns))
                    atomicOr(p.err, 16u);
            }
        }
    } else if (warp == 1) {
        // --------------------------- MMA issuer -----------------------------
        if (lane == 0) {
            const uint32_t ba = smem_u32(bh), va = smem_u32(bv), ha0 = smem_u32(hs);
            const uint32_t id1 = idesc_u8(kN1, false);
            const uint32_t id2 = idesc_u8(Tc, true);
            bool ok = true;
            auto product1 = [&](int j) -> bool {
                const int st = j % kXStages;
                if (!mbar_wait(&bars[X_FULL + st], (uint32_t)(j / kXStages) & 1u, p.wait_ns)) return false;
                tc_fence_after();
                const uint32_t xa = smem_u32(xs + st * kXBytes);
                for (int n0 = 0; n0 < Tc; n0 += kN1) {
                    for (int s = 0; s < K1c / 32; ++s) {
                        const int col = n0 + 32 * s;  // X column of this K step
                        const uint32_t a_addr = xa + (col >> 7) * kAtomBytes + (col & 127);
                        const uint64_t ad = desc_k_sw128(a_addr);
                        const uint64_t bd = desc_noswz(ba + s * 2 * kN1 * 16, kN1 * 16, 128);
                        mma_i8(tmem + kHCol + n0, ad, bd, id1, s > 0 ? 1u : 0u);
                    }
                }
                if (!(p.inject_missing_commit && j == 0)) mma_commit(&bars[H_FULL]);
                return true;
            };
            // product 2 of tile j: C = B_v * H(j), H(j) in shared-memory buffer j % 2
            auto product2 = [&](int j) -> bool {
                if (j >= 1 && !mbar_wait(&bars[C_EMPTY], (uint32_t)(j - 1) & 1u, p.wait_ns, kMmaSleepNs)) return false;
                tc_fence_after();
                const uint32_t ha = ha0 + (j & 1) * 128 * Tc;
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const uint64_t ad = desc_noswz(va + s * 2 * 128 * 16, 128 * 16, 128);
                    const uint64_t bd = desc_noswz(ha + s * 32 * 16, 128, 128 * 16);
                    mma_i8(tmem + kCCol, ad, bd, id2, s > 0 ? 1u : 0u);
                }
                mma_commit(&bars[C_FULL]);
                return true;
            };
            // Order per tile j: product 1 of tile j+1 as soon as H(j) has been read
            // back, then product 2 of tile j once C(j-1) has been read.
            ok = mine >= 1 ? product1(0) : true;
            for (int j = 0; j < mine && ok; ++j) {
                ok = mbar_wait(&bars[HS_FULL], (uint32_t)j & 1u, p.wait_ns, kMmaSleepNs);
                if (ok && j + 1 < mine) ok = product1(j + 1);
                if (ok) ok = product2(j);
            }
            if (!ok) atomicOr(p.err, 2u);
        }
    } else {
        // ---------------------------- epilogue ------------------------------
        const int q = warp & 3;                 // TMEM lane quarter of this warp
        const int grp = (warp - 2) >> 2;        // column group
        const int row = q * 32 + lane;          // H row / output row within the tile
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        const bool small = (2 * R + 1) * (2 * R + 1) <= 127;
        bool ok = true;
        // re-quantise H(j) to u8 into shared-memory buffer j % 2 (MN-major B operand of product 2)
        auto requant = [&](int j) -> bool {
            if (!mbar_wait(&bars[H_FULL], (uint32_t)j & 1u, p.wait_ns)) return false;
            tc_fence_after();
            uint8_t* hsb = hs + (j & 1) * 128 * Tc;
            tmem_walk16<kMaxChunks>(tmem + kHCol + lane_off, grp, kEpiGroups, Tc,
                                    [&](const uint32_t (&v)[8], int col) {
                                        uint4 w;
                                        w.x = low_bytes4(v[0], v[1]);
                                        w.y = low_bytes4(v[2], v[3]);
                                        w.z = low_bytes4(v[4], v[5]);
                                        w.w = low_bytes4(v[6], v[7]);
                                        *(uint4*)(hsb + ((col >> 4) * 128 + row) * 16) = w;
                                    });
            fence_proxy_async();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars[HS_FULL]);
            return true;
        };
        if (mine >= 1) ok = requant(0);
        int t = blockIdx.x;
        for (int j = 0; j < mine && ok; ++j, t += gridDim.x) {
            if (j + 1 < mine && !requant(j + 1)) {
                ok = false;
                break;
            }
            // rule + store C(j)
            if (!mbar_wait(&bars[C_FULL], (uint32_t)j & 1u, p.wait_ns)) {
                ok = false;
                break;
            }
            tc_fence_after();
            const int st = j % kXStages;
            const int ty = t / p.tiles_x, tx = t % p.tiles_x;
            const int r0 = ty * p.Tr, c0 = tx * Tc;
            const int gi = r0 + row;
            const bool row_ok = (row < p.Tr) && (gi < p.n);
            const int xr = row + R;
            const uint8_t* xrow = xs + st * kXBytes + (xr & 127) * 128;
            uint8_t* orow = p.out + (size_t)(p.H + gi) * (size_t)p.pitch + p.H + c0;
            tmem_walk16<kMaxChunks>(tmem + kCCol + lane_off, grp, kEpiGroups, Tc, [&](const uint32_t (&v)[8], int col) {
                if (!row_ok) return;
                const int xc = PADC + col;  // X column of these 16 cells
                const int atom = xc >> 7, ch = (xc & 127) >> 4;
                const uint4 s4 = *(const uint4*)(xrow + atom * kAtomBytes + ((ch ^ (xr & 7)) << 4));
                const uint32_t sw[4] = {s4.x, s4.y, s4.z, s4.w};  // compile-time indices only
                uint32_t o[4];
#pragma unroll
                for (int qq = 0; qq < 4; ++qq) {
                    const uint32_t* b = &v[2 * qq];  // cells 4qq .. 4qq+3 as two 16-bit pairs
                    if (small) {
                        o[qq] = rule_swar8(low_bytes4(b[0], b[1]), sw[qq], p.q);
                    } else {
                        uint32_t r = 0;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int B = (int)((b[e >> 1] >> (16 * (e & 1))) & 0xffffu);
                            const int sv = (sw[qq] >> (8 * e)) & 1;
                            const int lo = sv ? p.slo : p.blo, hi = sv ? p.shi : p.bhi;
                            r |= (uint32_t)((B >= lo) & (B <= hi)) << (8 * e);
                        }
                        o[qq] = r;
                    }
                }
                const int gj = c0 + col;
                if (gj + 16 <= p.n) {
                    *(uint4*)(orow + col) = make_uint4(o[0], o[1], o[2], o[3]);
                } else if (gj < p.n) {
                    const int cnt = p.n - gj;
#pragma unroll
                    for (int e = 0; e < 16; ++e)
                        if (e < cnt) orow[col + e] = (uint8_t)((o[e >> 2] >> (8 * (e & 3))) & 0xff);
                }
            });
            tc_fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&bars[C_EMPTY]);
                mbar_arrive(&bars[X_EMPTY + st]);
            }
        }
        if (!ok) atomicOr(p.err, 8u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        __syncwarp();
        tmem_dealloc(tmem, kTmemCols);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct TensorPlan {
    CUtensorMap map[2];  // source frame a / b
    TensorParams prm[2]; // destination frame b / a
    int smem_bytes;
    int grid;
    unsigned int* err;
};

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    }
    return fn;
}

static int pad_for(int R) { return (int)round_up((size_t)R, 16); }

int tensor_plan_halo_needed(int radius) { return std::max(16, pad_for(radius)); }

bool tensor_supported(int n, int radius, char* why, size_t why_len) {
    if (radius < 1 || radius > 32) {
        snprintf(why, why_len, "tensor variant supports 1 <= R <= 32 (got %d)", radius);
        return false;
    }
    if (n < radius) {
        snprintf(why, why_len, "n < R");
        return false;
    }
    return true;
}

TensorPlan* tensor_plan_create(const Frame& a, const Frame& b, const Rule& rule, int device, char* why,
                               size_t why_len) {
    if (!tensor_supported(a.n, rule.radius, why, why_len)) return nullptr;
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) {
        snprintf(why, why_len, "tcgen05 needs an sm_100 device (compute capability %d.x)", major);
        return nullptr;
    }
    auto encode = encode_fn();
    if (!encode) {
        snprintf(why, why_len, "cuTensorMapEncodeTiled not available");
        return nullptr;
    }
    TensorPlan* P = new TensorPlan();
    const int R = rule.radius;
    const int PADC = pad_for(R);
    const int Tc = ((kXCols - 2 * PADC) / kN1) * kN1;  // 224 for R <= 16, 192 for R <= 32
    const int Tr = 128 - 2 * R;
    const int K1c = (int)round_up((size_t)(kN1 + PADC + R), 32);
    if (Tc < kN1 || Tc > 16 * kEpiGroups * kMaxChunks || Tr < 1 || K1c > kN1 + 2 * PADC) {
        snprintf(why, why_len, "no tile shape for R=%d", R);
        delete P;
        return nullptr;
    }
    const Frame* src[2] = {&a, &b};
    const Frame* dst[2] = {&b, &a};
    for (int i = 0; i < 2; ++i) {
        const Frame& f = *src[i];
        cuuint64_t gdim[2] = {(cuuint64_t)f.pitch, (cuuint64_t)(f.n + 2 * f.H)};
        cuuint64_t gstride[1] = {(cuuint64_t)f.pitch};
        cuuint32_t box[2] = {128, 128};
        cuuint32_t estride[2] = {1, 1};
        CUresult cr = encode(&P->map[i], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)f.base, gdim, gstride, box, estride,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                             CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) {
            snprintf(why, why_len, "cuTensorMapEncodeTiled failed (%d)", (int)cr);
            delete P;
            return nullptr;
        }
        TensorParams& q = P->prm[i];
        q.out = dst[i]->base;
        q.n = f.n;
        q.H = f.H;
        q.pitch = (long long)f.pitch;
        q.R = R;
        q.PADC = PADC;
        q.Tr = Tr;
        q.Tc = Tc;
        q.K1c = K1c;
        q.tiles_x = (f.n + Tc - 1) / Tc;
        q.tiles_y = (f.n + Tr - 1) / Tr;
        q.q = make_rule_swar8(rule);
        q.slo = rule.smin + 1;
        q.shi = rule.smax + 1;
        q.blo = rule.bmin;
        q.bhi = rule.bmax;
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
    P->smem_bytes = smem_layout(Tc, K1c).total + 1024;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    P->grid = std::min(P->prm[0].tiles_x * P->prm[0].tiles_y, sms);
    if (cudaFuncSetAttribute(k_tensor_step, cudaFuncAttributeMaxDynamicSharedMemorySize, P->smem_bytes) !=
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
int tensor_plan_operand_bits(const TensorPlan*) { return 8; }
unsigned int* tensor_plan_error_flag(TensorPlan* p) { return p ? p->err : nullptr; }

cudaError_t launch_tensor_pass(TensorPlan* p, bool src_is_a, cudaStream_t s) {
    const int i = src_is_a ? 0 : 1;
    k_tensor_step<<<p->grid, kThreads, p->smem_bytes, s>>>(p->map[i], p->prm[i]);
    return cudaGetLastError();
}

}  // namespace ltl

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
//     128-byte-swizzled K-major layout the MMA reads (128 rows x 256 columns);
//   - product 1:  H = X * B_h   (row sums; M = 128 tile rows, N = 32-column
//     chunks, K = the chunk's column window; u8 x u8 -> s32 in TMEM);
//   - H (<= 2R+1) is read back with tcgen05.ld, re-quantised to u8 and stored
//     as the MN-major B operand of
//   - product 2:  C = B_v * H   (column sums; M = 128, N = Tc, K = 128) with
//     B_v[m][k] = [m <= k <= m + 2R], so the reference's transposed scatter
//     between the two products (AMXSolver.cpp:321-325) disappears;
//   - epilogue: C is the box count including the centre; the birth/survival
//     interval rule (HostSolver.tpp:47-73, k = C - centre) runs on four 8-bit
//     (R <= 5) or two 16-bit lanes per register, and the result bits are
//     gathered straight into the output word.
//
// Column order.  A packed word w spreads to bytes with (w >> k) & 0x01010101,
// k = 0..7: register k holds cells k, 8+k, 16+k, 24+k.  The shared-memory tile
// keeps that order: within each 32-column group, byte position 4k+j holds the
// group's cell 8j+k (the permutation pi(4k+j) = 8j+k).  Product 1 contracts over
// the positions, so B_h's rows follow pi, and its columns (the N order of H
// and C) are chosen so that the rule's result bits land in the output word's
// own bit order with one shift per register (sigma below).  No byte is moved
// to undo the permutation.
//
// Exactness: inputs are 0/1, H <= 2R+1 <= 65 fits u8, C <= (2R+1)^2 in s32.
//
// Every wait on an mbarrier is bounded (globaltimer, hardware-suspended
// tries); on timeout the kernel sets a bit in an error word that the host
// reads (ltl_synchronize), waits (bounded) for its own MMAs, frees its TMEM and
// returns.
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
constexpr int kMaxAtoms = 4;           // X tile: 2..4 atoms = 256..512 columns
constexpr int kMaxGroups = 4 * kMaxAtoms;  // 32-column groups per X row
constexpr int kMaxStages = 4;
constexpr int kHCol = 0;    // TMEM column of H
constexpr int kCCol = 256;  // TMEM column of C
constexpr int kN1 = 32;     // product-1 column chunk = one output word
constexpr int kGroups = 4;  // epilogue column groups
constexpr int kEpiWarps = 4 * kGroups;
constexpr int kUnpackWarps = 4;              // one X row per unpack thread
constexpr int kEpiWarp0 = 1 + kUnpackWarps;  // warp 0: MMA, 1..4: unpack, 5..20: epilogue
constexpr int kThreads = 32 * (kEpiWarp0 + kEpiWarps);
constexpr int kMaxChunks = 7;  // Tc <= 224
constexpr int kSmemLimit = 227 * 1024;
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait
// Back-off between barrier tries of the unpack and epilogue warps: they share
// every scheduler with the single MMA-issuing warp, whose issue rate sets the
// pace, so their spinning must not take its issue slots.
constexpr uint32_t kSleepNs = 64;

struct TcParams {
    const uint32_t* src;  // inner word (0, 0) of the current packed frame
    uint32_t* dst;        // inner word (0, 0) of the next packed frame
    long long wpitch;     // words per frame row
    int n, nw;
    int R, PADC, glo, K1;  // column halo of a tile (16 mod 32), first window group, product-1 K
    int Tr, Tc, nchunks;
    int half0;        // chunks of column half 0 (half 1 has nchunks - half0); each <= 4
    int atoms;        // X tile width = 128 * atoms columns
    int nb;           // 128-row X blocks per tile: product 2 contracts over 128 * nb rows
    int stages;       // X ring stages
    int nhs;          // H buffers in shared memory (1 or 2)
    int tiles_x, tiles_y;
    uint32_t nlo0, dlo, hiH0, dhi;  // rule constants (lane-broadcast; d* = live minus dead, mod 2^32)
    uint32_t rq_mask[kGroups];      // bit i: this epilogue group re-quantises chunk i
    unsigned int* err;
    unsigned long long wait_ns;
    int inject_missing_commit;  // test hook: product 1 of the first unit never signals
};

struct SmemLayout {
    int x_off, hs_off, bh_off, bv_off, bar_off, tmem_off, total;
};

enum Bar {
    X_FULL = 0,
    X_EMPTY = kMaxStages,
    H_FULL = 2 * kMaxStages,  // [2]: per TMEM column half
    HS_FULL = H_FULL + 2,     // [2]
    HS_EMPTY = HS_FULL + 2,   // [2]: per shared-memory H buffer
    C_FULL = HS_EMPTY + 2,    // [2]
    C_EMPTY = C_FULL + 2,     // [2]
    DRAIN = C_EMPTY + 2,
    NBARS
};

constexpr int kHalfCols = 128;  // TMEM columns of one half's H or C (4 chunks)

__host__ __device__ inline SmemLayout smem_layout(int stages, int atoms, int nhs, int K1, int nb) {
    SmemLayout L{};
    int o = 0;
    L.x_off = o;
    o += stages * atoms * kAtomBytes;  // 1024-aligned stages
    L.hs_off = o;
    o += nhs * 128 * kHalfCols;        // one half's H as u8, MN-major, one or two buffers
    L.bh_off = o;
    o += kN1 * K1;                     // B_h
    L.bv_off = o;
    o += 128 * 128 * nb;               // B_v, 128 x (128 nb)
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
__host__ __device__ constexpr int perm_sigma(int n, int lanes16) {
    return lanes16 ? 16 * (n & 1) + (n >> 1) : perm_pi(n);
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
// division in the loops).  Tiles t = blockIdx.x + j * gridDim.x, X blocks xi =
// j * nb + b, units u = 2 xi + h (h = column half).
struct Cursor {
    int u, h;        // unit and its column half
    int xi, b, j;    // X block, row block within the tile, tile count
    int st, sph;     // X ring stage of block xi and its phase parity ((xi / stages) & 1)
    int ty, tx;      // tile coordinates
    int step_x, step_y, tiles_x, nb, stages;

    __device__ void init(const TcParams& p) {
        u = h = xi = b = j = st = sph = 0;
        tiles_x = p.tiles_x;
        nb = p.nb;
        stages = p.stages;
        ty = (int)blockIdx.x / tiles_x;
        tx = (int)blockIdx.x - ty * tiles_x;
        step_y = (int)gridDim.x / tiles_x;
        step_x = (int)gridDim.x - step_y * tiles_x;
    }
    __device__ void next_block() {
        ++xi;
        if (++st == stages) {
            st = 0;
            sph ^= 1;
        }
        if (++b == nb) {
            b = 0;
            ++j;
            tx += step_x;
            ty += step_y;
            if (tx >= tiles_x) {
                tx -= tiles_x;
                ++ty;
            }
        }
    }
    __device__ void next_unit() {
        ++u;
        h ^= 1;
        if (h == 0) next_block();
    }
};

// The work is a stream of units u = ((tile j * nb + row block b) * 2 + column
// half h).  Per X block (j, b) the unpack warps fill one stage; per unit the MMA
// warp runs product 1 for the half's chunks into TMEM half h of H, the epilogue
// re-quantises it to shared memory, and product 2 adds B_v[:, 128b ..] * H to
// TMEM half h of C.  After a tile's last block the epilogue applies the rule to
// C half h.  The two halves use separate TMEM columns (H: [0, 256), C: [256,
// 512)), so the tensor core works on one half while the epilogue reads the other.
//
// LANES16: rule lanes (four 8-bit, or two 16-bit); CENTRE_SMEM: centre cells
// from the X tile (single-block tiles) or from the packed input word; FAST:
// n % 32 == 0 and large enough that rows and words wrap with one correction;
// ATOMS: X tile width in 128-column swizzle atoms; KS: product-1 K steps per
// chunk (K1 / 32).  The window of chunk i starts at X group i (PADC - R < 32).
template <bool LANES16, bool CENTRE_SMEM, bool FAST, int ATOMS, int KS>
__global__ void __launch_bounds__(kThreads, 1) k_tensor_step(const __grid_constant__ TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const SmemLayout L = smem_layout(p.stages, ATOMS, p.nhs, p.K1, p.nb);
    uint8_t* xs = smem + L.x_off;
    uint8_t* hs = smem + L.hs_off;
    uint8_t* bh = smem + L.bh_off;
    uint8_t* bv = smem + L.bv_off;
    uint64_t* bars = (uint64_t*)(smem + L.bar_off);
    uint32_t* tmem_slot = (uint32_t*)(smem + L.tmem_off);
    constexpr int kXB = ATOMS * kAtomBytes;  // bytes of one X stage
    constexpr int kNG = 4 * ATOMS;           // 32-column groups per X row

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = p.R, Tc = p.Tc, K1 = p.K1, nb = p.nb, S = p.stages, nhs = p.nhs;
    const int ntiles = p.tiles_x * p.tiles_y;
    const int mine = ntiles > (int)blockIdx.x ? (ntiles - 1 - (int)blockIdx.x) / (int)gridDim.x + 1 : 0;
    const int units = mine * nb * 2;
    constexpr uint32_t kTmemCols = 512;

    if (tid == 0) {
        for (int i = 0; i < S; ++i) {
            mbar_init(&bars[X_FULL + i], kUnpackWarps);
            mbar_init(&bars[X_EMPTY + i], CENTRE_SMEM ? kEpiWarps : 1);
        }
        for (int h = 0; h < 2; ++h) {
            mbar_init(&bars[H_FULL + h], 1);
            mbar_init(&bars[HS_FULL + h], kEpiWarps);
            mbar_init(&bars[HS_EMPTY + h], 1);
            mbar_init(&bars[C_FULL + h], 1);
            mbar_init(&bars[C_EMPTY + h], kEpiWarps);
        }
        mbar_init(&bars[DRAIN], 1);
        fence_mbar_init();
    }
    if (warp == 0) tmem_alloc(tmem_slot, kTmemCols);
    // B_h (K-major, no swizzle: [k / 16][n][16 bytes]), K1 x 32.  Row k is byte
    // position k of the chunk's window (group glo + k / 32, permuted by pi), column
    // n is accumulator column n (output cell sigma(n) of the chunk).
    for (int idx = tid; idx < kN1 * K1; idx += kThreads) {
        const int k = idx / kN1, nn = idx % kN1;
        const int xc = 32 * (p.glo + (k >> 5)) + perm_pi(k & 31);  // X column relative to the chunk
        const int d = xc - p.PADC - perm_sigma(nn, LANES16);
        bh[((k >> 4) * kN1 + nn) * 16 + (k & 15)] = (d >= -R && d <= R) ? 1 : 0;
    }
    // B_v[m][k] = [m <= k <= m + 2R], m < 128, k < 128 nb (K-major, no swizzle, 16 bytes per store)
    for (int idx = tid; idx < 8 * nb * 128; idx += kThreads) {
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
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;
    const int half0 = p.half0, nch = p.nchunks;

    if (warp == 0) {
        // --------------------------- MMA issuer -----------------------------
        // The whole warp runs the loop (waits and descriptor arithmetic are
        // warp-uniform); lane 0 alone issues the MMAs and the commits, so that
        // every commit tracks every MMA before it.  Descriptors are 64-bit bases
        // plus start-address offsets (in 16-byte units, within the 14-bit field).
        const uint32_t id1 = idesc_u8(kN1, false);
        const uint32_t id2a = idesc_u8(32 * half0, true), id2b = idesc_u8(32 * (nch - half0), true);
        const uint64_t xd0 = desc_k_sw128(smem_u32(xs));
        const uint64_t bhd0 = desc_noswz(smem_u32(bh), kN1 * 16, 128);
        const uint64_t bvd0 = desc_noswz(smem_u32(bv), 128 * 16, 128);
        const uint64_t hsd0 = desc_noswz(smem_u32(hs), 128, 128 * 16);
        const bool leader = lane == 0;
        Cursor c1, c2;  // product 1 runs two units ahead of product 2
        c1.init(p);
        c2.init(p);
        auto product1 = [&](const Cursor& c) -> bool {
            if (!__all_sync(0xffffffffu, mbar_wait(&bars[X_FULL + c.st], (uint32_t)c.sph, p.wait_ns))) return false;
            fence_after();
            if (leader) {
                const int i0 = c.h ? half0 : 0, nci = c.h ? nch - half0 : half0;  // this half's chunks
                const uint64_t xs0 = xd0 + (uint64_t)((c.st * kXB) >> 4);
                const uint32_t d0 = tmem + kHCol + kHalfCols * c.h;
#pragma unroll
                for (int ci = 0; ci < 4; ++ci) {
                    if (ci < nci) {
#pragma unroll
                        for (int s = 0; s < KS; ++s) {
                            const int g = i0 + ci + s;  // X group of this K step: 16-byte units (g / 4) atoms + 2 (g % 4)
                            const uint64_t ad = xs0 + (uint64_t)((g >> 2) * (kAtomBytes >> 4) + (g & 3) * 2);
                            mma_i8(d0 + kN1 * ci, ad, bhd0 + (uint64_t)(s * 2 * kN1), id1, s > 0 ? 1u : 0u);
                        }
                    }
                }
                if (!(p.inject_missing_commit && c.u == 0)) mma_commit(&bars[H_FULL + c.h]);
                // the centre cells come from global memory: the stage is free once both halves read it
                if (!CENTRE_SMEM && c.h == 1) mma_commit(&bars[X_EMPTY + c.st]);
            }
            __syncwarp();
            return true;
        };
        // product 2 of unit c: C[h] (+)= B_v[:, 128b ..] * H(u), H(u) in buffer u % nhs
        auto product2 = [&](const Cursor& c) -> bool {
            if (c.b == 0 && c.j >= 1 &&
                !__all_sync(0xffffffffu, mbar_wait(&bars[C_EMPTY + c.h], (uint32_t)(c.j - 1) & 1u, p.wait_ns)))
                return false;
            fence_after();
            if (leader) {
                const int hb = nhs == 2 ? c.h : 0;
                const uint64_t hd = hsd0 + (uint64_t)((hb * 128 * kHalfCols) >> 4);
                const uint64_t vd = bvd0 + (uint64_t)((4 * c.b * 2 * 128 * 16) >> 4);
                const uint32_t id2 = c.h ? id2b : id2a;
                const uint32_t d = tmem + kCCol + kHalfCols * c.h;
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    mma_i8(d, vd + (uint64_t)((s * 2 * 128 * 16) >> 4), hd + (uint64_t)((s * 32 * 16) >> 4), id2,
                           (c.b > 0 || s > 0) ? 1u : 0u);
                mma_commit(&bars[HS_EMPTY + hb]);
                if (c.b == nb - 1) mma_commit(&bars[C_FULL + c.h]);
            }
            __syncwarp();
            return true;
        };
        // Per unit u, once H(u) has been read back: product 2 of unit u (the
        // epilogue waits for it next), then product 1 of unit u+2 into the
        // TMEM half that H(u) has just left.
        bool ok = true;
        if (units >= 1) ok = product1(c1);
        c1.next_unit();
        if (ok && units >= 2) ok = product1(c1);
        c1.next_unit();
        for (; c2.u < units && ok; c2.next_unit(), c1.next_unit()) {
            ok = __all_sync(0xffffffffu, mbar_wait(&bars[HS_FULL + c2.h], (uint32_t)(c2.xi & 1), p.wait_ns));
            if (ok) ok = product2(c2);
            if (ok && c1.u < units) ok = product1(c1);
        }
        if (!ok && leader) atomicOr(p.err, 2u);
        // never leave with an MMA in flight (TMEM is freed below)
        if (leader) mma_commit(&bars[DRAIN]);
        __syncwarp();
        if (!__all_sync(0xffffffffu, mbar_wait(&bars[DRAIN], 0u, p.wait_ns)) && leader) atomicOr(p.err, 32u);
    } else if (warp < kEpiWarp0) {
        // ------------------------------ unpack ------------------------------
        // Thread `row` (0..127) fills X row `row` of every stage: the kNG groups
        // of 32 columns of one packed row.  The words of the next X block are
        // loaded right after this one is stored, so their latency is spent
        // waiting for a free stage rather than on the critical path.
        const int row = tid - 32;
        const int sw = row & 7;
        const int blocks = mine * nb;
        uint32_t w[kNG + 1];
        // FAST: the kNG + 1 words that hold X row `row` of the cursor's block (group
        // g = upper half of word g, lower half of word g + 1); otherwise the groups
        auto gather = [&](const Cursor& c) {
            const int gr0 = c.ty * p.Tr - R + 128 * c.b + row;
            const int cbase = c.tx * Tc - p.PADC;  // column of X-tile column 0 (16 mod 32)
            if (FAST) {
                int gr = gr0;
                if (gr < 0) gr += p.n;
                else if (gr >= p.n) gr -= p.n;
                const uint32_t* rp = p.src + (size_t)gr * (size_t)p.wpitch;
                int wi = (cbase - 16) >> 5;  // word holding X column 0
                if (wi < 0) wi += p.nw;
#pragma unroll
                for (int k = 0; k <= kNG; ++k) {
                    w[k] = __ldg(rp + wi);
                    if (++wi == p.nw) wi = 0;
                }
            } else {
                const uint32_t* rp = p.src + (size_t)wrap_slow(gr0, p.n) * (size_t)p.wpitch;
                int a = wrap_slow(cbase, p.n);
#pragma unroll
                for (int k = 0; k < kNG; ++k) {
                    w[k] = fetch32(rp, a, p.n);
                    a += 32;
                    while (a >= p.n) a -= p.n;
                }
            }
        };
        bool ok = true;
        Cursor c, cn;  // the block being stored and the one being loaded
        c.init(p);
        cn.init(p);
        if (blocks > 0) gather(cn);
        cn.next_block();
        for (; c.xi < blocks; c.next_block(), cn.next_block()) {
            if (c.xi >= S) {
                bool wt = true;
                if (lane == 0) wt = mbar_wait(&bars[X_EMPTY + c.st], (uint32_t)(c.sph ^ 1), p.wait_ns, kSleepNs);
                ok = __shfl_sync(0xffffffffu, wt, 0);
                if (!ok) break;
            }
            uint8_t* xrow = xs + c.st * kXB + row * 128;
#pragma unroll
            for (int g = 0; g < kNG; ++g) {
                const uint32_t x = FAST ? prmt(w[g], w[g + 1], 0x5432u) : w[g];
                uint32_t v[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) v[k] = (x >> k) & 0x01010101u;
                uint8_t* ap = xrow + (g >> 2) * kAtomBytes;
                const int ch = 2 * (g & 3);
                *(uint4*)(ap + ((ch ^ sw) << 4)) = make_uint4(v[0], v[1], v[2], v[3]);
                *(uint4*)(ap + (((ch + 1) ^ sw) << 4)) = make_uint4(v[4], v[5], v[6], v[7]);
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars[X_FULL + c.st]);
            if (cn.xi < blocks) gather(cn);
        }
        if (!ok && lane == 0) atomicOr(p.err, 4u);
    } else {
        // ---------------------------- epilogue ------------------------------
        const int ew = warp - kEpiWarp0;
        const int q = warp & 3;          // TMEM lane quarter this warp may access
        const int grp = ew >> 2;         // column group
        const int m = q * 32 + lane;     // tile row (TMEM lane)
        const uint32_t lane_off = (uint32_t)(q * 32) << 16;
        const uint32_t rq_mask = p.rq_mask[grp];
        const int aoff = (p.PADC - 16) >> 5;  // centre groups of chunk i: i + aoff, i + aoff + 1
        const uint32_t nlo0 = p.nlo0, dlo = p.dlo, hiH0 = p.hiH0, dhi = p.dhi;
        const int xr = min(m + R, 127);  // X row of this output row's centre cells (rows >= Tr are not stored)
        const int xsw = xr & 7;
        bool ok = true;
        auto wait_all = [&](uint64_t* bar, uint32_t ph) -> bool {
            const bool wt = mbar_wait(bar, ph, p.wait_ns, kSleepNs);
            return __all_sync(0xffffffffu, wt);
        };
        // Per step of the loop: the re-quantisation of unit cq (H of its column half
        // -> u8 in shared memory, the B operand of product 2) and the rule of unit
        // cr = cq - 1 (if that unit ends a tile).  Both TMEM loads are issued before
        // one wait, so their latencies overlap.  Each group has at most one chunk of
        // each per unit (a half has <= 4 chunks; the host plan spreads them).
        auto stage = [&](const Cursor* q, const Cursor* r) -> bool {
            int hb = 0;
            if (q) {
                if (!wait_all(&bars[H_FULL + q->h], (uint32_t)(q->xi & 1))) return false;
                hb = nhs == 2 ? q->h : 0;
                const int k = nhs == 2 ? q->xi : q->u;  // earlier uses of this buffer
                if (k >= 1 && !wait_all(&bars[HS_EMPTY + hb], (uint32_t)((k - 1) & 1))) return false;
            }
            if (r && !wait_all(&bars[C_FULL + r->h], (uint32_t)(r->j & 1))) return false;
            fence_after();
            // this group's chunks: at most one to re-quantise, at most one rule chunk
            int iq = -1, ir = -1, iq0 = 0, ir0 = 0;
            if (q) {
                iq0 = q->h ? half0 : 0;
                const int i1 = q->h ? nch : half0;
                for (int i = iq0; i < i1; ++i)
                    if ((rq_mask >> i) & 1u) iq = i;
            }
            if (r) {
                ir0 = r->h ? half0 : 0;
                const int i1 = r->h ? nch : half0;
                if (ir0 + grp < i1) ir = ir0 + grp;
            }
            uint32_t vq[16], vr[16];
            if (iq >= 0) tmem_ld32p(tmem + lane_off + kHCol + kHalfCols * q->h + kN1 * (iq - iq0), vq);
            if (ir >= 0) tmem_ld32p(tmem + lane_off + kCCol + kHalfCols * r->h + kN1 * (ir - ir0), vr);
            // rule operands that do not come from TMEM, fetched while the loads are in flight
            int gi = 0, wi = 0;
            bool store = false;
            uint32_t Ga[8], Gb[8];
            uint32_t cw = 0u;
            if (ir >= 0) {
                gi = r->ty * p.Tr + m;
                wi = r->tx * (Tc >> 5) + ir;
                store = (m < p.Tr) && (gi < p.n) && wi < p.nw;
                if (CENTRE_SMEM) {
                    // centre cells: groups ga and ga + 1 of the X row (8 words each)
                    const uint8_t* xrow = xs + r->st * kXB + xr * 128;  // one X block per tile
                    const int ga = ir + aoff, gb = ga + 1;
                    const uint4 a0 = *(const uint4*)(xrow + (ga >> 2) * kAtomBytes + (((2 * (ga & 3)) ^ xsw) << 4));
                    const uint4 a1 =
                        *(const uint4*)(xrow + (ga >> 2) * kAtomBytes + (((2 * (ga & 3) + 1) ^ xsw) << 4));
                    const uint4 b0 = *(const uint4*)(xrow + (gb >> 2) * kAtomBytes + (((2 * (gb & 3)) ^ xsw) << 4));
                    const uint4 b1 =
                        *(const uint4*)(xrow + (gb >> 2) * kAtomBytes + (((2 * (gb & 3) + 1) ^ xsw) << 4));
                    Ga[0] = a0.x; Ga[1] = a0.y; Ga[2] = a0.z; Ga[3] = a0.w;
                    Ga[4] = a1.x; Ga[5] = a1.y; Ga[6] = a1.z; Ga[7] = a1.w;
                    Gb[0] = b0.x; Gb[1] = b0.y; Gb[2] = b0.z; Gb[3] = b0.w;
                    Gb[4] = b1.x; Gb[5] = b1.y; Gb[6] = b1.z; Gb[7] = b1.w;
                } else {
                    // the output word's own cells in the current grid (word-aligned)
                    cw = store ? __ldg(p.src + (size_t)gi * (size_t)p.wpitch + wi) : 0u;
                }
            }
            tmem_wait_2x16(vq, vr);
            if (q) {
                if (iq >= 0) {
                    uint8_t* hsb = hs + hb * 128 * kHalfCols;
#pragma unroll
                    for (int hh = 0; hh < 2; ++hh) {
                        uint4 wv;
                        wv.x = prmt(vq[8 * hh + 0], vq[8 * hh + 1], 0x6420u);
                        wv.y = prmt(vq[8 * hh + 2], vq[8 * hh + 3], 0x6420u);
                        wv.z = prmt(vq[8 * hh + 4], vq[8 * hh + 5], 0x6420u);
                        wv.w = prmt(vq[8 * hh + 6], vq[8 * hh + 7], 0x6420u);
                        *(uint4*)(hsb + ((2 * (iq - iq0) + hh) * 128 + m) * 16) = wv;
                    }
                }
                fence_proxy_async();
                fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&bars[HS_FULL + q->h]);
            }
            if (r) {
                if (ir >= 0) {
                    uint32_t acc = 0u;
                    if (!LANES16) {
                        // accumulator column 4k+j = output cell 8j+k: four box counts per
                        // register, bit 7 of each byte lane = the rule's result
#pragma unroll
                        for (int k = 0; k < 8; ++k) {
                            const uint32_t B4 = prmt(vr[2 * k], vr[2 * k + 1], 0x6420u);
                            const uint32_t s4 = CENTRE_SMEM ? prmt(Ga[k], Gb[k], 0x5432u) : (cw >> k) & 0x01010101u;
                            const uint32_t ge = (B4 + nlo0) + s4 * dlo;  // bit 7: B >= lo(s)
                            const uint32_t le = (hiH0 + s4 * dhi) - B4;  // bit 7: B <= hi(s)
                            acc |= (ge & le & 0x80808080u) >> (7 - k);
                        }
                    } else {
                        // accumulator column 2r+e = output cell 16e+r: two box counts per
                        // register, bit 15 of each 16-bit lane = the rule's result
#pragma unroll
                        for (int k = 0; k < 16; ++k) {
                            const uint32_t hsel = (uint32_t)(k >> 3);
                            const uint32_t s2 = CENTRE_SMEM ? prmt(Ga[k & 7], Gb[k & 7],
                                                                   (2u + hsel) | 0x80u | ((4u + hsel) << 8) | 0x8000u)
                                                            : (cw >> k) & 0x00010001u;
                            const uint32_t ge = (vr[k] + nlo0) + s2 * dlo;
                            const uint32_t le = (hiH0 + s2 * dhi) - vr[k];
                            acc |= (ge & le & 0x80008000u) >> (15 - k);
                        }
                    }
                    if (store) p.dst[(size_t)gi * (size_t)p.wpitch + wi] = acc;
                }
                fence_before();
                __syncwarp();
                if (lane == 0) {
                    mbar_arrive(&bars[C_EMPTY + r->h]);
                    if (CENTRE_SMEM && r->h == 1) mbar_arrive(&bars[X_EMPTY + r->st]);
                }
            }
            return true;
        };
        Cursor cq, cr;  // the unit to re-quantise next, the unit whose rule comes next
        cq.init(p);
        cr.init(p);
        if (units >= 1) ok = stage(&cq, nullptr);
        cq.next_unit();
        for (; cr.u < units && ok; cr.next_unit()) {
            const bool has_q = cq.u < units;
            ok = stage(has_q ? &cq : nullptr, cr.b == nb - 1 ? &cr : nullptr);
            if (has_q) cq.next_unit();
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
    unsigned int* err;
};

// The instantiations that exist (R ranges as tensor_geometry lays them out):
//   R <= 5       8-bit lanes, single block, 2 atoms, 2 K steps
//   R 6..16      16-bit lanes, single block, 2 atoms, 2 K steps
//   R 17..32     16-bit lanes, single block, 2 atoms, 4 K steps
//   R 33..48     16-bit lanes, row blocks,   2 atoms, 4 K steps
//   R 49..80     16-bit lanes, row blocks,   3 atoms, 6 K steps
//   R 81..90     16-bit lanes, row blocks,   4 atoms, 8 K steps
template <bool L16, bool CS, int A, int KS>
static TcKernel pick_fast(bool fast) {
    return fast ? k_tensor_step<L16, CS, true, A, KS> : k_tensor_step<L16, CS, false, A, KS>;
}
static TcKernel pick_kernel(bool lanes16, bool centre_smem, bool fast, int atoms, int ks) {
    if (!lanes16) return (centre_smem && atoms == 2 && ks == 2) ? pick_fast<false, true, 2, 2>(fast) : nullptr;
    if (centre_smem) {
        if (atoms != 2) return nullptr;
        if (ks == 2) return pick_fast<true, true, 2, 2>(fast);
        if (ks == 4) return pick_fast<true, true, 2, 4>(fast);
        return nullptr;
    }
    if (atoms == 2 && ks == 4) return pick_fast<true, false, 2, 4>(fast);
    if (atoms == 3 && ks == 6) return pick_fast<true, false, 3, 6>(fast);
    if (atoms == 4 && ks == 8) return pick_fast<true, false, 4, 8>(fast);
    return nullptr;
}

// Largest radius of the tensor step: box counts (2R+1)^2 must fit the 16-bit
// rule lanes (< 2^15) and row sums 2R+1 the u8 operand of product 2.
constexpr int kTensorMaxRadius = 90;

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

// Tile geometry for radius R (also restated in tests/test_tensor_tiles.py):
//   PADC = 16 + 32a >= R columns of halo on each side of the Tc output columns
//          (16 mod 32, so that every X group straddles two packed words by halves);
//   the X tile is 2..4 swizzle atoms wide, chosen to minimise X columns per output
//          column, with Tc <= 224 so that H and C fit 512 TMEM columns;
//   nb = 1 row block for R <= 32 (Tr = 128 - 2R output rows per tile), else
//          enough 128-row blocks for Tr = 128 rows plus 2R halo rows;
//   K1 = the product-1 window of one 32-column chunk, whole 32-column groups.
struct TensorGeometry {
    int PADC, atoms, Tc, Tr, nb, glo, ghi, K1, nchunks, half0, lanes16, stages, nhs;
};

static bool tensor_geometry(int R, TensorGeometry& G) {
    G.PADC = R <= 16 ? 16 : 16 + 32 * ((R - 16 + 31) / 32);
    G.nb = R <= 32 ? 1 : (128 + 2 * R + 127) / 128;
    G.Tr = G.nb == 1 ? 128 - 2 * R : std::min(128, 128 * G.nb - 2 * R);
    G.atoms = 0;
    double best = 1e30;
    for (int a = 2; a <= kMaxAtoms; ++a) {
        const int tc = std::min(32 * kMaxChunks, ((128 * a - 2 * G.PADC) / 32) * 32);
        if (tc < 32) continue;
        const double cost = 128.0 * a / tc;
        if (cost < best - 1e-9) {
            best = cost;
            G.atoms = a;
            G.Tc = tc;
        }
    }
    if (!G.atoms || G.Tr < 1) return false;
    G.nchunks = G.Tc / 32;
    G.half0 = (G.nchunks + 1) / 2;  // <= 4 chunks = 128 TMEM columns per half
    G.glo = (G.PADC - R) / 32;
    G.ghi = (G.PADC + 31 + R) / 32;
    G.K1 = 32 * (G.ghi - G.glo + 1);
    G.lanes16 = (2 * R + 1) * (2 * R + 1) > 127 ? 1 : 0;
    const int ng = 4 * G.atoms;
    if ((G.nchunks - 1) + G.ghi > ng - 1) return false;                                   // product-1 windows
    if (G.nb == 1 && (G.nchunks - 1) + (G.PADC - 16) / 32 + 1 > ng - 1) return false;     // centre groups
    if ((2 * R + 1) * (2 * R + 1) >= (1 << 15) || 2 * R + 1 > 255) return false;
    // deepest X ring and double H buffers that fit, in that order of preference
    static const int pref[][2] = {{4, 2}, {3, 2}, {2, 2}, {2, 1}, {1, 2}, {1, 1}};
    for (const auto& pr : pref) {
        if (smem_layout(pr[0], G.atoms, pr[1], G.K1, G.nb).total + 1024 <= kSmemLimit) {
            G.stages = pr[0];
            G.nhs = pr[1];
            return true;
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
    TensorGeometry G{};
    if (!tensor_geometry(R, G)) {
        snprintf(why, why_len, "no tile shape for R=%d", R);
        return nullptr;
    }
    TensorPlan* P = new TensorPlan();
    const int bits = G.lanes16 ? 16 : 8;
    const uint32_t bcast = G.lanes16 ? 0x00010001u : 0x01010101u;
    int nlo_d, hiH_d, nlo_s, hiH_s;
    lane_consts(rule.bmin, rule.bmax, bits, nlo_d, hiH_d);
    lane_consts(rule.smin + 1, rule.smax + 1, bits, nlo_s, hiH_s);
    // epilogue balance, per column half (<= 4 chunks): the rule of the half's
    // chunk c runs on group c; its re-quantisations go first to the groups
    // without a rule chunk, then round-robin, so that no group has more than one
    // chunk of each kind per unit (the epilogue issues both TMEM loads at once)
    uint32_t rq_mask[kGroups] = {0, 0, 0, 0};
    for (int h = 0; h < 2; ++h) {
        const int c0 = h ? G.half0 : 0, c1 = h ? G.nchunks : G.half0;
        const int nc = c1 - c0;  // 1..4
        for (int k = 0; k < nc; ++k) rq_mask[(nc + k) % kGroups] |= 1u << (c0 + k);
    }
    const int ng = 4 * G.atoms;
    const int nw = a.nw;
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
        q.glo = G.glo;
        q.K1 = G.K1;
        q.Tr = G.Tr;
        q.Tc = G.Tc;
        q.nchunks = G.nchunks;
        q.half0 = G.half0;
        q.atoms = G.atoms;
        q.nb = G.nb;
        q.stages = G.stages;
        q.nhs = G.nhs;
        q.tiles_x = (a.n + G.Tc - 1) / G.Tc;
        q.tiles_y = (a.n + G.Tr - 1) / G.Tr;
        q.nlo0 = (uint32_t)nlo_d * bcast;
        q.dlo = (uint32_t)(nlo_s - nlo_d);
        q.hiH0 = (uint32_t)hiH_d * bcast;
        q.dhi = (uint32_t)(hiH_s - hiH_d);
        for (int g = 0; g < kGroups; ++g) q.rq_mask[g] = rq_mask[g];
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
    // one correction wraps a row (rows span [-R, n + 128 nb)) and a word index
    // (words span [-(PADC + 16) / 32, nw + ng)); groups are word halves
    const bool fast = a.n % 32 == 0 && nw > ng + 6 && a.n >= 128 * G.nb + R;
    P->kernel = G.glo == 0 ? pick_kernel(G.lanes16 != 0, G.nb == 1, fast, G.atoms, G.K1 / 32) : nullptr;
    if (!P->kernel) {
        snprintf(why, why_len, "no kernel instantiation for R=%d", R);
        cudaFree(P->err);
        delete P;
        return nullptr;
    }
    P->smem_bytes = smem_layout(G.stages, G.atoms, G.nhs, G.K1, G.nb).total + 1024;
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
int tensor_plan_operand_bits(const TensorPlan*) { return 8; }
unsigned int* tensor_plan_error_flag(TensorPlan* p) { return p ? p->err : nullptr; }

cudaError_t launch_tensor_pass(TensorPlan* p, bool src_is_a, cudaStream_t s) {
    const int i = src_is_a ? 0 : 1;
    p->kernel<<<p->grid, kThreads, p->smem_bytes, s>>>(p->prm[i]);
    return cudaGetLastError();
}

}  // namespace ltl

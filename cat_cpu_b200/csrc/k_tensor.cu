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
constexpr int kAtomBytes = 128 * 128;    // one 128-row x 128-byte swizzle atom
constexpr int kXBytes = 2 * kAtomBytes;  // X tile = 128 rows x 256 columns
constexpr int kXStages = 4;
constexpr int kHCol = 0;    // TMEM column of H
constexpr int kCCol = 256;  // TMEM column of C
constexpr int kN1 = 32;     // product-1 column chunk = one output word
constexpr int kGroups = 4;  // epilogue column groups
constexpr int kEpiWarps = 4 * kGroups;
constexpr int kUnpackWarps = 4;
constexpr int kEpiWarp0 = 1 + kUnpackWarps;  // warp 0: MMA, 1..4: unpack, 5..20: epilogue
constexpr int kThreads = 32 * (kEpiWarp0 + kEpiWarps);
constexpr int kMaxChunks = 7;  // Tc <= 224
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s: far above any legitimate wait

struct TcParams {
    const uint32_t* src;  // inner word (0, 0) of the current packed frame
    uint32_t* dst;        // inner word (0, 0) of the next packed frame
    long long wpitch;     // words per frame row
    int n, nw;
    int R, PADC, glo, K1;  // column halo of a tile (16 mod 32), first window group, product-1 K
    int Tr, Tc, nchunks;
    int tiles_x, tiles_y;
    int fast;     // n % 32 == 0 and n >= 256: word-aligned wrap with one correction
    int lanes16;  // rule lanes: 0 = four 8-bit lanes (R <= 5), 1 = two 16-bit lanes
    uint32_t nlo0, dlo, hiH0, dhi;  // rule constants (lane-broadcast; d* = live minus dead, mod 2^32)
    uint32_t rq_mask[kGroups];      // bit i: this epilogue group re-quantises chunk i
    unsigned int* err;
    unsigned long long wait_ns;
    int inject_missing_commit;  // test hook: product 1 of the first tile never signals
};

struct SmemLayout {
    int x_off, hs_off, bh_off, bv_off, bar_off, tmem_off, total;
};

enum Bar { X_FULL = 0, X_EMPTY = kXStages, H_FULL = 2 * kXStages, HS_FULL, C_FULL, C_EMPTY, DRAIN, NBARS };

__host__ __device__ inline SmemLayout smem_layout(int Tc, int K1) {
    SmemLayout L{};
    int o = 0;
    L.x_off = o;
    o += kXStages * kXBytes;  // 1024-aligned stages
    L.hs_off = o;
    o += 2 * 128 * Tc;        // H as u8, MN-major, two buffers (tile parity)
    L.bh_off = o;
    o += kN1 * K1;            // B_h
    L.bv_off = o;
    o += 128 * 128;           // B_v
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

__global__ void __launch_bounds__(kThreads, 1) k_tensor_step(const __grid_constant__ TcParams p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* smem = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    const SmemLayout L = smem_layout(p.Tc, p.K1);
    uint8_t* xs = smem + L.x_off;
    uint8_t* hs = smem + L.hs_off;
    uint8_t* bh = smem + L.bh_off;
    uint8_t* bv = smem + L.bv_off;
    uint64_t* bars = (uint64_t*)(smem + L.bar_off);
    uint32_t* tmem_slot = (uint32_t*)(smem + L.tmem_off);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int R = p.R, Tc = p.Tc, K1 = p.K1;
    const int ntiles = p.tiles_x * p.tiles_y;
    int mine = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) ++mine;
    constexpr uint32_t kTmemCols = 512;

    if (tid == 0) {
        for (int i = 0; i < kXStages; ++i) {
            mbar_init(&bars[X_FULL + i], kUnpackWarps);
            mbar_init(&bars[X_EMPTY + i], kEpiWarps);
        }
        mbar_init(&bars[H_FULL], 1);
        mbar_init(&bars[HS_FULL], kEpiWarps);
        mbar_init(&bars[C_FULL], 1);
        mbar_init(&bars[C_EMPTY], kEpiWarps);
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
        const int d = xc - p.PADC - perm_sigma(nn, p.lanes16);
        bh[((k >> 4) * kN1 + nn) * 16 + (k & 15)] = (d >= -R && d <= R) ? 1 : 0;
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
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *tmem_slot;

    if (warp == 0) {
        // --------------------------- MMA issuer -----------------------------
        if (lane == 0) {
            const uint32_t ba = smem_u32(bh), va = smem_u32(bv), ha0 = smem_u32(hs);
            const uint32_t id1 = idesc_u8(kN1, false);
            const uint32_t id2 = idesc_u8(Tc, true);
            const int ksteps = K1 / 32;
            auto product1 = [&](int j) -> bool {
                const int st = j % kXStages;
                if (!mbar_wait(&bars[X_FULL + st], (uint32_t)(j / kXStages) & 1u, p.wait_ns)) return false;
                fence_after();
                const uint32_t xa = smem_u32(xs + st * kXBytes);
                for (int i = 0; i < p.nchunks; ++i) {
                    for (int s = 0; s < ksteps; ++s) {
                        const int col = 32 * (i + p.glo + s);  // X column of this K step
                        const uint64_t ad = desc_k_sw128(xa + (col >> 7) * kAtomBytes + (col & 127));
                        const uint64_t bd = desc_noswz(ba + s * 2 * kN1 * 16, kN1 * 16, 128);
                        mma_i8(tmem + kHCol + kN1 * i, ad, bd, id1, s > 0 ? 1u : 0u);
                    }
                }
                if (!(p.inject_missing_commit && j == 0)) mma_commit(&bars[H_FULL]);
                return true;
            };
            // product 2 of tile j: C = B_v * H(j), H(j) in shared-memory buffer j % 2
            auto product2 = [&](int j) -> bool {
                if (j >= 1 && !mbar_wait(&bars[C_EMPTY], (uint32_t)(j - 1) & 1u, p.wait_ns)) return false;
                fence_after();
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
            bool ok = mine >= 1 ? product1(0) : true;
            for (int j = 0; j < mine && ok; ++j) {
                ok = mbar_wait(&bars[HS_FULL], (uint32_t)j & 1u, p.wait_ns);
                if (ok && j + 1 < mine) ok = product1(j + 1);
                if (ok) ok = product2(j);
            }
            if (!ok) atomicOr(p.err, 2u);
            // never leave with an MMA in flight (TMEM is freed below)
            mma_commit(&bars[DRAIN]);
            if (!mbar_wait(&bars[DRAIN], 0u, p.wait_ns)) atomicOr(p.err, 32u);
        }
    } else if (warp < kEpiWarp0) {
        // ------------------------------ unpack ------------------------------
        // 128 threads fill a stage: 128 rows x 8 groups of 32 columns.  Thread
        // ut always handles group g = ut % 8 of rows ut / 8 + 16 q, q = 0..7
        // (4 rows x 8 groups per warp and round).  The words of the next tile are
        // loaded while this one is spread and stored, so the loads' latency is
        // spent waiting for a free stage rather than on the critical path.
        const int ut = tid - 32;
        const int g = ut & 7;
        // the 8 groups (32 cells each, bit b = cell b) this thread stores for tile t
        auto gather = [&](int t, uint32_t (&x)[8]) {
            const int ty = t / p.tiles_x, tx = t % p.tiles_x;
            const int rbase = ty * p.Tr - R;
            const int cbase = tx * Tc - p.PADC;  // column of X-tile column 0 (16 mod 32)
            if (p.fast) {
                int wl = (cbase + 32 * g - 16) >> 5;  // word holding the group's first cell
                if (wl < 0) wl += p.nw;
                else if (wl >= p.nw) wl -= p.nw;
                const int wr = wl + 1 == p.nw ? 0 : wl + 1;
                uint32_t lo[8], hi[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    int gr = rbase + (ut >> 3) + 16 * q;
                    if (gr < 0) gr += p.n;
                    else if (gr >= p.n) gr -= p.n;
                    const uint32_t* rp = p.src + (size_t)gr * (size_t)p.wpitch;
                    lo[q] = __ldg(rp + wl);
                    hi[q] = __ldg(rp + wr);
                }
#pragma unroll
                for (int q = 0; q < 8; ++q) x[q] = prmt(lo[q], hi[q], 0x5432u);  // upper half of wl, lower of wr
            } else {
                const int a = wrap_slow(cbase + 32 * g, p.n);
                for (int q = 0; q < 8; ++q) {
                    const int gr = wrap_slow(rbase + (ut >> 3) + 16 * q, p.n);
                    x[q] = fetch32(p.src + (size_t)gr * (size_t)p.wpitch, a, p.n);
                }
            }
        };
        bool ok = true;
        int it = 0;
        uint32_t x[8];
        if ((int)blockIdx.x < ntiles) gather(blockIdx.x, x);
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
            const int st = it % kXStages;
            if (it >= kXStages) {
                bool w = true;
                if (lane == 0) w = mbar_wait(&bars[X_EMPTY + st], ((uint32_t)(it / kXStages) & 1u) ^ 1u, p.wait_ns);
                ok = __shfl_sync(0xffffffffu, w, 0);
                if (!ok) break;
            }
            uint8_t* xst = xs + st * kXBytes + (g >> 2) * kAtomBytes;
            const int ch = 2 * (g & 3);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int row = (ut >> 3) + 16 * q;
                uint32_t u[8];
#pragma unroll
                for (int k = 0; k < 8; ++k) u[k] = (x[q] >> k) & 0x01010101u;
                uint8_t* rowp = xst + row * 128;
                const int sw = row & 7;
                *(uint4*)(rowp + ((ch ^ sw) << 4)) = make_uint4(u[0], u[1], u[2], u[3]);
                *(uint4*)(rowp + (((ch + 1) ^ sw) << 4)) = make_uint4(u[4], u[5], u[6], u[7]);
            }
            fence_proxy_async();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bars[X_FULL + st]);
            if (t + (int)gridDim.x < ntiles) gather(t + gridDim.x, x);
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
        bool ok = true;
        auto wait_all = [&](uint64_t* bar, uint32_t ph) -> bool {
            const bool w = mbar_wait(bar, ph, p.wait_ns);
            return __all_sync(0xffffffffu, w);
        };
        // re-quantise H(j) to u8 into shared-memory buffer j % 2 (MN-major B operand of product 2)
        auto requant = [&](int j) -> bool {
            if (!wait_all(&bars[H_FULL], (uint32_t)j & 1u)) return false;
            fence_after();
            uint8_t* hsb = hs + (j & 1) * 128 * Tc;
            for (int i = 0; i < p.nchunks; ++i) {
                if (!((rq_mask >> i) & 1u)) continue;
                uint32_t v[16];
                tmem_ld32p(tmem + lane_off + kHCol + kN1 * i, v);
                tmem_wait16(v);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    uint4 w;
                    w.x = prmt(v[8 * h + 0], v[8 * h + 1], 0x6420u);
                    w.y = prmt(v[8 * h + 2], v[8 * h + 3], 0x6420u);
                    w.z = prmt(v[8 * h + 4], v[8 * h + 5], 0x6420u);
                    w.w = prmt(v[8 * h + 6], v[8 * h + 7], 0x6420u);
                    *(uint4*)(hsb + ((2 * i + h) * 128 + m) * 16) = w;
                }
            }
            fence_proxy_async();
            fence_before();
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
            if (!wait_all(&bars[C_FULL], (uint32_t)j & 1u)) {
                ok = false;
                break;
            }
            fence_after();
            const int st = j % kXStages;
            const int ty = t / p.tiles_x, tx = t % p.tiles_x;
            const int gi = ty * p.Tr + m;
            const bool row_ok = (m < p.Tr) && (gi < p.n);
            const int xr = min(m + R, 127);  // X row of this output row's centre cells (rows >= Tr are not stored)
            const uint8_t* xrow = xs + st * kXBytes + xr * 128;
            const int sw = xr & 7;
            uint32_t* orow = p.dst + (size_t)(row_ok ? gi : 0) * (size_t)p.wpitch;
            const int w0 = tx * (Tc >> 5);
            for (int i = grp; i < p.nchunks; i += kGroups) {
                uint32_t v[16];
                tmem_ld32p(tmem + lane_off + kCCol + kN1 * i, v);
                // centre cells: groups ga and ga + 1 of the X row (8 words each)
                const int ga = i + aoff, gb = ga + 1;
                const uint4 a0 = *(const uint4*)(xrow + (ga >> 2) * kAtomBytes + (((2 * (ga & 3)) ^ sw) << 4));
                const uint4 a1 = *(const uint4*)(xrow + (ga >> 2) * kAtomBytes + (((2 * (ga & 3) + 1) ^ sw) << 4));
                const uint4 b0 = *(const uint4*)(xrow + (gb >> 2) * kAtomBytes + (((2 * (gb & 3)) ^ sw) << 4));
                const uint4 b1 = *(const uint4*)(xrow + (gb >> 2) * kAtomBytes + (((2 * (gb & 3) + 1) ^ sw) << 4));
                const uint32_t Ga[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
                const uint32_t Gb[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
                tmem_wait16(v);
                uint32_t acc = 0u;
                if (!p.lanes16) {
                    // accumulator column 4k+j = output cell 8j+k: four box counts per
                    // register, bit 7 of each byte lane = the rule's result
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const uint32_t B4 = prmt(v[2 * k], v[2 * k + 1], 0x6420u);
                        const uint32_t s4 = prmt(Ga[k], Gb[k], 0x5432u);
                        const uint32_t ge = (B4 + p.nlo0) + s4 * p.dlo;  // bit 7: B >= lo(s)
                        const uint32_t le = (p.hiH0 + s4 * p.dhi) - B4;  // bit 7: B <= hi(s)
                        acc |= (ge & le & 0x80808080u) >> (7 - k);
                    }
                } else {
                    // accumulator column 2r+h = output cell 16h+r: two box counts per
                    // register, bit 15 of each 16-bit lane = the rule's result
#pragma unroll
                    for (int r = 0; r < 16; ++r) {
                        const uint32_t hsel = (uint32_t)(r >> 3);
                        const uint32_t s2 = prmt(Ga[r & 7], Gb[r & 7], (2u + hsel) | 0x80u | ((4u + hsel) << 8) | 0x8000u);
                        const uint32_t ge = (v[r] + p.nlo0) + s2 * p.dlo;
                        const uint32_t le = (p.hiH0 + s2 * p.dhi) - v[r];
                        acc |= (ge & le & 0x80008000u) >> (15 - r);
                    }
                }
                const int wi = w0 + i;
                if (row_ok && wi < p.nw) orow[wi] = acc;
            }
            fence_before();
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&bars[C_EMPTY]);
                mbar_arrive(&bars[X_EMPTY + st]);
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
struct TensorPlan {
    TcParams prm[2];  // source frame a -> b, b -> a
    int smem_bytes;
    int grid;
    unsigned int* err;
};

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
    TensorPlan* P = new TensorPlan();
    const int R = rule.radius;
    const int PADC = R <= 16 ? 16 : 48;
    const int Tc = 256 - 2 * PADC;  // 224 or 160
    const int Tr = 128 - 2 * R;
    const int glo = (PADC - R) / 32;
    const int ghi = (PADC + 31 + R) / 32;
    const int K1 = 32 * (ghi - glo + 1);
    const int nchunks = Tc / 32;
    const int lanes16 = (2 * R + 1) * (2 * R + 1) > 127 ? 1 : 0;
    const int bits = lanes16 ? 16 : 8;
    const uint32_t bcast = lanes16 ? 0x00010001u : 0x01010101u;
    int nlo_d, hiH_d, nlo_s, hiH_s;
    lane_consts(rule.bmin, rule.bmax, bits, nlo_d, hiH_d);
    lane_consts(rule.smin + 1, rule.smax + 1, bits, nlo_s, hiH_s);
    if (Tr < 1 || nchunks > kMaxChunks || (nchunks - 1) + (PADC - 16) / 32 + 1 > 7 || (nchunks - 1) + ghi > 7) {
        snprintf(why, why_len, "no tile shape for R=%d", R);
        delete P;
        return nullptr;
    }
    // epilogue balance: the rule of chunk i runs on group i % 4; each
    // re-quantisation (about a quarter of a rule chunk's work) goes to the
    // group with the least work so far
    uint32_t rq_mask[kGroups] = {0, 0, 0, 0};
    int load[kGroups] = {0, 0, 0, 0};
    for (int i = 0; i < nchunks; ++i) load[i % kGroups] += 4;
    for (int i = 0; i < nchunks; ++i) {
        int g = 0;
        for (int h = 1; h < kGroups; ++h)
            if (load[h] < load[g]) g = h;
        rq_mask[g] |= 1u << i;
        load[g] += 1;
    }
    const PackedFrame* src[2] = {&a, &b};
    const PackedFrame* dst[2] = {&b, &a};
    for (int i = 0; i < 2; ++i) {
        TcParams& q = P->prm[i];
        q.src = src[i]->words + (size_t)src[i]->HR * src[i]->wpitch + src[i]->HW;
        q.dst = dst[i]->words + (size_t)dst[i]->HR * dst[i]->wpitch + dst[i]->HW;
        q.wpitch = (long long)a.wpitch;
        q.n = a.n;
        q.nw = a.nw;
        q.R = R;
        q.PADC = PADC;
        q.glo = glo;
        q.K1 = K1;
        q.Tr = Tr;
        q.Tc = Tc;
        q.nchunks = nchunks;
        q.tiles_x = (a.n + Tc - 1) / Tc;
        q.tiles_y = (a.n + Tr - 1) / Tr;
        q.fast = (a.n % 32 == 0 && a.n >= 256) ? 1 : 0;
        q.lanes16 = lanes16;
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
    P->smem_bytes = smem_layout(Tc, K1).total + 1024;
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
    k_tensor_step<<<p->grid, kThreads, p->smem_bytes, s>>>(p->prm[i]);
    return cudaGetLastError();
}

}  // namespace ltl

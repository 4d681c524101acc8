// packed_core.cuh -- bit-sliced building blocks shared by the packed kernels
// (single grid: k_packed.cu, batched: k_batch.cu).
//
// Cells are bits of 32-bit words (cell j of a row = bit j % 32 of word j / 32).
// A count over many cells is kept "bit-sliced": plane i holds bit i of the count
// of each of the 32 lanes, so one logic operation works on 32 cells.
#pragma once

#include <algorithm>

#include "ltl_kernels.h"

namespace ltl {

__host__ __device__ constexpr int bits_for(int v) {
    int b = 0;
    while ((1 << b) <= v) ++b;
    return b;
}

// Three-input logic as single lop3 operations (the compiler does not always
// fuse these bit-sliced expressions into one instruction on its own):
//   xor3    a ^ b ^ c                       (sum of a full adder)     0x96
//   maj3    (a & b) | (a & c) | (b & c)     (carry of a full adder)   0xE8
//   borrow3 (~a & (b | c)) | (b & c)        (borrow out of a - b - c) 0x8E
__device__ __forceinline__ uint32_t xor3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ uint32_t maj3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0xE8;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}
__device__ __forceinline__ uint32_t borrow3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0x8E;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
    return d;
}

// Wallace reduction: out[0..P) = bit planes of the number of set inputs per lane.
template <int M, int L, int P>
__device__ __forceinline__ void wallace(const uint32_t* v, uint32_t* out) {
    if constexpr (L < P) {
        if constexpr (M == 0) {
            out[L] = 0u;
            wallace<0, L + 1, P>(v, out);
        } else {
            constexpr int NF = (M >= 3) ? (M - 1) / 2 : 0;
            constexpr int REM = M - 2 * NF;
            constexpr int NH = (REM == 2) ? 1 : 0;
            constexpr int NC = NF + NH;
            uint32_t carry[NC > 0 ? NC : 1];
            uint32_t acc = v[0];
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                uint32_t a = acc, b = v[1 + 2 * f], c = v[2 + 2 * f];
                acc = xor3(a, b, c);
                carry[f] = maj3(a, b, c);
            }
            if constexpr (NH == 1) {
                uint32_t b = v[M - 1];
                carry[NF] = acc & b;
                acc ^= b;
            }
            out[L] = acc;
            wallace<NC, L + 1, P>(carry, out);
        }
    }
}

// B -= h (h <= B per lane), B has PB planes, h has PH planes.
template <int PB, int PH>
__device__ __forceinline__ void planes_sub(uint32_t (&B)[PB], const uint32_t (&h)[PH]) {
    uint32_t br = 0u;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
        const uint32_t b = B[i];
        if (i < PH) {
            B[i] = xor3(b, h[i], br);
            br = borrow3(b, h[i], br);
        } else {
            B[i] = b ^ br;
            br = ~b & br;
        }
    }
}

// B += h
template <int PB, int PH>
__device__ __forceinline__ void planes_add(uint32_t (&B)[PB], const uint32_t (&h)[PH]) {
    uint32_t cy = 0u;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
        const uint32_t b = B[i];
        if (i < PH) {
            B[i] = xor3(b, h[i], cy);
            cy = maj3(b, h[i], cy);
        } else {
            B[i] = b ^ cy;
            cy = b & cy;
        }
    }
}

// One step of each comparator chain as a single three-input logic operation
// (written as lop3 so that the run-time mask operand costs one instruction):
//   ge_step(m, b, ge) = m ? (b & ge) : (b | ge)      truth table 0x8E
//   le_step(m, b, le) = m ? (~b | le) : (~b & le)    truth table 0xB2
__device__ __forceinline__ uint32_t ge_step(uint32_t m, uint32_t b, uint32_t ge) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0x8E;" : "=r"(d) : "r"(m), "r"(b), "r"(ge));
    return d;
}
__device__ __forceinline__ uint32_t le_step(uint32_t m, uint32_t b, uint32_t le) {
    uint32_t d;
    asm("lop3.b32 %0, %1, %2, %3, 0xB2;" : "=r"(d) : "r"(m), "r"(b), "r"(le));
    return d;
}

// Lanes where lo <= B <= hi, given the thresholds as per-plane masks (all-ones
// where the threshold's bit is set); lo, hi < 2^PB.  Two carry chains from the
// least significant plane up:
//   ge = carry out of B + ~lo + 1,  le = carry out of hi + ~B + 1.
template <int PB>
__device__ __forceinline__ uint32_t planes_in(const uint32_t (&B)[PB], const uint32_t* lm, const uint32_t* hm) {
    uint32_t ge = 0xffffffffu, le = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
        ge = ge_step(lm[i], B[i], ge);
        le = le_step(hm[i], B[i], le);
    }
    return ge & le;
}

constexpr int kMaxPlanes = 16;

// Birth (dead cell, index 0) and survival (live cell, index 1) intervals on the
// box count B, as per-plane bit masks (kernel parameters, so the comparator
// reads them from the constant bank).  `keep` is ~0u, or 0 for an empty interval.
struct PackedRule {
    uint32_t lo[2][kMaxPlanes];
    uint32_t hi[2][kMaxPlanes];
    uint32_t keep[2];
};

inline PackedRule make_packed_rule(const Rule& r) {
    const int maxB = (2 * r.radius + 1) * (2 * r.radius + 1);
    PackedRule p{};
    const int los[2] = {r.bmin, r.smin + 1};
    const int his[2] = {r.bmax, r.smax + 1};
    for (int k = 0; k < 2; ++k) {
        int lo = std::max(los[k], 0), hi = std::min(his[k], maxB);
        p.keep[k] = lo > hi ? 0u : 0xffffffffu;
        if (lo > hi) lo = hi = 0;
        for (int i = 0; i < kMaxPlanes; ++i) {
            p.lo[k][i] = ((lo >> i) & 1) ? 0xffffffffu : 0u;
            p.hi[k][i] = ((hi >> i) & 1) ? 0xffffffffu : 0u;
        }
    }
    return p;
}

// Horizontal window count of one frame row for word column fw (frame column).
// All lanes of the warp must call it together (shuffles).  kGlobal selects the
// read-only global load path; rows in shared memory use plain loads.
template <int R, int PH, bool kGlobal = true>
__device__ __forceinline__ void hcount(const uint32_t* __restrict__ row, int fw, bool active, int lane,
                                       uint32_t (&h)[PH]) {
    auto ld = [&](int i) -> uint32_t {
        if constexpr (kGlobal) {
            return __ldg(row + i);
        } else {
            return row[i];
        }
    };
    uint32_t own = active ? ld(fw) : 0u;
    uint32_t left = __shfl_up_sync(0xffffffffu, own, 1);
    uint32_t right = __shfl_down_sync(0xffffffffu, own, 1);
    if (lane == 0 && active) left = ld(fw - 1);
    if (lane == 31 && active) right = ld(fw + 1);
    uint32_t x[2 * R + 1];
#pragma unroll
    for (int d = -R; d <= R; ++d) {
        uint32_t v;
        if (d == 0)
            v = own;
        else if (d > 0)
            v = __funnelshift_rc(own, right, d);   // cells j + d: higher bits, then the right word
        else
            v = __funnelshift_lc(left, own, -d);   // cells j - |d|: lower bits, then the left word
        x[d + R] = v;
    }
    wallace<2 * R + 1, 0, PH>(x, h);
}

// Shared-memory ring of the last 2R+2 row counts h (PH planes per lane, one
// ring per warp), so that each row's horizontal count is computed once on
// entry and read back on exit.  Without it (kRing = false) the leaving row is
// counted again.
template <int R, int kWarps>
struct PackedRing {
    static constexpr int PH = bits_for(2 * R + 1);
    static constexpr int ROWS = 2 * R + 2;
    static constexpr int WARP_WORDS = ROWS * PH * 32;
    static constexpr int BYTES = WARP_WORDS * 4 * kWarps;
    static constexpr bool fits = BYTES <= 96 * 1024;
};

// One warp's band of output rows [r0, r1) of a packed frame, word column fw
// of each lane: next = s ? [smin+1 <= B <= smax+1] : [bmin <= B <= bmax] with
// B the box count (centre included), kept as PB bit planes and slid down the
// band (B -= h(r - R), B += h(r + R + 1)).  `cur`/`nxt` point at frame row 0,
// `HR` halo rows, `wp` words per frame row.  ring_lane = this warp's ring + lane
// (unused when !kRing).  All lanes of the warp must call it together.
// kFuse: the output frame's halo is written here too (one halo word per side,
// n a multiple of 32 and n >= 2R + 2): every halo word and halo row is a copy of
// an inner word or row, so the lane that computes a word also stores it where
// the torus repeats it -- inner word nw - 1 in the left halo word, word 0 in
// the right one, rows n - R .. n - 1 above the grid, rows 0 .. R below -- and
// no halo pass runs between generations.
template <int R, bool kRing, bool kFuse = false>
__device__ __forceinline__ void packed_band(const uint32_t* __restrict__ cur, uint32_t* __restrict__ nxt, size_t wp,
                                            int HR, int r0, int r1, int fw, bool active, bool outputs, int lane,
                                            uint32_t* ring_lane, const PackedRule& pr, int n = 0, int nw = 0) {
    constexpr int PH = bits_for(2 * R + 1);
    constexpr int PB = bits_for((2 * R + 1) * (2 * R + 1));
    constexpr int RING = 2 * R + 2;
    // row pointers advance by one frame row per output row; the ring slots of
    // rows r - R (read back) and r + R + 1 (written) advance with them
    const uint32_t* rin = cur + (size_t)(HR + r0 - R) * wp;   // next row to count
    const uint32_t* rs = cur + (size_t)(HR + r0) * wp + fw;   // centre row
    uint32_t* ro = nxt + (size_t)(HR + r0) * wp + fw;         // output row
    // kFuse: where this lane's word repeats in the same row (the other halo
    // word column, or 0), and the row distance of a repeated row
    const ptrdiff_t fdc = !kFuse ? 0 : fw - 1 == nw - 1 ? -(ptrdiff_t)nw : (fw - 1 == 0 ? (ptrdiff_t)nw : 0);
    const ptrdiff_t fnr = (ptrdiff_t)n * (ptrdiff_t)wp;
    uint32_t B[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) B[i] = 0u;
#pragma unroll 1
    for (int k = 0; k < 2 * R + 1; ++k, rin += wp) {
        uint32_t h[PH];
        hcount<R, PH>(rin, fw, active, lane, h);
        planes_add<PB, PH>(B, h);
        if constexpr (kRing) {
            uint32_t* sl = ring_lane + k * PH * 32;
#pragma unroll
            for (int i = 0; i < PH; ++i) sl[32 * i] = h[i];
        }
    }
    int out_slot = 0;  // ring slot of row r - R; row r + R + 1 goes to the slot before it
#pragma unroll 1
    for (int r = r0; r < r1; ++r, rs += wp, ro += wp, rin += wp) {
        if (outputs) {
            const uint32_t sv = __ldg(rs);
            const uint32_t in1 = planes_in<PB>(B, pr.lo[1], pr.hi[1]) & pr.keep[1];
            const uint32_t in0 = planes_in<PB>(B, pr.lo[0], pr.hi[0]) & pr.keep[0];
            const uint32_t val = (sv & in1) | (~sv & in0);
            *ro = val;
            if constexpr (kFuse) {
                if (fdc) ro[fdc] = val;
                if (r <= R || r >= n - R) {  // a row the torus repeats above or below the grid
                    const ptrdiff_t dr = r <= R ? fnr : -fnr;
                    ro[dr] = val;
                    if (fdc) ro[dr + fdc] = val;
                }
            }
        }
        if (r + 1 < r1) {
            uint32_t h[PH];
            const int in_slot = out_slot == 0 ? RING - 1 : out_slot - 1;
            if constexpr (kRing) {
                const uint32_t* sl = ring_lane + out_slot * PH * 32;
#pragma unroll
                for (int i = 0; i < PH; ++i) h[i] = sl[32 * i];
            } else {
                hcount<R, PH>(rin - (size_t)(2 * R + 1) * wp, fw, active, lane, h);
            }
            planes_sub<PB, PH>(B, h);
            hcount<R, PH>(rin, fw, active, lane, h);
            planes_add<PB, PH>(B, h);
            if constexpr (kRing) {
                uint32_t* sl = ring_lane + in_slot * PH * 32;
#pragma unroll
                for (int i = 0; i < PH; ++i) sl[32 * i] = h[i];
            }
            out_slot = out_slot + 1 == RING ? 0 : out_slot + 1;
        }
    }
}

// Horizontal window count for the segmented band walk below: lanes work in
// segments, and a lane at a segment's edge (edge_l / edge_r) loads its
// neighbouring word itself instead of taking it from the next lane.  Loads go
// through L1 without the read-only path (ld.global.ca), so words this CTA wrote
// before a __syncthreads are seen.
template <int R, int PH>
__device__ __forceinline__ void hcount_seg(const uint32_t* row, int fw, bool active, bool edge_l, bool edge_r,
                                           uint32_t (&h)[PH]) {
    const uint32_t own = active ? __ldca(row + fw) : 0u;
    uint32_t left = __shfl_up_sync(0xffffffffu, own, 1);
    uint32_t right = __shfl_down_sync(0xffffffffu, own, 1);
    if (edge_l && active) left = __ldca(row + fw - 1);
    if (edge_r && active) right = __ldca(row + fw + 1);
    uint32_t x[2 * R + 1];
#pragma unroll
    for (int d = -R; d <= R; ++d) {
        uint32_t v;
        if (d == 0)
            v = own;
        else if (d > 0)
            v = __funnelshift_rc(own, right, d);
        else
            v = __funnelshift_lc(left, own, -d);
        x[d + R] = v;
    }
    wallace<2 * R + 1, 0, PH>(x, h);
}

// packed_band for warps whose lanes work on different row bands: every lane
// has its own band [r0, r1) (the same for the lanes of one segment), and the
// whole warp runs `len` >= r1 - r0 iterations so that its shuffles stay
// converged; a lane stops loading and writing once its band has ended.  The
// h ring (kRing) is per lane, as in packed_band.  All lanes call it together.
template <int R, bool kRing>
__device__ __forceinline__ void packed_band_seg(const uint32_t* cur, uint32_t* nxt, size_t wp, int HR, int r0, int r1,
                                                int len, int fw, bool active, bool edge_l, bool edge_r,
                                                uint32_t* ring_lane, const PackedRule& pr) {
    constexpr int PH = bits_for(2 * R + 1);
    constexpr int PB = bits_for((2 * R + 1) * (2 * R + 1));
    constexpr int RING = 2 * R + 2;
    const uint32_t* rin = cur + (size_t)(HR + r0 - R) * wp;  // next row to count
    const uint32_t* rs = cur + (size_t)(HR + r0) * wp + fw;  // centre row
    uint32_t* ro = nxt + (size_t)(HR + r0) * wp + fw;        // output row
    uint32_t B[PB];
#pragma unroll
    for (int i = 0; i < PB; ++i) B[i] = 0u;
    const bool live0 = active && r0 < r1;
#pragma unroll 1
    for (int k = 0; k < 2 * R + 1; ++k, rin += wp) {
        uint32_t h[PH];
        hcount_seg<R, PH>(rin, fw, live0, edge_l, edge_r, h);
        planes_add<PB, PH>(B, h);
        if constexpr (kRing) {
            uint32_t* sl = ring_lane + k * PH * 32;
#pragma unroll
            for (int i = 0; i < PH; ++i) sl[32 * i] = h[i];
        }
    }
    int out_slot = 0;  // ring slot of row r - R; row r + R + 1 goes to the slot before it
#pragma unroll 1
    for (int k = 0; k < len; ++k, rs += wp, ro += wp, rin += wp) {
        const int r = r0 + k;
        if (active && r < r1) {
            const uint32_t sv = __ldca(rs);
            const uint32_t in1 = planes_in<PB>(B, pr.lo[1], pr.hi[1]) & pr.keep[1];
            const uint32_t in0 = planes_in<PB>(B, pr.lo[0], pr.hi[0]) & pr.keep[0];
            *ro = (sv & in1) | (~sv & in0);
        }
        if (k + 1 < len) {
            const bool live = active && r + 1 < r1;
            uint32_t h[PH];
            const int in_slot = out_slot == 0 ? RING - 1 : out_slot - 1;
            if constexpr (kRing) {
                const uint32_t* sl = ring_lane + out_slot * PH * 32;
#pragma unroll
                for (int i = 0; i < PH; ++i) h[i] = sl[32 * i];
            } else {
                hcount_seg<R, PH>(rin - (size_t)(2 * R + 1) * wp, fw, live, edge_l, edge_r, h);
            }
            planes_sub<PB, PH>(B, h);
            hcount_seg<R, PH>(rin, fw, live, edge_l, edge_r, h);
            planes_add<PB, PH>(B, h);
            if constexpr (kRing) {
                uint32_t* sl = ring_lane + in_slot * PH * 32;
#pragma unroll
                for (int i = 0; i < PH; ++i) sl[32 * i] = h[i];
            }
            out_slot = out_slot + 1 == RING ? 0 : out_slot + 1;
        }
    }
}

// Halo word fw of a packed frame row with one halo word per side (inner word w
// at frame word 1 + w): fw = 0 is the left halo (cells n-32 .. n-1), fw = nw
// the last inner word with its bits past n rewritten (cells 0 ..), fw = nw + 1
// the right halo (cells 32 nw - n .. 32 nw - n + 31).  For n >= 64 each is a
// funnel shift of two inner words; `slow` handles smaller grids bit by bit.
// Only inner bits (< n) are read, so concurrent writers of other halo words
// of the same row do not matter.
template <class Slow>
__device__ __forceinline__ uint32_t packed_halo_word(const uint32_t* row, int fw, int n, int nw, Slow&& slow) {
    if (n >= 64) {
        if (fw == nw) {
            const int ib = n - 32 * (nw - 1);  // inner bits of the last word, 1..32
            return ib >= 32 ? row[fw] : ((row[fw] & ((1u << ib) - 1u)) | (row[1] << ib));
        }
        const int c = fw == 0 ? n - 32 : 32 * nw - n;  // first cell of the word
        const uint32_t lo = row[1 + (c >> 5)];
        return (c & 31) ? __funnelshift_r(lo, row[2 + (c >> 5)], c & 31) : lo;
    }
    return slow();
}

}  // namespace ltl

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
                acc = a ^ b ^ c;
                carry[f] = (a & b) | (a & c) | (b & c);
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
        uint32_t b = B[i];
        uint32_t x = (i < PH) ? h[i] : 0u;
        B[i] = b ^ x ^ br;
        br = (~b & (x | br)) | (x & br);
    }
}

// B += h
template <int PB, int PH>
__device__ __forceinline__ void planes_add(uint32_t (&B)[PB], const uint32_t (&h)[PH]) {
    uint32_t cy = 0u;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
        uint32_t b = B[i];
        uint32_t x = (i < PH) ? h[i] : 0u;
        B[i] = b ^ x ^ cy;
        cy = (b & x) | (b & cy) | (x & cy);
    }
}

// Lanes where lo <= B <= hi, given the thresholds as per-plane masks (all-ones
// where the threshold's bit is set); lo, hi < 2^PB.  Two carry chains:
//   ge = carry out of B + ~lo + 1,  le = carry out of hi + ~B + 1.
template <int PB>
__device__ __forceinline__ uint32_t planes_in(const uint32_t (&B)[PB], const uint32_t* lm, const uint32_t* hm) {
    uint32_t ge = 0xffffffffu, le = 0xffffffffu;
#pragma unroll
    for (int i = 0; i < PB; ++i) {
        const uint32_t b = B[i];
        ge = (lm[i] & (b & ge)) | (~lm[i] & (b | ge));
        le = (hm[i] & (~b | le)) | (~hm[i] & (~b & le));
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

}  // namespace ltl

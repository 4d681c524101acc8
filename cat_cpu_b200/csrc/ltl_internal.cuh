// ltl_internal.cuh -- shared layout, rule and error helpers of libltl_b200.
//
// Device grid layout (every variant that stores one byte per cell):
//   a frame of (n + 2H) rows, `pitch` bytes per row, inner cell (i, j) at
//   base[(H + i) * pitch + H + j].  H is a multiple of 16 and >= R * depth, the
//   halo holds torus copies of inner cells (frame cell (r, c) = inner
//   ((r - H) mod n, (c - H) mod n)), refreshed by k_halo_fill before each pass.
//   This is the reference's CADataDomain layout (CADataDomain.tpp:4-98, inner
//   (i,j) at (i+h)*(n+2h) + j+h) with the halo rounded up to 16 bytes and the
//   pitch padded so that 16-byte vector and TMA accesses stay aligned and a
//   16-byte load that starts inside the right halo stays inside its row.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace ltl {

constexpr int kWarp = 32;

struct Frame {
    uint8_t* base;   // frame origin (row 0, column 0)
    int n;           // inner columns (and rows, unless `rows` is set)
    int H;           // halo width (cells)
    size_t pitch;    // bytes per frame row
    int rows = 0;    // inner rows of a rectangular torus (0: square, n rows)
    __host__ __device__ int nrows() const { return rows ? rows : n; }
    __host__ __device__ uint8_t* inner(int i, int j) const { return base + (size_t)(H + i) * pitch + H + j; }
    __host__ __device__ const uint8_t* cinner(int i, int j) const {
        return base + (size_t)(H + i) * pitch + H + j;
    }
};

__host__ __device__ inline size_t round_up(size_t v, size_t m) { return (v + m - 1) / m * m; }

inline int halo_for(int radius, int depth) {
    int h = radius * depth;
    if (h < 16) h = 16;
    return (int)round_up((size_t)h, 16);
}

inline size_t pitch_for(int n, int H) { return round_up((size_t)n + 2 * (size_t)H + 16, 64); }

// Rule in the reference's centre-excluded convention.
struct Rule {
    int radius, smin, smax, bmin, bmax;
};

// Thresholds on the box count B (centre INCLUDED) for 8-bit SWAR lanes holding
// B <= 127: alive cell survives iff slo <= B <= shi (slo = smin+1, shi = smax+1,
// since k = B - 1), dead cell is born iff blo <= B <= bhi.  Empty intervals are
// encoded lo = 128, hi = 0; lo is clamped to [0,128], hi to [0,127].  Each value
// is broadcast to the four byte lanes, lo as 0x80 - lo (so that B + (0x80 - lo)
// has bit 7 set iff B >= lo, without a carry into the next lane) and hi with
// the 0x80 marker bit (0x80 + hi - B has bit 7 set iff B <= hi).  `d*` hold the
// XOR of the dead and live values, for a one-operation select by the centre.
struct RuleSwar8 {
    uint32_t nlo0, hiH0;  // dead cell (birth interval)
    uint32_t dnlo, dhiH;  // XOR of the dead- and live-cell (survival) values
};

inline void clamp_interval8(int lo, int hi, uint32_t& nlo_out, uint32_t& hi_out) {
    if (lo < 0) lo = 0;
    if (hi > 127) hi = 127;
    if (hi < lo || lo > 127) {
        lo = 128;
        hi = 0;
    }
    nlo_out = (uint32_t)(0x80 - lo) * 0x01010101u;
    hi_out = ((uint32_t)hi | 0x80u) * 0x01010101u;
}

inline RuleSwar8 make_rule_swar8(const Rule& r) {
    uint32_t nlo0, hi0, nlo1, hi1;
    clamp_interval8(r.bmin, r.bmax, nlo0, hi0);
    clamp_interval8(r.smin + 1, r.smax + 1, nlo1, hi1);
    return RuleSwar8{nlo0, hi0, nlo0 ^ nlo1, hi0 ^ hi1};
}

// Per byte lane: 1 if the lane's cell is alive in the next generation.
// B: four box counts (centre included, each <= 127); s: four centre cells (0/1).
__device__ __forceinline__ uint32_t rule_swar8(uint32_t B, uint32_t s, const RuleSwar8& q) {
    const uint32_t m = s * 0xFFu;                     // 0x00 / 0xFF per lane
    const uint32_t nlo = q.nlo0 ^ (m & q.dnlo);
    const uint32_t hiH = q.hiH0 ^ (m & q.dhiH);
    const uint32_t ge = B + nlo;                      // bit 7 set iff B >= lo
    const uint32_t le = hiH - B;                      // bit 7 set iff hi >= B
    return ((ge & le) >> 7) & 0x01010101u;
}

__device__ __forceinline__ int rule_scalar(int k, int s, int smin, int smax, int bmin, int bmax) {
    return s ? (k >= smin && k <= smax) : (k >= bmin && k <= bmax);
}

__device__ __forceinline__ int wrap_mod(int v, int n) {
    int r = v % n;
    return r < 0 ? r + n : r;
}

}  // namespace ltl

// Host-side error reporting (ltl_abi.cu).
void ltl_set_error(const char* fmt, ...);

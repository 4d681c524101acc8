// k_noalloc.cu -- ltl_step_noalloc: the plain CUDA-core step for callers that
// cannot allocate device memory.
//
// Some callers may not call cudaMalloc at all:
//   - code that runs while a host framework owns every byte of device memory
//     through its own pool, where a raw allocation breaks the framework's budget
//     or fragments its pool;
//   - real-time or long-running services that allocate once at start-up and
//     forbid allocation (and the implicit synchronisation cudaMalloc/cudaFree
//     bring) on the hot path;
//   - plug-ins that are handed device buffers and a stream and nothing else.
// The regular entry points allocate two halo'd grids per solver.  This entry
// point instead keeps that scratch in one fixed array in device global memory
// that is part of the library image:
// every GPU that loads libltl_b200.so holds kNoAllocScratchBytes of it until
// the process exits, and no call allocates or frees anything.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/ltl.h"
#include "ltl_kernels.h"

namespace ltl {

// 32 MiB: two halo'd grids.  A grid needs round_up((n + 2H + 1) * pitch, 256)
// bytes with H = halo_for(R, 1) and pitch = round_up(n + 2H + 16, 64), so the
// limit is n <= 4048 for R <= 16 (H = 16) and smaller n for larger R.
constexpr size_t kNoAllocScratchBytes = 32ull << 20;

// The scratch.  Host code only sees a host-side stand-in for this symbol; the
// device address comes from cudaGetSymbolAddress (noalloc_scratch_address).
static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
static void* g_scratch_addr[kMaxDevices] = {};
static bool g_prepared[kMaxDevices][6] = {};  // radius 1..5 kernels' attributes set
static std::mutex g_mu;

// Device address of the scratch on `device` (which must be current), looked
// up once per device.
static cudaError_t noalloc_scratch_address(int device, void** out) {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[device] = p;
    }
    *out = g_scratch_addr[device];
    return cudaSuccess;
}

}  // namespace ltl

using namespace ltl;

extern "C" int ltl_step_noalloc(const uint8_t* dev_in, size_t in_pitch, uint8_t* dev_out, size_t out_pitch, int n,
                                int radius, int smin, int smax, int bmin, int bmax, int steps, void* stream) {
    if (!dev_in || !dev_out || n < 1 || radius < 1 || n < radius || steps < 0 || in_pitch < (size_t)n ||
        out_pitch < (size_t)n) {
        ltl_set_error("ltl_step_noalloc: bad arguments (n=%d, radius=%d, steps=%d)", n, radius, steps);
        return LTL_EINVAL;
    }
    const int H = halo_for(radius, 1);
    const size_t pitch = pitch_for(n, H);
    const size_t frame = round_up(((size_t)n + 2 * H + 1) * pitch, 256);
    const bool generic = !plain_swar8_supported(radius);
    const size_t need = 2 * frame;
    if (need > kNoAllocScratchBytes) {
        ltl_set_error("ltl_step_noalloc: n=%d, radius=%d needs %zu bytes of scratch; the fixed scratch holds %zu "
                      "(use ltl_create for larger grids)",
                      n, radius, need, (size_t)kNoAllocScratchBytes);
        return LTL_EINVAL;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0 || device >= kMaxDevices) {
        ltl_set_error("ltl_step_noalloc: no usable current CUDA device: %s", cudaGetErrorString(e));
        return LTL_ECUDA;
    }
    void* base = nullptr;
    e = noalloc_scratch_address(device, &base);
    if (e != cudaSuccess) {
        ltl_set_error("ltl_step_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return LTL_ECUDA;
    }
    if (!generic) {
        std::lock_guard<std::mutex> lock(g_mu);
        if (!g_prepared[device][radius]) {
            e = plain_prepare(radius);
            if (e != cudaSuccess) {
                ltl_set_error("ltl_step_noalloc: kernel setup failed: %s", cudaGetErrorString(e));
                return LTL_ECUDA;
            }
            g_prepared[device][radius] = true;
        }
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* scratch = (uint8_t*)base;
    Frame fa{scratch, n, H, pitch};
    Frame fb{scratch + frame, n, H, pitch};
    const Rule rule{radius, smin, smax, bmin, bmax};
    int band_rows = 0;
    if (!generic) band_rows = (int)tuning_lookup("plain", radius, n, "band_rows", plain_swar8_band_rows(n, device));
    // The frames are not cleared.  The inner cells are written by the copy and
    // the halo by the halo fill before any step reads them.  The kernels also
    // read bytes outside the halo'd grid (the wide kernel's loads past the right
    // halo into the pitch padding, the SWAR kernel's vector loads into the spare
    // row) and discard what they compute from them; those bytes hold whatever an
    // earlier call with another n left there.  That is safe because every byte
    // ever written to this array is a 0/1 cell, so the byte-lane sums that touch
    // stale bytes cannot carry into the lanes that are kept.  A kernel that
    // writes anything other than 0/1 cells here would break that.
    e = launch_copy_in(fa, dev_in, in_pitch, s);
    if (e == cudaSuccess) e = launch_halo_fill(fa, s);
    Frame* cur = &fa;
    Frame* nxt = &fb;
    for (int i = 0; i < steps && e == cudaSuccess; ++i) {
        e = generic ? launch_plain_generic(*cur, *nxt, rule, 0, s)
                    : launch_plain_swar8(*cur, *nxt, rule, band_rows, false, s);
        if (e == cudaSuccess) e = launch_halo_fill(*nxt, s);
        Frame* t = cur;
        cur = nxt;
        nxt = t;
    }
    if (e == cudaSuccess) e = launch_copy_out(*cur, dev_out, out_pitch, s);
    if (e != cudaSuccess) {
        ltl_set_error("ltl_step_noalloc: launch failed: %s", cudaGetErrorString(e));
        return LTL_ECUDA;
    }
    return LTL_OK;
}

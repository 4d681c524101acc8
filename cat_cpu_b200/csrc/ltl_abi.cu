// ltl_abi.cu -- the C ABI of libltl_b200 (include/ltl.h): solver contexts,
// variant dispatch, CUDA-graph replay of the step loop, status codes.
//
// The context plays the role of the reference's CASolver subclasses
// (src/CellularAutomata/Solvers/CASolver.h:7-28): it owns the two device
// grids (current / next, like HostSolver's dataDomain / dataDomainBuffer,
// HostSolver.tpp:5-45), uploads and downloads the host-visible grid, and runs
// doSteps as fill-halo -> step -> swap (CASolver.cpp:15-31) on one stream.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/ltl.h"
#include "ltl_kernels.h"

using namespace ltl;

static thread_local char g_err[512] = "";

void ltl_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

#define LTL_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            ltl_set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                          __LINE__);                                                       \
            return e_ == cudaErrorMemoryAllocation ? LTL_ENOMEM : LTL_ECUDA;               \
        }                                                                                  \
    } while (0)

struct ltl_ctx {
    int device = 0;
    int n = 0;       // columns (the side of a square torus)
    int rows = 0;    // rows (== n except for ltl_create_rect)
    Rule rule{};
    int variant = LTL_VARIANT_PLAIN;
    int depth = 1;
    Frame fa{}, fb{};
    bool cur_is_a = true;
    uint8_t* frames = nullptr;
    size_t frames_bytes = 0;
    unsigned long long* scratch = nullptr;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int band_rows = 64;         // plain: rows per work item
    bool plain_wrap = false;    // plain R <= 5: kernels apply the torus wrap, no halo refresh
    int packed_band_rows = 0;   // packed: rows per work item (0: heuristic)
    // packed and tensor variants: the grid lives in packed frames between steps
    PackedFrame pa{}, pb{};
    uint32_t* pwords = nullptr;
    size_t pwords_bytes = 0;
    // PACK-coded staging rows of ltl_upload_packed / ltl_download_packed (made on first use)
    uint64_t* pstage = nullptr;
    bool packed_valid = false;  // packed frames hold the current state
    // tensor variant
    TensorPlan* tplan = nullptr;
    unsigned long long wait_ns = 2000000000ull;
    bool inject = false;
    // graphs of kGraphPasses passes, one per starting buffer
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    // optional per-kernel timing (ltl_set_timing): event pairs around the main
    // step kernel(s) of every pass, and launch counters
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> ev;
    long long step_launches = 0;
    long long all_launches = 0;
};

static constexpr int kGraphPasses = 8;

static Frame& cur_frame(ltl_ctx* c) { return c->cur_is_a ? c->fa : c->fb; }
static Frame& nxt_frame(ltl_ctx* c) { return c->cur_is_a ? c->fb : c->fa; }
static PackedFrame& cur_packed(ltl_ctx* c) { return c->cur_is_a ? c->pa : c->pb; }
static PackedFrame& nxt_packed(ltl_ctx* c) { return c->cur_is_a ? c->pb : c->pa; }

static int check_ctx(const ltl_ctx* c) {
    if (!c) {
        ltl_set_error("null context");
        return LTL_EINVAL;
    }
    return LTL_OK;
}

static void free_events(ltl_ctx* c) {
    for (auto& p : c->ev) {
        cudaEventDestroy(p.first);
        cudaEventDestroy(p.second);
    }
    c->ev.clear();
}

static void release(ltl_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    free_events(c);
    for (auto& g : c->graph)
        if (g) cudaGraphExecDestroy(g);
    if (c->tplan) tensor_plan_destroy(c->tplan);
    if (c->frames) cudaFree(c->frames);
    if (c->pwords) cudaFree(c->pwords);
    if (c->pstage) cudaFree(c->pstage);
    if (c->scratch) cudaFree(c->scratch);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
}

static void drop_graphs(ltl_ctx* c) {
    for (auto& g : c->graph) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// rows x n torus (rows == n unless a rectangular form is asked for: plain and packed)
static int create_impl(ltl_ctx** out, int device, int rows, int n, int radius, int smin, int smax, int bmin,
                       int bmax, int variant) {
    if (!out) {
        ltl_set_error("ltl_create: out is NULL");
        return LTL_EINVAL;
    }
    *out = nullptr;
    if (n < 1 || radius < 1 || n < radius || rows < radius) {
        ltl_set_error("ltl_create: need n >= 1, radius >= 1 and n, rows >= radius (n=%d, rows=%d, radius=%d)", n,
                      rows, radius);
        return LTL_EINVAL;
    }
    if (rows != n && variant != LTL_VARIANT_PLAIN && variant != LTL_VARIANT_PACKED) {
        ltl_set_error("ltl_create_rect: rectangular grids are served by the plain and packed variants");
        return LTL_EUNSUPPORTED;
    }
    if (radius > 2047) {
        ltl_set_error("ltl_create: radius %d > 2047 is outside the exact range of every variant", radius);
        return LTL_EUNSUPPORTED;
    }
    if ((long long)rows * n > (1ll << 40)) {
        ltl_set_error("ltl_create: n=%d too large", n);
        return LTL_EINVAL;
    }
    if (variant == LTL_VARIANT_AUTO) variant = LTL_VARIANT_PLAIN;
    if (variant != LTL_VARIANT_PLAIN && variant != LTL_VARIANT_TENSOR && variant != LTL_VARIANT_PACKED) {
        ltl_set_error("ltl_create: unknown variant %d", variant);
        return LTL_EINVAL;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        ltl_set_error("ltl_create: CUDA device %d not available (%d devices)", device, ndev);
        return LTL_ECUDA;
    }
    if (variant == LTL_VARIANT_PLAIN && !plain_swar8_supported(radius) && !plain_generic_supported(radius)) {
        ltl_set_error("ltl_create: plain variant needs radius <= 2038 (got %d)", radius);
        return LTL_EUNSUPPORTED;
    }
    if (variant == LTL_VARIANT_PACKED && !packed_supported(n, radius)) {
        ltl_set_error("ltl_create: packed variant needs radius <= 32 (got %d)", radius);
        return LTL_EUNSUPPORTED;
    }
    char why[256] = "";
    if (variant == LTL_VARIANT_TENSOR && !tensor_supported(n, radius, why, sizeof(why))) {
        ltl_set_error("ltl_create: tensor variant: %s", why);
        return LTL_EUNSUPPORTED;
    }

    ltl_ctx* c = new (std::nothrow) ltl_ctx();
    if (!c) {
        ltl_set_error("ltl_create: host allocation failed");
        return LTL_ENOMEM;
    }
    c->device = device;
    c->n = n;
    c->rows = rows;
    c->rule = Rule{radius, smin, smax, bmin, bmax};
    c->variant = variant;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        ltl_set_error("ltl_create: %s", cudaGetErrorString(e));
        release(c);
        return LTL_ECUDA;
    }
    c->stream = c->own_stream;

    int depth = 1;
    const int H = halo_for(radius, 1);
    size_t pitch = pitch_for(n, H);
    size_t frows = (size_t)rows + 2 * H + 1;  // +1 spare row: vector loads may run past the last frame row
    size_t one = round_up(frows * pitch, 4096);
    c->frames_bytes = 2 * one;
    e = cudaMalloc(&c->frames, c->frames_bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(c->frames, 0, c->frames_bytes, c->stream);
    if (e == cudaSuccess) e = cudaMalloc(&c->scratch, 4 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        ltl_set_error("ltl_create: device allocation of %zu bytes failed: %s", c->frames_bytes,
                      cudaGetErrorString(e));
        release(c);
        return e == cudaErrorMemoryAllocation ? LTL_ENOMEM : LTL_ECUDA;
    }
    c->fa = Frame{c->frames, n, H, pitch, rows};
    c->fb = Frame{c->frames + one, n, H, pitch, rows};

    if (variant == LTL_VARIANT_PLAIN && plain_swar8_supported(radius)) {
        // generations per pass: the tuning table's value, else 2 where the
        // temporally blocked kernel applies (grids below 256 gain nothing)
        const int want = (int)tuning_lookup("plain", radius, n, "depth", n >= 256 ? 2 : 1);
        if (want > 1 && plain_tb_supported(radius, want) && H >= want * radius) depth = want;
        c->band_rows = (int)tuning_lookup("plain", radius, n, "band_rows", plain_swar8_band_rows(n, device));
        c->plain_wrap = plain_wrap_supported(n, rows);
    } else if (variant == LTL_VARIANT_PLAIN) {
        c->band_rows = (int)tuning_lookup("plain", radius, n, "band_rows", 0);  // 0: the launcher's choice
    }
    if (variant == LTL_VARIANT_PACKED) c->packed_band_rows = (int)tuning_lookup("packed", radius, n, "band_rows", 0);
    if (variant == LTL_VARIANT_PLAIN) e = plain_prepare(radius);
    if (variant == LTL_VARIANT_PLAIN && e == cudaSuccess) e = plain_tb_prepare(radius);
    if (variant == LTL_VARIANT_PACKED) e = packed_prepare(radius);
    if (e != cudaSuccess) {
        ltl_set_error("ltl_create: kernel setup failed: %s", cudaGetErrorString(e));
        release(c);
        return LTL_ECUDA;
    }
    if (variant == LTL_VARIANT_PACKED || variant == LTL_VARIANT_TENSOR) {
        // the packed step reads R + 1 halo rows; the tensor step wraps rows and
        // words itself and only needs the right halo word to exist
        PackedFrame p{};
        p.n = n;
        p.rows = rows;
        p.nw = (n + 31) / 32;
        p.HR = variant == LTL_VARIANT_PACKED ? radius + 1 : 1;
        p.HW = 1;
        p.wpitch = round_up((size_t)p.nw + 2 * p.HW + 1, 4);  // +1: edge lanes read one word past the halo
        size_t prow = (size_t)rows + 2 * p.HR;
        size_t pone = round_up(prow * p.wpitch * sizeof(uint32_t), 4096);
        c->pwords_bytes = 2 * pone;
        e = cudaMalloc(&c->pwords, c->pwords_bytes);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->pwords, 0, c->pwords_bytes, c->stream);
        if (e != cudaSuccess) {
            ltl_set_error("ltl_create: packed allocation failed: %s", cudaGetErrorString(e));
            release(c);
            return LTL_ENOMEM;
        }
        c->pa = p;
        c->pa.words = c->pwords;
        c->pb = p;
        c->pb.words = (uint32_t*)((uint8_t*)c->pwords + pone);
    }
    if (variant == LTL_VARIANT_TENSOR) {
        c->tplan = tensor_plan_create(c->pa, c->pb, c->rule, device, why, sizeof(why));
        if (!c->tplan) {
            ltl_set_error("ltl_create: tensor plan: %s", why);
            release(c);
            return LTL_EUNSUPPORTED;
        }
        depth = tensor_plan_depth(c->tplan);
    }
    c->depth = depth;
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) {
        ltl_set_error("ltl_create: %s", cudaGetErrorString(e));
        release(c);
        return LTL_ECUDA;
    }
    *out = c;
    return LTL_OK;
}

extern "C" int ltl_create(ltl_ctx** out, int device, int n, int radius, int smin, int smax, int bmin, int bmax,
                          int variant) {
    return create_impl(out, device, n, n, radius, smin, smax, bmin, bmax, variant);
}

extern "C" int ltl_create_rect(ltl_ctx** out, int device, int rows, int cols, int radius, int smin, int smax,
                               int bmin, int bmax) {
    return create_impl(out, device, rows, cols, radius, smin, smax, bmin, bmax, LTL_VARIANT_PLAIN);
}

extern "C" int ltl_create_rect_variant(ltl_ctx** out, int device, int rows, int cols, int radius, int smin,
                                       int smax, int bmin, int bmax, int variant) {
    if (variant == LTL_VARIANT_AUTO) variant = LTL_VARIANT_PLAIN;
    return create_impl(out, device, rows, cols, radius, smin, smax, bmin, bmax, variant);
}

extern "C" int ltl_destroy(ltl_ctx* c) {
    if (!c) return LTL_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    release(c);
    return LTL_OK;
}

extern "C" int ltl_set_stream(ltl_ctx* c, void* stream) {
    if (int r = check_ctx(c)) return r;
    cudaSetDevice(c->device);
    cudaStream_t s = stream ? (cudaStream_t)stream : c->own_stream;
    if (s != c->stream) drop_graphs(c);
    c->stream = s;
    return LTL_OK;
}

extern "C" int ltl_get_info(const ltl_ctx* c, ltl_info* info) {
    if (int r = check_ctx(c)) return r;
    if (!info) {
        ltl_set_error("ltl_get_info: info is NULL");
        return LTL_EINVAL;
    }
    info->variant = c->variant;
    info->n = c->n;
    info->rows = c->rows;
    info->radius = c->rule.radius;
    info->smin = c->rule.smin;
    info->smax = c->rule.smax;
    info->bmin = c->rule.bmin;
    info->bmax = c->rule.bmax;
    info->halo = c->fa.H;
    info->pitch = (long long)c->fa.pitch;
    info->temporal_depth = c->depth;
    info->operand_bits = c->tplan ? tensor_plan_operand_bits(c->tplan) : 0;
    info->device_bytes = (long long)(c->frames_bytes + c->pwords_bytes);
    return LTL_OK;
}

// Make the packed frames hold the byte frame's state (packed variant keeps its
// state packed between steps; the byte frame is refreshed on download).
static bool keeps_packed(const ltl_ctx* c) {
    return c->variant == LTL_VARIANT_PACKED || c->variant == LTL_VARIANT_TENSOR;
}

static int sync_to_packed(ltl_ctx* c) {
    Frame& f = cur_frame(c);
    LTL_CUDA(launch_pack_frame(f, cur_packed(c), c->stream));
    if (c->variant == LTL_VARIANT_PACKED) LTL_CUDA(launch_packed_halo(cur_packed(c), c->stream));
    c->packed_valid = true;
    return LTL_OK;
}

static int sync_from_packed(ltl_ctx* c) {
    if (!keeps_packed(c) || !c->packed_valid) return LTL_OK;
    LTL_CUDA(launch_unpack_frame(cur_packed(c), cur_frame(c), c->stream));
    return LTL_OK;
}

static int after_upload(ltl_ctx* c) {
    LTL_CUDA(launch_halo_fill(cur_frame(c), c->stream));
    c->packed_valid = false;
    if (keeps_packed(c)) return sync_to_packed(c);
    return LTL_OK;
}

__global__ void k_binarize(uint8_t* g, int n, int rows, int H, size_t pitch) {
    const long long total = (long long)rows * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int i = (int)(t / n), j = (int)(t % n);
        uint8_t* p = g + (size_t)(H + i) * pitch + H + j;
        *p = *p ? 1 : 0;
    }
}

extern "C" int ltl_upload(ltl_ctx* c, const uint8_t* inner, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (!inner || pitch < (size_t)c->n) {
        ltl_set_error("ltl_upload: bad buffer or pitch %zu < n %d", pitch, c->n);
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    Frame& f = cur_frame(c);
    LTL_CUDA(cudaMemcpy2DAsync(f.inner(0, 0), f.pitch, inner, pitch, c->n, c->rows, cudaMemcpyHostToDevice,
                               c->stream));
    long long total = (long long)c->rows * c->n;
    k_binarize<<<(int)std::min<long long>((total + 255) / 256, 148 * 32), 256, 0, c->stream>>>(
        f.base, c->n, c->rows, f.H, f.pitch);
    LTL_CUDA(cudaGetLastError());
    if (int r = after_upload(c)) return r;
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    return LTL_OK;
}

extern "C" int ltl_upload_device(ltl_ctx* c, const uint8_t* dev_inner, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (!dev_inner || pitch < (size_t)c->n) {
        ltl_set_error("ltl_upload_device: bad buffer or pitch");
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    LTL_CUDA(launch_copy_in(cur_frame(c), dev_inner, pitch, c->stream));
    return after_upload(c);
}

extern "C" int ltl_download(ltl_ctx* c, uint8_t* inner, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (!inner || pitch < (size_t)c->n) {
        ltl_set_error("ltl_download: bad buffer or pitch %zu < n %d", pitch, c->n);
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    if (int r = sync_from_packed(c)) return r;
    Frame& f = cur_frame(c);
    LTL_CUDA(cudaMemcpy2DAsync(inner, pitch, f.inner(0, 0), f.pitch, c->n, c->rows, cudaMemcpyDeviceToHost,
                               c->stream));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    return LTL_OK;
}

// ---------------------------------------------------------------------------
// Host transfers in the PACK coding (ceil(n / 64) uint64 words per row).
// ---------------------------------------------------------------------------
static int pack_args(ltl_ctx* c, const char* who, const void* words, size_t word_pitch_bytes) {
    if (!words || word_pitch_bytes < 8 * (size_t)((c->n + 63) / 64)) {
        ltl_set_error("%s: bad buffer or word pitch %zu < %d", who, word_pitch_bytes, 8 * ((c->n + 63) / 64));
        return LTL_EINVAL;
    }
    return LTL_OK;
}

static int pack_stage(ltl_ctx* c) {
    if (c->pstage) return LTL_OK;
    const size_t bytes = (size_t)c->rows * 8 * ((c->n + 63) / 64);
    cudaError_t e = cudaMalloc(&c->pstage, std::max<size_t>(bytes, 8));
    if (e != cudaSuccess) {
        ltl_set_error("packed transfer staging allocation failed: %s", cudaGetErrorString(e));
        return LTL_ENOMEM;
    }
    return LTL_OK;
}

extern "C" int ltl_upload_packed(ltl_ctx* c, const uint64_t* words, size_t word_pitch_bytes) {
    if (int r = check_ctx(c)) return r;
    if (int r = pack_args(c, "ltl_upload_packed", words, word_pitch_bytes)) return r;
    LTL_CUDA(cudaSetDevice(c->device));
    if (keeps_packed(c)) {
        // straight into the packed frame: a little-endian uint64 row is its 32-bit
        // word row; bits past n are rewritten by the halo pass (packed) or masked
        // by the step (tensor)
        PackedFrame& f = cur_packed(c);
        LTL_CUDA(cudaMemcpy2DAsync(f.words + (size_t)f.HR * f.wpitch + f.HW, f.wpitch * sizeof(uint32_t), words,
                                   word_pitch_bytes, (size_t)f.nw * sizeof(uint32_t), c->rows,
                                   cudaMemcpyHostToDevice, c->stream));
        if (c->variant == LTL_VARIANT_PACKED) LTL_CUDA(launch_packed_halo(f, c->stream));
        c->packed_valid = true;
    } else {
        if (int r = pack_stage(c)) return r;
        const size_t spitch = (size_t)(c->n + 63) / 64;  // words
        LTL_CUDA(cudaMemcpy2DAsync(c->pstage, spitch * 8, words, word_pitch_bytes, spitch * 8, c->rows,
                                   cudaMemcpyHostToDevice, c->stream));
        Frame& f = cur_frame(c);
        LTL_CUDA(launch_unpack(c->pstage, spitch, c->rows, c->n, f.inner(0, 0), f.pitch, c->stream));
        if (int r = after_upload(c)) return r;
    }
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    return LTL_OK;
}

extern "C" int ltl_download_packed(ltl_ctx* c, uint64_t* words, size_t word_pitch_bytes) {
    if (int r = check_ctx(c)) return r;
    if (int r = pack_args(c, "ltl_download_packed", words, word_pitch_bytes)) return r;
    LTL_CUDA(cudaSetDevice(c->device));
    if (int r = pack_stage(c)) return r;
    const size_t spitch = (size_t)(c->n + 63) / 64;  // words
    if (keeps_packed(c) && c->packed_valid) {
        LTL_CUDA(launch_frame_to_pack64(cur_packed(c), c->pstage, spitch, c->stream));
    } else {
        Frame& f = cur_frame(c);
        LTL_CUDA(launch_pack(f.inner(0, 0), f.pitch, c->rows, c->n, c->pstage, spitch, c->stream));
    }
    LTL_CUDA(cudaMemcpy2DAsync(words, word_pitch_bytes, c->pstage, spitch * 8, spitch * 8, c->rows,
                               cudaMemcpyDeviceToHost, c->stream));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    return LTL_OK;
}

extern "C" int ltl_download_device(ltl_ctx* c, uint8_t* dev_inner, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (!dev_inner || pitch < (size_t)c->n) {
        ltl_set_error("ltl_download_device: bad buffer or pitch");
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    if (int r = sync_from_packed(c)) return r;
    LTL_CUDA(launch_copy_out(cur_frame(c), dev_inner, pitch, c->stream));
    return LTL_OK;
}

// Row-range transfers (device buffers): rows [row0, row0 + nrows) of the
// current grid, `pitch` bytes apart in the caller's buffer.
static int check_rows(ltl_ctx* c, const char* who, int row0, int nrows, const void* dev, size_t pitch) {
    if (!dev || nrows < 0 || row0 < 0 || row0 + nrows > c->rows || pitch < (size_t)c->n) {
        ltl_set_error("%s: bad rows [%d, %d) of %d, buffer or pitch", who, row0, row0 + nrows, c->rows);
        return LTL_EINVAL;
    }
    return LTL_OK;
}

extern "C" int ltl_download_rows_device(ltl_ctx* c, int row0, int nrows, uint8_t* dev, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (int r = check_rows(c, "ltl_download_rows_device", row0, nrows, dev, pitch)) return r;
    if (nrows == 0) return LTL_OK;
    LTL_CUDA(cudaSetDevice(c->device));
    if (keeps_packed(c) && c->packed_valid) {
        // straight from the packed frame: only the asked rows are unpacked
        LTL_CUDA(launch_unpack_rows(cur_packed(c), row0, nrows, dev, pitch, c->stream));
        return LTL_OK;
    }
    Frame& f = cur_frame(c);
    LTL_CUDA(cudaMemcpy2DAsync(dev, pitch, f.inner(row0, 0), f.pitch, c->n, nrows, cudaMemcpyDeviceToDevice,
                               c->stream));
    return LTL_OK;
}

extern "C" int ltl_upload_rows_device(ltl_ctx* c, int row0, int nrows, const uint8_t* dev, size_t pitch) {
    if (int r = check_ctx(c)) return r;
    if (int r = check_rows(c, "ltl_upload_rows_device", row0, nrows, dev, pitch)) return r;
    if (nrows == 0) return LTL_OK;
    LTL_CUDA(cudaSetDevice(c->device));
    if (keeps_packed(c)) {
        // straight into the packed frame once it holds the current state (the
        // byte frame is staging only: every read of a packed grid unpacks it
        // again), then its halo
        if (!c->packed_valid) {
            if (int r = sync_to_packed(c)) return r;
        }
        LTL_CUDA(launch_pack_rows(dev, pitch, cur_packed(c), row0, nrows, c->stream));
        if (c->variant == LTL_VARIANT_PACKED) LTL_CUDA(launch_packed_halo(cur_packed(c), c->stream));
        return LTL_OK;
    }
    Frame& f = cur_frame(c);
    LTL_CUDA(cudaMemcpy2DAsync(f.inner(row0, 0), f.pitch, dev, pitch, c->n, nrows, cudaMemcpyDeviceToDevice,
                               c->stream));
    return after_upload(c);
}

// One pass = `gens` generations (c->depth, or fewer for the remainder of a
// step count; only the temporally blocked plain kernel takes more than 1).
// Leaves the result in nxt and swaps.
static cudaError_t enqueue_pass(ltl_ctx* c, int gens) {
    cudaError_t e = cudaSuccess;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (c->timing) {
        e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        if (e == cudaSuccess) e = cudaEventRecord(e0, c->stream);
        if (e != cudaSuccess) return e;
    }
    int step_kernels = 0, halo_kernels = 2;
    switch (c->variant) {
        case LTL_VARIANT_PLAIN: {
            Frame& a = cur_frame(c);
            Frame& b = nxt_frame(c);
            if (gens > 1) {
                e = launch_plain_tb(a, b, c->rule, c->band_rows, gens, c->plain_wrap, c->stream);
                step_kernels = 1;
            } else if (plain_swar8_supported(c->rule.radius)) {
                e = launch_plain_swar8(a, b, c->rule, c->band_rows, c->plain_wrap, c->stream);
                step_kernels = 1;
            } else {
                e = launch_plain_generic(a, b, c->rule, c->band_rows, c->stream);
                step_kernels = 1;
            }
            if (c->timing && e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
            // the SWAR kernels with plain_wrap read inner cells only: no halo to refresh
            const bool wrapped = c->plain_wrap && plain_swar8_supported(c->rule.radius);
            if (wrapped) halo_kernels = 0;
            else if (e == cudaSuccess) e = launch_halo_fill(b, c->stream);
            break;
        }
        case LTL_VARIANT_PACKED: {
            e = launch_packed_step(cur_packed(c), nxt_packed(c), c->rule, c->packed_band_rows, c->stream);
            step_kernels = 1;
            if (c->timing && e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
            if (packed_fused_halo(nxt_packed(c), c->rule.radius)) halo_kernels = 0;
            else if (e == cudaSuccess) e = launch_packed_halo(nxt_packed(c), c->stream);
            break;
        }
        case LTL_VARIANT_TENSOR: {
            // packed frames, torus wrap inside the kernel: no halo pass
            e = launch_tensor_pass(c->tplan, c->cur_is_a, c->stream);
            step_kernels = 1;
            halo_kernels = 0;
            if (c->timing && e == cudaSuccess) e = cudaEventRecord(e1, c->stream);
            break;
        }
    }
    if (c->timing) {
        c->ev.emplace_back(e0, e1);
        c->step_launches += step_kernels;
        c->all_launches += step_kernels + halo_kernels;
    }
    c->cur_is_a = !c->cur_is_a;
    return e;
}

static int build_graph(ltl_ctx* c, int which) {
    bool saved = c->cur_is_a;
    c->cur_is_a = (which == 0);
    cudaGraph_t g = nullptr;
    LTL_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = cudaSuccess;
    for (int p = 0; p < kGraphPasses && e == cudaSuccess; ++p) e = enqueue_pass(c, c->depth);
    cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
    c->cur_is_a = saved;
    if (e != cudaSuccess || e2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        ltl_set_error("graph capture failed: %s", cudaGetErrorString(e != cudaSuccess ? e : e2));
        return LTL_ECUDA;
    }
    cudaError_t e3 = cudaGraphInstantiate(&c->graph[which], g, 0);
    cudaGraphDestroy(g);
    if (e3 != cudaSuccess) {
        c->graph[which] = nullptr;
        ltl_set_error("graph instantiate failed: %s", cudaGetErrorString(e3));
        return LTL_ECUDA;
    }
    return LTL_OK;
}

extern "C" int ltl_step(ltl_ctx* c, int steps) {
    if (int r = check_ctx(c)) return r;
    if (steps < 0) {
        ltl_set_error("ltl_step: negative step count %d", steps);
        return LTL_EINVAL;
    }
    if (steps == 0) return LTL_OK;
    LTL_CUDA(cudaSetDevice(c->device));
    if (keeps_packed(c) && !c->packed_valid) {
        if (int r = sync_to_packed(c)) return r;
    }
    int passes = steps / c->depth;
    const int rest = steps % c->depth;  // a last, shorter pass
    while (!c->timing && passes >= kGraphPasses) {
        int which = c->cur_is_a ? 0 : 1;
        if (!c->graph[which]) {
            if (int r = build_graph(c, which)) return r;
        }
        LTL_CUDA(cudaGraphLaunch(c->graph[which], c->stream));
        // kGraphPasses is even: the parity of the current buffer is unchanged
        passes -= kGraphPasses;
    }
    for (int p = 0; p < passes; ++p) LTL_CUDA(enqueue_pass(c, c->depth));
    if (rest > 0) LTL_CUDA(enqueue_pass(c, rest));
    return LTL_OK;
}

extern "C" int ltl_synchronize(ltl_ctx* c) {
    if (int r = check_ctx(c)) return r;
    LTL_CUDA(cudaSetDevice(c->device));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    if (c->tplan) {
        unsigned int flag = 0;
        LTL_CUDA(cudaMemcpy(&flag, tensor_plan_error_flag(c->tplan), sizeof(flag), cudaMemcpyDeviceToHost));
        if (flag) {
            // clear it, so that the context stays usable after the caller re-uploads a state
            const unsigned int zero = 0;
            cudaMemcpy(tensor_plan_error_flag(c->tplan), &zero, sizeof(zero), cudaMemcpyHostToDevice);
            ltl_set_error("tensor kernel reported a bounded-wait timeout (flag 0x%x); the grid state is "
                          "unspecified until the next upload",
                          flag);
            return LTL_ETIMEOUT;
        }
    }
    return LTL_OK;
}

extern "C" int ltl_population(ltl_ctx* c, uint64_t* live) {
    if (int r = check_ctx(c)) return r;
    if (!live) {
        ltl_set_error("ltl_population: live is NULL");
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    if (int r = sync_from_packed(c)) return r;
    LTL_CUDA(launch_population(cur_frame(c), c->scratch, c->stream));
    unsigned long long v = 0;
    LTL_CUDA(cudaMemcpyAsync(&v, c->scratch, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    *live = v;
    return LTL_OK;
}

extern "C" int ltl_compare_device(ltl_ctx* c, const uint8_t* dev_expected, size_t pitch, uint64_t* mismatches,
                                  int64_t* first_index) {
    if (int r = check_ctx(c)) return r;
    if (!dev_expected || pitch < (size_t)c->n || !mismatches) {
        ltl_set_error("ltl_compare_device: bad arguments");
        return LTL_EINVAL;
    }
    LTL_CUDA(cudaSetDevice(c->device));
    if (int r = sync_from_packed(c)) return r;
    LTL_CUDA(launch_compare(cur_frame(c), dev_expected, pitch, c->scratch, c->stream));
    unsigned long long v[2] = {0, 0};
    LTL_CUDA(cudaMemcpyAsync(v, c->scratch, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    *mismatches = v[0];
    if (first_index) *first_index = v[0] ? (int64_t)v[1] : -1;
    return LTL_OK;
}

extern "C" int ltl_pack_device(const uint8_t* dev_cells, size_t cell_pitch, int rows, int cols,
                               uint64_t* dev_words, size_t word_pitch_bytes, void* stream) {
    if (!dev_cells || !dev_words || rows < 0 || cols < 0 || cell_pitch < (size_t)cols ||
        word_pitch_bytes % 8 != 0 || word_pitch_bytes < (size_t)((cols + 63) / 64) * 8) {
        ltl_set_error("ltl_pack_device: bad arguments");
        return LTL_EINVAL;
    }
    LTL_CUDA(launch_pack(dev_cells, cell_pitch, rows, cols, dev_words, word_pitch_bytes / 8, (cudaStream_t)stream));
    return LTL_OK;
}

extern "C" int ltl_unpack_device(const uint64_t* dev_words, size_t word_pitch_bytes, int rows, int cols,
                                 uint8_t* dev_cells, size_t cell_pitch, void* stream) {
    if (!dev_cells || !dev_words || rows < 0 || cols < 0 || cell_pitch < (size_t)cols ||
        word_pitch_bytes % 8 != 0 || word_pitch_bytes < (size_t)((cols + 63) / 64) * 8) {
        ltl_set_error("ltl_unpack_device: bad arguments");
        return LTL_EINVAL;
    }
    LTL_CUDA(launch_unpack(dev_words, word_pitch_bytes / 8, rows, cols, dev_cells, cell_pitch,
                           (cudaStream_t)stream));
    return LTL_OK;
}

extern "C" int ltl_set_param(ltl_ctx* c, const char* name, long long value) {
    if (int r = check_ctx(c)) return r;
    if (!name) {
        ltl_set_error("ltl_set_param: name is NULL");
        return LTL_EINVAL;
    }
    if (std::strcmp(name, "band_rows") == 0) {
        if (value != 0 && (value < 16 || value > 4096)) {
            ltl_set_error("ltl_set_param: band_rows must be 0 (built-in choice) or in [16, 4096]");
            return LTL_EINVAL;
        }
        if (c->variant == LTL_VARIANT_PLAIN && plain_swar8_supported(c->rule.radius))
            c->band_rows = value ? (int)value : plain_swar8_band_rows(c->n, c->device);
        else if (c->variant == LTL_VARIANT_PLAIN) c->band_rows = (int)value;
        else if (c->variant == LTL_VARIANT_PACKED) c->packed_band_rows = (int)value;
        else {
            ltl_set_error("ltl_set_param: band_rows applies to the plain and packed variants");
            return LTL_EUNSUPPORTED;
        }
        drop_graphs(c);
        return LTL_OK;
    }
    if (std::strcmp(name, "depth") == 0) {
        if (c->variant != LTL_VARIANT_PLAIN) {
            ltl_set_error("ltl_set_param: depth applies to the plain variant");
            return LTL_EUNSUPPORTED;
        }
        if (value != 1 && !(plain_tb_supported(c->rule.radius, (int)value) && c->fa.H >= value * c->rule.radius)) {
            ltl_set_error("ltl_set_param: depth %lld is not supported for R=%d (1, or 2..3 with depth*R <= 16 and R <= 5)",
                          value, c->rule.radius);
            return LTL_EINVAL;
        }
        c->depth = (int)value;
        drop_graphs(c);
        return LTL_OK;
    }
    if (std::strcmp(name, "wait_limit_ns") == 0 || std::strcmp(name, "inject_missing_commit") == 0) {
        if (c->variant != LTL_VARIANT_TENSOR) {
            ltl_set_error("ltl_set_param: %s applies to the tensor variant", name);
            return LTL_EUNSUPPORTED;
        }
        if (std::strcmp(name, "wait_limit_ns") == 0) {
            if (value < 1000000 || value > 10000000000ll) {
                ltl_set_error("ltl_set_param: wait_limit_ns must be in [1e6, 1e10]");
                return LTL_EINVAL;
            }
            c->wait_ns = (unsigned long long)value;
        } else {
            c->inject = value != 0;
        }
        tensor_plan_set_wait(c->tplan, c->wait_ns, c->inject ? 1 : 0);
        drop_graphs(c);
        return LTL_OK;
    }
    ltl_set_error("ltl_set_param: unknown parameter '%s'", name);
    return LTL_EINVAL;
}

extern "C" int ltl_set_timing(ltl_ctx* c, int enable) {
    if (int r = check_ctx(c)) return r;
    LTL_CUDA(cudaSetDevice(c->device));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    free_events(c);
    c->timing = enable != 0;
    c->step_launches = 0;
    c->all_launches = 0;
    return LTL_OK;
}

extern "C" int ltl_get_timing(ltl_ctx* c, double* step_kernel_ms, long long* step_kernel_launches,
                              long long* all_launches) {
    if (int r = check_ctx(c)) return r;
    LTL_CUDA(cudaSetDevice(c->device));
    LTL_CUDA(cudaStreamSynchronize(c->stream));
    double total = 0.0;
    for (auto& p : c->ev) {
        float ms = 0.f;
        LTL_CUDA(cudaEventElapsedTime(&ms, p.first, p.second));
        total += ms;
    }
    if (step_kernel_ms) *step_kernel_ms = total;
    if (step_kernel_launches) *step_kernel_launches = c->step_launches;
    if (all_launches) *all_launches = c->all_launches;
    return LTL_OK;
}

extern "C" const char* ltl_last_error(void) { return g_err; }

extern "C" const char* ltl_version(void) { return "libltl_b200 0.1 (sm_100a)"; }

// api.cu - the zap_tex_cuda C ABI (include/zap_tex_cuda.h): contexts, argument checks, host staging, dispatch.
//
// Host-pointer calls are synchronous like the reference functions they replace. Large images are cut into bands
// of block rows and pipelined over two streams, so the host->device copy of one band overlaps the kernels and
// the device->host copy of the previous one. Device-pointer (_dev) calls enqueue on the caller's stream and take
// their scratch from the stream-ordered allocator, so concurrent calls on different streams do not share it.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>

#include "../../include/zap_tex_cuda.h"
#include "ztc_common.cuh"
#include "ztc_internal.h"

#include <atomic>
#include <map>
#include <string>
#include <vector>

namespace ztc {
cudaError_t upload_mip_tables();
cudaError_t upload_astc_tables();

// ---------------------------------------------------------------- kernel tracing (events around each launch)
namespace {
struct TraceRec {
    const char *name;
    cudaEvent_t a, b;
    long units;                // blocks (or texels) the launch processed, when known on the host
    uint32_t *counter;         // pinned slot receiving a device-side count, or null
    const uint32_t *d_count;   // that count on the device, copied after the end event (outside the interval)
};
std::mutex g_trace_lock;
bool g_trace_on = false;
std::vector<TraceRec> g_trace;
thread_local std::vector<TraceRec> t_open;
uint32_t *g_slots = nullptr;  // pinned host slots for device-side unit counts
int g_slot_next = 0;
constexpr int kSlots = 1 << 16;
}  // namespace

void trace_begin(const char *name, cudaStream_t s) {
    if (!g_trace_on) return;
    TraceRec r{name, nullptr, nullptr, 0, nullptr, nullptr};
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) {  // nothing to time while capturing
        cudaGetLastError();
        t_open.push_back(r);
        return;
    }
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, s);
    t_open.push_back(r);
}
void trace_units(long n) {
    if (g_trace_on && !t_open.empty()) t_open.back().units = n;
}
void trace_units_dev(const uint32_t *d_count, cudaStream_t s) {  // the launch does not change the count it reads
    (void)s;
    if (g_trace_on && !t_open.empty() && t_open.back().a) t_open.back().d_count = d_count;
}
void trace_end(cudaStream_t s) {
    if (!g_trace_on || t_open.empty()) return;
    TraceRec r = t_open.back();
    t_open.pop_back();
    if (!r.a) return;  // began during a capture
    cudaEventRecord(r.b, s);
    std::lock_guard<std::mutex> g(g_trace_lock);
    if (r.d_count) {
        if (!g_slots && ztc_malloc_host((void **)&g_slots, kSlots * sizeof(uint32_t)) != cudaSuccess) g_slots = nullptr;
        if (g_slots && g_slot_next < kSlots) {
            uint32_t *slot = g_slots + g_slot_next++;
            *slot = 0;
            if (cudaMemcpyAsync(slot, r.d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s) == cudaSuccess) r.counter = slot;
        }
    }
    g_trace.push_back(r);
}
}  // namespace ztc

// Host-pointer pipeline: stream[0] copies bands in, stream[1] and stream[2] encode alternate bands, stream[3] copies
// blocks out; kOutLag bands behind the copies in, so a copy out (synchronous for pageable host memory) never holds
// up the issue of the next copy in.
constexpr int kStreams = 4, kOutLag = 2;

struct zap_tex_cuda_ctx {
    int device = 0;
    int sms = 148;
    cudaStream_t stream[kStreams] = {};
    cudaEvent_t ev_in = nullptr, ev_enc[kOutLag + 1] = {};  // band copied in; band encoded (ring)
    // host-call staging, grown on demand
    uint8_t *d_in = nullptr;
    size_t d_in_cap = 0;
    uint8_t *d_out = nullptr;
    size_t d_out_cap = 0;
    void *d_scratch[2] = {nullptr, nullptr};
    size_t d_scratch_cap[2] = {0, 0};
    bool owned_default = false;
};

namespace {

thread_local char g_err[512];

int fail(int status, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return status;
}
int cuda_fail(cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a sticky launch error so the context stays usable
    return fail(e == cudaErrorMemoryAllocation ? ZTC_ERR_NO_MEMORY : ZTC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
#define ZTC_CHECK(expr, what)                          \
    do {                                               \
        cudaError_t e_ = (expr);                       \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

std::mutex g_lock;
constexpr int kMaxDevices = 64;
bool g_tables_ready[kMaxDevices];
zap_tex_cuda_ctx *g_default[kMaxDevices];

int device_ok(int device) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) { cudaGetLastError(); return fail(ZTC_ERR_NO_DEVICE, "no CUDA device"); }
    if (device < 0 || device >= n || device >= kMaxDevices) return fail(ZTC_ERR_INVALID_ARG, "device %d out of range (%d devices)", device, n);
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (major != 10) return fail(ZTC_ERR_NO_DEVICE, "device %d is compute capability %d.x; this build targets sm_100a", device, major);
    return ZTC_OK;
}

int ensure_tables(int device) {  // caller holds g_lock, device is current
    if (g_tables_ready[device]) return ZTC_OK;
    ZTC_CHECK(ztc::upload_mip_tables(), "upload sRGB tables");
    ZTC_CHECK(ztc::upload_astc_tables(), "upload ASTC tables");
    g_tables_ready[device] = true;
    return ZTC_OK;
}

int create_ctx(int device, zap_tex_cuda_ctx **out) {
    int st = device_ok(device);
    if (st) return st;
    ZTC_CHECK(cudaSetDevice(device), "cudaSetDevice");
    {
        std::lock_guard<std::mutex> g(g_lock);
        st = ensure_tables(device);
        if (st) return st;
    }
    zap_tex_cuda_ctx *c = new (std::nothrow) zap_tex_cuda_ctx();
    if (!c) return fail(ZTC_ERR_NO_MEMORY, "context allocation");
    c->device = device;
    cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, device);
    for (int k = 0; k < kStreams; k++)
        if (cudaStreamCreateWithFlags(&c->stream[k], cudaStreamNonBlocking) != cudaSuccess) {
            zap_tex_cuda_destroy(c);
            return cuda_fail(cudaErrorUnknown, "stream creation");
        }
    for (int k = 0; k <= kOutLag + 1; k++)
        if (cudaEventCreateWithFlags(k ? &c->ev_enc[k - 1] : &c->ev_in, cudaEventDisableTiming) != cudaSuccess) {
            zap_tex_cuda_destroy(c);
            return cuda_fail(cudaErrorUnknown, "event creation");
        }
    *out = c;
    return ZTC_OK;
}

// ctx == NULL: the default context of the current device
int resolve(zap_tex_cuda_ctx *&ctx) {
    if (ctx) {
        ZTC_CHECK(cudaSetDevice(ctx->device), "cudaSetDevice");
        return ZTC_OK;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return fail(ZTC_ERR_NO_DEVICE, "no CUDA device"); }
    if (dev < 0 || dev >= kMaxDevices) return fail(ZTC_ERR_INVALID_ARG, "device %d", dev);
    {
        std::lock_guard<std::mutex> g(g_lock);
        if (g_default[dev]) { ctx = g_default[dev]; return ZTC_OK; }
    }
    zap_tex_cuda_ctx *c = nullptr;
    int st = create_ctx(dev, &c);
    if (st) return st;
    std::lock_guard<std::mutex> g(g_lock);
    if (g_default[dev]) { zap_tex_cuda_destroy(c); ctx = g_default[dev]; return ZTC_OK; }
    c->owned_default = true;
    g_default[dev] = c;
    ctx = c;
    return ZTC_OK;
}

int grow(void **p, size_t *cap, size_t need, const char *what) {
    if (*cap >= need) return ZTC_OK;
    if (*p) { cudaFree(*p); *p = nullptr; *cap = 0; }
    size_t n = need + need / 4 + 4096;
    ZTC_CHECK(ztc_malloc(p, n), what);
    *cap = n;
    return ZTC_OK;
}

bool valid_fmt_bc(int fmt) { return fmt >= ZTC_BC1 && fmt <= ZTC_BC7; }
// device pointers the kernels access with vector or word loads / stores must be aligned: blocks to their size,
// floats to 4 bytes, halfs to 2 (a misaligned vector access would be a device fault, so it is an argument error)
bool misaligned(const void *p, size_t a) { return ((uintptr_t)p) % a != 0; }
size_t block_bytes(int fmt) { return (fmt == ZTC_BC1 || fmt == ZTC_BC4) ? 8 : 16; }
size_t round16(size_t v) { return (v + 15) & ~(size_t)15; }

// one encoder launch over block rows [by0, by0 + nby) of a device image
int launch_encode(int fmt, const ztc::SrcU8 &src, const ztc::SrcHdr *hdr, int by0, int nby, uint8_t *out, void *scratch,
                  cudaStream_t s) {
    cudaError_t e;
    if (fmt == ZTC_BC7) e = ztc_launch_bc7(src, by0, nby, out, scratch, s);
    else if (fmt == ZTC_BC6H) e = ztc_launch_bc6h(*hdr, by0, nby, out, s);
    else if (fmt == ZTC_ASTC4X4) e = ztc_launch_astc(src, by0, nby, out, scratch, s);
    else e = ztc_launch_bcn(fmt, src, by0, nby, out, s);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return ZTC_OK;
}

size_t scratch_for(int fmt, size_t nblocks) {
    if (fmt == ZTC_BC7) return ztc::bc7_scratch_bytes(nblocks);
    if (fmt == ZTC_ASTC4X4) return ztc::astc_scratch_bytes(nblocks);
    return 0;
}

// Source bytes per band of the host-pointer pipeline: larger bands copy closer to the link's peak, smaller ones
// overlap more of the encode and the copy back with the copy in. Measured on a 2048x2048 BC7 call from pinned memory:
// 1 MB 0.51 ms, 2 MB 0.44 ms, 4 MB 0.46 ms (the 16.8 MB copy in alone takes 0.30-0.42 ms over PCIe).
#ifndef ZTC_HOST_BAND_BYTES
#define ZTC_HOST_BAND_BYTES (2u << 20)
#endif

// Host-pointer encode: stage rows to the device band by band, encode, copy blocks back.
// texel_bytes: 4 (RGBA8) or 16 (RGBA f32); src_stride in bytes.
int host_encode(zap_tex_cuda_ctx *ctx, int fmt, const void *src, int w, int h, size_t src_stride, size_t texel_bytes, void *out) {
    const int bw = (w + 3) / 4, bh = (h + 3) / 4;
    const size_t bs = fmt == ZTC_BC6H || fmt == ZTC_ASTC4X4 ? 16 : block_bytes(fmt);
    const size_t row_bytes = (size_t)w * texel_bytes, pitch = round16(row_bytes);
    // band height: about ZTC_HOST_BAND_BYTES of source per band, at least 8 block rows
    size_t band_rows = (size_t)ZTC_HOST_BAND_BYTES / (pitch * 4) + 1;
    if (band_rows < 8) band_rows = 8;
    if (band_rows > (size_t)bh) band_rows = (size_t)bh;
    const int nbands = (int)((bh + band_rows - 1) / band_rows);
    int st = grow((void **)&ctx->d_in, &ctx->d_in_cap, pitch * (size_t)h, "cudaMalloc(input)");
    if (!st) st = grow((void **)&ctx->d_out, &ctx->d_out_cap, (size_t)bw * bh * bs, "cudaMalloc(output)");
    const size_t scr = scratch_for(fmt, (size_t)band_rows * bw);
    for (int k = 0; k < 2 && !st && scr; k++) st = grow(&ctx->d_scratch[k], &ctx->d_scratch_cap[k], scr, "cudaMalloc(scratch)");
    if (st) return st;
    ztc::SrcU8 s8{ctx->d_in, pitch, w, h, 4, ((uintptr_t)ctx->d_in & 15u) == 0 && (pitch & 15u) == 0};
    ztc::SrcHdr sh{ctx->d_in, pitch / 4, w, h, 4, 1};
    auto band = [&](int b, int &by0, int &nby) {
        by0 = b * (int)band_rows;
        nby = by0 + (int)band_rows <= bh ? (int)band_rows : bh - by0;
    };
    cudaStream_t in = ctx->stream[0], out_s = ctx->stream[3];
    for (int b = 0; b < nbands + kOutLag && !st; b++) {
        int by0, nby;
        if (b < nbands) {
            band(b, by0, nby);
            const int y0 = by0 * 4, y1 = (by0 + nby) * 4 < h ? (by0 + nby) * 4 : h;
            cudaStream_t es = ctx->stream[1 + (b & 1)];
            ZTC_CHECK(cudaMemcpy2DAsync(ctx->d_in + (size_t)y0 * pitch, pitch, (const uint8_t *)src + (size_t)y0 * src_stride, src_stride,
                                        row_bytes, (size_t)(y1 - y0), cudaMemcpyHostToDevice, in),
                      "host->device copy");
            ZTC_CHECK(cudaEventRecord(ctx->ev_in, in), "event record");
            ZTC_CHECK(cudaStreamWaitEvent(es, ctx->ev_in, 0), "stream wait");
            st = launch_encode(fmt, s8, &sh, by0, nby, ctx->d_out + (size_t)by0 * bw * bs, ctx->d_scratch[b & 1], es);
            if (st) break;
            ZTC_CHECK(cudaEventRecord(ctx->ev_enc[b % (kOutLag + 1)], es), "event record");
        }
        const int ob = b - kOutLag;  // the band whose blocks go back now
        if (ob >= 0 && ob < nbands) {
            band(ob, by0, nby);
            ZTC_CHECK(cudaStreamWaitEvent(out_s, ctx->ev_enc[ob % (kOutLag + 1)], 0), "stream wait");
            ZTC_CHECK(cudaMemcpyAsync((uint8_t *)out + (size_t)by0 * bw * bs, ctx->d_out + (size_t)by0 * bw * bs, (size_t)nby * bw * bs,
                                      cudaMemcpyDeviceToHost, out_s),
                      "device->host copy");
        }
    }
    for (int k = 0; k < kStreams; k++) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream[k]);
        if (e != cudaSuccess && !st) st = cuda_fail(e, "encode");
    }
    return st;
}

// Blocks per encode launch at most (whole block rows): the kernels index a launch's blocks with 32-bit ints, and a
// texture a B200 can hold may have more than 2^31 blocks (2^31 blocks of RGBA8 are 128 GB of texels). The
// bounds-check build uses a small limit, so its tests run the chunked path on small images.
#ifndef ZTC_LAUNCH_BLOCKS
#ifdef ZTC_CHECKS
#define ZTC_LAUNCH_BLOCKS 4096
#else
#define ZTC_LAUNCH_BLOCKS (1 << 30)
#endif
#endif

int dev_encode(zap_tex_cuda_ctx *ctx, int fmt, const ztc::SrcU8 &s8, const ztc::SrcHdr *sh, int w, int h, void *out, cudaStream_t s) {
    const int bh = (h + 3) / 4, bw = (w + 3) / 4;
    const int rows = (int)std::min<size_t>((size_t)bh, std::max<size_t>(1, (size_t)ZTC_LAUNCH_BLOCKS / (size_t)bw));  // per launch
    const size_t bs = fmt == ZTC_BC6H || fmt == ZTC_ASTC4X4 ? 16 : block_bytes(fmt);
    const size_t scr = scratch_for(fmt, (size_t)bw * rows);
    void *scratch = nullptr;
    if (scr) ZTC_CHECK(ztc_malloc_async(&scratch, scr, s), "cudaMallocAsync(scratch)");
    int st = ZTC_OK;
    for (int y = 0; y < bh && !st; y += rows)  // launches on one stream, so they share the scratch in turn
        st = launch_encode(fmt, s8, sh, y, rows < bh - y ? rows : bh - y, (uint8_t *)out + (size_t)y * bw * bs, scratch, s);
    if (scratch) cudaFreeAsync(scratch, s);
    (void)ctx;
    return st;
}

// rate-distortion mode (zap_tex.h:223-306, :786-815): the base encodings of every block, then the RDO chain(s)
// over them in place; band_rows block rows per chain (0: one chain, as one reference call)
int rdo_encode(zap_tex_cuda_ctx *ctx, int fmt, const ztc::SrcU8 &s8, int w, int h, float lambda, int band_rows, void *out, cudaStream_t s) {
    int st = dev_encode(ctx, fmt, s8, nullptr, w, h, out, s);
    if (st) return st;
    ZTC_CHECK(ztc_launch_rdo(fmt, s8, (uint8_t *)out, lambda, band_rows, s), "rdo launch");
    return ZTC_OK;
}

// lambda as the reference reads it: <= 0 is the plain encode; a finite positive value selects RDO; NaN and
// infinities are rejected (the chain's choice rule relies on finite, non-negative costs)
int check_lambda(float rdo) {
    if (!(rdo == rdo) || rdo > 3.0e38f || rdo < -3.0e38f) return fail(ZTC_ERR_INVALID_ARG, "rdo must be a finite number");
    return ZTC_OK;
}

int check_image(const void *p, const void *out, int w, int h, size_t stride, size_t min_stride) {
    if (!p || !out) return fail(ZTC_ERR_INVALID_ARG, "null pointer");
    if (w < 1 || h < 1) return fail(ZTC_ERR_INVALID_ARG, "size %dx%d", w, h);
    if (w > (1 << 24) || h > (1 << 24)) return fail(ZTC_ERR_INVALID_ARG, "size %dx%d beyond 2^24", w, h);
    if (stride < min_stride) return fail(ZTC_ERR_INVALID_ARG, "stride %zu below %zu", stride, min_stride);
    return ZTC_OK;
}

}  // namespace

int ztc_set_error(int status, const char *msg) { return fail(status, "%s", msg); }

// ---------------------------------------------------------------- allocations (and the test hook that fails them)
namespace {
std::mutex g_alloc_lock;
long g_alloc_skip = 0, g_alloc_fail = 0;  // let g_alloc_skip allocations through, then fail g_alloc_fail
bool alloc_fault() {
    std::lock_guard<std::mutex> g(g_alloc_lock);
    if (g_alloc_skip > 0) { g_alloc_skip--; return false; }
    if (g_alloc_fail > 0) { g_alloc_fail--; return true; }
    return false;
}
}  // namespace
cudaError_t ztc_malloc(void **p, size_t n) {
    if (alloc_fault()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMalloc(p, n);
}
cudaError_t ztc_malloc_async(void **p, size_t n, cudaStream_t s) {
    if (alloc_fault()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMallocAsync(p, n, s);
}
cudaError_t ztc_malloc_host(void **p, size_t n) {
    if (alloc_fault()) { *p = nullptr; return cudaErrorMemoryAllocation; }
    return cudaMallocHost(p, n);
}

#ifdef ZTC_CHECKS
__device__ unsigned int ztc_check_word = 0u;  // the first failed bounds check of the ZTC_CHECKS build
#endif
int ztc_sm_count() {  // SMs of the current device, cached per device (148 on B200; a tuning input only)
    static std::atomic<int> cache[kMaxDevices];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) { cudaGetLastError(); return 148; }
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n <= 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) { cudaGetLastError(); n = 148; }
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}
int ztc_ctx_activate(zap_tex_cuda_ctx *ctx) { return resolve(ctx); }

extern "C" {

int zap_tex_cuda_version(void) { return ZAP_TEX_CUDA_VERSION; }

int zap_tex_cuda_debug_fail_allocations(int skip, int count) {
    if (skip < 0 || count < 0) return fail(ZTC_ERR_INVALID_ARG, "skip and count must be >= 0");
    std::lock_guard<std::mutex> g(g_alloc_lock);
    g_alloc_skip = skip;
    g_alloc_fail = count;
    return ZTC_OK;
}

int zap_tex_cuda_debug_checks(unsigned int *first_failure) {
    if (!first_failure) return fail(ZTC_ERR_INVALID_ARG, "null first_failure");
    *first_failure = 0u;
#ifdef ZTC_CHECKS
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return fail(ZTC_ERR_NO_DEVICE, "no CUDA device"); }
    ZTC_CHECK(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    ZTC_CHECK(cudaMemcpyFromSymbol(first_failure, ztc_check_word, sizeof(unsigned int)), "read the check word");
    const unsigned int zero = 0u;
    ZTC_CHECK(cudaMemcpyToSymbol(ztc_check_word, &zero, sizeof zero), "clear the check word");
    return ZTC_OK;
#else
    return fail(ZTC_ERR_UNSUPPORTED, "this library was built without ZTC_CHECKS (make -C zap_b200/csrc checks)");
#endif
}

const char *zap_tex_cuda_status_string(int status) {
    switch (status) {
    case ZTC_OK: return "ok";
    case ZTC_ERR_INVALID_ARG: return "invalid argument";
    case ZTC_ERR_UNSUPPORTED: return "unsupported";
    case ZTC_ERR_CUDA: return "CUDA error";
    case ZTC_ERR_NO_MEMORY: return "out of memory";
    case ZTC_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown status";
    }
}

const char *zap_tex_cuda_last_error(void) { return g_err; }

int zap_tex_cuda_trace_enable(int enable) {
    std::lock_guard<std::mutex> g(ztc::g_trace_lock);
    for (auto &r : ztc::g_trace) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    ztc::g_trace.clear();
    ztc::g_slot_next = 0;
    ztc::g_trace_on = enable != 0;
    return ZTC_OK;
}

int zap_tex_cuda_trace_report(char *buf, size_t cap) {
    std::lock_guard<std::mutex> g(ztc::g_trace_lock);
    struct Agg { long n = 0; double ms = 0; long units = 0; };
    std::map<std::string, Agg> agg;
    for (auto &r : ztc::g_trace) {
        float ms = 0.0f;
        if (cudaEventSynchronize(r.b) == cudaSuccess && cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            auto &e = agg[r.name];
            e.n += 1;
            e.ms += ms;
            e.units += r.counter ? (long)*r.counter : r.units;
        }
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    cudaGetLastError();
    ztc::g_trace.clear();
    ztc::g_slot_next = 0;
    std::string out;
    char line[200];
    for (auto &kv : agg) {
        std::snprintf(line, sizeof line, "%s %ld %.6f %ld\n", kv.first.c_str(), kv.second.n, kv.second.ms, kv.second.units);
        out += line;
    }
    if (buf && cap) {
        std::strncpy(buf, out.c_str(), cap - 1);
        buf[cap - 1] = 0;
    }
    return (int)out.size();
}

int zap_tex_cuda_create(int device, zap_tex_cuda_ctx **out) {
    ZTC_NVTX();
    if (!out) return fail(ZTC_ERR_INVALID_ARG, "null out");
    *out = nullptr;
    return create_ctx(device, out);
}

int zap_tex_cuda_destroy(zap_tex_cuda_ctx *c) {
    ZTC_NVTX();
    if (!c) return ZTC_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(c->device);
    for (int k = 0; k < kStreams; k++) if (c->stream[k]) { cudaStreamSynchronize(c->stream[k]); cudaStreamDestroy(c->stream[k]); }
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    for (int k = 0; k <= kOutLag; k++) if (c->ev_enc[k]) cudaEventDestroy(c->ev_enc[k]);
    cudaFree(c->d_in); cudaFree(c->d_out); cudaFree(c->d_scratch[0]); cudaFree(c->d_scratch[1]);
    if (c->owned_default) {
        std::lock_guard<std::mutex> g(g_lock);
        if (g_default[c->device] == c) g_default[c->device] = nullptr;
    }
    delete c;
    cudaSetDevice(prev);
    return ZTC_OK;
}

int zap_tex_cuda_reserve(zap_tex_cuda_ctx *ctx, size_t bytes) {
    ZTC_NVTX();
    int st = resolve(ctx);
    if (st) return st;
    // _dev calls draw scratch from the device's default memory pool: keep that much resident across frees
    cudaMemPool_t pool;
    ZTC_CHECK(cudaDeviceGetDefaultMemPool(&pool, ctx->device), "cudaDeviceGetDefaultMemPool");
    uint64_t keep = bytes;
    ZTC_CHECK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "cudaMemPoolSetAttribute");
    void *p = nullptr;
    ZTC_CHECK(ztc_malloc_async(&p, bytes ? bytes : 1, ctx->stream[0]), "cudaMallocAsync(reserve)");
    ZTC_CHECK(cudaFreeAsync(p, ctx->stream[0]), "cudaFreeAsync(reserve)");
    ZTC_CHECK(cudaStreamSynchronize(ctx->stream[0]), "reserve");
    return ZTC_OK;
}

size_t zap_tex_cuda_block_bytes(int fmt) { return block_bytes(fmt); }
size_t zap_tex_cuda_bc_size(int w, int h, int fmt) {
    if (w < 1 || h < 1) return 0;
    return (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4) * (fmt == ZTC_BC6H || fmt == ZTC_ASTC4X4 ? 16 : block_bytes(fmt));
}
int zap_tex_cuda_mip_levels(int w, int h) {
    int n = 1;
    while (w > 1 || h > 1) { w = w > 1 ? w / 2 : 1; h = h > 1 ? h / 2 : 1; n++; }
    return n;
}

// ------------------------------------------------------------------ host memory
int zap_tex_cuda_bc_encode(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, void *out) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (!valid_fmt_bc(fmt)) return fail(ZTC_ERR_UNSUPPORTED, "format %d", fmt);
    if ((st = check_lambda(rdo))) return st;
    if ((st = resolve(ctx))) return st;
    if (rdo <= 0.0f) return host_encode(ctx, fmt, rgba, w, h, stride, 4, out);
    // RDO: one chain over the whole image, so the image is staged whole (no bands)
    const size_t row = (size_t)w * 4, pitch = round16(row), bytes = (size_t)((w + 3) / 4) * ((h + 3) / 4) * block_bytes(fmt);
    if ((st = grow((void **)&ctx->d_in, &ctx->d_in_cap, pitch * (size_t)h, "cudaMalloc(input)"))) return st;
    if ((st = grow((void **)&ctx->d_out, &ctx->d_out_cap, bytes, "cudaMalloc(output)"))) return st;
    cudaStream_t s = ctx->stream[0];
    ZTC_CHECK(cudaMemcpy2DAsync(ctx->d_in, pitch, rgba, stride, row, (size_t)h, cudaMemcpyHostToDevice, s), "host->device copy");
    const ztc::SrcU8 s8{ctx->d_in, pitch, w, h, 4, ((uintptr_t)ctx->d_in & 15u) == 0};
    if ((st = rdo_encode(ctx, fmt, s8, w, h, rdo, 0, ctx->d_out, s))) return st;
    ZTC_CHECK(cudaMemcpyAsync(out, ctx->d_out, bytes, cudaMemcpyDeviceToHost, s), "device->host copy");
    ZTC_CHECK(cudaStreamSynchronize(s), "encode");
    return ZTC_OK;
}

int zap_tex_cuda_bc6h_encode(zap_tex_cuda_ctx *ctx, const float *rgba, int w, int h, size_t stride, void *out) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if ((st = resolve(ctx))) return st;
    return host_encode(ctx, ZTC_BC6H, rgba, w, h, stride * 4, 16, out);
}

int zap_tex_cuda_astc_encode(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, void *out) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if ((st = resolve(ctx))) return st;
    return host_encode(ctx, ZTC_ASTC4X4, rgba, w, h, stride, 4, out);
}

static int host_mip(zap_tex_cuda_ctx *ctx, const void *src, int w, int h, size_t stride_b, int srgb, void *dst, size_t dst_stride_b,
                    size_t texel) {
    const int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    const size_t pitch = round16((size_t)w * texel), dpitch = round16((size_t)nw * texel);
    int st = grow((void **)&ctx->d_in, &ctx->d_in_cap, pitch * h, "cudaMalloc(input)");
    if (!st) st = grow((void **)&ctx->d_out, &ctx->d_out_cap, dpitch * nh, "cudaMalloc(output)");
    if (st) return st;
    cudaStream_t s = ctx->stream[0];
    ZTC_CHECK(cudaMemcpy2DAsync(ctx->d_in, pitch, src, stride_b, (size_t)w * texel, h, cudaMemcpyHostToDevice, s), "host->device copy");
    cudaError_t e = texel == 4 ? ztc_launch_mip(ctx->d_in, w, h, pitch, srgb, ctx->d_out, dpitch, s)
                               : ztc_launch_mip_f((const float *)ctx->d_in, w, h, pitch / 4, (float *)ctx->d_out, dpitch / 4, s);
    if (e != cudaSuccess) return cuda_fail(e, "mip launch");
    ZTC_CHECK(cudaMemcpy2DAsync(dst, dst_stride_b, ctx->d_out, dpitch, (size_t)nw * texel, nh, cudaMemcpyDeviceToHost, s), "device->host copy");
    ZTC_CHECK(cudaStreamSynchronize(s), "mip");
    return ZTC_OK;
}

int zap_tex_cuda_mip_next(zap_tex_cuda_ctx *ctx, const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride) {
    ZTC_NVTX();
    int st = check_image(src, dst, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (dst_stride < (size_t)(w > 1 ? w / 2 : 1) * 4) return fail(ZTC_ERR_INVALID_ARG, "dst_stride %zu too small", dst_stride);
    if ((st = resolve(ctx))) return st;
    return host_mip(ctx, src, w, h, stride, srgb, dst, dst_stride, 4);
}

int zap_tex_cuda_mip_next_f(zap_tex_cuda_ctx *ctx, const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride) {
    ZTC_NVTX();
    int st = check_image(src, dst, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (dst_stride < (size_t)(w > 1 ? w / 2 : 1) * 4) return fail(ZTC_ERR_INVALID_ARG, "dst_stride %zu too small", dst_stride);
    if ((st = resolve(ctx))) return st;
    return host_mip(ctx, src, w, h, stride * 4, 0, dst, dst_stride * 4, 16);
}

// ------------------------------------------------------------------ device memory
int zap_tex_cuda_bc_encode_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, void *out,
                               void *stream) {
    ZTC_NVTX();
    if (!valid_fmt_bc(fmt)) return fail(ZTC_ERR_UNSUPPORTED, "format %d", fmt);
    int st = check_lambda(rdo);
    if (st) return st;
    if (rdo > 0.0f) return zap_tex_cuda_bc_encode_rdo_dev(ctx, rgba, w, h, stride, fmt, rdo, 0, out, stream);
    return zap_tex_cuda_bc_encode_u8_dev(ctx, rgba, 4, w, h, stride, fmt, out, stream);
}

int zap_tex_cuda_bc_encode_rdo_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, int band_rows,
                                   void *out, void *stream) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (!valid_fmt_bc(fmt)) return fail(ZTC_ERR_UNSUPPORTED, "format %d", fmt);
    if ((st = check_lambda(rdo))) return st;
    if (band_rows < 0) return fail(ZTC_ERR_INVALID_ARG, "band_rows %d", band_rows);
    if (misaligned(out, block_bytes(fmt))) return fail(ZTC_ERR_INVALID_ARG, "out must be aligned to the block size");
    if ((st = resolve(ctx))) return st;
    const ztc::SrcU8 s8{rgba, stride, w, h, 4, (((uintptr_t)rgba | stride) & 15u) == 0};
    if (rdo <= 0.0f) return dev_encode(ctx, fmt, s8, nullptr, w, h, out, (cudaStream_t)stream);
    return rdo_encode(ctx, fmt, s8, w, h, rdo, band_rows, out, (cudaStream_t)stream);
}

int zap_tex_cuda_bc_encode_u8_dev(zap_tex_cuda_ctx *ctx, const uint8_t *src, int channels, int w, int h, size_t stride, int fmt, void *out,
                                  void *stream) {
    ZTC_NVTX();
    if (channels != 1 && channels != 2 && channels != 4) return fail(ZTC_ERR_INVALID_ARG, "channels %d", channels);
    int st = check_image(src, out, w, h, stride, (size_t)w * channels);
    if (st) return st;
    if (!valid_fmt_bc(fmt) && fmt != ZTC_ASTC4X4) return fail(ZTC_ERR_UNSUPPORTED, "format %d", fmt);
    if (misaligned(out, block_bytes(fmt == ZTC_ASTC4X4 ? ZTC_BC7 : fmt))) return fail(ZTC_ERR_INVALID_ARG, "out must be aligned to the block size");
    if ((st = resolve(ctx))) return st;
    ztc::SrcU8 s8{src, stride, w, h, channels, channels == 4 && (((uintptr_t)src | stride) & 15u) == 0};
    return dev_encode(ctx, fmt, s8, nullptr, w, h, out, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- split / merge (zap_tex.h:1549-1571)
static int regroup_args(const void *in, size_t n, int fmt, const void *out) {
    if (!valid_fmt_bc(fmt)) return fail(ZTC_ERR_UNSUPPORTED, "format %d (split / merge take BC1..BC7)", fmt);
    if (n && (!in || !out)) return fail(ZTC_ERR_INVALID_ARG, "null pointer");
    const uint8_t *a = (const uint8_t *)in, *b = (const uint8_t *)out;
    if (n && a < b + n && b < a + n) return fail(ZTC_ERR_INVALID_ARG, "input and output overlap");
    return ZTC_OK;
}

static int host_regroup(zap_tex_cuda_ctx *ctx, const void *in, size_t n, int fmt, void *out, int to_planes) {
    int st = regroup_args(in, n, fmt, out);
    if (st || !n) return st;
    if ((st = resolve(ctx))) return st;
    if ((st = grow((void **)&ctx->d_in, &ctx->d_in_cap, n, "cudaMalloc(input)"))) return st;
    if ((st = grow((void **)&ctx->d_out, &ctx->d_out_cap, n, "cudaMalloc(output)"))) return st;
    cudaStream_t s = ctx->stream[0];
    ZTC_CHECK(cudaMemcpyAsync(ctx->d_in, in, n, cudaMemcpyHostToDevice, s), "host->device copy");
    ZTC_CHECK(ztc_launch_bc_regroup(ctx->d_in, ctx->d_out, n, fmt, to_planes, s), "split / merge launch");
    ZTC_CHECK(cudaMemcpyAsync(out, ctx->d_out, n, cudaMemcpyDeviceToHost, s), "device->host copy");
    ZTC_CHECK(cudaStreamSynchronize(s), "split / merge");
    return ZTC_OK;
}

static int dev_regroup(zap_tex_cuda_ctx *ctx, const void *in, size_t n, int fmt, void *out, int to_planes, void *stream) {
    int st = regroup_args(in, n, fmt, out);
    if (st || !n) return st;
    if ((st = resolve(ctx))) return st;
    ZTC_CHECK(ztc_launch_bc_regroup((const uint8_t *)in, (uint8_t *)out, n, fmt, to_planes, (cudaStream_t)stream), "split / merge launch");
    return ZTC_OK;
}

int zap_tex_cuda_bc_split(zap_tex_cuda_ctx *ctx, const void *bc, size_t n, int fmt, void *out) {
    ZTC_NVTX();
    return host_regroup(ctx, bc, n, fmt, out, 1);
}
int zap_tex_cuda_bc_merge(zap_tex_cuda_ctx *ctx, const void *planes, size_t n, int fmt, void *out) {
    ZTC_NVTX();
    return host_regroup(ctx, planes, n, fmt, out, 0);
}
int zap_tex_cuda_bc_split_dev(zap_tex_cuda_ctx *ctx, const void *bc, size_t n, int fmt, void *out, void *stream) {
    ZTC_NVTX();
    return dev_regroup(ctx, bc, n, fmt, out, 1, stream);
}
int zap_tex_cuda_bc_merge_dev(zap_tex_cuda_ctx *ctx, const void *planes, size_t n, int fmt, void *out, void *stream) {
    ZTC_NVTX();
    return dev_regroup(ctx, planes, n, fmt, out, 0, stream);
}

int zap_tex_cuda_bc_encode_split_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, void *out,
                                     void *stream) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (!valid_fmt_bc(fmt)) return fail(ZTC_ERR_UNSUPPORTED, "format %d (the split form exists for BC1..BC7)", fmt);
    if ((st = resolve(ctx))) return st;
    const ztc::SrcU8 s8{rgba, stride, w, h, 4, (((uintptr_t)rgba | stride) & 15u) == 0};
    const int bw = (w + 3) / 4, bh = (h + 3) / 4;
    const ztc::BlockOut planes{(uint8_t *)out, (size_t)bw * (size_t)bh, fmt, 1};
    cudaStream_t s = (cudaStream_t)stream;
    if (fmt != ZTC_BC7) {
        ZTC_CHECK(ztc_launch_bcn_to(fmt, s8, 0, bh, planes, 0, s), "kernel launch");
        return ZTC_OK;
    }
    void *scratch = nullptr;
    ZTC_CHECK(ztc_malloc_async(&scratch, ztc::bc7_scratch_bytes((size_t)bw * bh), s), "cudaMallocAsync(scratch)");
    cudaError_t e = ztc_launch_bc7_to(s8, 0, bh, planes, 0, scratch, s);
    cudaFreeAsync(scratch, s);
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    return ZTC_OK;
}

int zap_tex_cuda_bc6h_encode_dev(zap_tex_cuda_ctx *ctx, const float *rgba, int w, int h, size_t stride, void *out, void *stream) {
    ZTC_NVTX();
    int st = check_image(rgba, out, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (misaligned(rgba, 4) || misaligned(out, 16)) return fail(ZTC_ERR_INVALID_ARG, "misaligned texels (4 B) or blocks (16 B)");
    if ((st = resolve(ctx))) return st;
    ztc::SrcU8 none{};
    ztc::SrcHdr sh{rgba, stride, w, h, 4, 1};
    return dev_encode(ctx, ZTC_BC6H, none, &sh, w, h, out, (cudaStream_t)stream);
}

int zap_tex_cuda_bc6h_encode_half_dev(zap_tex_cuda_ctx *ctx, const uint16_t *src, int channels, int w, int h, size_t stride, void *out,
                                      void *stream) {
    ZTC_NVTX();
    if (channels != 3 && channels != 4) return fail(ZTC_ERR_INVALID_ARG, "channels %d", channels);
    int st = check_image(src, out, w, h, stride, (size_t)w * channels);
    if (st) return st;
    if (misaligned(src, 2) || misaligned(out, 16)) return fail(ZTC_ERR_INVALID_ARG, "misaligned texels (2 B) or blocks (16 B)");
    if ((st = resolve(ctx))) return st;
    ztc::SrcU8 none{};
    ztc::SrcHdr sh{src, stride, w, h, channels, 0};
    return dev_encode(ctx, ZTC_BC6H, none, &sh, w, h, out, (cudaStream_t)stream);
}

int zap_tex_cuda_astc_encode_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, void *out, void *stream) {
    ZTC_NVTX();
    return zap_tex_cuda_bc_encode_u8_dev(ctx, rgba, 4, w, h, stride, ZTC_ASTC4X4, out, stream);
}

int zap_tex_cuda_mip_next_dev(zap_tex_cuda_ctx *ctx, const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst,
                              size_t dst_stride, void *stream) {
    ZTC_NVTX();
    int st = check_image(src, dst, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if ((st = resolve(ctx))) return st;
    cudaError_t e = ztc_launch_mip(src, w, h, stride, srgb, dst, dst_stride, (cudaStream_t)stream);
    return e == cudaSuccess ? ZTC_OK : cuda_fail(e, "mip launch");
}

int zap_tex_cuda_mip_next_f_dev(zap_tex_cuda_ctx *ctx, const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride,
                                void *stream) {
    ZTC_NVTX();
    int st = check_image(src, dst, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if (misaligned(src, 4) || misaligned(dst, 4)) return fail(ZTC_ERR_INVALID_ARG, "float texels must be 4-byte aligned");
    if ((st = resolve(ctx))) return st;
    cudaError_t e = ztc_launch_mip_f(src, w, h, stride, dst, dst_stride, (cudaStream_t)stream);
    return e == cudaSuccess ? ZTC_OK : cuda_fail(e, "mip launch");
}

size_t zap_tex_cuda_mip_chain_bytes(int w, int h) {
    size_t total = 0;
    while (w > 1 || h > 1) {
        w = w > 1 ? w / 2 : 1; h = h > 1 ? h / 2 : 1;
        total += (size_t)w * h * 4;
    }
    return total;
}

int zap_tex_cuda_mip_chain_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int srgb, uint8_t *dst, void *stream) {
    ZTC_NVTX();
    int st = check_image(rgba, dst, w, h, stride, (size_t)w * 4);
    if (st) return st;
    if ((st = resolve(ctx))) return st;
    const uint8_t *prev = rgba;
    size_t prev_stride = stride;
    uint8_t *o = dst;
    while (w > 1 || h > 1) {
        int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
        cudaError_t e = ztc_launch_mip(prev, w, h, prev_stride, srgb, o, (size_t)nw * 4, (cudaStream_t)stream);
        if (e != cudaSuccess) return cuda_fail(e, "mip launch");
        prev = o; prev_stride = (size_t)nw * 4; o += (size_t)nw * nh * 4;
        w = nw; h = nh;
    }
    return ZTC_OK;
}

}  // extern "C"

// ztc_internal.h - launchers shared between the kernel files and the C-ABI layer (not installed).
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

enum { ZTC_FMT_BC1 = 0, ZTC_FMT_BC3 = 1, ZTC_FMT_BC4 = 2, ZTC_FMT_BC5 = 3, ZTC_FMT_BC7 = 4, ZTC_FMT_BC6H = 5, ZTC_FMT_ASTC = 6 };

namespace ztc {
struct SrcU8;

// Per-device constant tables (sRGB, ASTC). Uploaded once per device by the context.

// Half-float source for BC6H: `channels` halfs per texel (3 or 4), or float RGBA when f32 is set.
struct SrcHdr {
    const void *base;
    size_t stride;  // elements (floats or halfs) per row
    int w, h, channels, f32;
};

// An NVTX range over one C-ABI call, named after the entry point, so a timeline profiler shows each call with its
// copies and kernels under it. NVTX v3 is header-only: with no profiler attached, a push and a pop each test one
// pointer.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define ZTC_NVTX() ::ztc::NvtxRange ztc_nvtx_range_(__func__)

// Kernel tracing (off by default): CUDA events around each launch, aggregated per kernel name on report.
void trace_begin(const char *name, cudaStream_t s);
void trace_end(cudaStream_t s);
void trace_units(long n);                                     // units the open launch processes (host-known)
void trace_units_dev(const uint32_t *d_count, cudaStream_t s);  // ... or read from a device counter
struct TraceScope {
    cudaStream_t s;
    TraceScope(const char *name, cudaStream_t st) : s(st) { trace_begin(name, st); }
    ~TraceScope() { trace_end(s); }
};

// BC7 work-list scratch: one entry per block that mode 6 alone does not finish
struct Bc7Scratch {
    uint32_t *count;  // 1 counter (zeroed by the launcher)
    uint2 *items;     // (block index, mode-6 SSE), capacity = blocks of the launch
};
size_t bc7_scratch_bytes(size_t nblocks);
// ASTC work list: blocks that go on to the two-partition search
size_t astc_scratch_bytes(size_t nblocks);
}  // namespace ztc

// ---------------------------------------------------------------- batched encoder descriptors (device memory)
namespace ztc {
struct BatchLevel {     // one (texture, mip level) to encode
    const uint8_t *src; // RGBA8 texels of the level
    uint8_t *dst;       // its encoded blocks
    size_t pitch;       // bytes per texel row
    int w, h, bw, fmt;
    uint32_t gbase;     // BC7 levels: batch-wide id of the level's first block (ids run over the batch's BC7 levels)
    uint32_t pad;
};
struct BatchTile {      // count blocks of one level, from block index `first`
    int level, first, count;
    int tw;             // 0: a row strip, blocks first .. first + count - 1; else a 2-D tile tw blocks wide (row-major)
};
#ifdef __CUDACC__
// block index (raster order in a level bw blocks wide) of the tile's j-th block
__host__ __device__ inline int tile_block(const BatchTile &t, int bw, int j) {
    return t.tw ? t.first + (j / t.tw) * bw + (j % t.tw) : t.first + j;
}
#endif
struct BatchMip {       // one (texture, level d >= 1): built from level d - 1
    const uint8_t *src;
    uint8_t *dst;
    size_t src_pitch, dst_pitch;
    int w, h, nw, nh, srgb, pad;  // w, h: source level size
};
struct BatchMipTile {   // output texel pairs [first, first + count) of one BatchMip, row-major over (nw + 1) / 2 pairs
    int mip, first, count, pad;
};
}  // namespace ztc

// `regs`: 0 = the register cap of the single-image kernels (more resident CTAs), 1 = a looser cap (fewer spills)
cudaError_t ztc_launch_batch_bcn(int fmt, int cta, int regs, int grid, const ztc::BatchLevel *levels, const ztc::BatchTile *tiles, int ntiles,
                                 uint32_t *counter, cudaStream_t stream);
// BC7 in two launches: mode 6 over the tile queue, appending (batch-wide block id, SSE) of the blocks it does not
// finish to hard_items; then mode 5 over that list, appending its opaque blocks to opaque_items (opaque_count zeroed
// by the caller), and mode 1 over those (bases / level_of: the BC7 levels' first ids, ascending, and their indices in
// `levels`)
cudaError_t ztc_launch_batch_bc7_mode6(int cta, int regs, int grid, const ztc::BatchLevel *levels, const ztc::BatchTile *tiles, int ntiles,
                                       uint32_t *counter, uint32_t *hard_count, uint2 *hard_items, cudaStream_t stream);
cudaError_t ztc_launch_batch_bc7_hard(int grid, const ztc::BatchLevel *levels, const uint32_t *bases, const int *level_of, int nlevels,
                                      const uint32_t *hard_count, const uint2 *hard_items, uint32_t *opaque_count, uint2 *opaque_items,
                                      cudaStream_t stream);
namespace ztc { struct SrgbTables; }
cudaError_t ztc_launch_batch_mip(int grid, const ztc::BatchMip *mips, const ztc::BatchMipTile *tiles, int ntiles, const ztc::SrgbTables *srgb_tables,
                                 cudaStream_t stream);
const void *ztc_batch_bcn_kernel_fn(int fmt, int cta, int regs);
const void *ztc_batch_bc7_kernel_fn(int cta, int regs);  // the mode 6 tile-queue kernel
const void *ztc_batch_bc7_hard_kernel_fn();
const void *ztc_batch_mip_kernel_fn();
namespace ztc {
// The sRGB tables of the mip generator: linear value of each sRGB code (zap_tex.h:1360-1393), the thresholds where
// a code rounds up (:1394-1427, + an infinite sentinel), and a search start per bucket of linear values (bucket =
// the float's exponent and top 6 mantissa bits over [2^-16, 1], bucket 0 below): the answer at the bucket's lowest
// value, a lower bound for every value in it.
constexpr int kSrgbBuckets = 17 * 64;
struct SrgbTables {
    float lin[256], thr[256];
    uint8_t bucket[kSrgbBuckets];
};
void srgb_tables_host(SrgbTables &t);
}  // namespace ztc

// Every device and pinned-host allocation of the library goes through these (api.cu), so a test can make chosen
// ones fail (zap_tex_cuda_debug_fail_allocations) and check that each entry point reports ZTC_ERR_NO_MEMORY and the
// library keeps working afterwards.
cudaError_t ztc_malloc(void **p, size_t n);
cudaError_t ztc_malloc_async(void **p, size_t n, cudaStream_t s);
cudaError_t ztc_malloc_host(void **p, size_t n);

// records the calling thread's error message (zap_tex_cuda_last_error) and returns status
int ztc_set_error(int status, const char *msg);
// makes ctx's device current (NULL: the current device's default context) with its tables uploaded
struct zap_tex_cuda_ctx;
int ztc_ctx_activate(zap_tex_cuda_ctx *ctx);

cudaError_t ztc_launch_bcn(int fmt, const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, cudaStream_t stream);
cudaError_t ztc_launch_bc7(const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, void *scratch, cudaStream_t stream);
// the same encoders into a BlockOut (raster blocks or split field planes); b0: output index of the first block
namespace ztc { struct BlockOut; }
cudaError_t ztc_launch_bcn_to(int fmt, const ztc::SrcU8 &src, int by0, int nby, const ztc::BlockOut &out, size_t b0, cudaStream_t stream);
cudaError_t ztc_launch_bc7_to(const ztc::SrcU8 &src, int by0, int nby, const ztc::BlockOut &out, size_t b0, void *scratch,
                              cudaStream_t stream);
// RDO (lambda > 0) over base encodings already in `out`, in place: one chain per band_rows block rows (0: one)
// SMs of the current device (cached per device)
int ztc_sm_count();
cudaError_t ztc_launch_rdo(int fmt, const ztc::SrcU8 &src, uint8_t *out, float lambda, int band_rows, cudaStream_t stream);
// split (to_planes = 1) or merge n bytes of BC1..BC7 data, device to device (zap_tex.h:1549-1571)
cudaError_t ztc_launch_bc_regroup(const uint8_t *in, uint8_t *out, size_t n, int fmt, int to_planes, cudaStream_t stream);
cudaError_t ztc_launch_bc6h(const ztc::SrcHdr &src, int by0, int nby, uint8_t *out, cudaStream_t stream);
cudaError_t ztc_launch_astc(const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, void *scratch, cudaStream_t stream);
// zap_astc_decode (zap_tex.h:1344-1356), device to device; bc 16-byte aligned
cudaError_t ztc_launch_astc_decode(const uint8_t *bc, int w, int h, uint8_t *out, size_t stride, cudaStream_t stream);
cudaError_t ztc_launch_mip(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride,
                           cudaStream_t stream);
cudaError_t ztc_launch_mip_f(const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride, cudaStream_t stream);

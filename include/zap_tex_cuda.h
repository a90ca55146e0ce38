/* zap_tex_cuda.h - B200 (sm_100a) drop-in for the zap_tex.h texture encoders.
 *
 * A thin C ABI over hand-written CUDA kernels. Every entry point keeps the argument list and the output bytes
 * of the zap_tex.h function it replaces (zap 1.3.0; cited as zap_tex.h:line), adds a context as the first
 * argument, and returns an int status (ZTC_OK = 0) where the reference returns void. Block order and block
 * layout are the reference's: raster order over the ceil(w/4) x ceil(h/4) block grid, partial edge blocks
 * replicating the last column / row.
 *
 * Host-pointer functions are synchronous, like the reference: they return once `out` holds the blocks.
 * `_dev` functions take device pointers and enqueue on `stream` (a cudaStream_t passed as void *; NULL = the
 * legacy default stream); they return after the launch, with launch errors only.
 *
 * No CPU fallback exists: without a usable CUDA device every call returns ZTC_ERR_NO_DEVICE.
 * A context is not thread-safe; use one per host thread (ctx == NULL selects a per-device default context,
 * guarded by a lock).
 */
#ifndef ZAP_TEX_CUDA_H
#define ZAP_TEX_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZAP_TEX_CUDA_VERSION 10000 /* 1.0.0 */

#if defined(__GNUC__)
#define ZTC_API __attribute__((visibility("default")))
#else
#define ZTC_API
#endif

typedef enum zap_tex_cuda_status {
    ZTC_OK = 0,
    ZTC_ERR_INVALID_ARG = -1, /* null pointer, w or h < 1, stride too small, size beyond the limit */
    ZTC_ERR_UNSUPPORTED = -2, /* rdo != 0 (rate-distortion mode), or a format the call does not take */
    ZTC_ERR_CUDA = -3,        /* a CUDA runtime error; zap_tex_cuda_last_error() has the text */
    ZTC_ERR_NO_MEMORY = -4,   /* device or pinned-host allocation failed */
    /* -5 is not used: no kernel of this library waits on a flag, a peer or another launch */
    ZTC_ERR_NO_DEVICE = -6    /* no CUDA device, or the device is not sm_100 */
} zap_tex_cuda_status;

/* Formats: 0..4 are zap_bc_format (zap_tex.h:32); BC6H and ASTC 4x4 have ids for the batched API. */
enum { ZTC_BC1 = 0, ZTC_BC3 = 1, ZTC_BC4 = 2, ZTC_BC5 = 3, ZTC_BC7 = 4, ZTC_BC6H = 5, ZTC_ASTC4X4 = 6 };

typedef struct zap_tex_cuda_ctx zap_tex_cuda_ctx;

/* ---------------------------------------------------------------- library and context */
ZTC_API int zap_tex_cuda_version(void);
ZTC_API const char *zap_tex_cuda_status_string(int status);
/* the last error message of the calling thread ("" when none) */
ZTC_API const char *zap_tex_cuda_last_error(void);
/* creates a context on `device` (its own streams, scratch arena, constant tables); no reference counterpart */
ZTC_API int zap_tex_cuda_create(int device, zap_tex_cuda_ctx **out);
ZTC_API int zap_tex_cuda_destroy(zap_tex_cuda_ctx *ctx);
/* pre-sizes the context's device scratch arena so later _dev calls allocate nothing (e.g. before stream capture) */
ZTC_API int zap_tex_cuda_reserve(zap_tex_cuda_ctx *ctx, size_t scratch_bytes);

/* Kernel tracing, no reference counterpart (the reference times one call with timespec_get, tex_bench.c:208-210).
   enable != 0 starts recording CUDA events around every kernel launch (process-wide, off by default);
   report writes "name launches total_ms" lines into buf, clears the record, and returns the text length. */
ZTC_API int zap_tex_cuda_trace_enable(int enable);
ZTC_API int zap_tex_cuda_trace_report(char *buf, size_t cap);

/* ---------------------------------------------------------------- sizes (zap_tex.h:34-37, :1435-1439) */
ZTC_API size_t zap_tex_cuda_block_bytes(int fmt);          /* replaces zap_bc_block_bytes, zap_tex.h:34 */
ZTC_API size_t zap_tex_cuda_bc_size(int w, int h, int fmt); /* replaces zap_bc_size, zap_tex.h:35-37 (BC6H/ASTC: 16 B/block) */
ZTC_API int zap_tex_cuda_mip_levels(int w, int h);          /* replaces zap_mip_levels, zap_tex.h:1435-1439 */

/* ---------------------------------------------------------------- drop-in encoders, host memory */
/* replaces zap_bc_encode (zap_tex.h:1474). rdo <= 0: the plain encode; rdo > 0: rate-distortion mode
   (zap_tex.h:223-306, :786-815), the reference's bytes for one call over the whole image; rdo must be finite */
ZTC_API int zap_tex_cuda_bc_encode(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo,
                           void *out);
/* replaces zap_bc6h_encode (zap_tex.h:946); stride in floats per row */
ZTC_API int zap_tex_cuda_bc6h_encode(zap_tex_cuda_ctx *ctx, const float *rgba, int w, int h, size_t stride, void *out);
/* replaces zap_astc_encode (zap_tex.h:1291) */
ZTC_API int zap_tex_cuda_astc_encode(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, void *out);
/* replaces zap_mip_next (zap_tex.h:1442) */
ZTC_API int zap_tex_cuda_mip_next(zap_tex_cuda_ctx *ctx, const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst,
                          size_t dst_stride);
/* replaces zap_mip_next_f (zap_tex.h:1460); strides in floats */
ZTC_API int zap_tex_cuda_mip_next_f(zap_tex_cuda_ctx *ctx, const float *src, int w, int h, size_t stride, float *dst,
                            size_t dst_stride);

/* ---------------------------------------------------------------- device memory, asynchronous */
ZTC_API int zap_tex_cuda_bc_encode_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo,
                               void *out, void *stream);
/* Rate-distortion mode in bands, no single reference counterpart: the bytes of one zap_bc_encode call per band of
   band_rows block rows (4 * band_rows texel rows; 0 = one band), as callers that encode a texture in bands get them
   (samples/dx11/viewer.cpp:455-471 uses 8-block-row bands). Each band's choices form one serial chain on the
   device (one warp), so more bands run in parallel. rdo finite; rdo <= 0 is the plain encode. */
ZTC_API int zap_tex_cuda_bc_encode_rdo_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo,
                                           int band_rows, void *out, void *stream);
ZTC_API int zap_tex_cuda_bc6h_encode_dev(zap_tex_cuda_ctx *ctx, const float *rgba, int w, int h, size_t stride, void *out,
                                 void *stream);
ZTC_API int zap_tex_cuda_astc_encode_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, void *out,
                                 void *stream);
ZTC_API int zap_tex_cuda_mip_next_dev(zap_tex_cuda_ctx *ctx, const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst,
                              size_t dst_stride, void *stream);
ZTC_API int zap_tex_cuda_mip_next_f_dev(zap_tex_cuda_ctx *ctx, const float *src, int w, int h, size_t stride, float *dst,
                                size_t dst_stride, void *stream);

/* Narrow inputs, no reference counterpart: the reference takes RGBA8 (zap_tex.h:1474) and RGBA f32 (:946); these
   read 1-, 2- or 4-channel uint8 texels (channels absent from the source read as 0, alpha as 255) or RGB(A) half
   floats, and produce the bytes the reference produces for the same texels widened to its input type.
   stride: bytes per row for uint8, halfs per row for half. */
ZTC_API int zap_tex_cuda_bc_encode_u8_dev(zap_tex_cuda_ctx *ctx, const uint8_t *src, int channels, int w, int h, size_t stride,
                                  int fmt, void *out, void *stream);
ZTC_API int zap_tex_cuda_bc6h_encode_half_dev(zap_tex_cuda_ctx *ctx, const uint16_t *src, int channels, int w, int h, size_t stride,
                                      void *out, void *stream);

/* Full mip chain, no single reference counterpart: the caller loop of zap.c:336-342 (zap_mip_next per level).
   Writes levels 1..levels-1 of `rgba` into `dst` tightly packed (level l at max(1, w>>l) x max(1, h>>l),
   row pitch 4 * width), largest first. dst must hold zap_tex_cuda_mip_chain_bytes(w, h) bytes. */
ZTC_API size_t zap_tex_cuda_mip_chain_bytes(int w, int h);
ZTC_API int zap_tex_cuda_mip_chain_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int srgb,
                               uint8_t *dst, void *stream);

/* ---------------------------------------------------------------- device decoders
   replaces zap_bc_decode (zap_tex.h:1526; BC7 all modes) and zap_bc6h_decode (zap_tex.h:963; stride in uint16),
   device memory, asynchronous; only texels inside the image are written */
ZTC_API int zap_tex_cuda_bc_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride,
                                       void *stream);
ZTC_API int zap_tex_cuda_bc6h_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint16_t *rgba, size_t stride,
                                         void *stream);
/* replaces zap_astc_decode (zap_tex.h:1344-1356): void-extent blocks and the block modes the reference decodes
   (4x4 weight grid, power-of-two weight range, 1-2 partitions of CEM 8 / 12); any other block decodes to magenta */
ZTC_API int zap_tex_cuda_astc_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint8_t *rgba, size_t stride,
                                         void *stream);
/* the same three decoders with host memory, synchronous (zap_tex.h:1526, :963, :1344); block pointers of the _dev
   variants must be aligned to the block size (8 bytes for BC1 / BC4, else 16), ZTC_ERR_INVALID_ARG otherwise */
ZTC_API int zap_tex_cuda_bc_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride);
ZTC_API int zap_tex_cuda_bc6h_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint16_t *rgba, size_t stride);
ZTC_API int zap_tex_cuda_astc_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint8_t *rgba, size_t stride);

/* ---------------------------------------------------------------- split / merge (zap_tex.h:1549-1571)
   Plane k of the split form holds field k of every block, the planes one after another: BC1 {4, 4}, BC3
   {2, 6, 4, 4}, BC4 {2, 6}, BC5 {2, 6, 2, 6}, BC7 {8, 1, 7} bytes; bytes after the last whole block are copied
   unchanged. n bytes in, n bytes out; in and out must not overlap (ZTC_ERR_INVALID_ARG). */
/* replace zap_bc_split / zap_bc_merge (zap_tex.h:1567-1568), host memory, synchronous */
ZTC_API int zap_tex_cuda_bc_split(zap_tex_cuda_ctx *ctx, const void *bc, size_t n, int fmt, void *out);
ZTC_API int zap_tex_cuda_bc_merge(zap_tex_cuda_ctx *ctx, const void *planes, size_t n, int fmt, void *out);
/* the same, device memory, asynchronous on stream */
ZTC_API int zap_tex_cuda_bc_split_dev(zap_tex_cuda_ctx *ctx, const void *bc, size_t n, int fmt, void *out, void *stream);
ZTC_API int zap_tex_cuda_bc_merge_dev(zap_tex_cuda_ctx *ctx, const void *planes, size_t n, int fmt, void *out, void *stream);
/* Encode straight into the split form, no reference counterpart: the bytes of zap_bc_encode (rdo 0) followed by
   zap_bc_split (the caller sequence of tex_bench.c:209-212), with the encoders storing each
   field into its plane, so no second pass over the blocks. out holds zap_tex_cuda_bc_size(w, h, fmt) bytes. */
ZTC_API int zap_tex_cuda_bc_encode_split_dev(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt,
                                             void *out, void *stream);

/* ---------------------------------------------------------------- differentiable palette decode, refinement
   No reference counterpart. With indices held fixed, decoding is linear in the endpoints: texel i of subset s,
   stored channel c, decodes to
     a_i * E[2s][c] + (1 - a_i) * E[2s+1][c]
   a_i = {1, 0, 2/3, 1/3}[index] for BC1 (the 4-colour order; zap_tex.h:52-62) and 1 - w(index)/64 for BC7 with the
   mode's 2-, 3- or 4-bit weights (zap_tex.h:367-417). BC7 covers all eight modes: up to three subsets, separate
   colour / alpha index sets (modes 4, 5: alpha takes the second set's weight), the rotation (alpha swapped with
   channel rot - 1 after the interpolation; endpoints are in stored order, texels in decoded order), and modes
   without alpha bits (alpha decodes to 255, zero gradient); the reserved mode decodes to 0 with zero gradient.
   Endpoints in 8-bit units: float[b][2][4] for BC1 (RGB used; alpha decodes to 0), float[b][6][4] for BC7
   (endpoint 2s + k of subset s; unused rows 0); decoded float[b][16][4].
   block_endpoints: the stored endpoints, expanded; palette_adjoint: grad_endpoints = d(sum g . decoded)/d(endpoints).
   refine: per block, `steps` Adam steps (learning rate lr, 8-bit units) on the block MSE through the adjoint,
   requantise in the block's own mode (BC1 565; BC7 modes 6, 5 and 1, the modes the encoder writes, rotation and
   partition kept), re-fit the indices, keep the new block only if its squared error is lower; optional per-block
   squared errors before / after (uint32[nblocks], device). Device pointers, asynchronous. */
ZTC_API int zap_tex_cuda_block_endpoints_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, float *endpoints,
                                             void *stream);
ZTC_API int zap_tex_cuda_palette_decode_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *endpoints,
                                            float *decoded, void *stream);
ZTC_API int zap_tex_cuda_palette_adjoint_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *grad_decoded,
                                             float *grad_endpoints, void *stream);
ZTC_API int zap_tex_cuda_refine_dev(zap_tex_cuda_ctx *ctx, int fmt, const uint8_t *rgba, int w, int h, size_t stride, void *blocks,
                                    int steps, float lr, uint32_t *sse_before, uint32_t *sse_after, void *stream);

/* ---------------------------------------------------------------- batched encoding
   Many textures at once, each with its mip chain, mixed formats. No single reference counterpart: it replaces the
   caller loop of zap.c:330-342 (zap_bc_encode per level, zap_mip_next between levels) run over many textures.
   Output per item: its levels' blocks concatenated, largest first (the DDS order of zap.c:332-349); bytes are
   the reference's for every level. The plan (mip buffer, tile queues, CUDA graph) is built once by
   zap_tex_cuda_batch_create; zap_tex_cuda_batch_run replays it as one graph launch, reading the items' current
   source texels. Pointers are device pointers. */
typedef struct zap_tex_cuda_item {
    const uint8_t *src; /* level 0, RGBA8 */
    int w, h;           /* 1 .. 65536 */
    size_t stride;      /* bytes per row of src */
    int fmt;            /* ZTC_BC1 .. ZTC_BC7 */
    int srgb;           /* mip filter in linear light (forced off for BC4/BC5, like zap.c:325) */
    int levels;         /* 0 = full chain (zap_tex_cuda_mip_levels), else the number of levels to encode */
    uint8_t *dst;       /* zap_tex_cuda_batch_item_bytes(w, h, fmt, levels) bytes */
} zap_tex_cuda_item;
typedef struct zap_tex_cuda_batch zap_tex_cuda_batch;
/* AUTOTUNE: per format class, time on the batch's own levels, one knob at a time, and keep the fastest: CTA size
   (64/128/256), register cap (tight: the single-image kernels' resident CTAs; loose: fewer CTAs, fewer spills),
   blocks per tile (1/2/4 CTAs' worth), tile shape (row strip / 2-D tile), and for BC7 the modes-5/1 grid (1 or 2
   CTAs per SM, or all that fit). zap_tex_cuda_batch_info reports the choices and the timings.
   Without AUTOTUNE the plan is 128 threads, tight registers, 1 CTA's worth of blocks per tile, row strips, unless
   the TILES_2D / REGS_LOOSE / TILE_X2 / TILE_X4 / CTA_64 / CTA_256 flags set a knob for every class. */
#define ZTC_BATCH_AUTOTUNE 1
#define ZTC_BATCH_NO_GRAPH 2 /* launch the sequence directly instead of capturing it into a CUDA graph */
#define ZTC_BATCH_TILES_2D 4
#define ZTC_BATCH_REGS_LOOSE 8
#define ZTC_BATCH_TILE_X2 16
#define ZTC_BATCH_TILE_X4 32
#define ZTC_BATCH_CTA_64 64
#define ZTC_BATCH_CTA_256 128
ZTC_API size_t zap_tex_cuda_batch_item_bytes(int w, int h, int fmt, int levels);
ZTC_API int zap_tex_cuda_batch_create(zap_tex_cuda_ctx *ctx, const zap_tex_cuda_item *items, int n, int flags,
                                      zap_tex_cuda_batch **out);
ZTC_API int zap_tex_cuda_batch_run(zap_tex_cuda_batch *batch, void *stream);
/* the same work as one plain launch per texture and per level (the per-texture caller loop), for comparison */
ZTC_API int zap_tex_cuda_batch_run_plain(zap_tex_cuda_batch *batch, void *stream);
/* text: tile counts, chosen blocks per CTA and autotune timings per format */
ZTC_API int zap_tex_cuda_batch_info(zap_tex_cuda_batch *batch, char *buf, size_t cap);
ZTC_API int zap_tex_cuda_batch_destroy(zap_tex_cuda_batch *batch);

/* ---------------------------------------------------------------- texture containers (the CLI's tex, zap.c:309-355)
   zap_tex_cuda_dds_header: the header zap.c:344-349 writes before the levels: "DDS " and 124 bytes, plus the 20-byte
   DX10 extension for BC7 or sRGB (148 bytes in all). fmt ZTC_BC1..ZTC_BC7; mips != 0 declares the full chain; srgb
   picks the _SRGB DXGI code and is ignored for BC4/BC5 (zap.c:325). hdr holds 148 bytes; *hdr_bytes (optional)
   receives 128 or 148. Host only: no device work.
   zap_tex_cuda_astc_header: the 16-byte .astc header of zap.c:312-321 (4x4x1 blocks, 24-bit sizes, depth 1).
   With zap_tex_cuda_batch_item_bytes, a batch caller writes each item's header and then its dst.
   zap_tex_cuda_tex_file: the whole file `zap tex [-f fmt] [-r rdo] [-m] [-S] w h in out` writes, computed on the
   device: the header, then every level's blocks, largest first (level l + 1 is zap_mip_next of level l, in linear
   light with srgb; each level is one zap_bc_encode call, so rdo > 0 runs one chain per level). fmt ZTC_ASTC4X4
   gives the .astc file (one level; mips, srgb and rdo are ignored, as by the CLI). rgba and out are host memory;
   out holds zap_tex_cuda_tex_file_bytes(w, h, fmt, mips, srgb) bytes (out_cap is checked); synchronous. */
ZTC_API int zap_tex_cuda_dds_header(int w, int h, int fmt, int mips, int srgb, void *hdr, size_t *hdr_bytes);
ZTC_API int zap_tex_cuda_astc_header(int w, int h, void *hdr);
ZTC_API size_t zap_tex_cuda_tex_file_bytes(int w, int h, int fmt, int mips, int srgb);
ZTC_API int zap_tex_cuda_tex_file(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo,
                                  int mips, int srgb, void *out, size_t out_cap);

/* ---------------------------------------------------------------- diagnostics (no reference counterpart) */
/* Issue-rate probe for the encoders' ALU roofline: enqueues on `stream` one launch of 8 CTAs of 256 threads per
   SM, every thread running 8 independent chains of one instruction kind for iters x 256 instructions (kind 0
   mad.lo.u32, 1 fma.rn.f32, 2 dp4a, 3 mad.lo.u32 and fma.rn.f32 alternating). *instructions receives the number of
   probe instructions the launch executes; the caller times it (CUDA events) and divides. sink: 4 bytes of device
   memory the kernel may write. */
ZTC_API int zap_tex_cuda_alu_probe_dev(int kind, int iters, void *sink, void *stream, double *instructions);
/* Test hook: of the library's next device or pinned-host allocations, let `skip` succeed and make the `count` after
   them fail as if the device were out of memory, so a caller's tests can check that every entry point then returns
   ZTC_ERR_NO_MEMORY and works again afterwards. (0, 0) clears it. Process-wide. */
ZTC_API int zap_tex_cuda_debug_fail_allocations(int skip, int count);
/* The bounds-check build (make -C zap_b200/csrc checks: libzap_tex_cuda_checks.so, -DZTC_CHECKS) checks the
   kernels' global and shared-memory indices (texel gathers, work lists, per-CTA compacted lists); a failed check
   skips its access and records (site << 24) | index in a device word. This synchronises the device and returns
   that word (0: no failure) and clears it. The product build returns ZTC_ERR_UNSUPPORTED. */
ZTC_API int zap_tex_cuda_debug_checks(unsigned int *first_failure);

/* Allocation-free BC7 encode. No counterpart in the reference (zap_tex.h allocates nothing because it runs on the
   CPU); it exists for callers that cannot allocate device memory when they encode: real-time frame loops where an
   allocation would stall or is not allowed, engines with a fixed up-front GPU budget, plug-in hosts that only hand
   over their own buffers. Same bytes as zap_tex_cuda_bc_encode_dev(..., ZTC_BC7, ...), device pointers, async on `stream`.
   It never calls cudaMalloc/cudaFree: its work list is a static device array sized for at most 1048576 4x4
   blocks (4096 x 4096 texels, about 8 MB held by every GPU that loads the library); larger textures return
   ZTC_ERR_INVALID_ARG. The first call on a device looks up that array's address (make it before any stream
   capture) and keeps it for the life of the process: a cudaDeviceReset unloads the library's device code and
   leaves that address stale, so do not call this entry point again after resetting a device it has run on. All
   calls share the array: calls whose kernels overlap on the GPU race, so serialise them (one stream, or events). */
ZTC_API int zap_tex_cuda_bc7_encode_noalloc_dev(const uint8_t *rgba, int w, int h, size_t stride, void *out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* ZAP_TEX_CUDA_H */

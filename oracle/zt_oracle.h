/* zt_oracle.h - CPU restatement of the zap_tex.h texture path. TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this library, and only as the
 * checker. The product path (zap_b200) never calls it.
 *
 * Every function keeps the reference's semantics at rdo = 0 (zap_tex.h, zap 1.3.0): same block layout, same
 * float operation order, same strict-"<" tie breaking. Format ids follow zap_bc_format (zap_tex.h:32).
 */
#ifndef ZT_ORACLE_H
#define ZT_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ZO_BC1 = 0, ZO_BC3 = 1, ZO_BC4 = 2, ZO_BC5 = 3, ZO_BC7 = 4 };

size_t zo_bc_size(int w, int h, int fmt);                                                      /* zap_tex.h:34-37 */
int zo_bc_encode(const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, void *out); /* :1474 (rdo 0 only) */
void zo_bc_decode(const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride);           /* :1526 */
void zo_bc6h_encode(const float *rgba, int w, int h, size_t stride, void *out);                   /* :946 */
void zo_bc6h_decode(const void *bc, int w, int h, uint16_t *rgba, size_t stride);                 /* :963 */
void zo_astc_encode(const uint8_t *rgba, int w, int h, size_t stride, void *out);                 /* :1291 */
void zo_astc_decode(const void *bc, int w, int h, uint8_t *rgba, size_t stride);                  /* :1344 */
int zo_mip_levels(int w, int h);                                                                  /* :1435 */
void zo_mip_next(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride); /* :1442 */
void zo_mip_next_f(const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride);              /* :1460 */
void zo_bc_split(const void *bc, size_t n, int fmt, void *out);                                   /* :1567 */
void zo_bc_merge(const void *planes, size_t n, int fmt, void *out);                               /* :1568 */

/* the CLI's texture containers (zap.c:309-355): DDS header (returns 128 or 148 bytes), .astc header, and the whole
   file `zap tex [-f fmt] [-r rdo] [-m] [-S] w h in out` writes (fmt 6 = .astc; out NULL returns the size only) */
size_t zo_dds_header(int w, int h, int fmt, int mips, int srgb, uint8_t hdr[148]);
void zo_astc_header(int w, int h, uint8_t hdr[16]);
size_t zo_tex_file(const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, int mips, int srgb, uint8_t *out);

/* internals pinned by the reference's self-test (tex_bench.c:47-48, :104-125) */
uint16_t zo_f2h(float f);
float zo_h2f(uint16_t h);
int zo_astc_partition(int seed, int x, int y, int count);
void zo_srgb_tables(float lin[256], float thr[255]);
/* ISE put then get of n values in range `range` (0..20); returns bits written, or -1 if the read-back differs */
int zo_ise_roundtrip(int range, int n, const int *v, int *got);

/* the fields of one BC7 block, all modes (zap_tex.h:378-412): info = {mode (8 = reserved), subsets, partition,
   rotation, alpha has own bits}, expanded 8-bit endpoints (endpoint 2s + k of subset s), each texel's subset and its
   colour / alpha interpolation weight (0..64); returns 0 for the reserved mode. The decode is
   lerp64(ep[2s][c], ep[2s+1][c], w), then alpha swapped with channel rot - 1 when rot > 0. */
int zo_bc7_fields(const void *blk, int info[5], int ep[6][4], int subset[16], int cw[16], int aw[16]);

/* per-block BC7 mode histogram of an encoded BC7 image (modes 0..7, 8 = reserved) */
void zo_bc7_mode_hist(const void *bc, size_t nblocks, int hist[9]);

#ifdef __cplusplus
}
#endif
#endif

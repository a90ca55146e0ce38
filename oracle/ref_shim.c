/* ref_shim.c - TEST INFRASTRUCTURE ONLY (the oracle's "reference" leg).
 *
 * Compiles the reference's own zap_tex.h (included from the reference tree at build time; no source is
 * copied here) into oracle/_ref/libzapref.so with non-inline exported wrappers, so that tests, smoke() and
 * bench.py's CPU-baseline leg can call the unmodified reference encoder. Build flags are pinned by
 * oracle/Makefile: -std=c11 -O2 -ffp-contract=off (x86-64 SSE, no FMA contraction), which is the float
 * semantics the CUDA kernels reproduce.
 *
 * Besides the public entry points it exports:
 *  - a band-parallel encode that follows the reference's only multi-core texture path
 *    (samples/dx11/viewer.cpp:452-471: bands of 8 block rows handed out from an atomic counter), used as
 *    the all-cores CPU baseline;
 *  - a few internals the reference's own self-test pins (tex_bench.c:47-48, :104-121), so the oracle
 *    restatement can be checked against them.
 */
#include "zap_tex.h"
#include <pthread.h>
#include <stdatomic.h>
#include <stdlib.h>

#define ZR_API __attribute__((visibility("default")))

ZR_API size_t zr_bc_size(int w, int h, int f) { return zap_bc_size(w, h, (zap_bc_format)f); }
ZR_API void zr_bc_encode(const uint8_t *rgba, int w, int h, size_t stride, int f, float rdo, void *out) {
    zap_bc_encode(rgba, w, h, stride, (zap_bc_format)f, rdo, out);
}
ZR_API void zr_bc_decode(const void *bc, int w, int h, int f, uint8_t *rgba, size_t stride) {
    zap_bc_decode(bc, w, h, (zap_bc_format)f, rgba, stride);
}
ZR_API void zr_bc6h_encode(const float *rgba, int w, int h, size_t stride, void *out) { zap_bc6h_encode(rgba, w, h, stride, out); }
ZR_API void zr_bc6h_decode(const void *bc, int w, int h, uint16_t *rgba, size_t stride) { zap_bc6h_decode(bc, w, h, rgba, stride); }
ZR_API void zr_astc_encode(const uint8_t *rgba, int w, int h, size_t stride, void *out) { zap_astc_encode(rgba, w, h, stride, out); }
ZR_API void zr_astc_decode(const void *bc, int w, int h, uint8_t *rgba, size_t stride) { zap_astc_decode(bc, w, h, rgba, stride); }
ZR_API int zr_mip_levels(int w, int h) { return zap_mip_levels(w, h); }
ZR_API void zr_mip_next(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride) {
    zap_mip_next(src, w, h, stride, srgb, dst, dst_stride);
}
ZR_API void zr_mip_next_f(const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride) {
    zap_mip_next_f(src, w, h, stride, dst, dst_stride);
}
ZR_API void zr_bc_split(const void *bc, size_t n, int f, void *out) { zap_bc_split(bc, n, (zap_bc_format)f, out); }
ZR_API void zr_bc_merge(const void *planes, size_t n, int f, void *out) { zap_bc_merge(planes, n, (zap_bc_format)f, out); }

/* internals pinned by the reference's self-test */
ZR_API uint16_t zr_f2h(float f) { return zap__f2h(f); }
ZR_API float zr_h2f(uint16_t h) { return zap__h2f(h); }
ZR_API int zr_astc_part(int seed, int x, int y, int count) { return zap__astc_part(seed, x, y, count); }
ZR_API const float *zr_srgb_lin(void) { return ZAP__SRGB_LIN; }
ZR_API const float *zr_srgb_thr(void) { return ZAP__SRGB_THR; }

/* ---- band-parallel encode (viewer.cpp:455-471 scheme) ---- */
enum { ZR_BC = 0, ZR_BC6H = 1, ZR_ASTC = 2 };
typedef struct {
    int kind, fmt, w, h, bw, bands;
    const void *src;
    size_t stride; /* bytes for RGBA8, floats for RGBA f32 */
    uint8_t *out;
    atomic_int next;
} zr_job;

static void *zr_worker(void *arg) {
    zr_job *j = (zr_job *)arg;
    const int kBand = 8; /* block rows per band */
    for (;;) {
        int b = atomic_fetch_add(&j->next, 1);
        if (b >= j->bands) break;
        int y0 = b * kBand * 4, hh = j->h - y0 < kBand * 4 ? j->h - y0 : kBand * 4;
        size_t bb = j->kind == ZR_BC ? zap_bc_block_bytes((zap_bc_format)j->fmt) : 16;
        uint8_t *o = j->out + (size_t)b * kBand * (size_t)j->bw * bb;
        if (j->kind == ZR_BC)
            zap_bc_encode((const uint8_t *)j->src + (size_t)y0 * j->stride, j->w, hh, j->stride, (zap_bc_format)j->fmt, 0, o);
        else if (j->kind == ZR_ASTC)
            zap_astc_encode((const uint8_t *)j->src + (size_t)y0 * j->stride, j->w, hh, j->stride, o);
        else
            zap_bc6h_encode((const float *)j->src + (size_t)y0 * j->stride, j->w, hh, j->stride, o);
    }
    return NULL;
}

static int zr_run(zr_job *j, int threads) {
    int bh = (j->h + 3) / 4;
    j->bw = (j->w + 3) / 4;
    j->bands = (bh + 7) / 8;
    atomic_init(&j->next, 0);
    if (threads < 1) threads = 1;
    if (threads > 64) threads = 64;
    pthread_t th[64];
    int started = 0;
    for (int t = 1; t < threads; t++)
        if (pthread_create(&th[started], NULL, zr_worker, j) == 0) started++;
    zr_worker(j);
    for (int t = 0; t < started; t++) pthread_join(th[t], NULL);
    return started + 1;
}

/* returns the number of threads that ran */
ZR_API int zr_bc_encode_mt(const uint8_t *rgba, int w, int h, size_t stride, int f, void *out, int threads) {
    zr_job j = { .kind = ZR_BC, .fmt = f, .w = w, .h = h, .src = rgba, .stride = stride, .out = (uint8_t *)out };
    return zr_run(&j, threads);
}
ZR_API int zr_bc6h_encode_mt(const float *rgba, int w, int h, size_t stride, void *out, int threads) {
    zr_job j = { .kind = ZR_BC6H, .w = w, .h = h, .src = rgba, .stride = stride, .out = (uint8_t *)out };
    return zr_run(&j, threads);
}
ZR_API int zr_astc_encode_mt(const uint8_t *rgba, int w, int h, size_t stride, void *out, int threads) {
    zr_job j = { .kind = ZR_ASTC, .w = w, .h = h, .src = rgba, .stride = stride, .out = (uint8_t *)out };
    return zr_run(&j, threads);
}

/* abi_driver.c - every host-side path of the C ABI that runs without a GPU, for the AddressSanitizer /
 * UndefinedBehaviorSanitizer build of the library (tests/test_host_sanitizers.py): size helpers, the DDS / .astc
 * header writers, status strings, the trace record, the test hooks, and every entry point's argument checks with bad
 * arguments (each must return its status without touching memory it was not given) and with good ones (no usable
 * device here: ZTC_ERR_NO_DEVICE, never a CPU fallback). Prints "ok" and exits 0 when every expectation holds. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "zap_tex_cuda.h"

static int g_fail = 0;
#define EXPECT(cond)                                                          \
    do {                                                                      \
        if (!(cond)) { fprintf(stderr, "%s:%d: %s\n", __FILE__, __LINE__, #cond); g_fail = 1; } \
    } while (0)

int main(int argc, char **argv) {
    /* with a device present (argv[1] == "gpu") valid calls may succeed; without one they return NO_DEVICE */
    const int gpu = argc > 1 && strcmp(argv[1], "gpu") == 0;
    const int nodev = gpu ? ZTC_OK : ZTC_ERR_NO_DEVICE;
    (void)nodev;

    EXPECT(zap_tex_cuda_version() == ZAP_TEX_CUDA_VERSION);
    for (int s = -8; s <= 1; s++) EXPECT(zap_tex_cuda_status_string(s) != NULL && strlen(zap_tex_cuda_status_string(s)) > 0);
    EXPECT(zap_tex_cuda_last_error() != NULL);

    /* sizes (zap_tex.h:34-37, :1435-1439) */
    EXPECT(zap_tex_cuda_block_bytes(ZTC_BC1) == 8 && zap_tex_cuda_block_bytes(ZTC_BC4) == 8);
    EXPECT(zap_tex_cuda_block_bytes(ZTC_BC7) == 16 && zap_tex_cuda_block_bytes(ZTC_ASTC4X4) == 16);
    EXPECT(zap_tex_cuda_bc_size(5, 3, ZTC_BC1) == 16 && zap_tex_cuda_bc_size(0, 4, ZTC_BC1) == 0);
    EXPECT(zap_tex_cuda_bc_size(-7, 4, ZTC_BC7) == 0 && zap_tex_cuda_bc_size(65536, 65536, ZTC_BC7) == (size_t)16384 * 16384 * 16);
    EXPECT(zap_tex_cuda_mip_levels(256, 128) == 9 && zap_tex_cuda_mip_levels(1, 1) == 1 && zap_tex_cuda_mip_levels(5, 3) == 3);
    EXPECT(zap_tex_cuda_mip_chain_bytes(4, 4) == (size_t)(2 * 2 + 1) * 4);
    EXPECT(zap_tex_cuda_batch_item_bytes(4, 4, ZTC_BC1, 0) == 24 && zap_tex_cuda_batch_item_bytes(4, 4, 6, 0) == 0);
    EXPECT(zap_tex_cuda_batch_item_bytes(0, 4, ZTC_BC1, 0) == 0);

    /* container headers (zap.c:309-355): every format, with and without mips / sRGB, and their argument checks */
    uint8_t hdr[160];
    size_t hn = 0;
    for (int f = 0; f <= ZTC_BC7; f++)
        for (int m = 0; m < 2; m++)
            for (int s = 0; s < 2; s++) {
                memset(hdr, 0xCD, sizeof hdr);
                EXPECT(zap_tex_cuda_dds_header(37, 21, f, m, s, hdr, &hn) == ZTC_OK);
                EXPECT(hn == 128 || hn == 148);
                EXPECT(memcmp(hdr, "DDS ", 4) == 0 && hdr[hn] == 0xCD);
                EXPECT(zap_tex_cuda_tex_file_bytes(37, 21, f, m, s) > hn);
            }
    EXPECT(zap_tex_cuda_dds_header(37, 21, ZTC_ASTC4X4, 0, 0, hdr, &hn) != ZTC_OK);  /* .astc has its own header */
    EXPECT(zap_tex_cuda_dds_header(37, 21, ZTC_BC6H, 0, 0, hdr, &hn) != ZTC_OK);     /* the CLI writes no BC6H file */
    EXPECT(zap_tex_cuda_dds_header(0, 21, ZTC_BC1, 0, 0, hdr, &hn) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_dds_header(4, 4, ZTC_BC1, 0, 0, NULL, &hn) == ZTC_ERR_INVALID_ARG);
    memset(hdr, 0xCD, sizeof hdr);
    EXPECT(zap_tex_cuda_astc_header(37, 21, hdr) == ZTC_OK && hdr[16] == 0xCD);
    EXPECT(zap_tex_cuda_astc_header(37, 21, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_tex_file_bytes(37, 21, ZTC_ASTC4X4, 0, 0) == 16 + zap_tex_cuda_bc_size(37, 21, ZTC_BC7));

    /* trace record: enable, report into a small buffer (truncated, terminated), disable */
    char buf[8];
    EXPECT(zap_tex_cuda_trace_enable(1) == ZTC_OK);
    EXPECT(zap_tex_cuda_trace_report(buf, sizeof buf) >= 0 && strlen(buf) < sizeof buf);
    EXPECT(zap_tex_cuda_trace_report(NULL, 0) >= 0);
    EXPECT(zap_tex_cuda_trace_enable(0) == ZTC_OK);

    /* test hooks */
    unsigned int word = 1;
    EXPECT(zap_tex_cuda_debug_fail_allocations(-1, 0) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_debug_fail_allocations(2, 1) == ZTC_OK && zap_tex_cuda_debug_fail_allocations(0, 0) == ZTC_OK);
    EXPECT(zap_tex_cuda_debug_checks(NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_debug_checks(&word) == ZTC_ERR_UNSUPPORTED && word == 0);

    /* argument checks: each bad argument returns its status before any device work */
    const int W = 13, H = 9;
    uint8_t *img = calloc((size_t)W * H * 4, 1), *out = calloc(zap_tex_cuda_bc_size(W, H, ZTC_BC7) + 64, 1);
    float *fimg = calloc((size_t)W * H * 4, sizeof(float));
    EXPECT(img && out && fimg);
    EXPECT(zap_tex_cuda_bc_encode(NULL, NULL, W, H, W * 4, ZTC_BC1, 0.0f, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4, ZTC_BC1, 0.0f, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, 0, H, W * 4, ZTC_BC1, 0.0f, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, -3, W * 4, ZTC_BC1, 0.0f, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4 - 1, ZTC_BC1, 0.0f, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4, 9, 0.0f, out) == ZTC_ERR_UNSUPPORTED);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4, ZTC_BC1, NAN, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4, ZTC_BC1, INFINITY, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode(NULL, img, 1 << 25, H, (size_t)4 << 25, ZTC_BC1, 0.0f, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc6h_encode(NULL, NULL, W, H, W * 4, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc6h_encode(NULL, fimg, W, H, W * 4 - 1, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_astc_encode(NULL, img, W, 0, W * 4, out) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_mip_next(NULL, img, W, H, W * 4, 1, NULL, 4) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_mip_next(NULL, img, W, H, W * 4, 1, out, 1) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_mip_next_f(NULL, fimg, W, H, W * 4, NULL, W * 2) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode_dev(NULL, img, W, H, W * 4, ZTC_BC7, 0.0f, NULL, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode_dev(NULL, img, W, H, W * 4, ZTC_BC7, 0.0f, out + 1, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode_rdo_dev(NULL, img, W, H, W * 4, ZTC_BC1, NAN, 8, out, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_encode_u8_dev(NULL, img, 3, W, H, W * 3, ZTC_BC4, out, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc6h_encode_half_dev(NULL, (const uint16_t *)img, 2, W, H, W * 2, out, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_decode(NULL, NULL, W, H, ZTC_BC1, img, W * 4) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_decode(NULL, out, W, H, ZTC_BC1, img, 3) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc6h_decode(NULL, out, 0, H, (uint16_t *)img, W * 4) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_astc_decode(NULL, out, W, H, NULL, W * 4) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc_split(NULL, out, 32, 9, img) != ZTC_OK);                      /* no such format */
    EXPECT(zap_tex_cuda_bc_split(NULL, out, 32, ZTC_BC7, out) == ZTC_ERR_INVALID_ARG); /* in place */
    EXPECT(zap_tex_cuda_bc_merge(NULL, out, 32, 11, img) != ZTC_OK);
    EXPECT(zap_tex_cuda_block_endpoints_dev(NULL, ZTC_BC3, out, 4, fimg, NULL) == ZTC_ERR_UNSUPPORTED);
    EXPECT(zap_tex_cuda_palette_decode_dev(NULL, ZTC_BC7, out + 8, 1, fimg, fimg, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_refine_dev(NULL, ZTC_BC1, img, W, H, W * 4, out, -1, 1.0f, NULL, NULL, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc7_encode_noalloc_dev(NULL, W, H, W * 4, out, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_bc7_encode_noalloc_dev(img, 4100, 4096, 4100 * 4, out, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_alu_probe_dev(7, 1, out, NULL, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_create(0, NULL) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_destroy(NULL) == ZTC_OK);

    /* batched: bad items are refused before anything is allocated */
    zap_tex_cuda_item it = {img, W, H, (size_t)W * 4, ZTC_BC1, 1, 0, out};
    zap_tex_cuda_batch *b = (zap_tex_cuda_batch *)out;
    EXPECT(zap_tex_cuda_batch_create(NULL, &it, 0, 0, &b) == ZTC_ERR_INVALID_ARG);
    it.fmt = ZTC_ASTC4X4;
    EXPECT(zap_tex_cuda_batch_create(NULL, &it, 1, 0, &b) == ZTC_ERR_UNSUPPORTED && b == NULL);
    it.fmt = ZTC_BC7;
    it.dst = out + 8;
    EXPECT(zap_tex_cuda_batch_create(NULL, &it, 1, 0, &b) == ZTC_ERR_INVALID_ARG);
    EXPECT(zap_tex_cuda_batch_run(NULL, NULL) == ZTC_ERR_INVALID_ARG && zap_tex_cuda_batch_destroy(NULL) == ZTC_OK);
    EXPECT(zap_tex_cuda_batch_info(NULL, buf, sizeof buf) == ZTC_ERR_INVALID_ARG);

    /* whole CLI files: a too-small buffer is refused before any work */
    EXPECT(zap_tex_cuda_tex_file(NULL, img, W, H, W * 4, ZTC_BC1, 0.0f, 1, 1, out, 16) != ZTC_OK);

    if (!gpu) {  /* good arguments and no usable device: a status, never a CPU fallback */
        zap_tex_cuda_ctx *ctx = NULL;
        EXPECT(zap_tex_cuda_create(0, &ctx) == ZTC_ERR_NO_DEVICE && ctx == NULL);
        EXPECT(zap_tex_cuda_bc_encode(NULL, img, W, H, W * 4, ZTC_BC7, 0.0f, out) == ZTC_ERR_NO_DEVICE);
        EXPECT(zap_tex_cuda_bc6h_encode(NULL, fimg, W, H, W * 4, out) == ZTC_ERR_NO_DEVICE);
        EXPECT(zap_tex_cuda_astc_encode(NULL, img, W, H, W * 4, out) == ZTC_ERR_NO_DEVICE);
        EXPECT(zap_tex_cuda_bc_decode(NULL, out, W, H, ZTC_BC1, img, W * 4) == ZTC_ERR_NO_DEVICE);
        EXPECT(zap_tex_cuda_bc7_encode_noalloc_dev(img, W, H, W * 4, out, NULL) == ZTC_ERR_NO_DEVICE);
        it.dst = out;
        b = NULL;
        EXPECT(zap_tex_cuda_batch_create(NULL, &it, 1, ZTC_BATCH_AUTOTUNE, &b) == ZTC_ERR_NO_DEVICE && b == NULL);
        EXPECT(zap_tex_cuda_tex_file(NULL, img, W, H, W * 4, ZTC_BC1, 0.0f, 1, 1, out,
                                     zap_tex_cuda_tex_file_bytes(W, H, ZTC_BC1, 1, 1)) == ZTC_ERR_NO_DEVICE);
        EXPECT(strlen(zap_tex_cuda_last_error()) > 0);
    }
    free(img);
    free(out);
    free(fimg);
    if (!g_fail) printf("ok\n");
    return g_fail;
}

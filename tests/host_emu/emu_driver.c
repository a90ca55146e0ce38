/* emu_driver.c - runs the kernels' block logic compiled for the host (emu.cu) over images read from a file, for the
 * AddressSanitizer / UndefinedBehaviorSanitizer build of that code (tests/test_host_sanitizers.py).
 *
 *   emu_driver in.bin out.bin
 * in.bin: records of int32 w, h, kind (0: RGBA8, 1: RGBA f32) and the texels (rows packed). For every RGBA8 record
 * out.bin gets BC1, BC3, BC4, BC5 and BC7 blocks (BC7 followed by one byte per block: 1 where the second phase
 * revisits it), ASTC blocks with the same per-block bytes, and the mip level below with sRGB off then on; for every
 * f32 record, its BC6H blocks. Exit status 0 when every record was read and written. */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

int emu_bc_encode(const uint8_t *img, int w, int h, size_t stride, int fmt, uint8_t *out, uint8_t *hard);
int emu_bc6h_encode(const float *img, int w, int h, size_t stride, uint8_t *out);
int emu_astc_encode(const uint8_t *img, int w, int h, size_t stride, uint8_t *out, uint8_t *hard);
int emu_mip_next(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride);

static size_t blocks_of(int w, int h) { return (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4); }

int main(int argc, char **argv) {
    if (argc != 3) return 2;
    FILE *in = fopen(argv[1], "rb"), *out = fopen(argv[2], "wb");
    if (!in || !out) return 2;
    int32_t hdr[3];
    while (fread(hdr, sizeof hdr, 1, in) == 1) {
        const int w = hdr[0], h = hdr[1], kind = hdr[2];
        if (w < 1 || h < 1 || w > 4096 || h > 4096 || (kind != 0 && kind != 1)) return 3;
        const size_t npx = (size_t)w * h, nb = blocks_of(w, h);
        if (kind == 1) {
            float *img = malloc(npx * 16);
            uint8_t *bc = malloc(nb * 16);
            if (!img || !bc || fread(img, 16, npx, in) != npx) return 4;
            emu_bc6h_encode(img, w, h, (size_t)w * 4, bc);
            fwrite(bc, 16, nb, out);
            free(img);
            free(bc);
            continue;
        }
        uint8_t *img = malloc(npx * 4), *bc = malloc(nb * 16), *hard = malloc(nb);
        if (!img || !bc || !hard || fread(img, 4, npx, in) != npx) return 4;
        for (int fmt = 0; fmt < 5; fmt++) {
            const size_t bs = (fmt == 0 || fmt == 2) ? 8 : 16;
            emu_bc_encode(img, w, h, (size_t)w * 4, fmt, bc, fmt == 4 ? hard : NULL);
            fwrite(bc, bs, nb, out);
            if (fmt == 4) fwrite(hard, 1, nb, out);
        }
        emu_astc_encode(img, w, h, (size_t)w * 4, bc, hard);
        fwrite(bc, 16, nb, out);
        fwrite(hard, 1, nb, out);
        const int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
        uint8_t *mip = malloc((size_t)nw * nh * 4);
        if (!mip) return 4;
        for (int srgb = 0; srgb < 2; srgb++) {
            emu_mip_next(img, w, h, (size_t)w * 4, srgb, mip, (size_t)nw * 4);
            fwrite(mip, 4, (size_t)nw * nh, out);
        }
        free(mip);
        free(img);
        free(bc);
        free(hard);
    }
    fclose(in);
    return fclose(out) == 0 ? 0 : 5;
}

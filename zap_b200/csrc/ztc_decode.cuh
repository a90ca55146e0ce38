// ztc_decode.cuh - block decoders (zap_bc_decode, zap_tex.h:1508-1547; BC7 all modes, :367-417; BC6H mode 11,
// :933-943), host+device. Used by the device decode kernels and by the refinement statistics.
#pragma once
#include "ztc_common.cuh"

namespace ztc {
namespace dec {

// BC7 mode descriptors (format spec): subsets, partition bits, rotation bits, index-selector bits, colour bits,
// alpha bits, per-endpoint p-bit, shared p-bit, index bits, secondary index bits
struct Mode { uint8_t ns, pb, rb, isb, cb, ab, epb, spb, ib, ib2; };
ZTC_DEV Mode mode_info(int m) {
    switch (m) {
    case 0: return {3, 4, 0, 0, 4, 0, 1, 0, 3, 0};
    case 1: return {2, 6, 0, 0, 6, 0, 0, 1, 3, 0};
    case 2: return {3, 6, 0, 0, 5, 0, 0, 0, 2, 0};
    case 3: return {2, 6, 0, 0, 7, 0, 1, 0, 2, 0};
    case 4: return {1, 0, 2, 1, 5, 6, 0, 0, 2, 3};
    case 5: return {1, 0, 2, 0, 7, 8, 0, 0, 2, 2};
    case 6: return {1, 0, 0, 0, 7, 7, 1, 0, 4, 0};
    default: return {2, 6, 0, 0, 5, 5, 1, 0, 2, 0};
    }
}

constexpr uint32_t p3(const char *s) {
    uint32_t v = 0;
    for (int i = 0; i < 16; i++) v |= (uint32_t)(s[i] - '0') << (2 * i);
    return v;
}
// partitions (format spec): two-subset masks (bit i = subset 1) and three-subset rows (texel 0 first)
static __constant__ uint16_t kP2d[64] = {
    0xCCCC, 0x8888, 0xEEEE, 0xECC8, 0xC880, 0xFEEC, 0xFEC8, 0xEC80, 0xC800, 0xFFEC, 0xFE80, 0xE800, 0xFFE8, 0xFF00, 0xFFF0, 0xF000,
    0xF710, 0x008E, 0x7100, 0x08CE, 0x008C, 0x7310, 0x3100, 0x8CCE, 0x088C, 0x3110, 0x6666, 0x366C, 0x17E8, 0x0FF0, 0x718E, 0x399C,
    0xAAAA, 0xF0F0, 0x5A5A, 0x33CC, 0x3C3C, 0x55AA, 0x9696, 0xA55A, 0x73CE, 0x13C8, 0x324C, 0x3BDC, 0x6996, 0xC33C, 0x9966, 0x0660,
    0x0272, 0x04E4, 0x4E40, 0x2720, 0xC936, 0x936C, 0x39C6, 0x639C, 0x9336, 0x9CC6, 0x817E, 0xE718, 0xCCF0, 0x0FCC, 0x7744, 0xEE22};
static __constant__ uint32_t kP3d[64] = {
    p3("0011001102212222"), p3("0001001122112221"), p3("0000200122112211"), p3("0222002200110111"), p3("0000000011221122"),
    p3("0011001100220022"), p3("0022002211111111"), p3("0011001122112211"), p3("0000000011112222"), p3("0000111111112222"),
    p3("0000111122222222"), p3("0012001200120012"), p3("0112011201120112"), p3("0122012201220122"), p3("0011011211221222"),
    p3("0011200122002220"), p3("0001001101121122"), p3("0111001120012200"), p3("0000112211221122"), p3("0022002200221111"),
    p3("0111011102220222"), p3("0001000122212221"), p3("0000001101220122"), p3("0000110022102210"), p3("0122012200110000"),
    p3("0012001211222222"), p3("0110122112210110"), p3("0000011012211221"), p3("0022110211020022"), p3("0110011020022222"),
    p3("0011012201220011"), p3("0000200022112221"), p3("0000000211221222"), p3("0222002200120011"), p3("0011001200220222"),
    p3("0120012001200120"), p3("0000111122220000"), p3("0120120120120120"), p3("0120201212010120"), p3("0011220011220011"),
    p3("0011112222000011"), p3("0101010122222222"), p3("0000000021212121"), p3("0022112200221122"), p3("0022001100220011"),
    p3("0220122102201221"), p3("0101222222220101"), p3("0000212121212121"), p3("0101010101012222"), p3("0222011102220111"),
    p3("0002111200021112"), p3("0000211221122112"), p3("0222011101110222"), p3("0002111211120002"), p3("0110011001102222"),
    p3("0000000021122112"), p3("0110011022222222"), p3("0022001100110022"), p3("0022112211220022"), p3("0000000000002112"),
    p3("0002000100020001"), p3("0222122202221222"), p3("0101222222222222"), p3("0111201122012220")};
// anchor texels (format spec): subset 1 of two, subsets 1 and 2 of three
static __constant__ uint8_t kA2d[64] = {
    15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 2, 8, 2, 2, 8, 8, 15, 2, 8, 2, 2, 8, 8, 2, 2,
    15, 15, 6, 8, 2, 8, 15, 15, 2, 8, 2, 2, 2, 15, 15, 6, 6, 2, 6, 8, 15, 15, 2, 2, 15, 15, 15, 15, 15, 2, 2, 15};
static __constant__ uint8_t kA3ad[64] = {
    3, 3, 15, 15, 8, 3, 15, 15, 8, 8, 6, 6, 6, 5, 3, 3, 3, 3, 8, 15, 3, 3, 6, 10, 5, 8, 8, 6, 8, 5, 15, 15,
    8, 15, 3, 5, 6, 10, 8, 15, 15, 3, 15, 5, 15, 15, 15, 15, 3, 15, 5, 5, 5, 8, 5, 10, 5, 10, 8, 13, 15, 12, 3, 3};
static __constant__ uint8_t kA3bd[64] = {
    15, 8, 8, 3, 15, 15, 3, 8, 15, 15, 15, 15, 15, 15, 15, 8, 15, 8, 15, 3, 15, 8, 15, 8, 3, 15, 6, 10, 15, 15, 10, 8,
    15, 3, 15, 10, 10, 8, 9, 10, 6, 15, 8, 15, 3, 6, 6, 8, 15, 3, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 3, 15, 15, 8};

// partition tables are device constants: the multi-subset modes decode on the device only
ZTC_DEV int subset_of(int ns, int part, int i) {
    if (ns == 1) return 0;
#ifdef __CUDA_ARCH__
    if (ns == 2) return (kP2d[part] >> i) & 1;
    return (int)((kP3d[part] >> (2 * i)) & 3u);
#else
    return 0;  // not used on the host
#endif
}
ZTC_DEV int anchor_of(int ns, int part, int s) {
#ifdef __CUDA_ARCH__
    return s == 0 ? 0 : ns == 2 ? kA2d[part] : s == 1 ? kA3ad[part] : kA3bd[part];
#else
    return 0;
#endif
}

// A BC7 block's fields (zap_tex.h:378-412): mode (8 = reserved), subsets, partition, rotation, whether alpha has
// its own bits (else it decodes to 255), the expanded 8-bit endpoints (endpoint 2s + k of subset s) and each
// texel's subset and colour / alpha interpolation weight (0..64). The decode of texel i is
// lerp64(ep[2s][c], ep[2s+1][c], w) per channel, then alpha swapped with channel rot - 1 when rot > 0; with the
// weights held fixed it is linear in the endpoints, which the differentiable decode builds on.
struct Bc7Fields {
    int mode, ns, part, rot, ab;
    int ep[6][4];
    uint8_t subset[16], cw[16], aw[16];
};
ZTC_DEV bool bc7_parse(const uint32_t w[4], Bc7Fields &F) {
    int mode = 0;
    while (mode < 8 && !((w[0] >> mode) & 1u)) mode++;
    F.mode = mode;
    F.ns = 1; F.part = 0; F.rot = 0; F.ab = 0;
    if (mode == 8) return false;
    const Mode M = mode_info(mode);
    int pos = mode + 1;
    const int part = (int)get_bits128(w, pos, M.pb); pos += M.pb;
    const int rot = (int)get_bits128(w, pos, M.rb); pos += M.rb;
    const int isb = (int)get_bits128(w, pos, M.isb); pos += M.isb;
    const int ne = 2 * M.ns;
    int cb = M.cb, ab = M.ab;
    for (int c = 0; c < 3; c++)
        for (int e = 0; e < ne; e++) { F.ep[e][c] = (int)get_bits128(w, pos, cb); pos += cb; }
    for (int e = 0; e < ne; e++) {
        if (ab) { F.ep[e][3] = (int)get_bits128(w, pos, ab); pos += ab; }
        else F.ep[e][3] = 255;
    }
    if (M.epb || M.spb) {
        for (int e = 0; e < ne; e++) {
            if (!M.epb && (e & 1)) continue;
            int p = (int)get_bits128(w, pos, 1); pos += 1;
            int last = M.epb ? e : e + 1;
            for (int k = e; k <= last; k++) {
                for (int c = 0; c < 3; c++) F.ep[k][c] = (F.ep[k][c] << 1) | p;
                if (ab) F.ep[k][3] = (F.ep[k][3] << 1) | p;
            }
        }
        cb++;
        if (ab) ab++;
    }
    for (int e = 0; e < ne; e++) {
        for (int c = 0; c < 3; c++) F.ep[e][c] = expand_bits(F.ep[e][c], cb);
        if (ab) F.ep[e][3] = expand_bits(F.ep[e][3], ab);
    }
    for (int e = ne; e < 6; e++)
        for (int c = 0; c < 4; c++) F.ep[e][c] = 0;
    int i1[16], i2[16];
    for (int i = 0; i < 16; i++) {
        int anchor = i == anchor_of(M.ns, part, subset_of(M.ns, part, i));
        i1[i] = (int)get_bits128(w, pos, M.ib - anchor); pos += M.ib - anchor;
    }
    for (int i = 0; i < 16; i++) {
        i2[i] = 0;
        if (M.ib2) { i2[i] = (int)get_bits128(w, pos, M.ib2 - (i == 0)); pos += M.ib2 - (i == 0); }
    }
    for (int i = 0; i < 16; i++) {
        F.subset[i] = (uint8_t)subset_of(M.ns, part, i);
        const int cw = (M.ib2 && isb) ? wbits(M.ib2, i2[i]) : wbits(M.ib, i1[i]);
        F.cw[i] = (uint8_t)cw;
        F.aw[i] = (uint8_t)(!M.ib2 ? cw : isb ? wbits(M.ib, i1[i]) : wbits(M.ib2, i2[i]));
    }
    F.ns = M.ns; F.part = part; F.rot = rot; F.ab = M.ab > 0;
    return true;
}

// full BC7 decode, all 8 modes; reserved mode -> transparent black (zap_tex.h:378-417)
ZTC_DEV void bc7_block(const uint32_t w[4], uint32_t out[16]) {
    if ((w[0] & 0x7Fu) == 0x40u) {  // mode 6, the encoder's common case, straight from its fixed layout
        // R0 R1 G0 G1 B0 B1 A0 A1 (7 bits each) from bit 7, p-bits at 63 and 64, indices from bit 65 (texel 0: 3 bits)
        const uint64_t lo = w[0] | ((uint64_t)w[1] << 32), hi = w[2] | ((uint64_t)w[3] << 32);
        const int p0 = (int)(lo >> 63), p1 = (int)(hi & 1u);
        int x0[4], x1[4];
        #pragma unroll
        for (int c = 0; c < 4; c++) {
            x0[c] = (int)(((lo >> (7 + 14 * c)) & 0x7Fu) << 1) | p0;
            x1[c] = (int)(((lo >> (14 + 14 * c)) & 0x7Fu) << 1) | p1;
        }
        const Lerp4 row(x0, x1);
        #pragma unroll
        for (int i = 0; i < 16; i++) out[i] = row.at(w4(i == 0 ? (int)((hi >> 1) & 7u) : (int)((hi >> (4 * i)) & 15u)));
        return;
    }
    Bc7Fields F;
    if (!bc7_parse(w, F)) {
        for (int i = 0; i < 16; i++) out[i] = 0;
        return;
    }
    for (int i = 0; i < 16; i++) {
        const int s = F.subset[i];
        int px[4];
        for (int c = 0; c < 3; c++) px[c] = lerp64(F.ep[2 * s][c], F.ep[2 * s + 1][c], F.cw[i]);
        px[3] = lerp64(F.ep[2 * s][3], F.ep[2 * s + 1][3], F.aw[i]);
        if (F.rot) { int t = px[3]; px[3] = px[F.rot - 1]; px[F.rot - 1] = t; }
        out[i] = pack_rgba(px[0], px[1], px[2], px[3]);
    }
}

// BC1 colour block; four_always: the BC3 colour half (zap_tex.h:1508-1517)
ZTC_DEV void bc1_block(uint2 v, bool four_always, uint32_t out[16]) {
    uint32_t c0 = v.x & 0xFFFFu, c1 = v.x >> 16;
    int pal[4][3];
    for (int k = 0; k < 2; k++) {
        uint32_t c = k ? c1 : c0;
        int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
        pal[k][0] = (R << 3) | (R >> 2); pal[k][1] = (G << 2) | (G >> 4); pal[k][2] = (B << 3) | (B >> 2);
    }
    const bool four = four_always || c0 > c1;
    for (int c = 0; c < 3; c++) {
        int a = pal[0][c], b = pal[1][c];
        pal[2][c] = four ? (2 * a + b + 1) / 3 : (a + b + 1) / 2;
        pal[3][c] = four ? (a + 2 * b + 1) / 3 : 0;
    }
    for (int i = 0; i < 16; i++) {
        int k = (int)((v.y >> (2 * i)) & 3u);
        out[i] = pack_rgba(pal[k][0], pal[k][1], pal[k][2], (!four && k == 3) ? 0 : 255);
    }
}

// BC4 channel block (zap_tex.h:1519-1524)
ZTC_DEV void bc4_block(uint2 v, uint8_t out[16]) {
    int a0 = v.x & 0xFF, a1 = (v.x >> 8) & 0xFF, pal[8];
    pal[0] = a0; pal[1] = a1;
    if (a0 > a1) for (int i = 2; i < 8; i++) pal[i] = ((8 - i) * a0 + (i - 1) * a1 + 3) / 7;
    else { for (int i = 2; i < 6; i++) pal[i] = ((6 - i) * a0 + (i - 1) * a1 + 2) / 5; pal[6] = 0; pal[7] = 255; }
    uint64_t idx = (uint64_t)(v.x >> 16) | ((uint64_t)v.y << 16);
    for (int i = 0; i < 16; i++) out[i] = (uint8_t)pal[(idx >> (3 * i)) & 7u];
}

// one block of format fmt (0..4) to 16 RGBA8 texels (zap_tex.h:1526-1547)
// A decoded 4x4 block of RGBA8 texels (px[i]: texel i, R in the low byte) into an image: each row of four texels
// inside the image as one 16-byte store when vec (the image and its pitch 16-byte aligned), texels past the right
// or bottom edge left out, a row the right edge cuts texel by texel (4-byte stores if aligned4, else bytes).
ZTC_DEV void store_block_rgba8(uint8_t *out, size_t stride, int w, int h, int bx, int by, const uint32_t px[16], bool vec,
                               bool aligned4) {
    #pragma unroll
    for (int r = 0; r < 4; r++) {
        const int y = by * 4 + r, x0 = bx * 4;
        if (y >= h) break;
        uint8_t *row = out + (size_t)y * stride + (size_t)x0 * 4;
        if (vec && x0 + 3 < w) {
            *(uint4 *)row = make_uint4(px[4 * r], px[4 * r + 1], px[4 * r + 2], px[4 * r + 3]);
            continue;
        }
        #pragma unroll
        for (int c = 0; c < 4; c++) {
            if (x0 + c >= w) break;
            const uint32_t v = px[4 * r + c];
            if (aligned4) *(uint32_t *)(row + 4 * c) = v;
            else { row[4 * c] = (uint8_t)v; row[4 * c + 1] = (uint8_t)(v >> 8); row[4 * c + 2] = (uint8_t)(v >> 16); row[4 * c + 3] = (uint8_t)(v >> 24); }
        }
    }
}

ZTC_DEV void bcn_block(int fmt, const uint8_t *b, uint32_t out[16]) {
    if (fmt == 0) { bc1_block(*(const uint2 *)b, false, out); return; }
    if (fmt == 4) {
        uint4 v = *(const uint4 *)b;
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        bc7_block(w, out);
        return;
    }
    uint8_t v0[16], v1[16];
    if (fmt == 1) {
        bc1_block(*(const uint2 *)(b + 8), true, out);
        bc4_block(*(const uint2 *)b, v0);
        for (int i = 0; i < 16; i++) out[i] = (out[i] & 0x00FFFFFFu) | ((uint32_t)v0[i] << 24);
        return;
    }
    bc4_block(*(const uint2 *)b, v0);
    if (fmt == 3) bc4_block(*(const uint2 *)(b + 8), v1);
    else for (int i = 0; i < 16; i++) v1[i] = 0;
    for (int i = 0; i < 16; i++) out[i] = pack_rgba(v0[i], v1[i], 0, 255);
}

// BC6H mode 11 to half bits, alpha 1.0 (zap_tex.h:933-943); other modes decode to 0
ZTC_DEV void bc6h_block(const uint32_t w[4], uint16_t out[16][4]) {
    for (int i = 0; i < 16; i++) out[i][0] = out[i][1] = out[i][2] = out[i][3] = 0;
    if (get_bits128(w, 0, 5) != 3u) return;
    int e[2][3];
    for (int k = 0; k < 2; k++)
        for (int c = 0; c < 3; c++) {
            int q = (int)get_bits128(w, 5 + 10 * (3 * k + c), 10);
            e[k][c] = q == 0 ? 0 : q == 1023 ? 0xFFFF : ((q << 16) + 0x8000) >> 10;
        }
    for (int i = 0; i < 16; i++) {
        int idx = i == 0 ? (int)get_bits128(w, 65, 3) : (int)get_bits128(w, 68 + 4 * (i - 1), 4);
        int wt = w4(idx);
        for (int c = 0; c < 3; c++) out[i][c] = (uint16_t)((lerp64(e[0][c], e[1][c], wt) * 31) >> 6);
        out[i][3] = 0x3C00;
    }
}

}  // namespace dec
}  // namespace ztc

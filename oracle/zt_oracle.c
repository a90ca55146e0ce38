/* zt_oracle.c - CPU restatement of the zap_tex.h texture path. TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker, never the thing measured or shipped: only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it. It restates the reference's algorithm (zap_tex.h of zap 1.3.0, cited
 * per function as zap_tex.h:line) in plain C11, compiled with -O2 -ffp-contract=off so that every float
 * operation is one IEEE single-precision op in source order, exactly like the reference built the same way.
 * Parity is pinned two ways (tests/test_oracle.py): byte-identical output against the reference itself
 * (oracle/_ref, built from the reference's header by oracle/Makefile) and the known answers of the
 * reference's own self-test (tex_bench.c).
 *
 * Conventions shared with the reference: texel i of a 4x4 block is (x, y) = (i & 3, i >> 2); partial edge
 * blocks replicate the last column / row; searches keep the first candidate on ties (strict "<").
 */
#include "zt_oracle.h"
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef uint8_t tx4[4]; /* one RGBA8 texel */

/* Algorithmic op counts, compiled only into oracle/liboracle_ops.so (-DZO_COUNT_OPS; oracle/count_ops.py). One
 * texel-to-palette-entry distance over C channels counts 3C + 1 ops (C differences, C squares, C accumulations,
 * one comparison); the BC7 mode 1 ranking counts 9 additions per texel summed into a subset's moments. Counters
 * are plain globals: count with one thread. Slot 0: everything; slot 1: BC7 mode 6 only. */
#ifdef ZO_COUNT_OPS
static uint64_t g_ops[2];
#define ZO_OPS(n) (g_ops[0] += (uint64_t)(n))
void zo_ops_take(uint64_t out[2]) { out[0] = g_ops[0]; out[1] = g_ops[1]; g_ops[0] = g_ops[1] = 0; }
#else
#define ZO_OPS(n) ((void)0)
#endif

static int imin(int a, int b) { return a < b ? a : b; }
static int iclamp(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }
static float fclamp255(float v) { return v < 0 ? 0 : v > 255 ? 255 : v; } /* NaN passes through, as in the reference */
/* candidate k of {g - 1, g, g + 1} with two's-complement wrap: the reference's three-candidate loops, as compiled
   for x86-64, try exactly these even when g is INT_MIN (an out-of-range float -> int conversion) */
static int around(int g, int k) { return (int)((unsigned)g + (unsigned)k - 1u); }

/* ------------------------------------------------------------------ bit streams (LSB first) */
typedef struct { uint8_t *b; int pos; } bitw;
typedef struct { const uint8_t *b; int pos; } bitr;
static void put_bits(bitw *w, unsigned v, int n) {
    for (int i = 0; i < n; i++, w->pos++)
        if ((v >> i) & 1u) w->b[w->pos >> 3] |= (uint8_t)(1u << (w->pos & 7));
}
static unsigned get_bits(bitr *r, int n) {
    unsigned v = 0;
    for (int i = 0; i < n; i++, r->pos++) v |= (unsigned)((r->b[r->pos >> 3] >> (r->pos & 7)) & 1u) << i;
    return v;
}
static void store_le(uint8_t *p, uint64_t v, int n) { for (int i = 0; i < n; i++, v >>= 8) p[i] = (uint8_t)v; }
static uint64_t load_le(const uint8_t *p, int n) { uint64_t v = 0; for (int i = n - 1; i >= 0; i--) v = (v << 8) | p[i]; return v; }

/* gather one 4x4 block with edge replication (zap_tex.h:1483-1488) */
static void gather8(const uint8_t *img, int w, int h, size_t stride, int bx, int by, tx4 t[16]) {
    for (int i = 0; i < 16; i++) {
        int x = imin(bx * 4 + (i & 3), w - 1), y = imin(by * 4 + (i >> 2), h - 1);
        memcpy(t[i], img + (size_t)y * stride + (size_t)x * 4, 4);
    }
}

/* ================================================================== BC1 (zap_tex.h:39-168) */
static void unpack565(unsigned c, int rgb[3]) { /* :41-44 */
    int r = (c >> 11) & 31, g = (c >> 5) & 63, b = c & 31;
    rgb[0] = (r << 3) | (r >> 2); rgb[1] = (g << 2) | (g >> 4); rgb[2] = (b << 3) | (b >> 2);
}
static uint16_t pack565(float r, float g, float b) { /* :45-49; (int) keeps x86 truncation */
    int R = (int)(r * 31.0f / 255.0f + 0.5f), G = (int)(g * 63.0f / 255.0f + 0.5f), B = (int)(b * 31.0f / 255.0f + 0.5f);
    return (uint16_t)((iclamp(R, 0, 31) << 11) | (iclamp(G, 0, 63) << 5) | iclamp(B, 0, 31));
}
/* 4-colour palette (the encoder always evaluates in 4-colour order, :52-62 with force4) */
static void bc1_pal4(uint16_t c0, uint16_t c1, int pal[4][3]) {
    unpack565(c0, pal[0]); unpack565(c1, pal[1]);
    for (int k = 0; k < 3; k++) {
        int a = pal[0][k], b = pal[1][k];
        pal[2][k] = (2 * a + b + 1) / 3; pal[3][k] = (a + 2 * b + 1) / 3;
    }
}
static int d3(const uint8_t *p, const int *q) { int r = p[0] - q[0], g = p[1] - q[1], b = p[2] - q[2]; return r * r + g * g + b * b; }

/* endpoints -> canonical order (c0 > c1, or solid c0 == c1 with all indices 0), best indices, SSE (:70-94) */
static int bc1_eval_pair(const tx4 t[16], uint16_t *c0, uint16_t *c1, uint32_t *idx) {
    if (*c0 < *c1) { uint16_t s = *c0; *c0 = *c1; *c1 = s; }
    int pal[4][3], err = 0;
    bc1_pal4(*c0, *c1, pal);
    if (*c0 == *c1) {
        *idx = 0;
        ZO_OPS(16 * 10);
        for (int i = 0; i < 16; i++) err += d3(t[i], pal[0]);
        return err;
    }
    ZO_OPS(16 * 4 * 10);
    uint32_t bits = 0;
    for (int i = 0; i < 16; i++) {
        int bk = 0, be = d3(t[i], pal[0]);
        for (int k = 1; k < 4; k++) { int e = d3(t[i], pal[k]); if (e < be) { be = e; bk = k; } }
        bits |= (uint32_t)bk << (2 * i);
        err += be;
    }
    *idx = bits;
    return err;
}

/* quality BC1 search (:97-168): PCA axis, two starts with least-squares refits, then +-1 endpoint climb */
static int bc1_block(const tx4 t[16], uint16_t *o0, uint16_t *o1, uint32_t *oidx) {
    float mu[3] = { 0, 0, 0 }, C[6] = { 0, 0, 0, 0, 0, 0 };
    for (int i = 0; i < 16; i++) for (int k = 0; k < 3; k++) mu[k] += t[i][k] / 16.0f;
    for (int i = 0; i < 16; i++) {
        float r = t[i][0] - mu[0], g = t[i][1] - mu[1], b = t[i][2] - mu[2];
        C[0] += r * r; C[1] += r * g; C[2] += r * b; C[3] += g * g; C[4] += g * b; C[5] += b * b;
    }
    float v[3] = { 1, 1, 1 };
    for (int it = 0; it < 6; it++) {
        float x = C[0] * v[0] + C[1] * v[1] + C[2] * v[2];
        float y = C[1] * v[0] + C[3] * v[1] + C[4] * v[2];
        float z = C[2] * v[0] + C[4] * v[1] + C[5] * v[2];
        float m = fabsf(x);
        if (fabsf(y) > m) m = fabsf(y);
        if (fabsf(z) > m) m = fabsf(z);
        if (m < 1e-6f) break;
        v[0] = x / m; v[1] = y / m; v[2] = z / m;
    }
    float n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], tmin = 1e9f, tmax = -1e9f;
    for (int i = 0; i < 16; i++) {
        float s = (t[i][0] - mu[0]) * v[0] + (t[i][1] - mu[1]) * v[1] + (t[i][2] - mu[2]) * v[2];
        if (s < tmin) tmin = s;
        if (s > tmax) tmax = s;
    }
    static const float LSW[4] = { 1.0f, 0.0f, 2.0f / 3.0f, 1.0f / 3.0f }; /* weight of c0 for index 0..3 */
    uint16_t b0 = 0, b1 = 0;
    uint32_t bidx = 0;
    int best = 1 << 30;
    for (int start = 0; start < 2; start++) {
        float inset = start ? 0.0f : (tmax - tmin) / 16.0f, lo = (tmin + inset) / n2, hi = (tmax - inset) / n2;
        uint16_t c0 = pack565(mu[0] + v[0] * hi, mu[1] + v[1] * hi, mu[2] + v[2] * hi);
        uint16_t c1 = pack565(mu[0] + v[0] * lo, mu[1] + v[1] * lo, mu[2] + v[2] * lo);
        uint32_t idx = 0;
        int e = bc1_eval_pair(t, &c0, &c1, &idx);
        for (int it = 0; it < 3 && e > 0; it++) {
            float aa = 0, ab = 0, bb = 0, sa[3] = { 0, 0, 0 }, sb[3] = { 0, 0, 0 };
            for (int i = 0; i < 16; i++) {
                float wa = LSW[(idx >> (2 * i)) & 3], wb = 1.0f - wa;
                aa += wa * wa; ab += wa * wb; bb += wb * wb;
                for (int k = 0; k < 3; k++) { sa[k] += wa * t[i][k]; sb[k] += wb * t[i][k]; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) break;
            float A[3], B[3];
            for (int k = 0; k < 3; k++) { A[k] = (sa[k] * bb - sb[k] * ab) / det; B[k] = (sb[k] * aa - sa[k] * ab) / det; }
            uint16_t n0 = pack565(A[0], A[1], A[2]), n1 = pack565(B[0], B[1], B[2]);
            uint32_t ni = 0;
            int ne = bc1_eval_pair(t, &n0, &n1, &ni);
            if (ne >= e) break;
            e = ne; c0 = n0; c1 = n1; idx = ni;
        }
        if (e < best) { best = e; b0 = c0; b1 = c1; bidx = idx; }
    }
    static const int SH[3] = { 11, 5, 0 }, MX[3] = { 31, 63, 31 };
    int improved = 1;
    for (int pass = 0; improved && pass < 8 && best > 0; pass++) {
        improved = 0;
        for (int ep = 0; ep < 2; ep++)
            for (int ch = 0; ch < 3; ch++)
                for (int d = -1; d <= 1; d += 2) {
                    unsigned c = ep ? b1 : b0;
                    int f = (int)(c >> SH[ch]) & MX[ch];
                    if (f + d < 0 || f + d > MX[ch]) continue;
                    c = (c & ~((unsigned)MX[ch] << SH[ch])) | ((unsigned)(f + d) << SH[ch]);
                    uint16_t n0 = ep ? b0 : (uint16_t)c, n1 = ep ? (uint16_t)c : b1;
                    uint32_t ni = 0;
                    int ne = bc1_eval_pair(t, &n0, &n1, &ni);
                    if (ne < best) { best = ne; b0 = n0; b1 = n1; bidx = ni; improved = 1; }
                }
    }
    *o0 = b0; *o1 = b1; *oidx = bidx;
    return best;
}

static void bc1_store(uint8_t *o, uint16_t c0, uint16_t c1, uint32_t idx) { store_le(o, c0, 2); store_le(o + 2, c1, 2); store_le(o + 4, idx, 4); }

/* ================================================================== BC4 (zap_tex.h:170-213) */
static void bc4_pal(int a0, int a1, int pal[8]) {
    pal[0] = a0; pal[1] = a1;
    if (a0 > a1) for (int i = 2; i < 8; i++) pal[i] = ((8 - i) * a0 + (i - 1) * a1 + 3) / 7;
    else { for (int i = 2; i < 6; i++) pal[i] = ((6 - i) * a0 + (i - 1) * a1 + 2) / 5; pal[6] = 0; pal[7] = 255; }
}
static int bc4_block(const uint8_t v[16], uint8_t *oa0, uint8_t *oa1, uint64_t *oidx) {
    int lo = 255, hi = 0;
    for (int i = 0; i < 16; i++) { if (v[i] < lo) lo = v[i]; if (v[i] > hi) hi = v[i]; }
    int best = 1 << 30, ba0 = hi, ba1 = lo;
    uint64_t bidx = 0;
    for (int d0 = 0; d0 < 3; d0++)
        for (int d1 = 0; d1 < 3; d1++) {
            int a0 = hi - d0, a1 = lo + d1;
            if (a0 <= a1) { a0 = hi; a1 = lo; }
            int pal[8], err = 0;
            uint64_t bits = 0;
            bc4_pal(a0, a1, pal);
            ZO_OPS(a0 == a1 ? 16 * 4 : 16 * 8 * 4);
            for (int i = 0; i < 16; i++) {
                if (a0 == a1) { err += (v[i] - pal[0]) * (v[i] - pal[0]); continue; }
                int bk = 0, be = (v[i] - pal[0]) * (v[i] - pal[0]);
                for (int k = 1; k < 8; k++) { int e = (v[i] - pal[k]) * (v[i] - pal[k]); if (e < be) { be = e; bk = k; } }
                bits |= (uint64_t)bk << (3 * i);
                err += be;
            }
            if (err < best) { best = err; ba0 = a0; ba1 = a1; bidx = bits; }
        }
    *oa0 = (uint8_t)ba0; *oa1 = (uint8_t)ba1; *oidx = bidx;
    return best;
}
static void bc4_store(uint8_t *o, const uint8_t v[16]) {
    uint8_t a0, a1;
    uint64_t idx;
    bc4_block(v, &a0, &a1, &idx);
    o[0] = a0; o[1] = a1; store_le(o + 2, idx, 6);
}

/* ================================================================== BC7 (zap_tex.h:308-784) */
/* BC7 mode descriptors (format spec): subsets, partition bits, rotation bits, index-selector bits, colour bits,
   alpha bits, per-endpoint p-bit, per-subset p-bit, index bits, secondary index bits */
typedef struct { int ns, pb, rb, isb, cb, ab, epb, spb, ib, ib2; } bc7_mode;
static const bc7_mode BC7_MODES[8] = {
    { 3, 4, 0, 0, 4, 0, 1, 0, 3, 0 }, { 2, 6, 0, 0, 6, 0, 0, 1, 3, 0 }, { 3, 6, 0, 0, 5, 0, 0, 0, 2, 0 },
    { 2, 6, 0, 0, 7, 0, 1, 0, 2, 0 }, { 1, 0, 2, 1, 5, 6, 0, 0, 2, 3 }, { 1, 0, 2, 0, 7, 8, 0, 0, 2, 2 },
    { 1, 0, 0, 0, 7, 7, 1, 0, 4, 0 }, { 2, 6, 0, 0, 5, 5, 1, 0, 2, 0 } };
/* two-subset partitions (format spec): bit i set = texel i in subset 1 */
static const uint16_t BC7_P2[64] = {
    0xCCCC, 0x8888, 0xEEEE, 0xECC8, 0xC880, 0xFEEC, 0xFEC8, 0xEC80, 0xC800, 0xFFEC, 0xFE80, 0xE800, 0xFFE8, 0xFF00, 0xFFF0, 0xF000,
    0xF710, 0x008E, 0x7100, 0x08CE, 0x008C, 0x7310, 0x3100, 0x8CCE, 0x088C, 0x3110, 0x6666, 0x366C, 0x17E8, 0x0FF0, 0x718E, 0x399C,
    0xAAAA, 0xF0F0, 0x5A5A, 0x33CC, 0x3C3C, 0x55AA, 0x9696, 0xA55A, 0x73CE, 0x13C8, 0x324C, 0x3BDC, 0x6996, 0xC33C, 0x9966, 0x0660,
    0x0272, 0x04E4, 0x4E40, 0x2720, 0xC936, 0x936C, 0x39C6, 0x639C, 0x9336, 0x9CC6, 0x817E, 0xE718, 0xCCF0, 0x0FCC, 0x7744, 0xEE22 };
/* three-subset partitions (format spec), one row of 16 subset digits per partition, texel 0 first */
static const char *const BC7_P3_ROWS[64] = {
    "0011001102212222", "0001001122112221", "0000200122112211", "0222002200110111", "0000000011221122", "0011001100220022",
    "0022002211111111", "0011001122112211", "0000000011112222", "0000111111112222", "0000111122222222", "0012001200120012",
    "0112011201120112", "0122012201220122", "0011011211221222", "0011200122002220", "0001001101121122", "0111001120012200",
    "0000112211221122", "0022002200221111", "0111011102220222", "0001000122212221", "0000001101220122", "0000110022102210",
    "0122012200110000", "0012001211222222", "0110122112210110", "0000011012211221", "0022110211020022", "0110011020022222",
    "0011012201220011", "0000200022112221", "0000000211221222", "0222002200120011", "0011001200220222", "0120012001200120",
    "0000111122220000", "0120120120120120", "0120201212010120", "0011220011220011", "0011112222000011", "0101010122222222",
    "0000000021212121", "0022112200221122", "0022001100220011", "0220122102201221", "0101222222220101", "0000212121212121",
    "0101010101012222", "0222011102220111", "0002111200021112", "0000211221122112", "0222011101110222", "0002111211120002",
    "0110011001102222", "0000000021122112", "0110011022222222", "0022001100110022", "0022112211220022", "0000000000002112",
    "0002000100020001", "0222122202221222", "0101222222222222", "0111201122012220" };
/* anchor texel of subset 1 (two subsets) and of subsets 1 / 2 (three subsets) (format spec) */
static const uint8_t BC7_A2[64] = {
    15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 2, 8, 2, 2, 8, 8, 15, 2, 8, 2, 2, 8, 8, 2, 2,
    15, 15, 6, 8, 2, 8, 15, 15, 2, 8, 2, 2, 2, 15, 15, 6, 6, 2, 6, 8, 15, 15, 2, 2, 15, 15, 15, 15, 15, 2, 2, 15 };
static const uint8_t BC7_A3A[64] = {
    3, 3, 15, 15, 8, 3, 15, 15, 8, 8, 6, 6, 6, 5, 3, 3, 3, 3, 8, 15, 3, 3, 6, 10, 5, 8, 8, 6, 8, 5, 15, 15,
    8, 15, 3, 5, 6, 10, 8, 15, 15, 3, 15, 5, 15, 15, 15, 15, 3, 15, 5, 5, 5, 8, 5, 10, 5, 10, 8, 13, 15, 12, 3, 3 };
static const uint8_t BC7_A3B[64] = {
    15, 8, 8, 3, 15, 15, 3, 8, 15, 15, 15, 15, 15, 15, 15, 8, 15, 8, 15, 3, 15, 8, 15, 8, 3, 15, 6, 10, 15, 15, 10, 8,
    15, 3, 15, 10, 10, 8, 9, 10, 6, 15, 8, 15, 3, 6, 6, 8, 15, 3, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 3, 15, 15, 8 };
/* interpolation weights (format spec) */
static const int BC7_W2[4] = { 0, 21, 43, 64 }, BC7_W3[8] = { 0, 9, 18, 27, 37, 46, 55, 64 },
                 BC7_W4[16] = { 0, 4, 9, 13, 17, 21, 26, 30, 34, 38, 43, 47, 51, 55, 60, 64 };
static int bc7_weight(int bits, int i) { return bits == 2 ? BC7_W2[i] : bits == 3 ? BC7_W3[i] : BC7_W4[i]; }
static int bc7_subset_of(int ns, int part, int i) {
    if (ns == 1) return 0;
    if (ns == 2) return (BC7_P2[part] >> i) & 1;
    return BC7_P3_ROWS[part][i] - '0';
}
static int bc7_anchor_of(int ns, int part, int s) { return s == 0 ? 0 : ns == 2 ? BC7_A2[part] : s == 1 ? BC7_A3A[part] : BC7_A3B[part]; }
static int bc7_expand(int v, int n) { v <<= 8 - n; return v | (v >> n); } /* n-bit value -> 8 bits (:375) */
static int lerp64(int a, int b, int w) { return ((64 - w) * a + w * b + 32) >> 6; }

/* a block's fields (:378-412): mode (8 = reserved), subsets, partition, rotation, whether alpha has its own bits,
   the expanded 8-bit endpoints, and each texel's subset and colour / alpha interpolation weight (0..64) */
typedef struct { int mode, ns, part, rot, ab, ep[6][4], subset[16], cw[16], aw[16]; } bc7_fields;
static int bc7_parse(const uint8_t *blk, bc7_fields *F) {
    int mode = 0;
    while (mode < 8 && !((blk[0] >> mode) & 1)) mode++;
    memset(F, 0, sizeof *F);
    F->mode = mode;
    if (mode == 8) return 0;
    const bc7_mode *M = &BC7_MODES[mode];
    bitr r = { blk, mode + 1 };
    int part = (int)get_bits(&r, M->pb), rot = (int)get_bits(&r, M->rb), isb = (int)get_bits(&r, M->isb);
    int ne = 2 * M->ns, cb = M->cb, ab = M->ab;
    for (int c = 0; c < 3; c++) for (int e = 0; e < ne; e++) F->ep[e][c] = (int)get_bits(&r, cb);
    for (int e = 0; e < ne; e++) F->ep[e][3] = ab ? (int)get_bits(&r, ab) : 255;
    if (M->epb || M->spb) {
        for (int e = 0; e < ne; e++) {
            if (!M->epb && (e & 1)) continue; /* shared p-bit: read once per subset */
            int p = (int)get_bits(&r, 1), last = M->epb ? e : e + 1;
            for (int k = e; k <= last; k++) {
                for (int c = 0; c < 3; c++) F->ep[k][c] = (F->ep[k][c] << 1) | p;
                if (ab) F->ep[k][3] = (F->ep[k][3] << 1) | p;
            }
        }
        cb++;
        if (ab) ab++;
    }
    for (int e = 0; e < ne; e++) {
        for (int c = 0; c < 3; c++) F->ep[e][c] = bc7_expand(F->ep[e][c], cb);
        if (ab) F->ep[e][3] = bc7_expand(F->ep[e][3], ab);
    }
    int i1[16], i2[16] = { 0 };
    for (int i = 0; i < 16; i++) {
        int is_anchor = i == bc7_anchor_of(M->ns, part, bc7_subset_of(M->ns, part, i));
        i1[i] = (int)get_bits(&r, M->ib - is_anchor);
    }
    if (M->ib2) for (int i = 0; i < 16; i++) i2[i] = (int)get_bits(&r, M->ib2 - (i == 0));
    for (int i = 0; i < 16; i++) {
        F->subset[i] = bc7_subset_of(M->ns, part, i);
        F->cw[i] = (M->ib2 && isb) ? bc7_weight(M->ib2, i2[i]) : bc7_weight(M->ib, i1[i]);
        F->aw[i] = !M->ib2 ? F->cw[i] : isb ? bc7_weight(M->ib, i1[i]) : bc7_weight(M->ib2, i2[i]);
    }
    F->ns = M->ns; F->part = part; F->rot = rot; F->ab = M->ab > 0;
    return 1;
}

/* full decoder, all 8 modes; reserved mode decodes to transparent black (:378-417) */
static void bc7_decode_block(const uint8_t *blk, tx4 out[16]) {
    bc7_fields F;
    if (!bc7_parse(blk, &F)) { memset(out, 0, 64); return; }
    for (int i = 0; i < 16; i++) {
        int s = F.subset[i];
        for (int c = 0; c < 3; c++) out[i][c] = (uint8_t)lerp64(F.ep[2 * s][c], F.ep[2 * s + 1][c], F.cw[i]);
        out[i][3] = (uint8_t)lerp64(F.ep[2 * s][3], F.ep[2 * s + 1][3], F.aw[i]);
        if (F.rot) { uint8_t s2 = out[i][3]; out[i][3] = out[i][F.rot - 1]; out[i][F.rot - 1] = s2; }
    }
}
static int bc7_decoded_sse(const tx4 t[16], const uint8_t *blk) { /* :710-716 */
    tx4 d[16];
    int err = 0;
    bc7_decode_block(blk, d);
    for (int i = 0; i < 16; i++) for (int c = 0; c < 4; c++) { int x = t[i][c] - d[i][c]; err += x * x; }
    return err;
}

/* endpoint quantisation with a fixed p-bit: n total bits, low bit = p (:426-438) */
static int bc7_quant_pbit(const float *v, int nc, int n, int p, int *q, int *x8) {
    int err = 0, top = (1 << (n - 1)) - 1;
    for (int c = 0; c < nc; c++) {
        int g = (int)((v[c] / 255.0f * (float)((1 << n) - 1) - (float)p) / 2.0f + 0.5f), bq = 0, be = 1 << 30;
        for (int k = 0; k < 3; k++) {
            int tq = iclamp(around(g, k), 0, top);
            float d = (float)bc7_expand((tq << 1) | p, n) - v[c];
            if ((int)(d * d) < be) { be = (int)(d * d); bq = tq; }
        }
        q[c] = bq; x8[c] = bc7_expand((bq << 1) | p, n); err += be;
    }
    return err;
}

/* principal-axis endpoint estimate over a texel subset (:441-462); also used by ASTC */
static void pca_endpoints(const tx4 t[16], const int *sel, int cnt, int nc, float lo[4], float hi[4]) {
    float mu[4] = { 0, 0, 0, 0 }, C[4][4], ax[4] = { 1, 1, 1, 1 };
    memset(C, 0, sizeof C);
    for (int k = 0; k < cnt; k++) for (int c = 0; c < nc; c++) mu[c] += t[sel[k]][c] / (float)cnt;
    for (int k = 0; k < cnt; k++)
        for (int a = 0; a < nc; a++)
            for (int b = 0; b < nc; b++) C[a][b] += (t[sel[k]][a] - mu[a]) * (t[sel[k]][b] - mu[b]);
    for (int it = 0; it < 6; it++) {
        float nv[4] = { 0, 0, 0, 0 }, m = 0;
        for (int a = 0; a < nc; a++) {
            for (int b = 0; b < nc; b++) nv[a] += C[a][b] * ax[b];
            if (fabsf(nv[a]) > m) m = fabsf(nv[a]);
        }
        if (m < 1e-6f) break;
        for (int a = 0; a < nc; a++) ax[a] = nv[a] / m;
    }
    float n2 = 0, tl = 1e9f, th = -1e9f;
    for (int a = 0; a < nc; a++) n2 += ax[a] * ax[a];
    for (int k = 0; k < cnt; k++) {
        float s = 0;
        for (int c = 0; c < nc; c++) s += (t[sel[k]][c] - mu[c]) * ax[c];
        if (s < tl) tl = s;
        if (s > th) th = s;
    }
    for (int c = 0; c < nc; c++) { lo[c] = mu[c] + ax[c] * tl / n2; hi[c] = mu[c] + ax[c] * th / n2; }
    for (int c = nc; c < 4; c++) lo[c] = hi[c] = 255;
}

/* float endpoints -> best p-bits + quantised endpoints + indices for one subset (:466-486) */
static int bc7_subset_fit(const tx4 t[16], const int *sel, int cnt, int nc, int n, int ib, int shared_p,
                          const float lo[4], const float hi[4], int q[2][4], int pb[2], int *idx) {
    int best = 1 << 30, x8[2][4];
    for (int p0 = 0; p0 < 2; p0++)
        for (int p1 = 0; p1 < 2; p1++) {
            if (shared_p && p0 != p1) continue;
            int tq[2][4];
            int err = bc7_quant_pbit(lo, nc, n, p0, tq[0], x8[0]) + bc7_quant_pbit(hi, nc, n, p1, tq[1], x8[1]);
            if (err < best) { best = err; memcpy(q, tq, sizeof tq); pb[0] = p0; pb[1] = p1; }
        }
    for (int k = 0; k < 2; k++) for (int c = 0; c < nc; c++) x8[k][c] = bc7_expand((q[k][c] << 1) | pb[k], n);
    int pal[16][4], np = 1 << ib, err = 0;
    for (int j = 0; j < np; j++) for (int c = 0; c < nc; c++) pal[j][c] = lerp64(x8[0][c], x8[1][c], bc7_weight(ib, j));
    ZO_OPS(cnt * np * (3 * nc + 1));
    for (int k = 0; k < cnt; k++) {
        int bj = 0, be = 1 << 30;
        for (int j = 0; j < np; j++) {
            int d = 0;
            for (int c = 0; c < nc; c++) { int x = t[sel[k]][c] - pal[j][c]; d += x * x; }
            if (d < be) { be = d; bj = j; }
        }
        idx[k] = bj; err += be;
    }
    return err;
}

/* PCA start, fit, then up to two least-squares refits (:489-515) */
static int bc7_subset_encode(const tx4 t[16], const int *sel, int cnt, int nc, int n, int ib, int shared_p,
                             int q[2][4], int pb[2], int *idx) {
    float lo[4], hi[4];
    pca_endpoints(t, sel, cnt, nc, lo, hi);
    int err = bc7_subset_fit(t, sel, cnt, nc, n, ib, shared_p, lo, hi, q, pb, idx);
    for (int it = 0; it < 2 && err > 0; it++) {
        float aa = 0, ab = 0, bb = 0, sa[4] = { 0, 0, 0, 0 }, sb[4] = { 0, 0, 0, 0 };
        for (int k = 0; k < cnt; k++) {
            float w = bc7_weight(ib, idx[k]) / 64.0f, u = 1 - w;
            aa += u * u; ab += u * w; bb += w * w;
            for (int c = 0; c < nc; c++) { sa[c] += u * t[sel[k]][c]; sb[c] += w * t[sel[k]][c]; }
        }
        float det = aa * bb - ab * ab;
        if (det < 1e-6f && det > -1e-6f) break;
        float nlo[4], nhi[4];
        for (int c = 0; c < nc; c++) {
            nlo[c] = fclamp255((sa[c] * bb - sb[c] * ab) / det);
            nhi[c] = fclamp255((sb[c] * aa - sa[c] * ab) / det);
        }
        for (int c = nc; c < 4; c++) nlo[c] = nhi[c] = 255;
        int nq[2][4], npb[2], ni[16];
        int ne = bc7_subset_fit(t, sel, cnt, nc, n, ib, shared_p, nlo, nhi, nq, npb, ni);
        if (ne >= err) break;
        err = ne; memcpy(q, nq, sizeof nq); pb[0] = npb[0]; pb[1] = npb[1]; memcpy(idx, ni, sizeof(int) * (size_t)cnt);
    }
    return err;
}

/* mode 6: one subset RGBA, 7 bits + unique p-bit, 4-bit indices (:520-527, :582-593) */
static int bc7_mode6(const tx4 t[16], uint8_t out[16]) {
    int sel[16], q[2][4], pb[2], idx[16];
    for (int i = 0; i < 16; i++) sel[i] = i;
    int err = bc7_subset_encode(t, sel, 16, 4, 8, 4, 0, q, pb, idx);
    if (idx[0] & 8) { /* anchor MSB must be 0 */
        for (int c = 0; c < 4; c++) { int s = q[0][c]; q[0][c] = q[1][c]; q[1][c] = s; }
        int s = pb[0]; pb[0] = pb[1]; pb[1] = s;
        for (int i = 0; i < 16; i++) idx[i] = 15 - idx[i];
    }
    memset(out, 0, 16);
    bitw w = { out, 0 };
    put_bits(&w, 1u << 6, 7);
    for (int c = 0; c < 4; c++) for (int e = 0; e < 2; e++) put_bits(&w, (unsigned)q[e][c], 7);
    put_bits(&w, (unsigned)pb[0], 1); put_bits(&w, (unsigned)pb[1], 1);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)idx[i], i ? 4 : 3);
    return err;
}

/* mode 5 pieces (:597-657): 2-bit palettes on channels [c0, c0 + nc) */
static int m5_fit(const tx4 r[16], int c0, int nc, const int *e0, const int *e1, int idx[16]) {
    int pal[4][4], err = 0;
    for (int j = 0; j < 4; j++) for (int c = 0; c < nc; c++) pal[j][c] = lerp64(e0[c], e1[c], BC7_W2[j]);
    ZO_OPS(16 * 4 * (3 * nc + 1));
    for (int i = 0; i < 16; i++) {
        int bj = 0, be = 1 << 30;
        for (int j = 0; j < 4; j++) {
            int d = 0;
            for (int c = 0; c < nc; c++) { int x = r[i][c0 + c] - pal[j][c]; d += x * x; }
            if (d < be) { be = d; bj = j; }
        }
        idx[i] = bj; err += be;
    }
    return err;
}
static void m5_quant(const float *v, int nc, int n, int *q, int *x8) { /* no p-bit; nearest by truncated |diff| */
    int top = (1 << n) - 1;
    for (int c = 0; c < nc; c++) {
        int g = (int)(v[c] * (float)top / 255.0f + 0.5f), bq = 0, bd = 1 << 30;
        for (int k = 0; k < 3; k++) {
            int tq = iclamp(around(g, k), 0, top);
            float diff = (float)bc7_expand(tq, n) - v[c];
            int d = (int)(diff < 0 ? v[c] - (float)bc7_expand(tq, n) : diff);
            if (d < bd) { bd = d; bq = tq; }
        }
        q[c] = bq; x8[c] = bc7_expand(bq, n);
    }
}
static int m5_lsq(const tx4 r[16], int c0, int nc, const int idx[16], float lo[4], float hi[4]) {
    float aa = 0, ab = 0, bb = 0, sa[4] = { 0, 0, 0, 0 }, sb[4] = { 0, 0, 0, 0 };
    for (int i = 0; i < 16; i++) {
        float w = BC7_W2[idx[i]] / 64.0f, u = 1 - w;
        aa += u * u; ab += u * w; bb += w * w;
        for (int c = 0; c < nc; c++) { sa[c] += u * r[i][c0 + c]; sb[c] += w * r[i][c0 + c]; }
    }
    float det = aa * bb - ab * ab;
    if (det < 1e-6f && det > -1e-6f) return 0;
    for (int c = 0; c < nc; c++) { lo[c] = fclamp255((sa[c] * bb - sb[c] * ab) / det); hi[c] = fclamp255((sb[c] * aa - sa[c] * ab) / det); }
    return 1;
}
static int m5_part(const tx4 r[16], int c0, int nc, int n, float lo[4], float hi[4], int q[2][3], int idx[16]) {
    int x0[3], x1[3];
    m5_quant(lo, nc, n, q[0], x0); m5_quant(hi, nc, n, q[1], x1);
    int err = m5_fit(r, c0, nc, x0, x1, idx);
    for (int it = 0; it < 2 && err > 0; it++) {
        float nlo[4], nhi[4];
        int tq[2][3], ti[16];
        if (!m5_lsq(r, c0, nc, idx, nlo, nhi)) break;
        m5_quant(nlo, nc, n, tq[0], x0); m5_quant(nhi, nc, n, tq[1], x1);
        int e = m5_fit(r, c0, nc, x0, x1, ti);
        if (e >= err) break;
        err = e; memcpy(q, tq, sizeof tq); memcpy(idx, ti, sizeof ti);
    }
    return err;
}
/* mode 5: rotation x (RGB 7-bit + A 8-bit), separate 2-bit colour / alpha indices (:659-684) */
static void bc7_mode5(const tx4 t[16], uint8_t out[16]) {
    int best = 1 << 30, brot = 0, bcq[2][3] = { { 0 } }, baq[2][3] = { { 0 } }, bci[16] = { 0 }, bai[16] = { 0 };
    for (int rot = 0; rot < 4; rot++) {
        tx4 r[16];
        int sel[16], cq[2][3], aq[2][3], ci[16], ai[16];
        memcpy(r, t, sizeof r);
        for (int i = 0; i < 16; i++) {
            sel[i] = i;
            if (rot) { uint8_t s = r[i][3]; r[i][3] = r[i][rot - 1]; r[i][rot - 1] = s; }
        }
        float lo[4], hi[4], alo[4] = { 255, 0, 0, 0 }, ahi[4] = { 0, 0, 0, 0 };
        pca_endpoints((const tx4 *)r, sel, 16, 3, lo, hi);
        int err = m5_part((const tx4 *)r, 0, 3, 7, lo, hi, cq, ci);
        for (int i = 0; i < 16; i++) { if (r[i][3] < alo[0]) alo[0] = r[i][3]; if (r[i][3] > ahi[0]) ahi[0] = r[i][3]; }
        err += m5_part((const tx4 *)r, 3, 1, 8, alo, ahi, aq, ai);
        if (err < best) {
            best = err; brot = rot;
            memcpy(bcq, cq, sizeof cq); memcpy(baq, aq, sizeof aq); memcpy(bci, ci, sizeof ci); memcpy(bai, ai, sizeof ai);
        }
    }
    if (bci[0] & 2) { for (int c = 0; c < 3; c++) { int s = bcq[0][c]; bcq[0][c] = bcq[1][c]; bcq[1][c] = s; } for (int i = 0; i < 16; i++) bci[i] = 3 - bci[i]; }
    if (bai[0] & 2) { int s = baq[0][0]; baq[0][0] = baq[1][0]; baq[1][0] = s; for (int i = 0; i < 16; i++) bai[i] = 3 - bai[i]; }
    memset(out, 0, 16);
    bitw w = { out, 0 };
    put_bits(&w, 1u << 5, 6);
    put_bits(&w, (unsigned)brot, 2);
    for (int c = 0; c < 3; c++) for (int e = 0; e < 2; e++) put_bits(&w, (unsigned)bcq[e][c], 7);
    for (int e = 0; e < 2; e++) put_bits(&w, (unsigned)baq[e][0], 8);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)bci[i], i ? 2 : 1);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)bai[i], i ? 2 : 1);
}

/* mode 1: two subsets, RGB 6 bits + shared p-bit, 3-bit indices; out == NULL returns the fit SSE only (:687-708) */
static int bc7_mode1(const tx4 t[16], int part, uint8_t *out) {
    int sel[2][16], cnt[2] = { 0, 0 }, q[2][2][4], pb[2][2], idx[2][16], err = 0, full[16];
    for (int i = 0; i < 16; i++) { int s = (BC7_P2[part] >> i) & 1; sel[s][cnt[s]++] = i; }
    for (int s = 0; s < 2; s++) err += bc7_subset_encode(t, sel[s], cnt[s], 3, 7, 3, 1, q[s], pb[s], idx[s]);
    if (!out) return err;
    for (int s = 0; s < 2; s++) {
        for (int k = 0; k < cnt[s]; k++) full[sel[s][k]] = idx[s][k];
        int anchor = s ? BC7_A2[part] : 0;
        if (full[anchor] & 4) {
            for (int c = 0; c < 3; c++) { int x = q[s][0][c]; q[s][0][c] = q[s][1][c]; q[s][1][c] = x; }
            for (int k = 0; k < cnt[s]; k++) full[sel[s][k]] = 7 - full[sel[s][k]];
        }
    }
    memset(out, 0, 16);
    bitw w = { out, 0 };
    put_bits(&w, 2, 2);
    put_bits(&w, (unsigned)part, 6);
    for (int c = 0; c < 3; c++) for (int s = 0; s < 2; s++) for (int e = 0; e < 2; e++) put_bits(&w, (unsigned)q[s][e][c], 6);
    put_bits(&w, (unsigned)pb[0][0], 1); put_bits(&w, (unsigned)pb[1][0], 1);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)full[i], 3 - (i == 0 || i == BC7_A2[part]));
    return err;
}

/* cheap partition score from per-texel moments {r,g,b,rr,gg,bb,rg,rb,gb} (:722-748) */
static float bc7_partition_score(const float mo[16][9], const float tot[9], int part) {
    float s[2][9];
    int n1 = 0;
    for (int j = 0; j < 9; j++) s[1][j] = 0;
    for (int i = 0; i < 16; i++)
        if ((BC7_P2[part] >> i) & 1) { n1++; for (int j = 0; j < 9; j++) s[1][j] += mo[i][j]; }
    ZO_OPS(9 * n1);
    for (int j = 0; j < 9; j++) s[0][j] = tot[j] - s[1][j];
    float score = 0;
    for (int k = 0; k < 2; k++) {
        float n = (float)(k ? n1 : 16 - n1), *m = s[k];
        if (n < 2) continue;
        float S[3][3];
        S[0][0] = m[3] - m[0] * m[0] / n; S[0][1] = m[6] - m[0] * m[1] / n; S[0][2] = m[7] - m[0] * m[2] / n;
        S[1][1] = m[4] - m[1] * m[1] / n; S[1][2] = m[8] - m[1] * m[2] / n; S[2][2] = m[5] - m[2] * m[2] / n;
        S[1][0] = S[0][1]; S[2][0] = S[0][2]; S[2][1] = S[1][2];
        float tr = S[0][0] + S[1][1] + S[2][2], ax[3];
        int r0 = (S[0][0] >= S[1][1] && S[0][0] >= S[2][2]) ? 0 : S[1][1] >= S[2][2] ? 1 : 2;
        for (int c = 0; c < 3; c++) ax[c] = S[r0][c];
        for (int it = 0; it < 3; it++) {
            float v[3], mx = 1e-12f;
            for (int c = 0; c < 3; c++) {
                v[c] = S[c][0] * ax[0] + S[c][1] * ax[1] + S[c][2] * ax[2];
                mx = v[c] > mx ? v[c] : -v[c] > mx ? -v[c] : mx;
            }
            for (int c = 0; c < 3; c++) ax[c] = v[c] / mx;
        }
        float vv = ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2], vsv = 0;
        for (int c = 0; c < 3; c++) vsv += ax[c] * (S[c][0] * ax[0] + S[c][1] * ax[1] + S[c][2] * ax[2]);
        float lam = vv > 1e-12f ? vsv / vv : 0;
        score += tr - lam * (48.0f / 49.0f);
    }
    return score;
}

#define BC7_MODE1_TRIES 4 /* ZAP__BC7_M1K default (zap_tex.h:750-752) */

/* mode 6, early exit at SSE <= 64, then mode 5, then (opaque) mode 1 over the best-scored partitions (:755-784) */
static int bc7_block(const tx4 t[16], uint8_t out[16]) { /* returns the SSE of the block it wrote, as :755-784 */
#ifdef ZO_COUNT_OPS
    const uint64_t ops0 = g_ops[0];
#endif
    int err = bc7_mode6(t, out), opaque = 1;
#ifdef ZO_COUNT_OPS
    g_ops[1] += g_ops[0] - ops0;
#endif
    for (int i = 0; i < 16; i++) opaque &= t[i][3] == 255;
    if (err <= 16 * 4) return err;
    uint8_t m5[16];
    bc7_mode5(t, m5);
    int e5 = bc7_decoded_sse(t, m5);
    if (e5 < err) { memcpy(out, m5, 16); err = e5; }
    if (!opaque) return err;
    float mo[16][9], tot[9] = { 0 }, ce[BC7_MODE1_TRIES];
    int cand[BC7_MODE1_TRIES], bp = -1, be = err;
    for (int i = 0; i < 16; i++) {
        float r = t[i][0], g = t[i][1], b = t[i][2], v[9] = { r, g, b, r * r, g * g, b * b, r * g, r * b, g * b };
        for (int j = 0; j < 9; j++) { mo[i][j] = v[j]; tot[j] += v[j]; }
    }
    for (int j = 0; j < BC7_MODE1_TRIES; j++) { ce[j] = 1e30f; cand[j] = -1; }
    for (int part = 0; part < 64; part++) {
        float e = bc7_partition_score((const float(*)[9])mo, tot, part);
        for (int j = 0; j < BC7_MODE1_TRIES; j++)
            if (e < ce[j]) {
                for (int k = BC7_MODE1_TRIES - 1; k > j; k--) { ce[k] = ce[k - 1]; cand[k] = cand[k - 1]; }
                ce[j] = e; cand[j] = part;
                break;
            }
    }
    /* an unfilled slot (cand -1) would index the partition table out of bounds in the reference; skip it */
    for (int j = 0; j < BC7_MODE1_TRIES; j++) {
        if (cand[j] < 0) continue;
        int e = bc7_mode1(t, cand[j], NULL);
        if (e < be) { be = e; bp = cand[j]; }
    }
    if (bp >= 0) {
        uint8_t m1[16];
        bc7_mode1(t, bp, m1);
        int e1 = bc7_decoded_sse(t, m1);
        if (e1 < err) { memcpy(out, m1, 16); err = e1; }
    }
    return err;
}

/* ================================================================== RDO (zap_tex.h:223-306, :786-815)
 * With lambda > 0 each sub-block is picked among its own encoding and candidates rebuilt from the 16 blocks before
 * it in the call's raster order (the bytes already chosen for them), minimising SSE + lambda * rate. A field's rate
 * models zap's LZ on the split planes: 0 if it repeats the field at the current match distance, min(size, 3) if it
 * repeats one elsewhere in the window (a new match), else its size in literals. The choice is a sequential scan
 * with strict "<", so the first candidate of the lowest cost wins. */
#define RDO_WINDOW 16
typedef struct { int dist[2]; } rdo_state; /* current match distance of each field, per sub-block kind */

static float rdo_rate(const uint8_t *f, int n, const uint8_t *base, size_t cur, size_t stride, size_t off, int dist, int *nd) {
    *nd = dist;
    if (dist > 0 && (size_t)dist <= cur && memcmp(f, base + (cur - (size_t)dist) * stride + off, (size_t)n) == 0) return 0.0f;
    for (size_t j = 1; j <= RDO_WINDOW && j <= cur; j++)
        if (memcmp(f, base + (cur - j) * stride + off, (size_t)n) == 0) { *nd = (int)j; return n < 3 ? (float)n : 3.0f; }
    return (float)n;
}

/* BC1 palette for any endpoint order (:52-62): 3 colours + transparent black when c0 <= c1 and not force4 */
static int bc1_palette(uint16_t c0, uint16_t c1, int force4, int pal[4][3]) {
    int a[3], b[3], four = force4 || c0 > c1;
    unpack565(c0, a); unpack565(c1, b);
    for (int k = 0; k < 3; k++) {
        pal[0][k] = a[k]; pal[1][k] = b[k];
        pal[2][k] = four ? (2 * a[k] + b[k] + 1) / 3 : (a[k] + b[k] + 1) / 2;
        pal[3][k] = four ? (a[k] + 2 * b[k] + 1) / 3 : 0;
    }
    return four ? 4 : 3;
}
static int bc1_fit_any(const tx4 t[16], uint16_t c0, uint16_t c1, int force4, uint32_t *idx) { /* :66-77 */
    int pal[4][3], n = bc1_palette(c0, c1, force4, pal), err = 0;
    uint32_t bits = 0;
    for (int i = 0; i < 16; i++) {
        int bk = 0, be = d3(t[i], pal[0]);
        for (int k = 1; k < n; k++) { int e = d3(t[i], pal[k]); if (e < be) { be = e; bk = k; } }
        bits |= (uint32_t)bk << (2 * i);
        err += be;
    }
    *idx = bits;
    return err;
}
static int bc1_eval_idx(const tx4 t[16], uint16_t c0, uint16_t c1, int force4, uint32_t idx) { /* :79-84 */
    int pal[4][3], err = 0;
    bc1_palette(c0, c1, force4, pal);
    for (int i = 0; i < 16; i++) err += d3(t[i], pal[(idx >> (2 * i)) & 3]);
    return err;
}

static void bc1_rdo(const tx4 t[16], int force4, float lambda, uint8_t *base, size_t cur, size_t stride, size_t off, rdo_state *rs) {
    uint16_t c0, c1;
    uint32_t idx;
    const int e0 = bc1_block(t, &c0, &c1, &idx);
    uint8_t best[8], cand[8];
    bc1_store(best, c0, c1, idx);
    if (lambda > 0) {
        int bd0 = 0, bd1 = 0, d0, d1;
        float bj = (float)e0 + lambda * (rdo_rate(best, 4, base, cur, stride, off, rs->dist[0], &bd0) +
                                         rdo_rate(best + 4, 4, base, cur, stride, off + 4, rs->dist[1], &bd1));
        for (size_t j = 1; j <= RDO_WINDOW && j <= cur; j++) {
            const uint8_t *prev = base + (cur - j) * stride + off;
            const uint16_t p0 = (uint16_t)load_le(prev, 2), p1 = (uint16_t)load_le(prev + 2, 2);
            const uint32_t pi = (uint32_t)load_le(prev + 4, 4);
            for (int kind = 0; kind < 3; kind++) {
                int e;
                uint32_t fi;
                if (kind == 0) { e = bc1_fit_any(t, p0, p1, force4, &fi); bc1_store(cand, p0, p1, fi); } /* its endpoints */
                else if (kind == 1) { e = bc1_eval_idx(t, c0, c1, force4, pi); bc1_store(cand, c0, c1, pi); } /* its indices */
                else { e = bc1_eval_idx(t, p0, p1, force4, pi); memcpy(cand, prev, 8); } /* the whole block */
                if (!force4 && load_le(cand, 2) <= load_le(cand + 2, 2)) { /* 3-colour block: index 3 would be transparent */
                    const uint32_t ci = (uint32_t)load_le(cand + 4, 4);
                    int transparent = 0;
                    for (int i = 0; i < 16; i++) transparent |= ((ci >> (2 * i)) & 3) == 3;
                    if (transparent) continue;
                }
                float jj = (float)e;
                if (jj >= bj) continue;
                jj += lambda * (rdo_rate(cand, 4, base, cur, stride, off, rs->dist[0], &d0) +
                                rdo_rate(cand + 4, 4, base, cur, stride, off + 4, rs->dist[1], &d1));
                if (jj < bj) { bj = jj; memcpy(best, cand, 8); bd0 = d0; bd1 = d1; }
            }
        }
        rs->dist[0] = bd0; rs->dist[1] = bd1;
    }
    memcpy(base + cur * stride + off, best, 8);
}

static int bc4_fit_any(const uint8_t v[16], int a0, int a1, uint64_t *idx) { /* :178-189 */
    int pal[8], err = 0;
    uint64_t bits = 0;
    bc4_pal(a0, a1, pal);
    for (int i = 0; i < 16; i++) {
        int bk = 0, be = (v[i] - pal[0]) * (v[i] - pal[0]);
        for (int k = 1; k < 8; k++) { int e = (v[i] - pal[k]) * (v[i] - pal[k]); if (e < be) { be = e; bk = k; } }
        bits |= (uint64_t)bk << (3 * i);
        err += be;
    }
    *idx = bits;
    return err;
}
static int bc4_eval_idx(const uint8_t v[16], int a0, int a1, uint64_t idx) { /* :191-196 */
    int pal[8], err = 0;
    bc4_pal(a0, a1, pal);
    for (int i = 0; i < 16; i++) { int d = v[i] - pal[(idx >> (3 * i)) & 7]; err += d * d; }
    return err;
}
static void bc4_put(uint8_t *o, int a0, int a1, uint64_t idx) { o[0] = (uint8_t)a0; o[1] = (uint8_t)a1; store_le(o + 2, idx, 6); }

static void bc4_rdo(const uint8_t v[16], float lambda, uint8_t *base, size_t cur, size_t stride, size_t off, rdo_state *rs) {
    uint8_t a0, a1, best[8], cand[8];
    uint64_t idx;
    const int e0 = bc4_block(v, &a0, &a1, &idx);
    bc4_put(best, a0, a1, idx);
    if (lambda > 0) {
        int bd0 = 0, bd1 = 0, d0, d1;
        float bj = (float)e0 + lambda * (rdo_rate(best, 2, base, cur, stride, off, rs->dist[0], &bd0) +
                                         rdo_rate(best + 2, 6, base, cur, stride, off + 2, rs->dist[1], &bd1));
        for (size_t j = 1; j <= RDO_WINDOW && j <= cur; j++) {
            const uint8_t *prev = base + (cur - j) * stride + off;
            const uint64_t pi = load_le(prev + 2, 6);
            for (int kind = 0; kind < 3; kind++) {
                int e;
                uint64_t fi;
                if (kind == 0) { e = bc4_fit_any(v, prev[0], prev[1], &fi); bc4_put(cand, prev[0], prev[1], fi); }
                else if (kind == 1) { e = bc4_eval_idx(v, a0, a1, pi); bc4_put(cand, a0, a1, pi); }
                else { e = bc4_eval_idx(v, prev[0], prev[1], pi); memcpy(cand, prev, 8); }
                float jj = (float)e;
                if (jj >= bj) continue;
                jj += lambda * (rdo_rate(cand, 2, base, cur, stride, off, rs->dist[0], &d0) +
                                rdo_rate(cand + 2, 6, base, cur, stride, off + 2, rs->dist[1], &d1));
                if (jj < bj) { bj = jj; memcpy(best, cand, 8); bd0 = d0; bd1 = d1; }
            }
        }
        rs->dist[0] = bd0; rs->dist[1] = bd1;
    }
    memcpy(base + cur * stride + off, best, 8);
}

/* BC7 mode 6 pieces for RDO (:529-580): bytes 0-7 hold mode + endpoints, byte 8 straddles, bytes 9-15 indices */
static int bc7_is_mode6(const uint8_t *b) { return (b[0] & 0x7F) == 0x40; }
static void bc7_unpack_mode6(const uint8_t *b, int q[2][4], int pb[2], int idx[16]) {
    bitr r = { b, 7 };
    for (int c = 0; c < 4; c++) for (int e = 0; e < 2; e++) q[e][c] = (int)get_bits(&r, 7);
    pb[0] = (int)get_bits(&r, 1); pb[1] = (int)get_bits(&r, 1);
    for (int i = 0; i < 16; i++) idx[i] = (int)get_bits(&r, i ? 4 : 3);
}
static void bc7_pack_mode6(int q[2][4], const int pb[2], const int idx[16], uint8_t out[16]) {
    memset(out, 0, 16);
    bitw w = { out, 0 };
    put_bits(&w, 1u << 6, 7);
    for (int c = 0; c < 4; c++) for (int e = 0; e < 2; e++) put_bits(&w, (unsigned)q[e][c], 7);
    put_bits(&w, (unsigned)pb[0], 1); put_bits(&w, (unsigned)pb[1], 1);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)idx[i], i ? 4 : 3);
}
static void bc7_palette6(int q[2][4], const int pb[2], int pal[16][4]) {
    int x[2][4];
    for (int k = 0; k < 2; k++) for (int c = 0; c < 4; c++) x[k][c] = bc7_expand((q[k][c] << 1) | pb[k], 8);
    for (int j = 0; j < 16; j++) for (int c = 0; c < 4; c++) pal[j][c] = lerp64(x[0][c], x[1][c], BC7_W4[j]);
}
static int d4(const uint8_t *p, const int *q) { int s = 0; for (int c = 0; c < 4; c++) { int x = p[c] - q[c]; s += x * x; } return s; }
/* indices for given endpoints; texel 0 keeps to 0..7 so the block needs no anchor swap (:544-555) */
static int bc7_mode6_fit_indices(const tx4 t[16], int q[2][4], const int pb[2], int idx[16]) {
    int pal[16][4], err = 0;
    bc7_palette6(q, pb, pal);
    for (int i = 0; i < 16; i++) {
        int bj = 0, be = 1 << 30;
        for (int j = 0; j < (i ? 16 : 8); j++) { int d = d4(t[i], pal[j]); if (d < be) { be = d; bj = j; } }
        idx[i] = bj; err += be;
    }
    return err;
}
/* endpoints for given indices: least squares, then each endpoint's own best p-bit (:557-580) */
static int bc7_mode6_fit_endpoints(const tx4 t[16], const int idx[16], int q[2][4], int pb[2]) {
    float aa = 0, ab = 0, bb = 0, sa[4] = { 0, 0, 0, 0 }, sb[4] = { 0, 0, 0, 0 }, lo[4], hi[4];
    for (int i = 0; i < 16; i++) {
        float w = BC7_W4[idx[i]] / 64.0f, u = 1 - w;
        aa += u * u; ab += u * w; bb += w * w;
        for (int c = 0; c < 4; c++) { sa[c] += u * t[i][c]; sb[c] += w * t[i][c]; }
    }
    float det = aa * bb - ab * ab;
    for (int c = 0; c < 4; c++) {
        if (det < 1e-6f && det > -1e-6f) lo[c] = hi[c] = (sa[c] + sb[c]) / 16.0f; /* one index everywhere */
        else { lo[c] = (sa[c] * bb - sb[c] * ab) / det; hi[c] = (sb[c] * aa - sa[c] * ab) / det; }
        lo[c] = fclamp255(lo[c]); hi[c] = fclamp255(hi[c]);
    }
    int x0[4], x1[4], t0[4], t1[4], b0 = 1 << 30, b1 = 1 << 30;
    for (int p = 0; p < 2; p++) {
        int e0 = bc7_quant_pbit(lo, 4, 8, p, t0, x0), e1 = bc7_quant_pbit(hi, 4, 8, p, t1, x1);
        if (e0 < b0) { b0 = e0; memcpy(q[0], t0, sizeof t0); pb[0] = p; }
        if (e1 < b1) { b1 = e1; memcpy(q[1], t1, sizeof t1); pb[1] = p; }
    }
    int pal[16][4], err = 0;
    bc7_palette6(q, pb, pal);
    for (int i = 0; i < 16; i++) err += d4(t[i], pal[idx[i]]);
    return err;
}
static float bc7_rdo_rate(const uint8_t *c, const uint8_t *base, size_t cur, const rdo_state *rs, int d[2]) { /* :788-790 */
    return rdo_rate(c, 8, base, cur, 16, 0, rs->dist[0], &d[0]) + rdo_rate(c + 9, 7, base, cur, 16, 9, rs->dist[1], &d[1]) + 1;
}
static void bc7_rdo(const tx4 t[16], float lambda, uint8_t *base, size_t cur, rdo_state *rs) {
    uint8_t best[16], cand[16];
    const int e0 = bc7_block(t, best);
    if (lambda > 0) {
        int bd[2] = { 0, 0 }, d[2];
        float bj = (float)e0 + lambda * bc7_rdo_rate(best, base, cur, rs, bd);
        for (size_t j = 1; j <= RDO_WINDOW && j <= cur; j++) {
            const uint8_t *prev = base + (cur - j) * 16;
            int pq[2][4], ppb[2], pidx[16], nq[2][4], npb[2], nidx[16];
            const int six = bc7_is_mode6(prev);
            if (six) bc7_unpack_mode6(prev, pq, ppb, pidx);
            for (int kind = 0; kind < (six ? 3 : 1); kind++) {
                int e;
                if (kind == 0) { e = bc7_decoded_sse(t, prev); memcpy(cand, prev, 16); }
                else if (kind == 1) { e = bc7_mode6_fit_indices(t, pq, ppb, nidx); bc7_pack_mode6(pq, ppb, nidx, cand); }
                else { e = bc7_mode6_fit_endpoints(t, pidx, nq, npb); bc7_pack_mode6(nq, npb, pidx, cand); }
                if ((float)e >= bj) continue;
                float jj = (float)e + lambda * bc7_rdo_rate(cand, base, cur, rs, d);
                if (jj < bj) { bj = jj; memcpy(best, cand, 16); bd[0] = d[0]; bd[1] = d[1]; }
            }
        }
        rs->dist[0] = bd[0]; rs->dist[1] = bd[1];
    }
    memcpy(base + cur * 16, best, 16);
}

/* ================================================================== public BC entry (zap_tex.h:1474-1506) */
size_t zo_bc_size(int w, int h, int fmt) { return (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4) * (fmt == ZO_BC1 || fmt == ZO_BC4 ? 8u : 16u); }

int zo_bc_encode(const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, void *out_) {
    if (fmt < 0 || fmt > 4) return -1;
    uint8_t *out = (uint8_t *)out_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    size_t bs = (fmt == ZO_BC1 || fmt == ZO_BC4) ? 8 : 16;
    if (rdo > 0) { /* one chain over the call's blocks in raster order; a match state per sub-block kind */
        rdo_state rs[2] = { { { 1, 1 } }, { { 1, 1 } } };
        for (int by = 0; by < bh; by++)
            for (int bx = 0; bx < bw; bx++) {
                tx4 t[16];
                uint8_t ch[2][16];
                const size_t cur = (size_t)by * (size_t)bw + (size_t)bx;
                gather8(rgba, w, h, stride, bx, by, t);
                if (fmt == ZO_BC1) bc1_rdo((const tx4 *)t, 0, rdo, out, cur, bs, 0, &rs[0]);
                else if (fmt == ZO_BC3) {
                    for (int i = 0; i < 16; i++) ch[0][i] = t[i][3];
                    bc4_rdo(ch[0], rdo, out, cur, bs, 0, &rs[0]);
                    bc1_rdo((const tx4 *)t, 1, rdo, out, cur, bs, 8, &rs[1]);
                } else if (fmt == ZO_BC4 || fmt == ZO_BC5) {
                    for (int i = 0; i < 16; i++) { ch[0][i] = t[i][0]; ch[1][i] = t[i][1]; }
                    bc4_rdo(ch[0], rdo, out, cur, bs, 0, &rs[0]);
                    if (fmt == ZO_BC5) bc4_rdo(ch[1], rdo, out, cur, bs, 8, &rs[1]);
                } else {
                    bc7_rdo((const tx4 *)t, rdo, out, cur, &rs[0]);
                }
            }
        return 0;
    }
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            tx4 t[16];
            uint8_t ch[16];
            uint8_t *o = out + ((size_t)by * (size_t)bw + (size_t)bx) * bs;
            gather8(rgba, w, h, stride, bx, by, t);
            if (fmt == ZO_BC1 || fmt == ZO_BC3) {
                uint16_t c0, c1;
                uint32_t idx;
                if (fmt == ZO_BC3) { for (int i = 0; i < 16; i++) ch[i] = t[i][3]; bc4_store(o, ch); }
                bc1_block((const tx4 *)t, &c0, &c1, &idx);
                bc1_store(o + (fmt == ZO_BC3 ? 8 : 0), c0, c1, idx);
            } else if (fmt == ZO_BC4 || fmt == ZO_BC5) {
                for (int i = 0; i < 16; i++) ch[i] = t[i][0];
                bc4_store(o, ch);
                if (fmt == ZO_BC5) { for (int i = 0; i < 16; i++) ch[i] = t[i][1]; bc4_store(o + 8, ch); }
            } else {
                bc7_block((const tx4 *)t, o);
            }
        }
    return 0;
}

static void bc1_decode_block(const uint8_t *b, int four_always, tx4 out[16]) { /* :1508-1517 */
    uint16_t c0 = (uint16_t)load_le(b, 2), c1 = (uint16_t)load_le(b + 2, 2);
    int pal[4][3], four = four_always || c0 > c1;
    unpack565(c0, pal[0]); unpack565(c1, pal[1]);
    for (int k = 0; k < 3; k++) {
        int a = pal[0][k], c = pal[1][k];
        pal[2][k] = four ? (2 * a + c + 1) / 3 : (a + c + 1) / 2;
        pal[3][k] = four ? (a + 2 * c + 1) / 3 : 0;
    }
    uint32_t idx = (uint32_t)load_le(b + 4, 4);
    for (int i = 0; i < 16; i++) {
        int k = (idx >> (2 * i)) & 3;
        for (int c = 0; c < 3; c++) out[i][c] = (uint8_t)pal[k][c];
        out[i][3] = (uint8_t)(!four && k == 3 ? 0 : 255);
    }
}
static void bc4_decode_block(const uint8_t *b, uint8_t v[16]) {
    int pal[8];
    bc4_pal(b[0], b[1], pal);
    uint64_t idx = load_le(b + 2, 6);
    for (int i = 0; i < 16; i++) v[i] = (uint8_t)pal[(idx >> (3 * i)) & 7];
}

void zo_bc_decode(const void *bc_, int w, int h, int fmt, uint8_t *rgba, size_t stride) {
    const uint8_t *bc = (const uint8_t *)bc_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    size_t bs = (fmt == ZO_BC1 || fmt == ZO_BC4) ? 8 : 16;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const uint8_t *b = bc + ((size_t)by * (size_t)bw + (size_t)bx) * bs;
            tx4 px[16];
            uint8_t v0[16], v1[16];
            if (fmt == ZO_BC1) bc1_decode_block(b, 0, px);
            else if (fmt == ZO_BC7) bc7_decode_block(b, px);
            else if (fmt == ZO_BC3) { bc1_decode_block(b + 8, 1, px); bc4_decode_block(b, v0); for (int i = 0; i < 16; i++) px[i][3] = v0[i]; }
            else {
                bc4_decode_block(b, v0);
                if (fmt == ZO_BC5) bc4_decode_block(b + 8, v1); else memset(v1, 0, 16);
                for (int i = 0; i < 16; i++) { px[i][0] = v0[i]; px[i][1] = v1[i]; px[i][2] = 0; px[i][3] = 255; }
            }
            for (int i = 0; i < 16; i++) {
                int x = bx * 4 + (i & 3), y = by * 4 + (i >> 2);
                if (x < w && y < h) memcpy(rgba + (size_t)y * stride + (size_t)x * 4, px[i], 4);
            }
        }
}

/* split / merge (:1549-1571): plane k holds field k of every block, fields in block order; the planes follow one
 * another, and bytes after the last whole block are copied unchanged */
static int bc_fields(int fmt, int sz[4]) {
    static const int F[5][5] = { { 2, 4, 4 }, { 4, 2, 6, 4, 4 }, { 2, 2, 6 }, { 4, 2, 6, 2, 6 }, { 3, 8, 1, 7 } };
    for (int k = 0; k < F[fmt][0]; k++) sz[k] = F[fmt][k + 1];
    return F[fmt][0];
}
static void bc_regroup(const uint8_t *in, uint8_t *out, size_t n, int fmt, int to_planes) {
    int sz[4], nf = bc_fields(fmt, sz);
    size_t bs = (fmt == ZO_BC1 || fmt == ZO_BC4) ? 8 : 16, nb = n / bs, plane = 0, off = 0;
    for (int k = 0; k < nf; k++) {
        for (size_t b = 0; b < nb; b++) {
            size_t blk = b * bs + off, pl = plane + b * (size_t)sz[k];
            if (to_planes) memcpy(out + pl, in + blk, (size_t)sz[k]);
            else memcpy(out + blk, in + pl, (size_t)sz[k]);
        }
        plane += nb * (size_t)sz[k];
        off += (size_t)sz[k];
    }
    memcpy(out + nb * bs, in + nb * bs, n - nb * bs);
}
void zo_bc_split(const void *bc, size_t n, int fmt, void *out) { bc_regroup((const uint8_t *)bc, (uint8_t *)out, n, fmt, 1); }
void zo_bc_merge(const void *planes, size_t n, int fmt, void *out) { bc_regroup((const uint8_t *)planes, (uint8_t *)out, n, fmt, 0); }

int zo_bc7_fields(const void *blk, int info[5], int ep[6][4], int subset[16], int cw[16], int aw[16]) {
    bc7_fields F;
    int ok = bc7_parse((const uint8_t *)blk, &F);
    info[0] = F.mode; info[1] = F.ns; info[2] = F.part; info[3] = F.rot; info[4] = F.ab;
    memcpy(ep, F.ep, sizeof F.ep);
    memcpy(subset, F.subset, sizeof F.subset);
    memcpy(cw, F.cw, sizeof F.cw);
    memcpy(aw, F.aw, sizeof F.aw);
    return ok;
}

void zo_bc7_mode_hist(const void *bc, size_t nblocks, int hist[9]) {
    const uint8_t *b = (const uint8_t *)bc;
    for (int m = 0; m < 9; m++) hist[m] = 0;
    for (size_t k = 0; k < nblocks; k++) {
        int mode = 0;
        while (mode < 8 && !((b[k * 16] >> mode) & 1)) mode++;
        hist[mode]++;
    }
}

/* ================================================================== BC6H, unsigned mode 11 (zap_tex.h:817-975) */
uint16_t zo_f2h(float f) { /* :820-827 */
    uint32_t x;
    if (!(f > 0)) return 0;
    memcpy(&x, &f, 4);
    if (x >= 0x477FE000u) return 0x7BFF;
    if (x < 0x38800000u) return (uint16_t)(f * 16777216.0f + 0.5f);
    return (uint16_t)(((x - 0x38000000u) + 0x1000u) >> 13);
}
float zo_h2f(uint16_t h) { /* :828-835 */
    uint32_t e = (h >> 10) & 31, m = h & 1023u, x;
    float f;
    if (e == 0) return (float)m * (1.0f / 16777216.0f);
    x = ((e + 112u) << 23) | (m << 13);
    memcpy(&f, &x, 4);
    return f;
}
static int bc6_unquant(int e) { return e == 0 ? 0 : e == 1023 ? 0xFFFF : ((e << 16) + 0x8000) >> 10; }
static int bc6_finish(int u) { return (u * 31) >> 6; }
static int bc6_nearest(float u) { /* :841-851 */
    int g = (int)((u - 32.0f) / 64.0f + 0.5f), best = 0;
    float bd = 1e30f;
    for (int k = 0; k < 3; k++) {
        int e = iclamp(around(g, k), 0, 1023);
        float d = fabsf((float)bc6_unquant(e) - u);
        if (d < bd) { bd = d; best = e; }
    }
    return best;
}
/* the reference accumulates these integer squared errors in double, where they are exact; int64 is the same */
static int64_t bc6_fit(const uint16_t t[16][3], const int e[2][3], int idx[16]) { /* :854-871 */
    int pal[16][3];
    int64_t err = 0;
    for (int j = 0; j < 16; j++)
        for (int c = 0; c < 3; c++) pal[j][c] = bc6_finish(lerp64(bc6_unquant(e[0][c]), bc6_unquant(e[1][c]), BC7_W4[j]));
    ZO_OPS(16 * 16 * 10);
    for (int i = 0; i < 16; i++) {
        int64_t be = INT64_MAX;
        int bi = 0;
        for (int j = 0; j < 16; j++) {
            int64_t d = 0;
            for (int c = 0; c < 3; c++) { int64_t x = (int64_t)t[i][c] - pal[j][c]; d += x * x; }
            if (d < be) { be = d; bi = j; }
        }
        idx[i] = bi; err += be;
    }
    return err;
}
static void bc6_block(const uint16_t t[16][3], uint8_t out[16]) { /* :873-931 */
    float U[16][3], mu[3] = { 0, 0, 0 }, C[6] = { 0, 0, 0, 0, 0, 0 }, v[3] = { 1, 1, 1 };
    for (int i = 0; i < 16; i++) for (int c = 0; c < 3; c++) { U[i][c] = t[i][c] * 64.0f / 31.0f; mu[c] += U[i][c] / 16.0f; }
    for (int i = 0; i < 16; i++) {
        float r = U[i][0] - mu[0], g = U[i][1] - mu[1], b = U[i][2] - mu[2];
        C[0] += r * r; C[1] += r * g; C[2] += r * b; C[3] += g * g; C[4] += g * b; C[5] += b * b;
    }
    for (int it = 0; it < 6; it++) {
        float x = C[0] * v[0] + C[1] * v[1] + C[2] * v[2], y = C[1] * v[0] + C[3] * v[1] + C[4] * v[2];
        float z = C[2] * v[0] + C[4] * v[1] + C[5] * v[2], m = fabsf(x);
        if (fabsf(y) > m) m = fabsf(y);
        if (fabsf(z) > m) m = fabsf(z);
        if (m < 1e-6f) break;
        v[0] = x / m; v[1] = y / m; v[2] = z / m;
    }
    float n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], tl = 1e30f, th = -1e30f;
    float bl[3] = { 1e30f, 1e30f, 1e30f }, bh[3] = { 0, 0, 0 };
    for (int i = 0; i < 16; i++) {
        float d = (U[i][0] - mu[0]) * v[0] + (U[i][1] - mu[1]) * v[1] + (U[i][2] - mu[2]) * v[2];
        if (d < tl) tl = d;
        if (d > th) th = d;
        for (int c = 0; c < 3; c++) { if (U[i][c] < bl[c]) bl[c] = U[i][c]; if (U[i][c] > bh[c]) bh[c] = U[i][c]; }
    }
    int64_t best = INT64_MAX;
    int be[2][3] = { { 0 } }, bidx[16] = { 0 };
    for (int start = 0; start < 2; start++) {
        int e[2][3], idx[16];
        for (int c = 0; c < 3; c++) {
            float lo = start ? bl[c] : mu[c] + v[c] * tl / n2, hi = start ? bh[c] : mu[c] + v[c] * th / n2;
            e[0][c] = bc6_nearest(lo); e[1][c] = bc6_nearest(hi);
        }
        int64_t err = bc6_fit(t, (const int(*)[3])e, idx);
        for (int it = 0; it < 3 && err > 0; it++) {
            float aa = 0, ab = 0, bb = 0, sa[3] = { 0, 0, 0 }, sb[3] = { 0, 0, 0 };
            for (int i = 0; i < 16; i++) {
                float w = BC7_W4[idx[i]] / 64.0f, u = 1 - w;
                aa += u * u; ab += u * w; bb += w * w;
                for (int c = 0; c < 3; c++) { sa[c] += u * U[i][c]; sb[c] += w * U[i][c]; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) break;
            int ne[2][3], ni[16];
            for (int c = 0; c < 3; c++) { ne[0][c] = bc6_nearest((sa[c] * bb - sb[c] * ab) / det); ne[1][c] = bc6_nearest((sb[c] * aa - sa[c] * ab) / det); }
            int64_t e2 = bc6_fit(t, (const int(*)[3])ne, ni);
            if (e2 >= err) break;
            err = e2; memcpy(e, ne, sizeof ne); memcpy(idx, ni, sizeof ni);
        }
        if (err < best) { best = err; memcpy(be, e, sizeof e); memcpy(bidx, idx, sizeof idx); }
    }
    if (bidx[0] & 8) {
        for (int c = 0; c < 3; c++) { int x = be[0][c]; be[0][c] = be[1][c]; be[1][c] = x; }
        for (int i = 0; i < 16; i++) bidx[i] = 15 - bidx[i];
    }
    memset(out, 0, 16);
    bitw w = { out, 0 };
    put_bits(&w, 3, 5);
    for (int k = 0; k < 2; k++) for (int c = 0; c < 3; c++) put_bits(&w, (unsigned)be[k][c], 10);
    for (int i = 0; i < 16; i++) put_bits(&w, (unsigned)bidx[i], i ? 4 : 3);
}

void zo_bc6h_encode(const float *rgba, int w, int h, size_t stride, void *out_) {
    uint8_t *out = (uint8_t *)out_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            uint16_t t[16][3];
            for (int i = 0; i < 16; i++) {
                int x = imin(bx * 4 + (i & 3), w - 1), y = imin(by * 4 + (i >> 2), h - 1);
                for (int c = 0; c < 3; c++) t[i][c] = zo_f2h(rgba[(size_t)y * stride + (size_t)x * 4 + c]);
            }
            bc6_block((const uint16_t(*)[3])t, out + ((size_t)by * (size_t)bw + (size_t)bx) * 16);
        }
}

void zo_bc6h_decode(const void *bc_, int w, int h, uint16_t *rgba, size_t stride) {
    const uint8_t *bc = (const uint8_t *)bc_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            const uint8_t *b = bc + ((size_t)by * (size_t)bw + (size_t)bx) * 16;
            uint16_t px[16][4];
            memset(px, 0, sizeof px);
            bitr r = { b, 0 };
            if (get_bits(&r, 5) == 3) {
                int e[2][3];
                for (int k = 0; k < 2; k++) for (int c = 0; c < 3; c++) e[k][c] = bc6_unquant((int)get_bits(&r, 10));
                for (int i = 0; i < 16; i++) {
                    int wt = BC7_W4[get_bits(&r, i ? 4 : 3)];
                    for (int c = 0; c < 3; c++) px[i][c] = (uint16_t)bc6_finish(lerp64(e[0][c], e[1][c], wt));
                    px[i][3] = 0x3C00;
                }
            }
            for (int i = 0; i < 16; i++) {
                int x = bx * 4 + (i & 3), y = by * 4 + (i >> 2);
                if (x < w && y < h) memcpy(rgba + (size_t)y * stride + (size_t)x * 4, px[i], 8);
            }
        }
}

/* ================================================================== ASTC 4x4 LDR (zap_tex.h:977-1356) */
/* integer-sequence ranges (ASTC spec): levels, trit?, quint?, plain bits */
typedef struct { int levels, trit, quint, bits; } ise_range;
static const ise_range ISE[21] = {
    { 2, 0, 0, 1 }, { 3, 1, 0, 0 }, { 4, 0, 0, 2 }, { 5, 0, 1, 0 }, { 6, 1, 0, 1 }, { 8, 0, 0, 3 }, { 10, 0, 1, 1 },
    { 12, 1, 0, 2 }, { 16, 0, 0, 4 }, { 20, 0, 1, 2 }, { 24, 1, 0, 3 }, { 32, 0, 0, 5 }, { 40, 0, 1, 3 }, { 48, 1, 0, 4 },
    { 64, 0, 0, 6 }, { 80, 0, 1, 4 }, { 96, 1, 0, 5 }, { 128, 0, 0, 7 }, { 160, 0, 1, 5 }, { 192, 1, 0, 6 }, { 256, 0, 0, 8 } };
static int ise_nbits(const ise_range *r, int n) { return n * r->bits + (r->trit ? (8 * n + 4) / 5 : r->quint ? (7 * n + 2) / 3 : 0); }
static int astc_colour_range(int nvals, int avail) { /* largest range with >= 6 levels that fits (:996-999) */
    for (int i = 20; i >= 4; i--) if (ise_nbits(&ISE[i], nvals) <= avail) return i;
    return -1;
}
static int bit_replicate(int v, int n, int to) {
    int x = 0;
    for (int sh = to - n; sh > -n; sh -= n) x |= sh >= 0 ? v << sh : v >> -sh;
    return x & ((1 << to) - 1);
}
static int astc_colour_unquant(const ise_range *r, int v) { /* ASTC spec colour unquantisation (:1008-1027) */
    if (!r->trit && !r->quint) return bit_replicate(v, r->bits, 8);
    int n = r->bits, m = v & ((1 << n) - 1), D = v >> n;
    int a = m & 1, b = (m >> 1) & 1, c = (m >> 2) & 1, d = (m >> 3) & 1, e = (m >> 4) & 1, f = (m >> 5) & 1;
    int A = a ? 0x1FF : 0, B = 0, C = 0;
    switch (r->levels) {
    case 6: C = 204; break;
    case 10: C = 113; break;
    case 12: B = (b << 8) | (b << 4) | (b << 2) | (b << 1); C = 93; break;
    case 20: B = (b << 8) | (b << 3) | (b << 2); C = 54; break;
    case 24: B = (c << 8) | (b << 7) | (c << 3) | (b << 2) | (c << 1) | b; C = 44; break;
    case 40: B = (c << 8) | (b << 7) | (c << 2) | (b << 1) | c; C = 26; break;
    case 48: B = (d << 8) | (c << 7) | (b << 6) | (d << 2) | (c << 1) | b; C = 22; break;
    case 80: B = (d << 8) | (c << 7) | (b << 6) | (d << 1) | c; C = 13; break;
    case 96: B = (e << 8) | (d << 7) | (c << 6) | (b << 5) | (e << 1) | d; C = 11; break;
    case 160: B = (e << 8) | (d << 7) | (c << 6) | (b << 5) | e; C = 6; break;
    case 192: B = (f << 8) | (e << 7) | (d << 6) | (c << 5) | (b << 4) | f; C = 5; break;
    }
    int T = (D * C + B) ^ A;
    return (A & 0x80) | (T >> 2);
}
static int astc_weight_unquant(int w, int n) { int x = bit_replicate(w, n, 6); return x > 32 ? x + 1 : x; }

static void trit_unpack(int T, int t[5]) { /* ASTC spec: 8 bits -> 5 trits */
    int C;
    if (((T >> 2) & 7) == 7) { C = (((T >> 5) & 7) << 2) | (T & 3); t[4] = 2; t[3] = 2; }
    else {
        C = T & 31;
        if (((T >> 5) & 3) == 3) { t[4] = 2; t[3] = (T >> 7) & 1; }
        else { t[4] = (T >> 7) & 1; t[3] = (T >> 5) & 3; }
    }
    if ((C & 3) == 3) { t[2] = 2; t[1] = (C >> 4) & 1; t[0] = (((C >> 3) & 1) << 1) | (((C >> 2) & 1) & ~(C >> 3) & 1); }
    else if (((C >> 2) & 3) == 3) { t[2] = 2; t[1] = 2; t[0] = C & 3; }
    else { t[2] = (C >> 4) & 1; t[1] = (C >> 2) & 3; t[0] = (((C >> 1) & 1) << 1) | ((C & 1) & ~(C >> 1) & 1); }
}
static void quint_unpack(int Q, int q[3]) { /* ASTC spec: 7 bits -> 3 quints */
    if (((Q >> 1) & 3) == 3 && ((Q >> 5) & 3) == 0) {
        q[2] = ((Q & 1) << 2) | ((((Q >> 4) & 1) & ~Q & 1) << 1) | (((Q >> 3) & 1) & ~Q & 1);
        q[1] = 4; q[0] = 4;
        return;
    }
    int C;
    if (((Q >> 1) & 3) == 3) { q[2] = 4; C = (((Q >> 3) & 3) << 3) | ((~(Q >> 5) & 3) << 1) | (Q & 1); }
    else { q[2] = (Q >> 5) & 3; C = Q & 31; }
    if ((C & 7) == 5) { q[1] = 4; q[0] = (C >> 3) & 3; }
    else { q[1] = (C >> 3) & 3; q[0] = C & 7; }
}
static const int TRIT_SPLIT[5] = { 2, 2, 1, 2, 1 }, QUINT_SPLIT[3] = { 3, 2, 2 }; /* packed-code bits after each value */
static uint8_t TRIT_CODE[243], QUINT_CODE[125]; /* value combination -> smallest packed code that decodes to it */

static void ise_write(bitw *w, const ise_range *r, int n, const int *v) {
    int gs = r->trit ? 5 : r->quint ? 3 : 1, base = r->trit ? 3 : 5;
    const int *split = r->trit ? TRIT_SPLIT : QUINT_SPLIT;
    for (int g = 0; g < n; g += gs) {
        int cnt = imin(n - g, gs), X = 0, used = 0;
        if (gs > 1) {
            int key = 0;
            for (int k = gs - 1; k >= 0; k--) key = key * base + (k < cnt ? v[g + k] >> r->bits : 0);
            X = r->trit ? TRIT_CODE[key] : QUINT_CODE[key];
        }
        for (int k = 0; k < cnt; k++) {
            put_bits(w, (unsigned)(v[g + k] & ((1 << r->bits) - 1)), r->bits);
            if (gs > 1) { put_bits(w, (unsigned)(X >> used), split[k]); used += split[k]; }
        }
    }
}
static void ise_read(bitr *rd, const ise_range *r, int n, int *v) {
    int gs = r->trit ? 5 : r->quint ? 3 : 1;
    const int *split = r->trit ? TRIT_SPLIT : QUINT_SPLIT;
    for (int g = 0; g < n; g += gs) {
        int cnt = imin(n - g, gs), m[5], X = 0, used = 0, hi[5];
        for (int k = 0; k < cnt; k++) {
            m[k] = (int)get_bits(rd, r->bits);
            if (gs > 1) { X |= (int)get_bits(rd, split[k]) << used; used += split[k]; }
        }
        if (r->trit) trit_unpack(X, hi);
        else if (r->quint) quint_unpack(X, hi);
        for (int k = 0; k < cnt; k++) v[g + k] = gs > 1 ? (hi[k] << r->bits) | m[k] : m[k];
    }
}

static uint32_t astc_hash52(uint32_t p) { /* ASTC spec partition hash */
    p ^= p >> 15; p -= p << 17; p += p << 7; p += p << 4; p ^= p >> 5;
    p += p << 16; p ^= p >> 7; p ^= p >> 3; p ^= p << 6; p ^= p >> 17;
    return p;
}
int zo_astc_partition(int seed, int x, int y, int count) { /* ASTC spec partition selection, small block (:1102-1120) */
    x <<= 1; y <<= 1;
    seed += (count - 1) * 1024;
    uint32_t h = astc_hash52((uint32_t)seed);
    int s[8];
    for (int i = 0; i < 8; i++) s[i] = (int)((h >> (4 * i)) & 15);
    for (int i = 0; i < 8; i++) s[i] *= s[i];
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2) ? 4 : 5; sh2 = count == 3 ? 6 : 5; }
    else { sh1 = count == 3 ? 6 : 5; sh2 = (seed & 2) ? 4 : 5; }
    for (int i = 0; i < 8; i++) s[i] >>= (i & 1) ? sh2 : sh1;
    int a = (s[0] * x + s[1] * y + (int)(h >> 14)) & 0x3F, b = (s[2] * x + s[3] * y + (int)(h >> 10)) & 0x3F;
    int c = (s[4] * x + s[5] * y + (int)(h >> 6)) & 0x3F, d = (s[6] * x + s[7] * y + (int)(h >> 2)) & 0x3F;
    if (count < 4) d = 0;
    if (count < 3) c = 0;
    return (a >= b && a >= c && a >= d) ? 0 : (b >= c && b >= d) ? 1 : c >= d ? 2 : 3;
}

/* decoded RGBA endpoints of a CEM 8 / 12 pair from unquantised values r0 r1 g0 g1 b0 b1 [a0 a1] (:1122-1129) */
static void astc_endpoint_pair(int cem, const int *v, int e0[4], int e1[4]) {
    int a0 = cem == 12 ? v[6] : 255, a1 = cem == 12 ? v[7] : 255;
    if (v[1] + v[3] + v[5] >= v[0] + v[2] + v[4]) {
        e0[0] = v[0]; e0[1] = v[2]; e0[2] = v[4]; e0[3] = a0;
        e1[0] = v[1]; e1[1] = v[3]; e1[2] = v[5]; e1[3] = a1;
    } else { /* blue contraction */
        e0[0] = (v[1] + v[5]) >> 1; e0[1] = (v[3] + v[5]) >> 1; e0[2] = v[5]; e0[3] = a1;
        e1[0] = (v[0] + v[4]) >> 1; e1[1] = (v[2] + v[4]) >> 1; e1[2] = v[4]; e1[3] = a0;
    }
}
static int astc_lerp(int a, int b, int w) { return (((a * 257) * (64 - w) + (b * 257) * w + 32) >> 6) >> 8; }

static void astc_decode_block(const uint8_t *b, tx4 px[16]) { /* :1135-1168 */
    bitr r = { b, 0 };
    int mode = (int)get_bits(&r, 11);
    for (int i = 0; i < 16; i++) { px[i][0] = 255; px[i][1] = 0; px[i][2] = 255; px[i][3] = 255; }
    if ((mode & 0x1FF) == 0x1FC) {
        bitr v = { b, 64 };
        for (int c = 0; c < 4; c++) { int x = (int)get_bits(&v, 16) >> 8; for (int i = 0; i < 16; i++) px[i][c] = (uint8_t)x; }
        return;
    }
    if (!(mode & 3) || ((mode >> 2) & 3) || ((mode >> 5) & 3) != 2 || ((mode >> 7) & 3) || ((mode >> 10) & 1)) return;
    int R = ((mode & 1) << 1) | (((mode >> 1) & 1) << 2) | ((mode >> 4) & 1), H = (mode >> 9) & 1;
    static const int LEVELS[2][8] = { { 0, 0, 2, 3, 4, 5, 6, 8 }, { 0, 0, 10, 12, 16, 20, 24, 32 } };
    int levels = LEVELS[H][R], wb = levels == 2 ? 1 : levels == 4 ? 2 : levels == 8 ? 3 : levels == 16 ? 4 : levels == 32 ? 5 : 0;
    int parts = (int)get_bits(&r, 2) + 1, seed = 0, cem;
    if (!wb || parts > 2) return;
    if (parts == 2) {
        seed = (int)get_bits(&r, 10);
        int cf = (int)get_bits(&r, 6);
        if (cf & 3) return;
        cem = cf >> 2;
    } else cem = (int)get_bits(&r, 4);
    int nv = cem == 8 ? 6 : cem == 12 ? 8 : 0, v[16], e[2][2][4];
    if (!nv) return;
    int ri = astc_colour_range(nv * parts, 128 - r.pos - 16 * wb);
    if (ri < 0) return;
    ise_read(&r, &ISE[ri], nv * parts, v);
    for (int i = 0; i < nv * parts; i++) v[i] = astc_colour_unquant(&ISE[ri], v[i]);
    for (int k = 0; k < parts; k++) astc_endpoint_pair(cem, v + k * nv, e[k][0], e[k][1]);
    for (int i = 0; i < 16; i++) {
        int w = 0, k = parts == 2 ? zo_astc_partition(seed, i & 3, i >> 2, 2) : 0;
        for (int j = 0; j < wb; j++) { int bit = 127 - (i * wb + j); w |= ((b[bit >> 3] >> (bit & 7)) & 1) << j; }
        w = astc_weight_unquant(w, wb);
        for (int c = 0; c < 4; c++) px[i][c] = (uint8_t)astc_lerp(e[k][0][c], e[k][1][c], w);
    }
}

/* one trial configuration: endpoint mode, weight bits, partitions, colour range, 8-bit -> nearest code LUT */
typedef struct { int cem, wb, parts, nv, range; uint8_t q[256]; } astc_cfg;
static astc_cfg ASTC_CFG[8]; /* (cem, wb, parts): (8,4,1) (8,3,1) (8,5,1) (12,4,1) (12,3,1) (12,2,1) (8,3,2) (8,2,2) (:1298-1300) */
static uint16_t PAT_MASK[1024], PAT_SEED[1024];
static int PAT_COUNT;
static float SRGB_LIN[256], SRGB_THR[255];

static void astc_cfg_make(astc_cfg *c, int cem, int wb, int parts) { /* :1172-1180 */
    c->cem = cem; c->wb = wb; c->parts = parts; c->nv = cem == 8 ? 6 : 8;
    c->range = astc_colour_range(c->nv * parts, 128 - (parts == 1 ? 17 : 29) - 16 * wb);
    const ise_range *r = &ISE[c->range];
    for (int x = 0; x < 256; x++) {
        int best = 0, bd = 1 << 30;
        for (int v = 0; v < r->levels; v++) { int d = abs(astc_colour_unquant(r, v) - x); if (d < bd) { bd = d; best = v; } }
        c->q[x] = (uint8_t)best;
    }
}

/* sRGB tables: the reference's constants are the double-precision transfer function printed to 9 significant
   digits and read back as float; derive them the same way */
static float srgb_to_linear_9g(double c) {
    double lin = c <= 0.04045 ? c / 12.92 : pow((c + 0.055) / 1.055, 2.4);
    char buf[64];
    snprintf(buf, sizeof buf, "%.9g", lin);
    return strtof(buf, NULL);
}

static pthread_once_t ONCE = PTHREAD_ONCE_INIT;
static void tables_init(void) {
    for (int T = 255; T >= 0; T--) { int t[5]; trit_unpack(T, t); TRIT_CODE[t[0] + 3 * t[1] + 9 * t[2] + 27 * t[3] + 81 * t[4]] = (uint8_t)T; }
    for (int Q = 127; Q >= 0; Q--) { int q[3]; quint_unpack(Q, q); QUINT_CODE[q[0] + 5 * q[1] + 25 * q[2]] = (uint8_t)Q; }
    static const int CFG[8][3] = { { 8, 4, 1 }, { 8, 3, 1 }, { 8, 5, 1 }, { 12, 4, 1 }, { 12, 3, 1 }, { 12, 2, 1 }, { 8, 3, 2 }, { 8, 2, 2 } };
    for (int k = 0; k < 8; k++) astc_cfg_make(&ASTC_CFG[k], CFG[k][0], CFG[k][1], CFG[k][2]);
    PAT_COUNT = 0;
    for (int sd = 0; sd < 1024; sd++) {
        unsigned m = 0;
        for (int i = 0; i < 16; i++) m |= (unsigned)zo_astc_partition(sd, i & 3, i >> 2, 2) << i;
        if (m && m != 0xFFFFu) { PAT_MASK[PAT_COUNT] = (uint16_t)m; PAT_SEED[PAT_COUNT++] = (uint16_t)sd; }
    }
    for (int k = 0; k < 256; k++) SRGB_LIN[k] = srgb_to_linear_9g(k / 255.0);
    for (int k = 0; k < 255; k++) SRGB_THR[k] = srgb_to_linear_9g((k + 0.5) / 255.0);
}
static void ensure_tables(void) { pthread_once(&ONCE, tables_init); }

/* float endpoints -> codes + unquantised values; the pair with the larger RGB sum goes second (:1183-1194) */
static void astc_quant(const astc_cfg *c, const float lo[4], const float hi[4], int *code, int *uv) {
    const ise_range *r = &ISE[c->range];
    float s0 = lo[0] + lo[1] + lo[2], s1 = hi[0] + hi[1] + hi[2];
    const float *a = s1 >= s0 ? lo : hi, *b = s1 >= s0 ? hi : lo;
    for (int k = 0; k < c->nv / 2; k++) {
        int x0 = iclamp((int)(a[k] + 0.5f), 0, 255), x1 = iclamp((int)(b[k] + 0.5f), 0, 255);
        code[2 * k] = c->q[x0]; code[2 * k + 1] = c->q[x1];
        uv[2 * k] = astc_colour_unquant(r, code[2 * k]); uv[2 * k + 1] = astc_colour_unquant(r, code[2 * k + 1]);
    }
    if (uv[1] + uv[3] + uv[5] < uv[0] + uv[2] + uv[4])
        for (int k = 0; k < c->nv / 2; k++) {
            int s = code[2 * k]; code[2 * k] = code[2 * k + 1]; code[2 * k + 1] = s;
            s = uv[2 * k]; uv[2 * k] = uv[2 * k + 1]; uv[2 * k + 1] = s;
        }
}
static int astc_fit_weights(const tx4 px[16], const astc_cfg *c, const int *uv, const int *part, int nc, int w[16]) { /* :1197-1210 */
    int L = 1 << c->wb, pal[2][32][4], err = 0;
    for (int k = 0; k < c->parts; k++) {
        int e0[4], e1[4];
        astc_endpoint_pair(c->cem, uv + k * c->nv, e0, e1);
        for (int j = 0; j < L; j++) {
            int wt = astc_weight_unquant(j, c->wb);
            for (int ch = 0; ch < 4; ch++) pal[k][j][ch] = astc_lerp(e0[ch], e1[ch], wt);
        }
    }
    ZO_OPS(16 * L * (3 * nc + 1));
    for (int i = 0; i < 16; i++) {
        int bj = 0, be = 1 << 30, k = part[i];
        for (int j = 0; j < L; j++) {
            int d = 0;
            for (int ch = 0; ch < nc; ch++) { int x = px[i][ch] - pal[k][j][ch]; d += x * x; }
            if (d < be) { be = d; bj = j; }
        }
        w[i] = bj; err += be;
    }
    return err;
}
static int astc_trial(const tx4 px[16], const astc_cfg *c, const int *part, int code[16], int w[16]) { /* :1212-1244 */
    int nc = c->cem == 12 ? 4 : 3, uv[16], tc[16], tuv[16], tw[16];
    for (int k = 0; k < c->parts; k++) {
        int sel[16], cnt = 0;
        float lo[4], hi[4];
        for (int i = 0; i < 16; i++) if (part[i] == k) sel[cnt++] = i;
        if (!cnt) { sel[0] = 0; cnt = 1; }
        pca_endpoints(px, sel, cnt, nc, lo, hi);
        astc_quant(c, lo, hi, code + k * c->nv, uv + k * c->nv);
    }
    int err = astc_fit_weights(px, c, uv, part, nc, w);
    for (int it = 0; it < 3 && err > 0; it++) {
        memcpy(tc, code, sizeof tc); memcpy(tuv, uv, sizeof tuv);
        for (int k = 0; k < c->parts; k++) {
            float aa = 0, ab = 0, bb = 0, sa[4] = { 0, 0, 0, 0 }, sb[4] = { 0, 0, 0, 0 }, nlo[4], nhi[4];
            for (int i = 0; i < 16; i++) {
                if (part[i] != k) continue;
                float f = astc_weight_unquant(w[i], c->wb) / 64.0f, g = 1 - f;
                aa += g * g; ab += g * f; bb += f * f;
                for (int ch = 0; ch < nc; ch++) { sa[ch] += g * px[i][ch]; sb[ch] += f * px[i][ch]; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) continue;
            for (int ch = 0; ch < nc; ch++) { nlo[ch] = (sa[ch] * bb - sb[ch] * ab) / det; nhi[ch] = (sb[ch] * aa - sa[ch] * ab) / det; }
            for (int ch = nc; ch < 4; ch++) nlo[ch] = nhi[ch] = 255;
            astc_quant(c, nlo, nhi, tc + k * c->nv, tuv + k * c->nv);
        }
        int e = astc_fit_weights(px, c, tuv, part, nc, tw);
        if (e >= err) break;
        err = e; memcpy(code, tc, sizeof tc); memcpy(uv, tuv, sizeof tuv); memcpy(w, tw, sizeof tw);
    }
    return err;
}
static void astc_write_block(const astc_cfg *c, int seed, const int *code, const int w[16], uint8_t out[16]) { /* :1246-1260 */
    static const int RH[6][2] = { { 0, 0 }, { 0, 0 }, { 4, 0 }, { 7, 0 }, { 4, 1 }, { 7, 1 } }; /* weight bits -> (R, H) */
    int R = RH[c->wb][0], H = RH[c->wb][1];
    unsigned mode = (unsigned)(((R >> 1) & 1) | (((R >> 2) & 1) << 1) | ((R & 1) << 4) | (2 << 5) | (H << 9));
    memset(out, 0, 16);
    bitw bwr = { out, 0 };
    put_bits(&bwr, mode, 11);
    put_bits(&bwr, (unsigned)(c->parts - 1), 2);
    if (c->parts == 2) { put_bits(&bwr, (unsigned)seed, 10); put_bits(&bwr, (unsigned)c->cem << 2, 6); }
    else put_bits(&bwr, (unsigned)c->cem, 4);
    ise_write(&bwr, &ISE[c->range], c->nv * c->parts, code);
    uint8_t wbits[16] = { 0 };
    bitw ww = { wbits, 0 };
    for (int i = 0; i < 16; i++) put_bits(&ww, (unsigned)w[i], c->wb);
    for (int i = 0; i < ww.pos; i++)
        if ((wbits[i >> 3] >> (i & 7)) & 1) out[(127 - i) >> 3] |= (uint8_t)(1u << ((127 - i) & 7));
}
static unsigned astc_two_means(const tx4 px[16]) { /* :1263-1283 */
    float c[2][3];
    int lo = 0, hi = 0;
    for (int i = 1; i < 16; i++) {
        int s = px[i][0] + px[i][1] + px[i][2];
        if (s < px[lo][0] + px[lo][1] + px[lo][2]) lo = i;
        if (s > px[hi][0] + px[hi][1] + px[hi][2]) hi = i;
    }
    for (int k = 0; k < 3; k++) { c[0][k] = px[lo][k]; c[1][k] = px[hi][k]; }
    unsigned m = 0;
    for (int it = 0; it < 4; it++) {
        float sum[2][3] = { { 0, 0, 0 }, { 0, 0, 0 } };
        int n[2] = { 0, 0 };
        m = 0;
        for (int i = 0; i < 16; i++) {
            float d0 = 0, d1 = 0;
            for (int k = 0; k < 3; k++) { float a = px[i][k] - c[0][k], b = px[i][k] - c[1][k]; d0 += a * a; d1 += b * b; }
            int s = d1 < d0;
            m |= (unsigned)s << i; n[s]++;
            for (int k = 0; k < 3; k++) sum[s][k] += px[i][k];
        }
        for (int s = 0; s < 2; s++) if (n[s]) for (int k = 0; k < 3; k++) c[s][k] = sum[s][k] / n[s];
    }
    return m;
}
static int popcount16(unsigned x) { int n = 0; for (; x; x &= x - 1) n++; return n; }

void zo_astc_encode(const uint8_t *rgba, int w, int h, size_t stride, void *out_) { /* :1291-1342 */
    ensure_tables();
    uint8_t *out = (uint8_t *)out_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            tx4 px[16];
            int opaque = 1, part0[16] = { 0 };
            gather8(rgba, w, h, stride, bx, by, px);
            for (int i = 0; i < 16; i++) opaque &= px[i][3] == 255;
            int best = 1 << 30, bc = 0, bseed = 0, bcode[16], bwt[16], code[16], wt[16];
            for (int k = opaque ? 0 : 3; k < (opaque ? 3 : 6); k++) {
                int e = astc_trial((const tx4 *)px, &ASTC_CFG[k], part0, code, wt);
                if (e < best) { best = e; bc = k; memcpy(bcode, code, sizeof code); memcpy(bwt, wt, sizeof wt); }
            }
            if (opaque && best > 16 * 3 * 4) {
                unsigned km = astc_two_means((const tx4 *)px);
                int cand[4] = { -1, -1, -1, -1 }, cd[4] = { 99, 99, 99, 99 };
                for (int pi = 0; pi < PAT_COUNT && cd[3]; pi++) { /* top-4 by (distance, pattern order); stops at 4 exact */
                    int dd = popcount16(PAT_MASK[pi] ^ km), dist = dd < 16 - dd ? dd : 16 - dd;
                    for (int j = 0; j < 4; j++)
                        if (dist < cd[j]) {
                            for (int k = 3; k > j; k--) { cd[k] = cd[k - 1]; cand[k] = cand[k - 1]; }
                            cd[j] = dist; cand[j] = pi;
                            break;
                        }
                }
                for (int j = 0; j < 4 && cand[j] >= 0; j++) {
                    int part[16];
                    for (int i = 0; i < 16; i++) part[i] = (PAT_MASK[cand[j]] >> i) & 1;
                    for (int k = 6; k < 8; k++) {
                        int e = astc_trial((const tx4 *)px, &ASTC_CFG[k], part, code, wt);
                        if (e < best) { best = e; bc = k; bseed = PAT_SEED[cand[j]]; memcpy(bcode, code, sizeof code); memcpy(bwt, wt, sizeof wt); }
                    }
                }
            }
            astc_write_block(&ASTC_CFG[bc], bseed, bcode, bwt, out + ((size_t)by * (size_t)bw + (size_t)bx) * 16);
        }
}

void zo_astc_decode(const void *bc_, int w, int h, uint8_t *rgba, size_t stride) {
    ensure_tables();
    const uint8_t *bc = (const uint8_t *)bc_;
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            tx4 px[16];
            astc_decode_block(bc + ((size_t)by * (size_t)bw + (size_t)bx) * 16, px);
            for (int i = 0; i < 16; i++) {
                int x = bx * 4 + (i & 3), y = by * 4 + (i >> 2);
                if (x < w && y < h) memcpy(rgba + (size_t)y * stride + (size_t)x * 4, px[i], 4);
            }
        }
}

int zo_ise_roundtrip(int range, int n, const int *v, int *got) {
    ensure_tables();
    uint8_t b[32] = { 0 };
    bitw w = { b, 0 };
    ise_write(&w, &ISE[range], n, v);
    bitr r = { b, 0 };
    ise_read(&r, &ISE[range], n, got);
    if (r.pos != w.pos || w.pos != ise_nbits(&ISE[range], n)) return -1;
    for (int i = 0; i < n; i++) if (got[i] != v[i]) return -1;
    return w.pos;
}

/* ================================================================== mipmaps (zap_tex.h:1358-1469) */
void zo_srgb_tables(float lin[256], float thr[255]) {
    ensure_tables();
    memcpy(lin, SRGB_LIN, sizeof SRGB_LIN);
    memcpy(thr, SRGB_THR, sizeof SRGB_THR);
}
static uint8_t linear_to_srgb8(float v) { /* first k with v < threshold[k] (:1429-1433) */
    int lo = 0, hi = 255;
    while (lo < hi) { int mid = (lo + hi) >> 1; if (v < SRGB_THR[mid]) hi = mid; else lo = mid + 1; }
    return (uint8_t)lo;
}
int zo_mip_levels(int w, int h) {
    int n = 1;
    while (w > 1 || h > 1) { w = w > 1 ? w / 2 : 1; h = h > 1 ? h / 2 : 1; n++; }
    return n;
}
void zo_mip_next(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride) {
    ensure_tables();
    int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            int x0 = imin(2 * x, w - 1), x1 = imin(2 * x + 1, w - 1), y0 = imin(2 * y, h - 1), y1 = imin(2 * y + 1, h - 1);
            const uint8_t *p0 = src + (size_t)y0 * stride + (size_t)x0 * 4, *p1 = src + (size_t)y0 * stride + (size_t)x1 * 4;
            const uint8_t *p2 = src + (size_t)y1 * stride + (size_t)x0 * 4, *p3 = src + (size_t)y1 * stride + (size_t)x1 * 4;
            uint8_t *o = dst + (size_t)y * dst_stride + (size_t)x * 4;
            for (int c = 0; c < 4; c++) {
                if (srgb && c < 3) o[c] = linear_to_srgb8((SRGB_LIN[p0[c]] + SRGB_LIN[p1[c]] + SRGB_LIN[p2[c]] + SRGB_LIN[p3[c]]) * 0.25f);
                else o[c] = (uint8_t)((p0[c] + p1[c] + p2[c] + p3[c] + 2) >> 2);
            }
        }
}
void zo_mip_next_f(const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride) {
    int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            int x0 = imin(2 * x, w - 1), x1 = imin(2 * x + 1, w - 1), y0 = imin(2 * y, h - 1), y1 = imin(2 * y + 1, h - 1);
            for (int c = 0; c < 4; c++)
                dst[(size_t)y * dst_stride + (size_t)x * 4 + c] =
                    0.25f * (src[(size_t)y0 * stride + (size_t)x0 * 4 + c] + src[(size_t)y0 * stride + (size_t)x1 * 4 + c] +
                             src[(size_t)y1 * stride + (size_t)x0 * 4 + c] + src[(size_t)y1 * stride + (size_t)x1 * 4 + c]);
        }
}

/* ================================================================== texture containers (zap.c:309-355, the CLI's tex)
 * .astc: 16-byte header (magic 5CA1AB13 little-endian, block 4x4x1, 24-bit sizes, depth 1) then one level of ASTC blocks
 * (zap.c:312-321). DDS: "DDS " + 124-byte header; the 20-byte DX10 extension follows for BC7 and for sRGB (zap.c:344-349);
 * then every level's blocks, largest first. BC4/BC5 are never sRGB (zap.c:325). */
static void put32(uint8_t *p, uint32_t v) { for (int k = 0; k < 4; k++) p[k] = (uint8_t)(v >> (8 * k)); }

size_t zo_dds_header(int w, int h, int fmt, int mips, int srgb, uint8_t hdr[148]) {
    static const char *fourcc[5] = { "DXT1", "DXT5", "BC4U", "BC5U", "DX10" };
    static const uint32_t dxgi_unorm[5] = { 71, 77, 80, 83, 98 };
    if (fmt == ZO_BC4 || fmt == ZO_BC5) srgb = 0;
    int dx10 = fmt == ZO_BC7 || srgb != 0, levels = mips ? zo_mip_levels(w, h) : 1;
    memset(hdr, 0, 148);
    memcpy(hdr, "DDS ", 4);
    put32(hdr + 4, 124);
    put32(hdr + 8, 0x1u | 0x2u | 0x4u | 0x1000u | 0x80000u | (mips ? 0x20000u : 0u)); /* CAPS HEIGHT WIDTH PIXELFORMAT LINEARSIZE (MIPMAPCOUNT) */
    put32(hdr + 12, (uint32_t)h);
    put32(hdr + 16, (uint32_t)w);
    put32(hdr + 20, (uint32_t)zo_bc_size(w, h, fmt));
    put32(hdr + 28, (uint32_t)levels);
    put32(hdr + 76, 32);   /* pixel format size */
    put32(hdr + 80, 0x4);  /* FOURCC */
    memcpy(hdr + 84, dx10 ? "DX10" : fourcc[fmt], 4);
    put32(hdr + 108, 0x1000u | (mips ? 0x400008u : 0u));
    if (!dx10) return 128;
    put32(hdr + 128, dxgi_unorm[fmt] + (srgb ? 1u : 0u)); /* the _SRGB code follows each UNORM one */
    put32(hdr + 132, 3);   /* TEXTURE2D */
    put32(hdr + 140, 1);   /* array size */
    return 148;
}

void zo_astc_header(int w, int h, uint8_t hdr[16]) {
    static const uint8_t head[7] = { 0x13, 0xAB, 0xA1, 0x5C, 4, 4, 1 };
    memset(hdr, 0, 16);
    memcpy(hdr, head, 7);
    for (int k = 0; k < 3; k++) { hdr[7 + k] = (uint8_t)(w >> (8 * k)); hdr[10 + k] = (uint8_t)(h >> (8 * k)); }
    hdr[13] = 1;
}

/* the whole file `zap tex` writes; fmt 6 = .astc; out == NULL returns the size only */
size_t zo_tex_file(const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, int mips, int srgb, uint8_t *out) {
    if (fmt == 6) {
        size_t bn = zo_bc_size(w, h, ZO_BC7);
        if (out) { zo_astc_header(w, h, out); zo_astc_encode(rgba, w, h, stride, out + 16); }
        return 16 + bn;
    }
    if (fmt == ZO_BC4 || fmt == ZO_BC5) srgb = 0;
    uint8_t hdr[148];
    size_t hn = zo_dds_header(w, h, fmt, mips, srgb, hdr), total = 0;
    int levels = mips ? zo_mip_levels(w, h) : 1;
    for (int l = 0, lw = w, lh = h; l < levels; l++, lw = lw > 1 ? lw / 2 : 1, lh = lh > 1 ? lh / 2 : 1) total += zo_bc_size(lw, lh, fmt);
    if (!out) return hn + total;
    memcpy(out, hdr, hn);
    uint8_t *p = out + hn, *img = (uint8_t *)malloc((size_t)w * h * 4), *next = (uint8_t *)malloc((size_t)w * h * 4 + 4);
    for (int y = 0; y < h; y++) memcpy(img + (size_t)y * w * 4, rgba + (size_t)y * stride, (size_t)w * 4);
    for (int l = 0, lw = w, lh = h; l < levels; l++) {
        zo_bc_encode(img, lw, lh, (size_t)lw * 4, fmt, rdo, p);
        p += zo_bc_size(lw, lh, fmt);
        if (l + 1 < levels) {
            int nw = lw > 1 ? lw / 2 : 1, nh = lh > 1 ? lh / 2 : 1;
            zo_mip_next(img, lw, lh, (size_t)lw * 4, srgb, next, (size_t)nw * 4);
            lw = nw; lh = nh;
            memcpy(img, next, (size_t)lw * lh * 4);
        }
    }
    free(img); free(next);
    return hn + total;
}

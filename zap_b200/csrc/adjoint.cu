// adjoint.cu - differentiable palette decode and gradient endpoint refinement (no reference counterpart).
//
// With a block's indices held fixed, the BCn palette decode is linear in the endpoints. Texel i of subset s,
// stored channel c, decodes to
//   a_i * E[2s][c] + (1 - a_i) * E[2s+1][c]
// the continuous form of the integer palettes (zap_tex.h:52-62 for BC1, a_i = {1, 0, 2/3, 1/3}[idx] in 4-colour
// order; :367-417 for BC7, a_i = 1 - w(idx) / 64 with the mode's 2-, 3- or 4-bit weights). BC7 covers every mode:
// up to three subsets (endpoint 2s + k of subset s), mode 4/5's separate colour and alpha index sets (the alpha
// weight is the second set's), the rotation that swaps alpha with one colour channel after the interpolation, and
// the modes without alpha bits, whose alpha decodes to 255 whatever the endpoints are (zero gradient).
// Endpoints are in 8-bit units: float[b][2][4] for BC1 (RGB used), float[b][6][4] for BC7, in stored channel order
// (before the rotation), texels in decoded order. Its adjoint maps an upstream gradient on the decoded texels to
// the endpoints: dL/dE[2s][c] = sum_i a_i g_i,  dL/dE[2s+1][c] = sum_i (1 - a_i) g_i over the texels of subset s.
//
// zap_tex_cuda_refine_dev runs, per block, Adam steps on the block's MSE through that adjoint, requantises the
// endpoints in the block's own mode (BC1 565; BC7 mode 6: 7 bits + a p-bit per endpoint; mode 5: 7-bit colour and
// 8-bit alpha; mode 1: 6 bits + a p-bit shared per subset), re-fits the indices (anchor indices made valid by
// swapping a subset's endpoints, which leaves every decoded value unchanged because w(n-1-j) = 64 - w(j)), and keeps
// the new block only if its true squared error is lower than the encoder's. The encoder writes BC7 modes 6, 5 and 1
// only (zap_tex.h:755-784); blocks of other modes are left as they are.
#include <string>

#include "../../include/zap_tex_cuda.h"
#include "ztc_common.cuh"
#include "ztc_decode.cuh"
#include "ztc_internal.h"

namespace ztc {

ZTC_DEV int endpoint_floats(int fmt) { return fmt == ZTC_FMT_BC1 ? 8 : 24; }

// A block's linear form: per texel the weight of the subset's first endpoint for the colour channels (a) and for
// alpha (aa), the subset (bit i of `s1`: subset 1; `s2`: subset 2), the rotation, which channels the endpoints
// decide (nc: BC1 3, BC7 4; alpha_fixed: BC7 alpha without bits, 255), and the texels whose colour is a constant
// whatever the endpoints (`black`: index 3 of a BC1 3-colour block, zap_tex.h:1508-1517, which decodes to 0).
struct LinBlock {
    float a[16], aa[16];
    uint32_t s1, s2, black;
    int rot, nc, mode;
    bool covered, alpha_fixed;
};

// decoded (optional): the block's texels as the integer decoder gives them (zap_tex.h:1508-1517, :378-417)
ZTC_DEV void linear_form(int fmt, const uint8_t *blk, LinBlock &L, float e[6][4], uint32_t *decoded = nullptr) {
    L.s1 = L.s2 = L.black = 0u;
    L.rot = 0;
    L.alpha_fixed = false;
    if (fmt == ZTC_FMT_BC1) {
        uint2 v = *(const uint2 *)blk;
        uint32_t c0 = v.x & 0xFFFFu, c1 = v.x >> 16;
        L.nc = 3; L.mode = 0; L.covered = true;
        const bool four = c0 > c1;  // the decoder's rule: 4 colours, else 3 colours and black (zap_tex.h:1508-1517)
        #pragma unroll
        for (int i = 0; i < 16; i++) {
            const uint32_t k = (v.y >> (2 * i)) & 3u;
            if (four) L.a[i] = k == 0 ? 1.0f : k == 1 ? 0.0f : k == 2 ? 2.0f / 3.0f : 1.0f / 3.0f;
            else L.a[i] = k == 0 ? 1.0f : k == 1 ? 0.0f : k == 2 ? 0.5f : 0.0f;
            L.aa[i] = L.a[i];
            if (!four && k == 3) L.black |= 1u << i;
        }
        if (decoded) dec::bc1_block(v, false, decoded);
        for (int k = 0; k < 2; k++) {
            uint32_t c = k ? c1 : c0;
            int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
            e[k][0] = (float)((R << 3) | (R >> 2)); e[k][1] = (float)((G << 2) | (G >> 4)); e[k][2] = (float)((B << 3) | (B >> 2));
            e[k][3] = 255.0f;
        }
        for (int k = 2; k < 6; k++) for (int c = 0; c < 4; c++) e[k][c] = 0.0f;
        return;
    }
    uint4 v = *(const uint4 *)blk;
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    L.nc = 4;
    if ((w[0] & 0x7Fu) == 0x40u) {  // mode 6, the encoder's common case: its fixed layout read directly
        L.mode = 6; L.covered = true;  // R0 R1 G0 G1 B0 B1 A0 A1 (7 bits each), a p-bit per endpoint, 4-bit indices
        int ep[2][4];
        #pragma unroll
        for (int c = 0; c < 4; c++)
            #pragma unroll
            for (int k = 0; k < 2; k++) {
                ep[k][c] = (int)((get_bits128(w, 7 + 14 * c + 7 * k, 7) << 1) | get_bits128(w, 63 + k, 1));
                e[k][c] = (float)ep[k][c];
            }
        for (int k = 2; k < 6; k++) for (int c = 0; c < 4; c++) e[k][c] = 0.0f;
        #pragma unroll
        for (int i = 0; i < 16; i++) {
            const int wt = w4(i == 0 ? (int)get_bits128(w, 65, 3) : (int)get_bits128(w, 68 + 4 * (i - 1), 4));
            L.a[i] = L.aa[i] = 1.0f - (float)wt / 64.0f;
            if (decoded)
                decoded[i] = pack_rgba(lerp64(ep[0][0], ep[1][0], wt), lerp64(ep[0][1], ep[1][1], wt), lerp64(ep[0][2], ep[1][2], wt),
                                       lerp64(ep[0][3], ep[1][3], wt));
        }
        return;
    }
    dec::Bc7Fields F;
    L.covered = dec::bc7_parse(w, F);
    L.mode = F.mode;
    if (!L.covered) {  // reserved mode: decodes to 0, zero gradient
        #pragma unroll
        for (int i = 0; i < 16; i++) { L.a[i] = L.aa[i] = 0.0f; if (decoded) decoded[i] = 0u; }
        for (int k = 0; k < 6; k++) for (int c = 0; c < 4; c++) e[k][c] = 0.0f;
        return;
    }
    L.rot = F.rot;
    L.alpha_fixed = !F.ab;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        L.a[i] = 1.0f - (float)F.cw[i] / 64.0f;
        L.aa[i] = 1.0f - (float)F.aw[i] / 64.0f;
        L.s1 |= (uint32_t)(F.subset[i] == 1) << i;
        L.s2 |= (uint32_t)(F.subset[i] == 2) << i;
        if (decoded) {  // the decoder's texel (dec::bc7_block), from the same fields
            const int sb = F.subset[i];
            int px[4];
            for (int c = 0; c < 3; c++) px[c] = lerp64(F.ep[2 * sb][c], F.ep[2 * sb + 1][c], F.cw[i]);
            px[3] = lerp64(F.ep[2 * sb][3], F.ep[2 * sb + 1][3], F.aw[i]);
            if (F.rot) { int tmp = px[3]; px[3] = px[F.rot - 1]; px[F.rot - 1] = tmp; }
            decoded[i] = pack_rgba(px[0], px[1], px[2], px[3]);
        }
    }
    for (int k = 0; k < 6; k++) for (int c = 0; c < 4; c++) e[k][c] = (float)F.ep[k][c];
}

// stored channel of decoded channel c (the rotation swaps alpha with channel rot - 1 after the interpolation)
ZTC_DEV int stored_channel(int rot, int c) { return rot == 0 ? c : c == 3 ? rot - 1 : c == rot - 1 ? 3 : c; }
ZTC_DEV int subset_of_texel(const LinBlock &L, int i) { return ((L.s1 >> i) & 1u) ? 1 : ((L.s2 >> i) & 1u) ? 2 : 0; }

__global__ void endpoints_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, float *__restrict__ ep) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    LinBlock L;
    float e[6][4];
    linear_form(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), L, e);
    const int nf = endpoint_floats(fmt);
    for (int k = 0; k < nf / 4; k++) for (int c = 0; c < 4; c++) ep[(size_t)b * nf + 4 * k + c] = e[k][c];
}

__global__ void decode_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, const float *__restrict__ ep, float *__restrict__ out) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    LinBlock L;
    float e[6][4];
    linear_form(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), L, e);
    const int nf = endpoint_floats(fmt);
    const float *E = ep + (size_t)b * nf;
    for (int i = 0; i < 16; i++) {
        const int s = subset_of_texel(L, i);
        for (int c = 0; c < 4; c++) {
            const int sc = stored_channel(L.rot, c);
            float d = 0.0f;
            if (L.covered && c < L.nc && !((L.black >> i) & 1u)) {
                if (sc == 3 && L.alpha_fixed) d = 255.0f;
                else {
                    const float a = sc == 3 ? L.aa[i] : L.a[i];
                    d = a * E[4 * (2 * s) + sc] + (1.0f - a) * E[4 * (2 * s + 1) + sc];
                }
            }
            out[((size_t)b * 16 + i) * 4 + c] = d;
        }
    }
}

__global__ void adjoint_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, const float *__restrict__ g, float *__restrict__ ge) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    LinBlock L;
    float e[6][4], G[6][4];
    linear_form(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), L, e);
    for (int k = 0; k < 6; k++) for (int c = 0; c < 4; c++) G[k][c] = 0.0f;
    for (int i = 0; i < 16; i++) {
        const int s = subset_of_texel(L, i);
        for (int c = 0; c < 4; c++) {
            const int sc = stored_channel(L.rot, c);
            if (!L.covered || c >= L.nc || (sc == 3 && L.alpha_fixed) || ((L.black >> i) & 1u)) continue;
            const float gi = g[((size_t)b * 16 + i) * 4 + c], a = sc == 3 ? L.aa[i] : L.a[i];
            G[2 * s][sc] += a * gi;
            G[2 * s + 1][sc] += (1.0f - a) * gi;
        }
    }
    const int nf = endpoint_floats(fmt);
    for (int k = 0; k < nf / 4; k++) for (int c = 0; c < 4; c++) ge[(size_t)b * nf + 4 * k + c] = G[k][c];
}

// ---------------------------------------------------------------- refinement: requantise and re-fit per mode
ZTC_DEV uint32_t q565(float r, float g, float b) {  // zap_tex.h:45-49
    int R = f2i_x86(r * 31.0f / 255.0f + 0.5f), G = f2i_x86(g * 63.0f / 255.0f + 0.5f), B = f2i_x86(b * 31.0f / 255.0f + 0.5f);
    return ((uint32_t)clampi(R, 0, 31) << 11) | ((uint32_t)clampi(G, 0, 63) << 5) | (uint32_t)clampi(B, 0, 31);
}
ZTC_DEV void bc1_palette(uint32_t c0, uint32_t c1, int pal[4][3]) {
    for (int k = 0; k < 2; k++) {
        uint32_t c = k ? c1 : c0;
        int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
        pal[k][0] = (R << 3) | (R >> 2); pal[k][1] = (G << 2) | (G >> 4); pal[k][2] = (B << 3) | (B >> 2);
    }
    for (int c = 0; c < 3; c++) {
        int a = pal[0][c], b = pal[1][c];
        pal[2][c] = (2 * a + b + 1) / 3; pal[3][c] = (a + 2 * b + 1) / 3;
    }
}
// Nearest palette entry by squared distance over a texel's bytes: |t - p|^2 = |t|^2 + |p|^2 - 2 t.p, so with |t|^2
// fixed the entry minimising |p|^2 - 2 t.p wins (the first of equals, as in a plain scan); each candidate costs one
// four-byte dot product. Entries hold zero in the bytes the distance leaves out. Returns the index; `dist` gets
// |t - p|^2 for the texel's bytes masked like the entries.
template <int N>
ZTC_DEV int nearest_entry(uint32_t t, const uint32_t pal[N], const int pp[N], int tt, int &dist) {
    int bj = 0, be = 1 << 30;
    #pragma unroll
    for (int j = 0; j < N; j++) {
        const int s = pp[j] - 2 * (int)dot4(t, pal[j]);
        if (s < be) { be = s; bj = j; }
    }
    dist = be + tt;
    return bj;
}
template <int N>
ZTC_DEV void entry_norms(const uint32_t pal[N], int pp[N]) {
    #pragma unroll
    for (int j = 0; j < N; j++) pp[j] = (int)dot4(pal[j], pal[j]);
}

// canonical BC1 block for endpoints (c0 > c1 with best indices, or solid) and its SSE
ZTC_DEV int bc1_block_sse(const uint32_t t[16], uint32_t c0, uint32_t c1, uint2 &blk) {
    if (c0 < c1) { uint32_t s = c0; c0 = c1; c1 = s; }
    int pal[4][3], pp[4], err = 0;
    bc1_palette(c0, c1, pal);
    uint32_t pk[4];
    #pragma unroll
    for (int k = 0; k < 4; k++) pk[k] = pack_rgb(pal[k][0], pal[k][1], pal[k][2]);
    if (c0 == c1) pk[1] = pk[2] = pk[3] = pk[0];  // solid: every texel takes index 0 (the first of equals)
    entry_norms<4>(pk, pp);
    uint32_t bits = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t ti = t[i] & 0xFFFFFFu;
        int d;
        const int bk = nearest_entry<4>(ti, pk, pp, (int)dot4(ti, ti), d);
        bits |= (uint32_t)bk << (2 * i);
        err += d;
    }
    blk = make_uint2(c0 | (c1 << 16), bits);
    return err;
}

// nearest n-bit code (no p-bit) whose expansion is closest to v: the rounded guess and its neighbours
ZTC_DEV int quant_plain(float v, int n) {
    const int top = (1 << n) - 1;
    const int g = f2i_x86(v * (float)top / 255.0f + 0.5f);
    int bq = 0;
    float bd = 3.0e38f;
    #pragma unroll
    for (int k = 0; k < 3; k++) {
        const int q = clampi(around(g, k), 0, top);
        const float d = fabsf((float)expand_bits(q, n) - v);
        if (d < bd) { bd = d; bq = q; }
    }
    return bq;
}
// nearest (n-1)-bit code q with a fixed p-bit p, whose n-bit value (q << 1) | p expands closest to v; its distance
ZTC_DEV int quant_pbit(float v, int n, int p, float &dist) {
    const int top = (1 << (n - 1)) - 1;
    const int g = f2i_x86(((v * (float)((1 << n) - 1) / 255.0f) - (float)p) / 2.0f + 0.5f);
    int bq = 0;
    float bd = 3.0e38f;
    #pragma unroll
    for (int k = 0; k < 3; k++) {
        const int q = clampi(around(g, k), 0, top);
        const float d = fabsf((float)expand_bits((q << 1) | p, n) - v);
        if (d < bd) { bd = d; bq = q; }
    }
    dist = bd;
    return bq;
}

// BC7 mode 6 (zap_tex.h:520-527 layout): 7 bits + a p-bit per endpoint, 4-bit indices, anchor texel 0
ZTC_DEV int mode6_block_sse(const uint32_t t[16], const float e[6][4], uint4 &out) {
    int q[2][4], pb[2], x[2][4];
    #pragma unroll
    for (int k = 0; k < 2; k++) {
        float best = 3.0e38f;
        #pragma unroll
        for (int p = 0; p < 2; p++) {
            int qq[4];
            float err = 0.0f, d;
            #pragma unroll
            for (int c = 0; c < 4; c++) { qq[c] = quant_pbit(e[k][c], 8, p, d); err += d * d; }
            if (err < best) {
                best = err; pb[k] = p;
                #pragma unroll
                for (int c = 0; c < 4; c++) q[k][c] = qq[c];
            }
        }
        #pragma unroll
        for (int c = 0; c < 4; c++) x[k][c] = expand_bits((q[k][c] << 1) | pb[k], 8);
    }
    uint32_t pal[16];
    int pp[16];
    #pragma unroll
    for (int j = 0; j < 16; j++)
        pal[j] = pack_rgba(lerp64(x[0][0], x[1][0], w4(j)), lerp64(x[0][1], x[1][1], w4(j)), lerp64(x[0][2], x[1][2], w4(j)),
                           lerp64(x[0][3], x[1][3], w4(j)));
    entry_norms<16>(pal, pp);
    int idx[16], err = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        int d;
        idx[i] = nearest_entry<16>(t[i], pal, pp, (int)dot4(t[i], t[i]), d);
        err += d;
    }
    if (idx[0] >= 8) {  // anchor: swap the endpoints, mirror the indices (decoded values unchanged)
        #pragma unroll
        for (int c = 0; c < 4; c++) { int s = q[0][c]; q[0][c] = q[1][c]; q[1][c] = s; }
        int s = pb[0]; pb[0] = pb[1]; pb[1] = s;
        #pragma unroll
        for (int i = 0; i < 16; i++) idx[i] = 15 - idx[i];
    }
    Bits128 o;
    o.put(1u << 6, 7);
    #pragma unroll
    for (int c = 0; c < 4; c++) { o.put((uint32_t)q[0][c], 7); o.put((uint32_t)q[1][c], 7); }
    o.put((uint32_t)pb[0], 1); o.put((uint32_t)pb[1], 1);
    o.put((uint32_t)idx[0], 3);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((uint32_t)idx[i], 4);
    out = make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
    return err;
}

// BC7 mode 5 (zap_tex.h:597-684): rotation kept, 7-bit colour and 8-bit alpha endpoints (stored order), 2-bit
// colour and alpha indices, each set with its anchor at texel 0; ts: the texels in stored channel order
ZTC_DEV int mode5_block_sse(const uint32_t ts[16], const float e[6][4], int rot, uint4 &out) {
    int q[2][4], x[2][4];
    #pragma unroll
    for (int k = 0; k < 2; k++) {
        #pragma unroll
        for (int c = 0; c < 3; c++) { q[k][c] = quant_plain(e[k][c], 7); x[k][c] = expand_bits(q[k][c], 7); }
        q[k][3] = x[k][3] = clampi(f2i_x86(e[k][3] + 0.5f), 0, 255);
    }
    uint32_t pal[4];
    int pp[4], pa[4];
    #pragma unroll
    for (int j = 0; j < 4; j++) {
        pal[j] = pack_rgb(lerp64(x[0][0], x[1][0], w2(j)), lerp64(x[0][1], x[1][1], w2(j)), lerp64(x[0][2], x[1][2], w2(j)));
        pa[j] = lerp64(x[0][3], x[1][3], w2(j));
    }
    entry_norms<4>(pal, pp);
    int ci[16], ai[16], err = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t tc = ts[i] & 0xFFFFFFu;
        int d;
        ci[i] = nearest_entry<4>(tc, pal, pp, (int)dot4(tc, tc), d);
        const int ta = (int)(ts[i] >> 24);
        int bk = 0, bae = 1 << 30;
        #pragma unroll
        for (int j = 0; j < 4; j++) {
            const int y = ta - pa[j];
            if (y * y < bae) { bae = y * y; bk = j; }
        }
        ai[i] = bk;
        err += d + bae;
    }
    if (ci[0] >= 2) {
        #pragma unroll
        for (int c = 0; c < 3; c++) { int s = q[0][c]; q[0][c] = q[1][c]; q[1][c] = s; }
        #pragma unroll
        for (int i = 0; i < 16; i++) ci[i] = 3 - ci[i];
    }
    if (ai[0] >= 2) {
        int s = q[0][3]; q[0][3] = q[1][3]; q[1][3] = s;
        #pragma unroll
        for (int i = 0; i < 16; i++) ai[i] = 3 - ai[i];
    }
    Bits128 o;
    o.put(1u << 5, 6);
    o.put((uint32_t)rot, 2);
    #pragma unroll
    for (int c = 0; c < 3; c++) { o.put((uint32_t)q[0][c], 7); o.put((uint32_t)q[1][c], 7); }
    o.put((uint32_t)q[0][3], 8); o.put((uint32_t)q[1][3], 8);
    o.put((uint32_t)ci[0], 1);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((uint32_t)ci[i], 2);
    o.put((uint32_t)ai[0], 1);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((uint32_t)ai[i], 2);
    out = make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
    return err;
}

// BC7 mode 1 (zap_tex.h:687-708): partition kept, two subsets of 6-bit RGB endpoints with one p-bit per subset,
// 3-bit indices, anchors at texel 0 and at the partition's second-subset anchor; alpha decodes to 255
ZTC_DEV int mode1_block_sse(const uint32_t t[16], const float e[6][4], int part, uint4 &out) {
#ifdef __CUDA_ARCH__
    const uint32_t mask = dec::kP2d[part];
    const int anchor1 = dec::kA2d[part];
#else
    const uint32_t mask = 0u;
    const int anchor1 = 15;
#endif
    int q[4][3], pb[2], x[4][3];
    #pragma unroll
    for (int s = 0; s < 2; s++) {
        float best = 3.0e38f;
        #pragma unroll
        for (int p = 0; p < 2; p++) {
            int qq[2][3];
            float err = 0.0f, d;
            #pragma unroll
            for (int k = 0; k < 2; k++)
                #pragma unroll
                for (int c = 0; c < 3; c++) { qq[k][c] = quant_pbit(e[2 * s + k][c], 7, p, d); err += d * d; }
            if (err < best) {
                best = err; pb[s] = p;
                #pragma unroll
                for (int k = 0; k < 2; k++)
                    #pragma unroll
                    for (int c = 0; c < 3; c++) q[2 * s + k][c] = qq[k][c];
            }
        }
        #pragma unroll
        for (int k = 0; k < 2; k++)
            #pragma unroll
            for (int c = 0; c < 3; c++) x[2 * s + k][c] = expand_bits((q[2 * s + k][c] << 1) | pb[s], 7);
    }
    uint32_t pal[2][8];
    int pp[2][8];
    #pragma unroll
    for (int s = 0; s < 2; s++) {
        #pragma unroll
        for (int j = 0; j < 8; j++)
            pal[s][j] = pack_rgb(lerp64(x[2 * s][0], x[2 * s + 1][0], w3(j)), lerp64(x[2 * s][1], x[2 * s + 1][1], w3(j)),
                                 lerp64(x[2 * s][2], x[2 * s + 1][2], w3(j)));
        entry_norms<8>(pal[s], pp[s]);
    }
    int idx[16], err = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        const uint32_t tc = t[i] & 0xFFFFFFu;
        const bool s1 = (mask >> i) & 1u;
        uint32_t ps[8];
        int qs[8];
        #pragma unroll
        for (int j = 0; j < 8; j++) { ps[j] = s1 ? pal[1][j] : pal[0][j]; qs[j] = s1 ? pp[1][j] : pp[0][j]; }
        int d;
        idx[i] = nearest_entry<8>(tc, ps, qs, (int)dot4(tc, tc), d);
        const int ya = (int)chan(t[i], 3) - 255;
        err += d + ya * ya;
    }
    #pragma unroll
    for (int s = 0; s < 2; s++) {
        const int anchor = s ? anchor1 : 0;
        int ia = idx[0];
        #pragma unroll
        for (int i = 1; i < 16; i++) if (i == anchor) ia = idx[i];
        if (ia < 4) continue;
        #pragma unroll
        for (int c = 0; c < 3; c++) { int v = q[2 * s][c]; q[2 * s][c] = q[2 * s + 1][c]; q[2 * s + 1][c] = v; }
        #pragma unroll
        for (int i = 0; i < 16; i++) if ((int)((mask >> i) & 1u) == s) idx[i] = 7 - idx[i];
    }
    Bits128 o;
    o.put(1u << 1, 2);
    o.put((uint32_t)part, 6);
    #pragma unroll
    for (int c = 0; c < 3; c++)
        #pragma unroll
        for (int k = 0; k < 4; k++) o.put((uint32_t)q[k][c], 6);
    o.put((uint32_t)pb[0], 1); o.put((uint32_t)pb[1], 1);
    #pragma unroll
    for (int i = 0; i < 16; i++) o.put((uint32_t)idx[i], (i == 0 || i == anchor1) ? 2 : 3);
    out = make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
    return err;
}

// mode 5's rotation on a texel (swap A with R, G or B): decoded order <-> stored order
ZTC_DEV uint32_t swap_alpha(uint32_t v, int rot) {
    if (!rot) return v;
    const int sh = 8 * (rot - 1);
    const uint32_t a = v >> 24, c = (v >> sh) & 0xFFu;
    return (v & ~((0xFFu << sh) | 0xFF000000u)) | (a << sh) | (c << 24);
}

// `steps` Adam steps on the block's MSE through the adjoint, in stored channel order (the rotation only permutes
// channels, so the squared error is the same). NS subsets move: 1 (BC1, BC7 modes 6 and 5: endpoints 0 and 1) or
// 2 (mode 1: a texel of subset 1 moves endpoints 2 and 3); mode 1's alpha is fixed at 255 and not a parameter.
// Through the linear decode the gradient is affine in the endpoints. With a a texel's weight, b = 1 - a and t its
// value, per subset s and channel c
//   dL/dE[2s][c]   = n (Saa E[2s][c] + Sab E[2s+1][c] - Sat[c])
//   dL/dE[2s+1][c] = n (Sab E[2s][c] + Sbb E[2s+1][c] - Sbt[c]),   n = 2 / (16 nc)
// summed over the subset's texels (constant texels left out; alpha with its own weights), so the moments are summed
// once and a step costs a few operations per endpoint channel. Adam keeps its usual form, with eps^2 added under
// the root of the second moment rather than eps after it.
template <int NS>
ZTC_DEV void adam_refine(const LinBlock &L, const uint32_t ts[16], float e[6][4], int steps, float lr) {
    const int npar = L.alpha_fixed ? 3 : L.nc;
    float W[NS][2][3], T[NS][2][4];  // W[s][colour, alpha][aa, ab, bb]; T[s][a, b][c]
    #pragma unroll
    for (int s = 0; s < NS; s++)
        #pragma unroll
        for (int k = 0; k < 2; k++) {
            #pragma unroll
            for (int j = 0; j < 3; j++) W[s][k][j] = 0.0f;
            #pragma unroll
            for (int c = 0; c < 4; c++) T[s][k][c] = 0.0f;
        }
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        if ((L.black >> i) & 1u) continue;  // a constant: no gradient
        const bool in1 = NS == 2 && ((L.s1 >> i) & 1u);
        float w[2][3], tv[2][4];
        #pragma unroll
        for (int k = 0; k < 2; k++) {
            const float a = k ? L.aa[i] : L.a[i], b = 1.0f - a;
            w[k][0] = a * a; w[k][1] = a * b; w[k][2] = b * b;
        }
        #pragma unroll
        for (int c = 0; c < 4; c++) {
            const float a = c == 3 ? L.aa[i] : L.a[i], t = (float)chan(ts[i], c);
            tv[0][c] = a * t; tv[1][c] = (1.0f - a) * t;
        }
        #pragma unroll
        for (int s = 0; s < NS; s++) {
            if ((s == 1) != in1) continue;
            #pragma unroll
            for (int k = 0; k < 2; k++) {
                #pragma unroll
                for (int j = 0; j < 3; j++) W[s][k][j] += w[k][j];
                #pragma unroll
                for (int c = 0; c < 4; c++) T[s][k][c] += tv[k][c];
            }
        }
    }
    float m[NS][2][4], v[NS][2][4];
    #pragma unroll
    for (int s = 0; s < NS; s++)
        #pragma unroll
        for (int k = 0; k < 2; k++)
            #pragma unroll
            for (int c = 0; c < 4; c++) m[s][k][c] = v[s][k][c] = 0.0f;
    const float b1 = 0.9f, b2 = 0.999f, n = 2.0f / (16.0f * (float)L.nc);
    float p1 = 1.0f, p2 = 1.0f;
    #pragma unroll 1
    for (int st = 0; st < steps; st++) {
        p1 *= b1; p2 *= b2;
        const float c1 = lr / (1.0f - p1), c2 = 1.0f / (1.0f - p2);  // bias corrections
        #pragma unroll
        for (int s = 0; s < NS; s++)
            #pragma unroll
            for (int c = 0; c < 4; c++) {
                if (c >= npar) continue;
                const float *Wk = W[s][c == 3 ? 1 : 0];
                const float e0 = e[2 * s][c], e1 = e[2 * s + 1][c];
                const float g[2] = {n * (Wk[0] * e0 + Wk[1] * e1 - T[s][0][c]), n * (Wk[1] * e0 + Wk[2] * e1 - T[s][1][c])};
                #pragma unroll
                for (int k = 0; k < 2; k++) {
                    m[s][k][c] = b1 * m[s][k][c] + (1.0f - b1) * g[k];
                    v[s][k][c] = b2 * v[s][k][c] + (1.0f - b2) * g[k] * g[k];
                    const float upd = c1 * m[s][k][c] * rsqrtf(v[s][k][c] * c2 + 1e-16f);
                    e[2 * s + k][c] = fminf(255.0f, fmaxf(0.0f, e[2 * s + k][c] - upd));
                }
            }
    }
}

// 4 resident CTAs of 128 threads per SM
__global__ void __launch_bounds__(128, 4) refine_kernel(int fmt, SrcU8 src, int bw, int nblocks, uint8_t *__restrict__ blocks, int steps,
                                                        float lr, uint32_t *__restrict__ sse0, uint32_t *__restrict__ sse1) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const size_t bs = fmt == ZTC_FMT_BC1 ? 8 : 16;
    uint8_t *blk = blocks + (size_t)b * bs;
    uint32_t t[16], d[16];
    gather_block(src, b % bw, b / bw, t);
    LinBlock L;
    float e[6][4];
    linear_form(fmt, blk, L, e, d);  // one parse: the linear form and the decoder's texels
    const int nce = fmt == ZTC_FMT_BC1 ? 3 : 4;
    int before = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++)
        #pragma unroll
        for (int c = 0; c < 4; c++)
            if (c < nce) { const int x = (int)chan(t[i], c) - (int)chan(d[i], c); before += x * x; }
    int after = before;
    const bool refinable = fmt == ZTC_FMT_BC1 || L.mode == 6 || L.mode == 5 || L.mode == 1;
    if (refinable && before > 0) {
        uint32_t ts[16];
        #pragma unroll
        for (int i = 0; i < 16; i++) ts[i] = swap_alpha(t[i], L.rot);
        if (L.s1) adam_refine<2>(L, ts, e, steps, lr);
        else adam_refine<1>(L, ts, e, steps, lr);
        int ne = 1 << 30;
        if (fmt == ZTC_FMT_BC1) {
            uint2 nb;
            ne = bc1_block_sse(t, q565(e[0][0], e[0][1], e[0][2]), q565(e[1][0], e[1][1], e[1][2]), nb);
            if (ne < before) *(uint2 *)blk = nb;
        } else {
            uint4 nb;
            if (L.mode == 6) ne = mode6_block_sse(t, e, nb);
            else if (L.mode == 5) ne = mode5_block_sse(ts, e, L.rot, nb);
            else ne = mode1_block_sse(t, e, (int)get_bits128((const uint32_t *)blk, 2, 6), nb);
            if (ne < before) *(uint4 *)blk = nb;
        }
        if (ne < before) after = ne;
    }
    if (sse0) sse0[b] = (uint32_t)before;
    if (sse1) sse1[b] = (uint32_t)after;
}

}  // namespace ztc

// ---------------------------------------------------------------- C ABI
static int adj_check(int fmt, const void *p, int n) {
    if (fmt != ZTC_BC1 && fmt != ZTC_BC7) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "differentiable decode covers BC1 and BC7");
    if (!p || n < 0) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null pointer or negative block count");
    if ((uintptr_t)p % (fmt == ZTC_BC1 ? 8u : 16u)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "blocks must be aligned to the block size");
    return ZTC_OK;
}
static bool floats_misaligned(const void *a, const void *b = nullptr) { return ((uintptr_t)a | (uintptr_t)b) & 3u; }
static int launch_status(const char *what) {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZTC_OK : ztc_set_error(ZTC_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

extern "C" {

int zap_tex_cuda_block_endpoints_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, float *endpoints, void *stream) {
    ZTC_NVTX();
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!endpoints || floats_misaligned(endpoints)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned endpoints");
    if (nblocks) ztc::endpoints_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, endpoints);
    return launch_status("endpoints launch");
}

int zap_tex_cuda_palette_decode_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *endpoints, float *decoded,
                                    void *stream) {
    ZTC_NVTX();
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!endpoints || !decoded || floats_misaligned(endpoints, decoded))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned endpoints / decoded");
    if (nblocks) ztc::decode_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, endpoints, decoded);
    return launch_status("decode launch");
}

int zap_tex_cuda_palette_adjoint_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *grad_decoded,
                                     float *grad_endpoints, void *stream) {
    ZTC_NVTX();
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!grad_decoded || !grad_endpoints || floats_misaligned(grad_decoded, grad_endpoints))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned gradient pointer");
    if (nblocks)
        ztc::adjoint_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, grad_decoded,
                                                                                   grad_endpoints);
    return launch_status("adjoint launch");
}

int zap_tex_cuda_refine_dev(zap_tex_cuda_ctx *ctx, int fmt, const uint8_t *rgba, int w, int h, size_t stride, void *blocks, int steps,
                            float lr, uint32_t *sse_before, uint32_t *sse_after, void *stream) {
    ZTC_NVTX();
    int st = adj_check(fmt, blocks, 0);
    if (st) return st;
    if (!rgba || w < 1 || h < 1 || stride < (size_t)w * 4 || steps < 0 || steps > 1000 || !(lr >= 0.0f))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad image, steps or learning rate");
    if (floats_misaligned(sse_before, sse_after)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "misaligned SSE outputs");
    if ((st = ztc_ctx_activate(ctx))) return st;
    const int bw = (w + 3) / 4, nblocks = bw * ((h + 3) / 4);
    ztc::SrcU8 src{rgba, stride, w, h, 4, (((uintptr_t)rgba | stride) & 15u) == 0};
    ztc::TraceScope tr(fmt == ZTC_BC1 ? "refine_bc1" : "refine_bc7", (cudaStream_t)stream);
    ztc::trace_units(nblocks);
    ztc::refine_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, src, bw, nblocks, (uint8_t *)blocks, steps, lr, sse_before,
                                                                               sse_after);
    return launch_status("refine launch");
}

}  // extern "C"

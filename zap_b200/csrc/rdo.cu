// rdo.cu - rate-distortion encoding at lambda > 0 (zap_tex.h:223-306, :786-815) for sm_100a, bit-exact.
//
// The reference picks every sub-block among its own encoding and up to 48 candidates rebuilt from the 16 blocks
// chosen before it in the call's raster order (a neighbour's endpoints with refit indices, its indices with these
// endpoints, or the whole neighbour; for BC7: the whole neighbour, or for a mode-6 neighbour its endpoint bytes
// with refit indices or its index bytes with refit endpoints), minimising SSE + lambda * rate. The rate models
// zap's LZ on the split planes, per field: 0 if the field repeats the one at the current match distance,
// min(size, 3) for a new match in the window, its size in literals otherwise.
//
// Only that window makes the work serial. The base encodings do not depend on it, so the ordinary encoder kernels
// write them for every block first, in parallel. The chain then runs as one CTA per call (or per band of block
// rows: each band is its own call in the reference's banded callers; and per sub-block kind, whose chains are
// independent): per block, 16-lane groups evaluate the candidates side by side, one lane per texel, and a
// CTA-wide minimum of (cost, candidate order) picks the winner. That minimum is the
// reference's choice: its scan takes a candidate only if its cost is below the best so far (strict "<"), so it ends
// on the first candidate of the lowest cost, and its early "skip if SSE >= best" never changes that, because
// SSE + lambda * rate >= SSE in float arithmetic when lambda * rate >= 0 (finite lambda > 0: the entry points reject
// any other lambda). Costs are non-negative floats, whose bit patterns order like their values. The window of the
// last 16 chosen sub-blocks lives in shared memory; chosen blocks overwrite the base encodings in place.
#include "ztc_common.cuh"
#include "ztc_decode.cuh"
#include "ztc_internal.h"

namespace ztc {
namespace {

constexpr int kWindow = 16;          // ZAP_TEX_WINDOW (zap_tex.h:227)

enum SubType { kBc1 = 0, kBc4 = 1, kBc7 = 2 };
struct Sub {
    int type, chan, force4, off;  // chan: the BC4 channel; off: byte offset of the sub-block in the block
};
// the sub-blocks of a format's block, in the order the reference encodes them (zap_tex.h:1489-1503)
__host__ __device__ constexpr int sub_count(int fmt) { return fmt == ZTC_FMT_BC3 || fmt == ZTC_FMT_BC5 ? 2 : 1; }
__host__ __device__ constexpr Sub sub_of(int fmt, int s) {
    return fmt == ZTC_FMT_BC1   ? Sub{kBc1, 0, 0, 0}
           : fmt == ZTC_FMT_BC3 ? (s == 0 ? Sub{kBc4, 3, 0, 0} : Sub{kBc1, 0, 1, 8})
           : fmt == ZTC_FMT_BC4 ? Sub{kBc4, 0, 0, 0}
           : fmt == ZTC_FMT_BC5 ? (s == 0 ? Sub{kBc4, 0, 0, 0} : Sub{kBc4, 1, 0, 8})
                                : Sub{kBc7, 0, 0, 0};
}

// ---- BC1 sub-block (zap_tex.h:52-94): u16 c0, u16 c1, 2-bit indices; 3 colours + transparent when c0 <= c1
ZTC_DEV void bc1_entry(uint32_t c0, uint32_t c1, int force4, int k, int &r, int &g, int &b) {
    int r0, g0, b0, r1, g1, b1;
    unpack565(c0, r0, g0, b0); unpack565(c1, r1, g1, b1);
    const bool four = force4 || c0 > c1;
    if (k == 0) { r = r0; g = g0; b = b0; }
    else if (k == 1) { r = r1; g = g1; b = b1; }
    else if (k == 2) {
        if (four) { r = (2 * r0 + r1 + 1) / 3; g = (2 * g0 + g1 + 1) / 3; b = (2 * b0 + b1 + 1) / 3; }
        else { r = (r0 + r1 + 1) / 2; g = (g0 + g1 + 1) / 2; b = (b0 + b1 + 1) / 2; }
    } else {
        if (four) { r = (r0 + 2 * r1 + 1) / 3; g = (g0 + 2 * g1 + 1) / 3; b = (b0 + 2 * b1 + 1) / 3; }
        else { r = g = b = 0; }
    }
}
// ---- BC4 sub-block (zap_tex.h:172-196): u8 a0, u8 a1, 3-bit indices; 6 values + 0 and 255 when a0 <= a1
ZTC_DEV int bc4_entry(int a0, int a1, int k) {
    if (k == 0) return a0;
    if (k == 1) return a1;
    if (a0 > a1) return ((8 - k) * a0 + (k - 1) * a1 + 3) / 7;
    return k < 6 ? ((6 - k) * a0 + (k - 1) * a1 + 2) / 5 : k == 6 ? 0 : 255;
}
// ---- BC7 mode-6 blocks (zap_tex.h:529)
ZTC_DEV bool is_mode6(uint64_t lo) { return (lo & 0x7Fu) == 0x40u; }
// mode-6 fields: q[e][c] 7 bits each (c-major), p-bits, 4-bit indices (texel 0: 3 bits) packed into idx, 4 bits each
__device__ __forceinline__ uint64_t key_of(float cost, int order) { return ((uint64_t)__float_as_uint(cost) << 32) | (uint32_t)order; }

// ---------------------------------------------------------------- BC7: one lane per texel
// A BC7 candidate costs a whole palette search or least-squares solve, so this chain spreads each candidate over a
// 16-lane group: lane i takes texel i (and window slot i when the rate is counted). 25 warps = 50 groups:
// groups 0-15 kind 1 (neighbour j = group + 1: its endpoints, refit indices), 16-31 kind 2 (its indices, refit
// endpoints), 32-47 kind 0 (the whole neighbour), 48 the base, 49 loads the next block. Every chosen block enters
// the window with its decoded texels and, for mode 6, its palette and indices, so no candidate decodes a block:
// kind 0 compares the texels with the stored decode, kind 1 searches the stored palette. The base encodings are
// decoded for every block by a parallel pass before the chains. Kind 2's least-squares sums are exact in the
// reference's float accumulation (weights k/64, texels integers: every partial sum is a multiple of 1/4096 below
// 2^17 of them), so they are reduced as integers and scaled, which gives the same floats in any order.
constexpr int kB7Warps = 25, kB7Threads = kB7Warps * 32;

// Group collectives over a 16-lane group: gm names the caller's half-warp (each half of a warp passes its own
// mask, as 16-thread tiles do). ZTC_RDO_REDUX selects redux.sync (1) or xor-shuffle trees (0) for the sums and ORs;
// ZTC_RDO_MIN_REDUX the same for the warp-wide key minimum.
#ifndef ZTC_RDO_REDUX
#define ZTC_RDO_REDUX 0
#endif
#ifndef ZTC_RDO_MIN_REDUX
#define ZTC_RDO_MIN_REDUX 1
#endif
__device__ __forceinline__ int grp_sum(int v, unsigned gm) {
#if ZTC_RDO_REDUX
    return __reduce_add_sync(gm, v);
#else
    #pragma unroll
    for (int m = 8; m >= 1; m >>= 1) v += __shfl_xor_sync(gm, v, m, 16);
    return v;
#endif
}
__device__ __forceinline__ uint64_t grp_or64(uint64_t v, unsigned gm) {
#if ZTC_RDO_REDUX
    return ((uint64_t)__reduce_or_sync(gm, (uint32_t)(v >> 32)) << 32) | __reduce_or_sync(gm, (uint32_t)v);
#else
    #pragma unroll
    for (int m = 8; m >= 1; m >>= 1) {
        const uint32_t lo = __shfl_xor_sync(gm, (uint32_t)v, m, 16), hi = __shfl_xor_sync(gm, (uint32_t)(v >> 32), m, 16);
        v |= ((uint64_t)hi << 32) | lo;
    }
    return v;
#endif
}
// The mask a lane passes to its group's collectives: its half-warp, or (ZTC_RDO_FULL_MASK) the whole warp in
// warps 0-23, whose two groups run the same kind of candidate and meet every collective together; warp 24
// splits into the base and the loader, which run different code. Whole-warp masks measured faster on B200
// (512x512 one chain: BC7 30.6 -> 28.3 ms, BC1 25.8 -> 25.5 ms).
#ifndef ZTC_RDO_FULL_MASK
#define ZTC_RDO_FULL_MASK 1
#endif
__device__ __forceinline__ unsigned group_mask(int warp, int lane) {
    return ZTC_RDO_FULL_MASK && warp < 24 ? 0xFFFFFFFFu : 0xFFFFu << (lane & 16);
}
// warp-wide minimum of 64-bit keys
__device__ __forceinline__ uint64_t warp_min_redux(uint64_t k) {
#if ZTC_RDO_MIN_REDUX  // the high words' minimum, then the low words' among the lanes holding it
    const uint32_t hi = __reduce_min_sync(0xFFFFFFFFu, (uint32_t)(k >> 32));
    const uint32_t lo = __reduce_min_sync(0xFFFFFFFFu, (uint32_t)(k >> 32) == hi ? (uint32_t)k : 0xFFFFFFFFu);
    return ((uint64_t)hi << 32) | lo;
#else  // xor-shuffle tree
    #pragma unroll
    for (int m = 16; m >= 1; m >>= 1) {
        const uint32_t lo = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)k, m), hi = __shfl_xor_sync(0xFFFFFFFFu, (uint32_t)(k >> 32), m);
        const uint64_t o = ((uint64_t)hi << 32) | lo;
        k = o < k ? o : k;
    }
    return k;
#endif
}
ZTC_DEV int sq4px(uint32_t a, uint32_t b) {  // squared RGBA difference (zap__sq4 over 4 channels)
    int s = 0;
    #pragma unroll
    for (int c = 0; c < 4; c++) { const int d = (int)chan(a, c) - (int)chan(b, c); s += d * d; }
    return s;
}
ZTC_DEV uint32_t lerp_px(const int x0[4], const int x1[4], int w) {
    return pack_rgba(lerp64(x0[0], x1[0], w), lerp64(x0[1], x1[1], w), lerp64(x0[2], x1[2], w), lerp64(x0[3], x1[3], w));
}
// mode 6 bit layout: mode bits 0-6, R0 R1 G0 G1 B0 B1 A0 A1 (7 bits each) from bit 7, P0 bit 63, P1 bit 64, then
// the indices (texel 0: 3 bits, the others 4) from bit 65
ZTC_DEV void mode6_ends_of(uint64_t lo, uint64_t hi, int x0[4], int x1[4]) {  // expanded endpoints
    const int p0 = (int)(lo >> 63), p1 = (int)(hi & 1u);
    #pragma unroll
    for (int c = 0; c < 4; c++) {
        x0[c] = (int)(((lo >> (7 + 14 * c)) & 0x7Fu) << 1) | p0;
        x1[c] = (int)(((lo >> (14 + 14 * c)) & 0x7Fu) << 1) | p1;
    }
}
ZTC_DEV uint64_t mode6_idx_of(uint64_t hi) { return ((hi >> 1) & 7u) | (hi & ~0xFull); }  // 4 bits per texel
ZTC_DEV uint64_t mode6_hi(int p1, uint64_t idx) { return (uint64_t)p1 | ((idx & 7u) << 1) | (idx & ~0xFull); }

// the base encodings of blocks [0, nblocks), decoded: 16 texels per block
__global__ void __launch_bounds__(128) bc7_decode_bases_kernel(const uint8_t *__restrict__ blocks, int nblocks, uint4 *__restrict__ dec) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const uint4 v = *(const uint4 *)(blocks + (size_t)b * 16);
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    uint32_t px[16];
    dec::bc7_block(w, px);
    #pragma unroll
    for (int k = 0; k < 4; k++) dec[(size_t)b * 4 + k] = make_uint4(px[4 * k], px[4 * k + 1], px[4 * k + 2], px[4 * k + 3]);
}

// the loader group's work for block gk: its texels, decoded base, base and channel sums into slot ns
__device__ __forceinline__ void load_bc7_block(const SrcU8 &src, int bw, const uint8_t *out, const uint32_t *dec_base, int gk, int ns, int i,
                                               unsigned gm, uint32_t (*s_tex)[16], uint32_t (*s_dbase)[16], uint64_t (*s_base)[2],
                                               int (*s_sumx)[4]) {
    const uint32_t t = load_texel(src, min((gk % bw) * 4 + (i & 3), src.w - 1), min((gk / bw) * 4 + (i >> 2), src.h - 1));
    s_tex[ns][i] = t;
    s_dbase[ns][i] = dec_base[(size_t)gk * 16 + i];
    if (i < 2) s_base[ns][i] = *(const uint64_t *)(out + (size_t)gk * 16 + 8 * i);
    #pragma unroll
    for (int c = 0; c < 4; c++) {
        const int sx = grp_sum((int)chan(t, c), gm);
        if (i == c) s_sumx[ns][c] = sx;
    }
}

__global__ void __launch_bounds__(kB7Threads, 1) rdo_bc7_chain_kernel(SrcU8 src, int bw, int nby, int chain_rows, uint8_t *__restrict__ out,
                                                                      const uint32_t *__restrict__ dec_base, float lambda) {
    __shared__ uint64_t ring[kWindow][2];       // the last 16 chosen blocks, slot = block & 15
    __shared__ uint32_t ring_dec[kWindow][16];  // their decoded texels
    __shared__ uint32_t ring_pal[kWindow][16];  // mode 6: their palettes
    __shared__ uint64_t ring_idx[kWindow];      // mode 6: their indices, 4 bits per texel
    __shared__ uint32_t s_tex[3][16], s_dbase[3][16];  // block cur in slot cur % 3, loaded two blocks ahead
    __shared__ uint64_t s_base[3][2];
    __shared__ int s_sumx[3][4];                       // the block's channel sums
    __shared__ uint64_t s_key[kB7Warps];
    __shared__ int s_dist[2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, i = lane & 15, grp = tid >> 4;
    const int kind = grp < 16 ? 1 : grp < 32 ? 2 : grp < 48 ? 0 : grp == 48 ? -1 : -2, j = (grp & 15) + 1;
    const unsigned gm = group_mask(warp, lane);
    const int row0 = blockIdx.x * chain_rows, rows = min(chain_rows, nby - row0);
    if (rows <= 0) return;
    const int first = row0 * bw, count = rows * bw;
    if (kind == -2)
        for (int k = 0; k < 2 && k < count; k++) load_bc7_block(src, bw, out, dec_base, first + k, k, i, gm, s_tex, s_dbase, s_base, s_sumx);
    if (tid == 0) { s_dist[0] = 1; s_dist[1] = 1; }
    __syncthreads();
    for (int cur = 0; cur < count; cur++) {
        const int g = first + cur, slot = cur % 3, d0 = s_dist[0], d1 = s_dist[1];
        uint64_t key = ~0ull, clo = 0, chi = 0, cidx = 0;
        uint32_t dec = 0, pal = 0;
        int nd0 = 0, nd1 = 0;
        if (kind >= -1) {
            const uint32_t t = s_tex[slot][i];
            const int r = (cur - j) & (kWindow - 1);
            bool ok;
            int e;
            if (kind == -1) {  // the base (its SSE: the one the reference's encoder returns)
                clo = s_base[slot][0]; chi = s_base[slot][1];
                dec = s_dbase[slot][i];
                e = grp_sum(sq4px(t, dec), gm);
                int x0[4], x1[4];
                mode6_ends_of(clo, chi, x0, x1);
                pal = lerp_px(x0, x1, w4(i));
                cidx = mode6_idx_of(chi);
                ok = true;
            } else if (kind == 0) {  // the whole neighbour (zap__bc7_err)
                clo = ring[r][0]; chi = ring[r][1];
                dec = ring_dec[r][i]; pal = ring_pal[r][i]; cidx = ring_idx[r];
                e = grp_sum(sq4px(t, dec), gm);
                ok = j <= cur;
            } else if (kind == 1) {  // its endpoints, best indices; texel 0 keeps to 0..7 (zap__bc7_fit6_idx)
                const uint64_t nlo = ring[r][0], nhi = ring[r][1];
                ok = j <= cur && is_mode6(nlo);
                pal = ring_pal[r][i];
                int m = 0x7FFFFFFF;
                #pragma unroll
                for (int k = 0; k < 16; k++) {
                    const uint32_t pk = ring_pal[r][k];
                    const int kk = 16 * ((int)dot4(pk, pk) - 2 * (int)dot4(t, pk)) + k;
                    if ((i || k < 8) && kk < m) { m = kk; dec = pk; }
                }
                e = grp_sum((m >> 4) + (int)dot4(t, t), gm);
                cidx = grp_or64((uint64_t)(m & 15) << (4 * i), gm);
                clo = nlo; chi = mode6_hi((int)(nhi & 1u), cidx);
            } else {  // its indices, least-squares endpoints, each endpoint's own p-bit (zap__bc7_fit6_ep)
                const uint64_t nlo = ring[r][0], nhi = ring[r][1];
                ok = j <= cur && is_mode6(nlo);
                cidx = ring_idx[r];
                const int w = w4((int)((cidx >> (4 * i)) & 15u));
                const int ch = i & 3, ep = (i >> 2) & 1, p = i >> 3;
                // with u = 64 - w: sum u^2 = 16 * 4096 - 128 sum w + sum w^2, sum u w = 64 sum w - sum w^2,
                // sum u x = 64 sum x - sum w x; sum w (<= 1024) and sum w^2 (<= 65536) share one word
                const int W12 = grp_sum((w * w) << 11 | w, gm), W1 = W12 & 0x7FF, W2 = W12 >> 11;
                int SB = 0;
                #pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int sb = grp_sum(w * (int)chan(t, c), gm);
                    if (c == ch) SB = sb;
                }
                const int AA = 16 * 4096 - 128 * W1 + W2, AB = 64 * W1 - W2, BB = W2, SA = 64 * s_sumx[slot][ch] - SB;
                const float aa = (float)AA / 4096.0f, ab = (float)AB / 4096.0f, bb = (float)BB / 4096.0f;
                const float ax = (float)SA / 64.0f, bx = (float)SB / 64.0f, det = aa * bb - ab * ab;
                float v;
                if (det < 1e-6f && det > -1e-6f) v = (ax + bx) / 16.0f;  // one index everywhere: flat
                else v = ep ? (bx * aa - ax * ab) / det : (ax * bb - bx * ab) / det;
                v = clamp255(v);
                // lane (channel, endpoint, p-bit): zap__bc7q for one channel, 7 bits + p
                const int gq = f2i_x86((v / 255.0f * 255.0f - (float)p) / 2.0f + 0.5f);
                int bq = 0, be = 1 << 30;
                #pragma unroll
                for (int k = 0; k < 3; k++) {
                    const int tq = clampi(around(gq, k), 0, 127);
                    const float d = (float)((tq << 1) | p) - v;
                    const int ek = f2i_x86(d * d);
                    if (ek < be) { be = ek; bq = tq; }
                }
                int s4 = be + __shfl_xor_sync(gm, be, 1, 16);
                s4 += __shfl_xor_sync(gm, s4, 2, 16);
                const int e00 = __shfl_sync(gm, s4, 0, 16), e01 = __shfl_sync(gm, s4, 8, 16);
                const int e10 = __shfl_sync(gm, s4, 4, 16), e11 = __shfl_sync(gm, s4, 12, 16);
                const int pb0 = e01 < e00 ? 1 : 0, pb1 = e11 < e10 ? 1 : 0;
                int x0[4], x1[4];
                uint64_t lo = 0x40u | ((uint64_t)pb0 << 63);
                #pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int q0 = __shfl_sync(gm, bq, pb0 * 8 + c, 16), q1 = __shfl_sync(gm, bq, pb1 * 8 + 4 + c, 16);
                    x0[c] = (q0 << 1) | pb0; x1[c] = (q1 << 1) | pb1;
                    lo |= ((uint64_t)q0 << (7 + 14 * c)) | ((uint64_t)q1 << (14 + 14 * c));
                }
                dec = lerp_px(x0, x1, w);
                e = grp_sum(sq4px(t, dec), gm);
                pal = lerp_px(x0, x1, w4(i));
                clo = lo; chi = (nhi & ~1ull) | (uint64_t)pb1;
            }
            // rate (zap__bc7_rate): lane i compares the candidate's fields with window slot j' = i + 1
            const int rw = (cur - i - 1) & (kWindow - 1);
            const bool vw = i + 1 <= cur;
            const uint64_t wlo = ring[rw][0], whi = ring[rw][1];
            const unsigned sh = lane & 16;
            const unsigned mA = (__ballot_sync(gm, vw && wlo == clo) >> sh) & 0xFFFFu;
            const unsigned mB = (__ballot_sync(gm, vw && (whi >> 8) == (chi >> 8)) >> sh) & 0xFFFFu;
            float fa = 8.0f, fb = 7.0f;
            nd0 = d0; nd1 = d1;
            if (d0 > 0 && d0 <= cur && ((mA >> (d0 - 1)) & 1u)) fa = 0.0f;
            else if (mA) { nd0 = __ffs((int)mA); fa = 3.0f; }
            if (d1 > 0 && d1 <= cur && ((mB >> (d1 - 1)) & 1u)) fb = 0.0f;
            else if (mB) { nd1 = __ffs((int)mB); fb = 3.0f; }
            if (ok) key = key_of((float)e + lambda * (fa + fb + 1.0f), kind < 0 ? 0 : (j - 1) * 3 + kind + 1);
        } else if (cur + 2 < count) {  // the loader: the block after next
            load_bc7_block(src, bw, out, dec_base, g + 2, (cur + 2) % 3, i, gm, s_tex, s_dbase, s_base, s_sumx);
        }
        const uint64_t wk = warp_min_redux(key);
        if (lane == 0) s_key[warp] = wk;
        __syncthreads();
        const int order = (int)(uint32_t)warp_min_redux(lane < kB7Warps ? s_key[lane] : ~0ull);
        const int oc = order - 1, wkind = oc % 3, wgrp = order == 0 ? 48 : wkind == 1 ? oc / 3 : wkind == 2 ? 16 + oc / 3 : 32 + oc / 3;
        if (grp == wgrp) {  // the winner enters the window
            const int ws = cur & (kWindow - 1);
            ring_dec[ws][i] = dec;
            ring_pal[ws][i] = pal;
            if (i == 0) {
                ring[ws][0] = clo; ring[ws][1] = chi; ring_idx[ws] = cidx;
                s_dist[0] = nd0; s_dist[1] = nd1;
                if (order != 0) { *(uint64_t *)(out + (size_t)g * 16) = clo; *(uint64_t *)(out + (size_t)g * 16 + 8) = chi; }
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- BC1 / BC4 sub-blocks: one lane per texel
// The BC7 chain's layout for one sub-block of a BC1-BC5 block: groups 0-15 kind 0 (neighbour j = group + 1: its
// endpoints, fitted indices), 16-31 kind 1 (these endpoints, its indices), 32-47 kind 2 (the whole neighbour),
// 48 the base, 49 loads the next block. The two sub-blocks of a BC3 or BC5 block are independent chains (each
// looks only at its own fields of earlier blocks, with its own match distances, zap_tex.h:1494-1501), so each
// runs in its own CTA (blockIdx.y) and writes its own 8 bytes of the blocks.
ZTC_DEV void bc1_palette(uint32_t c0, uint32_t c1, int force4, uint32_t pal[4]) {  // entries as RGB texels
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        int r, g, b;
        bc1_entry(c0, c1, force4, k, r, g, b);
        pal[k] = pack_rgb(r, g, b);
    }
}
ZTC_DEV int sq3px(uint32_t t, uint32_t p) {
    int s = 0;
    #pragma unroll
    for (int c = 0; c < 3; c++) { const int d = (int)chan(t, c) - (int)chan(p, c); s += d * d; }
    return s;
}

__global__ void __launch_bounds__(kB7Threads, 1) rdo_sub_chain_kernel(SrcU8 src, int bw, int nby, int chain_rows, uint8_t *__restrict__ out,
                                                                      int bs, Sub S0, Sub S1, float lambda) {
    __shared__ uint64_t ring[kWindow];  // the sub-block of the last 16 chosen blocks, slot = block & 15
    __shared__ uint32_t s_tex[3][16];  // block cur in slot cur % 3, loaded two blocks ahead
    __shared__ uint64_t s_base[3];
    __shared__ uint64_t s_key[kB7Warps];
    __shared__ int s_dist[2];
    const Sub S = blockIdx.y ? S1 : S0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, i = lane & 15, grp = tid >> 4;
    const int kind = grp < 16 ? 0 : grp < 32 ? 1 : grp < 48 ? 2 : grp == 48 ? -1 : -2, j = (grp & 15) + 1;
    const unsigned gm = group_mask(warp, lane);
    const int row0 = blockIdx.x * chain_rows, rows = min(chain_rows, nby - row0);
    if (rows <= 0) return;
    const int first = row0 * bw, count = rows * bw;
    if (kind == -2)
        for (int k = 0; k < 2 && k < count; k++) {
            const int gk = first + k;
            s_tex[k][i] = load_texel(src, min((gk % bw) * 4 + (i & 3), src.w - 1), min((gk / bw) * 4 + (i >> 2), src.h - 1));
            if (i == 0) s_base[k] = *(const uint64_t *)(out + (size_t)gk * bs + S.off);
        }
    if (tid == 0) { s_dist[0] = 1; s_dist[1] = 1; }
    __syncthreads();
    // fields: BC1 {c0 c1, indices} = {4, 4} bytes, BC4 {a0 a1, indices} = {2, 6}
    const bool bc1 = S.type == kBc1;
    const int nA = bc1 ? 4 : 2, nB = bc1 ? 4 : 6;
    const uint64_t maskA = (1ull << (8 * nA)) - 1ull;
    const float newA = bc1 ? 3.0f : 2.0f, newB = 3.0f;  // min(size, 3)
    for (int cur = 0; cur < count; cur++) {
        const int g = first + cur, slot = cur % 3, d0 = s_dist[0], d1 = s_dist[1];
        uint64_t key = ~0ull, cand = 0;
        int nd0 = 0, nd1 = 0;
        if (kind >= -1) {
            const uint32_t t = s_tex[slot][i];
            const uint64_t base = s_base[slot], nb = ring[(cur - j) & (kWindow - 1)];
            bool ok = kind == -1 || j <= cur;
            int e;
            if (bc1) {  // the CTA's sub-block type: uniform
                const uint32_t p0 = (uint32_t)(nb & 0xFFFFu), p1 = (uint32_t)((nb >> 16) & 0xFFFFu);
                // kind 1 and the base: these endpoints; kinds 0 and 2: the neighbour's
                const uint32_t a = kind == 1 || kind == -1 ? (uint32_t)(base & 0xFFFFu) : p0;
                const uint32_t b = kind == 1 || kind == -1 ? (uint32_t)((base >> 16) & 0xFFFFu) : p1;
                uint32_t pal[4];
                bc1_palette(a, b, S.force4, pal);
                uint32_t idx;
                if (kind == 0) {  // zap__bc1_fit: best of the 4 (3 in 3-colour order) entries, first on ties
                    const int n = (S.force4 || a > b) ? 4 : 3;
                    int bk = 0, be = sq3px(t, pal[0]);
                    #pragma unroll
                    for (int k = 1; k < 4; k++) {
                        const int ek = sq3px(t, pal[k]);
                        if (k < n && ek < be) { be = ek; bk = k; }
                    }
                    e = grp_sum(be, gm);
                    idx = (uint32_t)grp_or64((uint64_t)bk << (2 * i), gm);
                } else {  // zap__bc1_eval with the base's or the neighbour's indices
                    idx = (uint32_t)((kind == -1 ? base : nb) >> 32);
                    const int k = (int)((idx >> (2 * i)) & 3u);
                    e = grp_sum(sq3px(t, k == 0 ? pal[0] : k == 1 ? pal[1] : k == 2 ? pal[2] : pal[3]), gm);
                }
                cand = (uint64_t)a | ((uint64_t)b << 16) | ((uint64_t)idx << 32);
                // a 3-colour block may not use index 3 (transparent); the base is never checked
                if (kind >= 0 && !S.force4 && a <= b && (idx & (idx >> 1) & 0x55555555u)) ok = false;
            } else {
                const int pa0 = (int)(nb & 0xFFu), pa1 = (int)((nb >> 8) & 0xFFu);
                const int a = kind == 1 || kind == -1 ? (int)(base & 0xFFu) : pa0, b = kind == 1 || kind == -1 ? (int)((base >> 8) & 0xFFu) : pa1;
                const int v = (int)chan(t, S.chan);
                uint64_t idx;
                if (kind == 0) {  // zap__bc4_fit
                    int bk = 0, be = (v - bc4_entry(a, b, 0)) * (v - bc4_entry(a, b, 0));
                    #pragma unroll
                    for (int k = 1; k < 8; k++) {
                        const int d = v - bc4_entry(a, b, k);
                        if (d * d < be) { be = d * d; bk = k; }
                    }
                    e = grp_sum(be, gm);
                    idx = grp_or64((uint64_t)bk << (3 * i), gm);
                } else {  // zap__bc4_eval
                    idx = (kind == -1 ? base : nb) >> 16;
                    const int d = v - bc4_entry(a, b, (int)((idx >> (3 * i)) & 7u));
                    e = grp_sum(d * d, gm);
                }
                cand = (uint64_t)a | ((uint64_t)b << 8) | (idx << 16);
            }
            // rate (zap__field_rate per field): lane i compares with window slot j' = i + 1
            const uint64_t w = ring[(cur - i - 1) & (kWindow - 1)];
            const bool vw = i + 1 <= cur;
            const unsigned sh = lane & 16;
            const unsigned mA = (__ballot_sync(gm, vw && (w & maskA) == (cand & maskA)) >> sh) & 0xFFFFu;
            const unsigned mB = (__ballot_sync(gm, vw && (w >> (8 * nA)) == (cand >> (8 * nA))) >> sh) & 0xFFFFu;
            float fa = (float)nA, fb = (float)nB;
            nd0 = d0; nd1 = d1;
            if (d0 > 0 && d0 <= cur && ((mA >> (d0 - 1)) & 1u)) fa = 0.0f;
            else if (mA) { nd0 = __ffs((int)mA); fa = newA; }
            if (d1 > 0 && d1 <= cur && ((mB >> (d1 - 1)) & 1u)) fb = 0.0f;
            else if (mB) { nd1 = __ffs((int)mB); fb = newB; }
            if (ok) key = key_of((float)e + lambda * (fa + fb), kind < 0 ? 0 : (j - 1) * 3 + kind + 1);
        } else if (cur + 2 < count) {  // the loader: texels and base sub-block of the block after next
            const int gn = g + 2, ns = (cur + 2) % 3;
            s_tex[ns][i] = load_texel(src, min((gn % bw) * 4 + (i & 3), src.w - 1), min((gn / bw) * 4 + (i >> 2), src.h - 1));
            if (i == 0) s_base[ns] = *(const uint64_t *)(out + (size_t)gn * bs + S.off);
        }
        const uint64_t wk = warp_min_redux(key);
        if (lane == 0) s_key[warp] = wk;
        __syncthreads();
        const int order = (int)(uint32_t)warp_min_redux(lane < kB7Warps ? s_key[lane] : ~0ull);
        const int oc = order - 1, wkind = oc % 3, wgrp = order == 0 ? 48 : wkind * 16 + oc / 3;
        if (grp == wgrp && i == 0) {  // the winner enters the window
            ring[cur & (kWindow - 1)] = cand;
            s_dist[0] = nd0; s_dist[1] = nd1;
            if (order != 0) *(uint64_t *)(out + (size_t)g * bs + S.off) = cand;
        }
        __syncthreads();
    }
}

}  // namespace
}  // namespace ztc

// RDO pass over an image whose base encodings `out` holds (raster blocks): one chain per band of band_rows block
// rows (band_rows >= the block-row count: one chain, the reference's single call). lambda: finite, > 0.
cudaError_t ztc_launch_rdo(int fmt, const ztc::SrcU8 &src, uint8_t *out, float lambda, int band_rows, cudaStream_t stream) {
    const int bw = (src.w + 3) / 4, nby = (src.h + 3) / 4;
    if (band_rows <= 0 || band_rows > nby) band_rows = nby;
    const int chains = (nby + band_rows - 1) / band_rows;
    ztc::TraceScope tr("rdo_chain", stream);
    ztc::trace_units((long)bw * nby);
    if (fmt == ZTC_FMT_BC7) {
        const int nblocks = bw * nby;
        uint32_t *dec = nullptr;
        cudaError_t e = ztc_malloc_async((void **)&dec, (size_t)nblocks * 64, stream);
        if (e != cudaSuccess) return e;
        ztc::bc7_decode_bases_kernel<<<(nblocks + 127) / 128, 128, 0, stream>>>(out, nblocks, (uint4 *)dec);
        ztc::rdo_bc7_chain_kernel<<<chains, ztc::kB7Threads, 0, stream>>>(src, bw, nby, band_rows, out, dec, lambda);
        e = cudaGetLastError();
        cudaFreeAsync(dec, stream);
        return e;
    }
    {
        const ztc::Sub S0 = ztc::sub_of(fmt, 0), S1 = ztc::sub_of(fmt, 1);
        const int ns = ztc::sub_count(fmt), bs = fmt == ZTC_FMT_BC1 || fmt == ZTC_FMT_BC4 ? 8 : 16;
        const dim3 grid(chains, ns);
        if (fmt < ZTC_FMT_BC1 || fmt > ZTC_FMT_BC5) return cudaErrorInvalidValue;
        ztc::rdo_sub_chain_kernel<<<grid, ztc::kB7Threads, 0, stream>>>(src, bw, nby, band_rows, out, bs, S0, S1, lambda);
        return cudaGetLastError();
    }
}

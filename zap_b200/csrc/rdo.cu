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


// ---------------------------------------------------------------- BC7
// A BC7 candidate costs a whole palette search or least-squares solve, so this chain spreads each candidate over a
// group of L lanes: lane q takes texels q*T .. q*T + T - 1 (T = 16 / L), and the window slots at those distances
// minus one when the rate is counted. Groups 0-15 kind 1 (neighbour j = group + 1: its endpoints, refit indices),
// 16-31 kind 2 (its indices, refit endpoints), 32-47 kind 0 (the whole neighbour), 48 the base; a last warp loads the
// blocks ahead, software-pipelined like the BC1 / BC4 chains' loader (its own warp, so its global loads hold no
// candidate's minimum). Every chosen block enters the window with its decoded texels and, for mode 6, its palette
// (with the entries' squared norms), indices and index weights, so no candidate decodes a block: kind 0 compares the
// texels with the stored decode, kind 1 searches the stored palette. The base encodings are decoded for every block
// by a parallel pass before the chains. Kind 2's least-squares sums are exact in the reference's float accumulation
// (weights k/64, texels integers: every partial sum is a multiple of 1/4096 below 2^17 of them), so they are integer
// dot products (the weights and the texels' channels a byte per texel), scaled, which gives the same floats in any
// order; its solve and quantisation are one (channel, endpoint) per lane, both p-bits.

// Collectives over a group of L lanes: gm names the lanes that meet the collective. Warps whose groups all run one
// kind of candidate pass the whole warp (every group meets each collective at the same point); whole-warp masks
// measured faster on B200 than each group passing its own (512x512 one chain: BC7 30.6 -> 28.3 ms, BC1 25.8 ->
// 25.5 ms), and redux.sync for the group sums slower than shuffle trees (BC7 30.6 -> 47 ms). ZTC_RDO_MIN_REDUX
// selects redux.sync (1) or an xor-shuffle tree (0) for the warp-wide key minimum.
#ifndef ZTC_RDO_MIN_REDUX
#define ZTC_RDO_MIN_REDUX 1
#endif
// sums and ORs over a group of L lanes (gm: the lanes that meet the collective)
template <int L> __device__ __forceinline__ int lsum(int v, unsigned gm) {
    #pragma unroll
    for (int m = L / 2; m >= 1; m >>= 1) v += __shfl_xor_sync(gm, v, m, L);
    return v;
}
template <int L> __device__ __forceinline__ uint32_t lor(uint32_t v, unsigned gm) {
    #pragma unroll
    for (int m = L / 2; m >= 1; m >>= 1) v |= __shfl_xor_sync(gm, v, m, L);
    return v;
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
// squared RGBA difference (zap__sq4 over 4 channels) as |a|^2 + |b|^2 - 2 a.b, three dp4a; aa = |a|^2
ZTC_DEV int sq4px(uint32_t a, int aa, uint32_t b) { return aa + (int)dot4(b, b) - 2 * (int)dot4(a, b); }
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

// The loader warp's registers for one block: lane i < 16 its texel i and decoded base texel i, every lane the base.
struct Bc7Fetch {
    uint32_t tex = 0, dec = 0;
    uint64_t lo = 0, hi = 0;
    __device__ __forceinline__ void fetch(const SrcU8 &src, int bw, const uint8_t *out, const uint32_t *dec_base, int gk, int lane) {
        if (lane < 16) {
            tex = load_texel(src, min((gk % bw) * 4 + (lane & 3), src.w - 1), min((gk / bw) * 4 + (lane >> 2), src.h - 1));
            dec = dec_base[(size_t)gk * 16 + lane];
        }
        lo = *(const uint64_t *)(out + (size_t)gk * 16);
        hi = *(const uint64_t *)(out + (size_t)gk * 16 + 8);
    }
    // into slot ns: texels, decoded base, base, the base's mode-6 palette, and the texels by channel (byte i of
    // texc[c] is channel c of texel i, for the least-squares sums as dp4a)
    __device__ __forceinline__ void store(int lane, int ns, uint32_t (*s_tex)[16], uint32_t (*s_dbase)[16], uint64_t (*s_base)[2],
                                          uint32_t (*s_bpal)[16], uint32_t (*s_texc)[4][4]) const {
        if (lane < 16) {
            s_tex[ns][lane] = tex;
            s_dbase[ns][lane] = dec;
            int x0[4], x1[4];
            mode6_ends_of(lo, hi, x0, x1);
            s_bpal[ns][lane] = lerp_px(x0, x1, w4(lane));
            #pragma unroll
            for (int c = 0; c < 4; c++) ((uint8_t *)s_texc[ns][c])[lane] = (uint8_t)chan(tex, c);
        }
        if (lane < 2) s_base[ns][lane] = lane ? hi : lo;
    }
};

template <int L> struct B7Chain {  // kWc candidate warps, then the loader warp
    static constexpr int T = 16 / L, kWc = (49 * L + 31) / 32, kThreads = (kWc + 1) * 32;
};
#ifndef ZTC_RDO_BC7_LANES
#define ZTC_RDO_BC7_LANES 8
#endif

template <int L>
__global__ void __launch_bounds__(B7Chain<L>::kThreads, 1) rdo_bc7_chain_kernel(SrcU8 src, int bw, int nby, int chain_rows, uint8_t *__restrict__ out,
                                                                                const uint32_t *__restrict__ dec_base, float lambda) {
    constexpr int T = B7Chain<L>::T, kW = B7Chain<L>::kWc;
    __shared__ uint64_t ring[kWindow][2];       // the last 16 chosen blocks, slot = block & 15
    __shared__ uint32_t ring_dec[kWindow][16];  // their decoded texels
    __shared__ __align__(16) uint32_t ring_pal[kWindow][16];  // mode 6: their palettes
    __shared__ __align__(16) int ring_pp[kWindow][16];        // and the entries' squared norms |p|^2
    __shared__ uint64_t ring_idx[kWindow];      // mode 6: their indices, 4 bits per texel
    __shared__ __align__(16) uint32_t ring_wp[kWindow][4];  // mode 6: their index weights w4(idx), a byte per texel
    __shared__ uint32_t s_tex[3][16], s_dbase[3][16];  // block cur in slot cur % 3, loaded two blocks ahead
    __shared__ uint64_t s_base[3][2];
    __shared__ uint32_t s_bpal[3][16];                 // the base's palette, if mode 6
    __shared__ __align__(16) uint32_t s_texc[3][4][4];  // the block's texels by channel, a byte per texel
    __shared__ uint64_t s_key[kW];
    __shared__ int s_dist[2];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = tid & (L - 1), grp = tid / L;
    const bool loader = warp == kW;
    const int kind = loader ? -2 : grp < 16 ? 1 : grp < 32 ? 2 : grp < 48 ? 0 : grp == 48 ? -1 : -3, j = (grp & 15) + 1;
    // the warps of groups 0-47 hold one kind each and meet every collective together; the base's group has its own
    const unsigned gm = warp < 48 * L / 32 ? 0xFFFFFFFFu : (((1u << L) - 1u) << (lane & ~(L - 1)));
    const int row0 = blockIdx.x * chain_rows, rows = min(chain_rows, nby - row0);
    if (rows <= 0) return;
    const int first = row0 * bw, count = rows * bw;
    Bc7Fetch fb;
    if (loader) {
        for (int k = 0; k < 2 && k < count; k++) {
            fb.fetch(src, bw, out, dec_base, first + k, lane);
            fb.store(lane, k, s_tex, s_dbase, s_base, s_bpal, s_texc);
        }
        if (count > 2) fb.fetch(src, bw, out, dec_base, first + 2, lane);
    }
    if (tid == 0) { s_dist[0] = 1; s_dist[1] = 1; }
    __syncthreads();
    for (int cur = 0; cur < count; cur++) {
        const int g = first + cur, slot = cur % 3, d0 = s_dist[0], d1 = s_dist[1];
        uint64_t key = ~0ull, clo = 0, chi = 0, cidx = 0;
        uint32_t dec[T];  // the candidate's decode of this lane's texels
        int nd0 = 0, nd1 = 0, x0[4], x1[4];  // x0, x1: kind 2's refit endpoints, expanded
        const int r = (cur - j) & (kWindow - 1);
        if (kind >= -1) {
            uint32_t t[T];
            int tt[T];
            #pragma unroll
            for (int u = 0; u < T; u++) { t[u] = s_tex[slot][q * T + u]; tt[u] = (int)dot4(t[u], t[u]); }
            bool ok;
            int e = 0;
            if (kind == -1) {  // the base (its SSE: the one the reference's encoder returns)
                clo = s_base[slot][0]; chi = s_base[slot][1];
                #pragma unroll
                for (int u = 0; u < T; u++) { dec[u] = s_dbase[slot][q * T + u]; e += sq4px(t[u], tt[u], dec[u]); }
                e = lsum<L>(e, gm);
                cidx = mode6_idx_of(chi);
                ok = true;
            } else if (kind == 0) {  // the whole neighbour (zap__bc7_err)
                clo = ring[r][0]; chi = ring[r][1]; cidx = ring_idx[r];
                #pragma unroll
                for (int u = 0; u < T; u++) { dec[u] = ring_dec[r][q * T + u]; e += sq4px(t[u], tt[u], dec[u]); }
                e = lsum<L>(e, gm);
                ok = j <= cur;
            } else if (kind == 1) {  // its endpoints, best indices; texel 0 keeps to 0..7 (zap__bc7_fit6_idx)
                const uint64_t nlo = ring[r][0], nhi = ring[r][1];
                ok = j <= cur && is_mode6(nlo);
                uint64_t bits = 0;
                #pragma unroll
                for (int u = 0; u < T; u++) {
                    // key 16 (|p|^2 - 2 t.p) + k per entry (its minimum is the first nearest entry), minimised as a tree
                    const int i = q * T + u;
                    int kk[16];
                    #pragma unroll
                    for (int k4 = 0; k4 < 4; k4++) {
                        const uint4 pk = *(const uint4 *)&ring_pal[r][4 * k4];
                        const int4 pp = *(const int4 *)&ring_pp[r][4 * k4];
                        kk[4 * k4 + 0] = 16 * (pp.x - 2 * (int)dot4(t[u], pk.x)) + 4 * k4 + 0;
                        kk[4 * k4 + 1] = 16 * (pp.y - 2 * (int)dot4(t[u], pk.y)) + 4 * k4 + 1;
                        kk[4 * k4 + 2] = 16 * (pp.z - 2 * (int)dot4(t[u], pk.z)) + 4 * k4 + 2;
                        kk[4 * k4 + 3] = 16 * (pp.w - 2 * (int)dot4(t[u], pk.w)) + 4 * k4 + 3;
                    }
                    if (i == 0) {  // the anchor texel's index has 3 bits
                        #pragma unroll
                        for (int k = 8; k < 16; k++) kk[k] = 0x7FFFFFFF;
                    }
                    #pragma unroll
                    for (int h = 8; h >= 1; h >>= 1)
                        #pragma unroll
                        for (int k = 0; k < h; k++) kk[k] = min(kk[k], kk[k + h]);
                    dec[u] = ring_pal[r][kk[0] & 15];
                    e += (kk[0] >> 4) + tt[u];
                    bits |= (uint64_t)(kk[0] & 15) << (4 * i);
                }
                e = lsum<L>(e, gm);
                cidx = ((uint64_t)lor<L>((uint32_t)(bits >> 32), gm) << 32) | lor<L>((uint32_t)bits, gm);
                clo = nlo; chi = mode6_hi((int)(nhi & 1u), cidx);
            } else {  // its indices, least-squares endpoints, each endpoint's own p-bit (zap__bc7_fit6_ep)
                const uint64_t nlo = ring[r][0], nhi = ring[r][1];
                ok = j <= cur && is_mode6(nlo);
                cidx = ring_idx[r];
                const int task = q & 7, ch = task >> 1, ep = task & 1;  // this lane's (channel, endpoint)
                // the neighbour's weights and this block's channel ch, a byte per texel: sum w, sum w^2 and sum w x
                // are four dp4a each; with u = 64 - w: sum u^2 = 16 * 4096 - 128 sum w + sum w^2,
                // sum u w = 64 sum w - sum w^2, sum u x = 64 sum x - sum w x
                const uint4 wp = *(const uint4 *)ring_wp[r], xc = *(const uint4 *)s_texc[slot][ch];
                const int W1 = (int)__dp4a(wp.w, 0x01010101u, __dp4a(wp.z, 0x01010101u, __dp4a(wp.y, 0x01010101u, dot4(wp.x, 0x01010101u))));
                const int W2 = (int)__dp4a(wp.w, wp.w, __dp4a(wp.z, wp.z, __dp4a(wp.y, wp.y, dot4(wp.x, wp.x))));
                const int SB = (int)__dp4a(wp.w, xc.w, __dp4a(wp.z, xc.z, __dp4a(wp.y, xc.y, dot4(wp.x, xc.x))));
                const int SX = (int)__dp4a(xc.w, 0x01010101u, __dp4a(xc.z, 0x01010101u, __dp4a(xc.y, 0x01010101u, dot4(xc.x, 0x01010101u))));
                const int AA = 16 * 4096 - 128 * W1 + W2, AB = 64 * W1 - W2, BB = W2, SA = 64 * SX - SB;
                const float aa = (float)AA / 4096.0f, ab = (float)AB / 4096.0f, bb = (float)BB / 4096.0f;
                const float ax = (float)SA / 64.0f, bx = (float)SB / 64.0f, det = aa * bb - ab * ab;
                float v;
                if (det < 1e-6f && det > -1e-6f) v = (ax + bx) / 16.0f;  // one index everywhere: flat
                else v = ep ? (bx * aa - ax * ab) / det : (ax * bb - bx * ab) / det;
                v = clamp255(v);
                // zap__bc7q for this (channel, endpoint), 7 bits + p, for both p-bits
                const float vv = div255(v) * 255.0f;  // v / 255 correctly rounded, without a division sequence
                int bq[2], be[2];
                #pragma unroll
                for (int p = 0; p < 2; p++) {
                    const int gq = f2i_x86((vv - (float)p) / 2.0f + 0.5f);
                    bq[p] = 0; be[p] = 1 << 30;
                    #pragma unroll
                    for (int k = 0; k < 3; k++) {
                        const int tq = clampi(around(gq, k), 0, 127);
                        const float d = (float)((tq << 1) | p) - v;
                        const int ek = f2i_x86(d * d);
                        if (ek < be[p]) { be[p] = ek; bq[p] = tq; }
                    }
                }
                // each endpoint's errors over the four channels, both p-bits in one word (each below 2^16: a
                // candidate lies within 2 of v); the endpoint keeps the p-bit of the smaller sum, p = 0 on ties
                int s2 = be[0] | (be[1] << 16);
                s2 += __shfl_xor_sync(gm, s2, 2, L);
                s2 += __shfl_xor_sync(gm, s2, 4, L);
                const int pbm = (s2 >> 16) < (s2 & 0xFFFF) ? 1 : 0, qm = pbm ? bq[1] : bq[0];
                const int pb0 = __shfl_sync(gm, pbm, 0, L), pb1 = __shfl_sync(gm, pbm, 1, L);
                uint64_t lo = 0x40u | ((uint64_t)pb0 << 63);
                #pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int q0 = __shfl_sync(gm, qm, 2 * c, L), q1 = __shfl_sync(gm, qm, 2 * c + 1, L);
                    x0[c] = (q0 << 1) | pb0; x1[c] = (q1 << 1) | pb1;
                    lo |= ((uint64_t)q0 << (7 + 14 * c)) | ((uint64_t)q1 << (14 + 14 * c));
                }
                #pragma unroll
                for (int u = 0; u < T; u++) {
                    dec[u] = lerp_px(x0, x1, w4((int)((cidx >> (4 * (q * T + u))) & 15u)));
                    e += sq4px(t[u], tt[u], dec[u]);
                }
                e = lsum<L>(e, gm);
                clo = lo; chi = (nhi & ~1ull) | (uint64_t)pb1;
            }
            // rate (zap__bc7_rate): bit d - 1 of a mask says the field equals the window's at distance d
            uint32_t mA = 0, mB = 0;
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const int d = q * T + u + 1, rw = (cur - d) & (kWindow - 1);
                if (d <= cur) {
                    mA |= (uint32_t)(ring[rw][0] == clo) << (d - 1);
                    mB |= (uint32_t)((ring[rw][1] >> 8) == (chi >> 8)) << (d - 1);
                }
            }
            mA = lor<L>(mA, gm);
            mB = lor<L>(mB, gm);
            float fa = 8.0f, fb = 7.0f;
            nd0 = d0; nd1 = d1;
            if (d0 > 0 && d0 <= cur && ((mA >> (d0 - 1)) & 1u)) fa = 0.0f;
            else if (mA) { nd0 = __ffs((int)mA); fa = 3.0f; }
            if (d1 > 0 && d1 <= cur && ((mB >> (d1 - 1)) & 1u)) fb = 0.0f;
            else if (mB) { nd1 = __ffs((int)mB); fb = 3.0f; }
            if (ok) key = key_of((float)e + lambda * (fa + fb + 1.0f), kind < 0 ? 0 : (j - 1) * 3 + kind + 1);
        } else if (loader) {  // block cur + 2 (fetched the iteration before) to shared memory; fetch block cur + 3
            if (cur + 2 < count) fb.store(lane, (cur + 2) % 3, s_tex, s_dbase, s_base, s_bpal, s_texc);
            if (cur + 3 < count) fb.fetch(src, bw, out, dec_base, g + 3, lane);
        }
        if (!loader) {
            const uint64_t wk = warp_min_redux(key);
            if (lane == 0) s_key[warp] = wk;
        }
        __syncthreads();
        const int order = loader ? -1 : (int)(uint32_t)warp_min_redux(lane < kW ? s_key[lane] : ~0ull);
        const int oc = order - 1, wkind = oc % 3, wgrp = order == 0 ? 48 : wkind == 1 ? oc / 3 : wkind == 2 ? 16 + oc / 3 : 32 + oc / 3;
        if (!loader && grp == wgrp) {  // the winner enters the window
            const int ws = cur & (kWindow - 1);
            // its decode, its mode-6 palette (the base's, built by the loader; the neighbour's, which kinds 0 and 1
            // keep: with j = 16 that slot is this one and each lane rewrites its own entries; or from the refit
            // endpoints) and its index weights
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const int i = q * T + u;
                ring_dec[ws][i] = dec[u];
                const uint32_t pal = order == 0 ? s_bpal[slot][i] : kind != 2 ? ring_pal[r][i] : lerp_px(x0, x1, w4(i));
                ring_pal[ws][i] = pal;
                ring_pp[ws][i] = (int)dot4(pal, pal);
                ((uint8_t *)ring_wp[ws])[i] = (uint8_t)w4((int)((cidx >> (4 * i)) & 15u));
            }
            if (q == 0) {
                ring[ws][0] = clo; ring[ws][1] = chi; ring_idx[ws] = cidx;
                s_dist[0] = nd0; s_dist[1] = nd1;
                if (order != 0) { *(uint64_t *)(out + (size_t)g * 16) = clo; *(uint64_t *)(out + (size_t)g * 16 + 8) = chi; }
            }
        }
        __syncthreads();
    }
}

// Word k of a sub-block's palette as the chain keeps it in shared memory: BC1 entries 0-3 as RGB texels (alpha
// byte 0), then words 4-7 their squared norms |p|^2, so a texel's squared distance to entry k is
// |t|^2 + |p_k|^2 - 2 t.p_k with t.p_k one dp4a; BC4 its 8 values. Each chosen sub-block enters the window with its
// palette and the loader builds each block's base palette two blocks ahead, so no candidate builds one.
ZTC_DEV int palette_word(const Sub &S, uint64_t v, int k) {
    if (S.type == kBc1) {
        int r, g, b;
        bc1_entry((uint32_t)(v & 0xFFFFu), (uint32_t)((v >> 16) & 0xFFFFu), S.force4, k & 3, r, g, b);
        const uint32_t p = pack_rgb(r, g, b);
        return k < 4 ? (int)p : (int)dot4(p, p);
    }
    return bc4_entry((int)(v & 0xFFu), (int)((v >> 8) & 0xFFu), k);
}

// ---------------------------------------------------------------- BC1 / BC4 sub-blocks
// One chain per CTA and sub-block kind, in two roles. The candidates of a block that do not involve the block
// chosen just before it (the base, and every neighbour at distance j >= 2) depend only on decisions at least two
// blocks back, so producer warps evaluate them one block ahead: while block b - 1 is being chosen, they compute
// block b's candidates (SSE, fields, and the match masks against window distances 2..16) into shared memory. A
// chooser warp then decides block b alone: it evaluates the three candidates of neighbour distance 1 itself, adds
// each other candidate's distance-1 match bit, turns the masks into rates and keys for all 49, and takes the minimum
// of (cost, candidate order) across its lanes. One barrier per block; no CTA-wide minimum. The 49 candidates are
// evaluated by groups of 8 lanes, lane q taking texels 2q, 2q + 1 and window distances 2q + 1, 2q + 2. Producer
// groups: 0-15 kind 0 (neighbour j = (group & 15) + 2: its endpoints, fitted indices), 16-31 kind 1 (these
// endpoints, its indices), 32-47 kind 2 (the whole neighbour), the last group of each kind idle (it repeats j = 16
// and keeps nothing), 48 the base; a last warp loads the blocks ahead, software-pipelined (block b + 2 stored while
// block b + 3 is fetched into registers), so no warp waits for a global load inside a step. The two sub-blocks of a
// BC3 or BC5 block are independent chains (each looks only at its own fields of earlier blocks, with its own match
// distances, zap_tex.h:1494-1501), so each runs in its own CTA (blockIdx.y) and writes its own 8 bytes of the blocks.
// The chooser is three warps: one fits the distance-1 kind-0 candidate, one evaluates kinds 1 and 2 (the same code
// path), and the deciding warp meanwhile turns the other 46 candidates into keys (they do not depend on the distance-1
// results); a named barrier over the three joins them, and the deciding warp adds the three distance-1 keys and takes
// the minimum. Phase timers (clock64, a scratch build) put the chooser's step at ~2,950 cycles per block with all
// three roles in one warp (the fit and evaluation branches serialised, then two candidates' keys per lane).
constexpr int kSubL = 8, kSubProducerWarps = 13, kSubFit = 13, kSubEval = 14, kSubDecide = 15, kSubLoader = 16,
              kSubThreads = 17 * 32;

struct SubCand {
    int e;
    uint64_t cand;
    bool ok;
    uint32_t mA, mB;  // bit d - 1: the field equals the window's at distance d (from distance dlo on)
};

// One candidate of chain block b on a group of 8 lanes (gm: the lanes that meet its collectives). kind -1: the base;
// 0: neighbour j's endpoints with fitted indices; 1: the base's endpoints with neighbour j's indices; 2: the whole
// neighbour j. Its window masks cover distances dlo..16 (up to b).
__device__ __forceinline__ SubCand sub_candidate(const Sub &S, int kind, int j, int b, int q, unsigned gm, int dlo,
                                                 const uint32_t (*s_tex)[16], const uint64_t *s_base, const int (*s_bpal)[8],
                                                 const uint64_t *ring, const int (*ring_pal)[8]) {
    constexpr int T = 16 / kSubL;
    const bool bc1 = S.type == kBc1;
    const int nA = bc1 ? 4 : 2, slot = b % 3;
    const uint64_t maskA = (1ull << (8 * nA)) - 1ull;
    uint32_t t[T];
    #pragma unroll
    for (int u = 0; u < T; u++) t[u] = s_tex[slot][q * T + u];
    const uint64_t base = s_base[slot], nb = ring[(b - j) & (kWindow - 1)];
    // kind 1 and the base: these endpoints (the base's palette); kinds 0 and 2: the neighbour's
    const bool own = kind == 1 || kind == -1;
    const int *P = own ? s_bpal[slot] : ring_pal[(b - j) & (kWindow - 1)];
    SubCand r;
    r.ok = kind == -1 || j <= b;
    int e = 0;
    if (bc1) {  // the CTA's sub-block type: uniform
        const uint32_t a = (uint32_t)((own ? base : nb) & 0xFFFFu), c = (uint32_t)(((own ? base : nb) >> 16) & 0xFFFFu);
        uint32_t idx;
        if (kind == 0) {  // zap__bc1_fit: best of the 4 (3 in 3-colour order) entries, first on ties
            const int4 pe = *(const int4 *)P, pn = *(const int4 *)(P + 4);
            const bool n4 = S.force4 || a > c;
            idx = 0;
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const uint32_t tc = t[u] & 0xFFFFFFu;
                int bk = 0, be = pn.x - 2 * (int)dot4(tc, (uint32_t)pe.x), sk;
                sk = pn.y - 2 * (int)dot4(tc, (uint32_t)pe.y); if (sk < be) { be = sk; bk = 1; }
                sk = pn.z - 2 * (int)dot4(tc, (uint32_t)pe.z); if (sk < be) { be = sk; bk = 2; }
                sk = pn.w - 2 * (int)dot4(tc, (uint32_t)pe.w); if (n4 && sk < be) { be = sk; bk = 3; }
                e += be + (int)dot4(tc, tc);
                idx |= (uint32_t)bk << (2 * (q * T + u));
            }
            e = lsum<kSubL>(e, gm);
            idx = lor<kSubL>(idx, gm);
        } else {  // zap__bc1_eval with the base's or the neighbour's indices
            idx = (uint32_t)((kind == -1 ? base : nb) >> 32);
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const uint32_t tc = t[u] & 0xFFFFFFu;
                const int k = (int)((idx >> (2 * (q * T + u))) & 3u);
                e += P[4 + k] - 2 * (int)dot4(tc, (uint32_t)P[k]) + (int)dot4(tc, tc);
            }
            e = lsum<kSubL>(e, gm);
        }
        r.cand = (uint64_t)a | ((uint64_t)c << 16) | ((uint64_t)idx << 32);
        // a 3-colour block may not use index 3 (transparent); the base is never checked
        if (kind >= 0 && !S.force4 && a <= c && (idx & (idx >> 1) & 0x55555555u)) r.ok = false;
    } else {
        const int a = (int)((own ? base : nb) & 0xFFu), c = (int)(((own ? base : nb) >> 8) & 0xFFu);
        uint64_t idx;
        if (kind == 0) {  // zap__bc4_fit
            const int4 p0 = *(const int4 *)P, p1 = *(const int4 *)(P + 4);
            const int pv[8] = {p0.x, p0.y, p0.z, p0.w, p1.x, p1.y, p1.z, p1.w};
            uint32_t part = 0;  // this lane's T 3-bit indices
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const int v = (int)chan(t[u], S.chan);
                int bk = 0, be = (v - pv[0]) * (v - pv[0]);
                #pragma unroll
                for (int k = 1; k < 8; k++) {
                    const int d = v - pv[k];
                    if (d * d < be) { be = d * d; bk = k; }
                }
                e += be;
                part |= (uint32_t)bk << (3 * u);
            }
            e = lsum<kSubL>(e, gm);
            // lane q's indices start at bit 3 q T: two 32-bit words of the 48
            const uint64_t mine = (uint64_t)part << (3 * q * T);
            idx = ((uint64_t)lor<kSubL>((uint32_t)(mine >> 32), gm) << 32) | lor<kSubL>((uint32_t)mine, gm);
        } else {  // zap__bc4_eval
            idx = (kind == -1 ? base : nb) >> 16;
            #pragma unroll
            for (int u = 0; u < T; u++) {
                const int d = (int)chan(t[u], S.chan) - P[(int)((idx >> (3 * (q * T + u))) & 7u)];
                e += d * d;
            }
            e = lsum<kSubL>(e, gm);
        }
        r.cand = (uint64_t)a | ((uint64_t)c << 8) | (idx << 16);
    }
    r.e = e;
    // rate inputs (zap__field_rate per field): which window fields equal this candidate's
    uint32_t mA = 0, mB = 0;
    #pragma unroll
    for (int u = 0; u < T; u++) {
        const int d = q * T + u + 1;
        const uint64_t w = ring[(b - d) & (kWindow - 1)];
        if (d >= dlo && d <= b) {
            mA |= (uint32_t)((w & maskA) == (r.cand & maskA)) << (d - 1);
            mB |= (uint32_t)((w >> (8 * nA)) == (r.cand >> (8 * nA))) << (d - 1);
        }
    }
    r.mA = lor<kSubL>(mA, gm);
    r.mB = lor<kSubL>(mB, gm);
    return r;
}

__global__ void __launch_bounds__(kSubThreads, 1) rdo_sub_chain_kernel(SrcU8 src, int bw, int nby, int chain_rows, uint8_t *__restrict__ out,
                                                                      int bs, Sub S0, Sub S1, float lambda) {
    __shared__ uint64_t ring[kWindow];  // the sub-block of the last 16 chosen blocks, slot = block & 15
    __shared__ __align__(16) int ring_pal[kWindow][8];  // their palettes (palette_word)
    __shared__ __align__(16) uint32_t s_tex[3][16];  // block b in slot b % 3
    __shared__ uint64_t s_base[3];
    __shared__ __align__(16) int s_bpal[3][8];  // the base sub-block's palette
    // the candidates of block b by candidate order (0 the base, (j - 1) * 3 + kind + 1 the others), buffer b & 1
    __shared__ uint64_t c_cand[2][49];
    __shared__ uint64_t c_meta[2][49];  // SSE (bit 31 set: not allowed) | mA << 32 | mB << 48
    const Sub S = blockIdx.y ? S1 : S0;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, q = tid & (kSubL - 1), grp = tid / kSubL;
    const int row0 = blockIdx.x * chain_rows, rows = min(chain_rows, nby - row0);
    if (rows <= 0) return;
    const int first = row0 * bw, count = rows * bw;
    // the loader warp: lane i < 16 fetches texel i of a block, every lane its base sub-block
    uint32_t r_tex = 0;
    uint64_t r_base = 0;
    auto fetch = [&](int gk) {
        if (lane < 16) r_tex = load_texel(src, min((gk % bw) * 4 + (lane & 3), src.w - 1), min((gk / bw) * 4 + (lane >> 2), src.h - 1));
        r_base = *(const uint64_t *)(out + (size_t)gk * bs + S.off);
    };
    auto store = [&](int ns) {  // the fetched block into slot ns, with the base's palette
        if (lane < 16) s_tex[ns][lane] = r_tex;
        if (lane < 8) s_bpal[ns][lane] = palette_word(S, r_base, lane);
        if (lane == 0) s_base[ns] = r_base;
    };
    if (warp == kSubLoader) {
        fetch(first);
        store(0);
        if (count > 1) fetch(first + 1);
    }
    __syncthreads();
    // producers: kind and neighbour distance of the group (the idle groups repeat j = 16), which warps hold one kind
    const int pkind = grp < 48 ? grp >> 4 : grp == 48 ? -1 : -3, pj = min((grp & 15) + 2, 16);
    const bool pkeep = grp < 48 ? (grp & 15) < 15 : grp == 48;
    const unsigned pgm = warp < 12 ? 0xFFFFFFFFu : 0xFFu << (lane & 24);
    // the chooser's fields and rates
    const bool bc1 = S.type == kBc1;
    const int nA = bc1 ? 4 : 2, nB = bc1 ? 4 : 6;
    const uint64_t maskA = (1ull << (8 * nA)) - 1ull;
    const float newA = bc1 ? 3.0f : 2.0f, newB = 3.0f;  // min(size, 3)
    int d0 = 1, d1 = 1;  // the chooser's current match distances (zap_tex.h:234)
    for (int it = -1; it < count; it++) {
        const int b = it + 1;  // the producers' block
        if (warp < kSubProducerWarps) {
            if (pkind >= -1 && b < count) {
                const SubCand c = sub_candidate(S, pkind, pj, b, q, pgm, 2, s_tex, s_base, s_bpal, ring, ring_pal);
                if (pkeep && q == 0) {
                    const int o = pkind < 0 ? 0 : (pj - 1) * 3 + pkind + 1;
                    c_cand[b & 1][o] = c.cand;
                    c_meta[b & 1][o] = (uint32_t)c.e | (c.ok ? 0u : 0x80000000u) | ((uint64_t)c.mA << 32) | ((uint64_t)c.mB << 48);
                }
            }
        } else if (warp == kSubFit || warp == kSubEval) {
            // the candidates of neighbour distance 1 (block it - 1, chosen in the previous step): kind 0 on the fit
            // warp's lanes 0-7, kinds 1 and 2 on the evaluation warp's lanes 0-7 and 8-15
            if (it >= 0) {
                const int ck = warp == kSubFit ? 0 : 1 + (lane >> 3);
                if (lane < (warp == kSubFit ? 8 : 16)) {
                    const SubCand c = sub_candidate(S, ck, 1, it, q, warp == kSubFit ? 0xFFu : 0xFFFFu, 1, s_tex, s_base, s_bpal, ring, ring_pal);
                    if (q == 0) {
                        c_cand[it & 1][ck + 1] = c.cand;
                        c_meta[it & 1][ck + 1] = (uint32_t)c.e | (c.ok ? 0u : 0x80000000u) | ((uint64_t)c.mA << 32) | ((uint64_t)c.mB << 48);
                    }
                }
                asm volatile("bar.sync 1, 96;" ::: "memory");  // with the deciding warp
            }
        } else if (warp == kSubDecide) {
            if (it >= 0) {
                const int cur = it, bi = cur & 1;
                const uint64_t w1 = ring[(cur - 1) & (kWindow - 1)];  // the block chosen in the previous step
                uint64_t best = ~0ull;
                int bd0 = d0, bd1 = d1;
                // candidate o's key (zap__field_rate per field, the window's distance-1 bits added for the candidates
                // the producers evaluated), kept if below the lane's best
                auto consider = [&](int o) {
                    const uint64_t cand = c_cand[bi][o], meta = c_meta[bi][o];
                    uint32_t mA = (uint32_t)(meta >> 32) & 0xFFFFu, mB = (uint32_t)(meta >> 48);
                    if ((o == 0 || o > 3) && cur >= 1) {
                        mA |= (uint32_t)((w1 & maskA) == (cand & maskA));
                        mB |= (uint32_t)((w1 >> (8 * nA)) == (cand >> (8 * nA)));
                    }
                    float fa = (float)nA, fb = (float)nB;
                    int nd0 = d0, nd1 = d1;
                    if (d0 > 0 && d0 <= cur && ((mA >> (d0 - 1)) & 1u)) fa = 0.0f;
                    else if (mA) { nd0 = __ffs((int)mA); fa = newA; }
                    if (d1 > 0 && d1 <= cur && ((mB >> (d1 - 1)) & 1u)) fb = 0.0f;
                    else if (mB) { nd1 = __ffs((int)mB); fb = newB; }
                    const int e = (int)(uint32_t)meta;
                    const uint64_t key = e >= 0 ? key_of((float)e + lambda * (fa + fb), o) : ~0ull;
                    if (key < best) { best = key; bd0 = nd0; bd1 = nd1; }
                };
                consider(lane == 0 ? 0 : lane + 3);  // the base and orders 4..34
                if (lane + 35 < 49) consider(lane + 35);  // orders 35..48
                asm volatile("bar.sync 1, 96;" ::: "memory");  // the distance-1 candidates are in
                if (lane >= 1 && lane <= 3) consider(lane);
                const int order = (int)(uint32_t)warp_min_redux(best);
                const int src = order <= 3 ? order : order <= 34 ? order - 3 : order - 35;  // the lane that keyed it
                d0 = __shfl_sync(0xFFFFFFFFu, bd0, src);
                d1 = __shfl_sync(0xFFFFFFFFu, bd1, src);
                // the winner enters the window with its palette (the base's, or the neighbour's: with j = 16 the
                // neighbour's slot is this one, and each lane rewrites its own word)
                const int oc = order - 1, wkind = oc % 3, wj = oc / 3 + 1;
                const uint64_t wc = c_cand[bi][order];
                if (lane < 8) {
                    const int *P = order == 0 || wkind == 1 ? s_bpal[cur % 3] : ring_pal[(cur - wj) & (kWindow - 1)];
                    ring_pal[cur & (kWindow - 1)][lane] = P[lane];
                }
                if (lane == 0) {
                    ring[cur & (kWindow - 1)] = wc;
                    if (order != 0) *(uint64_t *)(out + (size_t)(first + cur) * bs + S.off) = wc;
                }
            }
        } else {  // the loader: block it + 2 (fetched the step before) to shared memory; fetch block it + 3
            if (it + 2 < count) store((it + 2) % 3);
            if (it + 3 < count) fetch(first + it + 3);
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
        constexpr int L = ZTC_RDO_BC7_LANES;
        ztc::rdo_bc7_chain_kernel<L><<<chains, ztc::B7Chain<L>::kThreads, 0, stream>>>(src, bw, nby, band_rows, out, dec, lambda);
        e = cudaGetLastError();
        cudaFreeAsync(dec, stream);
        return e;
    }
    {
        const ztc::Sub S0 = ztc::sub_of(fmt, 0), S1 = ztc::sub_of(fmt, 1);
        const int ns = ztc::sub_count(fmt), bs = fmt == ZTC_FMT_BC1 || fmt == ZTC_FMT_BC4 ? 8 : 16;
        const dim3 grid(chains, ns);
        if (fmt < ZTC_FMT_BC1 || fmt > ZTC_FMT_BC5) return cudaErrorInvalidValue;
        ztc::rdo_sub_chain_kernel<<<grid, ztc::kSubThreads, 0, stream>>>(src, bw, nby, band_rows, out, bs, S0, S1, lambda);
        return cudaGetLastError();
    }
}

// bcn.cu - BC1 / BC3 / BC4 / BC5 block encoders for sm_100a, one thread per 4x4 block.
//
// Bit-exact with the reference encoder (zap_tex.h:39-213 at rdo = 0). The float part (PCA start, least-squares
// refits) keeps the reference's operation order; the palette searches are exact integer work arranged for the GPU:
// a texel's squared distance to palette entry k is |p|^2 + |c_k|^2 - 2 p.c_k, with p.c_k from one dp4a, and
// the key 4 * (|c_k|^2 - 2 p.c_k) + k orders candidates exactly like the reference's first-best scan.
#include "ztc_common.cuh"
#include "ztc_internal.h"

namespace ztc {

// ---------------------------------------------------------------- BC1 (zap_tex.h:39-168)
ZTC_DEV uint32_t pack565(float r, float g, float b) {  // zap_tex.h:45-49
    int R = f2i_x86(div255(r * 31.0f) + 0.5f), G = f2i_x86(div255(g * 63.0f) + 0.5f), B = f2i_x86(div255(b * 31.0f) + 0.5f);
    return ((uint32_t)clampi(R, 0, 31) << 11) | ((uint32_t)clampi(G, 0, 63) << 5) | (uint32_t)clampi(B, 0, 31);
}

struct Bc1Texels {
    uint32_t p[16];  // r, g, b bytes; alpha byte cleared
    int pp;          // sum of |p|^2
    int sr, sg, sb;  // channel sums
};

ZTC_DEV void bc1_prepare(const uint32_t t[16], Bc1Texels &T) {
    T.pp = 0; T.sr = T.sg = T.sb = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        T.p[i] = t[i] & 0x00FFFFFFu;
        T.pp += (int)dot4(T.p[i], T.p[i]);
        T.sr += (int)chan(t[i], 0); T.sg += (int)chan(t[i], 1); T.sb += (int)chan(t[i], 2);
    }
}

// best 2-bit indices and SSE for c0 > c1 (4-colour palette, zap_tex.h:52-80 with force4)
ZTC_DEV int bc1_fit4(const Bc1Texels &T, uint32_t c0, uint32_t c1, uint32_t &idx) {
    int r0, g0, b0, r1, g1, b1;
    unpack565(c0, r0, g0, b0); unpack565(c1, r1, g1, b1);
    uint32_t q0 = pack_rgb(r0, g0, b0), q1 = pack_rgb(r1, g1, b1);
    uint32_t q2 = pack_rgb((2 * r0 + r1 + 1) / 3, (2 * g0 + g1 + 1) / 3, (2 * b0 + b1 + 1) / 3);
    uint32_t q3 = pack_rgb((r0 + 2 * r1 + 1) / 3, (g0 + 2 * g1 + 1) / 3, (b0 + 2 * b1 + 1) / 3);
    int A0 = 4 * (int)dot4(q0, q0), A1 = 4 * (int)dot4(q1, q1) + 1, A2 = 4 * (int)dot4(q2, q2) + 2, A3 = 4 * (int)dot4(q3, q3) + 3;
    uint32_t bits = 0;
    int sum = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        uint32_t p = T.p[i];
        int k0 = A0 - 8 * (int)dot4(p, q0), k1 = A1 - 8 * (int)dot4(p, q1);
        int k2 = A2 - 8 * (int)dot4(p, q2), k3 = A3 - 8 * (int)dot4(p, q3);
        int m = min(min(k0, k1), min(k2, k3));
        sum += m;
        bits |= (uint32_t)(m & 3) << (2 * i);
    }
    idx = bits;
    int ksum = popc(bits & 0x55555555u) + 2 * popc(bits & 0xAAAAAAAAu);
    return ((sum - ksum) >> 2) + T.pp;
}

// canonical order (c0 > c1, or solid c0 == c1 with indices 0) + SSE (zap_tex.h:90-94)
ZTC_DEV int bc1_try(const Bc1Texels &T, uint32_t &c0, uint32_t &c1, uint32_t &idx) {
    if (c0 < c1) { uint32_t s = c0; c0 = c1; c1 = s; }
    if (c0 == c1) {
        int r, g, b;
        unpack565(c0, r, g, b);
        idx = 0;
        return T.pp + 16 * (r * r + g * g + b * b) - 2 * (T.sr * r + T.sg * g + T.sb * b);
    }
    return bc1_fit4(T, c0, c1, idx);
}

ZTC_DEV float bc1_lsw(uint32_t k) { return k == 0 ? 1.0f : k == 1 ? 0.0f : k == 2 ? 2.0f / 3.0f : 1.0f / 3.0f; }

// +-1 climb passes [first, last) over the six 565 channels of the two endpoints, first improvement taken
// immediately (zap_tex.h:146-165); the climb stops early at SSE 0 or after a pass without improvement. Returns
// whether the last pass that ran improved.
ZTC_DEV bool bc1_climb(const Bc1Texels &T, uint32_t &b0, uint32_t &b1, uint32_t &bidx, int &best, int first, int last) {
    bool improved = true;
    for (int pass = first; improved && pass < last && best > 0; pass++) {
        improved = false;
        for (int step = 0; step < 12; step++) {
            int ep = step / 6, ch = (step / 2) % 3, d = (step & 1) ? 1 : -1;
            int sh = ch == 0 ? 11 : ch == 1 ? 5 : 0, mx = ch == 1 ? 63 : 31;
            uint32_t c = ep ? b1 : b0;
            int f = (int)(c >> sh) & mx;
            if (f + d < 0 || f + d > mx) continue;
            c = (c & ~((uint32_t)mx << sh)) | ((uint32_t)(f + d) << sh);
            uint32_t n0 = ep ? b0 : c, n1 = ep ? c : b1, ni = 0;
            int ne = bc1_try(T, n0, n1, ni);
            if (ne < best) { best = ne; b0 = n0; b1 = n1; bidx = ni; improved = true; }
        }
    }
    return improved;
}

template <int UNROLL>
ZTC_DEV uint32_t bc1_texel(const Bc1Texels &T, TexRef tx, int i) { return UNROLL == 1 ? tx[i] : T.p[i]; }

// one start of the quality search (zap_tex.h:118-143): endpoints from the axis, then up to three least-squares refits
template <int UNROLL>
ZTC_DEV void bc1_one_start(const Bc1Texels &T, TexRef tx, int start, float mu0, float mu1, float mu2, float v0, float v1,
                           float v2, float n2, float tmin, float tmax, uint32_t &b0, uint32_t &b1, uint32_t &bidx, int &best) {
    float inset = start ? 0.0f : (tmax - tmin) / 16.0f, lo = (tmin + inset) / n2, hi = (tmax - inset) / n2;
    uint32_t c0 = pack565(mu0 + v0 * hi, mu1 + v1 * hi, mu2 + v2 * hi);
    uint32_t c1 = pack565(mu0 + v0 * lo, mu1 + v1 * lo, mu2 + v2 * lo);
    uint32_t idx = 0;
    int e = bc1_try(T, c0, c1, idx);
    for (int it = 0; it < 3 && e > 0; it++) {
        float aa = 0, ab = 0, bb = 0, sa0 = 0, sa1 = 0, sa2 = 0, sb0 = 0, sb1 = 0, sb2 = 0;
        for_texels<UNROLL>([&](int i) {
            float wa = bc1_lsw((idx >> (2 * i)) & 3u), wb = 1.0f - wa;
            aa = aa + wa * wa; ab = ab + wa * wb; bb = bb + wb * wb;
            const uint32_t x = bc1_texel<UNROLL>(T, tx, i);
            float r = (float)chan(x, 0), g = (float)chan(x, 1), b = (float)chan(x, 2);
            sa0 = sa0 + wa * r; sa1 = sa1 + wa * g; sa2 = sa2 + wa * b;
            sb0 = sb0 + wb * r; sb1 = sb1 + wb * g; sb2 = sb2 + wb * b;
        });
        float det = aa * bb - ab * ab;
        if (det < 1e-6f && det > -1e-6f) break;
        uint32_t n0 = pack565((sa0 * bb - sb0 * ab) / det, (sa1 * bb - sb1 * ab) / det, (sa2 * bb - sb2 * ab) / det);
        uint32_t n1 = pack565((sb0 * aa - sa0 * ab) / det, (sb1 * aa - sa1 * ab) / det, (sb2 * aa - sa2 * ab) / det);
        // the accepted pair again (bc1_try orders it c0 >= c1): the same fit and SSE, which ends the refits
        if (max(n0, n1) == c0 && min(n0, n1) == c1) break;
        uint32_t ni = 0;
        int ne = bc1_try(T, n0, n1, ni);
        if (ne >= e) break;
        e = ne; c0 = n0; c1 = n1; idx = ni;
    }
    if (e < best) { best = e; b0 = c0; b1 = c1; bidx = idx; }
}

// quality search up to the climb (zap_tex.h:97-145): PCA axis, two starts with least-squares refits (the colour
// channels of T.p are the texels' r, g, b)
// UNROLL 16: the texel loops unrolled over T.p (tx unused); UNROLL 1: rolled loops over tx, the block's texels in
// shared memory
template <int UNROLL = 16>
ZTC_DEV void bc1_start(const Bc1Texels &T, TexRef tx, uint32_t &b0, uint32_t &b1, uint32_t &bidx, int &best) {
    // the reference's mean sums x / 16 in texel order; every term and every partial sum is exact (a multiple of 1/16
    // below 256), so the float sum is the channel's integer sum / 16
    const float mu0 = (float)T.sr / 16.0f, mu1 = (float)T.sg / 16.0f, mu2 = (float)T.sb / 16.0f;
    float C0 = 0, C1 = 0, C2 = 0, C3 = 0, C4 = 0, C5 = 0;
    for_texels<UNROLL>([&](int i) {
        const uint32_t x = bc1_texel<UNROLL>(T, tx, i);
        float r = (float)chan(x, 0) - mu0, g = (float)chan(x, 1) - mu1, b = (float)chan(x, 2) - mu2;
        C0 = C0 + r * r; C1 = C1 + r * g; C2 = C2 + r * b; C3 = C3 + g * g; C4 = C4 + g * b; C5 = C5 + b * b;
    });
    float v0 = 1.0f, v1 = 1.0f, v2 = 1.0f;
    for (int it = 0; it < 6; it++) {
        float x = C0 * v0 + C1 * v1 + C2 * v2;
        float y = C1 * v0 + C3 * v1 + C4 * v2;
        float z = C2 * v0 + C4 * v1 + C5 * v2;
        float m = fabsf(x);
        if (fabsf(y) > m) m = fabsf(y);
        if (fabsf(z) > m) m = fabsf(z);
        if (m < 1e-6f) break;
        v0 = x / m; v1 = y / m; v2 = z / m;
    }
    float n2 = v0 * v0 + v1 * v1 + v2 * v2, tmin = 1e9f, tmax = -1e9f;
    for_texels<UNROLL>([&](int i) {
        const uint32_t x = bc1_texel<UNROLL>(T, tx, i);
        float s = ((float)chan(x, 0) - mu0) * v0 + ((float)chan(x, 1) - mu1) * v1 + ((float)chan(x, 2) - mu2) * v2;
        if (s < tmin) tmin = s;
        if (s > tmax) tmax = s;
    });
    b0 = 0; b1 = 0; bidx = 0;
    best = 1 << 30;
    #pragma unroll 1
    for (int start = 0; start < 2; start++)
        bc1_one_start<UNROLL>(T, tx, start, mu0, mu1, mu2, v0, v1, v2, n2, tmin, tmax, b0, b1, bidx, best);
}

// quality search (zap_tex.h:97-168), one thread
ZTC_DEV uint2 bc1_encode(const uint32_t t[16]) {
    Bc1Texels T;
    bc1_prepare(t, T);
    uint32_t b0, b1, bidx;
    int best;
    bc1_start(T, TexRef{nullptr, 0}, b0, b1, bidx, best);
    bc1_climb(T, b0, b1, bidx, best, 0, 8);
    return make_uint2(b0 | (b1 << 16), bidx);
}

// The quality search for the CTA's blocks, one per thread, with the climb past its second pass compacted. Every
// thread runs the starts and the first two climb passes of its block; the blocks whose climb goes on (about a
// tenth on photographic content, yet nearly every warp holds one) are listed in shared memory, and the first
// threads of the CTA climb them on to the end from the owners' texels, so the long tail of the climb costs about
// a tenth of the warps. Same bytes as bc1_encode. Every thread of the CTA calls it (it synchronises); a `valid`
// thread's block is in t and in column threadIdx.x of s_tex.
// ROLLED: the starts' principal axis and least-squares sums run in rolled loops over s_tex (less code, more
// instructions): faster in launches of several waves, slower in a launch of less than one wave, where each
// thread's own chain of dependent instructions sets the time (512x512 BC1: 0.0415 -> 0.0441 ms).
template <int CTA, bool ROLLED>
__device__ __forceinline__ uint2 bc1_encode_cta(bool valid, const uint32_t t[16], uint32_t (*s_tex)[CTA]) {
    static_assert(CTA % 32 == 0 && CTA <= 256, "whole warps, owners fit a byte");
    __shared__ uint32_t s_ends[CTA], s_idx[CTA];
    __shared__ int s_best[CTA], s_wcnt[CTA / 32];
    __shared__ uint8_t s_list[CTA];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    Bc1Texels T;
    uint32_t b0 = 0, b1 = 0, bidx = 0;
    int best = 0;
    if (valid) {
        bc1_prepare(t, T);
        if (ROLLED) bc1_start<1>(T, TexRef{&s_tex[0][tid], CTA}, b0, b1, bidx, best);
        else bc1_start(T, TexRef{nullptr, 0}, b0, b1, bidx, best);
    }
    bool active = valid;
    int owner = tid;
    #pragma unroll 1
    for (int round = 0; round < 2; round++) {
        bool more = false;
        if (active) more = bc1_climb(T, b0, b1, bidx, best, round ? 2 : 0, round ? 8 : 2) && best > 0;
        if (active) { s_ends[owner] = b0 | (b1 << 16); s_idx[owner] = bidx; s_best[owner] = best; }
        if (round == 1) break;
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, more);
        if (lane == 0) s_wcnt[warp] = __popc(bal);
        __syncthreads();
        int base = 0, total = 0;
        #pragma unroll
        for (int w = 0; w < CTA / 32; w++) { const int c = s_wcnt[w]; base += w < warp ? c : 0; total += c; }
        const int pos = base + __popc(bal & ((1u << lane) - 1u));
        if (more && ZTC_IN_BOUNDS(pos, CTA, 3)) s_list[pos] = (uint8_t)tid;
        __syncthreads();
        active = tid < total;
        if (active) owner = s_list[tid];
        if (active && !ZTC_IN_BOUNDS(owner, CTA, 8)) active = false;
        if (active) {
            uint32_t u[16];
            #pragma unroll
            for (int i = 0; i < 16; i++) u[i] = s_tex[i][owner];
            bc1_prepare(u, T);
            b0 = s_ends[owner] & 0xFFFFu; b1 = s_ends[owner] >> 16; bidx = s_idx[owner]; best = s_best[owner];
        }
    }
    __syncthreads();
    return make_uint2(s_ends[tid], s_idx[tid]);
}

// ---------------------------------------------------------------- BC4 (zap_tex.h:170-213)
ZTC_DEV uint2 bc4_encode(const uint32_t t[16], int c) {
    int v[16], lo = 255, hi = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) { v[i] = (int)chan(t[i], c); lo = min(lo, v[i]); hi = max(hi, v[i]); }
    int best = 1 << 30, ba0 = hi, ba1 = lo;
    uint64_t bidx = 0;
    for (int cand = 0; cand < 9; cand++) {
        int a0 = hi - cand / 3, a1 = lo + cand % 3;
        if (a0 <= a1) { a0 = hi; a1 = lo; }
        int err = 0;
        uint64_t bits = 0;
        if (a0 == a1) {
            #pragma unroll
            for (int i = 0; i < 16; i++) err += (v[i] - a0) * (v[i] - a0);
        } else {
            int p[8];
            p[0] = a0; p[1] = a1;
            #pragma unroll
            for (int k = 2; k < 8; k++) p[k] = ((8 - k) * a0 + (k - 1) * a1 + 3) / 7;
            #pragma unroll
            for (int i = 0; i < 16; i++) {
                int m = 1 << 30;
                #pragma unroll
                for (int k = 0; k < 8; k++) { int d = v[i] - p[k]; m = min(m, d * d * 8 + k); }
                err += m >> 3;
                bits |= (uint64_t)(m & 7) << (3 * i);
            }
        }
        if (err < best) { best = err; ba0 = a0; ba1 = a1; bidx = bits; }
    }
    return make_uint2((uint32_t)ba0 | ((uint32_t)ba1 << 8) | ((uint32_t)(bidx & 0xFFFFu) << 16), (uint32_t)(bidx >> 16));
}

// ---------------------------------------------------------------- kernel: one thread per block
// CTA sizes of the BC1-BC5 kernel. For BC1 / BC3 a larger CTA shares one list of compacted climbs among more
// blocks (2048x2048 BC1: 64 threads 0.217 ms, 128 0.189, 256 0.185; BC4 the same at all three); a launch smaller
// than one full wave of large CTAs takes the small size, which keeps more SMs busy. BC1 / BC3 take 224 threads at
// 4 CTAs per SM (72 registers; 2048x2048 BC1 fills 1.98 waves instead of 1.73: 0.172 -> 0.168 ms); BC4 / BC5 keep
// 256 (224 measured 0.0558 -> 0.0567 ms on BC4).
constexpr int kBcnSmall = 128;
template <int FMT>
constexpr int bcn_large() { return FMT == ZTC_FMT_BC1 || FMT == ZTC_FMT_BC3 ? 224 : 256; }
template <int FMT, int CTA>
__global__ void __launch_bounds__(CTA, ZTC_MINB_BCN * 128 / CTA) bcn_kernel(SrcU8 src, int bw, int by0, int nblocks, BlockOut out, size_t b0) {
    constexpr bool kColour = FMT == ZTC_FMT_BC1 || FMT == ZTC_FMT_BC3;
    __shared__ uint32_t s_tex[16][kColour ? CTA : 1];  // column threadIdx.x: this thread's block (BC1 / BC3)
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = b < nblocks;
    if (!kColour && !valid) return;  // BC4 / BC5 never synchronise
    uint32_t t[16];
    if (valid) {
        gather_block(src, b % bw, by0 + b / bw, t);
        if (kColour) {
            #pragma unroll
            for (int i = 0; i < 16; i++) s_tex[i][threadIdx.x] = t[i];
        }
    }
    const size_t ob = b0 + (size_t)b;  // the block's index in the output
    if (FMT == ZTC_FMT_BC1) {
        const uint2 c = bc1_encode_cta<CTA, CTA != kBcnSmall>(valid, t, (uint32_t(*)[CTA])s_tex);
        if (valid) put_block8(out, ob, c);
    } else if (FMT == ZTC_FMT_BC4) {
        put_block8(out, ob, bc4_encode(t, 0));
    } else if (FMT == ZTC_FMT_BC3) {
        uint2 a = valid ? bc4_encode(t, 3) : make_uint2(0u, 0u);
        const uint2 c = bc1_encode_cta<CTA, CTA != kBcnSmall>(valid, t, (uint32_t(*)[CTA])s_tex);
        if (valid) put_block16(out, ob, make_uint4(a.x, a.y, c.x, c.y));
    } else {  // BC5
        uint2 r = bc4_encode(t, 0), g = bc4_encode(t, 1);
        put_block16(out, ob, make_uint4(r.x, r.y, g.x, g.y));
    }
}

}  // namespace ztc

cudaError_t ztc_launch_bcn_to(int fmt, const ztc::SrcU8 &src, int by0, int nby, const ztc::BlockOut &out, size_t b0, cudaStream_t stream) {
    int bw = (src.w + 3) / 4, nblocks = bw * nby;
    if (nblocks <= 0) return cudaSuccess;
    static const char *names[4] = {"bc1_encode", "bc3_encode", "bc4_encode", "bc5_encode"};
    ztc::TraceScope tr(fmt >= 0 && fmt < 4 ? names[fmt] : "bcn_encode", stream);
    ztc::trace_units(nblocks);
#define ZTC_BCN_LAUNCH(F)                                                                                              \
    do {                                                                                                               \
        constexpr int kLarge = ztc::bcn_large<F>();                                                                    \
        const bool large = nblocks >= ztc_sm_count() * (ZTC_MINB_BCN * 128 / kLarge) * kLarge;                        \
        const int cta = large ? kLarge : ztc::kBcnSmall, grid = (nblocks + cta - 1) / cta;                            \
        if (large) ztc::bcn_kernel<F, kLarge><<<grid, cta, 0, stream>>>(src, bw, by0, nblocks, out, b0);               \
        else ztc::bcn_kernel<F, ztc::kBcnSmall><<<grid, cta, 0, stream>>>(src, bw, by0, nblocks, out, b0);            \
    } while (0)
    switch (fmt) {
    case ZTC_FMT_BC1: ZTC_BCN_LAUNCH(ZTC_FMT_BC1); break;
    case ZTC_FMT_BC3: ZTC_BCN_LAUNCH(ZTC_FMT_BC3); break;
    case ZTC_FMT_BC4: ZTC_BCN_LAUNCH(ZTC_FMT_BC4); break;
    case ZTC_FMT_BC5: ZTC_BCN_LAUNCH(ZTC_FMT_BC5); break;
    default: return cudaErrorInvalidValue;
    }
#undef ZTC_BCN_LAUNCH
    return cudaGetLastError();
}

cudaError_t ztc_launch_bcn(int fmt, const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, cudaStream_t stream) {
    return ztc_launch_bcn_to(fmt, src, by0, nby, ztc::BlockOut{out, 0, fmt, 0}, 0, stream);
}

// ---------------------------------------------------------------- batched: one persistent launch over a tile queue
// A CTA takes one tile at a time and runs it in chunks of CTA blocks (a tile holds a multiple of the CTA's blocks:
// blocks per tile and CTA size are separate knobs of the batch autotuner, as are the tile's shape, a row strip or a
// 2-D tile, and MINB, the minimum resident CTAs of 128 threads per SM that sets the register cap).
namespace ztc {
template <int FMT, int CTA, int MINB>
__global__ void __launch_bounds__(CTA, MINB * 128 / CTA) batch_bcn_kernel(const BatchLevel *__restrict__ levels, const BatchTile *__restrict__ tiles,
                                                                         int ntiles, uint32_t *__restrict__ counter) {
    constexpr bool kColour = FMT == ZTC_FMT_BC1 || FMT == ZTC_FMT_BC3;
    __shared__ int s_tile;
    __shared__ uint32_t s_tex[16][kColour ? CTA : 1];  // column threadIdx.x: this thread's block (BC1 / BC3)
    for (;;) {
        if (threadIdx.x == 0) s_tile = (int)atomicAdd(counter, 1u);
        __syncthreads();
        const int tile = s_tile;
        __syncthreads();  // every thread has read s_tile before thread 0 overwrites it
        if (tile >= ntiles) break;
        const BatchTile T = tiles[tile];
        const BatchLevel L = levels[T.level];
        const SrcU8 src{L.src, L.pitch, L.w, L.h, 4, (((uintptr_t)L.src | L.pitch) & 15u) == 0};
        for (int j0 = 0; j0 < T.count; j0 += CTA) {  // the same trip count in every thread: barriers stay uniform
            const int j = j0 + (int)threadIdx.x;
            const bool valid = j < T.count;
            if (!kColour && !valid) continue;  // BC4 / BC5 never synchronise inside a tile
            const int b = tile_block(T, L.bw, j);
            uint32_t t[16];
            if (valid) {
                gather_block(src, b % L.bw, b / L.bw, t);
                if (kColour) {
                    #pragma unroll
                    for (int i = 0; i < 16; i++) s_tex[i][threadIdx.x] = t[i];
                }
            }
            if (FMT == ZTC_FMT_BC1) {
                const uint2 c = bc1_encode_cta<CTA, true>(valid, t, (uint32_t(*)[CTA])s_tex);
                if (valid) store_block8(L.dst + (size_t)b * 8, c);
            } else if (FMT == ZTC_FMT_BC4) store_block8(L.dst + (size_t)b * 8, bc4_encode(t, 0));
            else if (FMT == ZTC_FMT_BC3) {
                const uint2 a = valid ? bc4_encode(t, 3) : make_uint2(0u, 0u);
                const uint2 c = bc1_encode_cta<CTA, true>(valid, t, (uint32_t(*)[CTA])s_tex);
                if (valid) store_block16(L.dst + (size_t)b * 16, make_uint4(a.x, a.y, c.x, c.y));
            } else {
                uint2 r = bc4_encode(t, 0), g = bc4_encode(t, 1);
                store_block16(L.dst + (size_t)b * 16, make_uint4(r.x, r.y, g.x, g.y));
            }
            if (kColour) __syncthreads();  // the next chunk overwrites s_tex
        }
    }
}

template <int FMT, int MINB>
static const void *batch_fn_cap(int cta) {
    switch (cta) {
    case 64: return (const void *)batch_bcn_kernel<FMT, 64, MINB>;
    case 128: return (const void *)batch_bcn_kernel<FMT, 128, MINB>;
    case 256: return (const void *)batch_bcn_kernel<FMT, 256, MINB>;
    default: return nullptr;
    }
}
template <int FMT>
static const void *batch_fn(int cta, int regs) {
    return regs ? batch_fn_cap<FMT, ZTC_MINB_BCN_BATCH_LOOSE>(cta) : batch_fn_cap<FMT, ZTC_MINB_BCN_BATCH>(cta);
}
}  // namespace ztc

const void *ztc_batch_bcn_kernel_fn(int fmt, int cta, int regs) {
    switch (fmt) {
    case ZTC_FMT_BC1: return ztc::batch_fn<ZTC_FMT_BC1>(cta, regs);
    case ZTC_FMT_BC3: return ztc::batch_fn<ZTC_FMT_BC3>(cta, regs);
    case ZTC_FMT_BC4: return ztc::batch_fn<ZTC_FMT_BC4>(cta, regs);
    case ZTC_FMT_BC5: return ztc::batch_fn<ZTC_FMT_BC5>(cta, regs);
    default: return nullptr;
    }
}

cudaError_t ztc_launch_batch_bcn(int fmt, int cta, int regs, int grid, const ztc::BatchLevel *levels, const ztc::BatchTile *tiles, int ntiles,
                                 uint32_t *counter, cudaStream_t stream) {
    const void *fn = ztc_batch_bcn_kernel_fn(fmt, cta, regs);
    if (!fn) return cudaErrorInvalidValue;
    void *args[] = {(void *)&levels, (void *)&tiles, (void *)&ntiles, (void *)&counter};
    return cudaLaunchKernel(fn, dim3(grid), dim3(cta), args, 0, stream);
}

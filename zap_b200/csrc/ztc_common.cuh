// ztc_common.cuh - device helpers shared by the zap_tex CUDA kernels (sm_100a).
//
// Numerics contract: the kernels reproduce the reference encoder's float results bit for bit. The build uses
// -fmad=false (no FMA contraction), IEEE division and square root, and every float accumulation keeps the
// reference's sequential order; integer searches keep the first candidate on ties (strict "<").
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

// Per-block encoder functions are host+device: the device build is the product; the host build lets the CPU test
// suite run the same block logic against the oracle without a GPU (tests/test_block_logic_on_host.py).
#define ZTC_DEV __host__ __device__ __forceinline__

// Minimum resident 128-thread CTAs per SM requested from the register allocator, per kernel (tuned on B200:
// more resident warps hide the latency of these long dependent integer / float chains; see the ncu summaries).
// Measured on 2048x2048 encodes (re-swept after the loops were rolled): bc7_mode6 0.120 -> 0.113 ms at 6 (85
// registers; the small spill stays in L1), BC1 -1.2 % at 8, ASTC single-partition -4 % at 5, BC6H (texels staged in
// shared memory) 0.383 -> 0.351 ms at 5 against 3; the batched BC7 mode-1 kernel (118 registers already allow 4
// CTAs) gains nothing from more.
#ifndef ZTC_MINB_BC7_MODE6
#define ZTC_MINB_BC7_MODE6 6
#endif
#ifndef ZTC_MINB_BC7_HARD
#define ZTC_MINB_BC7_HARD 1
#endif
// the mode-5 launches (single image and batch): resident 64-thread CTAs per SM
#ifndef ZTC_MINB_BC7_MODE5
#define ZTC_MINB_BC7_MODE5 8
#endif
#ifndef ZTC_MINB_BCN
#define ZTC_MINB_BCN 8
#endif
#ifndef ZTC_MINB_BCN_BATCH
#define ZTC_MINB_BCN_BATCH ZTC_MINB_BCN
#endif
// the batched encoder's second register cap (its autotuner picks per format): fewer resident CTAs, fewer spills
#ifndef ZTC_MINB_BCN_BATCH_LOOSE
#define ZTC_MINB_BCN_BATCH_LOOSE 5
#endif
#ifndef ZTC_MINB_BC7_BATCH_LOOSE
#define ZTC_MINB_BC7_BATCH_LOOSE 4
#endif
#ifndef ZTC_MINB_ASTC_SINGLE
#define ZTC_MINB_ASTC_SINGLE 5
#endif
#ifndef ZTC_MINB_BC6H
#define ZTC_MINB_BC6H 5
#endif

// ---------------------------------------------------------------- bounds checks (the ZTC_CHECKS build)
// ZTC_IN_BOUNDS(i, n, site) is true when 0 <= i < n. The checks build (-DZTC_CHECKS, relocatable device code,
// zap_b200/lib/libzap_tex_cuda_checks.so) also records a failure in the device word ztc_check_word, as
// (site << 24) | (i & 0xFFFFFF), keeping the first one, and the caller skips the access; no kernel traps or waits.
// zap_tex_cuda_debug_checks reads and clears the word. In the product build every check compiles to `true`.
// Sites: 1 texel gather, 2 BC7 mode-6 refit list, 3 BC1 climb list, 4 BC6H refit list, 5 ASTC fit list (shared
// memory), 6 BC7 work list, 7 ASTC work list (global memory), 8 a compacted list's owner (shared memory index),
// 9 a conversion-free truncation's argument outside the domain its caller proves (ZTC_TRUNC_DOMAIN; i = 0).
#ifdef ZTC_CHECKS
extern __device__ unsigned int ztc_check_word;
namespace ztc {
ZTC_DEV bool in_bounds(long long i, long long n, unsigned site) {
    const bool ok = i >= 0 && i < n;
#ifdef __CUDA_ARCH__
    if (!ok) atomicCAS(&ztc_check_word, 0u, (site << 24) | ((unsigned)i & 0xFFFFFFu));
#endif
    return ok;
}
}  // namespace ztc
#define ZTC_IN_BOUNDS(i, n, site) ::ztc::in_bounds((long long)(i), (long long)(n), (site))
#define ZTC_TRUNC_DOMAIN(x) ((void)::ztc::in_bounds(fabsf(x) < 4194304.0f ? 0 : -1, 1, 9))
#else
#define ZTC_IN_BOUNDS(i, n, site) true
#define ZTC_TRUNC_DOMAIN(x) ((void)0)
#endif

namespace ztc {

#ifdef __CUDA_ARCH__
ZTC_DEV uint32_t dot4(uint32_t a, uint32_t b) { return __dp4a(a, b, 0u); }  // sum of byte products (exact, unsigned)
ZTC_DEV int popc(uint32_t v) { return __popc(v); }
ZTC_DEV uint32_t f_as_u(float f) { return __float_as_uint(f); }
ZTC_DEV float u_as_f(uint32_t u) { return __uint_as_float(u); }
ZTC_DEV uint32_t brev(uint32_t v) { return __brev(v); }
ZTC_DEV int trunc_i(float f) { return __float2int_rz(f); }
ZTC_DEV float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
template <typename T> ZTC_DEV T ldg(const T *p) { return __ldg(p); }
#else
inline uint32_t dot4(uint32_t a, uint32_t b) {
    uint32_t s = 0;
    for (int k = 0; k < 4; k++) s += ((a >> (8 * k)) & 0xFFu) * ((b >> (8 * k)) & 0xFFu);
    return s;
}
inline int popc(uint32_t v) { return __builtin_popcount(v); }
inline uint32_t f_as_u(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float u_as_f(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint32_t brev(uint32_t v) { uint32_t r = 0; for (int k = 0; k < 32; k++) r |= ((v >> k) & 1u) << (31 - k); return r; }
inline int trunc_i(float f) { return (int)f; }  // only called on in-range values
inline float fma_rn(float a, float b, float c) { return std::fmaf(a, b, c); }
template <typename T> inline T ldg(const T *p) { return *p; }
#endif

// C's (int)f as the reference is compiled for x86-64 (cvttss2si): truncation toward zero, and INT_MIN for NaN or
// any value outside [-2^31, 2^31). CUDA's own conversion saturates instead, so out-of-range values (possible in
// degenerate least-squares solves) would otherwise decode differently.
ZTC_DEV int f2i_x86(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? trunc_i(f) : (int)0x80000000;
}
// min/max form on purpose: with nvcc 12.9 for sm_100a, the equivalent ternary chain followed by an equality test on
// the clamped value (the BC6H endpoint unquantiser) was observed to produce wrong results on the device (a
// mid-range value took the == 1023 branch); the host build and this form are correct.
ZTC_DEV int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }
// an integer in [0, 2^23) as a float, exactly: 2^23 + n has n as its mantissa bits, and subtracting 2^23 is exact
// (one logic op and one add instead of a conversion, which issues at a quarter of the rate)
ZTC_DEV float small_u2f(uint32_t n) { return u_as_f(0x4B000000u | n) - 8388608.0f; }
// (int)v for v in [0, 2^23): v + 2^23 rounded toward zero holds floor(v) in its mantissa bits (an add instead of a
// conversion)
ZTC_DEV int trunc_small(float v) {
#ifdef __CUDA_ARCH__
    return (int)(__float_as_uint(__fadd_rz(v, 8388608.0f)) & 0x7FFFFFu);
#else
    return (int)v;
#endif
}
// (int)v, truncation toward zero, for |v| < 2^23 (f2i_x86 on that domain), without a conversion
ZTC_DEV int trunc_mid(float v) {
#ifdef __CUDA_ARCH__
    const int m = (int)(__float_as_uint(__fadd_rz(fabsf(v), 8388608.0f)) & 0x7FFFFFu);
    return v < 0.0f ? -m : m;
#else
    return (int)v;
#endif
}
ZTC_DEV float clamp255(float v) { return v < 0.0f ? 0.0f : v > 255.0f ? 255.0f : v; }  // NaN passes through
// x / 255 correctly rounded, without a division instruction sequence: Markstein's method (P. Markstein,
// "Computation of elementary functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990):
// q = RN(x * RN(1/255)) is within an ulp of x / 255, the remainder x - 255 q is exact in one FMA, and
// RN(q + remainder * RN(1/255)) is the correctly rounded quotient. Equal to IEEE x / 255.0f for every finite float x
// (the host test checks all of them) except -0, which gives +0 (every caller adds to the quotient before it rounds
// to an integer, which erases the sign of a zero); NaN gives NaN.
ZTC_DEV float div255(float x) {
    constexpr float kInv = 0x1.010102p-8f;  // RN(1 / 255)
    const float q = x * kInv;
    return fma_rn(fma_rn(-255.0f, q, x), kInv, q);
}
// x / n for an integer-valued x in [0, 2^24) and an integer n in [1, 16] or n = 31, from ni = RN(1/n): the same
// correction as div255, exact on that whole domain (the host test enumerates it). The callers' operands are texel channel values
// or products of two sums of at most 16 of them (at most 4080^2 < 2^24), all exact integers in float.
ZTC_DEV float div_small(float x, float n, float ni) {
    const float q = x * ni;
    return fma_rn(fma_rn(-n, q, x), ni, q);
}
// candidate k of {g-1, g, g+1}, wrapping like the reference's compiled three-candidate loops
ZTC_DEV int around(int g, int k) { return (int)((unsigned)g + (unsigned)k - 1u); }

// BC7 / BC6H interpolation weights (format spec tables 0,21,43,64 / 0,9,..,64 / 0,4,..,64) as exact formulas
ZTC_DEV int w2(int j) { return (64 * j + 1) / 3; }
ZTC_DEV int w3(int j) { return (64 * j + 3) / 7; }
ZTC_DEV int w4(int j) { return (64 * j + 7) / 15; }
ZTC_DEV int wbits(int bits, int j) { return bits == 2 ? w2(j) : bits == 3 ? w3(j) : w4(j); }
ZTC_DEV int lerp64(int a, int b, int w) { return ((64 - w) * a + w * b + 32) >> 6; }
// lerp64 over four 8-bit channels at once, packed like a texel. The sum inside lerp64 is 64 a + 32 + (b - a) w, in
// [0, 2^14) for 8-bit a, b and 0 <= w <= 64, so two channels share a word as 16-bit fields (R with B, G with A):
// one multiply-add computes both (a negative slope borrows from the upper field, but both fields' results are exact
// and non-negative, so they separate), and bits 6..13 of each field are the channel's value
struct Lerp4 {
    uint32_t rb, ga, srb, sga;
    ZTC_DEV Lerp4(const int x0[4], const int x1[4]) {  // 8-bit endpoint channels
        rb = (uint32_t)(64 * x0[0] + 32) | ((uint32_t)(64 * x0[2] + 32) << 16);
        ga = (uint32_t)(64 * x0[1] + 32) | ((uint32_t)(64 * x0[3] + 32) << 16);
        srb = (uint32_t)(x1[0] - x0[0]) + ((uint32_t)(x1[2] - x0[2]) << 16);  // modulo 2^32, as the sums are
        sga = (uint32_t)(x1[1] - x0[1]) + ((uint32_t)(x1[3] - x0[3]) << 16);
    }
    ZTC_DEV uint32_t at(int w) const {  // the four channels' lerp64 at weight w, as a texel
        const uint32_t a = rb + srb * (uint32_t)w, b = ga + sga * (uint32_t)w;
        return ((a >> 6) & 0x00FF00FFu) | ((b << 2) & 0xFF00FF00u);
    }
};
ZTC_DEV int expand_bits(int v, int n) { v <<= 8 - n; return v | (v >> n); }  // n-bit -> 8-bit replication

// endpoint quantisation with a fixed p-bit (zap_tex.h:426-438); q: stored values, x8: expanded 8-bit values. The
// endpoints v are finite and within [-510, 765]: least-squares ones are clamped to [0, 255], and a principal-axis
// start is the mean (in the cube) plus an offset no longer than a texel's distance from it (at most 255 * 2).
// So the guess lies in (-256, 384) and d * d below 2^20, where the conversion-free truncations equal f2i_x86.
template <int NC>
ZTC_DEV int quant_pbit(const float v[4], int n, int p, int q[4], int x8[4]) {
    int err = 0, top = (1 << (n - 1)) - 1;
    #pragma unroll
    for (int c = 0; c < NC; c++) {
        const float gv = (div255(v[c]) * (float)((1 << n) - 1) - (float)p) / 2.0f + 0.5f;
        ZTC_TRUNC_DOMAIN(gv);
        int g = trunc_mid(gv), bq = 0, be = 1 << 30;
        #pragma unroll
        for (int k = 0; k < 3; k++) {
            int tq = clampi(around(g, k), 0, top);
            float d = small_u2f((uint32_t)expand_bits((tq << 1) | p, n)) - v[c];
            ZTC_TRUNC_DOMAIN(d * d);
            int e = trunc_small(d * d);
            if (e < be) { be = e; bq = tq; }
        }
        q[c] = bq; x8[c] = expand_bits((bq << 1) | p, n); err += be;
    }
    return err;
}

// 565 endpoint -> 8-bit RGB by bit replication (zap_tex.h:41-44)
ZTC_DEV void unpack565(uint32_t c, int &r, int &g, int &b) {
    int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
    r = (R << 3) | (R >> 2); g = (G << 2) | (G >> 4); b = (B << 3) | (B >> 2);
}

ZTC_DEV uint32_t chan(uint32_t t, int c) { return (t >> (8 * c)) & 0xFFu; }
ZTC_DEV uint32_t pack_rgb(int r, int g, int b) { return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16); }
ZTC_DEV uint32_t pack_rgba(int r, int g, int b, int a) { return pack_rgb(r, g, b) | ((uint32_t)a << 24); }

// 128-bit little-endian block assembled LSB-first in registers (the reference's bit-writer order)
struct Bits128 {
    uint32_t w[4];
    int pos;
    ZTC_DEV Bits128() : pos(0) { w[0] = w[1] = w[2] = w[3] = 0u; }
    ZTC_DEV void put(uint32_t v, int n) {  // n <= 16; v < 2^n
        int word = pos >> 5, sh = pos & 31;
        uint32_t lo = v << sh, hi = sh ? (v >> (32 - sh)) : 0u;
        #pragma unroll
        for (int k = 0; k < 4; k++) {
            if (k == word) w[k] |= lo;
            if (k == word + 1 && sh + n > 32) w[k] |= hi;
        }
        pos += n;
    }
    ZTC_DEV void set_bit(int bit) {
        #pragma unroll
        for (int k = 0; k < 4; k++) if (k == (bit >> 5)) w[k] |= 1u << (bit & 31);
    }
};
ZTC_DEV uint32_t get_bits128(const uint32_t w[4], int pos, int n) {  // n <= 16, pos + n <= 128
    uint64_t lo = 0;
    int word = pos >> 5, sh = pos & 31;
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        if (k == word) lo |= (uint64_t)w[k];
        if (k == word + 1) lo |= (uint64_t)w[k] << 32;
    }
    return (uint32_t)(lo >> sh) & ((1u << n) - 1u);
}

// ---------------------------------------------------------------- texel gather (zap_tex.h:1483-1488)
// Source description: texels of `channels` uint8 each (1, 2 or 4); missing channels read as 0, alpha as 255.
struct SrcU8 {
    const uint8_t *base;
    size_t stride;  // bytes per row
    int w, h, channels;
    int vec16;      // base and stride are 16-byte aligned and channels == 4
};

ZTC_DEV uint32_t load_texel(const SrcU8 &s, int x, int y) {
    const uint8_t *p = s.base + (size_t)y * s.stride + (size_t)x * (size_t)s.channels;
    if (s.channels == 4) {
        if ((((uintptr_t)p) & 3u) == 0) return ldg((const uint32_t *)p);
        return (uint32_t)ldg(p) | ((uint32_t)ldg(p + 1) << 8) | ((uint32_t)ldg(p + 2) << 16) | ((uint32_t)ldg(p + 3) << 24);
    }
    if (s.channels == 2) return (uint32_t)ldg(p) | ((uint32_t)ldg(p + 1) << 8) | 0xFF000000u;
    return (uint32_t)ldg(p) | 0xFF000000u;
}

// 16 texels of block (bx, by), texel i at (i & 3, i >> 2), clamped to the image like the reference
ZTC_DEV void gather_block(const SrcU8 &s, int bx, int by, uint32_t t[16]) {
    int x0 = bx * 4, y0 = by * 4;
    if (!ZTC_IN_BOUNDS(x0, s.w, 1) || !ZTC_IN_BOUNDS(y0, s.h, 1)) {  // a block outside the image: nothing is read
        for (int i = 0; i < 16; i++) t[i] = 0;
        return;
    }
    if (s.vec16 && x0 + 3 < s.w && y0 + 3 < s.h) {
        #pragma unroll
        for (int r = 0; r < 4; r++) {
            uint4 v = ldg((const uint4 *)(s.base + (size_t)(y0 + r) * s.stride + (size_t)x0 * 4));
            t[4 * r + 0] = v.x; t[4 * r + 1] = v.y; t[4 * r + 2] = v.z; t[4 * r + 3] = v.w;
        }
        return;
    }
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        int x = min(x0 + (i & 3), s.w - 1), y = min(y0 + (i >> 2), s.h - 1);
        t[i] = load_texel(s, x, y);
    }
}

// The block's texels as the rolled per-texel loops read them: texel i at p[i * stride]. On the device this is a
// shared-memory copy of the block, so those loops need not be unrolled over registers and the kernels' code stays
// small enough for the instruction cache (fully unrolled 16-texel x 16-entry palette scans, inlined at several
// call sites, leave the warps waiting on instruction fetch).
// f(0) .. f(15) in texel order: fully unrolled (UNROLL 16), or rolled (UNROLL 1) for loops over a TexRef
template <int UNROLL, typename F>
ZTC_DEV void for_texels(F &&f) {
    static_assert(UNROLL == 1 || UNROLL == 16, "rolled or fully unrolled");
    if (UNROLL == 1) {
        #pragma unroll 1
        for (int i = 0; i < 16; i++) f(i);
    } else {
        #pragma unroll
        for (int i = 0; i < 16; i++) f(i);
    }
}

struct TexRef {
    const uint32_t *p;
    int stride;
    ZTC_DEV uint32_t operator[](int i) const { return p[i * stride]; }
};

ZTC_DEV void store_block8(uint8_t *out, uint2 v) { *(uint2 *)out = v; }
ZTC_DEV void store_block16(uint8_t *out, uint4 v) { *(uint4 *)out = v; }

// ---------------------------------------------------------------- block fields (zap_tex.h:1549-1571)
// The split form of an encoded image: plane k holds field k of every block, the planes one after another.
// Fields, in block order: BC1 {4, 4} (endpoints, indices), BC3 {2, 6, 4, 4}, BC4 {2, 6}, BC5 {2, 6, 2, 6},
// BC7 {8, 1, 7}.
ZTC_DEV int bc_fields(int fmt, int sz[4]) {
    sz[0] = sz[1] = sz[2] = sz[3] = 0;
    switch (fmt) {
    case 0: sz[0] = 4; sz[1] = 4; return 2;
    case 1: sz[0] = 2; sz[1] = 6; sz[2] = 4; sz[3] = 4; return 4;
    case 2: sz[0] = 2; sz[1] = 6; return 2;
    case 3: sz[0] = 2; sz[1] = 6; sz[2] = 2; sz[3] = 6; return 4;
    case 4: sz[0] = 8; sz[1] = 1; sz[2] = 7; return 3;
    default: return 0;
    }
}

// Where an encoder puts block b: raster block order (base + b * block bytes), or, with split set, the field planes
// of an image of nblocks blocks (field k of block b at base + nblocks * (offset of field k) + b * (size of field k)),
// so a caller who stores or compresses the split form gets it without a second pass over the blocks.
struct BlockOut {
    uint8_t *base;
    size_t nblocks;
    int fmt, split;
};
ZTC_DEV void put_block(const BlockOut &o, size_t b, const uint32_t w[4], int bytes) {
    if (!o.split) {
        if (bytes == 8) store_block8(o.base + b * 8, make_uint2(w[0], w[1]));
        else store_block16(o.base + b * 16, make_uint4(w[0], w[1], w[2], w[3]));
        return;
    }
    int sz[4];
    const int nf = bc_fields(o.fmt, sz);
    int off = 0;
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        if (k >= nf) break;
        uint8_t *dst = o.base + o.nblocks * (size_t)off + b * (size_t)sz[k];
        for (int j = 0; j < sz[k]; j++) {
            const int i = off + j;  // byte i of the block (selects, not an indexed load: w stays in registers)
            const uint32_t x = i < 4 ? w[0] : i < 8 ? w[1] : i < 12 ? w[2] : w[3];
            dst[j] = (uint8_t)(x >> (8 * (i & 3)));
        }
        off += sz[k];
    }
}
ZTC_DEV void put_block8(const BlockOut &o, size_t b, uint2 v) { const uint32_t w[4] = {v.x, v.y, 0u, 0u}; put_block(o, b, w, 8); }
ZTC_DEV void put_block16(const BlockOut &o, size_t b, uint4 v) { const uint32_t w[4] = {v.x, v.y, v.z, v.w}; put_block(o, b, w, 16); }

}  // namespace ztc

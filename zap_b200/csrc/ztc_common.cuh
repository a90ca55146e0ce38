// ztc_common.cuh - device helpers shared by the zap_tex CUDA kernels (sm_100a).
//
// Numerics contract: the kernels reproduce the reference encoder's float results bit for bit. The build uses
// -fmad=false (no FMA contraction), IEEE division and square root, and every float accumulation keeps the
// reference's sequential order; integer searches keep the first candidate on ties (strict "<").
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#define ZTC_DEV __device__ __forceinline__

namespace ztc {

// C's (int)f as the reference is compiled for x86-64 (cvttss2si): truncation toward zero, and INT_MIN for NaN or
// any value outside [-2^31, 2^31). CUDA's own conversion saturates instead, so out-of-range values (possible in
// degenerate least-squares solves) would otherwise decode differently.
ZTC_DEV int f2i_x86(float f) {
    return (f >= -2147483648.0f && f < 2147483648.0f) ? __float2int_rz(f) : (int)0x80000000;
}
ZTC_DEV int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }
ZTC_DEV float clamp255(float v) { return v < 0.0f ? 0.0f : v > 255.0f ? 255.0f : v; }  // NaN passes through
// candidate k of {g-1, g, g+1}, wrapping like the reference's compiled three-candidate loops
ZTC_DEV int around(int g, int k) { return (int)((unsigned)g + (unsigned)k - 1u); }

// BC7 / BC6H interpolation weights (format spec tables 0,21,43,64 / 0,9,..,64 / 0,4,..,64) as exact formulas
ZTC_DEV int w2(int j) { return (64 * j + 1) / 3; }
ZTC_DEV int w3(int j) { return (64 * j + 3) / 7; }
ZTC_DEV int w4(int j) { return (64 * j + 7) / 15; }
ZTC_DEV int wbits(int bits, int j) { return bits == 2 ? w2(j) : bits == 3 ? w3(j) : w4(j); }
ZTC_DEV int lerp64(int a, int b, int w) { return ((64 - w) * a + w * b + 32) >> 6; }
ZTC_DEV int expand_bits(int v, int n) { v <<= 8 - n; return v | (v >> n); }  // n-bit -> 8-bit replication

ZTC_DEV uint32_t chan(uint32_t t, int c) { return (t >> (8 * c)) & 0xFFu; }
ZTC_DEV uint32_t pack_rgb(int r, int g, int b) { return (uint32_t)r | ((uint32_t)g << 8) | ((uint32_t)b << 16); }
ZTC_DEV uint32_t pack_rgba(int r, int g, int b, int a) { return pack_rgb(r, g, b) | ((uint32_t)a << 24); }
// sum of byte products of two packed texels (exact, unsigned)
ZTC_DEV uint32_t dot4(uint32_t a, uint32_t b) { return __dp4a(a, b, 0u); }

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
        if ((((uintptr_t)p) & 3u) == 0) return __ldg((const uint32_t *)p);
        return (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 8) | ((uint32_t)__ldg(p + 2) << 16) | ((uint32_t)__ldg(p + 3) << 24);
    }
    if (s.channels == 2) return (uint32_t)__ldg(p) | ((uint32_t)__ldg(p + 1) << 8) | 0xFF000000u;
    return (uint32_t)__ldg(p) | 0xFF000000u;
}

// 16 texels of block (bx, by), texel i at (i & 3, i >> 2), clamped to the image like the reference
ZTC_DEV void gather_block(const SrcU8 &s, int bx, int by, uint32_t t[16]) {
    int x0 = bx * 4, y0 = by * 4;
    if (s.vec16 && x0 + 3 < s.w && y0 + 3 < s.h) {
        #pragma unroll
        for (int r = 0; r < 4; r++) {
            uint4 v = __ldg((const uint4 *)(s.base + (size_t)(y0 + r) * s.stride + (size_t)x0 * 4));
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

ZTC_DEV void store_block8(uint8_t *out, uint2 v) { *(uint2 *)out = v; }
ZTC_DEV void store_block16(uint8_t *out, uint4 v) { *(uint4 *)out = v; }

}  // namespace ztc

// ztc_pca.cuh - principal-axis endpoint estimate over a texel subset (zap_tex.h:441-462), shared by the BC7 and
// ASTC kernels. The subset is a 16-bit mask (texel i selected when bit i is set); sums run over the selected
// texels in increasing texel order, exactly like the reference's sel[] lists.
#pragma once
#include "ztc_common.cuh"

namespace ztc {

// one power-iteration step on the axis ax; false (ax unchanged) when C ax vanishes
template <int NC>
ZTC_DEV bool pca_power_step(const float C[NC][NC], float ax[NC]) {
    float nv[NC], m = 0.0f;
    #pragma unroll
    for (int a = 0; a < NC; a++) {
        float s = 0.0f;
        #pragma unroll
        for (int b = 0; b < NC; b++) s = s + C[a][b] * ax[b];
        nv[a] = s;
        if (fabsf(s) > m) m = fabsf(s);
    }
    if (m < 1e-6f) return false;
    #pragma unroll
    for (int a = 0; a < NC; a++) ax[a] = nv[a] / m;
    return true;
}

// a byte or a small count as a float: a conversion, or (BITS) small_u2f's logic op and add; the same value either
// way, and which is faster depends on the kernel's other work
template <bool BITS>
ZTC_DEV float pca_u2f(uint32_t n) { return BITS ? small_u2f(n) : (float)n; }

// t: the texels in registers (uint32_t[16]) or a TexRef; UNROLL 1 rolls the texel loops and the power iteration
// (the same operations in the same order, in less code), UNROLL 16 unrolls them; U2F_BITS: pca_u2f's form
template <int NC, int UNROLL = 16, bool U2F_BITS = true, typename Tex>
ZTC_DEV void pca_endpoints(const Tex &t, uint32_t mask, float lo[4], float hi[4]) {
    const float cnt = pca_u2f<U2F_BITS>((uint32_t)popc(mask)), cnti = 1.0f / cnt;
    const bool whole = mask == 0xFFFFu;  // a compile-time constant for whole-block calls: x / 16 is a multiply there
    float mu[NC];
    if (whole) {
        // every term x / 16 and every partial sum of the mean is exact (a multiple of 1/16 below 256), so the
        // float sum is the channel's integer sum / 16; the four sums in two words of 16-bit fields
        uint32_t s02 = 0, s13 = 0;
        for_texels<UNROLL>([&](int i) {
            const uint32_t x = t[i];
            s02 += x & 0x00FF00FFu;
            s13 += (x >> 8) & 0x00FF00FFu;
        });
        const uint32_t S[4] = {s02 & 0xFFFFu, s13 & 0xFFFFu, s02 >> 16, s13 >> 16};
        #pragma unroll
        for (int c = 0; c < NC; c++) mu[c] = pca_u2f<U2F_BITS>(S[c]) / 16.0f;
    } else {
        #pragma unroll
        for (int c = 0; c < NC; c++) mu[c] = 0.0f;
        for_texels<UNROLL>([&](int i) {
            if ((mask >> i) & 1u) {
                #pragma unroll
                for (int c = 0; c < NC; c++) mu[c] = mu[c] + div_small(pca_u2f<U2F_BITS>(chan(t[i], c)), cnt, cnti);
            }
        });
    }
    // upper triangle only: cov[a][b] and cov[b][a] add bitwise-identical products in the same order
    float C[NC][NC];
    #pragma unroll
    for (int a = 0; a < NC; a++)
        #pragma unroll
        for (int b = 0; b < NC; b++) C[a][b] = 0.0f;
    for_texels<UNROLL>([&](int i) {
        if ((mask >> i) & 1u) {
            float d[NC];
            #pragma unroll
            for (int c = 0; c < NC; c++) d[c] = pca_u2f<U2F_BITS>(chan(t[i], c)) - mu[c];
            #pragma unroll
            for (int a = 0; a < NC; a++)
                #pragma unroll
                for (int b = a; b < NC; b++) C[a][b] = C[a][b] + d[a] * d[b];
        }
    });
    #pragma unroll
    for (int a = 0; a < NC; a++)
        #pragma unroll
        for (int b = 0; b < a; b++) C[a][b] = C[b][a];
    float ax[NC];
    #pragma unroll
    for (int c = 0; c < NC; c++) ax[c] = 1.0f;
    if (UNROLL == 1) {
        #pragma unroll 1
        for (int it = 0; it < 6; it++)
            if (!pca_power_step<NC>(C, ax)) break;
    } else {
        for (int it = 0; it < 6; it++)
            if (!pca_power_step<NC>(C, ax)) break;
    }
    float n2 = 0.0f, tl = 1e9f, th = -1e9f;
    #pragma unroll
    for (int a = 0; a < NC; a++) n2 = n2 + ax[a] * ax[a];
    for_texels<UNROLL>([&](int i) {
        if ((mask >> i) & 1u) {
            float s = 0.0f;
            #pragma unroll
            for (int c = 0; c < NC; c++) s = s + (pca_u2f<U2F_BITS>(chan(t[i], c)) - mu[c]) * ax[c];
            if (s < tl) tl = s;
            if (s > th) th = s;
        }
    });
    #pragma unroll
    for (int c = 0; c < 4; c++) {
        if (c < NC) { lo[c] = mu[c] + ax[c] * tl / n2; hi[c] = mu[c] + ax[c] * th / n2; }
        else { lo[c] = 255.0f; hi[c] = 255.0f; }
    }
}

}  // namespace ztc

// bc6h.cu - BC6H unsigned-float encoder, mode 11 (zap_tex.h:817-960), one thread per 4x4 block, bit-exact.
//
// Texels become unsigned half bits (zap__f2h); the search runs on the pre-finish values U = h * 64 / 31 in float
// (PCA start and bounding-box start, up to three least-squares refits each, in the reference's operation order).
// The reference sums squared half-bit differences in double; each is an integer below 2^32 and the block total
// below 2^38, so exact unsigned 32-bit terms and a 64-bit sum give the same values and the same comparisons.
#include "ztc_common.cuh"
#include "ztc_internal.h"

namespace ztc {

ZTC_DEV uint32_t f2h_unsigned(float f) {  // zap_tex.h:820-827
    if (!(f > 0.0f)) return 0;
    uint32_t x = f_as_u(f);
    if (x >= 0x477FE000u) return 0x7BFF;
    if (x < 0x38800000u) return (uint32_t)f2i_x86(f * 16777216.0f + 0.5f);
    return ((x - 0x38000000u) + 0x1000u) >> 13;
}
// an IEEE half widened to float, then f2h_unsigned: negatives and NaN -> 0, +inf -> 0x7BFF, the rest unchanged
ZTC_DEV uint32_t half_to_unsigned(uint32_t h) {
    if (h & 0x8000u) return 0;
    if (((h >> 10) & 31u) == 31u) return (h & 1023u) ? 0u : 0x7BFFu;
    return h;
}
// 10-bit endpoint -> 16-bit (zap_tex.h:837). Callers clamp e with clampi's min/max form (see ztc_common.cuh).
ZTC_DEV int bc6_unq(int e) { return e == 0 ? 0 : e == 1023 ? 0xFFFF : ((e << 16) + 0x8000) >> 10; }
ZTC_DEV int bc6_fin(int u) { return (u * 31) >> 6; }
ZTC_DEV int bc6_nearest(float u) {  // zap_tex.h:841-851
    int g = f2i_x86((u - 32.0f) / 64.0f + 0.5f), best = 0;
    float bd = 1e30f;
    #pragma unroll
    for (int k = 0; k < 3; k++) {
        int e = clampi(around(g, k), 0, 1023);
        float d = fabsf((float)bc6_unq(e) - u);
        if (d < bd) { bd = d; best = e; }
    }
    return best;
}

// A block's texels: unsigned half bits h and pre-finish values U = h * 64 / 31, texel i channel c at
// [(3 i + c) * stride] (a column of a per-CTA shared-memory array on the device, stride 1 on the host)
struct HalfRef {
    const uint16_t *t;
    const float *U;
    int stride;
    ZTC_DEV int h(int i, int c) const { return (int)t[(3 * i + c) * stride]; }
    ZTC_DEV float u(int i, int c) const { return U[(3 * i + c) * stride]; }
};

// best 4-bit indices and exact squared error for 10-bit endpoints e0, e1 (zap_tex.h:854-871)
ZTC_DEV uint64_t bc6_fit(const HalfRef &B, const int e0[3], const int e1[3], uint64_t &idx) {
    int pal[16][3];
    #pragma unroll
    for (int j = 0; j < 16; j++)
        #pragma unroll
        for (int c = 0; c < 3; c++) pal[j][c] = bc6_fin(lerp64(bc6_unq(e0[c]), bc6_unq(e1[c]), w4(j)));
    uint64_t err = 0, bits = 0;
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        const int tr = B.h(i, 0), tg = B.h(i, 1), tb = B.h(i, 2);
        uint32_t be = 0xFFFFFFFFu;
        int bj = 0;
        #pragma unroll
        for (int j = 0; j < 16; j++) {
            int dr = tr - pal[j][0], dg = tg - pal[j][1], db = tb - pal[j][2];
            uint32_t d = (uint32_t)(dr * dr) + (uint32_t)(dg * dg) + (uint32_t)(db * db);
            if (d < be) { be = d; bj = j; }
        }
        err += be;
        bits |= (uint64_t)bj << (4 * i);
    }
    idx = bits;
    return err;
}

// the search (zap_tex.h:873-931): PCA and bounding-box starts, each fitted and refitted by least squares up to
// three times (stopping at SSE 0, a singular system or the first refit that does not lower the SSE); the texel
// loops are rolled and the fit has one call site, which keeps the code small
ZTC_DEV uint4 bc6h_encode_block(const HalfRef &B) {
    float mu0 = 0.0f, mu1 = 0.0f, mu2 = 0.0f;
    #pragma unroll 1
    for (int i = 0; i < 16; i++) { mu0 = mu0 + B.u(i, 0) / 16.0f; mu1 = mu1 + B.u(i, 1) / 16.0f; mu2 = mu2 + B.u(i, 2) / 16.0f; }
    float C0 = 0, C1 = 0, C2 = 0, C3 = 0, C4 = 0, C5 = 0;
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        float r = B.u(i, 0) - mu0, g = B.u(i, 1) - mu1, b = B.u(i, 2) - mu2;
        C0 = C0 + r * r; C1 = C1 + r * g; C2 = C2 + r * b; C3 = C3 + g * g; C4 = C4 + g * b; C5 = C5 + b * b;
    }
    float v0 = 1.0f, v1 = 1.0f, v2 = 1.0f;
    for (int it = 0; it < 6; it++) {
        float x = C0 * v0 + C1 * v1 + C2 * v2, y = C1 * v0 + C3 * v1 + C4 * v2, z = C2 * v0 + C4 * v1 + C5 * v2;
        float m = fabsf(x);
        if (fabsf(y) > m) m = fabsf(y);
        if (fabsf(z) > m) m = fabsf(z);
        if (m < 1e-6f) break;
        v0 = x / m; v1 = y / m; v2 = z / m;
    }
    float n2 = v0 * v0 + v1 * v1 + v2 * v2, tl = 1e30f, th = -1e30f;
    float bl[3] = {1e30f, 1e30f, 1e30f}, bh[3] = {0.0f, 0.0f, 0.0f};
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        float d = (B.u(i, 0) - mu0) * v0 + (B.u(i, 1) - mu1) * v1 + (B.u(i, 2) - mu2) * v2;
        if (d < tl) tl = d;
        if (d > th) th = d;
        #pragma unroll
        for (int c = 0; c < 3; c++) { const float uc = B.u(i, c); if (uc < bl[c]) bl[c] = uc; if (uc > bh[c]) bh[c] = uc; }
    }
    const float mu[3] = {mu0, mu1, mu2}, ax[3] = {v0, v1, v2};
    uint64_t best = ~0ull, bidx = 0, idx = 0, err = 0;
    int be0[3] = {0, 0, 0}, be1[3] = {0, 0, 0}, e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0};
    int start = 0, pass = 0;  // pass 0: the start's first fit; 1..3: least-squares refits
    #pragma unroll 1
    for (;;) {
        int n0[3], n1[3];
        bool fit = true;
        if (pass == 0) {
            #pragma unroll
            for (int c = 0; c < 3; c++) {
                float lo = start ? bl[c] : mu[c] + ax[c] * tl / n2, hi = start ? bh[c] : mu[c] + ax[c] * th / n2;
                n0[c] = bc6_nearest(lo); n1[c] = bc6_nearest(hi);
            }
        } else {
            float aa = 0, ab = 0, bb = 0, sa[3] = {0, 0, 0}, sb[3] = {0, 0, 0};
            #pragma unroll 1
            for (int i = 0; i < 16; i++) {
                float w = (float)w4((int)((idx >> (4 * i)) & 15u)) / 64.0f, u = 1.0f - w;
                aa = aa + u * u; ab = ab + u * w; bb = bb + w * w;
                #pragma unroll
                for (int c = 0; c < 3; c++) { const float uc = B.u(i, c); sa[c] = sa[c] + u * uc; sb[c] = sb[c] + w * uc; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) fit = false;
            #pragma unroll
            for (int c = 0; c < 3; c++) { n0[c] = bc6_nearest((sa[c] * bb - sb[c] * ab) / det); n1[c] = bc6_nearest((sb[c] * aa - sa[c] * ab) / det); }
        }
        bool done = !fit;
        if (fit) {
            uint64_t ni;
            const uint64_t e2 = bc6_fit(B, n0, n1, ni);
            if (pass == 0 || e2 < err) {
                err = e2; idx = ni;
                #pragma unroll
                for (int c = 0; c < 3; c++) { e0[c] = n0[c]; e1[c] = n1[c]; }
                done = ++pass == 4 || err == 0;
            } else {
                done = true;
            }
        }
        if (done) {  // the start is finished: keep it if it is the best so far
            if (err < best) {
                best = err; bidx = idx;
                #pragma unroll
                for (int c = 0; c < 3; c++) { be0[c] = e0[c]; be1[c] = e1[c]; }
            }
            if (++start == 2) break;
            pass = 0;
        }
    }
    if (bidx & 8u) {  // anchor MSB must be 0
        #pragma unroll
        for (int c = 0; c < 3; c++) { int s = be0[c]; be0[c] = be1[c]; be1[c] = s; }
        bidx ^= ~0ull;
    }
    Bits128 o;
    o.put(3u, 5);  // mode 11
    #pragma unroll
    for (int c = 0; c < 3; c++) o.put((uint32_t)be0[c], 10);
    #pragma unroll
    for (int c = 0; c < 3; c++) o.put((uint32_t)be1[c], 10);
    o.put((uint32_t)(bidx & 7u), 3);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((uint32_t)((bidx >> (4 * i)) & 15u), 4);
    return make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
}

constexpr int kBc6hCta = 128;
__global__ void __launch_bounds__(kBc6hCta, ZTC_MINB_BC6H) bc6h_kernel(SrcHdr src, int bw, int by0, int nblocks, uint8_t *__restrict__ out) {
    // column threadIdx.x: this thread's block (read only by this thread)
    __shared__ uint16_t s_t[48][kBc6hCta];
    __shared__ float s_U[48][kBc6hCta];
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    int bx = b % bw, by = by0 + b / bw;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        int x = min(bx * 4 + (i & 3), src.w - 1), y = min(by * 4 + (i >> 2), src.h - 1);
        size_t off = (size_t)y * src.stride + (size_t)x * (size_t)src.channels;
        #pragma unroll
        for (int c = 0; c < 3; c++) {
            uint32_t h = src.f32 ? f2h_unsigned(__ldg((const float *)src.base + off + c))
                                 : half_to_unsigned(__ldg((const unsigned short *)src.base + off + c));
            s_t[3 * i + c][threadIdx.x] = (uint16_t)h;
            s_U[3 * i + c][threadIdx.x] = (float)h * 64.0f / 31.0f;
        }
    }
    store_block16(out + (size_t)b * 16, bc6h_encode_block(HalfRef{&s_t[0][threadIdx.x], &s_U[0][threadIdx.x], kBc6hCta}));
}

}  // namespace ztc

cudaError_t ztc_launch_bc6h(const ztc::SrcHdr &src, int by0, int nby, uint8_t *out, cudaStream_t stream) {
    int bw = (src.w + 3) / 4, nblocks = bw * nby;
    if (nblocks <= 0) return cudaSuccess;
    ztc::TraceScope tr("bc6h_encode", stream);
    ztc::trace_units(nblocks);
    ztc::bc6h_kernel<<<(nblocks + 127) / 128, 128, 0, stream>>>(src, bw, by0, nblocks, out);
    return cudaGetLastError();
}

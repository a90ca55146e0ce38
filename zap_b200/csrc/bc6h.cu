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

// Passes [first, last) of one start of the search (zap_tex.h:900-925): pass 0 fits the start's endpoints (lo, hi);
// pass k > 0 is the k-th least-squares refit on the indices idx holds, which does not run at SSE 0, stops at a
// singular system, and is dropped (ending the start) when it does not lower the SSE. e0, e1, idx, err take each
// accepted pass. Returns true when every pass ran and the SSE is still above 0, so pass `last` would run. The
// texel loops are rolled and the fit has one call site, which keeps the code small.
ZTC_DEV bool bc6_passes(const HalfRef &B, const float lo[3], const float hi[3], int first, int last, int e0[3], int e1[3],
                        uint64_t &idx, uint64_t &err) {
    #pragma unroll 1
    for (int pass = first; pass < last; pass++) {
        int n0[3], n1[3];
        if (pass == 0) {
            #pragma unroll
            for (int c = 0; c < 3; c++) { n0[c] = bc6_nearest(lo[c]); n1[c] = bc6_nearest(hi[c]); }
        } else {
            if (err == 0) return false;
            float aa = 0, ab = 0, bb = 0, sa[3] = {0, 0, 0}, sb[3] = {0, 0, 0};
            #pragma unroll 1
            for (int i = 0; i < 16; i++) {
                float w = (float)w4((int)((idx >> (4 * i)) & 15u)) / 64.0f, u = 1.0f - w;
                aa = aa + u * u; ab = ab + u * w; bb = bb + w * w;
                #pragma unroll
                for (int c = 0; c < 3; c++) { const float uc = B.u(i, c); sa[c] = sa[c] + u * uc; sb[c] = sb[c] + w * uc; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) return false;
            #pragma unroll
            for (int c = 0; c < 3; c++) { n0[c] = bc6_nearest((sa[c] * bb - sb[c] * ab) / det); n1[c] = bc6_nearest((sb[c] * aa - sa[c] * ab) / det); }
        }
        uint64_t ni;
        const uint64_t e2 = bc6_fit(B, n0, n1, ni);
        if (pass > 0 && e2 >= err) return false;
        err = e2; idx = ni;
        #pragma unroll
        for (int c = 0; c < 3; c++) { e0[c] = n0[c]; e1[c] = n1[c]; }
    }
    return err > 0;
}

// the two starts' endpoints (zap_tex.h:873-899): slo/shi[0] from the principal axis, [1] the bounding box
ZTC_DEV void bc6_starts(const HalfRef &B, float slo[2][3], float shi[2][3]) {
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
    #pragma unroll
    for (int c = 0; c < 3; c++) {
        slo[0][c] = mu[c] + ax[c] * tl / n2; shi[0][c] = mu[c] + ax[c] * th / n2;
        slo[1][c] = bl[c]; shi[1][c] = bh[c];
    }
}

// mode 11 block (zap_tex.h:926-931): anchor index MSB 0 (else swap the endpoints and invert the indices)
ZTC_DEV uint4 bc6_pack(int be0[3], int be1[3], uint64_t bidx) {
    if (bidx & 8u) {
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

// the search (zap_tex.h:873-931), one thread: both starts, all passes, the first start of least SSE
ZTC_DEV uint4 bc6h_encode_block(const HalfRef &B) {
    float slo[2][3], shi[2][3];
    bc6_starts(B, slo, shi);
    uint64_t best = ~0ull, bidx = 0;
    int be0[3] = {0, 0, 0}, be1[3] = {0, 0, 0};
    #pragma unroll 1
    for (int start = 0; start < 2; start++) {
        int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0};
        uint64_t idx = 0, err = 0;
        bc6_passes(B, slo[start], shi[start], 0, 4, e0, e1, idx, err);
        if (err < best) {
            best = err; bidx = idx;
            #pragma unroll
            for (int c = 0; c < 3; c++) { be0[c] = e0[c]; be1[c] = e1[c]; }
        }
    }
    return bc6_pack(be0, be1, bidx);
}

ZTC_DEV uint64_t pack_ends10(const int e0[3], const int e1[3]) {
    uint64_t v = 0;
    #pragma unroll
    for (int c = 0; c < 3; c++) v |= ((uint64_t)e0[c] << (10 * c)) | ((uint64_t)e1[c] << (30 + 10 * c));
    return v;
}
ZTC_DEV void unpack_ends10(uint64_t v, int e0[3], int e1[3]) {
    #pragma unroll
    for (int c = 0; c < 3; c++) { e0[c] = (int)((v >> (10 * c)) & 1023u); e1[c] = (int)((v >> (30 + 10 * c)) & 1023u); }
}

// The search for the CTA's blocks, one per thread, with each start's last least-squares refit compacted: every
// thread runs its block's two starts up to the third pass; the (block, start) pairs whose fourth pass would run
// (a tenth of them on the HDR test content, yet nearly every warp holds one) are listed in shared memory, and the
// first threads of the CTA run those passes on the owners' texels. Same bytes as bc6h_encode_block. Every thread
// of the CTA calls it (it synchronises); a `valid` thread's block is in column threadIdx.x of s_t / s_U.
template <int CTA>
__device__ __forceinline__ uint4 bc6h_encode_cta(bool valid, uint16_t (*s_t)[CTA], float (*s_U)[CTA]) {
    __shared__ uint64_t s_ends[2][CTA], s_idx[2][CTA], s_err[2][CTA];
    __shared__ int s_wcnt[2][CTA / 32];
    __shared__ uint16_t s_list[2 * CTA];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float slo[2][3], shi[2][3];
    if (valid) bc6_starts(HalfRef{&s_t[0][tid], &s_U[0][tid], CTA}, slo, shi);
    bool more0 = false, more1 = false;
    int total = 0;
    #pragma unroll 1
    for (int job = 0; job < 4; job++) {
        if (job == 2) {  // list the (block, start) pairs whose fourth pass would run, in thread order
            const unsigned b0 = __ballot_sync(0xFFFFFFFFu, more0), b1 = __ballot_sync(0xFFFFFFFFu, more1);
            if (lane == 0) { s_wcnt[0][warp] = __popc(b0); s_wcnt[1][warp] = __popc(b1); }
            __syncthreads();
            int base0 = 0, base1 = 0, t0 = 0, t1 = 0;
            #pragma unroll
            for (int w = 0; w < CTA / 32; w++) {
                const int c0 = s_wcnt[0][w], c1 = s_wcnt[1][w];
                base0 += w < warp ? c0 : 0; base1 += w < warp ? c1 : 0; t0 += c0; t1 += c1;
            }
            const unsigned below = (1u << lane) - 1u;
            if (more0) {
                const int p0 = base0 + __popc(b0 & below);
                if (ZTC_IN_BOUNDS(p0, 2 * CTA, 4)) s_list[p0] = (uint16_t)(tid << 1);
            }
            if (more1) {
                const int p1 = t0 + base1 + __popc(b1 & below);
                if (ZTC_IN_BOUNDS(p1, 2 * CTA, 4)) s_list[p1] = (uint16_t)((tid << 1) | 1);
            }
            total = t0 + t1;
            __syncthreads();
        }
        int owner = tid, st = job, first = 0, last = 3;
        bool active = valid;
        if (job >= 2) {
            const int k = tid + (job - 2) * CTA;
            active = k < total;
            if (active) { owner = s_list[k] >> 1; st = s_list[k] & 1; }
#ifdef ZTC_CHECKS
            if (active && !ZTC_IN_BOUNDS(owner, CTA, 8)) active = false;
#endif
            first = 3; last = 4;
        }
        if (active) {
            int e0[3] = {0, 0, 0}, e1[3] = {0, 0, 0};
            uint64_t idx = 0, err = 0;
            if (job >= 2) { unpack_ends10(s_ends[st][owner], e0, e1); idx = s_idx[st][owner]; err = s_err[st][owner]; }
            const uint64_t e_in = err;
            const bool more = bc6_passes(HalfRef{&s_t[0][owner], &s_U[0][owner], CTA}, slo[st], shi[st], first, last, e0, e1, idx, err);
            if (job < 2 || err < e_in) { s_ends[st][owner] = pack_ends10(e0, e1); s_idx[st][owner] = idx; s_err[st][owner] = err; }
            if (job == 0) more0 = more;
            if (job == 1) more1 = more;
        }
    }
    __syncthreads();
    if (!valid) return make_uint4(0, 0, 0, 0);
    const int st = s_err[1][tid] < s_err[0][tid] ? 1 : 0;  // the first start of least SSE
    int be0[3], be1[3];
    unpack_ends10(s_ends[st][tid], be0, be1);
    return bc6_pack(be0, be1, s_idx[st][tid]);
}

constexpr int kBc6hCta = 128;
__global__ void __launch_bounds__(kBc6hCta, ZTC_MINB_BC6H) bc6h_kernel(SrcHdr src, int bw, int by0, int nblocks, uint8_t *__restrict__ out) {
    __shared__ uint16_t s_t[48][kBc6hCta];  // column threadIdx.x: this thread's block
    __shared__ float s_U[48][kBc6hCta];
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = b < nblocks;
    if (valid) {
        const int bx = b % bw, by = by0 + b / bw;
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
    }
    const uint4 blk = bc6h_encode_cta<kBc6hCta>(valid, s_t, s_U);
    if (valid) store_block16(out + (size_t)b * 16, blk);
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

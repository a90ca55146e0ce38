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
// zap_tex.h:841-851. The reference truncates v = (u - 32) / 64 + 0.5 to g as x86 does (INT_MIN for NaN and
// out-of-range v) and keeps the first closest of g - 1, g, g + 1 clamped to [0, 1023]. Here v <= -2^31 keeps
// INT_MIN (its wrapped set {1023, 0, 0} picks 1023 once 65535 + |u| rounds to |u|), and other v are clamped to
// [0, 2048] before a conversion-free truncation, which changes no result: -2^31 < v < 0 means u < 0, where 0 comes
// first and is never farther than 1; v > 2048 gives candidates that all clamp to 1023, as the reference's do (for
// v >= 2^31 its set {1023, 0, 0} also picks 1023); a NaN u, and any u whose every candidate is 1e30 or more away,
// leaves 0 whatever the candidates. The host test checks every float.
ZTC_DEV int bc6_nearest(float u) {
    const float v = (u - 32.0f) / 64.0f + 0.5f;
    int g = v <= -2147483648.0f ? (int)0x80000000 : trunc_small(fminf(fmaxf(v, 0.0f), 2048.0f)), best = 0;
    float bd = 1e30f;
    #pragma unroll
    for (int k = 0; k < 3; k++) {
        int e = clampi(around(g, k), 0, 1023);
        float d = fabsf(small_u2f((uint32_t)bc6_unq(e)) - u);
        if (d < bd) { bd = d; best = e; }
    }
    return best;
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

// The block word: bits 15c..15c+14 hold the centre o_c = (min_c + max_c) >> 1 of channel c's half bits, bits 45..63
// Hq = ceil(H / 2^11) for H = sum_c h_c^2 with the half ranges h_c = max(max_c - o_c, o_c - min_c), so every
// centred texel has |t - o|^2 <= H <= Hq * 2^11.
ZTC_DEV uint64_t bc6_block_word(const int mn[3], const int mx[3]) {
    uint64_t w = 0;
    uint32_t H = 0;
    #pragma unroll
    for (int c = 0; c < 3; c++) {
        const int o = (mn[c] + mx[c]) >> 1, hc = max(mx[c] - o, o - mn[c]);
        H += (uint32_t)(hc * hc);
        w |= (uint64_t)o << (15 * c);
    }
    return w | ((uint64_t)((H + 2047u) >> 11) << 45);
}

// A block's texels: half bits centred on the block word's per-channel centre, t(i, c) = h - o_c, and pre-finish
// values U = h * 64 / 31, texel i channel c at [(3 i + c) * stride] (a column of a per-CTA shared-memory array on
// the device, stride 1 on the host), the block word cw and tsum = sum_i |t_i|^2 modulo 2^32 (exact whenever the
// fit's keys fit in 32 bits)
struct HalfRef {
    const int16_t *t;
    const float *U;
    int stride;
    uint64_t cw;
    uint32_t tsum;
    ZTC_DEV int h(int i, int c) const { return (int)t[(3 * i + c) * stride]; }
    ZTC_DEV float u(int i, int c) const { return U[(3 * i + c) * stride]; }
};

// best 4-bit indices and exact squared error for 10-bit endpoints `ends` (pack_ends10) (zap_tex.h:854-871).
// Distances are taken between centred values, (t - o) - (p - o) = t - p, so they are the reference's. With
// p'_c = p_c - o_c for the palette entries and H' = Hq * 2^11, the key of texel t' and entry j,
// 16 (|t' - p'_j|^2 - |t'|^2 + H') + j, is r_j + sum_c q_jc t'_c for q_jc = -32 p'_jc and
// r_j = 16 |p'_j|^2 + j + 16 H': three multiply-adds modulo 2^32. When every key is provably below 2^32 (the
// distance is at most 2 H' + 2 M, M = sum_c max_j p'_jc^2 from the two end entries, as each channel's palette is
// monotone in j), the texel's unsigned minimum key gives the least distance and, on ties, the lower index, as the
// reference's strict `<` scan; the block's squared error is then sum (key >> 4) + sum |t'|^2 - 16 H'. Otherwise
// (blocks whose range spans much of the half range) the plain scan of the squared differences runs.
ZTC_DEV uint64_t bc6_fit(const HalfRef &B, uint64_t ends, uint64_t &idx) {
    int e0[3], e1[3], a[3], b[3], o[3];
    unpack_ends10(ends, e0, e1);
    #pragma unroll
    for (int c = 0; c < 3; c++) { a[c] = bc6_unq(e0[c]); b[c] = bc6_unq(e1[c]); o[c] = (int)(B.cw >> (15 * c)) & 0x7FFF; }
    const uint32_t Hp = (uint32_t)(B.cw >> 45) << 11, c16 = Hp << 4;  // c16: modulo 2^32, used when the keys fit
    int q[16][3];
    uint32_t r[16];
    uint64_t M = 0;
    #pragma unroll
    for (int j = 0; j < 16; j++) {
        uint32_t P = 0;
        #pragma unroll
        for (int c = 0; c < 3; c++) {
            const int p = bc6_fin(lerp64(a[c], b[c], w4(j))) - o[c];  // |p| <= 31743
            q[j][c] = -32 * p;
            P += (uint32_t)(p * p);
        }
        r[j] = 16u * P + (uint32_t)j + c16;
    }
    #pragma unroll
    for (int c = 0; c < 3; c++) {
        const int p0 = q[0][c] / 32, p15 = q[15][c] / 32;  // exact: multiples of 32
        M += (uint64_t)(uint32_t)max(p0 * p0, p15 * p15);
    }
    uint64_t bits = 0;
    if (48ull * Hp + 32ull * M + 15ull < (1ull << 32)) {
        uint32_t acc = 0;  // < 16 * 2^28
        #pragma unroll 1
        for (int i = 0; i < 16; i++) {
            const uint32_t tr = (uint32_t)B.h(i, 0), tg = (uint32_t)B.h(i, 1), tb = (uint32_t)B.h(i, 2);
            uint32_t best = r[0] + (uint32_t)q[0][0] * tr + (uint32_t)q[0][1] * tg + (uint32_t)q[0][2] * tb;
            #pragma unroll
            for (int j = 1; j < 16; j++) best = min(best, r[j] + (uint32_t)q[j][0] * tr + (uint32_t)q[j][1] * tg + (uint32_t)q[j][2] * tb);
            acc += best >> 4;
            bits |= (uint64_t)(best & 15u) << (4 * i);
        }
        idx = bits;
        return (uint64_t)acc + B.tsum - ((uint64_t)Hp << 4);  // B.tsum <= 16 H' < 2^32 / 3 here
    }
    uint64_t err = 0;
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        const int tr = B.h(i, 0), tg = B.h(i, 1), tb = B.h(i, 2);
        uint32_t be = 0xFFFFFFFFu;
        int bj = 0;
        #pragma unroll
        for (int j = 0; j < 16; j++) {
            const int dr = tr + q[j][0] / 32, dg = tg + q[j][1] / 32, db = tb + q[j][2] / 32;  // t - p, |.| <= 31743
            const uint32_t d = (uint32_t)(dr * dr) + (uint32_t)(dg * dg) + (uint32_t)(db * db);
            if (d < be) { be = d; bj = j; }
        }
        err += be;
        bits |= (uint64_t)bj << (4 * i);
    }
    idx = bits;
    return err;
}

// Passes [first, last) of one start of the search (zap_tex.h:900-925): pass 0 fits the start's endpoints `start`;
// pass k > 0 is the k-th least-squares refit on the indices idx holds, which does not run at SSE 0, stops at a
// singular system, and is dropped (ending the start) when it does not lower the SSE. *ends, *idx, *err take each
// accepted pass (shared-memory slots on the device, which keeps them out of registers during the fits). Returns
// true when every pass ran and the SSE is still above 0, so pass `last` would run. The texel loops are rolled and
// the fit has one call site, which keeps the code small.
ZTC_DEV bool bc6_passes(const HalfRef &B, uint64_t start, int first, int last, uint64_t *ends, uint64_t *idx, uint64_t *err) {
    uint64_t n = start;
    #pragma unroll 1
    for (int pass = first; pass < last; pass++) {
        if (pass > 0) {
            if (*err == 0) return false;
            const uint64_t ix = *idx;
            float aa = 0, ab = 0, bb = 0, sa[3] = {0, 0, 0}, sb[3] = {0, 0, 0};
            #pragma unroll 1
            for (int i = 0; i < 16; i++) {
                float w = small_u2f((uint32_t)w4((int)((ix >> (4 * i)) & 15u))) / 64.0f, u = 1.0f - w;
                aa = aa + u * u; ab = ab + u * w; bb = bb + w * w;
                #pragma unroll
                for (int c = 0; c < 3; c++) { const float uc = B.u(i, c); sa[c] = sa[c] + u * uc; sb[c] = sb[c] + w * uc; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) return false;
            int n0[3], n1[3];
            #pragma unroll
            for (int c = 0; c < 3; c++) { n0[c] = bc6_nearest((sa[c] * bb - sb[c] * ab) / det); n1[c] = bc6_nearest((sb[c] * aa - sa[c] * ab) / det); }
            n = pack_ends10(n0, n1);
        }
        uint64_t ni;
        const uint64_t e2 = bc6_fit(B, n, ni);
        if (pass > 0 && e2 >= *err) return false;
        *err = e2; *idx = ni; *ends = n;
    }
    return *err > 0;
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

// the two starts' quantised endpoints (zap_tex.h:873-899 and pass 0's nearest 10-bit values, zap_tex.h:900-903):
// [0] from the principal axis, [1] from the bounding box
ZTC_DEV void bc6_start_ends(const HalfRef &B, uint64_t s[2]) {
    float slo[2][3], shi[2][3];
    bc6_starts(B, slo, shi);
    #pragma unroll
    for (int k = 0; k < 2; k++) {
        int n0[3], n1[3];
        #pragma unroll
        for (int c = 0; c < 3; c++) { n0[c] = bc6_nearest(slo[k][c]); n1[c] = bc6_nearest(shi[k][c]); }
        s[k] = pack_ends10(n0, n1);
    }
}

// the search (zap_tex.h:873-931), one thread: both starts, all passes, the first start of least SSE
ZTC_DEV uint4 bc6h_encode_block(const HalfRef &B) {
    uint64_t st[2];
    bc6_start_ends(B, st);
    uint64_t best = ~0ull, bidx = 0, bends = 0;
    #pragma unroll 1
    for (int start = 0; start < 2; start++) {
        uint64_t ends = 0, idx = 0, err = 0;
        bc6_passes(B, st[start], 0, 4, &ends, &idx, &err);
        if (err < best) { best = err; bidx = idx; bends = ends; }
    }
    int be0[3], be1[3];
    unpack_ends10(bends, be0, be1);
    return bc6_pack(be0, be1, bidx);
}

// A block's texels, half bits at tc[(3 i + c) * stride] (texel i, channel c; at most 0x7BFF), centred in place;
// returns the block word and sets tsum (HalfRef)
ZTC_DEV uint64_t bc6_center(int16_t *tc, int stride, uint32_t &tsum) {
    int mn[3] = {0x7FFF, 0x7FFF, 0x7FFF}, mx[3] = {0, 0, 0};
    #pragma unroll
    for (int k = 0; k < 48; k++) { const int v = tc[k * stride]; mn[k % 3] = min(mn[k % 3], v); mx[k % 3] = max(mx[k % 3], v); }
    const uint64_t cw = bc6_block_word(mn, mx);
    uint32_t ts = 0;
    #pragma unroll
    for (int k = 0; k < 48; k++) {
        const int v = (int)tc[k * stride] - (int)((cw >> (15 * (k % 3))) & 0x7FFF);
        tc[k * stride] = (int16_t)v;
        ts += (uint32_t)(v * v);
    }
    tsum = ts;
    return cw;
}

// The search for the CTA's blocks, one per thread, with each start's later passes compacted. Stage 0: every thread
// runs its block's two starts through passes 0 and 1 (all of them do). Stage 1: the (block, start) pairs whose
// pass 2 would run (about half of them on the HDR test content, yet nearly every warp holds several) are listed in
// shared memory and run by the first threads; stage 2 lists and runs those whose pass 3 would run (a tenth). A
// pair's state between stages is its shared-memory slots. Same bytes as bc6h_encode_block. Every thread of the
// CTA calls it (it synchronises); a `valid` thread's block is in column threadIdx.x of s_t / s_U, its block word
// and tsum in s_cw[threadIdx.x] and s_ts[threadIdx.x].
template <int CTA>
__device__ __forceinline__ uint4 bc6h_encode_cta(bool valid, int16_t (*s_t)[CTA], float (*s_U)[CTA], const uint64_t *s_cw, const uint32_t *s_ts) {
    __shared__ uint64_t s_ends[2][CTA], s_idx[2][CTA], s_err[2][CTA];
    __shared__ int s_wcnt[2][CTA / 32];
    __shared__ uint16_t s_list[2 * CTA];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (valid) {  // the starts' endpoints wait in the slots their passes fill
        uint64_t se[2];
        bc6_start_ends(HalfRef{&s_t[0][tid], &s_U[0][tid], CTA, s_cw[tid], s_ts[tid]}, se);
        s_ends[0][tid] = se[0];
        s_ends[1][tid] = se[1];
    }
    // the thread's two items of the stage (pairs as block << 1 | start) and whether each one's next pass would run
    int item0 = tid << 1, item1 = (tid << 1) | 1, total = 0;
    bool more0 = false, more1 = false;
    #pragma unroll 1
    for (int stage = 0; stage < 3; stage++) {
        if (stage > 0) {  // list the pairs whose next pass would run: round 0's in thread order, then round 1's
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
                if (ZTC_IN_BOUNDS(p0, 2 * CTA, 4)) s_list[p0] = (uint16_t)item0;
            }
            if (more1) {
                const int p1 = t0 + base1 + __popc(b1 & below);
                if (ZTC_IN_BOUNDS(p1, 2 * CTA, 4)) s_list[p1] = (uint16_t)item1;
            }
            total = t0 + t1;
            __syncthreads();
        }
        const int first = stage == 0 ? 0 : stage + 1, last = stage + 2;
        #pragma unroll 1
        for (int r = 0; r < 2; r++) {
            int it = r ? item1 : item0;
            bool active = valid;
            if (stage > 0) {
                const int k = tid + r * CTA;
                active = k < total;
                it = active ? (int)s_list[k] : 0;
            }
            const int owner = it >> 1, st = it & 1;
#ifdef ZTC_CHECKS
            if (active && !ZTC_IN_BOUNDS(owner, CTA, 8)) active = false;
#endif
            bool more = false;
            if (active)  // stage 0 starts from the start's endpoints, later stages from the pair's state
                more = bc6_passes(HalfRef{&s_t[0][owner], &s_U[0][owner], CTA, s_cw[owner], s_ts[owner]}, s_ends[st][owner],
                                  first, last, &s_ends[st][owner], &s_idx[st][owner], &s_err[st][owner]);
            if (r) { item1 = it; more1 = more; } else { item0 = it; more0 = more; }
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
    __shared__ int16_t s_t[48][kBc6hCta];  // column threadIdx.x: this thread's block, centred
    __shared__ float s_U[48][kBc6hCta];
    __shared__ uint64_t s_cw[kBc6hCta];  // the blocks' words
    __shared__ uint32_t s_ts[kBc6hCta];
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
                const uint32_t h = src.f32 ? f2h_unsigned(__ldg((const float *)src.base + off + c))
                                           : half_to_unsigned(__ldg((const unsigned short *)src.base + off + c));
                s_t[3 * i + c][threadIdx.x] = (int16_t)h;
                s_U[3 * i + c][threadIdx.x] = div_small(small_u2f(h) * 64.0f, 31.0f, 0x1.084210p-5f);  // h * 64 / 31; RN(1/31)
            }
        }
        uint32_t ts;
        s_cw[threadIdx.x] = bc6_center(&s_t[0][threadIdx.x], kBc6hCta, ts);
        s_ts[threadIdx.x] = ts;
    }
    const uint4 blk = bc6h_encode_cta<kBc6hCta>(valid, s_t, s_U, s_cw, s_ts);
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

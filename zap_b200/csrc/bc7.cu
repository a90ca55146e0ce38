// bc7.cu - BC7 encoder for sm_100a (modes 6, 5 and 1, as the reference encoder uses them; zap_tex.h:308-784).
//
// Two kernels over a device work list:
//   A  one thread per block: mode 6 (PCA start, p-bit search, two least-squares refits). Blocks whose SSE is
//      <= 64 are final (the reference's early exit, zap_tex.h:758); the others are appended to a work list.
//   B  over the listed blocks, in two passes per CTA:
//        mode 5  8 blocks per round, lane = block * 4 + rotation, the colour parts on one warp and the alpha parts
//                on the other, combined per rotation;
//        mode 1  the opaque ones, an 8-lane group per block: the 64 partitions are scored 8 per lane, the top 4 by
//                (score, partition) are merged across the group, then lane = (candidate, subset) fits the 8
//                subsets; with at most one listed block per CTA, the CTA's 64 threads score one partition each.
//      Decoded SSE checks of the reference (zap__bc7_err, zap_tex.h:761,780) equal the fit SSE here: the expand and
//      interpolation are the decoder's, anchor swaps preserve decoded values because every weight table satisfies
//      w(n-1-j) = 64 - w(j), mode 1 shares its p-bit between a subset's endpoints, and mode 1 decodes alpha 255
//      on the opaque blocks it is tried on. So kernel B compares fit errors directly.
// Every float expression keeps the reference's order; integer argmins keep the first candidate on ties.
#include <mutex>

#include "../../include/zap_tex_cuda.h"
#include "ztc_common.cuh"
#include "ztc_internal.h"
#include "ztc_pca.cuh"

namespace ztc {

// two-subset partitions (BC7 format spec): bit i set = texel i in subset 1; anchor texel of subset 1
__constant__ uint16_t kP2[64] = {
    0xCCCC, 0x8888, 0xEEEE, 0xECC8, 0xC880, 0xFEEC, 0xFEC8, 0xEC80, 0xC800, 0xFFEC, 0xFE80, 0xE800, 0xFFE8, 0xFF00, 0xFFF0, 0xF000,
    0xF710, 0x008E, 0x7100, 0x08CE, 0x008C, 0x7310, 0x3100, 0x8CCE, 0x088C, 0x3110, 0x6666, 0x366C, 0x17E8, 0x0FF0, 0x718E, 0x399C,
    0xAAAA, 0xF0F0, 0x5A5A, 0x33CC, 0x3C3C, 0x55AA, 0x9696, 0xA55A, 0x73CE, 0x13C8, 0x324C, 0x3BDC, 0x6996, 0xC33C, 0x9966, 0x0660,
    0x0272, 0x04E4, 0x4E40, 0x2720, 0xC936, 0x936C, 0x39C6, 0x639C, 0x9336, 0x9CC6, 0x817E, 0xE718, 0xCCF0, 0x0FCC, 0x7744, 0xEE22};
__constant__ uint8_t kA2[64] = {
    15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 15, 2, 8, 2, 2, 8, 8, 15, 2, 8, 2, 2, 8, 8, 2, 2,
    15, 15, 6, 8, 2, 8, 15, 15, 2, 8, 2, 2, 2, 15, 15, 6, 6, 2, 6, 8, 15, 15, 2, 2, 15, 15, 15, 15, 15, 2, 2, 15};

// ---------------------------------------------------------------- shared pieces (quant_pbit: ztc_common.cuh)
// Argmin over a (1 << IB)-entry palette for every selected texel: key = (|c|^2 - 2 p.c) * NP + j is ordered
// like the reference's first-best scan. idx: nibble i = index of texel i. Returns the SSE.
template <int NC, int IB>
ZTC_DEV int palette_fit(TexRef ts, uint32_t mask, const int x0[4], const int x1[4], uint64_t &idx) {
    constexpr int NP = 1 << IB;
    const uint32_t cm = NC == 4 ? 0xFFFFFFFFu : 0x00FFFFFFu;
    uint32_t pal[NP];
    int A[NP];
    const int y0[4] = {x0[0], x0[1], x0[2], NC == 4 ? x0[3] : 0}, y1[4] = {x1[0], x1[1], x1[2], NC == 4 ? x1[3] : 0};
    const Lerp4 row(y0, y1);
    #pragma unroll
    for (int j = 0; j < NP; j++) {
        const uint32_t e = row.at(wbits(IB, j)) & cm;
        pal[j] = e;
        A[j] = (int)dot4(e, e) * NP + j;
    }
    int err = 0;
    uint64_t bits = 0;
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        if (!((mask >> i) & 1u)) continue;
        const uint32_t p = ts[i] & cm;
        int m = A[0] - 2 * NP * (int)dot4(p, pal[0]);
        #pragma unroll
        for (int j = 1; j < NP; j++) m = min(m, A[j] - 2 * NP * (int)dot4(p, pal[j]));
        err += (m >> IB) + (int)dot4(p, p);
        bits |= (uint64_t)(m & (NP - 1)) << (4 * i);
    }
    idx = bits;
    return err;
}

// float endpoints -> best p-bits and quantised endpoints q (x0, x1: expanded to 8 bits) (zap_tex.h:466-486)
template <int NC>
ZTC_DEV void subset_quant(int n, bool shared_p, const float lo[4], const float hi[4], int q[2][4], int pb[2], int x0[4], int x1[4]) {
    int ql[2][4], qh[2][4], xl[2][4], xh[2][4], el[2], eh[2];
    #pragma unroll
    for (int p = 0; p < 2; p++) { el[p] = quant_pbit<NC>(lo, n, p, ql[p], xl[p]); eh[p] = quant_pbit<NC>(hi, n, p, qh[p], xh[p]); }
    int best = 1 << 30, b0 = 0, b1 = 0;
    #pragma unroll
    for (int combo = 0; combo < 4; combo++) {
        int p0 = combo >> 1, p1 = combo & 1;
        if (shared_p && p0 != p1) continue;
        int e = el[p0] + eh[p1];
        if (e < best) { best = e; b0 = p0; b1 = p1; }
    }
    #pragma unroll
    for (int c = 0; c < 4; c++) {
        q[0][c] = b0 ? ql[1][c] : ql[0][c]; q[1][c] = b1 ? qh[1][c] : qh[0][c];
        x0[c] = b0 ? xl[1][c] : xl[0][c]; x1[c] = b1 ? xh[1][c] : xh[0][c];
    }
    pb[0] = b0; pb[1] = b1;
}
// the quantised endpoints and p-bits q, pb equal a, apb (the channels the subset codes)
template <int NC>
ZTC_DEV bool same_ends(const int q[2][4], const int pb[2], const int a[2][4], const int apb[2]) {
    bool same = pb[0] == apb[0] && pb[1] == apb[1];
    #pragma unroll
    for (int c = 0; c < NC; c++) same = same && q[0][c] == a[0][c] && q[1][c] == a[1][c];
    return same;
}

// Passes [first, last) of a subset's fit sequence (zap_tex.h:489-515): pass 0 fits the endpoints (lo, hi); pass
// k > 0 is the k-th least-squares refit on the indices `idx` holds, which does not run at SSE 0, stops at a
// singular system, and is dropped (ending the sequence) when it does not lower the SSE. err: the SSE before
// `first`; q, pb, idx take each accepted pass. Returns the SSE; more: all the passes ran and the SSE is still
// above 0, so pass `last` would run. One fit call site keeps the code small. A refit that quantises to the
// accepted endpoints and p-bits would fit the same palette to the same texels and give the same SSE, which does not
// lower it: the sequence ends there without the fit.
template <int NC, int IB>
ZTC_DEV int subset_passes(TexRef ts, uint32_t mask, int n, bool shared_p, float lo[4], float hi[4], int first, int last, int err,
                          int q[2][4], int pb[2], uint64_t &idx, bool &more) {
    more = false;
    #pragma unroll 1
    for (int it = first; it < last; it++) {
        if (it > 0) {
            if (err <= 0) return err;
            float aa = 0.0f, ab = 0.0f, bb = 0.0f, sa[NC], sb[NC];
            #pragma unroll
            for (int c = 0; c < NC; c++) { sa[c] = 0.0f; sb[c] = 0.0f; }
            #pragma unroll 1
            for (int i = 0; i < 16; i++) {
                if (!((mask >> i) & 1u)) continue;
                float w = small_u2f((uint32_t)wbits(IB, (int)((idx >> (4 * i)) & 15u))) / 64.0f, u = 1.0f - w;
                aa = aa + u * u; ab = ab + u * w; bb = bb + w * w;
                const uint32_t x = ts[i];
                #pragma unroll
                for (int c = 0; c < NC; c++) { float xc = small_u2f(chan(x, c)); sa[c] = sa[c] + u * xc; sb[c] = sb[c] + w * xc; }
            }
            float det = aa * bb - ab * ab;
            if (det < 1e-6f && det > -1e-6f) return err;
            #pragma unroll
            for (int c = 0; c < 4; c++) {
                if (c < NC) { lo[c] = clamp255((sa[c] * bb - sb[c] * ab) / det); hi[c] = clamp255((sb[c] * aa - sa[c] * ab) / det); }
                else { lo[c] = 255.0f; hi[c] = 255.0f; }
            }
        }
        int nq[2][4], npb[2], x0[4], x1[4];
        subset_quant<NC>(n, shared_p, lo, hi, nq, npb, x0, x1);
        if (it > 0 && same_ends<NC>(nq, npb, q, pb)) return err;
        uint64_t ni;
        const int ne = palette_fit<NC, IB>(ts, mask, x0, x1, ni);
        if (it > 0 && ne >= err) return err;
        err = ne; idx = ni; pb[0] = npb[0]; pb[1] = npb[1];
        #pragma unroll
        for (int c = 0; c < 4; c++) { q[0][c] = nq[0][c]; q[1][c] = nq[1][c]; }
    }
    more = err > 0;
    return err;
}

// PCA start, fit, up to two least-squares refits (zap_tex.h:489-515). t: the texels in registers (for the
// principal axis), ts: the same texels for the rolled loops.
template <int NC, int IB>
ZTC_DEV int subset_encode(const uint32_t t[16], TexRef ts, uint32_t mask, int n, bool shared_p, int q[2][4], int pb[2],
                          uint64_t &idx) {
    float lo[4], hi[4];
    pca_endpoints<NC>(t, mask, lo, hi);
    bool more;
    return subset_passes<NC, IB>(ts, mask, n, shared_p, lo, hi, 0, 3, 0, q, pb, idx, more);
}

// ---------------------------------------------------------------- kernel A: mode 6 for every block
// mode-6 block from its fields (zap_tex.h:520-527): the anchor index's MSB must be 0, else the endpoints and
// p-bits swap and the indices invert (15 - i == i ^ 15)
ZTC_DEV uint4 pack_mode6_block(int q[2][4], int pb[2], uint64_t idx) {
    if (idx & 8u) {
        #pragma unroll
        for (int c = 0; c < 4; c++) { int s = q[0][c]; q[0][c] = q[1][c]; q[1][c] = s; }
        int s = pb[0]; pb[0] = pb[1]; pb[1] = s;
        idx ^= 0xFFFFFFFFFFFFFFFFull;
    }
    Bits128 o;
    o.put(1u << 6, 7);
    #pragma unroll
    for (int c = 0; c < 4; c++) { o.put((uint32_t)q[0][c], 7); o.put((uint32_t)q[1][c], 7); }
    o.put((uint32_t)pb[0], 1); o.put((uint32_t)pb[1], 1);
    o.put((uint32_t)(idx & 7u), 3);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((uint32_t)((idx >> (4 * i)) & 15u), 4);
    return make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
}

ZTC_DEV int mode6_encode(const uint32_t t[16], TexRef ts, uint4 &blk) {  // zap_tex.h:582-593
    int q[2][4], pb[2];
    uint64_t idx;
    int err = subset_encode<4, 4>(t, ts, 0xFFFFu, 8, false, q, pb, idx);
    blk = pack_mode6_block(q, pb, idx);
    return err;
}

// endpoints (7 bits each, endpoint-major) and p-bits of a mode-6 fit in one word
ZTC_DEV uint64_t pack_qp(const int q[2][4], const int pb[2]) {
    uint64_t v = (uint64_t)pb[0] << 56 | (uint64_t)pb[1] << 57;
    #pragma unroll
    for (int k = 0; k < 8; k++) v |= (uint64_t)q[k >> 2][k & 3] << (7 * k);
    return v;
}
ZTC_DEV void unpack_qp(uint64_t v, int q[2][4], int pb[2]) {
    #pragma unroll
    for (int k = 0; k < 8; k++) q[k >> 2][k & 3] = (int)((v >> (7 * k)) & 0x7Fu);
    pb[0] = (int)((v >> 56) & 1u); pb[1] = (int)((v >> 57) & 1u);
}

// Mode 6 for the CTA's blocks, one per thread, with the second least-squares refit compacted. Every thread runs
// the PCA, the first fit and the first refit of its block; the blocks whose second refit would run (about a fifth
// of them on photographic content, yet nearly every warp holds one) are listed in shared memory, and the first
// threads of the CTA run those refits on the owners' texels, so they cost about a fifth of the warps instead of
// nearly all. Same bytes and SSE as mode6_encode. Every thread of the CTA calls it (it synchronises); a `valid`
// thread's block is in t and in column threadIdx.x of s_tex.
// ROLLED: the principal axis in rolled loops over s_tex, for launches of several waves (see bc1_encode_cta)
template <int CTA, bool ROLLED>
__device__ __forceinline__ int mode6_encode_cta(bool valid, const uint32_t t[16], uint32_t (*s_tex)[CTA], uint4 &blk) {
    static_assert(CTA % 32 == 0 && CTA <= 1024, "whole warps");
    __shared__ uint64_t s_idx[CTA], s_qp[CTA];
    __shared__ int s_err[CTA], s_wcnt[CTA / 32];
    __shared__ uint16_t s_list[CTA];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float lo[4], hi[4];
    if (valid) {
        if (ROLLED) pca_endpoints<4, 1>(TexRef{&s_tex[0][tid], CTA}, 0xFFFFu, lo, hi);  // less code, no spills
        else pca_endpoints<4>(t, 0xFFFFu, lo, hi);
    }
    bool active = valid;
    int owner = tid, first = 0, err = 0, q[2][4], pb[2];  // q, pb, idx, err: the accepted fit (the owner's in round 1)
    uint64_t idx = 0;
    #pragma unroll 1
    for (int round = 0; round < 2; round++) {
        bool more = false;
        const int e_in = err;
        if (active)
            err = subset_passes<4, 4>(TexRef{&s_tex[0][owner], CTA}, 0xFFFFu, 8, false, lo, hi, first, round ? 3 : 2, err, q, pb, idx, more);
        if (active && (round == 0 || err < e_in)) { s_err[owner] = err; s_idx[owner] = idx; s_qp[owner] = pack_qp(q, pb); }
        if (round == 1) break;
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, more);
        if (lane == 0) s_wcnt[warp] = __popc(bal);
        __syncthreads();
        int base = 0, total = 0;
        #pragma unroll
        for (int w = 0; w < CTA / 32; w++) { const int c = s_wcnt[w]; base += w < warp ? c : 0; total += c; }
        const int pos = base + __popc(bal & ((1u << lane) - 1u));
        if (more && ZTC_IN_BOUNDS(pos, CTA, 2)) s_list[pos] = (uint16_t)tid;
        __syncthreads();
        active = tid < total;
        if (active) owner = s_list[tid];
        if (active && !ZTC_IN_BOUNDS(owner, CTA, 8)) active = false;
        if (active) { err = s_err[owner]; idx = s_idx[owner]; unpack_qp(s_qp[owner], q, pb); }
        first = 2;
    }
    __syncthreads();
    if (!valid) return 0;
    unpack_qp(s_qp[tid], q, pb);
    blk = pack_mode6_block(q, pb, s_idx[tid]);
    return s_err[tid];
}

// CTA sizes of the mode-6 kernel. A larger CTA shares one compacted-refit list among more blocks (2048x2048:
// 64 threads 0.119 ms, 128 0.105, 256 0.099, 384 0.100, 512 0.103); a launch smaller than one full wave of large
// CTAs takes the small size instead, which keeps more SMs busy (512x512 in 256-thread CTAs: 64 CTAs for 148 SMs).
// The large size is 224 threads at 4 CTAs per SM (72 registers): 896 threads per SM instead of 768 at 256 x 3,
// so 2048x2048 fills 1.98 waves instead of 2.31 (0.0980 -> 0.0966 ms).
constexpr int kMode6Small = 128, kMode6Large = 224;
template <int CTA>
constexpr int mode6_min_ctas() { return CTA == kMode6Large ? 4 : ZTC_MINB_BC7_MODE6 * 128 / CTA; }
template <int CTA>
__global__ void __launch_bounds__(CTA, mode6_min_ctas<CTA>()) bc7_mode6_kernel(SrcU8 src, int bw, int by0, int nblocks,
                                                        BlockOut out, size_t b0, uint32_t *__restrict__ count, uint2 *__restrict__ items) {
    __shared__ uint32_t s_tex[16][CTA];  // column threadIdx.x: this thread's block
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = b < nblocks;
    uint32_t t[16];
    if (valid) {
        gather_block(src, b % bw, by0 + b / bw, t);
        #pragma unroll
        for (int i = 0; i < 16; i++) s_tex[i][threadIdx.x] = t[i];
    }
    uint4 blk;
    const int err = mode6_encode_cta<CTA, CTA != kMode6Small>(valid, t, s_tex, blk);
    if (valid) put_block16(out, b0 + (size_t)b, blk);
    bool hard = valid && err > 16 * 4;  // zap_tex.h:758 early exit
    unsigned ballot = __ballot_sync(0xFFFFFFFFu, hard);
    if (ballot) {
        int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(ballot));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        const int pos = (int)base + __popc(ballot & ((1u << lane) - 1u));
        if (hard && ZTC_IN_BOUNDS(pos, nblocks, 6)) items[pos] = make_uint2((uint32_t)b, (uint32_t)err);
    }
}

// the mode-6 launch, at the CTA size that suits its block count
cudaError_t launch_mode6(const SrcU8 &src, int bw, int by0, int nblocks, const BlockOut &out, size_t b0, uint32_t *count, uint2 *items,
                         cudaStream_t s) {
    if (nblocks >= ztc_sm_count() * mode6_min_ctas<kMode6Large>() * kMode6Large)
        bc7_mode6_kernel<kMode6Large><<<(nblocks + kMode6Large - 1) / kMode6Large, kMode6Large, 0, s>>>(src, bw, by0, nblocks, out, b0, count, items);
    else
        bc7_mode6_kernel<kMode6Small><<<(nblocks + kMode6Small - 1) / kMode6Small, kMode6Small, 0, s>>>(src, bw, by0, nblocks, out, b0, count, items);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- kernel B pieces
// mode 5 part (zap_tex.h:597-657): 2-bit palette on the colour part (RGB of the rotated texels, 7-bit endpoints)
// or the alpha part (their A byte, 8-bit endpoints). Both kinds run the same code with nc = 3 or 1 channels, so
// the colour and alpha lanes of a group do not diverge: a part's texel holds its channels in the low bytes and
// zeros above, and unused palette channels are zero too, so the integer keys and sums are those of an nc-channel
// computation, and each used channel's float sums run in the reference's order.
ZTC_DEV uint32_t rotate_texel(uint32_t v, int rot) {  // mode 5 rotation: swap A with R (1), G (2) or B (3)
    if (rot) {
        const int sh = 8 * (rot - 1);
        const uint32_t a = v >> 24, c = (v >> sh) & 0xFFu;
        v = (v & ~((0xFFu << sh) | 0xFF000000u)) | (a << sh) | (c << 24);
    }
    return v;
}
// The mode 5 helpers take the part at compile time, KIND = kPartColour (rotated RGB, 7-bit endpoints) or kPartAlpha
// (rotated A, 8-bit endpoints): the alpha part's loops run over its one channel.
constexpr int kPartColour = 1, kPartAlpha = 2;

template <int KIND>
ZTC_DEV void m5_quant(const float v[3], int nc, int n, int q[3], int x8[3]) {
    const int top = (1 << n) - 1;
    #pragma unroll
    for (int c = 0; c < 3; c++) {
        if (c >= nc || (KIND == kPartAlpha && c > 0)) { q[c] = 0; x8[c] = 0; continue; }
        // finite v within [-510, 765] (clamped least-squares endpoints, or the starts), as for quant_pbit
        const float gv = div255(v[c] * (float)top) + 0.5f;
        ZTC_TRUNC_DOMAIN(gv);
        int g = trunc_mid(gv), bq = 0, bd = 1 << 30;
        #pragma unroll
        for (int k = 0; k < 3; k++) {
            int tq = clampi(around(g, k), 0, top);
            const float dv = fabsf(small_u2f((uint32_t)expand_bits(tq, n)) - v[c]);
            ZTC_TRUNC_DOMAIN(dv);
            int d = trunc_small(dv);
            if (d < bd) { bd = d; bq = tq; }
        }
        q[c] = bq; x8[c] = expand_bits(bq, n);
    }
}
// The part's texels p[16] are in registers (the colour part: rotated RGB in the low three bytes; the alpha part:
// the rotated alpha in byte 0), and the texel loops are unrolled: the modes-5/1 launch holds few warps per SM, so
// the length of each lane's dependent chain sets its time.
template <int KIND>
ZTC_DEV int m5_fit(const uint32_t p[16], const int x0[3], const int x1[3], uint32_t &idx) {
    uint32_t pal[4];
    int A[4];
    #pragma unroll
    for (int j = 0; j < 4; j++) {
        uint32_t e = 0;
        #pragma unroll
        for (int c = 0; c < (KIND == kPartAlpha ? 1 : 3); c++) e |= (uint32_t)lerp64(x0[c], x1[c], w2(j)) << (8 * c);
        pal[j] = e; A[j] = (int)dot4(e, e) * 4 + j;
    }
    int err = 0;
    uint32_t bits = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        int m = min(min(A[0] - 8 * (int)dot4(p[i], pal[0]), A[1] - 8 * (int)dot4(p[i], pal[1])),
                    min(A[2] - 8 * (int)dot4(p[i], pal[2]), A[3] - 8 * (int)dot4(p[i], pal[3])));
        err += (m >> 2) + (int)dot4(p[i], p[i]);
        bits |= (uint32_t)(m & 3) << (2 * i);
    }
    idx = bits;
    return err;
}
// Least-squares endpoints for fixed 2-bit indices (zap_tex.h:636-648). The reference sums floats, but every one of
// its sums is exact: w = k / 64 with k in {0, 21, 43, 64} and u = 1 - w, so u*u, u*w and w*w are multiples of 2^-12
// below 1, u*x and w*x multiples of 2^-6 below 256, and no partial sum of 16 terms needs more than 24 bits in those
// units. Integer sums scaled by 2^-12 and 2^-6 are therefore the reference's floats, bit for bit, in any order.
template <int KIND>
ZTC_DEV bool m5_lsq(const uint32_t p[16], int nc, uint32_t idx, float lo[3], float hi[3]) {
    constexpr int kC = KIND == kPartAlpha ? 1 : 3;
    int aa = 0, ab = 0, bb = 0, sa[3] = {0, 0, 0}, sb[3] = {0, 0, 0};
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        const int k = (int)((0x402B1500u >> (8 * ((idx >> (2 * i)) & 3u))) & 0xFFu), u = 64 - k;  // w2: 0, 21, 43, 64
        aa += u * u; ab += u * k; bb += k * k;
        #pragma unroll
        for (int c = 0; c < kC; c++) { const int x = (int)chan(p[i], c); sa[c] += u * x; sb[c] += k * x; }
    }
    const float faa = small_u2f((uint32_t)aa) * (1.0f / 4096.0f), fab = small_u2f((uint32_t)ab) * (1.0f / 4096.0f),
                fbb = small_u2f((uint32_t)bb) * (1.0f / 4096.0f);  // sums below 2^17
    float det = faa * fbb - fab * fab;
    if (det < 1e-6f && det > -1e-6f) return false;
    #pragma unroll
    for (int c = 0; c < kC; c++)
        if (c < nc) {
            const float fa = small_u2f((uint32_t)sa[c]) * (1.0f / 64.0f), fb = small_u2f((uint32_t)sb[c]) * (1.0f / 64.0f);  // below 2^18
            lo[c] = clamp255((fa * fbb - fb * fab) / det); hi[c] = clamp255((fb * faa - fa * fab) / det);
        }
    return true;
}
// quantise, fit, up to two least-squares refits (zap_tex.h:626-657); lo / hi: the start endpoints
template <int KIND>
ZTC_DEV int m5_part(const uint32_t p[16], float lo[3], float hi[3], int q[2][3], uint32_t &idx) {
    constexpr bool alpha = KIND == kPartAlpha;
    const int nc = alpha ? 1 : 3, n = alpha ? 8 : 7;
    int err = 0;
    #pragma unroll 1
    for (int it = 0; it < 3; it++) {
        if (it > 0 && !m5_lsq<KIND>(p, nc, idx, lo, hi)) break;
        int tq[2][3], x0[3], x1[3];
        m5_quant<KIND>(lo, nc, n, tq[0], x0); m5_quant<KIND>(hi, nc, n, tq[1], x1);
        if (it > 0) {  // the accepted endpoints again: the same fit and SSE, which ends the refits
            bool same = true;
            #pragma unroll
            for (int c = 0; c < 3; c++) same = same && (c >= nc || (tq[0][c] == q[0][c] && tq[1][c] == q[1][c]));
            if (same) break;
        }
        uint32_t ti;
        const int e = m5_fit<KIND>(p, x0, x1, ti);
        if (it > 0 && e >= err) break;
        err = e; idx = ti;
        #pragma unroll
        for (int c = 0; c < 3; c++) { q[0][c] = tq[0][c]; q[1][c] = tq[1][c]; }
        if (err <= 0) break;
    }
    return err;
}

// partition score (zap_tex.h:722-748) from the 9 moment sums of subset 1 (s1, over its n1 texels, added in texel
// order) and of the whole block (tot); subset 0's sums are tot - s1, as in the reference
ZTC_DEV float partition_score(const float s1[9], int n1, const float tot[9]) {
    float score = 0.0f;
    #pragma unroll 1
    for (int k = 0; k < 2; k++) {  // rolled (with the power iteration): one copy of the divisions
        float m[9];
        #pragma unroll
        for (int j = 0; j < 9; j++) m[j] = k ? s1[j] : tot[j] - s1[j];
        float n = small_u2f((uint32_t)(k ? n1 : 16 - n1));
        if (n < 2) continue;
        const float ni = 1.0f / n;  // the six quotients below: integer-valued numerators below 2^24 (div_small)
        float S00 = m[3] - div_small(m[0] * m[0], n, ni), S01 = m[6] - div_small(m[0] * m[1], n, ni);
        float S02 = m[7] - div_small(m[0] * m[2], n, ni), S11 = m[4] - div_small(m[1] * m[1], n, ni);
        float S12 = m[8] - div_small(m[1] * m[2], n, ni), S22 = m[5] - div_small(m[2] * m[2], n, ni);
        float tr = S00 + S11 + S22, a0, a1, a2;
        if (S00 >= S11 && S00 >= S22) { a0 = S00; a1 = S01; a2 = S02; }
        else if (S11 >= S22) { a0 = S01; a1 = S11; a2 = S12; }
        else { a0 = S02; a1 = S12; a2 = S22; }
        #pragma unroll 1
        for (int it = 0; it < 3; it++) {
            float v0 = S00 * a0 + S01 * a1 + S02 * a2;
            float v1 = S01 * a0 + S11 * a1 + S12 * a2;
            float v2 = S02 * a0 + S12 * a1 + S22 * a2;
            float mx = 1e-12f;
            mx = v0 > mx ? v0 : -v0 > mx ? -v0 : mx;
            mx = v1 > mx ? v1 : -v1 > mx ? -v1 : mx;
            mx = v2 > mx ? v2 : -v2 > mx ? -v2 : mx;
            a0 = v0 / mx; a1 = v1 / mx; a2 = v2 / mx;
        }
        float vv = a0 * a0 + a1 * a1 + a2 * a2, vsv = 0.0f;
        vsv = vsv + a0 * (S00 * a0 + S01 * a1 + S02 * a2);
        vsv = vsv + a1 * (S01 * a0 + S11 * a1 + S12 * a2);
        vsv = vsv + a2 * (S02 * a0 + S12 * a1 + S22 * a2);
        float lam = vv > 1e-12f ? vsv / vv : 0.0f;
        score = score + (tr - lam * (48.0f / 49.0f));
    }
    return score;
}

// (score, partition) lexicographic "less", with the reference's float "<" (so -0 == +0)
ZTC_DEV bool rank_less(float e, int p, float e2, int p2) { return e < e2 || (!(e2 < e) && p < p2); }

constexpr int kBc7Group = 8;
constexpr int kMode1Tries = 4;  // partitions fully fitted after ranking (ZAP__BC7_M1K, zap_tex.h:750-752)

__device__ __forceinline__ bool mode1_fits(TexRef ts, const int cand[kMode1Tries], int &err, uint4 &blk, const int l, const unsigned gmask);

// Mode 1's ranking of one opaque block (zap_tex.h:764-775) by the 8 lanes of a group (lane l, group mask gmask):
// cand[0..3] the partitions of the four least (score, partition), -1 past the last valid one (group-uniform).
// ts: the block's texels (the group's shared-memory copy).
__device__ __forceinline__ void group_rank(TexRef ts, int cand[kMode1Tries], const int l, const unsigned gmask) {
    // ---- mode 1 ranking: lane scores partitions l, l + 8, ..., l + 56 (zap_tex.h:764-775), four per round:
    // one pass over the texels adds each texel's 9 moments to the block totals and to the sums of the
    // four partitions' subset 1, every sum in texel order as the reference adds them
    float ce[kMode1Tries];
    int cp[kMode1Tries];
    #pragma unroll
    for (int j = 0; j < kMode1Tries; j++) { ce[j] = 1e30f; cp[j] = 64; }
    #pragma unroll 1
    for (int round = 0; round < 2; round++) {
        uint32_t pm[4];
        int n1[4];
        float s1[4][9], tot[9];
        #pragma unroll
        for (int k = 0; k < 4; k++) {
            pm[k] = kP2[l + kBc7Group * (4 * round + k)];
            n1[k] = 0;
            #pragma unroll
            for (int j = 0; j < 9; j++) s1[k][j] = 0.0f;
        }
        #pragma unroll
        for (int j = 0; j < 9; j++) tot[j] = 0.0f;
        #pragma unroll 1
        for (int i = 0; i < 16; i++) {
            const uint32_t x = ts[i];
            const float rr = small_u2f(chan(x, 0)), gg = small_u2f(chan(x, 1)), bb = small_u2f(chan(x, 2));
            const float mo[9] = {rr, gg, bb, rr * rr, gg * gg, bb * bb, rr * gg, rr * bb, gg * bb};
            #pragma unroll
            for (int j = 0; j < 9; j++) tot[j] = tot[j] + mo[j];
            #pragma unroll
            for (int k = 0; k < 4; k++)
                if ((pm[k] >> i) & 1u) {
                    n1[k]++;
                    #pragma unroll
                    for (int j = 0; j < 9; j++) s1[k][j] = s1[k][j] + mo[j];
                }
        }
        #pragma unroll 1
        for (int k = 0; k < 4; k++) {  // rolled: partition k's sums are at [0], the later ones shift down after it
            const int part = l + kBc7Group * (4 * round + k);
            const float e = partition_score(s1[0], n1[0], tot);
            #pragma unroll
            for (int r = 0; r < 3; r++) {
                n1[r] = n1[r + 1];
                #pragma unroll
                for (int j = 0; j < 9; j++) s1[r][j] = s1[r + 1][j];
            }
            // insertion keeps (score, partition) order; NaN and >= 1e30 never enter, as in the reference
            #pragma unroll
            for (int j = 0; j < kMode1Tries; j++) {
                if (e < ce[j]) {
                    #pragma unroll
                    for (int s = kMode1Tries - 1; s > j; s--) { ce[s] = ce[s - 1]; cp[s] = cp[s - 1]; }
                    ce[j] = e; cp[j] = part;
                    break;
                }
            }
        }
    }
    // merge the eight sorted lists: four rounds of a group-wide (score, partition) minimum
    #pragma unroll
    for (int j = 0; j < kMode1Tries; j++) {
        float he = ce[0];
        int hp = cp[0];
        #pragma unroll
        for (int m = 1; m < kBc7Group; m <<= 1) {
            float oe = __shfl_xor_sync(gmask, he, m, kBc7Group);
            int op = __shfl_xor_sync(gmask, hp, m, kBc7Group);
            if (rank_less(oe, op, he, hp)) { he = oe; hp = op; }
        }
        cand[j] = hp < 64 ? hp : -1;
        if (hp < 64 && (hp & (kBc7Group - 1)) == l) {  // owner pops its head
            #pragma unroll
            for (int s = 0; s < kMode1Tries - 1; s++) { ce[s] = ce[s + 1]; cp[s] = cp[s + 1]; }
            ce[kMode1Tries - 1] = 1e30f; cp[kMode1Tries - 1] = 64;
        }
    }
}

// Mode 1 of one opaque block (zap_tex.h:764-783) by the 8 lanes of a group: true, with err and blk updated, when the
// best of the ranked partitions has an SSE below err
__device__ __forceinline__ bool bc7_group_mode1(TexRef ts, int &err, uint4 &blk, const int l, const unsigned gmask) {
    int cand[kMode1Tries];
    group_rank(ts, cand, l, gmask);
    return mode1_fits(ts, cand, err, blk, l, gmask);
}

// Mode 1's ranking of one opaque block by all 64 threads of a CTA, one partition each (tid = partition; the same
// sums, scores and order as group_rank), then four rounds of a CTA-wide (score, partition) minimum; for lists of at
// most one block per CTA, where a block's ranking by one group (8 partitions per lane) is the longest chain of the
// launch. The CTA has 64 threads (two warps, one partition per thread), and every one of them calls it (it
// synchronises); s_e, s_p: two slots each. cand is the same in every thread.
__device__ __forceinline__ void cta_rank64(TexRef ts, int cand[kMode1Tries], float *s_e, int *s_p) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t pm = kP2[tid];
    float s1[9], tot[9];
    int n1 = 0;
    #pragma unroll
    for (int j = 0; j < 9; j++) { s1[j] = 0.0f; tot[j] = 0.0f; }
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        const uint32_t x = ts[i];
        const float rr = small_u2f(chan(x, 0)), gg = small_u2f(chan(x, 1)), bb = small_u2f(chan(x, 2));
        const float mo[9] = {rr, gg, bb, rr * rr, gg * gg, bb * bb, rr * gg, rr * bb, gg * bb};
        #pragma unroll
        for (int j = 0; j < 9; j++) tot[j] = tot[j] + mo[j];
        if ((pm >> i) & 1u) {
            n1++;
            #pragma unroll
            for (int j = 0; j < 9; j++) s1[j] = s1[j] + mo[j];
        }
    }
    const float e = partition_score(s1, n1, tot);
    const bool valid = e < 1e30f;  // NaN and >= 1e30 never enter, as in the reference
    float me = valid ? e : 1e30f;
    int mp = valid ? tid : 64;
    #pragma unroll 1
    for (int j = 0; j < kMode1Tries; j++) {
        float he = me;
        int hp = mp;
        #pragma unroll
        for (int m = 16; m >= 1; m >>= 1) {
            const float oe = __shfl_xor_sync(0xFFFFFFFFu, he, m);
            const int op = __shfl_xor_sync(0xFFFFFFFFu, hp, m);
            if (rank_less(oe, op, he, hp)) { he = oe; hp = op; }
        }
        if (lane == 0) { s_e[warp] = he; s_p[warp] = hp; }
        __syncthreads();
        const bool second = rank_less(s_e[1], s_p[1], s_e[0], s_p[0]);
        const int bp = second ? s_p[1] : s_p[0];
        cand[j] = bp < 64 ? bp : -1;
        if (bp < 64 && bp == tid) { me = 1e30f; mp = 64; }  // taken
        __syncthreads();  // the slots are written again next round
    }
}

// Mode 1's fits of the ranked partitions cand[0..3] (-1: none) by the 8 lanes of a group, lane = candidate * 2 +
// subset (zap_tex.h:687-708, 776): true, with err and blk updated, when the first candidate of the least SSE is
// below err. cand is group-uniform.
__device__ __forceinline__ bool mode1_fits(TexRef ts, const int cand[kMode1Tries], int &err, uint4 &blk, const int l, const unsigned gmask) {
    const int j = l >> 1, sub = l & 1;
    int pj = 0;
    #pragma unroll
    for (int k = 0; k < kMode1Tries; k++) if (k == j) pj = cand[k];
    int q1[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, pb1[2] = {0, 0}, e1 = 1 << 29;
    uint64_t i1 = 0;
    uint32_t pmask = 0;
    if (pj >= 0) {
        pmask = sub ? (uint32_t)kP2[pj] : (~(uint32_t)kP2[pj] & 0xFFFFu);
        float lo[4], hi[4];  // subset_encode with the principal axis taken in rolled loops over ts
        pca_endpoints<3, 1>(ts, pmask, lo, hi);
        bool more;
        e1 = subset_passes<3, 3>(ts, pmask, 7, true, lo, hi, 0, 3, 0, q1, pb1, i1, more);
        int anchor = sub ? (int)kA2[pj] : 0;
        if ((i1 >> (4 * anchor)) & 4u) {  // anchor MSB must be 0: swap, 7 - i == i ^ 7 on the subset's texels
            #pragma unroll
            for (int c = 0; c < 3; c++) { int s = q1[0][c]; q1[0][c] = q1[1][c]; q1[1][c] = s; }
            uint64_t sel = 0;
            #pragma unroll
            for (int i = 0; i < 16; i++) if ((pmask >> i) & 1u) sel |= 7ull << (4 * i);
            i1 ^= sel;
        }
    }
    int ecand = e1 + (int)__shfl_xor_sync(gmask, (uint32_t)e1, 1, kBc7Group);
    // first candidate (in rank order) with the smallest SSE below the current best
    uint32_t ckey = (pj >= 0 && ecand < err) ? (((uint32_t)ecand << 2) | (uint32_t)j) : 0xFFFFFFFFu;
    ckey = min(ckey, __shfl_xor_sync(gmask, ckey, 2, kBc7Group));
    ckey = min(ckey, __shfl_xor_sync(gmask, ckey, 4, kBc7Group));
    if (ckey != 0xFFFFFFFFu) {
        const int bj = (int)(ckey & 3u);
        uint32_t ew0 = (uint32_t)q1[0][0] | ((uint32_t)q1[0][1] << 6) | ((uint32_t)q1[0][2] << 12) | ((uint32_t)pb1[0] << 18);
        uint32_t ew1 = (uint32_t)q1[1][0] | ((uint32_t)q1[1][1] << 6) | ((uint32_t)q1[1][2] << 12);
        uint32_t ilo = (uint32_t)i1, ihi = (uint32_t)(i1 >> 32);
        uint32_t a0 = __shfl_sync(gmask, ew0, 2 * bj, kBc7Group), a1 = __shfl_sync(gmask, ew1, 2 * bj, kBc7Group);
        uint32_t b0w = __shfl_sync(gmask, ew0, 2 * bj + 1, kBc7Group), b1w = __shfl_sync(gmask, ew1, 2 * bj + 1, kBc7Group);
        uint32_t il = __shfl_sync(gmask, ilo, 2 * bj, kBc7Group) | __shfl_sync(gmask, ilo, 2 * bj + 1, kBc7Group);
        uint32_t ih = __shfl_sync(gmask, ihi, 2 * bj, kBc7Group) | __shfl_sync(gmask, ihi, 2 * bj + 1, kBc7Group);
        int part = __shfl_sync(gmask, pj, 2 * bj, kBc7Group);
        err = (int)(ckey >> 2);
        uint64_t full = (uint64_t)il | ((uint64_t)ih << 32);
        Bits128 o;
        o.put(2u, 2);
        o.put((uint32_t)part, 6);
        #pragma unroll
        for (int c = 0; c < 3; c++) {
            o.put((a0 >> (6 * c)) & 63u, 6); o.put((a1 >> (6 * c)) & 63u, 6);
            o.put((b0w >> (6 * c)) & 63u, 6); o.put((b1w >> (6 * c)) & 63u, 6);
        }
        o.put((a0 >> 18) & 1u, 1); o.put((b0w >> 18) & 1u, 1);
        const int anchor = (int)kA2[part];
        #pragma unroll
        for (int i = 0; i < 16; i++) o.put((uint32_t)((full >> (4 * i)) & 7u), (i == 0 || i == anchor) ? 2 : 3);
        blk = make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
        return true;
    }
    return false;
}

ZTC_DEV bool block_opaque(const uint32_t t[16]) {
    bool opaque = true;
    #pragma unroll
    for (int i = 0; i < 16; i++) opaque &= (t[i] >> 24) == 255u;
    return opaque;
}

// the group's shared-memory copy of its block (lane l writes texels l and l + 8), for the rolled loops
__device__ __forceinline__ TexRef stage_group_texels(uint32_t *gtex, const uint32_t t[16], int l, unsigned gmask) {
    __syncwarp(gmask);  // the group's reads of its previous block are done
    #pragma unroll
    for (int i = 0; i < 16; i++)
        if ((i & (kBc7Group - 1)) == l) gtex[i] = t[i];
    __syncwarp(gmask);
    return TexRef{gtex, 1};
}

// the mode-5 block (zap_tex.h:674-684) of rotation brot from its colour part (cq, cq2: the 7-bit endpoints, ci: the
// 2-bit indices, anchor already fixed) and its alpha part (aq: the 8-bit endpoints, ai: the indices)
__device__ __forceinline__ uint4 pack_mode5_block(int brot, uint32_t cq, uint32_t cq2, uint32_t ci, uint32_t aq, uint32_t ai) {
    Bits128 o;
    o.put(1u << 5, 6);
    o.put((uint32_t)brot, 2);
    const uint32_t c0[3] = {cq & 127u, (cq >> 7) & 127u, (cq >> 14) & 127u}, c1[3] = {(cq >> 21) & 127u, cq2 & 127u, (cq2 >> 7) & 127u};
    #pragma unroll
    for (int c = 0; c < 3; c++) { o.put(c0[c], 7); o.put(c1[c], 7); }
    o.put(aq & 255u, 8); o.put((aq >> 8) & 255u, 8);
    o.put(ci & 1u, 1);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((ci >> (2 * i)) & 3u, 2);
    o.put(ai & 1u, 1);
    #pragma unroll
    for (int i = 1; i < 16; i++) o.put((ai >> (2 * i)) & 3u, 2);
    return make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
}

// Modes 5 and 1 of single-image encodes over the mode-6 work list. A CTA of two warps takes 8 listed blocks at a
// time: warp 0 fits their mode-5 colour parts and warp 1 their alpha parts, lane = block * 4 + rotation, each warp
// on code specialised to its part (no lane of a warp waits on the other part's branch, and the alpha part's loops
// run over its one channel); the best rotation of each block is then chosen as the reference does, and mode 1 runs
// for the opaque ones, an 8-lane group per block.
constexpr int kHardBlocks = 8;

__device__ __forceinline__ int m5_colour_lane(TexRef ts, int rot, uint32_t &qw, uint32_t &qw2, uint32_t &idx) {
    uint32_t r[16];
    #pragma unroll
    for (int i = 0; i < 16; i++) r[i] = rotate_texel(ts[i], rot) & 0x00FFFFFFu;  // the colour part's texels
    float lo[4], hi[4];
    pca_endpoints<3>(r, 0xFFFFu, lo, hi);  // the colour part starts from the principal axis of the rotated RGB
    float lo5[3] = {lo[0], lo[1], lo[2]}, hi5[3] = {hi[0], hi[1], hi[2]};
    int q5[2][3] = {{0, 0, 0}, {0, 0, 0}};
    uint32_t i5 = 0;
    const int e5 = m5_part<kPartColour>(r, lo5, hi5, q5, i5);
    if (i5 & 2u) {  // anchor MSB must be 0 (zap_tex.h:673-674): swap, 3 - i == i ^ 3 for 2-bit indices
        #pragma unroll
        for (int c = 0; c < 3; c++) { int t = q5[0][c]; q5[0][c] = q5[1][c]; q5[1][c] = t; }
        i5 ^= 0xFFFFFFFFu;
    }
    qw = (uint32_t)q5[0][0] | ((uint32_t)q5[0][1] << 7) | ((uint32_t)q5[0][2] << 14) | ((uint32_t)q5[1][0] << 21);
    qw2 = (uint32_t)q5[1][1] | ((uint32_t)q5[1][2] << 7);
    idx = i5;
    return e5;
}

__device__ __forceinline__ int m5_alpha_lane(TexRef ts, int rot, uint32_t &qw, uint32_t &idx) {
    float lo5[3] = {255.0f, 0.0f, 0.0f}, hi5[3] = {0.0f, 0.0f, 0.0f};
    uint32_t r[16];
    #pragma unroll
    for (int i = 0; i < 16; i++) {  // the alpha part's texels; it starts from their range
        r[i] = rotate_texel(ts[i], rot) >> 24;
        const float a = small_u2f(r[i]);
        if (a < lo5[0]) lo5[0] = a;
        if (a > hi5[0]) hi5[0] = a;
    }
    int q5[2][3] = {{0, 0, 0}, {0, 0, 0}};
    uint32_t i5 = 0;
    const int e5 = m5_part<kPartAlpha>(r, lo5, hi5, q5, i5);
    if (i5 & 2u) {
        int t = q5[0][0]; q5[0][0] = q5[1][0]; q5[1][0] = t;
        i5 ^= 0xFFFFFFFFu;
    }
    qw = (uint32_t)q5[0][0] | ((uint32_t)q5[1][0] << 8);
    idx = i5;
    return e5;
}

__global__ void __launch_bounds__(64, ZTC_MINB_BC7_MODE5) bc7_hard_kernel(SrcU8 src, int bw, int by0, BlockOut out, size_t b0,
                                                        const uint32_t *__restrict__ count, uint2 *items) {
    __shared__ uint32_t s_tex[kHardBlocks][17];  // per block (padded: the groups of a warp hit distinct banks)
    __shared__ uint2 s_item[kHardBlocks];        // (block index, mode-6 SSE); x = ~0 past the list's end
    __shared__ int s_cerr[kHardBlocks][4], s_aerr[kHardBlocks][4];
    __shared__ uint32_t s_cq[kHardBlocks][4], s_cq2[kHardBlocks][4], s_ci[kHardBlocks][4], s_aq[kHardBlocks][4], s_ai[kHardBlocks][4];
    __shared__ int s_op[64], s_wcnt[2];          // pass 2: the list positions of a chunk's opaque blocks
    __shared__ float s_re[2];                    // cta_rank64's slots
    __shared__ int s_rp[2];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = (int)*(volatile const uint32_t *)count;
    // one round per CTA at most (short lists): pass 2 finds the round's blocks in shared memory; one block per CTA at
    // most (the shortest lists): that block's mode-1 ranking takes all 64 threads (these tests are grid-uniform)
    const bool one_round = n <= (int)gridDim.x * kHardBlocks, sparse = n <= (int)gridDim.x;
    const int per = sparse ? 1 : kHardBlocks;  // listed blocks per CTA and round
    // ---- pass 1, mode 5 (zap_tex.h:659-684) of every listed block the CTA holds, `per` per round: warp 0 fits the
    // colour parts and warp 1 the alpha parts, lane = block * 4 + rotation; the block is stored when mode 5 wins, and
    // its list entry keeps its SSE so far and, in bit 31 of the index, whether it is opaque (mode 1 is next)
    for (int base = blockIdx.x * per; base < n; base += gridDim.x * per) {
        if (tid < kHardBlocks) {  // one thread per block gathers its texels (16-byte row loads)
            const int it = base + tid;
            uint2 item = make_uint2(0xFFFFFFFFu, 0u);
            if (tid < per && it < n) {
                item = items[it];
                uint32_t t[16];
                gather_block(src, (int)item.x % bw, by0 + (int)item.x / bw, t);
                #pragma unroll
                for (int i = 0; i < 16; i++) s_tex[tid][i] = t[i];
            }
            s_item[tid] = item;
        }
        __syncthreads();
        {
            const int blk = lane >> 2, rot = lane & 3;
            if (s_item[blk].x != 0xFFFFFFFFu) {
                const TexRef ts{s_tex[blk], 1};
                uint32_t qw = 0, qw2 = 0, idx = 0;
                if (warp == 0) {
                    s_cerr[blk][rot] = m5_colour_lane(ts, rot, qw, qw2, idx);
                    s_cq[blk][rot] = qw; s_cq2[blk][rot] = qw2; s_ci[blk][rot] = idx;
                } else {
                    s_aerr[blk][rot] = m5_alpha_lane(ts, rot, qw, idx);
                    s_aq[blk][rot] = qw; s_ai[blk][rot] = idx;
                }
            }
        }
        __syncthreads();
        if (tid < kHardBlocks && s_item[tid].x != 0xFFFFFFFFu) {  // the best rotation: (SSE, rotation) lexicographic
            uint32_t key = 0xFFFFFFFFu;
            #pragma unroll
            for (int r = 0; r < 4; r++) key = min(key, ((uint32_t)(s_cerr[tid][r] + s_aerr[tid][r]) << 2) | (uint32_t)r);
            const int brot = (int)(key & 3u), best5 = (int)(key >> 2);
            const uint2 item = s_item[tid];
            int err = (int)item.y;
            if (best5 < err) {  // decoded SSE == fit SSE (see the file header)
                err = best5;
                put_block16(out, b0 + (size_t)item.x,
                            pack_mode5_block(brot, s_cq[tid][brot], s_cq2[tid][brot], s_ci[tid][brot], s_aq[tid][brot], s_ai[tid][brot]));
            }
            bool opaque = true;
            #pragma unroll
            for (int i = 0; i < 16; i++) opaque &= (s_tex[tid][i] >> 24) == 255u;
            const uint2 upd = make_uint2(item.x | (opaque ? 0x80000000u : 0u), (uint32_t)err);  // x < 2^31 - 1
            if (one_round) s_item[tid] = upd;
            else items[base + tid] = upd;
        }
        __syncthreads();  // the next round overwrites the shared arrays
    }
    // ---- pass 2, mode 1 (zap_tex.h:764-783) of the CTA's opaque blocks, an 8-lane group per block: the CTA's list
    // entries are read 64 at a time (its next 8 rounds) and the opaque ones compacted, so every group has a block
    // while any is left. Each warp runs one mode for long stretches instead of alternating with mode 5 every round
    // (an atlas of 64x64 textures, a quarter of its blocks listed: 0.98 -> 0.80 ms per 2048x2048 encode). After a
    // single round the blocks are still in shared memory, and group g takes slot g; with one block per CTA, the
    // whole CTA ranks its partitions and group 0 fits the four best.
    const int g = tid / kBc7Group, l = tid & (kBc7Group - 1);
    const unsigned gmask = 0xFFu << (lane & ~(kBc7Group - 1));
    for (int chunk = 0; (blockIdx.x + 8 * chunk * gridDim.x) * per < n; chunk++) {  // CTA-uniform
        int total = kHardBlocks;  // one round: group g takes slot g, whose own flag decides
        if (!one_round) {
            const int it = (blockIdx.x + (8 * chunk + (tid >> 3)) * gridDim.x) * kHardBlocks + (tid & 7);
            const bool op = it < n && (items[it].x >> 31) != 0u;
            const unsigned bal = __ballot_sync(0xFFFFFFFFu, op);
            if (lane == 0) s_wcnt[warp] = __popc(bal);
            __syncthreads();
            total = s_wcnt[0] + s_wcnt[1];
            const int pos = (warp ? s_wcnt[0] : 0) + __popc(bal & ((1u << lane) - 1u));
            if (op && ZTC_IN_BOUNDS(pos, 64, 9)) s_op[pos] = it;
            __syncthreads();
        }
        for (int k = g; k - g < total; k += kHardBlocks) {  // group-uniform: rounds of one block per group
            uint2 item = make_uint2(0xFFFFFFFFu, 0u);
            if (sparse) item = s_item[0];  // CTA-uniform
            else if (one_round) item = s_item[k];
            else if (k < total) item = items[s_op[k]];
            bool go = item.x != 0xFFFFFFFFu && (item.x >> 31) != 0u;
            const int slot = sparse ? 0 : g;
            TexRef ts{s_tex[slot], 1};
            int cand[kMode1Tries];
            if (sparse) {
                if (go) cta_rank64(ts, cand, s_re, s_rp);  // every thread of the CTA
                go = go && g == 0;
            } else if (go) {
                if (!one_round) {
                    const int b = (int)(item.x & 0x7FFFFFFFu);
                    uint32_t t[16];
                    gather_block(src, b % bw, by0 + b / bw, t);
                    ts = stage_group_texels(s_tex[g], t, l, gmask);
                }
                group_rank(ts, cand, l, gmask);
            }
            int err = (int)item.y;
            uint4 blk = make_uint4(0, 0, 0, 0);
            if (go && mode1_fits(ts, cand, err, blk, l, gmask) && l == 0) put_block16(out, b0 + (size_t)(item.x & 0x7FFFFFFFu), blk);
        }
        if (!one_round) __syncthreads();  // s_op, s_wcnt and s_tex are written again by the next chunk
    }
}

// the modes-5/1 launch over a work list of at most nblocks items
cudaError_t launch_hard(const SrcU8 &src, int bw, int by0, int nblocks, const BlockOut &out, size_t b0, const uint32_t *count,
                        uint2 *items, cudaStream_t s) {
    int ctas = (nblocks + kHardBlocks - 1) / kHardBlocks;
    const int cap = ztc_sm_count() * 8;
    ctas = ctas < cap ? ctas : cap;
    bc7_hard_kernel<<<ctas, 64, 0, s>>>(src, bw, by0, out, b0, count, items);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- batched: tile queue, then one batch-wide list
// Mode 6: each CTA takes tiles of consecutive blocks of one (texture, level) from a device counter, one thread per
// block, at the plain kernel's occupancy. Blocks above SSE 64 go to one work list for the whole batch, keyed by
// their batch-wide block id (the level's first id + the block index). Modes 5 and 1 then run as one persistent
// launch of 8-lane groups over that list, so every group has a block to work on until the list is drained.
template <int CTA, int MINB>
__global__ void __launch_bounds__(CTA, MINB * 128 / CTA)
batch_bc7_mode6_kernel(const BatchLevel *__restrict__ levels, const BatchTile *__restrict__ tiles, int ntiles,
                       uint32_t *__restrict__ counter, uint32_t *__restrict__ hard_count, uint2 *__restrict__ hard_items) {
    __shared__ int s_tile;
    __shared__ uint32_t s_tex[16][CTA];  // column threadIdx.x: this thread's block
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
            const int b = tile_block(T, L.bw, j);
            uint32_t t[16];
            if (valid) {
                gather_block(src, b % L.bw, b / L.bw, t);
                #pragma unroll
                for (int i = 0; i < 16; i++) s_tex[i][threadIdx.x] = t[i];
            }
            uint4 blk;
            const int err = mode6_encode_cta<CTA, true>(valid, t, s_tex, blk);
            if (valid) store_block16(L.dst + (size_t)b * 16, blk);
            const bool hard = valid && err > 16 * 4;  // zap_tex.h:758 early exit
            const unsigned ballot = __ballot_sync(0xFFFFFFFFu, hard);
            if (ballot) {
                const int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
                uint32_t base = 0;
                if (lane == leader) base = atomicAdd(hard_count, (uint32_t)__popc(ballot));
                base = __shfl_sync(0xFFFFFFFFu, base, leader);
                if (hard) hard_items[base + __popc(ballot & ((1u << lane) - 1u))] = make_uint2(L.gbase + (uint32_t)b, (uint32_t)err);
            }
            __syncthreads();  // the next chunk overwrites s_tex
        }
    }
}

// Batched mode 5 over the batch-wide list (bases[k]: batch-wide id of the first block of BC7 level k, ascending;
// level_of[k]: its index in `levels`), laid out like the single-image kernel: a CTA of two warps takes 8 listed
// blocks at a time, warp 0 fitting their colour parts and warp 1 their alpha parts (lane = block * 4 + rotation);
// the block is written when mode 5 wins, and each opaque block goes, with its SSE after mode 5, to the mode-1 list.
__global__ void __launch_bounds__(64, ZTC_MINB_BC7_MODE5) batch_bc7_mode5_kernel(const BatchLevel *__restrict__ levels, const uint32_t *__restrict__ bases,
                                                               const int *__restrict__ level_of, int nlevels,
                                                               const uint32_t *__restrict__ count, const uint2 *__restrict__ items,
                                                               uint32_t *__restrict__ next_count, uint2 *__restrict__ next_items) {
    __shared__ uint32_t s_tex[kHardBlocks][17];
    __shared__ uint2 s_item[kHardBlocks];
    __shared__ int s_cerr[kHardBlocks][4], s_aerr[kHardBlocks][4];
    __shared__ uint32_t s_cq[kHardBlocks][4], s_cq2[kHardBlocks][4], s_ci[kHardBlocks][4], s_aq[kHardBlocks][4], s_ai[kHardBlocks][4];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = (int)*(volatile const uint32_t *)count;
    uint8_t *dst = nullptr;  // threads 0..7: the level's blocks of their item, and the block's index there
    int bidx = 0;
    for (int base = blockIdx.x * kHardBlocks; base < n; base += gridDim.x * kHardBlocks) {
        if (tid < kHardBlocks) {
            const int it = base + tid;
            uint2 item = make_uint2(0xFFFFFFFFu, 0u);
            if (it < n) {
                item = items[it];
                int lo = 0, hi = nlevels - 1;  // last level whose first id is <= the block's id
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (__ldg(bases + mid) <= item.x) lo = mid; else hi = mid - 1;
                }
                const BatchLevel L = levels[__ldg(level_of + lo)];
                bidx = (int)(item.x - __ldg(bases + lo));
                dst = L.dst;
                const SrcU8 src{L.src, L.pitch, L.w, L.h, 4, (((uintptr_t)L.src | L.pitch) & 15u) == 0};
                uint32_t t[16];
                gather_block(src, bidx % L.bw, bidx / L.bw, t);
                #pragma unroll
                for (int i = 0; i < 16; i++) s_tex[tid][i] = t[i];
            }
            s_item[tid] = item;
        }
        __syncthreads();
        {
            const int blk = lane >> 2, rot = lane & 3;
            if (s_item[blk].x != 0xFFFFFFFFu) {
                const TexRef ts{s_tex[blk], 1};
                uint32_t qw = 0, qw2 = 0, idx = 0;
                if (warp == 0) {
                    s_cerr[blk][rot] = m5_colour_lane(ts, rot, qw, qw2, idx);
                    s_cq[blk][rot] = qw; s_cq2[blk][rot] = qw2; s_ci[blk][rot] = idx;
                } else {
                    s_aerr[blk][rot] = m5_alpha_lane(ts, rot, qw, idx);
                    s_aq[blk][rot] = qw; s_ai[blk][rot] = idx;
                }
            }
        }
        __syncthreads();
        if (tid < kHardBlocks && s_item[tid].x != 0xFFFFFFFFu) {
            uint32_t key = 0xFFFFFFFFu;
            #pragma unroll
            for (int r = 0; r < 4; r++) key = min(key, ((uint32_t)(s_cerr[tid][r] + s_aerr[tid][r]) << 2) | (uint32_t)r);
            const int brot = (int)(key & 3u), best5 = (int)(key >> 2);
            uint2 item = s_item[tid];
            if (best5 < (int)item.y) {  // decoded SSE == fit SSE (see the file header)
                item.y = (uint32_t)best5;
                put_block16(BlockOut{dst, 0, 4, 0}, (size_t)bidx,
                            pack_mode5_block(brot, s_cq[tid][brot], s_cq2[tid][brot], s_ci[tid][brot], s_aq[tid][brot], s_ai[tid][brot]));
            }
            bool opaque = true;
            #pragma unroll
            for (int i = 0; i < 16; i++) opaque &= (s_tex[tid][i] >> 24) == 255u;
            if (opaque) {
                const uint32_t pos = atomicAdd(next_count, 1u);
                next_items[pos] = item;
            }
        }
        __syncthreads();  // the next round overwrites the shared arrays
    }
}

// Batched mode 1 over the list of opaque blocks that batch_bc7_mode5_kernel appended (their SSE after mode 5),
// one block per 8-lane group. Groups take one block each per round with a CTA barrier between rounds, so the warps
// of a CTA run the same part of the search together (fewer instruction-fetch stalls than groups drifting apart).
__global__ void __launch_bounds__(128, ZTC_MINB_BC7_HARD)
batch_bc7_mode1_kernel(const BatchLevel *__restrict__ levels, const uint32_t *__restrict__ bases, const int *__restrict__ level_of,
                       int nlevels, const uint32_t *__restrict__ count, const uint2 *__restrict__ items) {
    __shared__ uint32_t s_gtex[128 / kBc7Group][17];
    const int lane = threadIdx.x & 31, l = lane & (kBc7Group - 1);
    const unsigned gmask = 0xFFu << (lane & ~(kBc7Group - 1));
    const int ngroups = gridDim.x * (blockDim.x / kBc7Group);
    const int n = (int)*(volatile const uint32_t *)count;
    uint32_t *gtex = s_gtex[threadIdx.x / kBc7Group];
    const int gid = blockIdx.x * (blockDim.x / kBc7Group) + (threadIdx.x / kBc7Group);
    const int rounds = (n + ngroups - 1) / ngroups;  // the same for every warp
    for (int r = 0; r < rounds; r++) {
        __syncthreads();
        const int it = r * ngroups + gid;
        if (it < n) {
            const uint2 item = items[it];
            int lo = 0, hi = nlevels - 1;  // last level whose first id is <= the block's id
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (__ldg(bases + mid) <= item.x) lo = mid; else hi = mid - 1;
            }
            const BatchLevel L = levels[__ldg(level_of + lo)];
            const int b = (int)(item.x - __ldg(bases + lo));
            const SrcU8 src{L.src, L.pitch, L.w, L.h, 4, (((uintptr_t)L.src | L.pitch) & 15u) == 0};
            uint32_t t[16];
            gather_block(src, b % L.bw, b / L.bw, t);
            const TexRef ts = stage_group_texels(gtex, t, l, gmask);
            int err = (int)item.y;
            uint4 blk = make_uint4(0, 0, 0, 0);
            if (bc7_group_mode1(ts, err, blk, l, gmask) && l == 0) put_block16(BlockOut{L.dst, 0, 4, 0}, (size_t)b, blk);
        }
    }
}

}  // namespace ztc

cudaError_t ztc_launch_batch_bc7_mode6(int cta, int regs, int grid, const ztc::BatchLevel *levels, const ztc::BatchTile *tiles, int ntiles,
                                       uint32_t *counter, uint32_t *hard_count, uint2 *hard_items, cudaStream_t stream) {
    const void *fn = ztc_batch_bc7_kernel_fn(cta, regs);
    if (!fn) return cudaErrorInvalidValue;
    void *args[] = {(void *)&levels, (void *)&tiles, (void *)&ntiles, (void *)&counter, (void *)&hard_count, (void *)&hard_items};
    return cudaLaunchKernel(fn, dim3(grid), dim3(cta), args, 0, stream);
}

cudaError_t ztc_launch_batch_bc7_hard(int grid, const ztc::BatchLevel *levels, const uint32_t *bases, const int *level_of, int nlevels,
                                      const uint32_t *hard_count, const uint2 *hard_items, uint32_t *opaque_count, uint2 *opaque_items,
                                      cudaStream_t stream) {
    ztc::batch_bc7_mode5_kernel<<<ztc_sm_count() * 8, 64, 0, stream>>>(levels, bases, level_of, nlevels, hard_count, hard_items,
                                                                       opaque_count, opaque_items);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    ztc::batch_bc7_mode1_kernel<<<grid, 128, 0, stream>>>(levels, bases, level_of, nlevels, opaque_count, opaque_items);
    return cudaGetLastError();
}

template <int MINB>
static const void *batch_bc7_fn_cap(int cta) {
    switch (cta) {
    case 64: return (const void *)ztc::batch_bc7_mode6_kernel<64, MINB>;
    case 128: return (const void *)ztc::batch_bc7_mode6_kernel<128, MINB>;
    case 256: return (const void *)ztc::batch_bc7_mode6_kernel<256, MINB>;
    default: return nullptr;
    }
}
const void *ztc_batch_bc7_kernel_fn(int cta, int regs) {
    return regs ? batch_bc7_fn_cap<ZTC_MINB_BC7_BATCH_LOOSE>(cta) : batch_bc7_fn_cap<ZTC_MINB_BC7_MODE6>(cta);
}

const void *ztc_batch_bc7_hard_kernel_fn() { return (const void *)ztc::batch_bc7_mode1_kernel; }  // the tuned modes-5/1 grid is mode 1's

size_t ztc::bc7_scratch_bytes(size_t nblocks) { return 256 + nblocks * sizeof(uint2); }

cudaError_t ztc_launch_bc7_to(const ztc::SrcU8 &src, int by0, int nby, const ztc::BlockOut &out, size_t b0, void *scratch,
                              cudaStream_t stream) {
    int bw = (src.w + 3) / 4, nblocks = bw * nby;
    if (nblocks <= 0) return cudaSuccess;
    uint32_t *count = (uint32_t *)scratch;
    uint2 *items = (uint2 *)((uint8_t *)scratch + 256);
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    {
        ztc::TraceScope tr("bc7_mode6", stream);
        ztc::trace_units(nblocks);
        e = ztc::launch_mode6(src, bw, by0, nblocks, out, b0, count, items, stream);
        if (e != cudaSuccess) return e;  // launch_mode6 read (and cleared) the launch error; the list is not valid
    }
    ztc::TraceScope tr("bc7_modes51", stream);
    ztc::trace_units_dev(count, stream);
    return ztc::launch_hard(src, bw, by0, nblocks, out, b0, count, items, stream);
}

cudaError_t ztc_launch_bc7(const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, void *scratch, cudaStream_t stream) {
    return ztc_launch_bc7_to(src, by0, nby, ztc::BlockOut{out, 0, ZTC_FMT_BC7, 0}, 0, scratch, stream);
}

// ---------------------------------------------------------------- allocation-free BC7 entry point
// Some callers cannot allocate device memory at encode time: code running inside a real-time frame loop where an
// allocation would stall or be forbidden, engines that own a fixed GPU memory
// budget handed out up front, or plug-in hosts that give a texture tool only the buffers it is called with.
// zap_tex_cuda_bc7_encode_noalloc_dev serves them: its BC7 work list lives in the file-scope array below, sized
// for at most kNoAllocMaxBlocks 4x4 blocks (a 4096 x 4096 texture), which every GPU that loads this library holds
// until the process exits (about 8 MB). The first call on a device looks up the array's device address.
namespace ztc {
constexpr size_t kNoAllocMaxBlocks = size_t(1) << 20;
constexpr size_t kNoAllocBytes = 256 + kNoAllocMaxBlocks * sizeof(uint2);
static __device__ __align__(256) unsigned char g_bc7_noalloc_scratch[kNoAllocBytes];
}  // namespace ztc

namespace {
std::mutex g_noalloc_lock;
void *g_noalloc_addr[64];  // per device: device address of g_bc7_noalloc_scratch
}  // namespace

extern "C" __attribute__((visibility("default"))) int zap_tex_cuda_bc7_encode_noalloc_dev(const uint8_t *rgba, int w, int h,
                                                                                           size_t stride, void *out, void *stream) {
    ZTC_NVTX();
    if (!rgba || !out) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null pointer");
    if (w < 1 || h < 1 || w > (1 << 24) || h > (1 << 24)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "size out of range");
    if (stride < (size_t)w * 4) return ztc_set_error(ZTC_ERR_INVALID_ARG, "stride below 4 * width");
    if ((uintptr_t)out % 16u)
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "out must be 16-byte aligned (BC7 blocks are stored 16 bytes at a time)");
    const size_t bw = (size_t)(w + 3) / 4, bh = (size_t)(h + 3) / 4;
    if (bw * bh > ztc::kNoAllocMaxBlocks)
        return ztc_set_error(ZTC_ERR_INVALID_ARG,
                             "texture has more 4x4 blocks than the allocation-free BC7 entry point holds (1048576)");
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return ztc_set_error(ZTC_ERR_NO_DEVICE, "no CUDA device");
    }
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return ztc_set_error(ZTC_ERR_NO_DEVICE, "this build targets sm_100a");
    void *scratch = nullptr;
    {
        std::lock_guard<std::mutex> g(g_noalloc_lock);
        if (!g_noalloc_addr[dev]) {  // set-up, once per device, with that device current
            cudaError_t e = cudaGetSymbolAddress(&g_noalloc_addr[dev], ztc::g_bc7_noalloc_scratch);
            if (e != cudaSuccess) {
                g_noalloc_addr[dev] = nullptr;
                cudaGetLastError();
                return ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e));
            }
        }
        scratch = g_noalloc_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    ztc::SrcU8 src{rgba, stride, w, h, 4, (((uintptr_t)rgba | stride) & 15u) == 0};
    uint32_t *count = (uint32_t *)scratch;
    uint2 *items = (uint2 *)((uint8_t *)scratch + 256);
    const int nblocks = (int)(bw * bh);
    const ztc::BlockOut blocks{(uint8_t *)out, 0, ZTC_FMT_BC7, 0};
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), s);  // the list must start empty on every call
    if (e == cudaSuccess) e = ztc::launch_mode6(src, (int)bw, 0, nblocks, blocks, 0, count, items, s);
    if (e == cudaSuccess) e = ztc::launch_hard(src, (int)bw, 0, nblocks, blocks, 0, count, items, s);  // over the list mode 6 filled
    if (e != cudaSuccess) { cudaGetLastError(); return ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e)); }
    return ZTC_OK;
}

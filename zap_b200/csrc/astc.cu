// astc.cu - ASTC 4x4 LDR encoder (zap_tex.h:977-1342) for sm_100a, bit-exact with the reference.
//
// Kernel A, one thread per block: the three single-partition configurations (CEM 8 for opaque blocks, CEM 12
// otherwise), each a PCA start, a quantisation, a weight fit and up to three least-squares refits. Opaque blocks
// still above SSE 192 go to a work list.
// Kernel B, one 8-lane group per listed block: 2-means split, then the ~1000 usable two-partition patterns are
// scanned 8-way by Hamming distance and the top 4 by (distance, pattern order) merged across the group (the
// reference's early stop at four exact matches yields the same four); lane = (candidate, configuration) fits the
// 8 trials, and the first-best trial below the single-partition SSE is packed by the lane that found it.
// Tables the reference rebuilds on every call (zap_tex.h:1293-1305) are built once per device.
#include <cstring>

#include <cstddef>

#include "ztc_common.cuh"
#include "ztc_decode.cuh"
#include "ztc_internal.h"
#include "ztc_pca.cuh"

namespace ztc {

// ---------------------------------------------------------------- ASTC spec rules (host and device)
struct IseRange { int levels, trit, quint, bits; };
// integer-sequence range i of the ASTC spec's 21 (2, 3, 4, 5, 6, 8, 10, 12, 16, 20, ..., 192, 256 levels): after
// the first two the ranges repeat (2^(k+2) values, 5 * 2^k with a quint, 3 * 2^(k+1) with a trit), k = 0, 1, ...
ZTC_DEV IseRange ise_range(int i) {
    if (i == 0) return {2, 0, 0, 1};
    if (i == 1) return {3, 1, 0, 0};
    const int m = (i - 2) % 3, k = (i - 2) / 3;
    if (m == 0) return {1 << (k + 2), 0, 0, k + 2};
    if (m == 1) return {5 << k, 0, 1, k};
    return {3 << (k + 1), 1, 0, k + 1};
}

struct AstcCfg { int cem, wb, parts, nv, trit, quint, bits; };
struct AstcTables {
    AstcCfg cfg[8];
    uint8_t q[8][256];   // 8-bit target -> nearest colour code (first on ties)
    uint8_t uq[8][256];  // colour code -> unquantised 0..255
    uint8_t trit_code[256], quint_code[128];  // value combination -> smallest packed code
    uint8_t wq[4][32];   // weight code -> 0..64 for 2, 3, 4, 5 weight bits
    uint16_t pat_mask[1024], pat_seed[1024];
    int pat_count;
};
__constant__ AstcTables kAstc;
// the same tables in global memory: the kernels stage them into shared memory once per CTA, each thread reading
// consecutive words (coalesced loads; the constant cache would serialise the threads' different addresses)
__device__ AstcTables gAstc;

ZTC_DEV int ise_bits(const IseRange &r, int n) { return n * r.bits + (r.trit ? (8 * n + 4) / 5 : r.quint ? (7 * n + 2) / 3 : 0); }
// the largest range with at least 6 levels whose nvals values fit in avail bits (zap_tex.h:996-999)
ZTC_DEV int colour_range(int nvals, int avail) {
    for (int i = 20; i >= 4; i--) if (ise_bits(ise_range(i), nvals) <= avail) return i;
    return -1;
}
ZTC_DEV int replicate(int v, int n, int to) {
    int x = 0;
    for (int sh = to - n; sh > -n; sh -= n) x |= sh >= 0 ? v << sh : v >> -sh;
    return x & ((1 << to) - 1);
}
ZTC_DEV int colour_unquant(const IseRange &r, int v) {  // ASTC spec colour unquantisation
    if (!r.trit && !r.quint) return replicate(v, r.bits, 8);
    int n = r.bits, m = v & ((1 << n) - 1), D = v >> n;
    int a = m & 1, b = (m >> 1) & 1, c = (m >> 2) & 1, d = (m >> 3) & 1, e = (m >> 4) & 1, f = (m >> 5) & 1;
    int A = a ? 0x1FF : 0, B = 0, C = 0;
    switch (r.levels) {
    case 6: C = 204; break;
    case 10: C = 113; break;
    case 12: B = (b << 8) | (b << 4) | (b << 2) | (b << 1); C = 93; break;
    case 20: B = (b << 8) | (b << 3) | (b << 2); C = 54; break;
    case 24: B = (c << 8) | (b << 7) | (c << 3) | (b << 2) | (c << 1) | b; C = 44; break;
    case 40: B = (c << 8) | (b << 7) | (c << 2) | (b << 1) | c; C = 26; break;
    case 48: B = (d << 8) | (c << 7) | (b << 6) | (d << 2) | (c << 1) | b; C = 22; break;
    case 80: B = (d << 8) | (c << 7) | (b << 6) | (d << 1) | c; C = 13; break;
    case 96: B = (e << 8) | (d << 7) | (c << 6) | (b << 5) | (e << 1) | d; C = 11; break;
    case 160: B = (e << 8) | (d << 7) | (c << 6) | (b << 5) | e; C = 6; break;
    case 192: B = (f << 8) | (e << 7) | (d << 6) | (c << 5) | (b << 4) | f; C = 5; break;
    }
    int T = (D * C + B) ^ A;
    return (A & 0x80) | (T >> 2);
}
ZTC_DEV void trit_unpack(int T, int t[5]) {  // ASTC spec: 8 bits -> 5 trits
    int C;
    if (((T >> 2) & 7) == 7) { C = (((T >> 5) & 7) << 2) | (T & 3); t[4] = 2; t[3] = 2; }
    else {
        C = T & 31;
        if (((T >> 5) & 3) == 3) { t[4] = 2; t[3] = (T >> 7) & 1; }
        else { t[4] = (T >> 7) & 1; t[3] = (T >> 5) & 3; }
    }
    if ((C & 3) == 3) { t[2] = 2; t[1] = (C >> 4) & 1; t[0] = (((C >> 3) & 1) << 1) | (((C >> 2) & 1) & ~(C >> 3) & 1); }
    else if (((C >> 2) & 3) == 3) { t[2] = 2; t[1] = 2; t[0] = C & 3; }
    else { t[2] = (C >> 4) & 1; t[1] = (C >> 2) & 3; t[0] = (((C >> 1) & 1) << 1) | ((C & 1) & ~(C >> 1) & 1); }
}
ZTC_DEV void quint_unpack(int Q, int q[3]) {  // ASTC spec: 7 bits -> 3 quints
    if (((Q >> 1) & 3) == 3 && ((Q >> 5) & 3) == 0) {
        q[2] = ((Q & 1) << 2) | ((((Q >> 4) & 1) & ~Q & 1) << 1) | (((Q >> 3) & 1) & ~Q & 1);
        q[1] = 4; q[0] = 4;
        return;
    }
    int C;
    if (((Q >> 1) & 3) == 3) { q[2] = 4; C = (((Q >> 3) & 3) << 3) | ((~(Q >> 5) & 3) << 1) | (Q & 1); }
    else { q[2] = (Q >> 5) & 3; C = Q & 31; }
    if ((C & 7) == 5) { q[1] = 4; q[0] = (C >> 3) & 3; }
    else { q[1] = (C >> 3) & 3; q[0] = C & 7; }
}
ZTC_DEV uint32_t hash52(uint32_t p) {  // ASTC spec partition hash
    p ^= p >> 15; p -= p << 17; p += p << 7; p += p << 4; p ^= p >> 5;
    p += p << 16; p ^= p >> 7; p ^= p >> 3; p ^= p << 6; p ^= p >> 17;
    return p;
}
ZTC_DEV int astc_partition(int seed, int x, int y, int count) {  // ASTC spec partition selection, small block
    x <<= 1; y <<= 1;
    seed += (count - 1) * 1024;
    uint32_t h = hash52((uint32_t)seed);
    int s[8];
    for (int i = 0; i < 8; i++) { s[i] = (int)((h >> (4 * i)) & 15); s[i] *= s[i]; }
    int sh1, sh2;
    if (seed & 1) { sh1 = (seed & 2) ? 4 : 5; sh2 = count == 3 ? 6 : 5; }
    else { sh1 = count == 3 ? 6 : 5; sh2 = (seed & 2) ? 4 : 5; }
    for (int i = 0; i < 8; i++) s[i] >>= (i & 1) ? sh2 : sh1;
    int a = (s[0] * x + s[1] * y + (int)(h >> 14)) & 0x3F, b = (s[2] * x + s[3] * y + (int)(h >> 10)) & 0x3F;
    int c = (s[4] * x + s[5] * y + (int)(h >> 6)) & 0x3F, d = (s[6] * x + s[7] * y + (int)(h >> 2)) & 0x3F;
    if (count < 4) d = 0;
    if (count < 3) c = 0;
    return (a >= b && a >= c && a >= d) ? 0 : (b >= c && b >= d) ? 1 : c >= d ? 2 : 3;
}

ZTC_DEV int wunq(int j, int wb) {  // weight n-bit -> 0..64 (power-of-two ranges, zap_tex.h:1030)
    int x = 0;
    for (int sh = 6 - wb; sh > -wb; sh -= wb) x |= sh >= 0 ? j << sh : j >> -sh;
    x &= 63;
    return x > 32 ? x + 1 : x;
}

static void build_tables(AstcTables &T) {
    std::memset(&T, 0, sizeof T);
    for (int wb = 2; wb <= 5; wb++)
        for (int j = 0; j < (1 << wb); j++) T.wq[wb - 2][j] = (uint8_t)wunq(j, wb);
    // (CEM, weight bits, partitions) of the eight trial configurations (zap_tex.h:1298-1300)
    static const int CFG[8][3] = {{8, 4, 1}, {8, 3, 1}, {8, 5, 1}, {12, 4, 1}, {12, 3, 1}, {12, 2, 1}, {8, 3, 2}, {8, 2, 2}};
    for (int k = 0; k < 8; k++) {
        AstcCfg &c = T.cfg[k];
        c.cem = CFG[k][0]; c.wb = CFG[k][1]; c.parts = CFG[k][2]; c.nv = c.cem == 8 ? 6 : 8;
        int ri = colour_range(c.nv * c.parts, 128 - (c.parts == 1 ? 17 : 29) - 16 * c.wb);
        const IseRange r = ise_range(ri);
        c.trit = r.trit; c.quint = r.quint; c.bits = r.bits;
        for (int v = 0; v < 256; v++) T.uq[k][v] = v < r.levels ? (uint8_t)colour_unquant(r, v) : 0;
        for (int x = 0; x < 256; x++) {
            int best = 0, bd = 1 << 30;
            for (int v = 0; v < r.levels; v++) {
                int d = colour_unquant(r, v) - x;
                d = d < 0 ? -d : d;
                if (d < bd) { bd = d; best = v; }
            }
            T.q[k][x] = (uint8_t)best;
        }
    }
    for (int t = 255; t >= 0; t--) { int v[5]; trit_unpack(t, v); T.trit_code[v[0] + 3 * v[1] + 9 * v[2] + 27 * v[3] + 81 * v[4]] = (uint8_t)t; }
    for (int q = 127; q >= 0; q--) { int v[3]; quint_unpack(q, v); T.quint_code[v[0] + 5 * v[1] + 25 * v[2]] = (uint8_t)q; }
    T.pat_count = 0;
    for (int sd = 0; sd < 1024; sd++) {
        unsigned m = 0;
        for (int i = 0; i < 16; i++) m |= (unsigned)astc_partition(sd, i & 3, i >> 2, 2) << i;
        if (m && m != 0xFFFFu) { T.pat_mask[T.pat_count] = (uint16_t)m; T.pat_seed[T.pat_count++] = (uint16_t)sd; }
    }
}

cudaError_t upload_astc_tables() {
    static AstcTables T;
    static bool built = false;
    if (!built) { build_tables(T); built = true; }
    cudaError_t e = cudaMemcpyToSymbol(kAstc, &T, sizeof T);
    return e == cudaSuccess ? cudaMemcpyToSymbol(gAstc, &T, sizeof T) : e;
}

// ---------------------------------------------------------------- device pieces
struct __align__(16) AstcSmem {  // staged as 32-bit words
    uint8_t q[8][256], uq[8][256];
    AstcCfg cfg[8];
    uint8_t trit_code[256], quint_code[128];
    uint8_t wq[4][32];
};

static_assert(offsetof(AstcTables, q) % 4 == 0 && offsetof(AstcTables, trit_code) % 4 == 0 && offsetof(AstcTables, quint_code) % 4 == 0 &&
                  offsetof(AstcTables, wq) % 4 == 0 && offsetof(AstcTables, pat_mask) % 4 == 0 && offsetof(AstcTables, pat_seed) % 4 == 0 &&
                  offsetof(AstcSmem, trit_code) % 4 == 0 && offsetof(AstcSmem, quint_code) % 4 == 0 && offsetof(AstcSmem, wq) % 4 == 0,
              "the tables are staged as 32-bit words");
__device__ __forceinline__ void load_smem(AstcSmem &S) {
    const uint32_t *src = (const uint32_t *)&gAstc.q[0][0];
    uint32_t *dst = (uint32_t *)&S.q[0][0];
    for (int k = threadIdx.x; k < (int)(sizeof(S.q) + sizeof(S.uq)) / 4; k += blockDim.x) dst[k] = __ldg(src + k);
    for (int k = threadIdx.x; k < 256 / 4; k += blockDim.x) ((uint32_t *)S.trit_code)[k] = __ldg((const uint32_t *)gAstc.trit_code + k);
    for (int k = threadIdx.x; k < 128 / 4; k += blockDim.x) ((uint32_t *)S.quint_code)[k] = __ldg((const uint32_t *)gAstc.quint_code + k);
    for (int k = threadIdx.x; k < 128 / 4; k += blockDim.x) ((uint32_t *)&S.wq[0][0])[k] = __ldg((const uint32_t *)&gAstc.wq[0][0] + k);
    if (threadIdx.x < 8) S.cfg[threadIdx.x] = kAstc.cfg[threadIdx.x];
}

ZTC_DEV int astc_lerp(int a, int b, int w) { return (((a * 257) * (64 - w) + (b * 257) * w + 32) >> 6) >> 8; }
// astc_lerp over the four channels of one endpoint pair as an affine function of w: the sum inside astc_lerp is
// a * 257 * 64 + 32 + (b - a) * 257 * w, never negative, and (x >> 6) >> 8 = x >> 14, so an entry is
// (base + slope * w) >> 14 per channel, astc_lerp's value with two operations a channel
struct LerpRow {
    int base[4], slope[4];
    ZTC_DEV LerpRow(const int e0[4], const int e1[4]) {
        #pragma unroll
        for (int c = 0; c < 4; c++) { base[c] = 64 * 257 * e0[c] + 32; slope[c] = 257 * (e1[c] - e0[c]); }
    }
    ZTC_DEV uint32_t at(int w) const {
        return pack_rgba((base[0] + slope[0] * w) >> 14, (base[1] + slope[1] * w) >> 14, (base[2] + slope[2] * w) >> 14,
                         (base[3] + slope[3] * w) >> 14);
    }
};
ZTC_DEV uint32_t get8(const uint32_t a[4], int i) { return (a[i >> 2] >> (8 * (i & 3))) & 0xFFu; }
ZTC_DEV void set8(uint32_t a[4], int i, uint32_t v) {
    #pragma unroll
    for (int k = 0; k < 4; k++)
        if (k == (i >> 2)) a[k] = (a[k] & ~(0xFFu << (8 * (i & 3)))) | (v << (8 * (i & 3)));
}

// CEM 8 / 12 endpoint pair from unquantised values r0 r1 g0 g1 b0 b1 [a0 a1] (zap_tex.h:1125-1129)
ZTC_DEV void endpoint_pair(int cem, const int v[8], int e0[4], int e1[4]) {
    int a0 = cem == 12 ? v[6] : 255, a1 = cem == 12 ? v[7] : 255;
    if (v[1] + v[3] + v[5] >= v[0] + v[2] + v[4]) {
        e0[0] = v[0]; e0[1] = v[2]; e0[2] = v[4]; e0[3] = a0;
        e1[0] = v[1]; e1[1] = v[3]; e1[2] = v[5]; e1[3] = a1;
    } else {  // blue contraction
        e0[0] = (v[1] + v[5]) >> 1; e0[1] = (v[3] + v[5]) >> 1; e0[2] = v[5]; e0[3] = a1;
        e1[0] = (v[0] + v[4]) >> 1; e1[1] = (v[2] + v[4]) >> 1; e1[2] = v[4]; e1[3] = a0;
    }
}

// float endpoints -> codes + unquantised values of one partition (zap_tex.h:1183-1194)
ZTC_DEV void astc_quant(const AstcSmem &S, int cfg, int nv, const float lo[4], const float hi[4], int code[8], int uv[8]) {
    float s0 = lo[0] + lo[1] + lo[2], s1 = hi[0] + hi[1] + hi[2];
    const bool keep = s1 >= s0;
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        if (2 * k >= nv) break;
        float a = keep ? lo[k] : hi[k], b = keep ? hi[k] : lo[k];
        int x0 = clampi(f2i_x86(a + 0.5f), 0, 255), x1 = clampi(f2i_x86(b + 0.5f), 0, 255);
        code[2 * k] = S.q[cfg][x0]; code[2 * k + 1] = S.q[cfg][x1];
        uv[2 * k] = S.uq[cfg][code[2 * k]]; uv[2 * k + 1] = S.uq[cfg][code[2 * k + 1]];
    }
    if (uv[1] + uv[3] + uv[5] < uv[0] + uv[2] + uv[4]) {
        #pragma unroll
        for (int k = 0; k < 4; k++) {
            if (2 * k >= nv) break;
            int s = code[2 * k]; code[2 * k] = code[2 * k + 1]; code[2 * k + 1] = s;
            s = uv[2 * k]; uv[2 * k] = uv[2 * k + 1]; uv[2 * k + 1] = s;
        }
    }
}

// best weights for fixed endpoints (zap_tex.h:1197-1210); pm: bit i set = texel i in partition 1; cm masks the
// channels the configuration codes (alpha is left out for CEM 8); wq: weight code -> 0..64 for this weight range
template <int LMAX, int PARTS>
ZTC_DEV int astc_fit_weights(TexRef ts, uint32_t cm, int cem, int wb, const uint8_t *wq, uint32_t pm, const int uv[PARTS][8],
                             uint32_t wt[4]) {
    const int L = 1 << wb;
    uint32_t pal[PARTS][LMAX];
    int A[PARTS][LMAX];
    #pragma unroll
    for (int k = 0; k < PARTS; k++) {
        int e0[4], e1[4];
        endpoint_pair(cem, uv[k], e0, e1);
        const LerpRow row(e0, e1);
        #pragma unroll
        for (int j = 0; j < LMAX; j++) {
            if (j >= L) break;
            const uint32_t e = row.at(wq[j]) & cm;
            pal[k][j] = e;
            A[k][j] = (int)dot4(e, e) * LMAX + j;
        }
    }
    int err = 0;
    uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;  // texel i's weight enters at the top byte and is shifted down
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        const int k = PARTS == 2 ? (int)((pm >> i) & 1u) : 0;
        const uint32_t p = ts[i] & cm;
        int m = 0x7FFFFFFF;
        #pragma unroll
        for (int j = 0; j < LMAX; j++) {
            if (j >= L) break;
            uint32_t pj = PARTS == 2 ? (k ? pal[1][j] : pal[0][j]) : pal[0][j];
            int aj = PARTS == 2 ? (k ? A[PARTS - 1][j] : A[0][j]) : A[0][j];
            m = min(m, aj - 2 * LMAX * (int)dot4(p, pj));
        }
        // key = (|c|^2 - 2 p.c) * LMAX + j keeps the first best j
        const int q = m >= 0 ? m / LMAX : -((-m + LMAX - 1) / LMAX);
        err += q + (int)dot4(p, p);
        w0 = (w0 >> 8) | (w1 << 24); w1 = (w1 >> 8) | (w2 << 24); w2 = (w2 >> 8) | (w3 << 24);
        w3 = (w3 >> 8) | ((uint32_t)(m - q * LMAX) << 24);
    }
    wt[0] = w0; wt[1] = w1; wt[2] = w2; wt[3] = w3;
    return err;
}

// The same fit for one partition with the loops turned inside out: entries outer (rolled), the 16 texels inner
// (unrolled, in registers), each texel keeping its least key. The keys are unique ((|c|^2 - 2 p.c) * LMAX + j), so
// the minimum, and with it every weight and the SSE, is the one the texel-outer loop finds; the state is the texels
// and their 16 best keys instead of a palette and key table of up to 2 x 32 registers.
template <int LMAX>
ZTC_DEV int astc_fit_weights_1p(TexRef ts, uint32_t cm, int cem, int wb, const uint8_t *wq, const int uv[8], uint32_t wt[4]) {
    const int L = 1 << wb;
    int e0[4], e1[4];
    endpoint_pair(cem, uv, e0, e1);
    const LerpRow row(e0, e1);
    uint32_t p[16];
    int best[16];
    #pragma unroll
    for (int i = 0; i < 16; i++) { p[i] = ts[i] & cm; best[i] = 0x7FFFFFFF; }
    #pragma unroll 1
    for (int j = 0; j < L; j++) {
        const uint32_t e = row.at(wq[j]) & cm;
        const int a = (int)dot4(e, e) * LMAX + j;
        #pragma unroll
        for (int i = 0; i < 16; i++) best[i] = min(best[i], a - 2 * LMAX * (int)dot4(p[i], e));
    }
    int err = 0;
    uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        const int m = best[i];
        const int q = m >= 0 ? m / LMAX : -((-m + LMAX - 1) / LMAX);
        err += q + (int)dot4(p[i], p[i]);
        const uint32_t wi = (uint32_t)(m - q * LMAX);
        if (i < 4) w0 |= wi << (8 * i);
        else if (i < 8) w1 |= wi << (8 * (i - 4));
        else if (i < 12) w2 |= wi << (8 * (i - 8));
        else w3 |= wi << (8 * (i - 12));
    }
    wt[0] = w0; wt[1] = w1; wt[2] = w2; wt[3] = w3;
    return err;
}

// Passes [first, last) of one trial configuration (zap_tex.h:1212-1244): pass 0 fits the weights to the endpoint
// codes code / uv; pass k > 0 is the k-th least-squares refit on the weights wt holds, which stops at SSE 0 or at
// the first refit that does not lower the SSE (a partition whose system is singular keeps its codes). code, uv, wt
// and err take each accepted pass. Returns true when every pass ran and the SSE is still above 0, so pass `last`
// would run. One fit call site keeps the code small.
template <int LMAX, int PARTS>
ZTC_DEV bool astc_passes(TexRef ts, const AstcSmem &S, int cfg, int nc, uint32_t pm, int first, int last, int code[PARTS][8],
                         int uv[PARTS][8], uint32_t wt[4], int &err) {
    const AstcCfg &C = S.cfg[cfg];
    const int cem = C.cem, wb = C.wb, nv = C.nv;
    const uint32_t cm = nc == 4 ? 0xFFFFFFFFu : 0x00FFFFFFu;
    const uint8_t *wq = S.wq[wb - 2];
    #pragma unroll 1
    for (int it = first; it < last; it++) {
        int tc[PARTS][8], tuv[PARTS][8];
        #pragma unroll
        for (int k = 0; k < PARTS; k++)
            #pragma unroll
            for (int v = 0; v < 8; v++) { tc[k][v] = code[k][v]; tuv[k][v] = uv[k][v]; }
        if (it > 0) {
            #pragma unroll
            for (int k = 0; k < PARTS; k++) {
                const uint32_t m = PARTS == 2 ? (k ? pm : (~pm & 0xFFFFu)) : 0xFFFFu;
                float aa = 0.0f, ab = 0.0f, bb = 0.0f, sa[4] = {0.0f, 0.0f, 0.0f, 0.0f}, sb[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                uint32_t a0 = wt[0], a1 = wt[1], a2 = wt[2], a3 = wt[3];
                #pragma unroll 1
                for (int i = 0; i < 16; i++) {
                    const uint32_t wi = a0 & 0xFFu;
                    a0 = (a0 >> 8) | (a1 << 24); a1 = (a1 >> 8) | (a2 << 24); a2 = (a2 >> 8) | (a3 << 24); a3 >>= 8;
                    if (!((m >> i) & 1u)) continue;
                    const uint32_t x = ts[i];
                    float f = (float)wq[wi] / 64.0f, g = 1.0f - f;
                    aa = aa + g * g; ab = ab + g * f; bb = bb + f * f;
                    // the alpha sums are computed for CEM 8 too and then not used: each channel's sums are
                    // independent, so the RGB results are the same as a three-channel loop's
                    #pragma unroll
                    for (int c = 0; c < 4; c++) { float xc = (float)chan(x, c); sa[c] = sa[c] + g * xc; sb[c] = sb[c] + f * xc; }
                }
                float det = aa * bb - ab * ab;
                if (det < 1e-6f && det > -1e-6f) continue;
                float nlo[4], nhi[4];
                #pragma unroll
                for (int c = 0; c < 4; c++) {
                    if (c < nc) { nlo[c] = (sa[c] * bb - sb[c] * ab) / det; nhi[c] = (sb[c] * aa - sa[c] * ab) / det; }
                    else { nlo[c] = 255.0f; nhi[c] = 255.0f; }
                }
                astc_quant(S, cfg, nv, nlo, nhi, tc[k], tuv[k]);
            }
        }
        uint32_t tw[4];
        const int e = PARTS == 1 ? astc_fit_weights_1p<LMAX>(ts, cm, cem, wb, wq, tuv[0], tw)
                                 : astc_fit_weights<LMAX, PARTS>(ts, cm, cem, wb, wq, pm, tuv, tw);
        if (it > 0 && e >= err) return false;
        err = e;
        #pragma unroll
        for (int k = 0; k < 4; k++) wt[k] = tw[k];
        #pragma unroll
        for (int k = 0; k < PARTS; k++)
            #pragma unroll
            for (int v = 0; v < 8; v++) { code[k][v] = tc[k][v]; uv[k][v] = tuv[k][v]; }
        if (err <= 0) return false;
    }
    return true;
}

// a trial's starting endpoint codes (code) and unquantised values (uv) from the partitions' endpoints lo / hi
template <int LMAX, int PARTS>
ZTC_DEV void astc_trial_codes(const AstcSmem &S, int cfg, const float lo[PARTS][4], const float hi[PARTS][4], int code[PARTS][8],
                              int uv[PARTS][8]) {
    const int nv = S.cfg[cfg].nv;
    #pragma unroll
    for (int k = 0; k < PARTS; k++) {
        #pragma unroll
        for (int v = 0; v < 8; v++) { code[k][v] = 0; uv[k][v] = 0; }
        astc_quant(S, cfg, nv, lo[k], hi[k], code[k], uv[k]);
    }
}
// the codes as the block stores them: a byte per value, partition 0 first
template <int PARTS>
ZTC_DEV void astc_codes_bytes(const AstcSmem &S, int cfg, const int code[PARTS][8], uint32_t codes[4]) {
    const int nv = S.cfg[cfg].nv;
    #pragma unroll
    for (int k = 0; k < 4; k++) codes[k] = 0;
    #pragma unroll
    for (int k = 0; k < PARTS; k++)
        #pragma unroll
        for (int v = 0; v < 8; v++)
            if (v < nv) set8(codes, k * nv + v, (uint32_t)code[k][v]);
}
// one trial configuration (zap_tex.h:1212-1244) from the partitions' principal-axis endpoints lo / hi (which do
// not depend on the configuration, so callers compute them once per block and partition). nc: 3 (CEM 8) or 4
// (CEM 12) channels. codes: byte per value, partition 0 first. Returns the SSE; wt: 16 weight bytes.
template <int LMAX, int PARTS>
ZTC_DEV int astc_try(TexRef ts, const AstcSmem &S, int cfg, int nc, uint32_t pm, const float lo[PARTS][4], const float hi[PARTS][4],
                     uint32_t codes[4], uint32_t wt[4]) {
    int code[PARTS][8], uv[PARTS][8], err = 0;
    astc_trial_codes<LMAX, PARTS>(S, cfg, lo, hi, code, uv);
    astc_passes<LMAX, PARTS>(ts, S, cfg, nc, pm, 0, 4, code, uv, wt, err);
    astc_codes_bytes<PARTS>(S, cfg, code, codes);
    return err;
}

// the three single-partition trials of one block (zap_tex.h:1306-1318): CEM 8 for opaque blocks, CEM 12 otherwise.
// t: the texels in registers (for the principal axis), ts: the same texels for the rolled loops.
ZTC_DEV int astc_single_block(const uint32_t t[16], TexRef ts, const AstcSmem &S, bool opaque, int &bc, uint32_t bcodes[4],
                              uint32_t bwt[4]) {
    float lo[1][4], hi[1][4];
    if (opaque) pca_endpoints<3, 16, false>(t, 0xFFFFu, lo[0], hi[0]);
    else pca_endpoints<4, 16, false>(t, 0xFFFFu, lo[0], hi[0]);
    int best = 1 << 30;
    bc = 0;
    #pragma unroll 1
    for (int k = 0; k < 3; k++) {
        const int cfg = opaque ? k : 3 + k;
        uint32_t codes[4], wt[4];
        const int e = astc_try<32, 1>(ts, S, cfg, opaque ? 3 : 4, 0u, lo, hi, codes, wt);
        if (e < best) {
            best = e; bc = cfg;
            #pragma unroll
            for (int q = 0; q < 4; q++) { bcodes[q] = codes[q]; bwt[q] = wt[q]; }
        }
    }
    return best;
}

ZTC_DEV uint64_t bytes8(const int v[8]) {
    uint64_t r = 0;
    #pragma unroll
    for (int k = 0; k < 8; k++) r |= (uint64_t)(v[k] & 0xFF) << (8 * k);
    return r;
}
ZTC_DEV void unbytes8(uint64_t r, int v[8]) {
    #pragma unroll
    for (int k = 0; k < 8; k++) v[k] = (int)((r >> (8 * k)) & 0xFFu);
}

// The three single-partition trials for the CTA's blocks, one per thread, with each trial's third and fourth fits
// compacted: every thread runs its block's trials up to the second fit; the (block, trial) pairs whose third fit
// would run (a third of them on the test content, yet nearly every warp holds one) are listed in shared memory and
// the first threads of the CTA finish them on the owners' texels. Same result as astc_single_block. Every thread of
// the CTA calls it (it synchronises); a `valid` thread's block is in t and in column threadIdx.x of s_tex.
template <int CTA>
__device__ __forceinline__ int astc_single_cta(bool valid, const uint32_t t[16], uint32_t (*s_tex)[CTA], const AstcSmem &S, bool opaque,
                                               int &bc, uint32_t bcodes[4], uint32_t bwt[4]) {
    __shared__ uint64_t s_code[3][CTA], s_uv[3][CTA];
    __shared__ uint4 s_wt[3][CTA];
    __shared__ int s_err[3][CTA], s_wcnt[3][CTA / 32];
    __shared__ uint16_t s_list[3 * CTA];
    __shared__ uint8_t s_opq[CTA];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    float lo[1][4], hi[1][4];
    if (valid) {  // principal axis in rolled loops over the block's column of s_tex
        const TexRef own{&s_tex[0][tid], CTA};
        if (opaque) pca_endpoints<3, 1, false>(own, 0xFFFFu, lo[0], hi[0]);
        else pca_endpoints<4, 1, false>(own, 0xFFFFu, lo[0], hi[0]);
        s_opq[tid] = opaque;
    }
    unsigned mores = 0;  // bit k: trial k's third fit would run
    int total = 0;
    #pragma unroll 1
    for (int job = 0; job < 6; job++) {
        if (job == 3) {  // list the (block, trial) pairs whose third fit would run, trial by trial in thread order
            unsigned bal[3];
            #pragma unroll
            for (int k = 0; k < 3; k++) {
                bal[k] = __ballot_sync(0xFFFFFFFFu, (mores >> k) & 1u);
                if (lane == 0) s_wcnt[k][warp] = __popc(bal[k]);
            }
            __syncthreads();
            int off = 0;
            #pragma unroll
            for (int k = 0; k < 3; k++) {
                int base = 0, tk = 0;
                #pragma unroll
                for (int w = 0; w < CTA / 32; w++) { const int c = s_wcnt[k][w]; base += w < warp ? c : 0; tk += c; }
                const int pos = off + base + __popc(bal[k] & ((1u << lane) - 1u));
                if (((mores >> k) & 1u) && ZTC_IN_BOUNDS(pos, 3 * CTA, 5)) s_list[pos] = (uint16_t)((tid << 2) | k);
                off += tk;
            }
            total = off;
            __syncthreads();
        }
        int owner = tid, k = job, first = 0, last = 2;
        bool active = valid;
        if (job >= 3) {
            const int q = tid + (job - 3) * CTA;
            active = q < total;
            if (active) { owner = s_list[q] >> 2; k = s_list[q] & 3; }
            if (active && !ZTC_IN_BOUNDS(owner, CTA, 8)) active = false;
            first = 2; last = 4;
        }
        if (active) {
            const bool opq = job < 3 ? opaque : s_opq[owner] != 0;
            const int cfg = opq ? k : 3 + k;
            int code[1][8], uv[1][8], err = 0;
            uint32_t wt[4] = {0, 0, 0, 0};
            if (job < 3) {
                astc_trial_codes<32, 1>(S, cfg, lo, hi, code, uv);
            } else {
                unbytes8(s_code[k][owner], code[0]); unbytes8(s_uv[k][owner], uv[0]);
                const uint4 w = s_wt[k][owner];
                wt[0] = w.x; wt[1] = w.y; wt[2] = w.z; wt[3] = w.w;
                err = s_err[k][owner];
            }
            const int e_in = err;
            const bool more = astc_passes<32, 1>(TexRef{&s_tex[0][owner], CTA}, S, cfg, opq ? 3 : 4, 0u, first, last, code, uv, wt, err);
            if (job < 3 || err < e_in) {
                s_code[k][owner] = bytes8(code[0]); s_uv[k][owner] = bytes8(uv[0]);
                s_wt[k][owner] = make_uint4(wt[0], wt[1], wt[2], wt[3]); s_err[k][owner] = err;
            }
            if (job < 3 && more) mores |= 1u << k;
        }
    }
    __syncthreads();
    int best = 1 << 30;
    bc = 0;
    if (!valid) return best;
    #pragma unroll 1
    for (int k = 0; k < 3; k++) {  // the first trial of least SSE (zap_tex.h:1306-1318)
        const int e = s_err[k][tid];
        if (e < best) {
            best = e; bc = opaque ? k : 3 + k;
            int code[1][8];
            unbytes8(s_code[k][tid], code[0]);
            astc_codes_bytes<1>(S, bc, code, bcodes);
            const uint4 w = s_wt[k][tid];
            bwt[0] = w.x; bwt[1] = w.y; bwt[2] = w.z; bwt[3] = w.w;
        }
    }
    return best;
}

// integer-sequence encoding of n codes (zap_tex.h:1080-1095)
ZTC_DEV void ise_write(Bits128 &o, const AstcSmem &S, const AstcCfg &c, int n, const uint32_t codes[4]) {
    const int bits = c.bits, mask = (1 << bits) - 1;
    if (!c.trit && !c.quint) {
        for (int i = 0; i < n; i++) o.put(get8(codes, i) & (uint32_t)mask, bits);
        return;
    }
    const int gs = c.trit ? 5 : 3, base = c.trit ? 3 : 5;
    for (int g = 0; g < n; g += gs) {
        int cnt = min(n - g, gs), key = 0;
        for (int k = gs - 1; k >= 0; k--) key = key * base + (k < cnt ? (int)(get8(codes, g + k) >> bits) : 0);
        uint32_t X = c.trit ? S.trit_code[key] : S.quint_code[key];
        int used = 0;
        for (int k = 0; k < cnt; k++) {
            o.put(get8(codes, g + k) & (uint32_t)mask, bits);
            int xb = c.trit ? (k == 2 || k == 4 ? 1 : 2) : (k == 0 ? 3 : 2);  // packed-code bits after each value
            o.put((X >> used) & ((1u << xb) - 1u), xb);
            used += xb;
        }
    }
}

// block layout (zap_tex.h:1246-1260): mode, partitions, seed / CEM, ISE colours, weights reversed from bit 127
ZTC_DEV uint4 astc_pack(const AstcSmem &S, int cfg, int seed, const uint32_t codes[4], const uint32_t wt[4]) {
    const AstcCfg c = S.cfg[cfg];
    const int R = c.wb == 2 ? 4 : c.wb == 3 ? 7 : c.wb == 4 ? 4 : 7, H = c.wb >= 4 ? 1 : 0;
    uint32_t mode = (uint32_t)(((R >> 1) & 1) | (((R >> 2) & 1) << 1) | ((R & 1) << 4) | (2 << 5) | (H << 9));
    Bits128 o;
    o.put(mode, 11);
    o.put((uint32_t)(c.parts - 1), 2);
    if (c.parts == 2) { o.put((uint32_t)seed, 10); o.put((uint32_t)c.cem << 2, 6); }
    else o.put((uint32_t)c.cem, 4);
    ise_write(o, S, c, c.nv * c.parts, codes);
    Bits128 ws;
    for (int i = 0; i < 16; i++) ws.put(get8(wt, i), c.wb);
    // stream bit i -> block bit 127 - i
    return make_uint4(o.w[0] | brev(ws.w[3]), o.w[1] | brev(ws.w[2]), o.w[2] | brev(ws.w[1]), o.w[3] | brev(ws.w[0]));
}

__global__ void __launch_bounds__(128, ZTC_MINB_ASTC_SINGLE) astc_single_kernel(SrcU8 src, int bw, int by0, int nblocks, uint8_t *__restrict__ out,
                                                          uint32_t *__restrict__ count, uint2 *__restrict__ items) {
    __shared__ AstcSmem S;
    __shared__ uint32_t s_tex[16][128];  // column threadIdx.x: this thread's block
    load_smem(S);
    __syncthreads();
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    bool valid = b < nblocks, hard = false, opaque = true;
    uint32_t t[16];
    if (valid) {
        gather_block(src, b % bw, by0 + b / bw, t);
        #pragma unroll
        for (int i = 0; i < 16; i++) { opaque &= (t[i] >> 24) == 255u; s_tex[i][threadIdx.x] = t[i]; }
    }
    int bc = 0;
    uint32_t bcodes[4] = {0, 0, 0, 0}, bwt[4] = {0, 0, 0, 0};
    const int best = astc_single_cta<128>(valid, t, s_tex, S, opaque, bc, bcodes, bwt);
    if (valid) {
        store_block16(out + (size_t)b * 16, astc_pack(S, bc, 0, bcodes, bwt));
        hard = opaque && best > 16 * 3 * 4;  // zap_tex.h:1323
    }
    unsigned ballot = __ballot_sync(0xFFFFFFFFu, hard);
    if (ballot) {
        int lane = threadIdx.x & 31, leader = __ffs(ballot) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(count, (uint32_t)__popc(ballot));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        const int pos = (int)base + __popc(ballot & ((1u << lane) - 1u));
        if (hard && ZTC_IN_BOUNDS(pos, nblocks, 7)) items[pos] = make_uint2((uint32_t)b, (uint32_t)best);
    }
}

// 2-means on RGB (zap_tex.h:1263-1283): bit i set = texel i in cluster 1
ZTC_DEV uint32_t two_means(const uint32_t t[16]) {
    int lo = 0, hi = 0, slo = (int)(chan(t[0], 0) + chan(t[0], 1) + chan(t[0], 2)), shi = slo;
    #pragma unroll
    for (int i = 1; i < 16; i++) {
        int s = (int)(chan(t[i], 0) + chan(t[i], 1) + chan(t[i], 2));
        if (s < slo) { lo = i; slo = s; }
        if (s > shi) { hi = i; shi = s; }
    }
    float c0[3], c1[3];
    #pragma unroll
    for (int k = 0; k < 3; k++) {
        uint32_t tl = t[0], th = t[0];
        #pragma unroll
        for (int i = 1; i < 16; i++) { if (i == lo) tl = t[i]; if (i == hi) th = t[i]; }
        c0[k] = (float)chan(tl, k); c1[k] = (float)chan(th, k);
    }
    uint32_t m = 0;
    for (int it = 0; it < 4; it++) {
        float s0[3] = {0, 0, 0}, s1[3] = {0, 0, 0};
        int n0 = 0, n1 = 0;
        m = 0;
        #pragma unroll
        for (int i = 0; i < 16; i++) {
            float d0 = 0.0f, d1 = 0.0f;
            #pragma unroll
            for (int k = 0; k < 3; k++) {
                float x = (float)chan(t[i], k), a = x - c0[k], b = x - c1[k];
                d0 = d0 + a * a; d1 = d1 + b * b;
            }
            bool s = d1 < d0;
            m |= (uint32_t)s << i;
            #pragma unroll
            for (int k = 0; k < 3; k++) {
                float x = (float)chan(t[i], k);
                if (s) s1[k] = s1[k] + x; else s0[k] = s0[k] + x;
            }
            n1 += s; n0 += !s;
        }
        #pragma unroll
        for (int k = 0; k < 3; k++) {
            if (n0) c0[k] = s0[k] / (float)n0;
            if (n1) c1[k] = s1[k] / (float)n1;
        }
    }
    return m;
}

constexpr int kAstcGroup = 8;

__global__ void __launch_bounds__(128) astc_two_part_kernel(SrcU8 src, int bw, int by0, uint8_t *__restrict__ out,
                                                            const uint32_t *__restrict__ count, const uint2 *__restrict__ items) {
    __shared__ AstcSmem S;
    __shared__ __align__(16) uint16_t pmask[1024], pseed[1024];  // staged as 32-bit words
    __shared__ uint32_t s_tex[128 / kAstcGroup][17];  // per group: its block's texels (padded: no bank conflicts)
    // listed blocks go to the CTAs in turn (group g of CTA c takes items c, c + grid, ... of its share), so a short
    // list spreads over every SM, and CTAs with nothing to do leave before staging the tables
    const int n = (int)*(volatile const uint32_t *)count;
    if ((int)blockIdx.x >= n) return;
    load_smem(S);
    const int npat = kAstc.pat_count;
    for (int k = threadIdx.x; k < npat / 2; k += blockDim.x) {
        ((uint32_t *)pmask)[k] = __ldg((const uint32_t *)gAstc.pat_mask + k);
        ((uint32_t *)pseed)[k] = __ldg((const uint32_t *)gAstc.pat_seed + k);
    }
    if ((npat & 1) && threadIdx.x == 0) { pmask[npat - 1] = gAstc.pat_mask[npat - 1]; pseed[npat - 1] = gAstc.pat_seed[npat - 1]; }
    __syncthreads();
    const int lane = threadIdx.x & 31, l = lane & (kAstcGroup - 1);
    const unsigned gmask = 0xFFu << (lane & ~(kAstcGroup - 1));
    const int ngroups = gridDim.x * (blockDim.x / kAstcGroup);
    uint32_t *gtex = s_tex[threadIdx.x / kAstcGroup];
    for (int it = (threadIdx.x / kAstcGroup) * gridDim.x + blockIdx.x; it < n; it += ngroups) {
        const uint2 item = items[it];
        const int b = (int)item.x, best = (int)item.y;
        uint32_t t[16];
        gather_block(src, b % bw, by0 + b / bw, t);
        __syncwarp(gmask);  // the group's reads of the previous block are done
        #pragma unroll
        for (int i = 0; i < 16; i++)
            if ((i & (kAstcGroup - 1)) == l) gtex[i] = t[i];
        __syncwarp(gmask);
        const uint32_t km = two_means(t);
        // local top 4 by (distance, pattern order) over patterns l, l + 8, ...
        int cd[4] = {99, 99, 99, 99}, cp[4] = {1 << 20, 1 << 20, 1 << 20, 1 << 20};
        for (int pi = l; pi < npat; pi += kAstcGroup) {
            int dd = __popc((uint32_t)pmask[pi] ^ km), dist = min(dd, 16 - dd);
            if (dist < cd[3]) {
                int pos = 3;
                #pragma unroll
                for (int j = 2; j >= 0; j--) if (dist < cd[j]) pos = j;
                #pragma unroll
                for (int j = 3; j > 0; j--) if (j > pos) { cd[j] = cd[j - 1]; cp[j] = cp[j - 1]; }
                #pragma unroll
                for (int j = 0; j < 4; j++) if (j == pos) { cd[j] = dist; cp[j] = pi; }
            }
        }
        int cand[4];
        #pragma unroll
        for (int j = 0; j < 4; j++) {  // group-wide (distance, pattern) minimum, owner pops
            uint32_t key = ((uint32_t)cd[0] << 21) | (uint32_t)cp[0];
            #pragma unroll
            for (int m = 1; m < kAstcGroup; m <<= 1) key = min(key, __shfl_xor_sync(gmask, key, m, kAstcGroup));
            int p = (int)(key & 0x1FFFFFu);
            cand[j] = (key >> 21) < 99 ? p : -1;
            if (cand[j] >= 0 && (p & (kAstcGroup - 1)) == l) {
                #pragma unroll
                for (int s = 0; s < 3; s++) { cd[s] = cd[s + 1]; cp[s] = cp[s + 1]; }
                cd[3] = 99; cp[3] = 1 << 20;
            }
        }
        // lane = candidate * 2 + configuration (6: 3 weight bits, 7: 2 weight bits)
        const int j = l >> 1, cfg = 6 + (l & 1);
        int pj = -1;
        #pragma unroll
        for (int k = 0; k < 4; k++) if (k == j) pj = cand[k];
        uint32_t codes[4] = {0, 0, 0, 0}, wt[4] = {0, 0, 0, 0};
        int e = 1 << 30;
        if (pj >= 0) {
            const uint32_t pm = pmask[pj];
            float lo[2][4], hi[2][4];
            #pragma unroll
            for (int k = 0; k < 2; k++) {
                uint32_t m = k ? pm : (~pm & 0xFFFFu);
                if (!m) m = 1u;  // empty partition: the reference fits texel 0
                pca_endpoints<3, 16, false>(t, m, lo[k], hi[k]);
            }
            e = astc_try<8, 2>(TexRef{gtex, 1}, S, cfg, 3, pm, lo, hi, codes, wt);
        }
        uint32_t key = (pj >= 0 && e < best) ? (((uint32_t)e << 3) | (uint32_t)l) : 0xFFFFFFFFu;
        #pragma unroll
        for (int m = 1; m < kAstcGroup; m <<= 1) key = min(key, __shfl_xor_sync(gmask, key, m, kAstcGroup));
        if (key != 0xFFFFFFFFu && (int)(key & 7u) == l) store_block16(out + (size_t)b * 16, astc_pack(S, cfg, pseed[pj], codes, wt));
    }
}

// ---------------------------------------------------------------- decoder (zap_tex.h:1135-1168, :1344-1356)
// The blocks the reference decodes: void-extent blocks, and 4x4 weight grids with a power-of-two weight range and
// one or two partitions sharing CEM 8 or 12. Any other block decodes to magenta (255, 0, 255, 255), as there.
ZTC_DEV uint32_t take_bits(const uint32_t w[4], int &pos, int n) {  // LSB-first, n <= 16 (zap__bits)
    const uint32_t v = n ? get_bits128(w, pos, n) : 0u;
    pos += n;
    return v;
}
ZTC_DEV uint32_t bit_at(const uint32_t w[4], int p) {
    const uint32_t x = p < 32 ? w[0] : p < 64 ? w[1] : p < 96 ? w[2] : w[3];
    return (x >> (p & 31)) & 1u;
}
ZTC_DEV void astc_decode_block(const uint32_t w[4], uint32_t px[16]) {
    #pragma unroll
    for (int i = 0; i < 16; i++) px[i] = 0xFFFF00FFu;  // magenta
    int pos = 0;
    const int mode = (int)take_bits(w, pos, 11);
    if ((mode & 0x1FF) == 0x1FC) {  // void extent: one colour, 16-bit UNORM RGBA at bits 64..127
        uint32_t c = 0;
        #pragma unroll
        for (int k = 0; k < 4; k++) c |= (get_bits128(w, 64 + 16 * k, 16) >> 8) << (8 * k);
        #pragma unroll
        for (int i = 0; i < 16; i++) px[i] = c;
        return;
    }
    const int R = ((mode & 1) << 1) | (((mode >> 1) & 1) << 2) | ((mode >> 4) & 1), H = (mode >> 9) & 1;
    if (!(mode & 3) || ((mode >> 2) & 3) || ((mode >> 5) & 3) != 2 || ((mode >> 7) & 3) || ((mode >> 10) & 1)) return;
    // weight levels (R, H): {-, -, 2, 3, 4, 5, 6, 8} and {-, -, 10, 12, 16, 20, 24, 32}; only powers of two decode
    const int wb = !H ? (R == 2 ? 1 : R == 4 ? 2 : R == 7 ? 3 : 0) : (R == 4 ? 4 : R == 7 ? 5 : 0);
    const int parts = (int)take_bits(w, pos, 2) + 1;
    if (!wb || parts > 2) return;
    int seed = 0, cem;
    if (parts == 2) {
        seed = (int)take_bits(w, pos, 10);
        const int cf = (int)take_bits(w, pos, 6);
        if (cf & 3) return;  // both partitions must use the same endpoint mode
        cem = cf >> 2;
    } else {
        cem = (int)take_bits(w, pos, 4);
    }
    const int nv = cem == 8 ? 6 : cem == 12 ? 8 : 0, n = nv * parts;
    if (!nv) return;
    const int ri = colour_range(n, 128 - pos - 16 * wb);
    if (ri < 0) return;
    const IseRange r = ise_range(ri);
    int v[16];
    const int gs = r.trit ? 5 : r.quint ? 3 : 1;
    for (int g = 0; g < n; g += gs) {  // integer-sequence decode (zap__ise_get, zap_tex.h:1065-1078)
        const int cnt = min(n - g, gs);
        int m[5] = {0, 0, 0, 0, 0}, t[5] = {0, 0, 0, 0, 0}, X = 0, xp = 0;
        for (int k = 0; k < cnt; k++) {
            m[k] = (int)take_bits(w, pos, r.bits);
            if (gs > 1) {
                const int xb = r.trit ? ((k == 2 || k == 4) ? 1 : 2) : (k == 0 ? 3 : 2);  // packed-code bits after value k
                X |= (int)take_bits(w, pos, xb) << xp;
                xp += xb;
            }
        }
        if (r.trit) trit_unpack(X, t);
        else if (r.quint) quint_unpack(X, t);
        for (int k = 0; k < cnt; k++) v[g + k] = colour_unquant(r, gs > 1 ? (t[k] << r.bits) | m[k] : m[k]);
    }
    int e0[2][4], e1[2][4];
    for (int k = 0; k < parts; k++) endpoint_pair(cem, v + k * nv, e0[k], e1[k]);
    #pragma unroll 1
    for (int i = 0; i < 16; i++) {
        const int k = parts == 2 ? astc_partition(seed, i & 3, i >> 2, 2) : 0;
        int wt = 0;
        for (int j = 0; j < wb; j++) wt |= (int)bit_at(w, 127 - (i * wb + j)) << j;  // weights run down from bit 127
        wt = wunq(wt, wb);
        const int *a = k ? e0[1] : e0[0], *b = k ? e1[1] : e1[0];
        px[i] = pack_rgba(astc_lerp(a[0], b[0], wt), astc_lerp(a[1], b[1], wt), astc_lerp(a[2], b[2], wt), astc_lerp(a[3], b[3], wt));
    }
}

__global__ void __launch_bounds__(128) astc_decode_kernel(const uint8_t *__restrict__ bc, int w, int h, uint8_t *__restrict__ out,
                                                          size_t stride) {
    const int bw = (w + 3) / 4;
    const long nblocks = (long)bw * ((h + 3) / 4), b = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const uint4 q = __ldg((const uint4 *)(bc + (size_t)b * 16));
    const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
    uint32_t px[16];
    astc_decode_block(wd, px);
    const bool vec = (((uintptr_t)out | stride) & 15u) == 0, aligned4 = (((uintptr_t)out | stride) & 3u) == 0;
    dec::store_block_rgba8(out, stride, w, h, (int)(b % bw), (int)(b / bw), px, vec, aligned4);
}

}  // namespace ztc

// zap_astc_decode (zap_tex.h:1344-1356) into device memory; bc must be 16-byte aligned
cudaError_t ztc_launch_astc_decode(const uint8_t *bc, int w, int h, uint8_t *out, size_t stride, cudaStream_t stream) {
    const long nblocks = (long)((w + 3) / 4) * ((h + 3) / 4);
    if (nblocks <= 0) return cudaSuccess;
    ztc::TraceScope tr("astc_decode", stream);
    ztc::trace_units(nblocks);
    ztc::astc_decode_kernel<<<(unsigned)((nblocks + 127) / 128), 128, 0, stream>>>(bc, w, h, out, stride);
    return cudaGetLastError();
}

size_t ztc::astc_scratch_bytes(size_t nblocks) { return 256 + nblocks * sizeof(uint2); }

cudaError_t ztc_launch_astc(const ztc::SrcU8 &src, int by0, int nby, uint8_t *out, void *scratch, cudaStream_t stream) {
    int bw = (src.w + 3) / 4, nblocks = bw * nby;
    if (nblocks <= 0) return cudaSuccess;
    uint32_t *count = (uint32_t *)scratch;
    uint2 *items = (uint2 *)((uint8_t *)scratch + 256);
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(uint32_t), stream);
    if (e != cudaSuccess) return e;
    {
        ztc::TraceScope tr("astc_single", stream);
        ztc::trace_units(nblocks);
        ztc::astc_single_kernel<<<(nblocks + 127) / 128, 128, 0, stream>>>(src, bw, by0, nblocks, out, count, items);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int groups_per_cta = 128 / ztc::kAstcGroup, ctas = (nblocks + groups_per_cta - 1) / groups_per_cta;
    ctas = ctas < sms * 8 ? ctas : sms * 8;
    ztc::TraceScope tr("astc_two_part", stream);
    ztc::trace_units_dev(count, stream);
    ztc::astc_two_part_kernel<<<ctas, 128, 0, stream>>>(src, bw, by0, out, count, items);
    return cudaGetLastError();
}

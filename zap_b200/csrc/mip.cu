// mip.cu - 2x2 box-filter mip generator (zap_tex.h:1358-1469), bit-exact, HBM-bound.
//
// RGBA8: with srgb, RGB goes through the sRGB->linear table, the four values are summed left to right and scaled
// by 0.25f, and the result maps back to sRGB as the first k whose threshold exceeds it (the reference's binary
// search; here a scan from a per-bucket start, below). Alpha (and RGB without srgb) is (a + b + c + d + 2) >> 2.
// Odd sizes drop the last row / column.
// The fast path gives each thread two output texels: one 16-byte load from each of the two source rows and one
// 8-byte store; edge and unaligned texels take a clamped scalar path.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "ztc_common.cuh"
#include "ztc_internal.h"

namespace ztc {

__device__ SrgbTables gSrgb;  // staged into shared memory by each CTA (coalesced loads)

// the bucket of a linear value: 0 below 2^-16 (and for negative values), else its exponent and top 6 mantissa bits
ZTC_DEV int srgb_bucket(float v) {
    const uint32_t u = f_as_u(v);
    if (u < 0x37800000u || (u & 0x80000000u)) return 0;
    const int q = (int)(u >> 17) - (0x37800000 >> 17);
    return q < kSrgbBuckets - 1 ? q : kSrgbBuckets - 1;
}
// first k with v < thr[k] (zap_tex.h:1429-1433), 255 when there is none: the reference's binary search finds it in
// eight steps; here the scan starts at the bucket's lower bound, one to three steps for the mip generator's values
ZTC_DEV uint32_t lin_to_srgb(const float *thr, const uint8_t *bucket, float v) {
    int k = bucket[srgb_bucket(v)];
    while (k < 255 && !(v < thr[k])) k++;
    return (uint32_t)k;
}

ZTC_DEV uint32_t box4(uint32_t a, uint32_t b, uint32_t c, uint32_t d, bool srgb, const SrgbTables &T) {
    uint32_t o = 0;
    #pragma unroll
    for (int k = 0; k < 4; k++) {
        uint32_t v0 = chan(a, k), v1 = chan(b, k), v2 = chan(c, k), v3 = chan(d, k), r;
        if (srgb && k < 3) r = lin_to_srgb(T.thr, T.bucket, (T.lin[v0] + T.lin[v1] + T.lin[v2] + T.lin[v3]) * 0.25f);
        else r = (v0 + v1 + v2 + v3 + 2) >> 2;
        o |= r << (8 * k);
    }
    return o;
}

// every thread of the CTA calls it: the tables from global memory into shared memory, 32-bit words
__device__ __forceinline__ void stage_srgb(SrgbTables &S, const SrgbTables *src) {
    static_assert(sizeof(SrgbTables) % 4 == 0, "staged as 32-bit words");
    const uint32_t *g = (const uint32_t *)src;
    uint32_t *d = (uint32_t *)&S;
    for (int k = threadIdx.x; k < (int)(sizeof(SrgbTables) / 4); k += blockDim.x) d[k] = __ldg(g + k);
    __syncthreads();
}

ZTC_DEV uint32_t ld_texel(const uint8_t *p) {
    if ((((uintptr_t)p) & 3u) == 0) return ldg((const uint32_t *)p);
    return (uint32_t)ldg(p) | ((uint32_t)ldg(p + 1) << 8) | ((uint32_t)ldg(p + 2) << 16) | ((uint32_t)ldg(p + 3) << 24);
}
ZTC_DEV void st_texel(uint8_t *p, uint32_t v) {
    if ((((uintptr_t)p) & 3u) == 0) { *(uint32_t *)p = v; return; }
    p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}

__global__ void __launch_bounds__(256) mip_rgba8_kernel(const uint8_t *__restrict__ src, int w, int h, size_t stride, int srgb,
                                                        uint8_t *__restrict__ dst, size_t dst_stride, int nw, int nh, int vec) {
    __shared__ SrgbTables S;
    if (srgb) stage_srgb(S, &gSrgb);
    const int pairs = (nw + 1) >> 1;
    const long total = (long)pairs * nh;
    for (long id = (long)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (long)gridDim.x * blockDim.x) {
        int y = (int)(id / pairs), xp = (int)(id % pairs), x = 2 * xp;
        int y0 = min(2 * y, h - 1), y1 = min(2 * y + 1, h - 1);
        const uint8_t *r0 = src + (size_t)y0 * stride, *r1 = src + (size_t)y1 * stride;
        uint8_t *o = dst + (size_t)y * dst_stride + (size_t)x * 4;
        if (vec && 2 * x + 3 < w && x + 1 < nw) {
            uint4 a = __ldg((const uint4 *)(r0 + (size_t)x * 8)), b = __ldg((const uint4 *)(r1 + (size_t)x * 8));
            uint32_t o0 = box4(a.x, a.y, b.x, b.y, srgb, S), o1 = box4(a.z, a.w, b.z, b.w, srgb, S);
            *(uint2 *)o = make_uint2(o0, o1);
        } else {
            for (int k = 0; k < 2 && x + k < nw; k++) {
                int xx = x + k, x0 = min(2 * xx, w - 1), x1 = min(2 * xx + 1, w - 1);
                uint32_t v = box4(ld_texel(r0 + (size_t)x0 * 4), ld_texel(r0 + (size_t)x1 * 4), ld_texel(r1 + (size_t)x0 * 4),
                                  ld_texel(r1 + (size_t)x1 * 4), srgb, S);
                st_texel(o + (size_t)k * 4, v);
            }
        }
    }
}

// float RGBA (linear): 0.25f * (a + b + c + d) per channel (zap_tex.h:1460-1469)
__global__ void __launch_bounds__(256) mip_f32_kernel(const float *__restrict__ src, int w, int h, size_t stride,
                                                      float *__restrict__ dst, size_t dst_stride, int nw, int nh, int vec) {
    const long total = (long)nw * nh;
    for (long id = (long)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += (long)gridDim.x * blockDim.x) {
        int y = (int)(id / nw), x = (int)(id % nw);
        int x0 = min(2 * x, w - 1), x1 = min(2 * x + 1, w - 1), y0 = min(2 * y, h - 1), y1 = min(2 * y + 1, h - 1);
        const float *a = src + (size_t)y0 * stride + (size_t)x0 * 4, *b = src + (size_t)y0 * stride + (size_t)x1 * 4;
        const float *c = src + (size_t)y1 * stride + (size_t)x0 * 4, *d = src + (size_t)y1 * stride + (size_t)x1 * 4;
        float *o = dst + (size_t)y * dst_stride + (size_t)x * 4;
        if (vec) {
            float4 A = __ldg((const float4 *)a), B = __ldg((const float4 *)b), C = __ldg((const float4 *)c), D = __ldg((const float4 *)d);
            *(float4 *)o = make_float4(0.25f * (A.x + B.x + C.x + D.x), 0.25f * (A.y + B.y + C.y + D.y),
                                       0.25f * (A.z + B.z + C.z + D.z), 0.25f * (A.w + B.w + C.w + D.w));
        } else {
            #pragma unroll
            for (int k = 0; k < 4; k++) o[k] = 0.25f * (__ldg(a + k) + __ldg(b + k) + __ldg(c + k) + __ldg(d + k));
        }
    }
}

// The reference's sRGB constants are the double-precision transfer function printed with 9 significant digits
// and read back as float (checked bit for bit against the reference's tables by the test suite).
static float srgb_to_linear_9g(double c) {
    double lin = c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
    char buf[64];
    std::snprintf(buf, sizeof buf, "%.9g", lin);
    return std::strtof(buf, nullptr);
}

void srgb_tables_host(SrgbTables &t) {
    for (int k = 0; k < 256; k++) t.lin[k] = srgb_to_linear_9g(k / 255.0);
    for (int k = 0; k < 255; k++) t.thr[k] = srgb_to_linear_9g((k + 0.5) / 255.0);
    t.thr[255] = INFINITY;
    for (int q = 0; q < kSrgbBuckets; q++) {  // the answer at the bucket's lowest value (0 for bucket 0)
        uint32_t u = q ? (uint32_t)(q + (0x37800000 >> 17)) << 17 : 0u;
        float lo;
        std::memcpy(&lo, &u, 4);
        int k = 0;
        while (k < 255 && !(lo < t.thr[k])) k++;
        t.bucket[q] = (uint8_t)k;
    }
}

cudaError_t upload_mip_tables() {
    SrgbTables T;
    srgb_tables_host(T);
    return cudaMemcpyToSymbol(gSrgb, &T, sizeof T);
}

static int grid_for(long work, int threads) {
    long g = (work + threads - 1) / threads;
    return (int)(g < 148L * 32 ? (g < 1 ? 1 : g) : 148L * 32);
}

}  // namespace ztc

cudaError_t ztc_launch_mip(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride,
                           cudaStream_t stream) {
    int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    int vec = ((((uintptr_t)src) | stride) & 15u) == 0 && ((((uintptr_t)dst) | dst_stride) & 7u) == 0;
    long work = (long)((nw + 1) / 2) * nh;
    ztc::TraceScope tr("mip_rgba8", stream);
    ztc::trace_units((long)nw * nh);
    ztc::mip_rgba8_kernel<<<ztc::grid_for(work, 256), 256, 0, stream>>>(src, w, h, stride, srgb ? 1 : 0, dst, dst_stride, nw, nh, vec);
    return cudaGetLastError();
}

cudaError_t ztc_launch_mip_f(const float *src, int w, int h, size_t stride, float *dst, size_t dst_stride, cudaStream_t stream) {
    int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    int vec = ((((uintptr_t)src) | (stride * 4)) & 15u) == 0 && ((((uintptr_t)dst) | (dst_stride * 4)) & 15u) == 0;
    long work = (long)nw * nh;
    ztc::TraceScope tr("mip_f32", stream);
    ztc::trace_units((long)nw * nh);
    ztc::mip_f32_kernel<<<ztc::grid_for(work, 256), 256, 0, stream>>>(src, w, h, stride, dst, dst_stride, nw, nh, vec);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- batched: one launch per mip depth, all textures
namespace ztc {
__global__ void __launch_bounds__(256) batch_mip_kernel(const BatchMip *__restrict__ mips, const BatchMipTile *__restrict__ tiles, int ntiles,
                                                        const SrgbTables *__restrict__ tables) {
    __shared__ SrgbTables S;
    stage_srgb(S, tables);
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const BatchMipTile T = tiles[tile];
        if ((int)threadIdx.x >= T.count) continue;
        const BatchMip M = mips[T.mip];
        const int pairs = (M.nw + 1) >> 1, id = T.first + (int)threadIdx.x;
        const int y = id / pairs, x = 2 * (id % pairs);
        const int y0 = min(2 * y, M.h - 1), y1 = min(2 * y + 1, M.h - 1);
        const uint8_t *r0 = M.src + (size_t)y0 * M.src_pitch, *r1 = M.src + (size_t)y1 * M.src_pitch;
        uint8_t *o = M.dst + (size_t)y * M.dst_pitch + (size_t)x * 4;
        const bool vec = ((((uintptr_t)M.src) | M.src_pitch) & 15u) == 0 && ((((uintptr_t)M.dst) | M.dst_pitch) & 7u) == 0;
        if (vec && 2 * x + 3 < M.w && x + 1 < M.nw) {
            uint4 a = ldg((const uint4 *)(r0 + (size_t)x * 8)), b = ldg((const uint4 *)(r1 + (size_t)x * 8));
            *(uint2 *)o = make_uint2(box4(a.x, a.y, b.x, b.y, M.srgb, S), box4(a.z, a.w, b.z, b.w, M.srgb, S));
        } else {
            for (int k = 0; k < 2 && x + k < M.nw; k++) {
                int xx = x + k, x0 = min(2 * xx, M.w - 1), x1 = min(2 * xx + 1, M.w - 1);
                st_texel(o + (size_t)k * 4, box4(ld_texel(r0 + (size_t)x0 * 4), ld_texel(r0 + (size_t)x1 * 4), ld_texel(r1 + (size_t)x0 * 4),
                                                 ld_texel(r1 + (size_t)x1 * 4), M.srgb != 0, S));
            }
        }
    }
}
}  // namespace ztc

const void *ztc_batch_mip_kernel_fn() { return (const void *)ztc::batch_mip_kernel; }

cudaError_t ztc_launch_batch_mip(int grid, const ztc::BatchMip *mips, const ztc::BatchMipTile *tiles, int ntiles, const ztc::SrgbTables *srgb_tables,
                                 cudaStream_t stream) {
    if (ntiles <= 0) return cudaSuccess;
    ztc::batch_mip_kernel<<<grid, 256, 0, stream>>>(mips, tiles, ntiles, srgb_tables);
    return cudaGetLastError();
}

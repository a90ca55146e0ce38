// adjoint.cu - differentiable palette decode and gradient endpoint refinement (no reference counterpart).
//
// With a block's indices held fixed, the BCn palette decode is linear in the endpoints:
//   decoded_i = a_i * e0 + (1 - a_i) * e1
// with a_i = {1, 0, 2/3, 1/3}[idx_i] for BC1 (4-colour order) and a_i = 1 - w4(idx_i) / 64 for BC7 mode 6
// (the continuous form of the integer palettes of zap_tex.h:52-62 and :538-542; endpoints in 8-bit units).
// Its adjoint maps an upstream gradient on the decoded texels to the endpoints:
//   dL/de0 = sum_i a_i g_i,   dL/de1 = sum_i (1 - a_i) g_i.
// zap_tex_cuda_refine_dev runs, per block, 8 Adam steps on the block's MSE through that adjoint, requantises the
// endpoints (565 for BC1; 7 bits + best p-bit per endpoint for BC7 mode 6), re-fits the indices, and keeps the new
// block only if its true squared error is lower than the encoder's. BC7 blocks in modes other than 6 are left as
// they are (their adjoint is reported as zero).
#include <string>

#include "../../include/zap_tex_cuda.h"
#include "ztc_common.cuh"
#include "ztc_decode.cuh"
#include "ztc_internal.h"

namespace ztc {

// per-texel weight of endpoint 0 and channel count; returns false for blocks the adjoint does not cover
ZTC_DEV bool block_weights(int fmt, const uint8_t *blk, float a[16], int &nc) {
    if (fmt == ZTC_FMT_BC1) {
        uint2 v = *(const uint2 *)blk;
        uint32_t c0 = v.x & 0xFFFFu, c1 = v.x >> 16;
        nc = 3;
        #pragma unroll
        for (int i = 0; i < 16; i++) {
            uint32_t k = (v.y >> (2 * i)) & 3u;
            if (c0 <= c1) k = k == 1 ? 1u : 0u;  // solid / 3-colour blocks: our encoder only emits index 0 there
            a[i] = k == 0 ? 1.0f : k == 1 ? 0.0f : k == 2 ? 2.0f / 3.0f : 1.0f / 3.0f;
        }
        return true;
    }
    uint4 v = *(const uint4 *)blk;
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    nc = 4;
    if ((w[0] & 0x7Fu) != 0x40u) {  // not mode 6
        #pragma unroll
        for (int i = 0; i < 16; i++) a[i] = 0.0f;
        return false;
    }
    #pragma unroll
    for (int i = 0; i < 16; i++) {
        int idx = i == 0 ? (int)get_bits128(w, 65, 3) : (int)get_bits128(w, 68 + 4 * (i - 1), 4);
        a[i] = 1.0f - (float)w4(idx) / 64.0f;
    }
    return true;
}

// expanded 8-bit endpoints of a block as floats [2][4]
ZTC_DEV void block_endpoints(int fmt, const uint8_t *blk, float e[2][4]) {
    if (fmt == ZTC_FMT_BC1) {
        uint2 v = *(const uint2 *)blk;
        for (int k = 0; k < 2; k++) {
            uint32_t c = k ? (v.x >> 16) : (v.x & 0xFFFFu);
            int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
            e[k][0] = (float)((R << 3) | (R >> 2)); e[k][1] = (float)((G << 2) | (G >> 4)); e[k][2] = (float)((B << 3) | (B >> 2));
            e[k][3] = 255.0f;
        }
        return;
    }
    uint4 v = *(const uint4 *)blk;
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    if ((w[0] & 0x7Fu) != 0x40u) {
        for (int k = 0; k < 2; k++) for (int c = 0; c < 4; c++) e[k][c] = 0.0f;
        return;
    }
    for (int c = 0; c < 4; c++)
        for (int k = 0; k < 2; k++) {
            int q = (int)get_bits128(w, 7 + 14 * c + 7 * k, 7), p = (int)get_bits128(w, 63 + k, 1);
            e[k][c] = (float)((q << 1) | p);
        }
}

__global__ void endpoints_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, float *__restrict__ ep) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float e[2][4];
    block_endpoints(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), e);
    for (int k = 0; k < 2; k++) for (int c = 0; c < 4; c++) ep[(size_t)b * 8 + 4 * k + c] = e[k][c];
}

__global__ void decode_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, const float *__restrict__ ep, float *__restrict__ out) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float a[16];
    int nc;
    const bool covered = block_weights(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), a, nc);
    const float *e = ep + (size_t)b * 8;
    for (int i = 0; i < 16; i++)
        for (int c = 0; c < 4; c++)
            out[((size_t)b * 16 + i) * 4 + c] = (covered && c < nc) ? a[i] * e[c] + (1.0f - a[i]) * e[4 + c] : 0.0f;
}

__global__ void adjoint_kernel(int fmt, const uint8_t *__restrict__ blocks, int n, const float *__restrict__ g, float *__restrict__ ge) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n) return;
    float a[16];
    int nc;
    const bool covered = block_weights(fmt, blocks + (size_t)b * (fmt == ZTC_FMT_BC1 ? 8 : 16), a, nc);
    float g0[4] = {0, 0, 0, 0}, g1[4] = {0, 0, 0, 0};
    for (int i = 0; i < 16; i++)
        for (int c = 0; c < 4; c++) {
            float gi = (covered && c < nc) ? g[((size_t)b * 16 + i) * 4 + c] : 0.0f;
            g0[c] += a[i] * gi;
            g1[c] += (1.0f - a[i]) * gi;
        }
    for (int c = 0; c < 4; c++) { ge[(size_t)b * 8 + c] = g0[c]; ge[(size_t)b * 8 + 4 + c] = g1[c]; }
}

// ---------------------------------------------------------------- refinement
ZTC_DEV uint32_t q565(float r, float g, float b) {  // zap_tex.h:45-49
    int R = f2i_x86(r * 31.0f / 255.0f + 0.5f), G = f2i_x86(g * 63.0f / 255.0f + 0.5f), B = f2i_x86(b * 31.0f / 255.0f + 0.5f);
    return ((uint32_t)clampi(R, 0, 31) << 11) | ((uint32_t)clampi(G, 0, 63) << 5) | (uint32_t)clampi(B, 0, 31);
}
ZTC_DEV void bc1_palette(uint32_t c0, uint32_t c1, int pal[4][3]) {
    for (int k = 0; k < 2; k++) {
        uint32_t c = k ? c1 : c0;
        int R = (c >> 11) & 31, G = (c >> 5) & 63, B = c & 31;
        pal[k][0] = (R << 3) | (R >> 2); pal[k][1] = (G << 2) | (G >> 4); pal[k][2] = (B << 3) | (B >> 2);
    }
    for (int c = 0; c < 3; c++) {
        int a = pal[0][c], b = pal[1][c];
        pal[2][c] = (2 * a + b + 1) / 3; pal[3][c] = (a + 2 * b + 1) / 3;
    }
}
// canonical BC1 block for endpoints (c0 > c1 with best indices, or solid) and its SSE
ZTC_DEV int bc1_block_sse(const uint32_t t[16], uint32_t c0, uint32_t c1, uint2 &blk) {
    if (c0 < c1) { uint32_t s = c0; c0 = c1; c1 = s; }
    int pal[4][3], err = 0;
    bc1_palette(c0, c1, pal);
    uint32_t bits = 0;
    for (int i = 0; i < 16; i++) {
        int bk = 0, be = 1 << 30;
        for (int k = 0; k < (c0 == c1 ? 1 : 4); k++) {
            int d = 0;
            for (int c = 0; c < 3; c++) { int x = (int)chan(t[i], c) - pal[k][c]; d += x * x; }
            if (d < be) { be = d; bk = k; }
        }
        bits |= (uint32_t)bk << (2 * i);
        err += be;
    }
    blk = make_uint2(c0 | (c1 << 16), bits);
    return err;
}
// BC7 mode-6 block for expanded endpoints (7 bits + p-bit chosen per endpoint), indices re-fitted with texel 0
// limited to 0..7 so no swap is needed, and its SSE
ZTC_DEV int mode6_block_sse(const uint32_t t[16], const float e[2][4], uint4 &out) {
    int q[2][4], pb[2], x[2][4];
    for (int k = 0; k < 2; k++) {
        int best = 1 << 30;
        for (int p = 0; p < 2; p++) {
            int qq[4], xx[4], err = 0;
            for (int c = 0; c < 4; c++) {
                int g = clampi(f2i_x86((e[k][c] - (float)p) / 2.0f + 0.5f), 0, 127);
                qq[c] = g; xx[c] = (g << 1) | p;
                int d = xx[c] - f2i_x86(e[k][c] + 0.5f);
                err += d * d;
            }
            if (err < best) { best = err; pb[k] = p; for (int c = 0; c < 4; c++) { q[k][c] = qq[c]; x[k][c] = xx[c]; } }
        }
    }
    uint32_t pal[16];
    for (int j = 0; j < 16; j++) {
        uint32_t v = 0;
        for (int c = 0; c < 4; c++) v |= (uint32_t)lerp64(x[0][c], x[1][c], w4(j)) << (8 * c);
        pal[j] = v;
    }
    int err = 0;
    uint64_t idx = 0;
    for (int i = 0; i < 16; i++) {
        int bj = 0, be = 1 << 30;
        for (int j = 0; j < (i ? 16 : 8); j++) {
            int d = 0;
            for (int c = 0; c < 4; c++) { int y = (int)chan(t[i], c) - (int)chan(pal[j], c); d += y * y; }
            if (d < be) { be = d; bj = j; }
        }
        idx |= (uint64_t)bj << (4 * i);
        err += be;
    }
    Bits128 o;
    o.put(1u << 6, 7);
    for (int c = 0; c < 4; c++) { o.put((uint32_t)q[0][c], 7); o.put((uint32_t)q[1][c], 7); }
    o.put((uint32_t)pb[0], 1); o.put((uint32_t)pb[1], 1);
    o.put((uint32_t)(idx & 7u), 3);
    for (int i = 1; i < 16; i++) o.put((uint32_t)((idx >> (4 * i)) & 15u), 4);
    out = make_uint4(o.w[0], o.w[1], o.w[2], o.w[3]);
    return err;
}
// squared error of the block as stored (the decoder's integer palette)
ZTC_DEV int stored_sse(int fmt, const uint32_t t[16], const uint8_t *blk) {
    if (fmt == ZTC_FMT_BC1) {
        uint2 v = *(const uint2 *)blk;
        uint32_t c0 = v.x & 0xFFFFu, c1 = v.x >> 16;
        int pal[4][3];
        bc1_palette(c0, c1, pal);
        if (c0 <= c1) for (int c = 0; c < 3; c++) { pal[2][c] = (pal[0][c] + pal[1][c] + 1) / 2; pal[3][c] = 0; }
        int err = 0;
        for (int i = 0; i < 16; i++) {
            int k = (v.y >> (2 * i)) & 3;
            for (int c = 0; c < 3; c++) { int d = (int)chan(t[i], c) - pal[k][c]; err += d * d; }
        }
        return err;
    }
    uint4 v = *(const uint4 *)blk;
    const uint32_t w[4] = {v.x, v.y, v.z, v.w};
    float e[2][4];
    block_endpoints(fmt, blk, e);
    int err = 0;
    for (int i = 0; i < 16; i++) {
        int idx = i == 0 ? (int)get_bits128(w, 65, 3) : (int)get_bits128(w, 68 + 4 * (i - 1), 4);
        for (int c = 0; c < 4; c++) { int d = (int)chan(t[i], c) - lerp64((int)e[0][c], (int)e[1][c], w4(idx)); err += d * d; }
    }
    return err;
}

__global__ void __launch_bounds__(128) refine_kernel(int fmt, SrcU8 src, int bw, int nblocks, uint8_t *__restrict__ blocks, int steps,
                                                     float lr, uint32_t *__restrict__ sse0, uint32_t *__restrict__ sse1) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    const size_t bs = fmt == ZTC_FMT_BC1 ? 8 : 16;
    uint8_t *blk = blocks + (size_t)b * bs;
    uint32_t t[16];
    gather_block(src, b % bw, b / bw, t);
    float a[16], e[2][4];
    int nc;
    const bool covered = !(fmt == ZTC_FMT_BC7 && (blk[0] & 0x7F) != 0x40);
    int before;
    if (covered) before = stored_sse(fmt, t, blk);
    else {  // modes 5 / 1: not refined; their error still counts in the statistics
        uint32_t d[16];
        dec::bcn_block(ZTC_FMT_BC7, blk, d);
        before = 0;
        for (int i = 0; i < 16; i++)
            for (int c = 0; c < 4; c++) { int x = (int)chan(t[i], c) - (int)chan(d[i], c); before += x * x; }
    }
    int after = before;
    if (covered && before > 0 && block_weights(fmt, blk, a, nc)) {
        block_endpoints(fmt, blk, e);
        float m[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}}, v[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
        const float b1 = 0.9f, b2 = 0.999f, inv_n = 2.0f / (16.0f * (float)nc);
        float p1 = 1.0f, p2 = 1.0f;
        for (int s = 0; s < steps; s++) {
            float g[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
            for (int i = 0; i < 16; i++)
                for (int c = 0; c < nc; c++) {  // forward decode, residual, adjoint
                    float r = (a[i] * e[0][c] + (1.0f - a[i]) * e[1][c] - (float)chan(t[i], c)) * inv_n;
                    g[0][c] += a[i] * r;
                    g[1][c] += (1.0f - a[i]) * r;
                }
            p1 *= b1; p2 *= b2;
            for (int k = 0; k < 2; k++)
                for (int c = 0; c < nc; c++) {
                    m[k][c] = b1 * m[k][c] + (1.0f - b1) * g[k][c];
                    v[k][c] = b2 * v[k][c] + (1.0f - b2) * g[k][c] * g[k][c];
                    float mh = m[k][c] / (1.0f - p1), vh = v[k][c] / (1.0f - p2);
                    e[k][c] = fminf(255.0f, fmaxf(0.0f, e[k][c] - lr * mh / (sqrtf(vh) + 1e-8f)));
                }
        }
        if (fmt == ZTC_FMT_BC1) {
            uint2 nb;
            int ne = bc1_block_sse(t, q565(e[0][0], e[0][1], e[0][2]), q565(e[1][0], e[1][1], e[1][2]), nb);
            if (ne < before) { *(uint2 *)blk = nb; after = ne; }
        } else {
            uint4 nb;
            int ne = mode6_block_sse(t, e, nb);
            if (ne < before) { *(uint4 *)blk = nb; after = ne; }
        }
    }
    if (sse0) sse0[b] = (uint32_t)before;
    if (sse1) sse1[b] = (uint32_t)after;
}

}  // namespace ztc

// ---------------------------------------------------------------- C ABI
static int adj_check(int fmt, const void *p, int n) {
    if (fmt != ZTC_BC1 && fmt != ZTC_BC7) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "differentiable decode covers BC1 and BC7 mode 6");
    if (!p || n < 0) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null pointer or negative block count");
    if ((uintptr_t)p % (fmt == ZTC_BC1 ? 8u : 16u)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "blocks must be aligned to the block size");
    return ZTC_OK;
}
static bool floats_misaligned(const void *a, const void *b = nullptr) { return ((uintptr_t)a | (uintptr_t)b) & 3u; }
static int launch_status(const char *what) {
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZTC_OK : ztc_set_error(ZTC_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

extern "C" {

int zap_tex_cuda_block_endpoints_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, float *endpoints, void *stream) {
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!endpoints || floats_misaligned(endpoints)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned endpoints");
    if (nblocks) ztc::endpoints_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, endpoints);
    return launch_status("endpoints launch");
}

int zap_tex_cuda_palette_decode_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *endpoints, float *decoded,
                                    void *stream) {
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!endpoints || !decoded || floats_misaligned(endpoints, decoded))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned endpoints / decoded");
    if (nblocks) ztc::decode_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, endpoints, decoded);
    return launch_status("decode launch");
}

int zap_tex_cuda_palette_adjoint_dev(zap_tex_cuda_ctx *ctx, int fmt, const void *blocks, int nblocks, const float *grad_decoded,
                                     float *grad_endpoints, void *stream) {
    int st = adj_check(fmt, blocks, nblocks);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!grad_decoded || !grad_endpoints || floats_misaligned(grad_decoded, grad_endpoints))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "null or misaligned gradient pointer");
    if (nblocks)
        ztc::adjoint_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)blocks, nblocks, grad_decoded,
                                                                                   grad_endpoints);
    return launch_status("adjoint launch");
}

int zap_tex_cuda_refine_dev(zap_tex_cuda_ctx *ctx, int fmt, const uint8_t *rgba, int w, int h, size_t stride, void *blocks, int steps,
                            float lr, uint32_t *sse_before, uint32_t *sse_after, void *stream) {
    int st = adj_check(fmt, blocks, 0);
    if (st || (st = ztc_ctx_activate(ctx))) return st;
    if (!rgba || w < 1 || h < 1 || stride < (size_t)w * 4 || steps < 0 || steps > 1000 || !(lr >= 0.0f))
        return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad image, steps or learning rate");
    if (floats_misaligned(sse_before, sse_after)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "misaligned SSE outputs");
    const int bw = (w + 3) / 4, nblocks = bw * ((h + 3) / 4);
    ztc::SrcU8 src{rgba, stride, w, h, 4, (((uintptr_t)rgba | stride) & 15u) == 0};
    ztc::TraceScope tr(fmt == ZTC_BC1 ? "refine_bc1" : "refine_bc7", (cudaStream_t)stream);
    ztc::trace_units(nblocks);
    ztc::refine_kernel<<<(nblocks + 127) / 128, 128, 0, (cudaStream_t)stream>>>(fmt, src, bw, nblocks, (uint8_t *)blocks, steps, lr, sse_before,
                                                                               sse_after);
    return launch_status("refine launch");
}

}  // extern "C"

// decode.cu - device block decoders: zap_bc_decode (zap_tex.h:1526-1547, BC7 all modes), zap_bc6h_decode
// (zap_tex.h:963-975) and zap_astc_decode (zap_tex.h:1344-1356, kernel in astc.cu), device and host memory. One
// thread per block; only texels inside the image are written (partial edge blocks).
// They give on-device quality checks for encoded batches without a host round trip.
#include <string>

#include "../../include/zap_tex_cuda.h"
#include "ztc_decode.cuh"
#include "ztc_internal.h"

namespace ztc {

__global__ void __launch_bounds__(128) bcn_decode_kernel(int fmt, const uint8_t *__restrict__ bc, int w, int h, uint8_t *__restrict__ out,
                                                         size_t stride) {
    const int bw = (w + 3) / 4, nblocks = bw * ((h + 3) / 4);
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    uint32_t px[16];
    dec::bcn_block(fmt, bc + (size_t)b * ((fmt == 0 || fmt == 2) ? 8 : 16), px);
    const bool vec = (((uintptr_t)out | stride) & 15u) == 0, aligned4 = (((uintptr_t)out | stride) & 3u) == 0;
    dec::store_block_rgba8(out, stride, w, h, b % bw, b / bw, px, vec, aligned4);
}

__global__ void __launch_bounds__(128) bc6h_decode_kernel(const uint8_t *__restrict__ bc, int w, int h, uint16_t *__restrict__ out, size_t stride) {
    const int bw = (w + 3) / 4, nblocks = bw * ((h + 3) / 4);
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nblocks) return;
    uint4 v = *(const uint4 *)(bc + (size_t)b * 16);
    const uint32_t wd[4] = {v.x, v.y, v.z, v.w};
    uint16_t px[16][4];
    dec::bc6h_block(wd, px);
    const int bx = b % bw, by = b / bw;
    // a row of four texels inside the image as two 16-byte stores when the image and its pitch (stride halves) are
    // 16-byte aligned; else element by element
    const bool vec = ((uintptr_t)out & 15u) == 0 && (stride & 7u) == 0;
    #pragma unroll
    for (int r = 0; r < 4; r++) {
        const int y = by * 4 + r, x0 = bx * 4;
        if (y >= h) break;
        uint16_t *row = out + (size_t)y * stride + (size_t)x0 * 4;
        if (vec && x0 + 3 < w) {
            uint32_t q[8];
            #pragma unroll
            for (int k = 0; k < 8; k++) q[k] = (uint32_t)px[4 * r + (k >> 1)][2 * (k & 1)] | ((uint32_t)px[4 * r + (k >> 1)][2 * (k & 1) + 1] << 16);
            ((uint4 *)row)[0] = make_uint4(q[0], q[1], q[2], q[3]);
            ((uint4 *)row)[1] = make_uint4(q[4], q[5], q[6], q[7]);
            continue;
        }
        for (int c = 0; c < 4; c++) {
            if (x0 + c >= w) break;
            for (int k = 0; k < 4; k++) row[4 * c + k] = px[4 * r + c][k];
        }
    }
}

}  // namespace ztc

namespace {

enum Kind { kBcn, kBc6h, kAstc };

// block bytes of the format, and the alignment the decoder's block loads need
size_t block_bytes_of(Kind k, int fmt) { return k == kBcn && (fmt == ZTC_BC1 || fmt == ZTC_BC4) ? 8 : 16; }

int check_decode(Kind k, const void *bc, int w, int h, int fmt, const void *rgba, size_t stride, size_t texel_units) {
    if (!bc || !rgba || w < 1 || h < 1 || stride < (size_t)w * texel_units) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad decode arguments");
    if ((long)((w + 3) / 4) * ((h + 3) / 4) >= (1L << 31)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "more than 2^31 - 1 blocks");
    if (k == kBcn && (fmt < ZTC_BC1 || fmt > ZTC_BC7)) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "decode format must be BC1..BC7");
    if ((uintptr_t)bc % block_bytes_of(k, fmt)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "blocks must be aligned to the block size");
    return ZTC_OK;
}

cudaError_t launch_decode(Kind k, const void *bc, int w, int h, int fmt, void *rgba, size_t stride, cudaStream_t s) {
    const long nblocks = (long)((w + 3) / 4) * ((h + 3) / 4);
    const unsigned grid = (unsigned)((nblocks + 127) / 128);
    if (k == kAstc) return ztc_launch_astc_decode((const uint8_t *)bc, w, h, (uint8_t *)rgba, stride, s);
    if (k == kBc6h) ztc::bc6h_decode_kernel<<<grid, 128, 0, s>>>((const uint8_t *)bc, w, h, (uint16_t *)rgba, stride);
    else ztc::bcn_decode_kernel<<<grid, 128, 0, s>>>(fmt, (const uint8_t *)bc, w, h, (uint8_t *)rgba, stride);
    return cudaGetLastError();
}

int dev_decode(Kind k, zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, void *rgba, size_t stride, void *stream) {
    int st = check_decode(k, bc, w, h, fmt, rgba, stride, 4);
    if (st) return st;
    if ((st = ztc_ctx_activate(ctx))) return st;
    cudaError_t e = launch_decode(k, bc, w, h, fmt, rgba, stride, (cudaStream_t)stream);
    if (e != cudaSuccess) { cudaGetLastError(); return ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e)); }
    return ZTC_OK;
}

// host memory in and out, synchronous: blocks to a device buffer, decode, texel rows back with the caller's stride
int host_decode(Kind k, zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, void *rgba, size_t stride, size_t texel_bytes) {
    // host blocks need no alignment (they are copied): the check sees a stand-in aligned address
    int st = check_decode(k, (const void *)16, w, h, fmt, rgba, stride * (k == kBc6h ? 2 : 1), texel_bytes);
    if (!st && !bc) st = ztc_set_error(ZTC_ERR_INVALID_ARG, "bad decode arguments");
    if (st) return st;
    if ((st = ztc_ctx_activate(ctx))) return st;
    const size_t nb = (size_t)((w + 3) / 4) * ((h + 3) / 4) * block_bytes_of(k, fmt), row = (size_t)w * texel_bytes;
    const size_t host_stride = k == kBc6h ? stride * 2 : stride;  // BC6H strides count uint16 elements
    cudaStream_t s = cudaStreamPerThread;
    uint8_t *d_bc = nullptr, *d_px = nullptr;
    cudaError_t e = ztc_malloc_async((void **)&d_bc, nb, s);
    if (e == cudaSuccess) e = ztc_malloc_async((void **)&d_px, row * (size_t)h, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_bc, bc, nb, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = launch_decode(k, d_bc, w, h, fmt, d_px, k == kBc6h ? (size_t)w * 4 : row, s);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(rgba, host_stride, d_px, row, row, (size_t)h, cudaMemcpyDeviceToHost, s);
    if (d_px) cudaFreeAsync(d_px, s);
    if (d_bc) cudaFreeAsync(d_bc, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) {
        cudaGetLastError();
        return ztc_set_error(e == cudaErrorMemoryAllocation ? ZTC_ERR_NO_MEMORY : ZTC_ERR_CUDA, cudaGetErrorString(e));
    }
    return ZTC_OK;
}

}  // namespace

extern "C" {

int zap_tex_cuda_bc_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride, void *stream) {
    ZTC_NVTX();
    return dev_decode(kBcn, ctx, bc, w, h, fmt, rgba, stride, stream);
}

int zap_tex_cuda_bc6h_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint16_t *rgba, size_t stride, void *stream) {
    ZTC_NVTX();
    return dev_decode(kBc6h, ctx, bc, w, h, ZTC_BC6H, rgba, stride, stream);
}

int zap_tex_cuda_astc_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint8_t *rgba, size_t stride, void *stream) {
    ZTC_NVTX();
    return dev_decode(kAstc, ctx, bc, w, h, ZTC_ASTC4X4, rgba, stride, stream);
}

int zap_tex_cuda_bc_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride) {
    ZTC_NVTX();
    return host_decode(kBcn, ctx, bc, w, h, fmt, rgba, stride, 4);
}

int zap_tex_cuda_bc6h_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint16_t *rgba, size_t stride) {
    ZTC_NVTX();
    return host_decode(kBc6h, ctx, bc, w, h, ZTC_BC6H, rgba, stride, 8);
}

int zap_tex_cuda_astc_decode(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint8_t *rgba, size_t stride) {
    ZTC_NVTX();
    return host_decode(kAstc, ctx, bc, w, h, ZTC_ASTC4X4, rgba, stride, 4);
}

}  // extern "C"

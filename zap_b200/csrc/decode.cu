// decode.cu - device block decoders: zap_bc_decode (zap_tex.h:1526-1547, BC7 all modes) and zap_bc6h_decode
// (zap_tex.h:963-975). One thread per block; only texels inside the image are written (partial edge blocks).
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
    const int bx = b % bw, by = b / bw;
    for (int i = 0; i < 16; i++) {
        int x = bx * 4 + (i & 3), y = by * 4 + (i >> 2);
        if (x < w && y < h) {
            uint8_t *p = out + (size_t)y * stride + (size_t)x * 4;
            p[0] = (uint8_t)px[i]; p[1] = (uint8_t)(px[i] >> 8); p[2] = (uint8_t)(px[i] >> 16); p[3] = (uint8_t)(px[i] >> 24);
        }
    }
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
    for (int i = 0; i < 16; i++) {
        int x = bx * 4 + (i & 3), y = by * 4 + (i >> 2);
        if (x < w && y < h)
            for (int c = 0; c < 4; c++) out[(size_t)y * stride + (size_t)x * 4 + c] = px[i][c];
    }
}

}  // namespace ztc

extern "C" {

int zap_tex_cuda_bc_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, int fmt, uint8_t *rgba, size_t stride, void *stream) {
    if (!bc || !rgba || w < 1 || h < 1 || stride < (size_t)w * 4) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad decode arguments");
    if (fmt < ZTC_BC1 || fmt > ZTC_BC7) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "decode format must be BC1..BC7");
    int st = ztc_ctx_activate(ctx);
    if (st) return st;
    const long nblocks = (long)((w + 3) / 4) * ((h + 3) / 4);
    ztc::bcn_decode_kernel<<<(unsigned)((nblocks + 127) / 128), 128, 0, (cudaStream_t)stream>>>(fmt, (const uint8_t *)bc, w, h, rgba, stride);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZTC_OK : ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e));
}

int zap_tex_cuda_bc6h_decode_dev(zap_tex_cuda_ctx *ctx, const void *bc, int w, int h, uint16_t *rgba, size_t stride, void *stream) {
    if (!bc || !rgba || w < 1 || h < 1 || stride < (size_t)w * 4) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad decode arguments");
    int st = ztc_ctx_activate(ctx);
    if (st) return st;
    const long nblocks = (long)((w + 3) / 4) * ((h + 3) / 4);
    ztc::bc6h_decode_kernel<<<(unsigned)((nblocks + 127) / 128), 128, 0, (cudaStream_t)stream>>>((const uint8_t *)bc, w, h, rgba, stride);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ZTC_OK : ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e));
}

}  // extern "C"

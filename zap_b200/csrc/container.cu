// container.cu - the CLI's texture containers (zap.c:309-355): DDS and .astc headers, and whole files whose mip
// chain and blocks are computed on the device.
//
// DDS layout (zap.c:344-349): "DDS " and the 124-byte header; for BC7, or when sRGB is requested, the 20-byte DX10
// extension follows (DXGI code, 2D, one element); then each level's blocks, largest first. The .astc layout
// (zap.c:312-321): 16 bytes (magic 0x5CA1AB13 little-endian, block 4x4x1, 24-bit width / height / depth) and the one
// level's blocks. The field values follow the CLI so that a file written here is the CLI's file byte for byte.
#include <cstring>

#include "../../include/zap_tex_cuda.h"
#include "ztc_internal.h"

namespace {

void put32(uint8_t *p, uint32_t v) {
    for (int k = 0; k < 4; k++) p[k] = (uint8_t)(v >> (8 * k));
}
bool dds_format(int fmt) { return fmt >= ZTC_BC1 && fmt <= ZTC_BC7; }
int effective_srgb(int fmt, int srgb) { return fmt == ZTC_BC4 || fmt == ZTC_BC5 ? 0 : srgb != 0; }  // zap.c:325
size_t dds_header_bytes(int fmt, int srgb) { return fmt == ZTC_BC7 || effective_srgb(fmt, srgb) ? 148 : 128; }
int file_levels(int w, int h, int fmt, int mips) { return mips && fmt != ZTC_ASTC4X4 ? zap_tex_cuda_mip_levels(w, h) : 1; }

size_t blocks_bytes(int w, int h, int fmt, int levels) {
    size_t total = 0;
    for (int l = 0; l < levels; l++, w = w > 1 ? w / 2 : 1, h = h > 1 ? h / 2 : 1) total += zap_tex_cuda_bc_size(w, h, fmt);
    return total;
}

int cuda_status(cudaError_t e) {
    cudaGetLastError();
    return ztc_set_error(e == cudaErrorMemoryAllocation ? ZTC_ERR_NO_MEMORY : ZTC_ERR_CUDA, cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int zap_tex_cuda_dds_header(int w, int h, int fmt, int mips, int srgb, void *hdr, size_t *hdr_bytes) {
    static const char kFourcc[5][5] = {"DXT1", "DXT5", "BC4U", "BC5U", "DX10"};
    static const uint32_t kDxgiUnorm[5] = {71, 77, 80, 83, 98};  // BC1..BC7 UNORM; the _SRGB code is the next one
    if (!hdr || w < 1 || h < 1) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad DDS header arguments");
    if (!dds_format(fmt)) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "DDS header format must be BC1..BC7");
    const int s = effective_srgb(fmt, srgb);
    const size_t n = dds_header_bytes(fmt, srgb);
    uint8_t *p = (uint8_t *)hdr;
    std::memset(p, 0, n);
    std::memcpy(p, "DDS ", 4);
    put32(p + 4, 124);
    // CAPS | HEIGHT | WIDTH | PIXELFORMAT | LINEARSIZE, and MIPMAPCOUNT with a chain
    put32(p + 8, 0x1u | 0x2u | 0x4u | 0x1000u | 0x80000u | (mips ? 0x20000u : 0u));
    put32(p + 12, (uint32_t)h);
    put32(p + 16, (uint32_t)w);
    put32(p + 20, (uint32_t)zap_tex_cuda_bc_size(w, h, fmt));
    put32(p + 28, (uint32_t)file_levels(w, h, fmt, mips));
    put32(p + 76, 32);   // pixel-format structure size
    put32(p + 80, 0x4);  // its FOURCC field is valid
    std::memcpy(p + 84, n == 148 ? "DX10" : kFourcc[fmt], 4);
    put32(p + 108, 0x1000u | (mips ? 0x400008u : 0u));  // TEXTURE, plus COMPLEX | MIPMAP with a chain
    if (n == 148) {
        put32(p + 128, kDxgiUnorm[fmt] + (uint32_t)s);
        put32(p + 132, 3);  // 2D texture
        put32(p + 140, 1);  // one array element
    }
    if (hdr_bytes) *hdr_bytes = n;
    return ZTC_OK;
}

int zap_tex_cuda_astc_header(int w, int h, void *hdr) {
    if (!hdr || w < 1 || h < 1) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad .astc header arguments");
    uint8_t *p = (uint8_t *)hdr;
    const uint8_t head[7] = {0x13, 0xAB, 0xA1, 0x5C, 4, 4, 1};
    std::memset(p, 0, 16);
    std::memcpy(p, head, 7);
    for (int k = 0; k < 3; k++) {
        p[7 + k] = (uint8_t)(w >> (8 * k));
        p[10 + k] = (uint8_t)(h >> (8 * k));
    }
    p[13] = 1;  // depth
    return ZTC_OK;
}

size_t zap_tex_cuda_tex_file_bytes(int w, int h, int fmt, int mips, int srgb) {
    if (w < 1 || h < 1) return 0;
    if (fmt == ZTC_ASTC4X4) return 16 + zap_tex_cuda_bc_size(w, h, ZTC_ASTC4X4);
    if (!dds_format(fmt)) return 0;
    return dds_header_bytes(fmt, srgb) + blocks_bytes(w, h, fmt, file_levels(w, h, fmt, mips));
}

int zap_tex_cuda_tex_file(zap_tex_cuda_ctx *ctx, const uint8_t *rgba, int w, int h, size_t stride, int fmt, float rdo, int mips,
                          int srgb, void *out, size_t out_cap) {
    ZTC_NVTX();
    if (!rgba || !out || w < 1 || h < 1 || stride < (size_t)w * 4) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad texture file arguments");
    if (!dds_format(fmt) && fmt != ZTC_ASTC4X4) return ztc_set_error(ZTC_ERR_UNSUPPORTED, "file format must be BC1..BC7 or ASTC 4x4");
    const size_t need = zap_tex_cuda_tex_file_bytes(w, h, fmt, mips, srgb);
    if (out_cap < need) return ztc_set_error(ZTC_ERR_INVALID_ARG, "out_cap below zap_tex_cuda_tex_file_bytes");
    int st = ztc_ctx_activate(ctx);
    if (st) return st;

    uint8_t *o = (uint8_t *)out;
    size_t hn = 16;
    if (fmt == ZTC_ASTC4X4) st = zap_tex_cuda_astc_header(w, h, o);
    else st = zap_tex_cuda_dds_header(w, h, fmt, mips, srgb, o, &hn);
    if (st) return st;

    const int levels = file_levels(w, h, fmt, mips), s = effective_srgb(fmt, srgb);
    const size_t base = (size_t)w * h * 4, chain = levels > 1 ? zap_tex_cuda_mip_chain_bytes(w, h) : 0;
    const size_t total = need - hn;
    cudaStream_t cs = cudaStreamPerThread;
    uint8_t *d_img = nullptr, *d_blocks = nullptr;
    cudaError_t e = ztc_malloc_async((void **)&d_img, base + chain, cs);
    if (e == cudaSuccess) e = ztc_malloc_async((void **)&d_blocks, total, cs);
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(d_img, (size_t)w * 4, rgba, stride, (size_t)w * 4, (size_t)h, cudaMemcpyHostToDevice, cs);
    if (e != cudaSuccess) st = cuda_status(e);
    // levels 1.. of the chain, each zap_mip_next of the one before (zap.c:339-341)
    if (!st && levels > 1) st = zap_tex_cuda_mip_chain_dev(ctx, d_img, w, h, (size_t)w * 4, s, d_img + base, cs);
    const uint8_t *lsrc = d_img;
    uint8_t *ldst = d_blocks;
    for (int l = 0, lw = w, lh = h; l < levels && !st; l++) {
        // one encoder call per level, as the CLI calls zap_bc_encode (zap.c:337): rdo > 0 runs one chain per level
        if (fmt == ZTC_ASTC4X4) st = zap_tex_cuda_astc_encode_dev(ctx, lsrc, lw, lh, (size_t)lw * 4, ldst, cs);
        else st = zap_tex_cuda_bc_encode_rdo_dev(ctx, lsrc, lw, lh, (size_t)lw * 4, fmt, rdo, 0, ldst, cs);
        ldst += zap_tex_cuda_bc_size(lw, lh, fmt);
        lsrc = l == 0 ? d_img + base : lsrc + (size_t)lw * lh * 4;  // the chain packs levels 1.. tightly
        lw = lw > 1 ? lw / 2 : 1;
        lh = lh > 1 ? lh / 2 : 1;
    }
    if (!st && (e = cudaMemcpyAsync(o + hn, d_blocks, total, cudaMemcpyDeviceToHost, cs)) != cudaSuccess) st = cuda_status(e);
    if (d_blocks) cudaFreeAsync(d_blocks, cs);
    if (d_img) cudaFreeAsync(d_img, cs);
    e = cudaStreamSynchronize(cs);
    if (!st && e != cudaSuccess) st = cuda_status(e);
    return st;
}

}  // extern "C"

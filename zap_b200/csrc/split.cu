// split.cu - split / merge of encoded BC1-BC7 images into field planes (zap_tex.h:1549-1571), for sm_100a.
//
// The split form puts field k of every block into plane k (BC7: the 8 endpoint bytes, the straddling byte 8, the
// 7 index bytes), which an LZ-style compressor finds far more repetitive than interleaved blocks. One thread per
// block: split reads the block with one vector load and writes its fields to the planes; merge gathers the fields
// and writes the block with one vector store. Stray bytes after the last whole block are copied unchanged. The
// encoders can also write the split form directly (BlockOut in ztc_common.cuh), with no pass of this kernel.
#include "ztc_common.cuh"
#include "ztc_internal.h"

namespace ztc {

__global__ void __launch_bounds__(256) bc_regroup_kernel(const uint8_t *__restrict__ in, uint8_t *__restrict__ out, size_t nb, int fmt,
                                                         int bs, int to_planes, int aligned) {
    for (size_t b = (size_t)blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += (size_t)gridDim.x * blockDim.x) {
        uint32_t w[4] = {0u, 0u, 0u, 0u};
        if (to_planes) {
            const uint8_t *src = in + b * bs;
            if (aligned && bs == 16) { const uint4 v = __ldg((const uint4 *)src); w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w; }
            else if (aligned) { const uint2 v = __ldg((const uint2 *)src); w[0] = v.x; w[1] = v.y; }
            else
                for (int i = 0; i < bs; i++) w[i >> 2] |= (uint32_t)__ldg(src + i) << (8 * (i & 3));
            put_block(BlockOut{out, nb, fmt, 1}, b, w, bs);
        } else {
            int sz[4];
            const int nf = bc_fields(fmt, sz);
            int off = 0;
            for (int k = 0; k < nf; k++) {
                const uint8_t *src = in + nb * (size_t)off + b * (size_t)sz[k];
                for (int j = 0; j < sz[k]; j++) {
                    const int i = off + j;
                    const uint32_t v = (uint32_t)__ldg(src + j) << (8 * (i & 3));
                    if (i < 4) w[0] |= v; else if (i < 8) w[1] |= v; else if (i < 12) w[2] |= v; else w[3] |= v;
                }
                off += sz[k];
            }
            uint8_t *dst = out + b * bs;
            if (aligned) put_block(BlockOut{out, 0, fmt, 0}, b, w, bs);
            else
                for (int i = 0; i < bs; i++) {
                    const uint32_t x = i < 4 ? w[0] : i < 8 ? w[1] : i < 12 ? w[2] : w[3];
                    dst[i] = (uint8_t)(x >> (8 * (i & 3)));
                }
        }
    }
}

}  // namespace ztc

// n bytes of blocks (to_planes) or planes (merge) from `in` to `out` (device memory, not overlapping)
cudaError_t ztc_launch_bc_regroup(const uint8_t *in, uint8_t *out, size_t n, int fmt, int to_planes, cudaStream_t stream) {
    const int bs = (fmt == ZTC_FMT_BC1 || fmt == ZTC_FMT_BC4) ? 8 : 16;
    const size_t nb = n / (size_t)bs, tail = n - nb * (size_t)bs;
    if (nb) {
        const int aligned = ((((uintptr_t)in) | ((uintptr_t)out)) & (uintptr_t)(bs - 1)) == 0;
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const size_t want = (nb + 255) / 256, cap = (size_t)sms * 8;
        const int grid = (int)(want < cap ? want : cap);
        ztc::TraceScope tr(to_planes ? "bc_split" : "bc_merge", stream);
        ztc::trace_units((long)nb);
        ztc::bc_regroup_kernel<<<grid, 256, 0, stream>>>(in, out, nb, fmt, bs, to_planes, aligned);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    if (tail) return cudaMemcpyAsync(out + nb * bs, in + nb * bs, tail, cudaMemcpyDeviceToDevice, stream);
    return cudaSuccess;
}

// alu_probe.cu - issue-rate probe for the ALU roofline of the encoders (a diagnostic; no reference counterpart).
//
// The encoders are bound by the SMs' instruction issue, not by HBM: a 4x4 block costs thousands of integer and
// float operations against 80 bytes of traffic. The roofline they are measured against is the rate at which a
// B200 executes the instruction kinds their inner loops are made of, measured here rather than derived from a
// data sheet: every thread runs 8 independent chains of one kind (no chain waits on another, so with 64 warps
// per SM the latency is hidden and the probe measures throughput), 256 probe instructions per loop iteration.
//   kind 0  mad.lo.u32    (integer multiply-add: the palette distance and error sums)
//   kind 1  fma.rn.f32    (float multiply-add: the principal-axis and least-squares arithmetic)
//   kind 2  dp4a.u32.u32  (four byte products summed: the texel-to-palette distances)
//   kind 3  kinds 0 and 1 alternating (the encoders' integer/float mix)
// Each chain is written in inline PTX so the instruction kind and count are fixed by the source; the result is
// stored only under a condition the compiler cannot decide, so no chain is removed as dead code.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/zap_tex_cuda.h"
#include "ztc_internal.h"

namespace ztc {
namespace {
constexpr int kProbeThreads = 256, kProbeCtasPerSm = 8, kChains = 8, kUnroll = 32;

template <int KIND>
__global__ void __launch_bounds__(kProbeThreads) alu_probe_kernel(uint32_t *sink, int iters, uint32_t m, uint32_t c) {
    uint32_t a[kChains];
    float f[kChains];
    #pragma unroll
    for (int j = 0; j < kChains; j++) {
        a[j] = threadIdx.x * (2u * j + 1u) + blockIdx.x;
        f[j] = (float)a[j] * 1e-6f;
    }
    const float fm = __uint_as_float(0x3F7FFFF0u + (m & 7u)), fc = (float)(c & 255u) * 1e-3f;  // |f| stays bounded
    for (int i = 0; i < iters; i++) {
        #pragma unroll
        for (int r = 0; r < kUnroll; r++) {
            #pragma unroll
            for (int j = 0; j < kChains; j++) {
                if (KIND == 0 || (KIND == 3 && (j & 1) == 0))
                    asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[j]) : "r"(m), "r"(c));
                else if (KIND == 1 || KIND == 3)
                    asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(f[j]) : "f"(fm), "f"(fc));
                else
                    asm volatile("dp4a.u32.u32 %0, %0, %1, %0;" : "+r"(a[j]) : "r"(m));
            }
        }
    }
    uint32_t acc = 0;
    #pragma unroll
    for (int j = 0; j < kChains; j++) acc ^= a[j] ^ __float_as_uint(f[j]);
    if (acc == c) sink[0] = acc;  // almost never true; keeps every chain live
}
}  // namespace
}  // namespace ztc

extern "C" ZTC_API int zap_tex_cuda_alu_probe_dev(int kind, int iters, void *sink, void *stream, double *instructions) {
    ZTC_NVTX();
    if (kind < 0 || kind > 3 || iters < 1 || !sink || ((uintptr_t)sink & 3u)) return ztc_set_error(ZTC_ERR_INVALID_ARG, "bad probe arguments");
    int dev = 0, major = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) { cudaGetLastError(); return ztc_set_error(ZTC_ERR_NO_DEVICE, "no CUDA device"); }
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return ztc_set_error(ZTC_ERR_NO_DEVICE, "this build targets sm_100a");
    const int grid = ztc_sm_count() * ztc::kProbeCtasPerSm;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t *p = (uint32_t *)sink;
    const uint32_t m = 0x01010101u * 3u + 0x10000u, c = 0x9E3779B9u;
    switch (kind) {
    case 0: ztc::alu_probe_kernel<0><<<grid, ztc::kProbeThreads, 0, s>>>(p, iters, m, c); break;
    case 1: ztc::alu_probe_kernel<1><<<grid, ztc::kProbeThreads, 0, s>>>(p, iters, m, c); break;
    case 2: ztc::alu_probe_kernel<2><<<grid, ztc::kProbeThreads, 0, s>>>(p, iters, m, c); break;
    default: ztc::alu_probe_kernel<3><<<grid, ztc::kProbeThreads, 0, s>>>(p, iters, m, c); break;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ztc_set_error(ZTC_ERR_CUDA, cudaGetErrorString(e));
    if (instructions)
        *instructions = (double)grid * ztc::kProbeThreads * (double)iters * ztc::kUnroll * ztc::kChains;
    return ZTC_OK;
}

// emu.cu - TEST INFRASTRUCTURE: the per-block encoder logic of zap_b200/csrc, compiled for the host.
//
// The kernels' block functions (ztc::bc1_encode, ztc::mode6_encode, ztc::bc6h_encode_block, ...) are
// __host__ __device__; this file includes the kernel sources and runs those functions block by block on the CPU,
// so tests/test_block_logic_on_host.py can diff the device logic against the oracle without a GPU. It is a
// debugging aid beside the GPU parity tests, not a substitute for them: warp-cooperative kernels (the BC7 mode 5/1
// and ASTC two-partition work lists) are not emulated, and only blocks those kernels do not revisit are compared.
#include "../../zap_b200/csrc/astc.cu"
#include "../../zap_b200/csrc/bc6h.cu"
#include "../../zap_b200/csrc/bc7.cu"
#include "../../zap_b200/csrc/bcn.cu"
#include "../../zap_b200/csrc/mip.cu"

namespace ztc {  // the launchers' tracing hooks live in api.cu, which is not part of this build
void trace_begin(const char *, cudaStream_t) {}
void trace_end(cudaStream_t) {}
void trace_units(long) {}
void trace_units_dev(const uint32_t *, cudaStream_t) {}
}  // namespace ztc
int ztc_set_error(int status, const char *) { return status; }
int ztc_sm_count() { return 148; }  // launch sizing only; no launch runs in this build

using namespace ztc;

extern "C" {

// BC1/BC3/BC4/BC5 exactly; BC7: mode-6 blocks, hard[b] = 1 where kernel B would revisit the block
__attribute__((visibility("default"))) int emu_bc_encode(const uint8_t *img, int w, int h, size_t stride, int fmt, uint8_t *out,
                                                         uint8_t *hard) {
    SrcU8 s{img, stride, w, h, 4, 0};
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            uint32_t t[16];
            gather_block(s, bx, by, t);
            size_t b = (size_t)by * bw + bx;
            if (fmt == ZTC_FMT_BC1) { uint2 v = bc1_encode(t); memcpy(out + b * 8, &v, 8); }
            else if (fmt == ZTC_FMT_BC4) { uint2 v = bc4_encode(t, 0); memcpy(out + b * 8, &v, 8); }
            else if (fmt == ZTC_FMT_BC3) { uint2 a = bc4_encode(t, 3), c = bc1_encode(t); memcpy(out + b * 16, &a, 8); memcpy(out + b * 16 + 8, &c, 8); }
            else if (fmt == ZTC_FMT_BC5) { uint2 r = bc4_encode(t, 0), g = bc4_encode(t, 1); memcpy(out + b * 16, &r, 8); memcpy(out + b * 16 + 8, &g, 8); }
            else if (fmt == ZTC_FMT_BC7) {
                uint4 v;
                int err = mode6_encode(t, TexRef{t, 1}, v);
                memcpy(out + b * 16, &v, 16);
                if (hard) hard[b] = err > 64;
            } else return -1;
        }
    return 0;
}

__attribute__((visibility("default"))) int emu_bc6h_encode(const float *img, int w, int h, size_t stride, uint8_t *out) {
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            int16_t t[48];
            float U[48];
            for (int i = 0; i < 16; i++) {
                int x = std::min(bx * 4 + (i & 3), w - 1), y = std::min(by * 4 + (i >> 2), h - 1);
                for (int c = 0; c < 3; c++) {
                    uint32_t hb = f2h_unsigned(img[(size_t)y * stride + (size_t)x * 4 + c]);
                    t[3 * i + c] = (int16_t)hb;
                    U[3 * i + c] = (float)hb * 64.0f / 31.0f;
                }
            }
            uint32_t ts;
            const uint64_t cw = bc6_center(t, 1, ts);
            uint4 v = bc6h_encode_block(HalfRef{t, U, 1, cw, ts});
            memcpy(out + ((size_t)by * bw + bx) * 16, &v, 16);
        }
    return 0;
}

// single-partition ASTC blocks; hard[b] = 1 where the two-partition kernel would revisit the block
__attribute__((visibility("default"))) int emu_astc_encode(const uint8_t *img, int w, int h, size_t stride, uint8_t *out, uint8_t *hard) {
    static AstcTables T;
    static AstcSmem S;
    static bool ready = false;
    if (!ready) {
        build_tables(T);
        memcpy(S.q, T.q, sizeof S.q); memcpy(S.uq, T.uq, sizeof S.uq); memcpy(S.cfg, T.cfg, sizeof S.cfg);
        memcpy(S.trit_code, T.trit_code, sizeof S.trit_code); memcpy(S.quint_code, T.quint_code, sizeof S.quint_code);
        memcpy(S.wq, T.wq, sizeof S.wq);
        ready = true;
    }
    SrcU8 s{img, stride, w, h, 4, 0};
    int bw = (w + 3) / 4, bh = (h + 3) / 4;
    for (int by = 0; by < bh; by++)
        for (int bx = 0; bx < bw; bx++) {
            uint32_t t[16];
            gather_block(s, bx, by, t);
            bool opaque = true;
            for (int i = 0; i < 16; i++) opaque &= (t[i] >> 24) == 255u;
            int bc = 0;
            uint32_t bcodes[4] = {0, 0, 0, 0}, bwt[4] = {0, 0, 0, 0};
            const int best = astc_single_block(t, TexRef{t, 1}, S, opaque, bc, bcodes, bwt);
            uint4 v = astc_pack(S, bc, 0, bcodes, bwt);
            size_t b = (size_t)by * bw + bx;
            memcpy(out + b * 16, &v, 16);
            if (hard) hard[b] = opaque && best > 192;
        }
    return 0;
}

__attribute__((visibility("default"))) int emu_mip_next(const uint8_t *src, int w, int h, size_t stride, int srgb, uint8_t *dst, size_t dst_stride) {
    SrgbTables T;
    srgb_tables_host(T);
    int nw = w > 1 ? w / 2 : 1, nh = h > 1 ? h / 2 : 1;
    for (int y = 0; y < nh; y++)
        for (int x = 0; x < nw; x++) {
            int x0 = std::min(2 * x, w - 1), x1 = std::min(2 * x + 1, w - 1), y0 = std::min(2 * y, h - 1), y1 = std::min(2 * y + 1, h - 1);
            uint32_t v = box4(ld_texel(src + (size_t)y0 * stride + (size_t)x0 * 4), ld_texel(src + (size_t)y0 * stride + (size_t)x1 * 4),
                              ld_texel(src + (size_t)y1 * stride + (size_t)x0 * 4), ld_texel(src + (size_t)y1 * stride + (size_t)x1 * 4),
                              srgb != 0, T);
            memcpy(dst + (size_t)y * dst_stride + (size_t)x * 4, &v, 4);
        }
    return 0;
}

// floats v with bit patterns in [lo, hi) for which the mip generator's bucketed sRGB search differs from the
// reference's binary search (zap_tex.h:1429-1433)
__attribute__((visibility("default"))) uint64_t emu_srgb_search_mismatches(uint64_t lo, uint64_t hi) {
    SrgbTables T;
    srgb_tables_host(T);
    uint64_t bad = 0;
    for (uint64_t b = lo; b < hi; b++) {
        const uint32_t u = (uint32_t)b;
        float v;
        memcpy(&v, &u, 4);
        int l = 0, h = 255;
        while (l < h) { const int mid = (l + h) >> 1; if (v < T.thr[mid]) h = mid; else l = mid + 1; }
        bad += lin_to_srgb(T.thr, T.bucket, v) != (uint32_t)l;
    }
    return bad;
}

// endpoint pairs and weights for which ztc::Lerp4 (two channels per word) differs from four lerp64 calls: every
// (a, b) pair in the low fields (R, G) and in the high fields (B, A) at every weight 0..64, against extreme and
// mixed values in the other field (the low field's negative slopes borrow from the high field)
__attribute__((visibility("default"))) uint64_t emu_lerp4_mismatches() {
    const int other[6][2] = {{0, 0}, {255, 255}, {0, 255}, {255, 0}, {17, 200}, {200, 17}};
    uint64_t bad = 0;
    for (int hi_field = 0; hi_field < 2; hi_field++)
        for (int a = 0; a < 256; a++)
            for (int b = 0; b < 256; b++)
                for (int o = 0; o < 6; o++) {
                    int x0[4], x1[4];
                    for (int c = 0; c < 4; c++) {
                        const bool mine = (c >= 2) == (hi_field == 1);
                        x0[c] = mine ? a : other[o][0];
                        x1[c] = mine ? b : other[o][1];
                    }
                    const Lerp4 row(x0, x1);
                    for (int w = 0; w <= 64; w++) {
                        const uint32_t want = pack_rgba(lerp64(x0[0], x1[0], w), lerp64(x0[1], x1[1], w), lerp64(x0[2], x1[2], w),
                                                        lerp64(x0[3], x1[3], w));
                        bad += row.at(w) != want;
                    }
                }
    return bad;
}

// finite floats x with bit patterns in [lo, hi) for which ztc::div255(x) differs bitwise from the division x / 255.0f
// (-0, whose documented quotient is +0, excepted)
__attribute__((visibility("default"))) uint64_t emu_div255_mismatches(uint64_t lo, uint64_t hi) {
    volatile float d = 255.0f;  // a runtime divisor: the host compiler emits a true division
    uint64_t bad = 0;
    for (uint64_t u = lo; u < hi; u++) {
        float x;
        const uint32_t b = (uint32_t)u;
        std::memcpy(&x, &b, 4);
        if (!std::isfinite(x) || b == 0x80000000u) continue;
        const float a = x / d, m = div255(x);
        if (std::memcmp(&a, &m, 4) != 0) bad++;
    }
    return bad;
}

// floats u with bit patterns in [lo, hi) for which ztc::bc6_nearest(u) differs from the reference's rule as written
// (zap_tex.h:841-851): g truncated as x86 does, candidates g - 1, g, g + 1 clamped, the first of least distance
__attribute__((visibility("default"))) uint64_t emu_bc6_nearest_mismatches(uint64_t lo, uint64_t hi) {
    uint64_t bad = 0;
    for (uint64_t b = lo; b < hi; b++) {
        const float u = u_as_f((uint32_t)b);
        const int g = f2i_x86((u - 32.0f) / 64.0f + 0.5f);
        int best = 0;
        float bd = 1e30f;
        for (int k = 0; k < 3; k++) {
            const int e = clampi(around(g, k), 0, 1023);
            const float d = std::fabs((float)bc6_unq(e) - u);
            if (d < bd) { bd = d; best = e; }
        }
        if (bc6_nearest(u) != best) bad++;
    }
    return bad;
}

// (x, n) pairs, x an integer in [0, 2^24) and the given n, for which ztc::div_small(x, n, 1 / n) differs bitwise from
// the division x / n
__attribute__((visibility("default"))) uint64_t emu_div_small_mismatches(int n) {
    volatile float dv = (float)n;  // a runtime divisor: the host compiler emits true divisions
    const float ni = 1.0f / dv;
    uint64_t bad = 0;
    for (uint32_t v = 0; v < (1u << 24); v++) {
        const float x = (float)v, a = x / dv, m = div_small(x, dv, ni);
        if (std::memcmp(&a, &m, 4) != 0) bad++;
    }
    return bad;
}

}  // extern "C"

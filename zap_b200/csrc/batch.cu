// batch.cu - batched encoder: thousands of textures of uneven size, full mip chains, mixed formats.
//
// No single reference counterpart: it replaces the caller loop of zap.c:330-342 (per level: zap_bc_encode, then
// zap_mip_next) run over many textures. A batch is planned once (zap_tex_cuda_batch_create):
//   - mip levels 1..L-1 of every texture go to one device buffer; depth d of all textures is built by one
//     persistent launch over tiles of 256 output texel pairs (level-synchronous, L-1 launches in all);
//   - every (texture, level) is cut into tiles of consecutive blocks; one persistent launch per format class pulls
//     tiles from a device counter (largest levels first); for BC7 that launch runs mode 6 and lists the blocks it
//     does not finish in one batch-wide work list, which a second persistent launch (8-lane groups, modes 5 / 1)
//     drains;
//   - an optional autotuner times, per format class, on the batch's own levels: the CTA size (64/128/256 threads),
//     the register cap (the single-image kernels' minimum resident CTAs, or a looser one), the blocks per tile
//     (1, 2 or 4 CTAs' worth, a CTA running its tile in chunks), the tile shape (a row strip of consecutive blocks
//     or a 2-D tile of block rows), and for BC7 the grid of the modes-5/1 launches (1 or 2 CTAs per SM, or as many
//     as fit); one knob at a time, in that order, each keeping the fastest setting;
//   - the whole sequence (counter resets, mip launches, concurrent encode launches) is captured into one CUDA
//     graph; zap_tex_cuda_batch_run is one graph launch.
// zap_tex_cuda_batch_run_plain issues the same work as one plain launch per texture and per level (the
// per-texture path a caller would write), for comparison; both produce the same bytes.
#include <algorithm>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/zap_tex_cuda.h"
#include "ztc_common.cuh"
#include "ztc_internal.h"

namespace {

constexpr int kClasses = 5;  // BC1, BC3, BC4, BC5, BC7 (format id == class id)
constexpr int kHardCounter = 8;  // d_counters slots of the BC7 work-list lengths: after mode 6 (8), after mode 5 (9)
const int kCtaChoices[3] = {64, 128, 256};
const int kTileMult[3] = {1, 2, 4};  // blocks per tile = CTA size x this

// one format class's launch configuration (the autotuner's knobs)
struct ClassPlan {
    int cta = 128, regs = 0, mult = 1, shape = 0;  // shape 0: row strip, 1: 2-D tile
    int tile_w = 0, tile_h = 0;                     // the 2-D tile in blocks
};

struct HostLevel {
    int item, level, w, h, fmt, srgb;
    const uint8_t *src;
    size_t pitch;
    uint8_t *dst;
    int bw, bh;
};

size_t block_bytes(int fmt) { return (fmt == ZTC_BC1 || fmt == ZTC_BC4) ? 8 : 16; }
size_t level_bytes(int w, int h, int fmt) { return (size_t)((w + 3) / 4) * (size_t)((h + 3) / 4) * block_bytes(fmt); }
int full_levels(int w, int h) { return zap_tex_cuda_mip_levels(w, h); }

}  // namespace

struct zap_tex_cuda_batch {
    int device = 0, sms = 148;
    cudaStream_t stream = nullptr, side[kClasses] = {};
    cudaEvent_t fork = nullptr, join[kClasses] = {};
    std::vector<HostLevel> levels;          // every (item, level), item-major
    std::vector<std::vector<ztc::BatchMip>> mips;  // per depth d >= 1
    uint8_t *mip_buf = nullptr;
    size_t mip_bytes = 0;
    ztc::BatchLevel *d_levels = nullptr;
    ztc::BatchTile *d_tiles[kClasses] = {};
    int ntiles[kClasses] = {}, grid[kClasses] = {};
    ClassPlan plan[kClasses];
    std::vector<ztc::BatchMip *> d_mips;
    std::vector<ztc::BatchMipTile *> d_mip_tiles;
    std::vector<int> n_mip_tiles;
    uint32_t *d_counters = nullptr;          // [f]: tile counter of class f; [kHardCounter]: BC7 work-list length
    uint2 *d_hard_items = nullptr;           // BC7 work lists: (batch-wide block id, SSE) after mode 6, then after mode 5
    uint32_t *d_bc7_bases = nullptr;         // first batch-wide id of each BC7 level, ascending
    int *d_bc7_level_of = nullptr;           // ... and that level's index in d_levels
    int n_bc7_levels = 0, hard_grid = 1, hard_per_sm = 1;
    ztc::SrgbTables *d_srgb = nullptr;
    void *plain_scratch = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::string tune_log[kClasses];  // the autotuner's timings, per knob
    long pixels = 0, blocks[kClasses] = {};
};

namespace {

int cuda_err(cudaError_t e, const char *what) {
    cudaGetLastError();
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    return ztc_set_error(e == cudaErrorMemoryAllocation ? ZTC_ERR_NO_MEMORY : ZTC_ERR_CUDA, m.c_str());
}
#define BCHECK(expr, what)                                 \
    do {                                                   \
        cudaError_t e_ = (expr);                           \
        if (e_ != cudaSuccess) return cuda_err(e_, what);  \
    } while (0)

// the tiles of class f under plan p, largest levels first: row strips of cta x mult consecutive blocks, or 2-D
// tiles of that many blocks (tile_w x tile_h, clipped at the level's edges)
std::vector<ztc::BatchTile> make_tiles(const zap_tex_cuda_batch *b, int f, const ClassPlan &p) {
    std::vector<int> order;
    for (int i = 0; i < (int)b->levels.size(); i++) if (b->levels[i].fmt == f) order.push_back(i);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return (long)b->levels[x].bw * b->levels[x].bh > (long)b->levels[y].bw * b->levels[y].bh;
    });
    const int per_tile = p.cta * p.mult;
    std::vector<ztc::BatchTile> t;
    for (int i : order) {
        const int bw = b->levels[i].bw, bh = b->levels[i].bh, n = bw * bh;
        if (p.shape == 0 || bw <= p.tile_w) {  // strips (a level no wider than a tile: its strips are its rows)
            for (int first = 0; first < n; first += per_tile) t.push_back({i, first, std::min(per_tile, n - first), 0});
            continue;
        }
        for (int by = 0; by < bh; by += p.tile_h)
            for (int bx = 0; bx < bw; bx += p.tile_w) {
                const int tw = std::min(p.tile_w, bw - bx), th = std::min(p.tile_h, bh - by);
                t.push_back({i, by * bw + bx, tw * th, tw});
            }
    }
    return t;
}

int upload_tiles(zap_tex_cuda_batch *b, int f, ClassPlan p) {
    int lg = 0;
    while ((1 << (lg + 1)) <= p.cta * p.mult) lg++;
    p.tile_w = 1 << ((lg + 1) / 2);  // 2-D tiles as square as a power of two allows (wider than high)
    p.tile_h = (p.cta * p.mult) / p.tile_w;
    std::vector<ztc::BatchTile> t = make_tiles(b, f, p);
    if (b->d_tiles[f]) { cudaFree(b->d_tiles[f]); b->d_tiles[f] = nullptr; }
    b->ntiles[f] = (int)t.size();
    b->plan[f] = p;
    if (t.empty()) return ZTC_OK;
    BCHECK(ztc_malloc((void **)&b->d_tiles[f], t.size() * sizeof(ztc::BatchTile)), "cudaMalloc(tiles)");
    BCHECK(cudaMemcpy(b->d_tiles[f], t.data(), t.size() * sizeof(ztc::BatchTile), cudaMemcpyHostToDevice), "upload tiles");
    const void *fn = f == ZTC_BC7 ? ztc_batch_bc7_kernel_fn(p.cta, p.regs) : ztc_batch_bcn_kernel_fn(f, p.cta, p.regs);
    int per_sm = 1;
    BCHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, p.cta, 0), "occupancy");
    b->grid[f] = std::max(1, std::min(b->ntiles[f], per_sm * b->sms));
    return ZTC_OK;
}

cudaError_t launch_encode(zap_tex_cuda_batch *b, int f, cudaStream_t s) {
    if (!b->ntiles[f]) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(b->d_counters + f, 0, sizeof(uint32_t), s);
    if (e != cudaSuccess) return e;
    if (f == ZTC_BC7) {
        uint32_t *hard_count = b->d_counters + kHardCounter;
        if ((e = cudaMemsetAsync(hard_count, 0, 2 * sizeof(uint32_t), s)) != cudaSuccess) return e;
        {
            ztc::TraceScope tr("batch_bc7_mode6", s);
            ztc::trace_units(b->blocks[f]);
            e = ztc_launch_batch_bc7_mode6(b->plan[f].cta, b->plan[f].regs, b->grid[f], b->d_levels, b->d_tiles[f], b->ntiles[f],
                                           b->d_counters + f, hard_count, b->d_hard_items, s);
            if (e != cudaSuccess) return e;
        }
        ztc::TraceScope tr("batch_bc7_modes51", s);
        ztc::trace_units_dev(hard_count, s);
        return ztc_launch_batch_bc7_hard(b->hard_grid, b->d_levels, b->d_bc7_bases, b->d_bc7_level_of, b->n_bc7_levels, hard_count,
                                         b->d_hard_items, hard_count + 1, b->d_hard_items + b->blocks[f], s);
    }
    ztc::TraceScope tr(f == ZTC_BC1 ? "batch_bc1" : f == ZTC_BC3 ? "batch_bc3" : f == ZTC_BC4 ? "batch_bc4" : "batch_bc5", s);
    ztc::trace_units(b->blocks[f]);
    return ztc_launch_batch_bcn(f, b->plan[f].cta, b->plan[f].regs, b->grid[f], b->d_levels, b->d_tiles[f], b->ntiles[f],
                                b->d_counters + f, s);
}

cudaError_t launch_mips(zap_tex_cuda_batch *b, cudaStream_t s) {
    for (size_t d = 0; d < b->d_mips.size(); d++) {
        if (!b->n_mip_tiles[d]) continue;
        ztc::TraceScope tr("batch_mip", s);
        long units = 0;
        for (auto &m : b->mips[d]) units += (long)m.nw * m.nh;
        ztc::trace_units(units);
        int grid = std::max(1, std::min(b->n_mip_tiles[d], b->sms * 8));
        cudaError_t e = ztc_launch_batch_mip(grid, b->d_mips[d], b->d_mip_tiles[d], b->n_mip_tiles[d], b->d_srgb, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// the batch's whole sequence on one stream, encode classes forked onto side streams
cudaError_t enqueue_all(zap_tex_cuda_batch *b, cudaStream_t s) {
    cudaError_t e = launch_mips(b, s);
    if (e != cudaSuccess) return e;
    if ((e = cudaEventRecord(b->fork, s)) != cudaSuccess) return e;
    for (int f = 0; f < kClasses; f++) {
        if (!b->ntiles[f]) continue;
        if ((e = cudaStreamWaitEvent(b->side[f], b->fork, 0)) != cudaSuccess) return e;
        if ((e = launch_encode(b, f, b->side[f])) != cudaSuccess) return e;
        if ((e = cudaEventRecord(b->join[f], b->side[f])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, b->join[f], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Coordinate search per format class on the batch's own levels: each knob in turn (CTA size, register cap,
// blocks per tile, tile shape; BC7: then the modes-5/1 grid) is timed at each of its settings with the others held,
// and the fastest is kept. One warm-up launch per setting, then one timed launch (CUDA events).
int autotune(zap_tex_cuda_batch *b) {
    cudaEvent_t e0, e1;
    BCHECK(cudaEventCreate(&e0), "event");
    BCHECK(cudaEventCreate(&e1), "event");
    int st = launch_mips(b, b->stream) == cudaSuccess ? ZTC_OK : cuda_err(cudaGetLastError(), "mip launch");
    auto time_class = [&](int f, double &ms) -> int {
        cudaError_t e = launch_encode(b, f, b->stream);  // warm-up
        if (e == cudaSuccess) e = cudaEventRecord(e0, b->stream);
        if (e == cudaSuccess) e = launch_encode(b, f, b->stream);
        if (e == cudaSuccess) e = cudaEventRecord(e1, b->stream);
        if (e == cudaSuccess) e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return cuda_err(e, "autotune");
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        ms = t;
        return ZTC_OK;
    };
    char buf[96];
    for (int f = 0; f < kClasses && !st; f++) {
        bool any = false;
        for (auto &l : b->levels) any |= l.fmt == f;
        if (!any) continue;
        ClassPlan best;
        std::string log;
        for (int knob = 0; knob < 4 && !st; knob++) {
            const int nset = knob == 1 || knob == 3 ? 2 : 3;
            ClassPlan keep = best;
            double best_ms = 1e30;
            log += knob == 0 ? " cta" : knob == 1 ? " regs" : knob == 2 ? " tile_ctas" : " shape";
            for (int k = 0; k < nset && !st; k++) {
                ClassPlan p = best;
                if (knob == 0) p.cta = kCtaChoices[k];
                else if (knob == 1) p.regs = k;
                else if (knob == 2) p.mult = kTileMult[k];
                else p.shape = k;
                double ms = 0;
                if (!(st = upload_tiles(b, f, p)) && !(st = time_class(f, ms))) {
                    std::snprintf(buf, sizeof buf, "%s%.3f", k ? "/" : ":", ms);
                    log += buf;
                    if (ms < best_ms) { best_ms = ms; keep = p; }
                }
            }
            best = keep;
        }
        if (!st) st = upload_tiles(b, f, best);
        if (f == ZTC_BC7 && !st && b->n_bc7_levels) {  // the modes-5/1 grid: 1, 2 or all resident CTAs per SM
            const int choices[3] = {1, 2, b->hard_per_sm};
            int best_grid = b->hard_grid;
            double best_ms = 1e30;
            log += " hard_ctas_per_sm";
            for (int k = 0; k < 3 && !st; k++) {
                if (k == 2 && (choices[2] <= 2)) break;
                b->hard_grid = choices[k] * b->sms;
                double ms = 0;
                if (!(st = time_class(f, ms))) {
                    std::snprintf(buf, sizeof buf, "%s%.3f", k ? "/" : ":", ms);
                    log += buf;
                    if (ms < best_ms) { best_ms = ms; best_grid = b->hard_grid; }
                }
            }
            b->hard_grid = best_grid;
        }
        b->tune_log[f] = "tuned_ms" + log;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}

}  // namespace

extern "C" {

size_t zap_tex_cuda_batch_item_bytes(int w, int h, int fmt, int levels) {
    if (w < 1 || h < 1 || fmt < ZTC_BC1 || fmt > ZTC_BC7) return 0;
    int L = levels <= 0 ? full_levels(w, h) : std::min(levels, full_levels(w, h));
    size_t total = 0;
    for (int l = 0; l < L; l++) {
        total += level_bytes(w, h, fmt);
        w = w > 1 ? w / 2 : 1; h = h > 1 ? h / 2 : 1;
    }
    return total;
}

int zap_tex_cuda_batch_destroy(zap_tex_cuda_batch *b) {
    ZTC_NVTX();
    if (!b) return ZTC_OK;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (int f = 0; f < kClasses; f++) {
        cudaFree(b->d_tiles[f]);
        if (b->side[f]) cudaStreamDestroy(b->side[f]);
        if (b->join[f]) cudaEventDestroy(b->join[f]);
    }
    for (auto p : b->d_mips) cudaFree(p);
    for (auto p : b->d_mip_tiles) cudaFree(p);
    cudaFree(b->mip_buf); cudaFree(b->d_levels); cudaFree(b->d_counters); cudaFree(b->d_srgb); cudaFree(b->plain_scratch);
    cudaFree(b->d_hard_items); cudaFree(b->d_bc7_bases); cudaFree(b->d_bc7_level_of);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    cudaSetDevice(prev);
    return ZTC_OK;
}

int zap_tex_cuda_batch_create(zap_tex_cuda_ctx *ctx, const zap_tex_cuda_item *items, int n, int flags, zap_tex_cuda_batch **out) {
    ZTC_NVTX();
    if (!out || !items || n < 1) return ztc_set_error(ZTC_ERR_INVALID_ARG, "batch: null items / out or n < 1");
    *out = nullptr;
    for (int i = 0; i < n; i++) {
        const zap_tex_cuda_item &it = items[i];
        if (!it.src || !it.dst || it.w < 1 || it.h < 1 || it.w > (1 << 16) || it.h > (1 << 16) || it.stride < (size_t)it.w * 4)
            return ztc_set_error(ZTC_ERR_INVALID_ARG, ("batch item " + std::to_string(i) + ": bad pointer, size or stride").c_str());
        if (it.fmt < ZTC_BC1 || it.fmt > ZTC_BC7)
            return ztc_set_error(ZTC_ERR_UNSUPPORTED, ("batch item " + std::to_string(i) + ": format must be BC1..BC7").c_str());
        if ((uintptr_t)it.dst % block_bytes(it.fmt))  // blocks are stored 8 or 16 bytes at a time
            return ztc_set_error(ZTC_ERR_INVALID_ARG, ("batch item " + std::to_string(i) + ": dst not aligned to the block size").c_str());
    }
    int st0 = ztc_ctx_activate(ctx);  // makes the context's device current (NULL: the current device's default context)
    if (st0) return st0;
    int dev = 0;
    cudaGetDevice(&dev);
    zap_tex_cuda_batch *b = new (std::nothrow) zap_tex_cuda_batch();
    if (!b) return ztc_set_error(ZTC_ERR_NO_MEMORY, "batch allocation");
    b->device = dev;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
    auto fail = [&](int st) { zap_tex_cuda_batch_destroy(b); return st; };
#define BTRY(expr, what)                                              \
    do {                                                              \
        cudaError_t e_ = (expr);                                      \
        if (e_ != cudaSuccess) return fail(cuda_err(e_, what));       \
    } while (0)
    BTRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "stream");
    BTRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "event");
    for (int f = 0; f < kClasses; f++) {
        BTRY(cudaStreamCreateWithFlags(&b->side[f], cudaStreamNonBlocking), "stream");
        BTRY(cudaEventCreateWithFlags(&b->join[f], cudaEventDisableTiming), "event");
    }
    // ---- plan levels and the mip buffer
    std::vector<size_t> mip_off;  // per (item, level >= 1) in b->levels order; offsets into mip_buf
    size_t mip_total = 0;
    int max_levels = 1;
    for (int i = 0; i < n; i++) {
        const zap_tex_cuda_item &it = items[i];
        int L = it.levels <= 0 ? full_levels(it.w, it.h) : std::min(it.levels, full_levels(it.w, it.h));
        max_levels = std::max(max_levels, L);
        int w = it.w, h = it.h;
        size_t out_off = 0;
        for (int l = 0; l < L; l++) {
            int srgb = (it.fmt == ZTC_BC4 || it.fmt == ZTC_BC5) ? 0 : (it.srgb != 0);  // channel data is never sRGB (zap.c:325)
            HostLevel hl{i, l, w, h, it.fmt, srgb, nullptr, 0, it.dst + out_off, (w + 3) / 4, (h + 3) / 4};
            mip_off.push_back(mip_total);
            if (l > 0) mip_total += ((size_t)w * h * 4 + 15) & ~(size_t)15;
            b->levels.push_back(hl);
            b->pixels += (long)w * h;
            b->blocks[it.fmt] += (long)((w + 3) / 4) * ((h + 3) / 4);
            out_off += level_bytes(w, h, it.fmt);
            w = w > 1 ? w / 2 : 1; h = h > 1 ? h / 2 : 1;
        }
    }
    b->mip_bytes = mip_total;
    if (mip_total) BTRY(ztc_malloc((void **)&b->mip_buf, mip_total), "cudaMalloc(mip levels)");
    for (size_t k = 0; k < b->levels.size(); k++) {
        HostLevel &hl = b->levels[k];
        if (hl.level == 0) { hl.src = items[hl.item].src; hl.pitch = items[hl.item].stride; }
        else { hl.src = b->mip_buf + mip_off[k]; hl.pitch = (size_t)hl.w * 4; }
    }
    // ---- mip work per depth
    b->mips.resize(max_levels > 1 ? max_levels - 1 : 0);
    for (size_t k = 0; k < b->levels.size(); k++) {
        const HostLevel &hl = b->levels[k];
        if (hl.level == 0) continue;
        const HostLevel &prev = b->levels[k - 1];
        b->mips[hl.level - 1].push_back({prev.src, (uint8_t *)hl.src, prev.pitch, hl.pitch, prev.w, prev.h, hl.w, hl.h, hl.srgb, 0});
    }
    for (auto &depth : b->mips) {
        std::vector<ztc::BatchMipTile> tiles;
        for (int m = 0; m < (int)depth.size(); m++) {
            int pairs = ((depth[m].nw + 1) / 2) * depth[m].nh;
            for (int first = 0; first < pairs; first += 256) tiles.push_back({m, first, std::min(256, pairs - first), 0});
        }
        ztc::BatchMip *dm = nullptr;
        ztc::BatchMipTile *dt = nullptr;
        BTRY(ztc_malloc((void **)&dm, std::max<size_t>(1, depth.size()) * sizeof(ztc::BatchMip)), "cudaMalloc(mips)");
        b->d_mips.push_back(dm);
        BTRY(ztc_malloc((void **)&dt, std::max<size_t>(1, tiles.size()) * sizeof(ztc::BatchMipTile)), "cudaMalloc(mip tiles)");
        b->d_mip_tiles.push_back(dt);
        b->n_mip_tiles.push_back((int)tiles.size());
        if (!depth.empty()) BTRY(cudaMemcpy(dm, depth.data(), depth.size() * sizeof(ztc::BatchMip), cudaMemcpyHostToDevice), "upload mips");
        if (!tiles.empty()) BTRY(cudaMemcpy(dt, tiles.data(), tiles.size() * sizeof(ztc::BatchMipTile), cudaMemcpyHostToDevice), "upload mip tiles");
    }
    // ---- level descriptors, tables, counters
    std::vector<ztc::BatchLevel> dl;
    std::vector<uint32_t> bc7_bases;
    std::vector<int> bc7_level_of;
    size_t max_blocks = 1, bc7_blocks = 0;
    for (size_t k = 0; k < b->levels.size(); k++) {
        const HostLevel &hl = b->levels[k];
        const size_t nb = (size_t)hl.bw * hl.bh;
        uint32_t gbase = 0;
        if (hl.fmt == ZTC_BC7) {
            gbase = (uint32_t)bc7_blocks;
            bc7_bases.push_back(gbase);
            bc7_level_of.push_back((int)k);
            bc7_blocks += nb;
        }
        dl.push_back({hl.src, hl.dst, hl.pitch, hl.w, hl.h, hl.bw, hl.fmt, gbase, 0});
        max_blocks = std::max(max_blocks, nb);
    }
    if (bc7_blocks >= ((size_t)1 << 32))
        return fail(ztc_set_error(ZTC_ERR_INVALID_ARG, "batch: more than 2^32 - 1 BC7 blocks in one batch; split it"));
    BTRY(ztc_malloc((void **)&b->d_levels, dl.size() * sizeof(ztc::BatchLevel)), "cudaMalloc(levels)");
    BTRY(cudaMemcpy(b->d_levels, dl.data(), dl.size() * sizeof(ztc::BatchLevel), cudaMemcpyHostToDevice), "upload levels");
    if (bc7_blocks) {  // BC7 work list: room for every BC7 block of the batch
        b->n_bc7_levels = (int)bc7_bases.size();
        BTRY(ztc_malloc((void **)&b->d_hard_items, 2 * bc7_blocks * sizeof(uint2)), "cudaMalloc(BC7 work lists)");
        BTRY(ztc_malloc((void **)&b->d_bc7_bases, bc7_bases.size() * sizeof(uint32_t)), "cudaMalloc(BC7 level bases)");
        BTRY(ztc_malloc((void **)&b->d_bc7_level_of, bc7_level_of.size() * sizeof(int)), "cudaMalloc(BC7 level map)");
        BTRY(cudaMemcpy(b->d_bc7_bases, bc7_bases.data(), bc7_bases.size() * sizeof(uint32_t), cudaMemcpyHostToDevice), "upload BC7 bases");
        BTRY(cudaMemcpy(b->d_bc7_level_of, bc7_level_of.data(), bc7_level_of.size() * sizeof(int), cudaMemcpyHostToDevice),
             "upload BC7 level map");
        int per_sm = 1;
        BTRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, ztc_batch_bc7_hard_kernel_fn(), 128, 0), "occupancy");
        b->hard_per_sm = std::max(1, per_sm);
        b->hard_grid = b->hard_per_sm * b->sms;
    }
    ztc::SrgbTables tables;
    ztc::srgb_tables_host(tables);
    BTRY(ztc_malloc((void **)&b->d_srgb, sizeof tables), "cudaMalloc(srgb)");
    BTRY(cudaMemcpy(b->d_srgb, &tables, sizeof tables, cudaMemcpyHostToDevice), "upload srgb");
    BTRY(ztc_malloc((void **)&b->d_counters, 64 * sizeof(uint32_t)), "cudaMalloc(counters)");
    BTRY(ztc_malloc((void **)&b->plain_scratch, ztc::bc7_scratch_bytes(max_blocks)), "cudaMalloc(plain scratch)");
    // ---- tiles (autotuned or 128 blocks per CTA)
    int st = ZTC_OK;
    if (flags & ZTC_BATCH_AUTOTUNE) st = autotune(b);
    else
        for (int f = 0; f < kClasses && !st; f++) {
            ClassPlan p;
            p.cta = (flags & ZTC_BATCH_CTA_64) ? 64 : (flags & ZTC_BATCH_CTA_256) ? 256 : 128;
            p.regs = (flags & ZTC_BATCH_REGS_LOOSE) ? 1 : 0;
            p.mult = (flags & ZTC_BATCH_TILE_X4) ? 4 : (flags & ZTC_BATCH_TILE_X2) ? 2 : 1;
            p.shape = (flags & ZTC_BATCH_TILES_2D) ? 1 : 0;
            st = upload_tiles(b, f, p);
        }
    if (st) return fail(st);
    // ---- one CUDA graph for the whole batch
    if (!(flags & ZTC_BATCH_NO_GRAPH)) {
        BTRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
        cudaError_t e = enqueue_all(b, b->stream);
        cudaGraph_t g = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(b->stream, &g);
        if (e != cudaSuccess || e2 != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return fail(cuda_err(e != cudaSuccess ? e : e2, "graph capture"));
        }
        b->graph = g;
        BTRY(cudaGraphInstantiate(&b->exec, g, 0), "graph instantiate");
    }
    BTRY(cudaStreamSynchronize(b->stream), "batch create");
    *out = b;
    return ZTC_OK;
#undef BTRY
}

int zap_tex_cuda_batch_run(zap_tex_cuda_batch *b, void *stream) {
    ZTC_NVTX();
    if (!b) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null batch");
    BCHECK(cudaSetDevice(b->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    if (b->exec) {
        ztc::TraceScope tr("batch_graph", s);
        ztc::trace_units(b->pixels);
        BCHECK(cudaGraphLaunch(b->exec, s), "graph launch");
        return ZTC_OK;
    }
    BCHECK(enqueue_all(b, s), "batch launch");
    return ZTC_OK;
}

int zap_tex_cuda_batch_run_plain(zap_tex_cuda_batch *b, void *stream) {
    if (!b) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null batch");
    BCHECK(cudaSetDevice(b->device), "cudaSetDevice");
    cudaStream_t s = (cudaStream_t)stream;
    for (size_t k = 0; k < b->levels.size(); k++) {
        const HostLevel &hl = b->levels[k];
        if (hl.level > 0) {  // this level's texels from the previous level: one plain mip launch
            const HostLevel &prev = b->levels[k - 1];
            BCHECK(ztc_launch_mip(prev.src, prev.w, prev.h, prev.pitch, hl.srgb, (uint8_t *)hl.src, hl.pitch, s), "mip launch");
        }
        ztc::SrcU8 src{hl.src, hl.pitch, hl.w, hl.h, 4, (((uintptr_t)hl.src | hl.pitch) & 15u) == 0};
        cudaError_t e = hl.fmt == ZTC_BC7 ? ztc_launch_bc7(src, 0, hl.bh, hl.dst, b->plain_scratch, s)
                                          : ztc_launch_bcn(hl.fmt, src, 0, hl.bh, hl.dst, s);
        BCHECK(e, "encode launch");
    }
    return ZTC_OK;
}

int zap_tex_cuda_batch_info(zap_tex_cuda_batch *b, char *buf, size_t cap) {
    if (!b) return ztc_set_error(ZTC_ERR_INVALID_ARG, "null batch");
    std::string s;
    char line[256];
    std::snprintf(line, sizeof line, "levels %zu pixels %ld mip_bytes %zu graph %d\n", b->levels.size(), b->pixels, b->mip_bytes, b->exec != nullptr);
    s += line;
    const char *names[kClasses] = {"bc1", "bc3", "bc4", "bc5", "bc7"};
    for (int f = 0; f < kClasses; f++) {
        if (!b->ntiles[f]) continue;
        const ClassPlan &p = b->plan[f];
        char shape[32];
        if (p.shape) std::snprintf(shape, sizeof shape, "2d_%dx%d", p.tile_w, p.tile_h);
        else std::snprintf(shape, sizeof shape, "strip");
        std::snprintf(line, sizeof line, "%s tiles %d cta %d regs %s blocks_per_tile %d shape %s grid %d", names[f], b->ntiles[f], p.cta,
                      p.regs ? "loose" : "tight", p.cta * p.mult, shape, b->grid[f]);
        s += line;
        if (f == ZTC_BC7) {
            std::snprintf(line, sizeof line, " hard_grid %d", b->hard_grid);
            s += line;
        }
        if (!b->tune_log[f].empty()) s += " " + b->tune_log[f];
        s += "\n";
    }
    if (buf && cap) { std::strncpy(buf, s.c_str(), cap - 1); buf[cap - 1] = 0; }
    return (int)s.size();
}

}  // extern "C"

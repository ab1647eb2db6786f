// dl_render.cu — host orchestration of the renderer's device pipeline.
//
// One frame (any number of views of one device-resident scene):
//   project_k -> depth sort (4 onesweep passes) -> emit_k -> pair_digits_k
//   -> pair sort (1-3 onesweep passes; the last one lowers the tile offsets,
//      bound_init_k / bound_fill_k around it) -> rasterize_k
// No host synchronisation happens inside the frame: every size a later stage
// needs (visible count, pair count, tile offsets) stays in device memory.
// Pair buffers are sized from an upper bound; if a frame overflows them the
// emit kernel flags it, the host grows the buffers and re-runs the pair stages.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>

#include "dl_internal.h"
#include "dl_render_kernels.cuh"
#include "dl_sort.cuh"

namespace {

constexpr int kScratchWords = 32;
enum {
    SC_DEPTH_CTR = 0,      // 4 counters
    SC_EMIT_CTR = 4,
    SC_PAIR_CTR = 5,       // 4 counters
    SC_WORK_CTR = 9,
    SC_ERR = 10,
    SC_DEPTH_TILES = 11,
    SC_PAIR_TILES = 12,
    SC_OVF = 13,
    SC_SCHED_CTR = 14,     // 4 counters
    SC_SCHED_TILES = 18,
    SC_DEPTH_TILES2 = 19,  // tiles of the depth sort after its first pass
    SC_RASTER_CTR = 20     // kReadBackGroups work counters of view-range rasterizer launches
};

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

int ensure_pinned(void** p, size_t* cap, size_t need) {
    if (need <= *cap && *p) return DL_OK;
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    *cap = 0;
    if (cudaMallocHost(p, need) != cudaSuccess) {
        *p = nullptr;
        dl_set_error("cudaMallocHost failed");
        return DL_E_OOM;
    }
    *cap = need;
    return DL_OK;
}

template <int BITS>
void launch_pass(const dlsort::Pass& p, uint32_t grid, cudaStream_t st, const dlsort::Bound& b) {
    if (p.drop_max) dlsort::pass_k<BITS, true><<<dlsort::pass_grid(grid), dlsort::kThreads, 0, st>>>(p);
    else if (b.bound) dlsort::pass_k<BITS, false, true><<<dlsort::pass_grid(grid), dlsort::kThreads, 0, st>>>(p, b);
    else dlsort::pass_k<BITS><<<dlsort::pass_grid(grid), dlsort::kThreads, 0, st>>>(p);
}

void launch_pass_bits(int bits, const dlsort::Pass& p, uint32_t grid, cudaStream_t st,
                      const dlsort::Bound& b = dlsort::Bound()) {
    if (bits == 8) launch_pass<8>(p, grid, st, b);
    else if (bits == 7) launch_pass<7>(p, grid, st, b);
    else launch_pass<6>(p, grid, st, b);
}

// SH in 16 bits, repacked per Gaussian: in[g][c * M + k] (channel-major, as
// SplatData) -> out[g][3 k + c], blocks of P = round_up(3M, 8) halves, zero pads.
__global__ void sh_to_half_k(const float* in, uint16_t* out, uint64_t n, int M, int P, int kind) {
    const uint64_t total = n * (uint64_t)P;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t g = i / P;
        const int j = (int)(i - g * P);
        float f = 0.0f;
        if (j < 3 * M) f = in[g * 3 * M + (uint64_t)((j % 3) * M + j / 3)];
        out[i] = kind == 1 ? __half_as_ushort(__float2half_rn(f)) : __bfloat16_as_ushort(__float2bfloat16_rn(f));
    }
}


}  // namespace

int dl_make_view(const dl_camera* cam, const float bg[4], uint32_t maxCov, DlView* v) {
    if (!cam) { dl_set_error("camera is NULL"); return DL_E_INVALID_ARG; }
    if (cam->projection != DL_PINHOLE && cam->projection != DL_EQUIRECT) {
        dl_set_error("camera.projection must be DL_PINHOLE or DL_EQUIRECT");
        return DL_E_INVALID_ARG;
    }
    std::memset(v, 0, sizeof(*v));
    std::memcpy(v->view, cam->view, sizeof(v->view));
    // src/render/camera.ts:32-46 in f64, stored into the f32 uniform (pipeline.ts:490-497)
    const double focal = (double)cam->height / (2.0 * std::tan(cam->fov_y / 2.0));
    v->width = (float)cam->width;
    v->height = (float)cam->height;
    v->focal = (float)focal;
    v->cx = (float)((double)cam->width / 2.0);
    v->cy = (float)((double)cam->height / 2.0);
    v->near_f = (float)cam->near_plane;
    v->far_f = (float)cam->far_plane;
    v->near_d = cam->near_plane;
    v->far_d = cam->far_plane;
    v->W = cam->width;
    v->H = cam->height;
    v->tilesX = (cam->width + DL_TILE - 1) / DL_TILE;
    v->tilesY = (cam->height + DL_TILE - 1) / DL_TILE;
    if (v->tilesX > 0x7fffu || v->tilesY > 0x7fffu || (uint64_t)v->tilesX * v->tilesY >= (1u << 20)) {
        dl_set_error("image too large: at most 2^20 16x16 tiles and 32767 tiles per axis");
        return DL_E_CAPACITY;
    }
    v->numTiles = v->tilesX * v->tilesY;
    v->projection = cam->projection;
    v->maxCoverage = maxCov;
    v->tileW = DL_TILE;
    v->tileH = DL_TILE;
    v->refTilesX = v->tilesX;
    v->refTilesY = v->tilesY;
    v->binCap = maxCov;
    const float dflt[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    for (int k = 0; k < 4; k++) v->bg[k] = bg ? bg[k] : dflt[k];
    return DL_OK;
}

int dl_upload_convert_sh(const DlUploadChunks* up, uint32_t g0, uint32_t g1, cudaStream_t st, uint64_t* launches) {
    if (!up->sh_dst || g1 <= g0) return DL_OK;
    sh_to_half_k<<<std::min<uint32_t>((g1 - g0 + 31) / 32, 1024), 256, 0, st>>>(
        up->sh_src + 3ull * up->sh_M * g0, up->sh_dst + (uint64_t)up->sh_P * g0, g1 - g0, up->sh_M, up->sh_P,
        up->sh_kind);
    if (launches) (*launches)++;
    DL_CK(cudaGetLastError());
    return DL_OK;
}

int dl_upload_scene(dl_scene* s, const dl_splats* d, int precision, cudaStream_t st, DlUploadChunks* chunks) {
    if (!d) { dl_set_error("splats is NULL"); return DL_E_INVALID_ARG; }
    if (d->sh_bands < 0 || d->sh_bands > 3) { dl_set_error("sh_bands must be 0..3"); return DL_E_INVALID_ARG; }
    if (d->count >= (1ull << 30)) { dl_set_error("at most 2^30 - 1 splats"); return DL_E_CAPACITY; }
    const uint64_t n = d->count;
    if (n > 0 && (!d->positions || !d->rotations || !d->log_scales || !d->opacity_logits || !d->colors_dc)) {
        dl_set_error("splats: a required array is NULL");
        return DL_E_INVALID_ARG;
    }
    if (precision < DL_PREC_F32 || precision > DL_PREC_BF16) { dl_set_error("bad precision"); return DL_E_INVALID_ARG; }
    // SH coefficients absent: the reference packs zeros (preprocess.ts:127-135), which adds
    // exactly zero to the colour, so the splats render as band 0.
    const int bands = d->colors_sh ? d->sh_bands : 0;
    const int M = bands == 0 ? 0 : bands == 1 ? 3 : bands == 2 ? 8 : 15;
    const uint64_t a = 256;
    const uint64_t oPos = 0, oRot = round_up(oPos + 12 * n, a), oLsc = round_up(oRot + 16 * n, a);
    const uint64_t oOpl = round_up(oLsc + 12 * n, a), oDc = round_up(oOpl + 4 * n, a);
    const uint64_t oSh = round_up(oDc + 12 * n, a);
    const uint32_t P16 = (uint32_t)round_up((uint64_t)3 * M, 8);
    const uint64_t shBytes = precision == DL_PREC_F32 ? (uint64_t)3 * M * n * 4 : (uint64_t)P16 * n * 2;
    const uint64_t oTmp = round_up(oSh + shBytes, a);
    const uint64_t total = (precision == DL_PREC_F32 || M == 0) ? oTmp : oTmp + (uint64_t)3 * M * n * 4;
    DL_TRY(s->mem.ensure(total));
    char* b = s->mem.as<char>();
    // one splat range [g0, g1) of every array (the SH too when withSh)
    // (by value: a chunked upload runs from chunks->issue after this returns)
    auto upload = [=](uint64_t g0, uint64_t g1, bool withSh) -> int {
        const uint64_t c = g1 - g0;
        auto h2d = [&](uint64_t off, const void* src, uint64_t elem) {
            return cudaMemcpyAsync(b + off + elem * g0, (const char*)src + elem * g0, elem * c,
                                   cudaMemcpyHostToDevice, st);
        };
        DL_CK(h2d(oPos, d->positions, 12));
        DL_CK(h2d(oRot, d->rotations, 16));
        DL_CK(h2d(oLsc, d->log_scales, 12));
        DL_CK(h2d(oOpl, d->opacity_logits, 4));
        DL_CK(h2d(oDc, d->colors_dc, 12));
        if (M && withSh) {
            if (precision == DL_PREC_F32) {
                DL_CK(h2d(oSh, d->colors_sh, 12ull * M));
            } else {
                DL_CK(h2d(oTmp, d->colors_sh, 12ull * M));
                sh_to_half_k<<<1024, 256, 0, st>>>((const float*)(b + oTmp) + 3ull * M * g0,
                                                   (uint16_t*)(b + oSh) + (uint64_t)P16 * g0, c, M, (int)P16,
                                                   precision);
                DL_CK(cudaGetLastError());
            }
        }
        return DL_OK;
    };
    if (chunks) {
        // the geometry in equal splat ranges, each followed by its event; then
        // the SH (the bulk of the bytes) in the same ranges, each followed by
        // its event, and sh_event after all of them
        chunks->count = kUploadChunks;
        chunks->sh_separate = M > 0;
        chunks->issued = false;
        chunks->sh_src = M ? (const float*)(b + (precision == DL_PREC_F32 ? oSh : oTmp)) : nullptr;
        chunks->sh_dst = (M && precision != DL_PREC_F32) ? (uint16_t*)(b + oSh) : nullptr;
        chunks->sh_M = M;
        chunks->sh_P = (int)P16;
        chunks->sh_kind = precision;
        for (int k = 0; k <= kUploadChunks; k++) chunks->bounds[k] = (uint32_t)(n * (uint64_t)k / kUploadChunks);
        chunks->issue = [=]() -> int {
            for (int k = 0; k < kUploadChunks; k++) {
                if (chunks->bounds[k + 1] > chunks->bounds[k])
                    DL_TRY(upload(chunks->bounds[k], chunks->bounds[k + 1], false));
                DL_CK(cudaEventRecord(chunks->events[k], st));
            }
            if (M) {
                // in the same ranges: copies issued later on other streams (a
                // frame's view tables) queue behind one copy at most.  The
                // copies run back to back, each chunk followed by its event; the
                // frame converts a chunk to 16 bits on its own stream (a
                // conversion between two copies here would hold the next copy
                // until it has run beside the frame's kernels)
                for (int k = 0; k < kUploadChunks; k++) {
                    const uint64_t g0 = chunks->bounds[k], g1 = chunks->bounds[k + 1];
                    if (g1 > g0) {
                        const uint64_t e = 12ull * M;
                        DL_CK(cudaMemcpyAsync(b + (precision == DL_PREC_F32 ? oSh : oTmp) + e * g0,
                                              (const char*)d->colors_sh + e * g0, e * (g1 - g0),
                                              cudaMemcpyHostToDevice, st));
                    }
                    DL_CK(cudaEventRecord(chunks->sh_events[k], st));
                }
                DL_CK(cudaEventRecord(chunks->sh_event, st));
            }
            chunks->issued = true;
            return DL_OK;
        };
    } else if (n) {
        DL_TRY(upload(0, n, true));
    }
    s->precision = precision;
    s->d.pos = (const float*)(b + oPos);
    s->d.rot = (const float*)(b + oRot);
    s->d.lsc = (const float*)(b + oLsc);
    s->d.opl = (const float*)(b + oOpl);
    s->d.dc = (const float*)(b + oDc);
    s->d.sh = (M && precision == DL_PREC_F32) ? (const float*)(b + oSh) : nullptr;
    s->d.sh16 = (M && precision != DL_PREC_F32) ? (const uint16_t*)(b + oSh) : nullptr;
    s->d.sh16_stride = (M && precision != DL_PREC_F32) ? P16 : 0;
    s->d.n = (uint32_t)n;
    s->d.bands = bands;
    s->d.sh_kind = M ? precision : 0;
    return DL_OK;
}

namespace {

// Device pointers of one frame's working set (renderer buffers or the static array).
struct FramePtrs {
    DlView* views;
    uint32_t* tileBase;            // [V+1] first global tile of each view
    uint64_t* segStart;
    uint32_t* segLen;
    uint32_t* segTileBase;
    uint32_t* scr;
    uint32_t *keys0, *keys1, *vals0, *vals1;
    float4* recA;
    float4* recBC;
    uint4* recH;
    uint2* bbox;
    uint32_t* nvis;
    uint32_t* depthHist;
    uint32_t* sortStatus;
    uint32_t** outs;
    uint32_t* tileOff;
    uint64_t *pairBase, *pairCap;
    unsigned long long* npairs;
    uint32_t *pairSegLen, *pairSegTileBase, *pairGlob, *pairHist;
    unsigned long long* emitStatus;
    uint32_t *pkeys0, *pkeys1, *pvals0, *pvals1;
    float4* accum;
    unsigned long long* evalCount;
    const uint32_t* work;          // optional tile order for the rasterizer
    uint32_t* tileEvals;           // optional per-tile counters (cost logging)
    uint32_t* tileCycles;
    // a scene upload still in flight: projection per splat range after its event
    const DlUploadChunks* upload;
    uint32_t* visMask;             // colours deferred until each SH range has arrived (upload->sh_events)
    // host outputs read back per view range while the next range rasterizes
    int rbGroups;                  // 0: one rasterizer launch, no read-back here
    uint8_t* const* rbHost;        // [V] host destinations
    uint32_t* const* rbDev;        // [V] device images
    const DlView* rbViews;         // host view table (sizes)
    const uint32_t* rbTileBase;    // host [V+1] first global tile of each view
    cudaStream_t rbStream;
    cudaEvent_t rbEvent;
    cudaStream_t rasterStream2;    // with rbGroups: the odd view ranges rasterize here (NULL: all on the frame's)
    cudaEvent_t rasterEv[2];
    // learned schedule: features -> MLP -> longest-first tile order
    float* feat;                   // [total tiles][12], or NULL
    float* pred;
    const dl_mlp* sched;           // NULL: no learned order
    uint32_t *skeys0, *skeys1, *svals0, *svals1, *sstatus, *shist;
    uint64_t* ssegStart;
    uint32_t *ssegLen, *ssegTileBase;
};

struct FrameDims {
    uint32_t V = 1, N = 0, maxT = 1, TS = 2, totalTiles = 0, rasterGrid = 148;
    uint64_t stride = 64, cap = 0;
    uint32_t depthGrid = 1, emitTilesPerView = 1, pairGrid = 1;
    int pbits = 8, ppasses = 0;
    bool f16rec = false, fastExp = false, f64deg = false, cullOff = false;
    int subLw = 3;                       // rasterizer work item width log2 (8x4)
    bool ppl2 = false;                   // two pixels per lane (8x8 work items)
    bool x2 = false;                     // two splats per step in f32x2 arithmetic (fast variant)
    bool tileCta = false;                // one CTA per 256-pixel tile, the slice read once (fast variant)
    bool tileK = false;                  // one CTA per 256-pixel tile, records read in place (both variants)
    int iptLg = 3;                       // log2 of the rasterizer work items per binning tile
};

// Staging margin of the rasterizer (pixels): a splat is staged for a work
// item when its box widened by this much reaches a pixel centre of the item.
// 1/64 px is far above the f32 rounding of the box test (under 1e-3 px at
// the largest image coordinates) and below the 0.1% relative margin between
// a splat's box and the region where its alpha reaches 1/255.
// DL_STAGE_PAD overrides it (pixels) for measurements.
float stage_pad() {
    static float pad = -1.0f;
    if (pad < 0.0f) {
        const char* e = getenv("DL_STAGE_PAD");
        pad = e ? std::max(0.015625f, (float)atof(e)) : 0.015625f;
    }
    return pad;
}

// Bin a frame's views with tw x th-pixel tiles instead of the reference's
// 16x16.  Only when no view can truncate a splat's coverage (maxCoverage at
// least the view's 16x16 tile count), because the truncation keeps a
// row-major prefix of 16x16 tiles (src/render/shaders/emit-pairs.ts:46-53);
// without it every pixel is offered the same splats under any tile, so the
// pixels are the same.  Returns false (views unchanged) when that does not hold
// or the grid is too large.
bool dl_retile_views(DlView* v, uint32_t V, uint32_t tw, uint32_t th) {
    for (uint32_t i = 0; i < V; i++) {
        const uint64_t ref = (uint64_t)v[i].refTilesX * v[i].refTilesY;
        const uint64_t tx = (v[i].W + tw - 1) / tw, ty = (v[i].H + th - 1) / th;
        if (v[i].maxCoverage < ref || tx > 0x7fffu || ty > 0x7fffu || tx * ty >= (1u << 20)) return false;
    }
    for (uint32_t i = 0; i < V; i++) {
        v[i].tileW = tw;
        v[i].tileH = th;
        v[i].tilesX = (v[i].W + tw - 1) / tw;
        v[i].tilesY = (v[i].H + th - 1) / th;
        v[i].numTiles = v[i].tilesX * v[i].tilesY;
        v[i].binCap = 0xffffffffu;
    }
    return true;
}

// Persistent rasterizer grid: every SM filled to its occupancy limit.
uint32_t raster_grid(bool fastExp, bool ppl2, bool x2, bool tileCta, bool tileK) {
    static int cached[64][8] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const int kind = tileK ? (fastExp ? 7 : 6) : tileCta ? 5 : x2 ? 4 : (fastExp ? 1 : 0) + (ppl2 ? 2 : 0);
    int* c = (dev >= 0 && dev < 64) ? &cached[dev][kind] : nullptr;
    if (c && *c) return (uint32_t)*c;
    int sms = 148, per = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (tileK) {
        if (fastExp) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_tile_k<false, false>,
                                                                   dlr::kRasterThreads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_tile_k<true, false>,
                                                           dlr::kRasterThreads, 0);
    } else if (tileCta) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_tile_x2_k<false>, dlr::kRasterThreads, 0);
    } else if (x2) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_x2_k<false>, dlr::kRasterThreads, 0);
    } else if (ppl2) {
        if (fastExp) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize2_k<false>, dlr::kRasterThreads, 0);
        else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize2_k<true>, dlr::kRasterThreads, 0);
    } else if (fastExp) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_k<false>, dlr::kRasterThreads, 0);
    } else {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dlr::rasterize_k<true>, dlr::kRasterThreads, 0);
    }
    const int g = std::max(sms, 1) * std::max(per, 1);
    if (c) *c = g;
    return (uint32_t)g;
}

FrameDims frame_dims(const DlView* hv, uint32_t V, uint32_t N, uint64_t cap, uint32_t flags,
                     const DlTuning& t = DlTuning()) {
    FrameDims d;
    d.pbits = (t.pair_bits >= 6 && t.pair_bits <= 8) ? t.pair_bits : 8;
    d.subLw = t.shape == 1 ? 4 : t.shape == 2 ? 2 : 3;
    d.ppl2 = t.shape == 3;
    d.V = V;
    d.N = N;
    d.stride = round_up(std::max<uint32_t>(N, 1), 64);
    for (uint32_t v = 0; v < V; v++) {
        d.maxT = std::max(d.maxT, hv[v].numTiles);
        d.totalTiles += hv[v].numTiles;
    }
    d.TS = d.maxT + 1;
    d.depthGrid = std::max<uint32_t>(1, V * (uint32_t)((N + dlsort::kTile - 1) / dlsort::kTile));
    d.emitTilesPerView = (uint32_t)((d.stride + dlr::kEmitRanks - 1) / dlr::kEmitRanks);
    int keyBits = 0;
    while ((1u << keyBits) < d.maxT) keyBits++;
    d.ppasses = (keyBits + d.pbits - 1) / d.pbits;
    if (d.ppasses > 4) {                 // the digit tables hold 4 passes
        d.pbits = 8;
        d.ppasses = (keyBits + 7) / 8;
    }
    d.cap = cap;
    d.pairGrid = std::max<uint32_t>(1, (uint32_t)(V * ((cap + dlsort::kTile - 1) / dlsort::kTile)));
    d.f16rec = (flags & DL_BATCH_F16_RECORDS) != 0;
    d.fastExp = (flags & DL_BATCH_FAST_EXP) != 0;
    d.f64deg = (flags & DL_BATCH_F64_DEGENERATE) != 0;
    d.cullOff = (flags & DL_BATCH_CULL_OFFSCREEN) != 0;
    d.x2 = (t.shape == 4 || t.shape == 5) && d.fastExp;    // the packed variants have the fast arithmetic only
    // work items must fit the binning tile (every view of a frame has the same tile)
    const uint32_t tw = V ? hv[0].tileW : DL_TILE, th = V ? hv[0].tileH : DL_TILE;
    d.tileCta = t.shape == 5 && d.fastExp && tw * th == 256u;   // 8 warps of 8x4 items per tile
    d.tileK = t.shape == 6 && tw * th == 256u;
    const uint32_t iw = d.ppl2 ? 8u : (1u << d.subLw), ih = d.ppl2 ? 8u : (32u >> d.subLw);
    if (iw > tw || ih > th) { d.subLw = 3; d.ppl2 = false; }
    const uint32_t ipt = (d.tileCta || d.tileK) ? 1u : tw * th / (d.ppl2 ? 64u : 32u);
    d.iptLg = 0;
    while ((1u << d.iptLg) < ipt) d.iptLg++;
    d.rasterGrid = raster_grid(d.fastExp, d.ppl2, d.x2, d.tileCta, d.tileK);
    if (t.ctas_per_sm > 0) {
        int dev = 0, sms = 148;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        d.rasterGrid = std::min<uint32_t>(d.rasterGrid, (uint32_t)(std::max(sms, 1) * t.ctas_per_sm));
    }
    return d;
}

inline void rec_event(cudaEvent_t* ev, int i, cudaStream_t st) {
    if (ev) cudaEventRecord(ev[i], st);
}

// Deferred colours of upload ranges [k0, k1) on the frame's stream, each once
// its SH range has arrived (converted to 16 bits first).  The frame launches
// them between its later stages, so that they neither wait behind persistent
// kernels that hold every SM nor hold back the rasterizer.
int launch_colours(const FramePtrs& f, const FrameDims& d, const DlSceneDev& sc, cudaStream_t st, int k0, int k1,
                   uint64_t* launches) {
    if (!f.visMask || !d.N) return DL_OK;
    const DlUploadChunks& up = *f.upload;
    dlr::ColourArgs ca;
    ca.sc = sc;
    ca.views = f.views;
    ca.num_views = d.V;
    ca.view_stride = d.stride;
    ca.vis_mask = f.visMask;
    ca.recBC = d.f16rec ? nullptr : f.recBC;
    ca.recH = d.f16rec ? f.recH : nullptr;
    for (int k = std::max(k0, 0); k < std::min(k1, up.count); k++) {
        const uint32_t g0 = up.bounds[k], g1 = up.bounds[k + 1];
        DL_CK(cudaStreamWaitEvent(st, up.sh_events[k], 0));
        if (g1 == g0) continue;
        DL_TRY(dl_upload_convert_sh(&up, g0, g1, st, launches));
        ca.g_begin = g0;
        ca.g_end = g1;
        if (d.fastExp) dlr::colour_k<true><<<(g1 - g0 + 255) / 256, 256, 0, st>>>(ca);
        else dlr::colour_k<false><<<(g1 - g0 + 255) / 256, 256, 0, st>>>(ca);
        (*launches)++;
        DL_CK(cudaGetLastError());
    }
    return DL_OK;
}

// project + depth sort.  Expects views, segment tables, nvis and scratch words
// already uploaded / cleared on the stream.
int launch_front(const FramePtrs& f, const FrameDims& d, const DlSceneDev& sc, cudaStream_t st, cudaEvent_t* ev,
                 uint64_t* launches) {
    rec_event(ev, 0, st);
    dlr::ProjectArgs pa;
    pa.sc = sc;
    pa.views = f.views;
    pa.num_views = d.V;
    pa.view_stride = d.stride;
    pa.keys = f.keys0;
    pa.recA = f.recA;
    pa.recBC = d.f16rec ? nullptr : f.recBC;
    pa.recH = d.f16rec ? f.recH : nullptr;
    pa.bbox = f.bbox;
    pa.nvis = f.nvis;
    pa.f64_degenerate = d.f64deg ? 1 : 0;
    pa.cull_offscreen = d.cullOff ? 1 : 0;
    pa.g_begin = 0;
    pa.g_end = d.N;
    pa.vis_mask = f.visMask;
    if (f.upload) {
        for (int k = 0; k < f.upload->count; k++) {
            DL_CK(cudaStreamWaitEvent(st, f.upload->events[k], 0));
            pa.g_begin = f.upload->bounds[k];
            pa.g_end = f.upload->bounds[k + 1];
            if (pa.g_end > pa.g_begin) {
                if (d.fastExp) dlr::project_k<true><<<(pa.g_end - pa.g_begin + 255) / 256, 256, 0, st>>>(pa);
                else dlr::project_k<false><<<(pa.g_end - pa.g_begin + 255) / 256, 256, 0, st>>>(pa);
                (*launches)++;
                DL_CK(cudaGetLastError());
            }
        }
    } else if (d.N) {
        if (d.fastExp) dlr::project_k<true><<<(d.N + 255) / 256, 256, 0, st>>>(pa);
        else dlr::project_k<false><<<(d.N + 255) / 256, 256, 0, st>>>(pa);
        (*launches)++;
    }
    DL_CK(cudaGetLastError());
    rec_event(ev, 1, st);
    // depth sort: stable LSD, 4 x 8-bit digits, one segment per view
    if (d.N) {
        dlsort::Segs ds;
        ds.start = f.segStart; ds.len = f.segLen; ds.tile_base = f.segTileBase;
        ds.total_tiles = f.scr + SC_DEPTH_TILES; ds.num = d.V;
        dlsort::prepare_k<<<1, 32, 0, st>>>(ds);
        // the first pass drops the culled keys (0xffffffff) and compacts the
        // visible ones, in a stable order, to each view's segment start; the
        // other passes sort the nvis[v] visible keys only
        dlsort::Segs ds2 = ds;
        ds2.len = f.nvis; ds2.tile_base = f.segTileBase + d.V; ds2.total_tiles = f.scr + SC_DEPTH_TILES2;
        dlsort::prepare_k<<<1, 32, 0, st>>>(ds2);
        DL_CK(cudaMemsetAsync(f.depthHist, 0, 4ull * d.V * 4 * 256, st));
        dlsort::hist_k<8><<<std::min<uint32_t>(d.depthGrid, 4096), dlsort::kThreads, 0, st>>>(f.keys0, ds, 4, 0,
                                                                                               f.depthHist, 1);
        dlsort::scan_hist_k<8><<<std::min<uint32_t>(4 * d.V, 1024), 256, 0, st>>>(f.depthHist, 4 * d.V);
        *launches += 4;
        uint32_t *kin = f.keys0, *kout = f.keys1, *vin = nullptr, *vout = f.vals1;
        for (int p = 0; p < 4; p++) {
            DL_CK(cudaMemsetAsync(f.sortStatus, 0, 4ull * 256 * d.depthGrid, st));
            dlsort::Pass sp;
            sp.keys_in = kin; sp.vals_in = vin; sp.keys_out = kout; sp.vals_out = vout;
            sp.segs = p == 0 ? ds : ds2; sp.glob_off = f.depthHist;
            sp.status = f.sortStatus; sp.counter = f.scr + SC_DEPTH_CTR + p; sp.err = f.scr + SC_ERR;
            sp.shift = 8 * p; sp.pass = p; sp.passes = 4; sp.drop_max = p == 0 ? 1 : 0;
            sp.spin_limit = g_dl_wait.spin_limit;
            if (p == 0) sp.withhold_tile = g_dl_wait.withheld(DL_WAIT_STAGE_DEPTH_SORT);
            launch_pass_bits(8, sp, d.depthGrid, st);
            (*launches)++;
            std::swap(kin, kout);
            vin = vout;
            vout = (vout == f.vals1) ? f.vals0 : f.vals1;
        }
        DL_CK(cudaGetLastError());
    }
    // deferred colours: the first half of the upload ranges (their SH has
    // arrived by the end of the depth sort on the headline batch)
    if (f.visMask) DL_TRY(launch_colours(f, d, sc, st, 0, f.upload->count / 2, launches));
    rec_event(ev, 2, st);
    // after 4 passes keys0 / vals0 hold the sorted keys / splat indices
    return DL_OK;
}

// emit -> pair digits -> pair sort -> boundaries -> rasterize.  Expects
// pairBase / pairCap uploaded.  *finalVals receives the sorted pair values.
int launch_back(const FramePtrs& f, const FrameDims& d, const DlSceneDev& sc, cudaStream_t st, cudaEvent_t* ev,
                uint64_t* launches, uint32_t** finalVals) {
    DL_CK(cudaMemsetAsync(f.pairHist, 0, 4ull * d.V * 4 * 256, st));
    DL_CK(cudaMemsetAsync(f.emitStatus, 0, 8ull * d.V * d.emitTilesPerView, st));
    DL_CK(cudaMemsetAsync(f.scr + SC_EMIT_CTR, 0, 4ull * 6, st));   // emit + pair counters + work counter
    DL_CK(cudaMemsetAsync(f.scr + SC_OVF, 0, 4, st));
    rec_event(ev, 3, st);
    dlr::EmitArgs ea;
    ea.sorted_vals = f.vals0;
    ea.bbox = f.bbox;
    ea.nvis = f.nvis;
    ea.views = f.views;
    ea.view_stride = d.stride;
    ea.tiles_per_view = d.emitTilesPerView;
    ea.pair_base = f.pairBase;
    ea.pair_cap = f.pairCap;
    ea.pair_keys = f.pkeys0;
    ea.pair_vals = f.pvals0;
    ea.npairs = f.npairs;
    ea.digit_hist = f.pairHist;
    ea.bits = d.pbits;
    ea.passes = d.ppasses;
    ea.status = f.emitStatus;
    ea.counter = f.scr + SC_EMIT_CTR;
    ea.err = f.scr + SC_ERR;
    ea.ovf = f.scr + SC_OVF;
    ea.spin_limit = g_dl_wait.spin_limit;
    ea.withhold_tile = g_dl_wait.withheld(DL_WAIT_STAGE_EMIT);
    dlr::emit_k<<<d.V * d.emitTilesPerView, dlr::kEmitThreads, 0, st>>>(ea);
    (*launches)++;
    DL_CK(cudaGetLastError());
    // deferred colours: the next three eighths of the upload ranges after the
    // emission, the rest after the first pair-sort pass
    const int colMid = f.visMask ? f.upload->count / 2 : 0;
    const int colLate = f.visMask ? f.upload->count * 7 / 8 : 0;
    if (f.visMask) DL_TRY(launch_colours(f, d, sc, st, colMid, colLate, launches));
    rec_event(ev, 4, st);

    dlr::PairDigitArgs pd;
    pd.digit_hist = f.pairHist;
    pd.glob_off = f.pairGlob;
    pd.npairs = f.npairs;
    pd.pair_cap = f.pairCap;
    pd.seg_len = f.pairSegLen;
    pd.bits = d.pbits;
    pd.passes = d.ppasses;
    pd.err = f.scr + SC_ERR;
    dlr::pair_digits_k<<<d.V, 32, 0, st>>>(pd);
    (*launches)++;
    DL_CK(cudaGetLastError());
    rec_event(ev, 5, st);

    // pair sort by tile id (stable: depth-rank order kept inside each tile)
    uint32_t* vals = f.pvals0;
    uint32_t* keys = f.pkeys0;
    if (d.ppasses > 0) {
        dlsort::Segs ps;
        ps.start = f.pairBase; ps.len = f.pairSegLen; ps.tile_base = f.pairSegTileBase;
        ps.total_tiles = f.scr + SC_PAIR_TILES; ps.num = d.V;
        dlsort::prepare_k<<<1, 32, 0, st>>>(ps);
        (*launches)++;
        uint32_t *kin = f.pkeys0, *kout = f.pkeys1, *vin = f.pvals0, *vout = f.pvals1;
        // the last pass lowers the tile offsets itself (bound_init_k presets them)
        dlr::BoundArgs bi;
        bi.views = f.views; bi.keys = nullptr; bi.pair_base = f.pairBase; bi.seg_len = f.pairSegLen;
        bi.tile_off = f.tileOff; bi.tile_stride = d.TS; bi.err = f.scr + SC_ERR;
        dlr::bound_init_k<<<dim3((d.TS + 255) / 256, d.V), 256, 0, st>>>(bi);
        (*launches)++;
        for (int p = 0; p < d.ppasses; p++) {
            DL_CK(cudaMemsetAsync(f.sortStatus, 0, 4ull * 256 * d.pairGrid, st));
            dlsort::Pass sp;
            const bool last = p + 1 == d.ppasses;
            sp.keys_in = kin; sp.vals_in = vin; sp.keys_out = last ? nullptr : kout; sp.vals_out = vout;
            dlsort::Bound bd;
            if (last) { bd.bound = f.tileOff; bd.stride = d.TS; }
            sp.segs = ps; sp.glob_off = f.pairGlob;
            sp.status = f.sortStatus; sp.counter = f.scr + SC_PAIR_CTR + p; sp.err = f.scr + SC_ERR;
            sp.shift = d.pbits * p; sp.pass = p; sp.passes = d.ppasses;
            sp.spin_limit = g_dl_wait.spin_limit;
            if (p == 0) sp.withhold_tile = g_dl_wait.withheld(DL_WAIT_STAGE_PAIR_SORT);
            launch_pass_bits(d.pbits, sp, d.pairGrid, st, bd);
            (*launches)++;
            if (p == 0 && f.visMask) DL_TRY(launch_colours(f, d, sc, st, colLate, f.upload->count, launches));
            std::swap(kin, kout);
            std::swap(vin, vout);
        }
        keys = kin;
        vals = vin;
        DL_CK(cudaGetLastError());
    }
    dlr::BoundArgs ba;
    ba.views = f.views;
    ba.keys = keys;
    ba.pair_base = f.pairBase;
    ba.seg_len = f.pairSegLen;
    ba.tile_off = f.tileOff;
    ba.tile_stride = d.TS;
    ba.err = f.scr + SC_ERR;
    if (d.ppasses > 0) {
        dlr::bound_fill_k<<<d.V, dlr::kFillThreads, 0, st>>>(ba);
    } else {                            // one tile per view: the keys are all 0
        const uint32_t bgrid = (uint32_t)std::min<uint64_t>(std::max<uint64_t>((d.cap + 256) / 256, 1), 2048);
        dlr::boundaries_k<<<dim3(bgrid, d.V), 256, 0, st>>>(ba);
    }
    (*launches)++;
    DL_CK(cudaGetLastError());

    if (d.ppasses == 0 && f.visMask) DL_TRY(launch_colours(f, d, sc, st, colLate, f.upload->count, launches));

    // learned schedule: per-tile features, predicted cost, tiles in decreasing order
    const uint32_t* work = f.work;
    if (f.feat && !f.sched && d.totalTiles) {
        dlr::tile_features_k<<<(d.totalTiles + 255) / 256, 256, 0, st>>>(f.views, d.V, f.tileBase, f.tileOff, d.TS,
                                                                         d.totalTiles, f.feat);
        (*launches)++;
        DL_CK(cudaGetLastError());
    }
    if (f.sched && d.totalTiles) {
        const uint32_t g = std::min<uint32_t>((d.totalTiles + dlr::kSchedThreads - 1) / dlr::kSchedThreads, 2048);
        DL_CK(cudaMemsetAsync(f.shist, 0, 4ull * 256 * d.V, st));
        // the views that end a rasterizer launch are reordered
        const uint32_t tailEvery = f.rbGroups > 1 ? (d.V + (uint32_t)f.rbGroups - 1) / (uint32_t)f.rbGroups : d.V;
        dlr::sched_pred_k<<<g, dlr::kSchedThreads, 0, st>>>(f.views, d.V, f.tileBase, f.tileOff, d.TS, d.totalTiles,
                                                            (const __nv_bfloat16*)dl_mlp_weights(f.sched), f.svals1,
                                                            f.shist, tailEvery, f.svals0);
        dlr::sched_scan_k<<<d.V, 32, 0, st>>>(f.tileBase, f.shist);
        dlr::sched_scatter_k<<<std::min<uint32_t>((d.totalTiles + 255) / 256, 2048), 256, 0, st>>>(
            f.svals1, d.totalTiles, f.shist, f.svals0);
        *launches += 3;
        DL_CK(cudaGetLastError());
        work = f.svals0;
    }
    rec_event(ev, 6, st);

    dlr::RasterArgs ra;
    std::memset(&ra, 0, sizeof(ra));
    ra.views = f.views;
    ra.num_views = d.V;
    ra.tile_base = f.tileBase;
    ra.tile_off = f.tileOff;
    ra.tile_stride = d.TS;
    ra.pair_vals = vals;
    ra.pair_base = f.pairBase;
    ra.recA = f.recA;
    ra.recBC = d.f16rec ? nullptr : f.recBC;
    ra.recH = d.f16rec ? f.recH : nullptr;
    ra.view_stride = d.stride;
    ra.outs = f.outs;
    ra.accum = f.accum;
    ra.work = work;
    const bool count = f.evalCount || f.tileEvals;
    // counting frames run the 8x4 warp-item kernel: 8 items per 256-pixel tile
    const int iptLg = ((d.tileCta || d.tileK) && count) ? 3 : d.iptLg;
    ra.item_base = 0;
    ra.num_items = (1u << iptLg) * d.totalTiles;
    ra.ipt_lg = iptLg;
    ra.work_counter = f.scr + SC_WORK_CTR;
    ra.eval_count = f.evalCount;
    ra.tile_evals = f.tileEvals;
    ra.tile_cycles = f.tileCycles;
    ra.sub_lw = d.subLw;
    ra.rec_box = d.cullOff ? 1 : 0;
    ra.stage_pad = stage_pad();
    auto raster = [&](const dlr::RasterArgs& x, cudaStream_t rs) {
        if (d.tileK && !count) {
            if (d.fastExp) {
                if (x.tile_cycles) dlr::rasterize_tile_k<false, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
                else dlr::rasterize_tile_k<false, false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            } else {
                if (x.tile_cycles) dlr::rasterize_tile_k<true, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
                else dlr::rasterize_tile_k<true, false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            }
        } else if (d.tileCta && !count) {
            if (x.tile_cycles) dlr::rasterize_tile_x2_k<true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            else dlr::rasterize_tile_x2_k<false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
        } else if (d.x2 && !count) {
            if (x.tile_cycles) dlr::rasterize_x2_k<true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            else dlr::rasterize_x2_k<false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
        } else if (d.ppl2) {
            if (d.fastExp) {
                if (count) dlr::rasterize2_k<false, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
                else dlr::rasterize2_k<false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            } else {
                if (count) dlr::rasterize2_k<true, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
                else dlr::rasterize2_k<true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            }
        } else if (d.fastExp) {
            if (count) dlr::rasterize_k<false, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            else dlr::rasterize_k<false><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
        } else {
            if (count) dlr::rasterize_k<true, true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
            else dlr::rasterize_k<true><<<d.rasterGrid, dlr::kRasterThreads, 0, rs>>>(x);
        }
        (*launches)++;
    };
    if (f.rbGroups > 1 && d.V > 1) {
        // One launch per view range (the work queue is view-major in both
        // orders, so a range of views is a range of items); each range's images
        // go back to the host on the read-back stream while the next rasterizes.
        const uint32_t per = (d.V + (uint32_t)f.rbGroups - 1) / (uint32_t)f.rbGroups;
        const uint32_t ipt = 1u << iptLg;
        static_assert(SC_RASTER_CTR + kReadBackGroups <= kScratchWords, "scratch words");
        DL_CK(cudaMemsetAsync(f.scr + SC_RASTER_CTR, 0, 4ull * kReadBackGroups, st));
        // Ranges alternate between the frame's stream and a second one, so
        // that the next range's CTAs take the SMs that the current range's
        // persistent CTAs leave at its end (ranges of one stream run in order;
        // at most two ranges are in flight).
        const bool two = f.rasterStream2 != nullptr;
        if (two) {
            DL_CK(cudaEventRecord(f.rasterEv[0], st));
            DL_CK(cudaStreamWaitEvent(f.rasterStream2, f.rasterEv[0], 0));
        }
        for (uint32_t v0 = 0, g = 0; v0 < d.V; v0 += per, g++) {
            const uint32_t v1 = std::min(d.V, v0 + per);
            cudaStream_t rs = (two && (g & 1u)) ? f.rasterStream2 : st;
            dlr::RasterArgs x = ra;
            x.item_base = ipt * f.rbTileBase[v0];
            x.num_items = ipt * f.rbTileBase[v1];
            x.work_counter = f.scr + SC_RASTER_CTR + g;      // g < rbGroups <= kReadBackGroups
            raster(x, rs);
            DL_CK(cudaGetLastError());
            DL_CK(cudaEventRecord(f.rbEvent, rs));
            DL_CK(cudaStreamWaitEvent(f.rbStream, f.rbEvent, 0));
            for (uint32_t v = v0; v < v1; v++)
                DL_CK(cudaMemcpyAsync(f.rbHost[v], f.rbDev[v], (uint64_t)f.rbViews[v].W * f.rbViews[v].H * 4,
                                      cudaMemcpyDeviceToHost, f.rbStream));
        }
        if (two) {                       // the frame's stream continues after both
            DL_CK(cudaEventRecord(f.rasterEv[1], f.rasterStream2));
            DL_CK(cudaStreamWaitEvent(st, f.rasterEv[1], 0));
        }
    } else {
        raster(ra, st);
    }
    DL_CK(cudaGetLastError());
    rec_event(ev, 7, st);
    *finalVals = vals;
    return DL_OK;
}

}  // namespace

int dl_render_views(dl_renderer* r, const DlSceneDev& sc, const DlView* hv, uint32_t V, uint32_t* const* d_outs,
                    uint32_t flags, const DlOverlap* overlap) {
    cudaStream_t st = r->stream;
    const uint32_t N = sc.n;
    if (r->pair_cap_per_view == 0) r->pair_cap_per_view = std::max<uint64_t>(1u << 20, 4ull * N);
    // the plain path keeps the default knobs
    const DlTuning tune = (flags & DL_BATCH_PLAIN) ? DlTuning() : r->tune;
    std::vector<DlView> retiled;
    if (tune.bin_tile == 1 || tune.bin_tile == 2) {
        const uint32_t tw = tune.bin_tile == 1 ? 8u : 32u, th = 8u;
        retiled.assign(hv, hv + V);
        if (dl_retile_views(retiled.data(), V, tw, th)) hv = retiled.data();
    }
    FrameDims d = frame_dims(hv, V, N, r->pair_cap_per_view, flags, tune);
    const bool countEvals = (flags & DL_BATCH_COUNT_EVALS) != 0;
    r->launches = 0;

    // ---- buffers
    if (d.totalTiles >= (1u << 29)) { dl_set_error("more than 2^29 tiles in one batch"); return DL_E_CAPACITY; }
    DL_TRY(r->views.ensure(sizeof(DlView) * V));
    DL_TRY(r->tileBase.ensure(4ull * (V + 1)));
    DL_TRY(r->segStart.ensure(8ull * V));
    DL_TRY(r->segLen.ensure(4ull * V));
    DL_TRY(r->segTileBase.ensure(8ull * V));
    DL_TRY(r->scratch.ensure(4ull * kScratchWords));
    DL_TRY(r->keys0.ensure(4ull * V * d.stride));
    DL_TRY(r->keys1.ensure(4ull * V * d.stride));
    DL_TRY(r->vals0.ensure(4ull * V * d.stride));
    DL_TRY(r->vals1.ensure(4ull * V * d.stride));
    DL_TRY(r->recA.ensure(16ull * V * d.stride));
    if (d.f16rec) DL_TRY(r->recH.ensure(16ull * V * d.stride));
    else DL_TRY(r->recBC.ensure(32ull * V * d.stride));
    DL_TRY(r->bbox.ensure(8ull * V * d.stride));
    DL_TRY(r->nvis.ensure(4ull * V));
    DL_TRY(r->depthHist.ensure(4ull * V * 4 * 256));
    DL_TRY(r->outs.ensure(sizeof(uint32_t*) * V));
    DL_TRY(r->tileOff.ensure(4ull * V * d.TS));
    DL_TRY(r->pairBase.ensure(8ull * V));
    DL_TRY(r->pairCap.ensure(8ull * V));
    DL_TRY(r->npairs.ensure(8ull * V));
    DL_TRY(r->pairSegLen.ensure(4ull * V));
    DL_TRY(r->pairSegTileBase.ensure(4ull * V));
    DL_TRY(r->pairGlob.ensure(4ull * V * 4 * 256));
    DL_TRY(r->tileCount.ensure(4ull * V * 4 * 256));          // tile-id digit histograms of the pair sort
    DL_TRY(r->emitStatus.ensure(8ull * V * d.emitTilesPerView));
    DL_TRY(r->sortStatus.ensure(4ull * 256 * d.depthGrid));
    if (r->keep_accum && V == 1) DL_TRY(r->accum.ensure(16ull * hv[0].W * hv[0].H));
    if (countEvals) DL_TRY(r->evalCount.ensure(8));

    // learned schedule (batched frames only) and tile-cost logging
    const bool useSched = r->sched && !(flags & (DL_BATCH_PLAIN | DL_BATCH_STATIC));
    const bool logTiles = (flags & DL_BATCH_LOG_TILES) != 0;
    if (useSched || logTiles) {
        DL_TRY(r->feat.ensure(48ull * d.totalTiles));
        DL_TRY(r->pred.ensure(4ull * d.totalTiles));
    }
    if (useSched) {
        const uint64_t sg = (d.totalTiles + dlsort::kTile - 1) / dlsort::kTile;
        DL_TRY(r->skeys0.ensure(4ull * d.totalTiles));
        DL_TRY(r->skeys1.ensure(4ull * d.totalTiles));
        DL_TRY(r->svals0.ensure(4ull * d.totalTiles));
        DL_TRY(r->svals1.ensure(4ull * d.totalTiles));
        DL_TRY(r->sstatus.ensure(4ull * 256 * std::max<uint64_t>(sg, 1)));
        DL_TRY(r->shist.ensure(4ull * 256 * std::max<uint32_t>(V, 4)));
        DL_TRY(r->sseg.ensure(64));
    }
    if (logTiles) DL_TRY(r->tileCycles.ensure(4ull * d.totalTiles));

    FramePtrs f;
    std::memset(&f, 0, sizeof(f));
    if (useSched || logTiles) { f.feat = r->feat.as<float>(); f.pred = r->pred.as<float>(); }
    if (useSched) {
        f.sched = r->sched;
        f.skeys0 = r->skeys0.as<uint32_t>(); f.skeys1 = r->skeys1.as<uint32_t>();
        f.svals0 = r->svals0.as<uint32_t>(); f.svals1 = r->svals1.as<uint32_t>();
        f.sstatus = r->sstatus.as<uint32_t>(); f.shist = r->shist.as<uint32_t>();
        f.ssegStart = r->sseg.as<uint64_t>();
        f.ssegLen = (uint32_t*)(f.ssegStart + 1);
        f.ssegTileBase = f.ssegLen + 1;
    }
    if (logTiles) f.tileCycles = r->tileCycles.as<uint32_t>();
    f.views = r->views.as<DlView>();
    f.tileBase = r->tileBase.as<uint32_t>();
    f.segStart = r->segStart.as<uint64_t>();
    f.segLen = r->segLen.as<uint32_t>();
    f.segTileBase = r->segTileBase.as<uint32_t>();
    f.scr = r->scratch.as<uint32_t>();
    f.keys0 = r->keys0.as<uint32_t>(); f.keys1 = r->keys1.as<uint32_t>();
    f.vals0 = r->vals0.as<uint32_t>(); f.vals1 = r->vals1.as<uint32_t>();
    f.recA = r->recA.as<float4>();
    f.recBC = d.f16rec ? nullptr : r->recBC.as<float4>();
    f.recH = d.f16rec ? r->recH.as<uint4>() : nullptr;
    f.bbox = r->bbox.as<uint2>();
    f.nvis = r->nvis.as<uint32_t>();
    f.depthHist = r->depthHist.as<uint32_t>();
    f.outs = r->outs.as<uint32_t*>();
    f.tileOff = r->tileOff.as<uint32_t>();
    f.pairBase = r->pairBase.as<uint64_t>();
    f.pairCap = r->pairCap.as<uint64_t>();
    f.npairs = r->npairs.as<unsigned long long>();
    f.pairSegLen = r->pairSegLen.as<uint32_t>();
    f.pairSegTileBase = r->pairSegTileBase.as<uint32_t>();
    f.pairGlob = r->pairGlob.as<uint32_t>();
    f.pairHist = r->tileCount.as<uint32_t>();
    f.emitStatus = r->emitStatus.as<unsigned long long>();
    f.accum = (r->keep_accum && V == 1) ? r->accum.as<float4>() : nullptr;
    f.evalCount = countEvals ? r->evalCount.as<unsigned long long>() : nullptr;

    // ---- host-side tables (pinned staging), one upload
    const size_t hbytes = sizeof(DlView) * V + 8ull * V + 4ull * V + sizeof(void*) * V + 4ull * (V + 1) + 128;
    DL_TRY(ensure_pinned((void**)&r->h_views, &r->h_views_cap, hbytes));
    char* hb = (char*)r->h_views;
    std::memcpy(hb, hv, sizeof(DlView) * V);
    uint64_t* hSegStart = (uint64_t*)(hb + sizeof(DlView) * V);
    uint32_t* hSegLen = (uint32_t*)(hSegStart + V);
    for (uint32_t v = 0; v < V; v++) { hSegStart[v] = (uint64_t)v * d.stride; hSegLen[v] = N; }
    void** hOuts = (void**)(hSegLen + V + (V & 1));
    for (uint32_t v = 0; v < V; v++) hOuts[v] = d_outs[v];
    uint32_t* hTileBase = (uint32_t*)(hOuts + V);
    hTileBase[0] = 0;
    for (uint32_t v = 0; v < V; v++) hTileBase[v + 1] = hTileBase[v] + hv[v].numTiles;
    DL_CK(cudaMemcpyAsync(f.tileBase, hTileBase, 4ull * (V + 1), cudaMemcpyHostToDevice, st));
    if (useSched) {
        uint64_t* hs = (uint64_t*)(hTileBase + V + 1 + ((V + 1) & 1));
        hs[0] = 0;
        reinterpret_cast<uint32_t*>(hs + 1)[0] = d.totalTiles;
        reinterpret_cast<uint32_t*>(hs + 1)[1] = 0;
        DL_CK(cudaMemcpyAsync(f.ssegStart, hs, 16, cudaMemcpyHostToDevice, st));
    }
    DL_CK(cudaMemcpyAsync(f.views, hb, sizeof(DlView) * V, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.segStart, hSegStart, 8ull * V, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.segLen, hSegLen, 4ull * V, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.outs, hOuts, sizeof(void*) * V, cudaMemcpyHostToDevice, st));
    cudaEvent_t* ev = r->profiling ? r->ev : nullptr;
    f.sortStatus = r->sortStatus.as<uint32_t>();
    // frames that overlap copies with their kernels run outside a graph
    std::vector<uint32_t> rbTileBase;
    if (overlap) {
        f.upload = overlap->upload;
        if (f.upload && f.upload->sh_separate) {
            DL_TRY(r->visMask.ensure(4ull * ((V + 31) / 32) * std::max<uint32_t>(N, 1)));
            f.visMask = r->visMask.as<uint32_t>();
        }
        if (overlap->groups > 1 && V > 1) {
            rbTileBase.assign(hTileBase, hTileBase + V + 1);
            f.rbGroups = std::min(overlap->groups, kReadBackGroups);
            f.rbHost = overlap->host;
            f.rbDev = d_outs;
            f.rbViews = hv;
            f.rbTileBase = rbTileBase.data();
            f.rbStream = overlap->stream;
            f.rbEvent = overlap->event;
            if (!r->raster_stream) DL_CK(cudaStreamCreateWithFlags(&r->raster_stream, cudaStreamNonBlocking));
            for (auto& e : r->raster_ev)
                if (!e) DL_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            f.rasterStream2 = r->raster_stream;
            f.rasterEv[0] = r->raster_ev[0];
            f.rasterEv[1] = r->raster_ev[1];
        }
    }
    const bool useGraph = !(flags & DL_BATCH_NO_GRAPH) && !(flags & DL_BATCH_PLAIN) && V > 1 && !r->profiling &&
                          !overlap && st != nullptr && st != cudaStreamLegacy && st != cudaStreamPerThread;

    // a frame that cannot fit leaves the capacity where it found it, so the
    // renderer keeps serving batches that do fit
    const uint64_t capOnEntry = r->pair_cap_per_view;
    for (int attempt = 0; attempt < 3; attempt++) {
        const uint64_t cap = r->pair_cap_per_view;
        if (cap >= (1ull << 30)) {
            r->pair_cap_per_view = capOnEntry;
            dl_set_error("more than 2^30 tile pairs in one view");
            return DL_E_CAPACITY;
        }
        d = frame_dims(hv, V, N, cap, flags, tune);
        DL_TRY(r->pkeys0.ensure(4ull * V * cap));
        DL_TRY(r->pvals0.ensure(4ull * V * cap));
        DL_TRY(r->pkeys1.ensure(4ull * V * cap));
        DL_TRY(r->pvals1.ensure(4ull * V * cap));
        DL_TRY(r->sortStatus.ensure(4ull * 256 * std::max(d.pairGrid, d.depthGrid)));
        f.sortStatus = r->sortStatus.as<uint32_t>();
        f.pkeys0 = r->pkeys0.as<uint32_t>(); f.pkeys1 = r->pkeys1.as<uint32_t>();
        f.pvals0 = r->pvals0.as<uint32_t>(); f.pvals1 = r->pvals1.as<uint32_t>();
        DL_TRY(ensure_pinned((void**)&r->h_u64, &r->h_u64_cap, 16ull * V + 64));
        for (uint32_t v = 0; v < V; v++) { r->h_u64[v] = (uint64_t)v * cap; r->h_u64[V + v] = cap; }
        DL_CK(cudaMemcpyAsync(f.pairBase, r->h_u64, 8ull * V, cudaMemcpyHostToDevice, st));
        DL_CK(cudaMemcpyAsync(f.pairCap, r->h_u64 + V, 8ull * V, cudaMemcpyHostToDevice, st));
        // a pending scene upload goes behind this frame's small copies
        if (f.upload && !f.upload->issued) DL_TRY(f.upload->issue());
        uint32_t* finalVals = nullptr;
        // the device sequence of the frame: clears, project, depth sort, pair stages
        auto sequence = [&]() -> int {
            DL_CK(cudaMemsetAsync(f.scr, 0, 4ull * kScratchWords, st));
            DL_CK(cudaMemsetAsync(f.nvis, 0, 4ull * V, st));
            if (f.evalCount) DL_CK(cudaMemsetAsync(f.evalCount, 0, 8, st));
            if (f.tileCycles) DL_CK(cudaMemsetAsync(f.tileCycles, 0, 4ull * d.totalTiles, st));
            uint64_t n = 0;
            DL_TRY(launch_front(f, d, sc, st, ev, &n));
            DL_TRY(launch_back(f, d, sc, st, ev, &n, &finalVals));
            r->launches = n;
            return DL_OK;
        };
        if (!useGraph) {
            DL_TRY(sequence());
        } else {
            // key: every pointer and size baked into the captured launches
            std::vector<uint64_t> key;
            const uint64_t* fp = reinterpret_cast<const uint64_t*>(&f);
            key.assign(fp, fp + sizeof(FramePtrs) / 8);
            const uint64_t* sp = reinterpret_cast<const uint64_t*>(&sc);
            key.insert(key.end(), sp, sp + sizeof(DlSceneDev) / 8);
            key.insert(key.end(), {V, N, d.maxT, d.TS, d.totalTiles, d.stride, d.cap, (uint64_t)flags, d.rasterGrid,
                                   (uint64_t)d.pbits, (uint64_t)d.subLw, (uint64_t)d.ppl2, (uint64_t)d.x2,
                                   (uint64_t)d.iptLg, (uint64_t)hv[0].tileW, (uint64_t)hv[0].tileH,
                                   (uint64_t)d.tileCta, (uint64_t)d.tileK,
                                   g_dl_wait.spin_limit,
                                   g_dl_wait.withheld(DL_WAIT_STAGE_DEPTH_SORT), g_dl_wait.withheld(DL_WAIT_STAGE_EMIT),
                                   g_dl_wait.withheld(DL_WAIT_STAGE_PAIR_SORT)});
            if (!r->graph_exec || key != r->graph_key) {
                if (r->graph_exec) { cudaGraphExecDestroy(r->graph_exec); r->graph_exec = nullptr; }
                cudaGraph_t g = nullptr;
                DL_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
                const int cs = sequence();
                const cudaError_t ce = cudaStreamEndCapture(st, &g);
                if (cs != DL_OK) { if (g) cudaGraphDestroy(g); return cs; }
                if (ce != cudaSuccess) { dl_set_error(std::string("stream capture: ") + cudaGetErrorString(ce)); return DL_E_CUDA; }
                const cudaError_t ie = cudaGraphInstantiate(&r->graph_exec, g, 0);
                cudaGraphDestroy(g);
                if (ie != cudaSuccess) { r->graph_exec = nullptr; dl_set_error(std::string("graph instantiate: ") + cudaGetErrorString(ie)); return DL_E_CUDA; }
                r->graph_key = key;
                r->graph_launches = r->launches;
                r->graph_final_vals = finalVals;
            } else {
                finalVals = r->graph_final_vals;
                r->launches = r->graph_launches;
            }
            DL_CK(cudaGraphLaunch(r->graph_exec, st));
            r->graph_replays++;
        }

        // one sync per frame: error word and pair totals
        DL_CK(cudaMemcpyAsync(r->h_u64, f.npairs, 8ull * V, cudaMemcpyDeviceToHost, st));
        DL_CK(cudaMemcpyAsync(r->h_u64 + V, f.scr + SC_ERR, 4, cudaMemcpyDeviceToHost, st));
        DL_CK(cudaMemcpyAsync(r->h_u64 + V + 1, f.scr + SC_OVF, 4, cudaMemcpyDeviceToHost, st));
        DL_CK(cudaStreamSynchronize(st));
        const uint32_t err = (uint32_t)(r->h_u64[V] & 0xffffffffu) | (uint32_t)(r->h_u64[V + 1] & 0xffffffffu);
        if (r->profiling) {
            float ms;
            const int from[6] = {0, 1, 3, 4, 5, 6}, to[6] = {1, 2, 4, 5, 6, 7};
            for (int k = 0; k < 6; k++)
                if (cudaEventElapsedTime(&ms, r->ev[from[k]], r->ev[to[k]]) == cudaSuccess) r->stage_ms[k] += ms;
        }
        if (err & DL_DEVERR_TIMEOUT) {
            dl_set_error("a bounded device-side wait timed out");
            return DL_E_TIMEOUT;
        }
        uint64_t maxPairs = 0;
        for (uint32_t v = 0; v < V; v++) maxPairs = std::max<uint64_t>(maxPairs, r->h_u64[v]);
        if (err & DL_DEVERR_OVERFLOW) {
            r->pair_cap_per_view = maxPairs + maxPairs / 4 + 4096;
            continue;
        }
        r->last_max_pairs = maxPairs;
        r->last_n = N;
        r->last_stride = (uint32_t)d.stride;
        r->last_T = hv[0].numTiles;
        r->last_W = hv[0].W;
        r->last_H = hv[0].H;
        r->last_pairs_final = (uint32_t)r->h_u64[0];
        r->last_rec_kind = d.f16rec ? 1 : 0;
        r->last_final_vals = finalVals;
        r->last_V = V;
        r->log_tiles = logTiles ? d.totalTiles : 0;
        return DL_OK;
    }
    r->pair_cap_per_view = capOnEntry;
    dl_set_error("pair buffers overflowed repeatedly");
    return DL_E_CAPACITY;
}

// ============================================================================
// dl_render_static: the single-view render with every piece of device scratch
// taken from one fixed, file-scope device array instead of cudaMalloc.
//
// Who needs it: code that runs inside a host application which owns all of
// the GPU's memory (an engine or framework that reserves the device up front
// with its own allocator and forbids foreign cudaMalloc/cudaFree), or a
// real-time loop that may not allocate after start-up.  Such callers can still
// render a small scene: this path allocates nothing, neither device memory nor
// pinned host memory; it only copies the caller's host arrays into the array
// below and the finished image back out.
//
// Limits (checked before anything runs, DL_E_CAPACITY with a message):
//   at most kStaticMaxSplats Gaussians, kStaticMaxPixels output pixels,
//   kStaticMaxTiles 16x16 tiles and kStaticMaxPairs tile pairs.
// The array is kStaticBytes (16 MiB) on every GPU that loads this library,
// held until the process exits.
//
// Sharing: every call on a device uses the same array and leaves the last
// call's contents in it; everything a call reads is written or cleared by that
// call first.  Calls whose GPU work overlaps (two host threads, or calls on
// different streams of one device) race on the array and must be serialised
// by the caller.  The first call on each device looks up the array's device
// address (cudaGetSymbolAddress) with that device current; make that first
// call before any stream capture on the device.  The address is kept for the
// life of the process: a cudaDeviceReset (or a reset of the primary context)
// unloads the array, and calls after it are not supported.
//
// Stream: the calling thread's per-thread default stream (cudaStreamPerThread),
// so the call does not wait on the other streams of the device; it
// synchronises that stream before returning.  Its copies from pageable host
// memory are not allowed while another thread captures a CUDA graph in
// cudaStreamCaptureModeGlobal.
// ============================================================================
namespace {

constexpr uint32_t kStaticMaxSplats = 16384;
constexpr uint64_t kStaticMaxPixels = 1280ull * 720ull;
constexpr uint32_t kStaticMaxTiles = 4096;
constexpr uint64_t kStaticMaxPairs = 1ull << 18;
constexpr size_t kStaticBytes = 16ull << 20;

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

constexpr int kStaticMaxDevices = 64;
// device address of g_static_scratch per device ordinal; threads that make
// their first call at once look it up alike and store the same value
std::atomic<unsigned char*> g_static_addr[kStaticMaxDevices] = {};

// Carves 256-byte-aligned pieces out of the array, in call order.
struct Carver {
    unsigned char* base;
    size_t off = 0;
    template <typename T> T* take(size_t bytes) {
        T* p = reinterpret_cast<T*>(base + off);
        off = (off + bytes + 255) / 256 * 256;
        return p;
    }
};

}  // namespace

extern "C" int dl_render_static(const dl_splats* data, const dl_camera* cam, const float bg[4],
                                uint32_t max_coverage, uint8_t* out_rgba, size_t out_len) {
    if (!data || !cam) { dl_set_error("dl_render_static: NULL argument"); return DL_E_INVALID_ARG; }
    const uint64_t pixels = (uint64_t)cam->width * cam->height;
    if (pixels == 0) return DL_OK;
    if (!out_rgba || out_len < pixels * 4) {
        dl_set_error("dl_render_static: output buffer smaller than width*height*4");
        return DL_E_INVALID_ARG;
    }
    if (data->count > kStaticMaxSplats) {
        dl_set_error("dl_render_static: at most " + std::to_string(kStaticMaxSplats) + " Gaussians (got " +
                     std::to_string(data->count) + ")");
        return DL_E_CAPACITY;
    }
    if (pixels > kStaticMaxPixels) {
        dl_set_error("dl_render_static: at most " + std::to_string(kStaticMaxPixels) + " pixels per image");
        return DL_E_CAPACITY;
    }
    DlView v;
    DL_TRY(dl_make_view(cam, bg, max_coverage ? max_coverage : 16384u, &v));
    if (v.numTiles > kStaticMaxTiles) {
        dl_set_error("dl_render_static: at most " + std::to_string(kStaticMaxTiles) + " 16x16 tiles per image");
        return DL_E_CAPACITY;
    }
    if (data->sh_bands < 0 || data->sh_bands > 3) { dl_set_error("sh_bands must be 0..3"); return DL_E_INVALID_ARG; }
    const uint64_t n = data->count;
    if (n > 0 && (!data->positions || !data->rotations || !data->log_scales || !data->opacity_logits || !data->colors_dc)) {
        dl_set_error("splats: a required array is NULL");
        return DL_E_INVALID_ARG;
    }
    int dev = 0;
    DL_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kStaticMaxDevices) { dl_set_error("dl_render_static: device ordinal too large"); return DL_E_CAPACITY; }
    unsigned char* base = g_static_addr[dev].load(std::memory_order_acquire);
    if (!base) {
        void* p = nullptr;
        DL_CK(cudaGetSymbolAddress(&p, g_static_scratch));
        base = static_cast<unsigned char*>(p);
        g_static_addr[dev].store(base, std::memory_order_release);
    }
    cudaStream_t st = cudaStreamPerThread;

    // ---- carve the array (same layout on every call)
    const int bands = data->colors_sh ? data->sh_bands : 0;
    const int M = bands == 0 ? 0 : bands == 1 ? 3 : bands == 2 ? 8 : 15;
    const uint32_t N = (uint32_t)n;
    const FrameDims d = frame_dims(&v, 1, N, kStaticMaxPairs, 0);
    Carver c{base};
    float* dPos = c.take<float>(12ull * kStaticMaxSplats);
    float* dRot = c.take<float>(16ull * kStaticMaxSplats);
    float* dLsc = c.take<float>(12ull * kStaticMaxSplats);
    float* dOpl = c.take<float>(4ull * kStaticMaxSplats);
    float* dDc = c.take<float>(12ull * kStaticMaxSplats);
    float* dSh = c.take<float>(180ull * kStaticMaxSplats);
    FramePtrs f;
    std::memset(&f, 0, sizeof(f));
    f.views = c.take<DlView>(sizeof(DlView));
    f.tileBase = c.take<uint32_t>(8);
    f.segStart = c.take<uint64_t>(8);
    f.segLen = c.take<uint32_t>(4);
    f.segTileBase = c.take<uint32_t>(8);
    f.scr = c.take<uint32_t>(4ull * kScratchWords);
    f.keys0 = c.take<uint32_t>(4ull * kStaticMaxSplats);
    f.keys1 = c.take<uint32_t>(4ull * kStaticMaxSplats);
    f.vals0 = c.take<uint32_t>(4ull * kStaticMaxSplats);
    f.vals1 = c.take<uint32_t>(4ull * kStaticMaxSplats);
    f.recA = c.take<float4>(16ull * kStaticMaxSplats);
    f.recBC = c.take<float4>(32ull * kStaticMaxSplats);
    f.bbox = c.take<uint2>(8ull * kStaticMaxSplats);
    f.nvis = c.take<uint32_t>(4);
    f.depthHist = c.take<uint32_t>(4ull * 4 * 256);
    const uint32_t maxSortTiles = (uint32_t)((kStaticMaxPairs + dlsort::kTile - 1) / dlsort::kTile);
    f.sortStatus = c.take<uint32_t>(4ull * 256 * maxSortTiles);
    f.outs = c.take<uint32_t*>(sizeof(void*));
    f.tileOff = c.take<uint32_t>(4ull * (kStaticMaxTiles + 1));
    f.pairBase = c.take<uint64_t>(8);
    f.pairCap = c.take<uint64_t>(8);
    f.npairs = c.take<unsigned long long>(8);
    f.pairSegLen = c.take<uint32_t>(4);
    f.pairSegTileBase = c.take<uint32_t>(4);
    f.pairGlob = c.take<uint32_t>(4ull * 4 * 256);
    f.pairHist = c.take<uint32_t>(4ull * 4 * 256);
    f.emitStatus = c.take<unsigned long long>(8ull * ((kStaticMaxSplats + dlr::kEmitRanks - 1) / dlr::kEmitRanks));
    f.pkeys0 = c.take<uint32_t>(4ull * kStaticMaxPairs);
    f.pkeys1 = c.take<uint32_t>(4ull * kStaticMaxPairs);
    f.pvals0 = c.take<uint32_t>(4ull * kStaticMaxPairs);
    f.pvals1 = c.take<uint32_t>(4ull * kStaticMaxPairs);
    uint32_t* rgba = c.take<uint32_t>(4ull * kStaticMaxPixels);
    if (c.off > kStaticBytes) { dl_set_error("dl_render_static: scratch layout exceeds the array"); return DL_E_CAPACITY; }

    // ---- inputs (pageable host copies are staged by the driver; nothing is allocated here)
    if (n) {
        DL_CK(cudaMemcpyAsync(dPos, data->positions, 12 * n, cudaMemcpyHostToDevice, st));
        DL_CK(cudaMemcpyAsync(dRot, data->rotations, 16 * n, cudaMemcpyHostToDevice, st));
        DL_CK(cudaMemcpyAsync(dLsc, data->log_scales, 12 * n, cudaMemcpyHostToDevice, st));
        DL_CK(cudaMemcpyAsync(dOpl, data->opacity_logits, 4 * n, cudaMemcpyHostToDevice, st));
        DL_CK(cudaMemcpyAsync(dDc, data->colors_dc, 12 * n, cudaMemcpyHostToDevice, st));
        if (M) DL_CK(cudaMemcpyAsync(dSh, data->colors_sh, 12ull * M * n, cudaMemcpyHostToDevice, st));
    }
    const uint64_t segStart = 0;
    const uint32_t segLen = N;
    uint32_t* outPtr = rgba;
    const uint64_t pairBaseH = 0, pairCapH = kStaticMaxPairs;
    DL_CK(cudaMemcpyAsync(f.views, &v, sizeof(DlView), cudaMemcpyHostToDevice, st));
    const uint32_t tileBaseH[2] = {0u, v.numTiles};
    DL_CK(cudaMemcpyAsync(f.tileBase, tileBaseH, 8, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.segStart, &segStart, 8, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.segLen, &segLen, 4, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.outs, &outPtr, sizeof(void*), cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.pairBase, &pairBaseH, 8, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemcpyAsync(f.pairCap, &pairCapH, 8, cudaMemcpyHostToDevice, st));
    DL_CK(cudaMemsetAsync(f.scr, 0, 4ull * kScratchWords, st));
    DL_CK(cudaMemsetAsync(f.nvis, 0, 4, st));

    DlSceneDev sc{};
    sc.pos = dPos; sc.rot = dRot; sc.lsc = dLsc; sc.opl = dOpl; sc.dc = dDc;
    sc.sh = M ? dSh : nullptr; sc.sh16 = nullptr; sc.sh16_stride = 0; sc.n = N; sc.bands = bands; sc.sh_kind = 0;

    uint64_t launches = 0;
    uint32_t* finalVals = nullptr;
    DL_TRY(launch_front(f, d, sc, st, nullptr, &launches));
    DL_TRY(launch_back(f, d, sc, st, nullptr, &launches, &finalVals));

    uint32_t flagsH[2] = {0, 0};
    DL_CK(cudaMemcpyAsync(&flagsH[0], f.scr + SC_ERR, 4, cudaMemcpyDeviceToHost, st));
    DL_CK(cudaMemcpyAsync(&flagsH[1], f.scr + SC_OVF, 4, cudaMemcpyDeviceToHost, st));
    DL_CK(cudaMemcpyAsync(out_rgba, rgba, pixels * 4, cudaMemcpyDeviceToHost, st));
    DL_CK(cudaStreamSynchronize(st));
    if (flagsH[0] & DL_DEVERR_TIMEOUT) { dl_set_error("a bounded device-side wait timed out"); return DL_E_TIMEOUT; }
    if (flagsH[1] & DL_DEVERR_OVERFLOW) {
        dl_set_error("dl_render_static: more than " + std::to_string(kStaticMaxPairs) + " tile pairs in this view");
        return DL_E_CAPACITY;
    }
    return DL_OK;
}

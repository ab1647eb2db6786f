// dl_internal.h — host-side internals shared by the C-ABI translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <functional>
#include <vector>

#include "../../include/droplet_b200.h"
#include "dl_common.cuh"

void dl_set_error(const std::string& msg);

#define DL_CK(call)                                                                          \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) {                                                             \
            dl_set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                \
            return e_ == cudaErrorMemoryAllocation ? DL_E_OOM : DL_E_CUDA;                   \
        }                                                                                    \
    } while (0)

#define DL_TRY(expr)                  \
    do {                              \
        int s_ = (expr);              \
        if (s_ != DL_OK) return s_;   \
    } while (0)

// Test hook (dl_test_fail_allocation): the number of device allocations that
// still succeed before one is refused as if the device were out of memory;
// negative: none is refused.
extern int g_dl_alloc_budget;

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int ensure(size_t need) {
        if (need <= bytes && p) return DL_OK;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        const size_t alloc = need < 256 ? 256 : need;
        if (g_dl_alloc_budget == 0) {
            g_dl_alloc_budget = -1;
            dl_set_error(std::string("cudaMalloc(") + std::to_string(alloc) + "): out of memory (refused by the test hook)");
            return DL_E_OOM;
        }
        if (g_dl_alloc_budget > 0) g_dl_alloc_budget--;
        cudaError_t e = cudaMalloc(&p, alloc);
        if (e != cudaSuccess) {
            p = nullptr;
            dl_set_error(std::string("cudaMalloc(") + std::to_string(alloc) + "): " + cudaGetErrorString(e));
            return DL_E_OOM;
        }
        bytes = alloc;
        return DL_OK;
    }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T* as() const { return static_cast<T*>(p); }
};

// Bounded device waits (decoupled look-backs): how many polls of an
// unpublished predecessor a CTA makes before it gives up with
// DL_DEVERR_TIMEOUT, and a test hook that makes one CTA of one stage withhold
// its status so that its successors run into that limit (dl_test_* entry
// points; the defaults leave every stage as it is).
enum { DL_WAIT_STAGE_NONE = 0, DL_WAIT_STAGE_DEPTH_SORT = 1, DL_WAIT_STAGE_EMIT = 2, DL_WAIT_STAGE_PAIR_SORT = 3 };
struct DlWaitPlan {
    uint32_t spin_limit = DL_SPIN_LIMIT;
    int withhold_stage = DL_WAIT_STAGE_NONE;
    uint32_t withhold_tile = 0xffffffffu;
    uint32_t withheld(int stage) const { return withhold_stage == stage ? withhold_tile : 0xffffffffu; }
};
extern DlWaitPlan g_dl_wait;

struct dl_mlp;
struct VoxBufs;

struct dl_device {
    int ordinal = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    VoxBufs* vox = nullptr;             // the voxelizer's grow-only device buffers
    dl_mlp* vox_sched = nullptr;        // block-cost model ordering the voxel work queue
};

// dl_voxel.cu: releases the voxelizer's buffers of a device
void dl_vox_release(dl_device* dev);

struct dl_scene {
    dl_device* dev = nullptr;
    DevBuf mem;
    DlSceneDev d{};
    int precision = DL_PREC_F32;
};

// Knobs of a batched frame that change timing only (dl_tuning in the ABI).
struct DlTuning {
    int pair_bits = 8;        // pair-sort digit width 6..8
    int shape = 5;            // rasterizer: 0 8x4, 1 16x2, 2 4x8, 3 8x8 (two pixels per lane) warp items,
                              // 4 8x4 packed, 5 one CTA per tile packed (fast frames; others use 0), 6 one CTA
                              // per tile in place
    int ctas_per_sm = 0;      // persistent rasterizer CTAs per SM; 0 = occupancy limit
    int bin_tile = 0;         // binning tile: 0 16x16 (the reference's), 1 8x8, 2 32x8
};

constexpr int kUploadChunks = 8;   // splat ranges of an upload that overlaps projection
constexpr int kReadBackGroups = 8; // view ranges of a rasterizer whose images are read back meanwhile

// Host-side state of the tile-binned renderer.
struct dl_renderer {
    dl_device* dev = nullptr;
    uint32_t chunk_cap = 200000;
    uint32_t max_cov = 16384;
    cudaStream_t stream = nullptr;      // effective stream
    cudaStream_t own_stream = nullptr;

    // frame buffers (grow-only)
    DevBuf views, tileBase, segStart, segLen, segTileBase, scratch;     // scratch: counters + error word
    DevBuf keys0, keys1, vals0, vals1, recA, recBC, recH, bbox, nvis;
    DevBuf depthHist, sortStatus;
    DevBuf pairBase, pairCap, pkeys0, pkeys1, pvals0, pvals1, npairs, emitStatus;
    DevBuf tileCount, tileOff, pairSegLen, pairSegTileBase, pairGlob, outs, accum, tileEvals, work;
    dl_scene own_scene;                 // upload target of dl_render()

    // host mirrors
    DlView* h_views = nullptr;          // pinned
    size_t h_views_cap = 0;
    uint64_t* h_u64 = nullptr;          // pinned scratch
    size_t h_u64_cap = 0;
    uint64_t pair_cap_per_view = 0;
    uint64_t last_max_pairs = 0;          // largest view's tile pairs in the last frame that fit

    // last frame (single view) for debug copies
    uint32_t last_n = 0, last_stride = 0, last_T = 0, last_W = 0, last_H = 0, last_pairs_final = 0;
    int last_rec_kind = 0;
    uint32_t* last_final_vals = nullptr;
    uint32_t last_V = 0;
    DevBuf evalCount;
    DevBuf rgba;                        // device output of dl_render()
    bool keep_accum = false;
    bool keep_depth_keys = true;

    // profiling
    bool profiling = false;
    cudaEvent_t ev[8] = {};
    double stage_ms[6] = {0, 0, 0, 0, 0, 0};
    uint64_t launches = 0;

    // CUDA graph of the last batched frame, replayed while its key matches
    cudaGraphExec_t graph_exec = nullptr;
    std::vector<uint64_t> graph_key;
    uint64_t graph_launches = 0;
    uint64_t graph_replays = 0;
    uint32_t* graph_final_vals = nullptr;

    // learned schedule and tile-cost logging
    dl_mlp* sched = nullptr;
    DevBuf visMask;           // deferred-colour record bits [ceil(V/32)][N]
    DevBuf feat, pred, skeys0, skeys1, svals0, svals1, sseg, sstatus, shist, tileCycles;
    uint32_t log_tiles = 0;

    DlTuning tune;                      // dl_renderer_set_tuning / dl_renderer_autotune
    DevBuf tuneOut;                     // autotuner's device images

    // read-back of host-output batches, overlapped with rendering
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t copy_event = nullptr;
    // host-output frames: the odd rasterizer view ranges run on a second stream
    cudaStream_t raster_stream = nullptr;
    cudaEvent_t raster_ev[2] = {nullptr, nullptr};
    cudaEvent_t upload_events[2 * kUploadChunks + 1] = {};   // geometry chunks, SH chunks, all SH
};

struct dl_mlp;
int dl_mlp_infer_launch(const dl_mlp* mlp, const float* X, uint32_t n, float* out, cudaStream_t st);
const void* dl_mlp_weights(const dl_mlp* mlp);   // device BF16 parameters

// dl_render.cu
// A scene upload issued in splat ranges on a second stream: chunk c holds
// splats [bounds[c], bounds[c+1]) and is complete when events[c] has fired.
// With SH bands, the SH coefficients follow the geometry of all chunks,
// complete when sh_event has fired (sh_separate = 1), so that frames can defer
// colours until then.  dl_upload_scene lays the scene out and returns; the
// frame calls issue() once its own small host-to-device copies are queued, so
// that they do not wait behind the upload.  The SH arrives chunk by chunk as
// f32 at sh_src (sh_events[c]: chunk c's coefficients are there); with a
// 16-bit scene (sh_dst set) the frame converts them to the scene's layout
// (sh_P halves per splat, dl_upload_convert_sh) once they have arrived.
struct DlUploadChunks {
    int count;
    uint32_t bounds[kUploadChunks + 1];
    cudaEvent_t events[kUploadChunks];
    int sh_separate;
    cudaEvent_t sh_event;
    cudaEvent_t sh_events[kUploadChunks];
    const float* sh_src = nullptr;
    uint16_t* sh_dst = nullptr;
    int sh_M = 0, sh_P = 0, sh_kind = 0;
    std::function<int()> issue;
    bool issued = false;
};
// Copies that overlap a frame's kernels: projection of each uploaded splat
// range starts when its chunk has arrived, and the rasterizer runs as `groups`
// launches over view ranges, each range's images copied to host[v] on `stream`
// while the next range rasterizes.  The caller synchronises `stream`.
struct DlOverlap {
    int groups;
    uint8_t* const* host;
    cudaStream_t stream;
    cudaEvent_t event;
    const DlUploadChunks* upload;  // NULL: the scene is resident
};
int dl_render_views(dl_renderer* r, const DlSceneDev& sc, const DlView* hviews, uint32_t V,
                    uint32_t* const* d_outs, uint32_t flags, const DlOverlap* overlap = nullptr);
int dl_upload_scene(dl_scene* s, const dl_splats* data, int precision, cudaStream_t stream,
                    DlUploadChunks* chunks = nullptr);
int dl_make_view(const dl_camera* cam, const float bg[4], uint32_t maxCov, DlView* out);
// Converts splats [g0, g1) of a chunked upload's SH to the scene's 16-bit
// layout on st (nothing for an f32 scene); the caller orders it after the
// chunks' sh_events.
int dl_upload_convert_sh(const DlUploadChunks* up, uint32_t g0, uint32_t g1, cudaStream_t st, uint64_t* launches);

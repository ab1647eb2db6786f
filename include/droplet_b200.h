/* droplet_b200.h — C ABI of libdroplet_b200.so, the B200 (sm_100a) engine
 * behind droplet's TypeScript API.
 *
 * The TypeScript surface stays as it is (src/index.ts:16-38); a thin shim
 * calls these entry points through bun:ffi.  Each entry point cites the
 * reference interface it replaces.  Paths are relative to the droplet
 * repository.
 *
 * Conventions
 *   - Every function returns an int status: DL_OK (0) or a DL_E_* code; the
 *     message of the last failure on the calling thread is dl_last_error().
 *     The shim turns a non-zero status into `throw new Error(msg)`, which is
 *     how the reference reports setup failures (src/gpu/device.ts:27-41).
 *   - Host arrays are borrowed read-only for the duration of a call
 *     (src/render/preprocess.ts:90-138 copies them the same way); outputs are
 *     written into caller-allocated memory.
 *   - Handles are not thread-safe: one caller at a time per handle (the
 *     reference's Renderer shares scratch between calls the same way,
 *     src/render/pipeline.ts:5-8); distinct handles are independent.
 */
#ifndef DROPLET_B200_H
#define DROPLET_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DL_OK = 0,
    DL_E_INVALID_ARG = 1,   /* bad pointer, size or option */
    DL_E_OOM = 2,           /* device or pinned allocation failed */
    DL_E_CUDA = 3,          /* a CUDA runtime call failed */
    DL_E_TIMEOUT = 4,       /* a bounded device-side wait gave up (no hang) */
    DL_E_CAPACITY = 5,      /* a size exceeds a documented limit */
    DL_E_NO_DEVICE = 6      /* no usable CUDA device */
};

enum { DL_PINHOLE = 0, DL_EQUIRECT = 1 };              /* src/types.ts:70 Projection */
enum { DL_PREC_F32 = 0, DL_PREC_F16 = 1, DL_PREC_BF16 = 2 };

typedef struct dl_device dl_device;
typedef struct dl_renderer dl_renderer;
typedef struct dl_scene dl_scene;
typedef struct dl_vox_result dl_vox_result;

/* src/types.ts:23-32 SplatData: struct of arrays, all float32, N = count.
 * colors_sh: per Gaussian 3*M channel-major terms (R[M], G[M], B[M]),
 * M = 0/3/8/15 for sh_bands 0..3 (src/types.ts:35-37); may be NULL. */
typedef struct dl_splats {
    uint64_t count;
    const float* positions;       /* 3N xyz */
    const float* rotations;       /* 4N [w, x, y, z] */
    const float* log_scales;      /* 3N */
    const float* opacity_logits;  /* N */
    const float* colors_dc;       /* 3N */
    const float* colors_sh;       /* 3MN or NULL */
    int32_t sh_bands;             /* 0..3 */
} dl_splats;

/* src/types.ts:74-82 RenderCamera (JS numbers are f64 here). */
typedef struct dl_camera {
    uint32_t width, height;
    float view[16];               /* world->camera, column-major (Float32Array) */
    double fov_y, near_plane, far_plane;
    int32_t projection;           /* DL_PINHOLE or DL_EQUIRECT */
} dl_camera;

/* src/render/pipeline.ts:43-48 RendererOptions; 0 selects the default. */
typedef struct dl_renderer_opts {
    uint32_t chunk_cap;               /* default 200000; results never depend on it */
    uint32_t max_coverage_per_splat;  /* default 16384 */
} dl_renderer_opts;

/* src/voxel/voxelize.ts:29-36 VoxelizeOptions. */
typedef struct dl_vox_opts {
    double voxel_resolution;      /* default 0.05 when <= 0 is passed with use_defaults */
    double opacity_cutoff;        /* default 0.1 */
    int32_t use_defaults;         /* 1: ignore the two fields above */
    int32_t has_bounds;           /* 1: use bounds_min/bounds_max (opts.bounds) */
    double bounds_min[3];
    double bounds_max[3];
    /* Multi-GPU sharding (no reference counterpart): with shard_count > 1 the
     * call voxelizes only shard shard_index of the grid's z rows of 16^3-block
     * batches, split into shard_count contiguous row ranges of about equal
     * Gaussian-block pair counts (equal row counts when opacity_cutoff <= 0).  Bounds and dims stay those of the whole
     * grid; concatenating the block lists of shards 0..count-1 gives the
     * unsharded list in the reference's order.  0 / 0 voxelizes everything. */
    int32_t shard_index;
    int32_t shard_count;
    /* 1: keep per-block features and measured cost (dl_vox_result_block_log) */
    int32_t log_blocks;
    /* DL_VOX_FAST_EXP: the density exponentials use the hardware ex2 instead
     * of the library's exact-rounding exp; voxels whose opacity lies within
     * about 1e-5 of the cutoff may then change (no reference counterpart). */
    uint32_t flags;
} dl_vox_opts;
#define DL_VOX_FAST_EXP 1u
/* DL_VOX_PROFILE: record the device time of the call's stages, read by
 * dl_vox_result_stage_times */
#define DL_VOX_PROFILE 2u

/* ---- errors ------------------------------------------------------------ */
/* Message of the last failure on this thread ("" if none). */
const char* dl_last_error(void);

/* ---- device: src/gpu/device.ts:27-41 createDevice ---------------------- */
int dl_device_open(int ordinal, dl_device** out);
int dl_device_close(dl_device* dev);

/* ---- renderer: src/render/pipeline.ts:76-84 constructor, :581-591 destroy */
int dl_renderer_create(dl_device* dev, const dl_renderer_opts* opts, dl_renderer** out);
int dl_renderer_destroy(dl_renderer* r);
/* Run the renderer's kernels on a caller-provided cudaStream_t (NULL: the
 * renderer's own stream).  Lets a caller time kernels with its own events. */
int dl_renderer_set_stream(dl_renderer* r, void* cuda_stream);

/* src/render/pipeline.ts:181-426 Renderer.render(data, camera, background):
 * writes width*height RGBA8 pixels (finalize.ts packing) into out_rgba.
 * bg = (r, g, b, a) in [0, 1]; NULL means (0, 0, 0, 1). */
int dl_render(dl_renderer* r, const dl_splats* data, const dl_camera* cam, const float bg[4],
              uint8_t* out_rgba, size_t out_len);

/* ---- device-resident scenes and batched views (no reference counterpart:
 * the reference re-uploads SplatData on every render, pipeline.ts:221-228) */
int dl_scene_upload(dl_renderer* r, const dl_splats* data, int sh_precision, dl_scene** out);
int dl_scene_free(dl_scene* s);

enum {
    DL_BATCH_OUT_DEVICE = 1,      /* outs[i] are device pointers */
    DL_BATCH_PLAIN = 2,           /* one launch sequence per view, f32 records, static schedule */
    DL_BATCH_F16_RECORDS = 4,     /* projected conic/alpha/colour stored as f16 */
    DL_BATCH_NO_GRAPH = 8,        /* launch directly instead of replaying a CUDA graph */
    DL_BATCH_STATIC = 16,         /* rasterize tiles in launch order, not cost order */
    DL_BATCH_FAST_EXP = 32,       /* hardware ex2 in the rasterizer (+-1 LSB) */
    DL_BATCH_COUNT_EVALS = 64,    /* count evaluated (pixel, splat) pairs ("evals") */
    DL_BATCH_LOG_TILES = 128,     /* keep per-tile features and measured cost (dl_renderer_tile_log) */
    DL_BATCH_F64_DEGENERATE = 256,/* f64 determinant and inverse for near-degenerate 2D covariances
                                     (det < 2^-10 c00 c11); culling and tile ranges unchanged */
    DL_BATCH_SH16 = 512,          /* dl_render_many: keep the uploaded SH coefficients in f16 */
    DL_BATCH_CULL_OFFSCREEN = 1024 /* work that cannot change a pixel is left out: splats with no tile on
                                      the image, and splats whose alpha reaches 1/255 nowhere, leave the
                                      depth order; untruncated splats are binned by the box of their
                                      ellipse q <= min(9.5, 1.002 qa + 0.01), qa = -2 ln(exp(-4.5) +
                                      1/(255 opacity)) being the q where alpha falls to 1/255; and the
                                      screen record ("recA") holds (x, y, half-width, half-height) of the
                                      box the rasterizer tests.  Pixels are unchanged; tile lists and
                                      depth ranks then differ from the reference's. */
};
/* Render n views of one resident scene; outs[i] receives cams[i].width *
 * cams[i].height RGBA8 pixels (host or device memory, per flags). */
int dl_render_batch(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4],
                    uint8_t* const* outs, uint32_t flags);

/* Renderer.render(data, camera, bg) (src/render/pipeline.ts:181-426) for n
 * cameras of one host SplatData in one call: the splats are uploaded into the
 * renderer's own grow-only scene buffer, all views are rendered as one batch,
 * and each RGBA8 image is copied to outs[i] (host memory).  With 8 or more
 * views the copies overlap the frame on a second stream: the splats' geometry
 * uploads in 8 ranges, each projected as soon as it has arrived, the SH
 * coefficients follow while depth sort, binning and pair sort run (colours are
 * evaluated once they have arrived), and the rasterizer runs over 8 view
 * ranges, each range's images copied back while the next range rasterizes
 * (dl_render_batch with host outputs and 8+ views does the same read-back).
 * The data arrays must stay unchanged until the call returns. */
int dl_render_many(dl_renderer* r, const dl_splats* data, const dl_camera* cams, int n, const float bg[4],
                   uint8_t* const* outs, uint32_t flags);

/* No counterpart in the reference.  For callers that cannot allocate GPU
 * memory (an application that owns the whole device through its own
 * allocator, or a real-time loop that may not allocate after start-up): the
 * single-view render of dl_render with no renderer handle, on the current CUDA
 * device, with all device scratch taken from one 16 MiB array that the
 * library reserves statically on every GPU that loads it.  Limits: 16384
 * Gaussians, 921600 pixels (e.g. 1280x720), 4096 16x16 tiles, 262144 tile
 * pairs; beyond them it returns DL_E_CAPACITY.  Calls that overlap on one GPU
 * race on the shared array.  The first call on a device looks the array up
 * and should come before any stream capture there; after a cudaDeviceReset
 * of that device the call is not supported.  It runs on the calling thread's
 * per-thread default stream (no wait on the device's other streams) and
 * returns after that stream has finished; its pageable host copies are not
 * allowed while another thread captures a graph in global capture mode.
 * max_coverage 0 selects the default 16384. */
int dl_render_static(const dl_splats* data, const dl_camera* cam, const float bg[4], uint32_t max_coverage,
                     uint8_t* out_rgba, size_t out_len);

/* ---- tuning (no reference counterpart) -----------------------------------
 * Knobs of rendered frames that change timing only, never a pixel.  The
 * binning tile may be 8x8 or 32x8 instead of the reference's 16x16 TILE_SIZE
 * only for frames where no splat's coverage can be truncated (every view's
 * 16x16 tile count at most maxCoveragePerSplat); the truncation keeps a
 * row-major prefix of 16x16 tiles, so other frames bin with 16x16 tiles. */
typedef struct dl_tuning {
    int32_t pair_sort_bits;       /* digit width of the tile-pair sort: 6, 7 or 8 (default 8) */
    int32_t raster_shape;         /* rasterizer (default 5): pixels of one work item (one warp): 0 = 8x4, 1 = 16x2, 2 = 4x8,
                                     3 = 8x8 with two pixels per lane, 4 = 8x4 taking two splats per step
                                     in packed f32x2 arithmetic, 5 = the same with one CTA per 256-pixel
                                     tile reading the tile's pairs once (4 and 5: DL_BATCH_FAST_EXP frames,
                                     others use 0; 5 with 8x8 tiles uses 4), 6 = one CTA per 256-pixel tile
                                     compositing the staged records in place, either arithmetic (with 8x8
                                     tiles it uses 0) */
    int32_t raster_ctas_per_sm;   /* persistent rasterizer CTAs per SM, 1..5; 0 = the occupancy limit */
    int32_t bin_tile;             /* binning tile: 0 = 16x16 (default), 1 = 8x8, 2 = 32x8; work items that do
                                     not fit the tile fall back to 8x4 */
} dl_tuning;
int dl_renderer_set_tuning(dl_renderer* r, const dl_tuning* t);
int dl_renderer_get_tuning(dl_renderer* r, dl_tuning* t);
/* Autotuner: renders the n views of s (flags as dl_render_batch, outputs kept
 * on the device) under candidate tunings — coordinate descent over the four
 * knobs from the current tuning — timing each as the median of `reps` frames
 * (CUDA events on the renderer's stream, after one warm-up frame), keeps the
 * fastest on the renderer and returns it with its frame time in ms. */
int dl_renderer_autotune(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4],
                         uint32_t flags, int reps, dl_tuning* best, double* best_ms);

/* ---- learned schedule (no reference counterpart: the reference rasterizes
 * tiles in dispatch order, src/render/pipeline.ts:402-422).  A small MLP
 * (DL_MLP_IN features -> 64 -> 64 -> 1, ReLU, BF16 weights, FP32 accumulation)
 * predicts each tile's rasterizer cost; with a scheduler attached, batched
 * frames (not DL_BATCH_PLAIN / DL_BATCH_STATIC) rasterize tiles in decreasing
 * predicted cost.  The order changes timing only, never a pixel. */
#define DL_MLP_IN 12
#define DL_MLP_HIDDEN 64
#define DL_MLP_PARAMS (DL_MLP_IN * DL_MLP_HIDDEN + DL_MLP_HIDDEN + DL_MLP_HIDDEN * DL_MLP_HIDDEN + DL_MLP_HIDDEN + \
                       DL_MLP_HIDDEN + 1)
typedef struct dl_mlp dl_mlp;
int dl_mlp_create(dl_device* dev, uint64_t seed, dl_mlp** out);
int dl_mlp_destroy(dl_mlp* mlp);
/* FP32 master parameters, layout W1[IN][H], b1[H], W2[H][H], b2[H], W3[H], b3. */
int dl_mlp_get_params(dl_mlp* mlp, float* out, size_t n);
int dl_mlp_set_params(dl_mlp* mlp, const float* in, size_t n);
/* X: n x DL_MLP_IN row-major host array; out: n predictions. */
int dl_mlp_predict(dl_mlp* mlp, const float* X, uint64_t n, float* out);
/* Gradient of the mean squared error over the n samples w.r.t. the parameters. */
int dl_mlp_grad(dl_mlp* mlp, const float* X, const float* y, uint64_t n, float* grad_out, float* loss_out);
/* Adam on mini-batches of `batch` samples, reshuffled each epoch from `seed`. */
int dl_mlp_train(dl_mlp* mlp, const float* X, const float* y, uint64_t n, int epochs, int batch, float lr,
                 uint64_t seed, float* loss_out);
/* Attach (or with NULL detach) the cost model that orders batched frames. */
int dl_renderer_set_scheduler(dl_renderer* r, dl_mlp* mlp);
/* After a frame rendered with DL_BATCH_LOG_TILES: per tile (views in order,
 * tiles row-major) its DL_MLP_IN features and measured cost (SM cycles / 16
 * summed over the tile's warps).  *n receives the tile count. */
int dl_renderer_tile_log(dl_renderer* r, float* features, float* cost, uint64_t cap, uint64_t* n);

/* ---- voxelizer: src/voxel/voxelize.ts:59-248 voxelize(device, data, opts) */
int dl_voxelize(dl_device* dev, const dl_splats* data, const dl_vox_opts* opts, dl_vox_result** out);
/* VoxelizeResult {bounds, numBlocksX/Y/Z} (voxelize.ts:38-45) and the block
 * count of its BlockMaskBuffer (block-mask-buffer.ts:57).  dims may be
 * -Infinity for an empty input, as in the reference. */
int dl_vox_result_info(const dl_vox_result* res, double bounds_min[3], double bounds_max[3],
                       double dims[3], uint64_t* block_count);
/* BlockMaskBuffer.blocks (block-mask-buffer.ts:27) in the reference's order:
 * flat block index, low 32 voxel bits, high 32 voxel bits. */
int dl_vox_result_copy(const dl_vox_result* res, uint32_t* block_idx, uint32_t* mask_lo, uint32_t* mask_hi);
int dl_vox_result_free(dl_vox_result* res);
/* No counterpart in the reference (its BlockMaskBuffer answers get(blockIdx) one
 * block at a time on the CPU, src/voxel/block-mask-buffer.ts:41-58): occupancy of
 * npoints points (x, y, z f32, host memory) against a block-mask buffer (the
 * arrays dl_vox_result_copy returns, or any BlockMaskBuffer's; a block listed
 * twice is OR-merged as addBlock does), on the device — a collision test against
 * the voxelizer's output.  A point lies in voxel floor((p - bounds_min) /
 * voxel_resolution) per axis (f64); out[i] (host) = 1 when that voxel's bit is
 * set in its block (flat index bx + by*dims[0] + bz*dims[0]*dims[1], bit
 * (z&3)*16 + (y&3)*4 + (x&3) of the voxel in the block, lo = bits 0-31), else 0,
 * also for points outside the 4*dims voxel grid, non-finite points and an
 * empty grid.  Synchronous; device memory is allocated for the call. */
int dl_vox_query(dl_device* dev, const uint32_t* block_idx, const uint32_t* mask_lo, const uint32_t* mask_hi,
                 uint64_t nblocks, const double bounds_min[3], double voxel_resolution, const double dims[3],
                 const float* points, uint64_t npoints, uint8_t* out);
/* No counterpart in the reference (its voxelize.ts:1-14 names carve among the
 * downstream stages of the block-mask buffer without building it): A minus B,
 * block by block, on the device.  Each of A's na entries (host arrays as
 * dl_vox_result_copy returns them) keeps the bits that B's entries with the same
 * flat index (OR-merged) do not set; entries left empty are dropped and the rest
 * keep A's order.  out_idx/out_lo/out_hi (host) hold na entries; *out_n gets the
 * count written.  Synchronous; device memory is allocated for the call. */
int dl_vox_carve(dl_device* dev, const uint32_t* a_idx, const uint32_t* a_lo, const uint32_t* a_hi, uint64_t na,
                 const uint32_t* b_idx, const uint32_t* b_lo, const uint32_t* b_hi, uint64_t nb, uint32_t* out_idx,
                 uint32_t* out_lo, uint32_t* out_hi, uint64_t* out_n);
/* Learned block order (no reference counterpart: the reference evaluates
 * batches in dispatch order, voxelize.ts:186-248).  With a model attached,
 * dl_voxelize on this device evaluates blocks in decreasing cost predicted
 * from DL_MLP_IN per-block features (the block's and its neighbours' list
 * lengths, a sample of its Gaussians' opacity and size, its place in the
 * batch, the cutoff); the order changes timing only, never a bit.  NULL detaches. */
int dl_device_set_voxel_scheduler(dl_device* dev, dl_mlp* mlp);
/* After dl_voxelize with log_blocks: per evaluated block, in block order of
 * each slab, its DL_MLP_IN features and measured cost (SM cycles / 16). */
int dl_vox_result_block_log(const dl_vox_result* res, float* features, float* cost, uint64_t cap, uint64_t* n);
/* Device ms per stage of a call made with DL_VOX_PROFILE (no reference
 * counterpart): prep (upload, extents, bounds, batch counts), binning, sort,
 * block heads (and the learned order), evaluation, compaction, and the time
 * the device waits for the host between slabs (set-up, result copies). */
int dl_vox_result_stage_times(const dl_vox_result* res, double* ms, int n);

/* ---- src/io/ply.ts:120-239 loadPlySplats --------------------------------
 * Parses a 3DGS PLY held in memory (bytes, len) into the SoA arrays of a
 * dl_splats, with the reference loader's header rules, transforms (flipY:
 * y, and the quaternion's x and z, negated; f_dc times SH_C0; quaternions
 * normalized) and error messages (DL_E_INVALID_ARG, message in
 * dl_last_error).  With DL_PLY_PINNED the arrays are page-locked host memory,
 * so that dl_scene_upload / dl_render move them to the device without a
 * staging copy (needs a CUDA device); otherwise ordinary host memory.  The
 * arrays live until dl_ply_free; dl_ply_splats points a dl_splats at them. */
#define DL_PLY_PINNED 1u
typedef struct dl_ply dl_ply;
int dl_ply_load(const uint8_t* bytes, size_t len, int flip_y, uint32_t flags, dl_ply** out);
int dl_ply_splats(const dl_ply* p, dl_splats* out);
int dl_ply_free(dl_ply* p);

/* ---- src/gpu/radix-sort.ts:91-216 GpuRadixSorter ----------------------- */
/* Stable LSD radix sort of n u32 keys with u32 values in device memory (the
 * reference's sorter is not stable; a stable order is one it may return).
 * keys must be below 2^key_bits (key_bits 0 means 32), as the reference
 * assumes.  vals may be NULL: values are then the input positions (an
 * argsort).  On return *out_keys / *out_vals point at the sorted arrays —
 * the inputs or the sorter's own grow-only pong buffers, valid until the next
 * sort or destroy — as GpuRadixSorter.sort returns its buffer pair
 * (radix-sort.ts:137-215).  Input arrays are overwritten.  The call returns
 * after the sort has finished on the sorter's stream. */
typedef struct dl_sorter dl_sorter;
int dl_sorter_create(dl_device* dev, dl_sorter** out);        /* radix-sort.ts:101-123 */
int dl_sorter_destroy(dl_sorter* s);
int dl_sorter_set_stream(dl_sorter* s, void* cuda_stream);
/* digit width of the passes: 6, 7 or 8 bits (default 8) */
int dl_sorter_set_digit_bits(dl_sorter* s, int bits);
int dl_sorter_sort(dl_sorter* s, uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits,
                   uint32_t** out_keys, uint32_t** out_vals);

/* ---- instrumentation (no reference counterpart) ------------------------ */
/* Copy a named device array of the last single-view render into dst (cap
 * bytes); *bytes receives its size.  Names: "depth_keys", "sorted_idx",
 * "recA", "recBC", "bbox", "tile_off", "pair_vals", "accum", "nvis", "npairs"
 * (one u64 per view of the last frame), "evals" (u64, with DL_BATCH_COUNT_EVALS). */
int dl_renderer_debug_get(dl_renderer* r, const char* name, void* dst, size_t cap, size_t* bytes);
/* Per-stage device time (ms) accumulated while profiling is on, in the order
 * project, depth_sort, emit, tile_offsets, pair_sort, rasterize. */
int dl_renderer_set_profiling(dl_renderer* r, int on);
int dl_renderer_stage_times(dl_renderer* r, double* ms, int n);
/* Kernel launches issued by the last render call. */
int dl_renderer_launch_count(dl_renderer* r, uint64_t* count);
/* Keep the last single-view frame's f32 accumulator (r, g, b, T) for "accum". */
int dl_renderer_set_debug(dl_renderer* r, int keep_intermediates);

/* ---- bounded device waits (no reference counterpart; the reference throws
 * on device set-up failure, src/gpu/device.ts:29-35, and has no device-side
 * waits).  Every decoupled look-back (depth sort, pair emission, pair sort,
 * the sorter, the voxelizer's binning, block heads and compaction) polls an
 * unpublished predecessor at most `polls` times, then sets a timeout bit that
 * the call returns as DL_E_TIMEOUT; the kernels after it skip their work, so
 * the device stays usable.  polls 0 restores the default (2^21, about 0.2 s).
 * Process-wide; for tests of the failure path. */
int dl_test_set_wait_limit(uint32_t polls);
/* Test hook: CTA `tile` (a global CTA index) of one stage publishes no status,
 * so that its successors run into the wait limit.  stage: 0 none (default),
 * 1 the depth sort's first pass, 2 pair emission, 3 the pair sort's first pass. */
int dl_test_withhold_status(int stage, uint32_t tile);
/* Test hook: the library's next `after` device allocations succeed and the
 * one after them fails as cudaMalloc does when the device is out of memory
 * (the call returns DL_E_OOM); then the hook switches itself off.  Negative:
 * off.  Process-wide. */
int dl_test_fail_allocation(int after);

#ifdef __cplusplus
}
#endif
#endif /* DROPLET_B200_H */

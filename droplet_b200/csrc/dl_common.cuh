// dl_common.cuh — shared device-side definitions for the droplet_b200 kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "dl_math.h"

// Renderer constants, src/render/shaders/constants.ts:19-26,37-38 (WGSL f32 literals).
#define DL_TILE 16u
#define DL_SIGMA_CUTOFF 3.0f
#define DL_AA_DILATION 0.3f
#define DL_OPACITY_CAP 0.999f
#define DL_MIN_T 0.0001f
#define DL_MIN_ALPHA 0.00392156862745098f
#define DL_GAUSS_FLOOR 1.1108996538e-2f
#define DL_FADE_START_FRAC 0.9481481481481482f
#define DL_FADE_END_FRAC 1.8962962962962964f

// Device error word bits (set by kernels, read by the host after a sync).
#define DL_DEVERR_TIMEOUT 1u    // a bounded look-back wait gave up
#define DL_DEVERR_OVERFLOW 2u   // a pair / list buffer was too small (host grows and re-runs)

// Bounded spin: polls with nanosleep back-off; ~0.2 s worst case per wait.
#define DL_SPIN_LIMIT (1u << 21)

__device__ __forceinline__ uint32_t dl_ld_volatile(const uint32_t* p) {
    return *(const volatile uint32_t*)p;
}
__device__ __forceinline__ void dl_st_volatile(uint32_t* p, uint32_t v) { *(volatile uint32_t*)p = v; }
__device__ __forceinline__ unsigned long long dl_ld_volatile64(const unsigned long long* p) {
    return *(const volatile unsigned long long*)p;
}
__device__ __forceinline__ void dl_st_volatile64(unsigned long long* p, unsigned long long v) {
    *(volatile unsigned long long*)p = v;
}

__device__ __forceinline__ uint32_t dl_lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Per-view camera parameters as the project shader's uniform block holds
// them (src/render/pipeline.ts:475-506): f32 copies of the f64 host values,
// plus the f64 values the CPU cull uses (src/render/camera.ts:56-99).
struct DlView {
    float view[16];              // column-major world->camera
    float width, height, focal, cx, cy, near_f, far_f;
    double near_d, far_d;
    uint32_t W, H;
    uint32_t tilesX, tilesY, numTiles;   // the binning tile grid (tileW x tileH-pixel tiles)
    int32_t projection;          // 0 pinhole, 1 equirect
    uint32_t maxCoverage;        // the reference's maxCoveragePerSplat, counted in 16x16 tiles
    float bg[4];
    uint32_t tileW, tileH;       // binning tile size: 16x16 (the reference's TILE_SIZE) unless tuned
    uint32_t refTilesX, refTilesY;   // the reference's 16x16 tile grid (coverage count, phantom rule)
    uint32_t binCap;             // binning tiles one splat may take: maxCoverage at 16x16, else no cap
};

// Device-resident scene (struct of arrays, as SplatData).
struct DlSceneDev {
    const float* pos;      // 3N
    const float* rot;      // 4N
    const float* lsc;      // 3N
    const float* opl;      // N
    const float* dc;       // 3N
    const float* sh;       // 3MN (f32) or NULL
    const uint16_t* sh16;  // f16 / bf16 bits, or NULL: per Gaussian a block of sh16_stride halves,
                           // coefficient-major (entry 3k + c = coefficient k of channel c), zero-padded
    uint32_t sh16_stride;  // round_up(3M, 8): 16-byte aligned blocks
    uint32_t n;
    int32_t bands;
    int32_t sh_kind;       // 0 f32, 1 f16, 2 bf16
};

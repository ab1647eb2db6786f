// ORACLE — test infrastructure only; parity unpinned (see oracle_render.cpp).  Plain C structs
// mirroring droplet's SplatData / RenderCamera (src/types.ts:23-32,74-82).
#pragma once
#include <stdint.h>
#include "dl_math.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_splats {
    uint64_t count;
    const float* positions;       // 3N
    const float* rotations;       // 4N, [w, x, y, z]
    const float* log_scales;      // 3N
    const float* opacity_logits;  // N
    const float* colors_dc;       // 3N
    const float* colors_sh;       // 3*M*N channel-major per Gaussian, or NULL
    int32_t sh_bands;             // 0..3
} orc_splats;

typedef struct orc_camera {
    uint32_t width, height;
    float view[16];               // column-major world->camera
    double fov_y, near_plane, far_plane;
    int32_t projection;           // 0 pinhole, 1 equirect
} orc_camera;

void* orc_render_run(const orc_splats* data, const orc_camera* cam, uint32_t maxCoverage,
                     uint32_t chunkCap, const float bg[4], int withF64);
int64_t orc_render_get(void* h, const char* name, void* dst, int64_t cap);
void orc_render_free(void* h);

void* orc_voxelize_run(const orc_splats* data, double voxelRes, double opacityCutoff,
                       const double* bounds6, int order, float eps, int64_t zrow_lo, int64_t zrow_hi);
int64_t orc_voxelize_get(void* h, const char* name, void* dst, int64_t cap);
void orc_voxelize_free(void* h);

#ifdef __cplusplus
}
#endif

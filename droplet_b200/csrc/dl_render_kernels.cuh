// dl_render_kernels.cuh — CUDA kernels of the tile-binned forward renderer.
//
// Stage map (reference -> here):
//   camera.ts:56-99 cull + radix-sort.ts key   -> project_k (f64 cull, depth key)
//   project.ts:59-234 project                    -> project_k (same f32 op order)
//   radix-sort.ts:65-117 CPU depth sort          -> dlsort passes (dl_sort.cuh)
//   prefix-sum.ts + pipeline.ts:277-304 scan     -> emit_k (decoupled look-back)
//   (pair-sort digit offsets)                    -> pair_digits_k
//   emit-pairs.ts:28-57 emit                    -> emit_k (load-balanced emission)
//   pipeline.ts:544-578 stable pair sort          -> dlsort passes on tile ids
//   find-boundaries.ts:17-99 tile offsets         -> lowered by the pair sort's last pass (dl_sort.cuh
//                                                    Bound), bound_init_k / bound_fill_k; boundaries_k
//                                                    (direct writes) when a view has one tile
//   rasterize.ts:36-82 + finalize.ts:30-43    -> rasterize_k (fused)
//
// All f32 arithmetic that feeds an integer decision or an output byte is
// written in the shaders' evaluation order and compiled with --fmad=false,
// so results are bit-identical to the CPU restatement of the reference.
#pragma once
#include "dl_common.cuh"
#include <cuda_fp16.h>
#include <cuda_bf16.h>

#include "dl_mlp.cuh"

namespace dlr {

// ------------------------------------------------------------------ project
struct ProjectArgs {
    DlSceneDev sc;
    const DlView* views;
    uint32_t num_views;
    uint64_t view_stride;     // elements between views' per-splat arrays (>= N)
    uint32_t* keys;           // [V][stride] sortable depth key, 0xffffffff if culled
    float4* recA;             // [V][stride] (screenX, screenY, radius, depth)
    float4* recBC;            // [V][stride][2] (A, B, C, alpha), (r, g, b, 0)   (f32 records)
    uint4* recH;              // [V][stride] half records: (A,B) (C,alpha) (r,g) (b,0)  (f16 records)
    uint2* bbox;              // [V][stride] (minX | minY<<16, maxX | maxY<<16), bit 15 of each max
                              // field = box entirely left of / above the image; empty if minX > maxX
    uint32_t* nvis;           // [V] visible count
    int f64_degenerate;       // recompute det / conic / AA factor in f64 for near-degenerate splats
    int cull_offscreen;       // also cull splats with no tile on the image (no pair can touch a pixel)
    uint32_t g_begin, g_end;  // this launch projects splats [g_begin, g_end)
    uint32_t* vis_mask;       // non-NULL: colours deferred to colour_k; [ceil(V/32)][N] record bits
};

// A 2D covariance is near-degenerate when its f32 determinant has lost at
// least 10 of its 24 bits to cancellation: det < 2^-10 * c00 * c11.
constexpr float kDegenerateRel = 1.0f / 1024.0f;

struct Cov3 { float c00, c01, c02, c11, c12, c22; };

__device__ __forceinline__ void quat_rot(const float q[4], float vx, float vy, float vz, float o[3]) {
    // project.ts:50-53 — t = 2*cross(q.yzw, v); v + q.x*t + cross(q.yzw, t)
    const float qx = q[1], qy = q[2], qz = q[3];
    const float c0 = qy * vz - qz * vy, c1 = qz * vx - qx * vz, c2 = qx * vy - qy * vx;
    const float t0 = 2.0f * c0, t1 = 2.0f * c1, t2 = 2.0f * c2;
    const float d0 = qy * t2 - qz * t1, d1 = qz * t0 - qx * t2, d2 = qx * t1 - qy * t0;
    o[0] = (vx + q[0] * t0) + d0;
    o[1] = (vy + q[0] * t1) + d1;
    o[2] = (vz + q[0] * t2) + d2;
}

// project.ts:86-98 — view-independent, computed once per splat.
__device__ __forceinline__ Cov3 make_cov3(const float rot[4], const float s[3]) {
    float rx[3], ry[3], rz[3];
    quat_rot(rot, 1.0f, 0.0f, 0.0f, rx);
    quat_rot(rot, 0.0f, 1.0f, 0.0f, ry);
    quat_rot(rot, 0.0f, 0.0f, 1.0f, rz);
    for (int k = 0; k < 3; k++) { rx[k] = rx[k] * s[0]; ry[k] = ry[k] * s[1]; rz[k] = rz[k] * s[2]; }
    Cov3 c;
    c.c00 = (rx[0] * rx[0] + ry[0] * ry[0]) + rz[0] * rz[0];
    c.c01 = (rx[0] * rx[1] + ry[0] * ry[1]) + rz[0] * rz[1];
    c.c02 = (rx[0] * rx[2] + ry[0] * ry[2]) + rz[0] * rz[2];
    c.c11 = (rx[1] * rx[1] + ry[1] * ry[1]) + rz[1] * rz[1];
    c.c12 = (rx[1] * rx[2] + ry[1] * ry[2]) + rz[1] * rz[2];
    c.c22 = (rx[2] * rx[2] + ry[2] * ry[2]) + rz[2] * rz[2];
    return c;
}

__device__ __forceinline__ float sh_coef(const DlSceneDev& sc, uint64_t i) {
    return __ldg(sc.sh + i);
}

// Division and square root of the projection: correctly rounded, as the
// shader's f32 operations (bit-exact with the oracle), or in the +-1 LSB
// arithmetic of DL_BATCH_FAST_EXP frames (kFast) the hardware approximations
// (relative error about 2^-22: far inside the margins of every integer
// decision they feed, which are pixels or 0.2% of a box).
template <bool kFast>
__device__ __forceinline__ float pdiv(float a, float b) { return kFast ? __fdividef(a, b) : a / b; }
template <bool kFast>
__device__ __forceinline__ float psqrt(float x) {
    if (!kFast) return sqrtf(x);
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// acc + b * c: the shader's separate multiply and add, or (kFma, the +-1 LSB
// arithmetic of DL_BATCH_FAST_EXP frames) one fused multiply-add
template <bool kFma>
__device__ __forceinline__ float sh_acc(float acc, float b, float c) {
    return kFma ? __fmaf_rn(b, c, acc) : acc + b * c;
}

// project.ts:264-331 evalSH (channel-major coefficients, camera-space direction)
template <bool kFma>
__device__ __forceinline__ void eval_sh(const DlSceneDev& sc, uint64_t base, int M, float x, float y, float z,
                                        float& r, float& g, float& b) {
    const float SH1 = 0.4886025119029199f, nSH1 = -0.4886025119029199f;
    const float b1[3] = {nSH1 * y, SH1 * z, nSH1 * x};
    r = 0.0f; g = 0.0f; b = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        r = sh_acc<kFma>(r, b1[k], sh_coef(sc, base + k));
        g = sh_acc<kFma>(g, b1[k], sh_coef(sc, base + M + k));
        b = sh_acc<kFma>(b, b1[k], sh_coef(sc, base + 2 * M + k));
    }
    if (sc.bands >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        const float xy = x * y, yz = y * z, xz = x * z;
        const float b2[5] = {1.0925484305920792f * xy, -1.0925484305920792f * yz,
                             0.31539156525252005f * (((2.0f * zz) - xx) - yy), -1.0925484305920792f * xz,
                             0.5462742152960396f * (xx - yy)};
#pragma unroll
        for (int k = 0; k < 5; k++) {
            r = sh_acc<kFma>(r, b2[k], sh_coef(sc, base + 3 + k));
            g = sh_acc<kFma>(g, b2[k], sh_coef(sc, base + M + 3 + k));
            b = sh_acc<kFma>(b, b2[k], sh_coef(sc, base + 2 * M + 3 + k));
        }
        if (sc.bands >= 3) {
            const float b3[7] = {(-0.5900435899266435f * y) * ((3.0f * xx) - yy),
                                 (2.890611442640554f * xy) * z,
                                 (-0.4570457994644658f * y) * (((4.0f * zz) - xx) - yy),
                                 (0.3731763325901154f * z) * (((2.0f * zz) - (3.0f * xx)) - (3.0f * yy)),
                                 (-0.4570457994644658f * x) * (((4.0f * zz) - xx) - yy),
                                 (1.445305721320277f * z) * (xx - yy),
                                 (-0.5900435899266435f * x) * (xx - (3.0f * yy))};
#pragma unroll
            for (int k = 0; k < 7; k++) {
                r = sh_acc<kFma>(r, b3[k], sh_coef(sc, base + 8 + k));
                g = sh_acc<kFma>(g, b3[k], sh_coef(sc, base + M + 8 + k));
                b = sh_acc<kFma>(b, b3[k], sh_coef(sc, base + 2 * M + 8 + k));
            }
        }
    }
}

// evalSH on the 16-bit SH block of one Gaussian (same basis, same summation
// order as eval_sh): the block is read with 128-bit loads.  kHalf: FP16
// coefficients, else BF16 (a compile-time choice, so that each coefficient
// costs one conversion and no select).
template <int BANDS, bool kFma, bool kHalf>
__device__ __forceinline__ void eval_sh16(const DlSceneDev& sc, uint32_t g, float x, float y, float z,
                                          float& r, float& gr, float& b) {
    constexpr int M = BANDS == 1 ? 3 : BANDS == 2 ? 8 : 15;
    constexpr int CH = (3 * M + 7) / 8;
    const uint4* blk = reinterpret_cast<const uint4*>(sc.sh16 + (uint64_t)g * sc.sh16_stride);
    uint32_t w[CH * 4];
#pragma unroll
    for (int c = 0; c < CH; c++) {
        const uint4 q = __ldg(blk + c);
        w[4 * c] = q.x; w[4 * c + 1] = q.y; w[4 * c + 2] = q.z; w[4 * c + 3] = q.w;
    }
    auto coef = [&](int k, int ch) -> float {
        const int e = 3 * k + ch;
        const uint32_t word = w[e >> 1];
        if (kHalf) return __half2float(__ushort_as_half((uint16_t)(word >> ((e & 1) * 16))));
        return __uint_as_float((e & 1) ? (word & 0xffff0000u) : (word << 16));   // BF16: the high half of an f32
    };
    const float SH1 = 0.4886025119029199f, nSH1 = -0.4886025119029199f;
    const float b1[3] = {nSH1 * y, SH1 * z, nSH1 * x};
    r = 0.0f; gr = 0.0f; b = 0.0f;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        r = sh_acc<kFma>(r, b1[k], coef(k, 0));
        gr = sh_acc<kFma>(gr, b1[k], coef(k, 1));
        b = sh_acc<kFma>(b, b1[k], coef(k, 2));
    }
    if (BANDS >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        const float xy = x * y, yz = y * z, xz = x * z;
        const float b2[5] = {1.0925484305920792f * xy, -1.0925484305920792f * yz,
                             0.31539156525252005f * (((2.0f * zz) - xx) - yy), -1.0925484305920792f * xz,
                             0.5462742152960396f * (xx - yy)};
#pragma unroll
        for (int k = 0; k < 5; k++) {
            r = sh_acc<kFma>(r, b2[k], coef(3 + k, 0));
            gr = sh_acc<kFma>(gr, b2[k], coef(3 + k, 1));
            b = sh_acc<kFma>(b, b2[k], coef(3 + k, 2));
        }
        if (BANDS >= 3) {
            const float b3[7] = {(-0.5900435899266435f * y) * ((3.0f * xx) - yy),
                                 (2.890611442640554f * xy) * z,
                                 (-0.4570457994644658f * y) * (((4.0f * zz) - xx) - yy),
                                 (0.3731763325901154f * z) * (((2.0f * zz) - (3.0f * xx)) - (3.0f * yy)),
                                 (-0.4570457994644658f * x) * (((4.0f * zz) - xx) - yy),
                                 (1.445305721320277f * z) * (xx - yy),
                                 (-0.5900435899266435f * x) * (xx - (3.0f * yy))};
#pragma unroll
            for (int k = 0; k < 7; k++) {
                r = sh_acc<kFma>(r, b3[k], coef(8 + k, 0));
                gr = sh_acc<kFma>(gr, b3[k], coef(8 + k, 1));
                b = sh_acc<kFma>(b, b3[k], coef(8 + k, 2));
            }
        }
    }
}

__device__ __forceinline__ uint32_t pack_h2(float a, float b) {
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Camera-space position (project.ts:79-84): the shader's order, or in the
// +-1 LSB arithmetic of DL_BATCH_FAST_EXP frames (kFma) fused multiply-adds.
// project_k and colour_k both call this, so deferred colours are bit-identical.
template <bool kFma>
__device__ __forceinline__ void cam_pos(const float* V, const float pos[3], float& pcx, float& pcy, float& pcz) {
    if (kFma) {
        pcx = __fmaf_rn(V[8], pos[2], __fmaf_rn(V[4], pos[1], V[0] * pos[0])) + V[12];
        pcy = __fmaf_rn(V[9], pos[2], __fmaf_rn(V[5], pos[1], V[1] * pos[0])) + V[13];
        pcz = __fmaf_rn(V[10], pos[2], __fmaf_rn(V[6], pos[1], V[2] * pos[0])) + V[14];
    } else {
        pcx = ((V[0] * pos[0] + V[4] * pos[1]) + V[8] * pos[2]) + V[12];
        pcy = ((V[1] * pos[0] + V[5] * pos[1]) + V[9] * pos[2]) + V[13];
        pcz = ((V[2] * pos[0] + V[6] * pos[1]) + V[10] * pos[2]) + V[14];
    }
}

// Splat colour for one view (project.ts:236-251): DC plus the SH bands
// evaluated along the normalised view-space position, + 0.5, clamped at 0.
// project_k and colour_k both call this, so deferred colours are bit-identical.
template <bool kFma>
__device__ __forceinline__ void splat_colour(const DlSceneDev& sc, uint32_t g, int M, const float dc[3], float pcx,
                                             float pcy, float pcz, float& c0, float& c1, float& c2) {
    float col0 = dc[0], col1 = dc[1], col2 = dc[2];
    if (sc.bands > 0) {
        const float len = psqrt<kFma>(kFma ? __fmaf_rn(pcz, pcz, __fmaf_rn(pcy, pcy, pcx * pcx))
                                           : (pcx * pcx + pcy * pcy) + pcz * pcz);
        float sr, sg, sb;
        const float dxn = pdiv<kFma>(pcx, len), dyn = pdiv<kFma>(pcy, len), dzn = pdiv<kFma>(pcz, len);
        if (sc.sh16 && sc.sh_kind == 1) {
            if (sc.bands == 1) eval_sh16<1, kFma, true>(sc, g, dxn, dyn, dzn, sr, sg, sb);
            else if (sc.bands == 2) eval_sh16<2, kFma, true>(sc, g, dxn, dyn, dzn, sr, sg, sb);
            else eval_sh16<3, kFma, true>(sc, g, dxn, dyn, dzn, sr, sg, sb);
        } else if (sc.sh16) {
            if (sc.bands == 1) eval_sh16<1, kFma, false>(sc, g, dxn, dyn, dzn, sr, sg, sb);
            else if (sc.bands == 2) eval_sh16<2, kFma, false>(sc, g, dxn, dyn, dzn, sr, sg, sb);
            else eval_sh16<3, kFma, false>(sc, g, dxn, dyn, dzn, sr, sg, sb);
        } else {
            eval_sh<kFma>(sc, (uint64_t)g * 3 * M, M, dxn, dyn, dzn, sr, sg, sb);
        }
        col0 = col0 + sr; col1 = col1 + sg; col2 = col2 + sb;
    }
    c0 = fmaxf(col0 + 0.5f, 0.0f);
    c1 = fmaxf(col1 + 0.5f, 0.0f);
    c2 = fmaxf(col2 + 0.5f, 0.0f);
}

// One splat, all views.  Thread per splat, index order (coalesced SoA reads).
constexpr int kProjectMaxViews = 4096;          // views per frame (per-CTA visible counters)

constexpr uint32_t kProjectSmemViews = 64;      // view tables staged in shared memory up to this count
static_assert(sizeof(DlView) % 4 == 0, "DlView is copied as 32-bit words");

// kFma: DL_BATCH_FAST_EXP frames evaluate the camera-space position, the 2D
// covariance and the SH colour with fused multiply-adds (64 registers, 4 CTAs
// per SM; the shader's order needs 80 registers, 3 CTAs per SM)
template <bool kFma>
__global__ void __launch_bounds__(256, kFma ? 4 : 3) project_k(ProjectArgs a) {
    __shared__ uint32_t s_vis[kProjectMaxViews];
    __shared__ DlView s_views[kProjectSmemViews];
    for (uint32_t v = threadIdx.x; v < a.num_views; v += blockDim.x) s_vis[v] = 0;
    const bool staged = a.num_views <= kProjectSmemViews;
    if (staged) {
        const uint32_t words = a.num_views * (uint32_t)(sizeof(DlView) / 4);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.views);
        uint32_t* dst = reinterpret_cast<uint32_t*>(s_views);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const DlView* vtab = staged ? s_views : a.views;
    const uint32_t g = a.g_begin + blockIdx.x * blockDim.x + threadIdx.x;
    const bool inRange = g < a.g_end;
    float pos[3] = {0, 0, 0}, rot[4] = {1, 0, 0, 0}, s[3] = {1, 1, 1}, dc[3] = {0, 0, 0}, opl = 0.0f;
    if (inRange) {
        pos[0] = __ldg(a.sc.pos + 3ull * g); pos[1] = __ldg(a.sc.pos + 3ull * g + 1); pos[2] = __ldg(a.sc.pos + 3ull * g + 2);
        const float4 q = __ldg(reinterpret_cast<const float4*>(a.sc.rot) + g);
        rot[0] = q.x; rot[1] = q.y; rot[2] = q.z; rot[3] = q.w;
        s[0] = dl_expf(__ldg(a.sc.lsc + 3ull * g));
        s[1] = dl_expf(__ldg(a.sc.lsc + 3ull * g + 1));
        s[2] = dl_expf(__ldg(a.sc.lsc + 3ull * g + 2));
        opl = __ldg(a.sc.opl + g);
        dc[0] = __ldg(a.sc.dc + 3ull * g); dc[1] = __ldg(a.sc.dc + 3ull * g + 1); dc[2] = __ldg(a.sc.dc + 3ull * g + 2);
    }
    const Cov3 cv = make_cov3(rot, s);
    const float sig = dl_sigmoidf(opl);
    const int M = a.sc.bands == 0 ? 0 : a.sc.bands == 1 ? 3 : a.sc.bands == 2 ? 8 : 15;
    uint32_t mword = 0;                           // deferred colour: views of this word with a record

    for (uint32_t v = 0; v < a.num_views; v++) {
        if (a.vis_mask && v && (v & 31u) == 0) {
            if (inRange) a.vis_mask[(uint64_t)((v >> 5) - 1) * a.sc.n + g] = mword;
            mword = 0;
        }
        const DlView& u = vtab[v];
        const float* V = u.view;
        const uint64_t o = (uint64_t)v * a.view_stride + g;
        // ---- camera.ts:56-99: f64 cull and depth key
        bool visible = false;
        float depthKey = 0.0f;
        if (inRange) {
            const double x = pos[0], y = pos[1], z = pos[2];
            if (u.projection == 0) {
                const double cz = (((double)V[2] * x + (double)V[6] * y) + (double)V[10] * z) + (double)V[14];
                const double depth = -cz;
                visible = depth > u.near_d && depth < u.far_d;
                depthKey = (float)depth;
            } else {
                const double cx = (((double)V[0] * x + (double)V[4] * y) + (double)V[8] * z) + (double)V[12];
                const double cy = (((double)V[1] * x + (double)V[5] * y) + (double)V[9] * z) + (double)V[13];
                const double cz = (((double)V[2] * x + (double)V[6] * y) + (double)V[10] * z) + (double)V[14];
                const double r2 = (cx * cx + cy * cy) + cz * cz;
                visible = r2 > u.near_d * u.near_d;
                depthKey = (float)sqrt(r2);
            }
            if (!a.cull_offscreen || !visible) a.keys[o] = visible ? dl_sortable_key(depthKey) : 0xffffffffu;
        }
        if (!a.cull_offscreen) {
            const uint32_t ballot = __ballot_sync(0xffffffffu, visible);
            if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(&s_vis[v], (uint32_t)__popc(ballot));
        }
        if (!visible) continue;

        // ---- project.ts:79-84
        float pcx, pcy, pcz;
        cam_pos<kFma>(V, pos, pcx, pcy, pcz);
        const float depth = -pcz;
        float screenX, screenY;
        bool culled = false;
        if (u.projection == 0) {
            culled = depth <= u.near_f || depth >= u.far_f;
            screenX = pdiv<kFma>(pcx * u.focal, -pcz) + u.cx;
            screenY = pdiv<kFma>(-pcy * u.focal, -pcz) + u.cy;
        } else {
            const float r = sqrtf((pcx * pcx + pcy * pcy) + pcz * pcz);
            culled = r <= u.near_f;
            const float lon = dl_atan2f(pcx, -pcz);
            const float lat = dl_asinf(pcy / r);
            screenX = (lon / 6.2831853f + 0.5f) * u.width;
            screenY = (0.5f - lat / 3.14159265f) * u.height;
        }
        float conicA = 0, conicB = 0, conicC = 0, radius = 0, radiusFade = 0, aaFactor = 0;
        if (!culled) {
            float c00o, c01, c11o;
            if (kFma) {
                // +-1 LSB frames: the same 2D covariance J W Σ Wᵀ Jᵀ (W: the view
                // rotation) associated as (J W) Σ (J W)ᵀ, in fused multiply-adds:
                // 45 operations where the shader's order takes 99
                const float invZ = pdiv<true>(1.0f, pcz);
                const float j00 = u.focal * invZ;
                const float j02 = ((-u.focal * pcx) * invZ) * invZ;
                const float j12 = ((-u.focal * pcy) * invZ) * invZ;
                const float t00 = __fmaf_rn(j02, V[2], j00 * V[0]), t01 = __fmaf_rn(j02, V[6], j00 * V[4]);
                const float t02 = __fmaf_rn(j02, V[10], j00 * V[8]);
                const float t10 = __fmaf_rn(j12, V[2], j00 * V[1]), t11 = __fmaf_rn(j12, V[6], j00 * V[5]);
                const float t12 = __fmaf_rn(j12, V[10], j00 * V[9]);
                const float s0 = __fmaf_rn(cv.c02, t02, __fmaf_rn(cv.c01, t01, cv.c00 * t00));
                const float s1 = __fmaf_rn(cv.c12, t02, __fmaf_rn(cv.c11, t01, cv.c01 * t00));
                const float s2 = __fmaf_rn(cv.c22, t02, __fmaf_rn(cv.c12, t01, cv.c02 * t00));
                const float q0 = __fmaf_rn(cv.c02, t12, __fmaf_rn(cv.c01, t11, cv.c00 * t10));
                const float q1 = __fmaf_rn(cv.c12, t12, __fmaf_rn(cv.c11, t11, cv.c01 * t10));
                const float q2 = __fmaf_rn(cv.c22, t12, __fmaf_rn(cv.c12, t11, cv.c02 * t10));
                c00o = __fmaf_rn(t02, s2, __fmaf_rn(t01, s1, t00 * s0));
                c01 = __fmaf_rn(t12, s2, __fmaf_rn(t11, s1, t10 * s0));
                c11o = __fmaf_rn(t12, q2, __fmaf_rn(t11, q1, t10 * q0));
            } else {
                // Σ_cam = V Σ Vᵀ (project.ts:103-123)
                const float v00 = V[0], v01 = V[4], v02 = V[8], v10 = V[1], v11 = V[5], v12 = V[9];
                const float v20 = V[2], v21 = V[6], v22 = V[10];
                const float a00 = (v00 * cv.c00 + v01 * cv.c01) + v02 * cv.c02;
                const float a01 = (v00 * cv.c01 + v01 * cv.c11) + v02 * cv.c12;
                const float a02 = (v00 * cv.c02 + v01 * cv.c12) + v02 * cv.c22;
                const float a10 = (v10 * cv.c00 + v11 * cv.c01) + v12 * cv.c02;
                const float a11 = (v10 * cv.c01 + v11 * cv.c11) + v12 * cv.c12;
                const float a12 = (v10 * cv.c02 + v11 * cv.c12) + v12 * cv.c22;
                const float a20 = (v20 * cv.c00 + v21 * cv.c01) + v22 * cv.c02;
                const float a21 = (v20 * cv.c01 + v21 * cv.c11) + v22 * cv.c12;
                const float a22 = (v20 * cv.c02 + v21 * cv.c12) + v22 * cv.c22;
                const float cc00 = (a00 * v00 + a01 * v01) + a02 * v02;
                const float cc01 = (a00 * v10 + a01 * v11) + a02 * v12;
                const float cc02 = (a00 * v20 + a01 * v21) + a02 * v22;
                const float cc11 = (a10 * v10 + a11 * v11) + a12 * v12;
                const float cc12 = (a10 * v20 + a11 * v21) + a12 * v22;
                const float cc22 = (a20 * v20 + a21 * v21) + a22 * v22;
                // EWA Jacobian as written (project.ts:128-149)
                const float invZ = pdiv<kFma>(1.0f, pcz);
                const float j00 = u.focal * invZ;
                const float j02 = ((-u.focal * pcx) * invZ) * invZ;
                const float j11 = u.focal * invZ;
                const float j12 = ((-u.focal * pcy) * invZ) * invZ;
                const float b00 = j00 * cc00 + j02 * cc02;
                const float b01 = j00 * cc01 + j02 * cc12;
                const float b02 = j00 * cc02 + j02 * cc22;
                const float b11 = j11 * cc11 + j12 * cc12;
                const float b12 = j11 * cc12 + j12 * cc22;
                c00o = b00 * j00 + b02 * j02;
                c01 = b01 * j11 + b02 * j12;
                c11o = b11 * j11 + b12 * j12;
            }
            const float c01s = c01 * c01;
            const float detOrig = kFma ? __fmaf_rn(c00o, c11o, -c01s) : c00o * c11o - c01s;
            const float c00 = c00o + DL_AA_DILATION;
            const float c11 = c11o + DL_AA_DILATION;
            const float det = kFma ? __fmaf_rn(c00, c11, -c01s) : c00 * c11 - c01s;
            aaFactor = psqrt<kFma>(fmaxf(pdiv<kFma>(detOrig, det), 0.0f));
            if (det <= 1.0e-6f) {
                culled = true;
            } else if (a.f64_degenerate && det < kDegenerateRel * (c00 * c11)) {
                // precision variant: determinants and inverse in f64 from the f32
                // covariance (products of two f32 are exact in f64); the cull,
                // radius and tile decisions below keep the f32 determinant
                const double d64 = (double)c00 * (double)c11 - (double)c01 * (double)c01;
                const double o64 = (double)c00o * (double)c11o - (double)c01 * (double)c01;
                conicA = (float)((double)c11 / d64);
                conicB = (float)(-(double)c01 / d64);
                conicC = (float)((double)c00 / d64);
                aaFactor = (float)sqrt(fmax(o64 / d64, 0.0));
            } else {
                const float invDet = pdiv<kFma>(1.0f, det);
                conicA = c11 * invDet;
                conicB = -c01 * invDet;
                conicC = c00 * invDet;
            }
            if (!culled) {
                const float mid = 0.5f * (c00 + c11);
                const float radiusEig = psqrt<kFma>(fmaxf(0.1f, kFma ? __fmaf_rn(mid, mid, -det) : mid * mid - det));
                const float lambda1 = mid + radiusEig;
                const float radiusRaw = DL_SIGMA_CUTOFF * psqrt<kFma>(lambda1);
                const float fadeStart = DL_FADE_START_FRAC * u.height;
                const float fadeEnd = DL_FADE_END_FRAC * u.height;
                radiusFade = fminf(fmaxf(pdiv<kFma>(fadeEnd - radiusRaw, fadeEnd - fadeStart), 0.0f), 1.0f);
                if (radiusFade <= 0.0f) culled = true;
                else radius = ceilf(fminf(radiusRaw, fadeEnd));
            }
        }
        if (culled) {
            if (a.cull_offscreen) {
                a.keys[o] = 0xffffffffu;
            } else {
                a.recA[o] = make_float4(0.0f, 0.0f, -1.0f, 0.0f);
                a.bbox[o] = make_uint2(0xffffu, 0u);
            }
            continue;
        }
        // project.ts:224-233 tile AABB (u32() saturates: off-screen left/top splats land in row/col 0)
        uint32_t minTX = dl_sat_u32(fmaxf(0.0f, floorf((screenX - radius) / 16.0f)));
        uint32_t minTY = dl_sat_u32(fmaxf(0.0f, floorf((screenY - radius) / 16.0f)));
        float fx1 = floorf((screenX + radius) / 16.0f), fy1 = floorf((screenY + radius) / 16.0f);
        uint32_t maxTX = dl_sat_u32(fminf((float)u.refTilesX - 1.0f, fx1));
        uint32_t maxTY = dl_sat_u32(fminf((float)u.refTilesY - 1.0f, fy1));
        const float alpha = (sig * radiusFade) * aaFactor;
        float boxX = radius, boxY = radius;          // half-extents the rasterizer tests (cull mode)
        // the rasterizer's alpha is opacity * (exp(-q/2) - exp(-4.5)) with the
        // opacity as stored; below 1/255 it is skipped
        const float alSt = a.recBC ? alpha : __half2float(__float2half_rn(alpha));
        if (a.cull_offscreen && alSt * (1.0f - DL_GAUSS_FLOOR) < 0.999f * DL_MIN_ALPHA) {
            // alpha < 1/255 at every pixel (exp(-q/2) <= 1): no pixel composites it
            a.keys[o] = 0xffffffffu;
            continue;
        }
        if (a.cull_offscreen && maxTX >= minTX && maxTY >= minTY &&
            (maxTX - minTX + 1u) * (maxTY - minTY + 1u) <= u.maxCoverage) {
            // Bin by the box of the ellipse q <= level (q: the rasterizer's
            // quadratic form, from the conic as it is stored) when the reference's
            // square box is not truncated.  Outside it alpha < 1/255 is skipped:
            // q > 9 gives exp(-q/2) < exp(-4.5); and alpha >= 1/255 needs
            // q <= qa = -2 ln(exp(-4.5) + 1/(255 opacity)).  The level takes qa
            // with 0.2% + 0.01 to spare, which keeps alpha at least 0.5% below
            // 1/255 outside the box, far above the f32 error of q and exp.
            float cA = conicA, cB = conicB, cC = conicC;
            if (!a.recBC) {
                cA = __half2float(__float2half_rn(cA));
                cB = __half2float(__float2half_rn(cB));
                cC = __half2float(__float2half_rn(cC));
            }
            const float ac = cA * cC, dt = kFma ? __fmaf_rn(-cB, cB, ac) : ac - cB * cB;
            if (dt > 0.0f && ac <= 1024.0f * dt) {
                const float lx = DL_GAUSS_FLOOR + pdiv<kFma>(DL_MIN_ALPHA, alSt);
                const float qa = -2.0f * (kFma ? __logf(lx) : logf(lx));
                const float level = fmaxf(0.0f, fminf(9.5f, 1.002f * qa + 0.01f));
                const float s = pdiv<kFma>(level, dt);
                const float ex = fminf(radius, psqrt<kFma>(cC * s)), ey = fminf(radius, psqrt<kFma>(cA * s));
                boxX = ex;
                boxY = ey;
                minTX = dl_sat_u32(fmaxf(0.0f, floorf((screenX - ex) / 16.0f)));
                minTY = dl_sat_u32(fmaxf(0.0f, floorf((screenY - ey) / 16.0f)));
                fx1 = floorf((screenX + ex) / 16.0f);
                fy1 = floorf((screenY + ey) / 16.0f);
                maxTX = dl_sat_u32(fminf((float)u.refTilesX - 1.0f, fx1));
                maxTY = dl_sat_u32(fminf((float)u.refTilesY - 1.0f, fy1));
            }
        }
        // A box right edge left of x = 0 (or bottom edge above y = 0) still counts
        // column (row) 0 after the saturation, but no pixel centre can pass its
        // box test there: flag it so the rasterizer skips these pairs unread.
        uint32_t phantom = ((fx1 < 0.0f) ? 0x8000u : 0u) | ((fy1 < 0.0f) ? 0x80000000u : 0u);
        bool hasTiles = maxTX >= minTX && maxTY >= minTY;
        if (a.cull_offscreen) {
            // a splat with no tile, or only phantom tiles, touches no pixel:
            // leaving it out of the depth order changes no tile list's order
            if (!hasTiles || phantom) { a.keys[o] = 0xffffffffu; continue; }
            a.keys[o] = dl_sortable_key(depthKey);
            const uint32_t m = __activemask();
            if ((threadIdx.x & 31) == (uint32_t)(__ffs(m) - 1)) atomicAdd(&s_vis[v], (uint32_t)__popc(m));
        }
        if (u.tileW != DL_TILE || u.tileH != DL_TILE) {
            // A tuned binning tile: the splat goes to the tiles of that grid that
            // its box (the one the rasterizer tests, or the radius square) meets
            // on the image.  The host uses another tile only when the reference's
            // maxCoverage cannot truncate any splat of the view, so every pixel
            // is offered the same splats as with 16x16 tiles; splats that meet
            // no tile of the image get none (they touch no pixel).
            const float bx = a.cull_offscreen ? boxX : radius, by = a.cull_offscreen ? boxY : radius;
            const float tw = (float)u.tileW, th = (float)u.tileH;
            const float x0 = floorf((screenX - bx) / tw), x1 = floorf((screenX + bx) / tw);
            const float y0 = floorf((screenY - by) / th), y1 = floorf((screenY + by) / th);
            hasTiles = x1 >= 0.0f && y1 >= 0.0f && x0 <= (float)u.tilesX - 1.0f && y0 <= (float)u.tilesY - 1.0f &&
                       x1 >= x0 && y1 >= y0;
            if (hasTiles) {
                minTX = (uint32_t)fmaxf(x0, 0.0f);
                minTY = (uint32_t)fmaxf(y0, 0.0f);
                maxTX = (uint32_t)fminf(x1, (float)u.tilesX - 1.0f);
                maxTY = (uint32_t)fminf(y1, (float)u.tilesY - 1.0f);
            }
            phantom = 0u;
        }
        // deferred: colour_k fills the colour once the SH has arrived
        float col0 = 0.0f, col1 = 0.0f, col2 = 0.0f;
        if (a.vis_mask) mword |= 1u << (v & 31u);
        else splat_colour<kFma>(a.sc, g, M, dc, pcx, pcy, pcz, col0, col1, col2);
        // cull mode: the screen record carries the half-extents of the box the
        // rasterizer tests (the ellipse's box, or the radius square) instead of
        // (radius, depth), which it does not read there
        a.recA[o] = a.cull_offscreen ? make_float4(screenX, screenY, boxX, boxY)
                                     : make_float4(screenX, screenY, radius, depth);
        if (a.recBC) {
            a.recBC[2 * o] = make_float4(conicA, conicB, conicC, alpha);
            a.recBC[2 * o + 1] = make_float4(col0, col1, col2, 0.0f);
        } else {
            a.recH[o] = make_uint4(pack_h2(conicA, conicB), pack_h2(conicC, alpha), pack_h2(col0, col1),
                                   pack_h2(col2, 0.0f));
        }
        if (hasTiles)
            a.bbox[o] = make_uint2(minTX | (minTY << 16), (maxTX | (maxTY << 16)) | phantom);
        else
            a.bbox[o] = make_uint2(0xffffu, 0u);
    }
    if (a.vis_mask && inRange && a.num_views)
        a.vis_mask[(uint64_t)((a.num_views - 1) >> 5) * a.sc.n + g] = mword;
    __syncthreads();
    for (uint32_t v = threadIdx.x; v < a.num_views; v += blockDim.x)
        if (s_vis[v]) atomicAdd(&a.nvis[v], s_vis[v]);
}

// Deferred colour: thread per splat, SH read once for all views; writes the
// colour of every (splat, view) whose record project_k wrote (vis_mask
// [ceil(V/32)][N], bit v % 32 of word v / 32), with the arithmetic of
// project_k (splat_colour).  Lets projection, sorting and binning run while
// the SH coefficients are still being uploaded.
struct ColourArgs {
    DlSceneDev sc;
    const DlView* views;
    uint32_t num_views;
    uint64_t view_stride;
    const uint32_t* vis_mask;
    float4* recBC;
    uint4* recH;
    uint32_t g_begin, g_end;       // the splat range coloured by this launch
};

template <bool kFma>
__global__ void __launch_bounds__(256) colour_k(ColourArgs a) {
    __shared__ DlView s_views[kProjectSmemViews];
    const bool staged = a.num_views <= kProjectSmemViews;
    if (staged) {
        const uint32_t words = a.num_views * (uint32_t)(sizeof(DlView) / 4);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.views);
        uint32_t* dst = reinterpret_cast<uint32_t*>(s_views);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const DlView* vtab = staged ? s_views : a.views;
    const uint32_t g = a.g_begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= a.g_end) return;
    const int M = a.sc.bands == 0 ? 0 : a.sc.bands == 1 ? 3 : a.sc.bands == 2 ? 8 : 15;
    float pos[3], dc[3];
    pos[0] = __ldg(a.sc.pos + 3ull * g); pos[1] = __ldg(a.sc.pos + 3ull * g + 1); pos[2] = __ldg(a.sc.pos + 3ull * g + 2);
    dc[0] = __ldg(a.sc.dc + 3ull * g); dc[1] = __ldg(a.sc.dc + 3ull * g + 1); dc[2] = __ldg(a.sc.dc + 3ull * g + 2);
    // views in the same order in every lane, so that the lanes of a warp
    // write one view's records together (consecutive splats, coalesced)
    uint32_t m = 0;
    for (uint32_t v = 0; v < a.num_views; v++) {
        if ((v & 31u) == 0) m = __ldg(a.vis_mask + (uint64_t)(v >> 5) * a.sc.n + g);
        if (!((m >> (v & 31u)) & 1u)) continue;
        {
            float pcx, pcy, pcz;
            cam_pos<kFma>(vtab[v].view, pos, pcx, pcy, pcz);
            float c0, c1, c2;
            splat_colour<kFma>(a.sc, g, M, dc, pcx, pcy, pcz, c0, c1, c2);
            const uint64_t o = (uint64_t)v * a.view_stride + g;
            if (a.recBC) a.recBC[2 * o + 1] = make_float4(c0, c1, c2, 0.0f);
            else reinterpret_cast<uint2*>(a.recH + o)[1] = make_uint2(pack_h2(c0, c1), pack_h2(c2, 0.0f));
        }
    }
}

// ------------------------------------------------------------------ emit
// Fused: gather tile counts in depth-rank order, exclusive scan with a
// decoupled look-back across CTAs (replaces the two scan kernels and the host
// block-sum scan), then write every pair of the CTA's contiguous output range
// with consecutive threads on consecutive slots (load-balanced, coalesced).
constexpr int kEmitThreads = 256;
constexpr int kEmitItems = 4;
constexpr int kEmitRanks = kEmitThreads * kEmitItems;   // 1024 ranks per CTA
constexpr unsigned long long kEmitAgg = 1ull << 62;
constexpr unsigned long long kEmitPrefix = 2ull << 62;
constexpr unsigned long long kEmitMask = (1ull << 62) - 1;

struct EmitArgs {
    const uint32_t* sorted_vals;   // [V][stride] rank -> splat
    const uint2* bbox;             // [V][stride]
    const uint32_t* nvis;          // [V]
    const DlView* views;
    uint64_t view_stride;
    uint32_t tiles_per_view;       // ceil(stride / kEmitRanks)
    const uint64_t* pair_base;     // [V]
    const uint64_t* pair_cap;      // [V]
    uint32_t* pair_keys;
    uint32_t* pair_vals;
    unsigned long long* npairs;    // [V] out
    uint32_t* digit_hist;          // [V][4][256] (zeroed): tile-id digit counts for the pair sort
    int bits, passes;              // digit width and count of the pair sort
    unsigned long long* status;    // [V][tiles_per_view] (zeroed)
    uint32_t* counter;
    uint32_t* err;                 // DL_DEVERR_TIMEOUT
    uint32_t* ovf;                 // DL_DEVERR_OVERFLOW
    uint32_t spin_limit;           // look-back polls before giving up
    uint32_t withhold_tile;        // test hook: this CTA tile publishes no status (0xffffffff: none)
};

// Pair values carry this bit for splats whose box lies entirely left of or
// above the image (see project_k); the splat index is in the low 30 bits.
constexpr uint32_t kPhantomBit = 0x80000000u;

__device__ __forceinline__ uint32_t bbox_count(uint2 bb, uint32_t maxCov) {
    const uint32_t minX = bb.x & 0xffffu, minY = bb.x >> 16, maxX = bb.y & 0x7fffu, maxY = (bb.y >> 16) & 0x7fffu;
    if (maxX < minX || maxY < minY) return 0u;
    const uint32_t c = (maxX - minX + 1u) * (maxY - minY + 1u);
    return c > maxCov ? maxCov : c;
}

__global__ void __launch_bounds__(kEmitThreads, 8) emit_k(EmitArgs a) {
    __shared__ uint32_t s_excl[kEmitRanks + 1];
    __shared__ uint32_t s_g[kEmitRanks];
    __shared__ uint32_t s_min[kEmitRanks];
    __shared__ uint16_t s_span[kEmitRanks];
    __shared__ uint32_t s_wsum[kEmitThreads / 32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_prefix;
    __shared__ uint32_t s_skip;
    __shared__ uint32_t s_dh[4 * 256];
    __shared__ uint32_t s_own[kEmitThreads / 32][32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // after a timed-out depth sort the sorted indices may hold unwritten slots
    if (__syncthreads_or(tid == 0 && (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT))) return;
    if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
    for (int i = tid; i < 4 * 256; i += kEmitThreads) s_dh[i] = 0;
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t v = tile / a.tiles_per_view;
    const uint32_t lt = tile - v * a.tiles_per_view;
    const uint32_t n = a.nvis[v];
    const uint32_t r0 = lt * kEmitRanks;
    if (r0 >= n) {
        if (lt == 0 && tid == 0) a.npairs[v] = 0ull;
        return;
    }
    const DlView& u = a.views[v];
    const uint64_t vo = (uint64_t)v * a.view_stride;

    uint32_t cnt[kEmitItems], gs[kEmitItems], mins[kEmitItems], spans[kEmitItems];
    uint32_t local = 0;
#pragma unroll
    for (int j = 0; j < kEmitItems; j++) {
        const uint32_t r = r0 + tid * kEmitItems + j;
        cnt[j] = 0; gs[j] = 0; mins[j] = 0; spans[j] = 1;
        if (r < n) {
            const uint32_t g = a.sorted_vals[vo + r];
            const uint2 bb = a.bbox[vo + g];
            gs[j] = g | ((bb.y & 0x80008000u) ? kPhantomBit : 0u);
            cnt[j] = bbox_count(bb, u.binCap);
            mins[j] = bb.x;
            spans[j] = (bb.y & 0x7fffu) - (bb.x & 0xffffu) + 1u;
        }
        local += cnt[j];
    }
    // block exclusive scan of per-thread sums
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
#pragma unroll
    for (int w = 0; w < kEmitThreads / 32; w++) { if (w < warp) wpre += s_wsum[w]; total += s_wsum[w]; }
    uint32_t run = wpre + inc - local;
#pragma unroll
    for (int j = 0; j < kEmitItems; j++) {
        const int i = tid * kEmitItems + j;
        s_excl[i] = run;
        s_g[i] = gs[j];
        s_min[i] = mins[j];
        s_span[i] = (uint16_t)spans[j];
        run += cnt[j];
    }
    if (tid == 0) s_excl[kEmitRanks] = total;

    // decoupled look-back over this view's earlier CTAs, by warp 0: each step
    // reads the 32 nearest unread predecessors at once.  No fence: a status
    // word carries its own value, and no other data passes between CTAs.
    if (warp == 0) {
        unsigned long long* st = a.status + (uint64_t)v * a.tiles_per_view;
        unsigned long long excl = 0;
        const bool publish = tile != a.withhold_tile;
        if (lt == 0) {
            if (lane == 0 && publish) dl_st_volatile64(&st[0], kEmitPrefix | (unsigned long long)total);
        } else {
            if (lane == 0 && publish) dl_st_volatile64(&st[lt], kEmitAgg | (unsigned long long)total);
            int64_t q = (int64_t)lt - 1;                 // nearest predecessor not yet added
            uint32_t spins = 0;
            while (true) {
                // tile 0 always publishes an inclusive prefix, so a walk never passes it
                const unsigned long long w = (q - lane >= 0) ? dl_ld_volatile64(&st[q - lane]) : kEmitPrefix;
                const unsigned long long flag = w & ~kEmitMask;
                const uint32_t notReady = __ballot_sync(0xffffffffu, flag == 0ull);
                const uint32_t prefix = __ballot_sync(0xffffffffu, flag == kEmitPrefix);
                const int firstNR = notReady ? __ffs(notReady) - 1 : 32;
                const int firstP = prefix ? __ffs(prefix) - 1 : 32;
                // lanes before the first unpublished one (through the first prefix) are added
                const int take = firstP < firstNR ? firstP + 1 : firstNR;
                unsigned long long add = lane < take ? (w & kEmitMask) : 0ull;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xffffffffu, add, o);
                excl += add;
                if (firstP < firstNR) break;
                q -= take;
                if (take == 0) {
                    if (++spins > a.spin_limit) { if (lane == 0) atomicOr(a.err, DL_DEVERR_TIMEOUT); break; }
                    __nanosleep(32);
                }
            }
            if (lane == 0 && publish) dl_st_volatile64(&st[lt], kEmitPrefix | ((excl + total) & kEmitMask));
        }
        if (lane == 0) {
            s_prefix = excl;
            if (r0 + kEmitRanks >= n) a.npairs[v] = excl + total;    // last CTA of the view
            const bool over = excl + total > a.pair_cap[v];
            if (over) atomicOr(a.ovf, DL_DEVERR_OVERFLOW);
            s_skip = over ? 1u : 0u;
        }
    }
    __syncthreads();
    if (s_skip) return;
    const uint64_t outBase = a.pair_base[v] + s_prefix;
    const uint32_t dmask = (1u << a.bits) - 1u;
    // Each warp walks a contiguous share of the CTA's pairs, 32 at a time.  A
    // pair o belongs to the last rank slot whose exclusive offset is <= o: one
    // binary search finds the slot of the warp's first pair, then each window
    // of 32 pairs takes its slots from the 32 slots after the previous one —
    // each marks the window position where it starts (the last of equal
    // starts: slots without pairs are passed over) and a max-scan over the
    // lanes counts the slots starting at or before each pair (another 32 slots
    // when all of them do).
    constexpr uint32_t kEmitWarps = kEmitThreads / 32;
    const uint32_t per = ((total + kEmitWarps - 1u) / kEmitWarps + 31u) & ~31u;
    const uint32_t wb = min(total, (uint32_t)warp * per), we = min(total, wb + per);
    uint32_t* own = s_own[warp];
    uint32_t base = 0;
    if (wb < we) {
        uint32_t hi = kEmitRanks;
        while (hi - base > 1) {
            const uint32_t mid = (base + hi) >> 1;
            if (s_excl[mid] <= wb) base = mid; else hi = mid;
        }
    }
    for (uint32_t o0 = wb; o0 < we; o0 += 32u) {
        const uint32_t o = o0 + (uint32_t)lane;
        uint32_t lo = base, b = base;
        bool resolved = false;
        while (true) {
            own[lane] = 0u;
            __syncwarp();
            // slot b + 1 + lane starts at o0 + q (q >= 0: slot b ends at or after o0)
            const uint32_t idx = b + 1u + (uint32_t)lane;
            const uint32_t q = idx <= (uint32_t)kEmitRanks ? s_excl[idx] - o0 : 0xffffffffu;
            const uint32_t qn = __shfl_down_sync(0xffffffffu, q, 1);
            if (q < 32u && (lane == 31 || qn != q)) own[q] = (uint32_t)lane + 1u;
            __syncwarp();
            uint32_t m = own[lane];
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, m, d);
                if (lane >= d) m = max(m, t);
            }
            if (!resolved && m < 32u) { lo = b + m; resolved = true; }
            if (!__any_sync(0xffffffffu, o < we && !resolved)) break;
            b += 32u;
            __syncwarp();                                   // own[] is cleared next
        }
        base = __shfl_sync(0xffffffffu, lo, 31);
        if (o >= we) continue;
        const uint32_t w = o - s_excl[lo];
        const uint32_t span = s_span[lo];
        const uint32_t mn = s_min[lo];
        // w / span and w % span: the approximate float quotient is within 1/16
        // of w / span (which is below 2^16, a tile row), so one step corrects it
        uint32_t row = __float2uint_rz(__fdividef((float)w, (float)span));
        int col = (int)w - (int)(row * span);
        if (col < 0) { row--; col += (int)span; }
        else if (col >= (int)span) { row++; col -= (int)span; }
        const uint32_t ty = (mn >> 16) + row;
        const uint32_t tx = (mn & 0xffffu) + (uint32_t)col;
        const uint32_t tileId = ty * u.tilesX + tx;
        a.pair_keys[outBase + o] = tileId;
        a.pair_vals[outBase + o] = s_g[lo];
        for (int p = 0; p < a.passes; p++) atomicAdd(&s_dh[p * 256 + ((tileId >> (p * a.bits)) & dmask)], 1u);
    }
    __syncthreads();
    uint32_t* gh = a.digit_hist + (uint64_t)v * 4 * 256;
    for (int i = tid; i < a.passes * 256; i += kEmitThreads)
        if (s_dh[i]) atomicAdd(&gh[i], s_dh[i]);
}

// ------------------------------------------------------------------ pair digits
// Per view: exclusive scan of the emit kernel's tile-id digit histograms (the
// pair sort's global digit offsets) and the pair-sort segment length (0 when
// the view overflowed its pair buffer).  One CTA per view.
struct PairDigitArgs {
    const uint32_t* digit_hist;    // [V][4][256]
    uint32_t* glob_off;            // [V][passes][radix]
    const unsigned long long* npairs;
    const uint64_t* pair_cap;
    uint32_t* seg_len;
    int bits, passes;
    const uint32_t* err;           // DL_DEVERR_TIMEOUT: the pair lists are not complete
};

__global__ void pair_digits_k(PairDigitArgs a) {
    const uint32_t v = blockIdx.x;
    const int radix = 1 << a.bits;
    if (threadIdx.x < (unsigned)a.passes) {
        const int p = threadIdx.x;
        const uint32_t* h = a.digit_hist + ((uint64_t)v * 4 + p) * 256;
        uint32_t* o = a.glob_off + ((uint64_t)v * a.passes + p) * radix;
        uint32_t acc = 0;
        for (int d = 0; d < radix; d++) { o[d] = acc; acc += h[d]; }
    }
    if (threadIdx.x == 0) {
        // an overflowed view, or any view of a frame with a timed-out wait,
        // sorts and bins no pairs: nothing downstream reads unwritten slots
        const bool ok = a.npairs[v] <= a.pair_cap[v] && !(dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT);
        a.seg_len[v] = ok ? (uint32_t)a.npairs[v] : 0u;
    }
}

// ------------------------------------------------------------------ boundaries
// find-boundaries.ts:31-99 on the sorted tile ids, with direct writes: the
// thread at pair i writes tileOffsets[t] = i for every tile t in
// (key[i-1], key[i]]; the thread at i = n writes n for the tiles after the
// last key and the sentinel tileOffsets[T].  Each entry has exactly one writer.
struct BoundArgs {
    const DlView* views;
    const uint32_t* keys;          // sorted tile ids, view v at pair_base[v]
    const uint64_t* pair_base;
    const uint32_t* seg_len;       // [V] pairs per view (0 on overflow)
    uint32_t* tile_off;            // [V][tile_stride]
    uint32_t tile_stride;
    const uint32_t* err;           // DL_DEVERR_TIMEOUT: the sorted keys are not complete
};

__global__ void boundaries_k(BoundArgs a) {
    const uint32_t v = blockIdx.y;
    // after a timed-out pair sort every view gets empty tiles
    const uint32_t n = (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT) ? 0u : a.seg_len[v];
    const uint32_t T = a.views[v].numTiles;
    const uint32_t* k = a.keys + a.pair_base[v];
    uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i <= n; i += gridDim.x * blockDim.x) {
        const int64_t prev = i == 0 ? -1 : (int64_t)k[i - 1];
        const int64_t cur = i == n ? (int64_t)T : (int64_t)k[i];
        for (int64_t t = prev + 1; t <= cur; t++) to[t] = i;
    }
}

// The same offsets without the sorted tile ids: the pair sort's last pass
// lowers tileOffsets[t] (atomicMin) to the position of the first pair of tile
// t it writes; bound_init_k presets every entry of a view to its pair count
// before that pass, and bound_fill_k then gives each empty tile the start of
// the next non-empty one (a suffix minimum; positions grow with the tile id),
// which is find-boundaries.ts's result: the first pair index with tile >= t.
__global__ void bound_init_k(BoundArgs a) {
    const uint32_t v = blockIdx.y;
    const uint32_t n = a.seg_len[v];
    const uint32_t T = a.views[v].numTiles;
    uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t <= T; t += gridDim.x * blockDim.x) to[t] = n;
}

constexpr int kFillThreads = 1024;

__global__ void __launch_bounds__(kFillThreads) bound_fill_k(BoundArgs a) {
    __shared__ uint32_t s_w[kFillThreads / 32];
    __shared__ uint32_t s_carry;
    const uint32_t v = blockIdx.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t T = a.views[v].numTiles;
    uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    // after a timed-out pair sort every view gets empty tiles
    if (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT) {
        for (uint32_t t = tid; t <= T; t += kFillThreads) to[t] = 0u;
        return;
    }
    if (tid == 0) s_carry = 0xffffffffu;
    // chunks of kFillThreads entries from the end: suffix minimum inside the
    // chunk, then with the minimum of everything after it
    for (int64_t hi = (int64_t)T + 1; hi > 0; hi -= kFillThreads) {
        const int64_t lo = hi - kFillThreads;
        const int64_t t = lo + tid;
        uint32_t x = t >= 0 ? to[t] : 0xffffffffu;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_down_sync(0xffffffffu, x, o);
            if (lane + o < 32) x = min(x, y);
        }
        if (lane == 0) s_w[warp] = x;                 // minimum of the warp's entries
        __syncthreads();
        uint32_t later = s_carry;
        for (int w = warp + 1; w < kFillThreads / 32; w++) later = min(later, s_w[w]);
        x = min(x, later);
        if (t >= 0) to[t] = x;
        __syncthreads();                              // s_w and s_carry are rewritten next
        if (tid == 0) s_carry = x;                    // the chunk's minimum: its first entry
        __syncthreads();
    }
}

// ------------------------------------------------------------------ tile features
// The 12 inputs of the learned cost model for tile t of view u, from the tile
// offsets alone (available after bound_fill_k, before the rasterizer).
__device__ __forceinline__ void tile_features(const DlView& u, const uint32_t* to, uint32_t t, float* x) {
    const int tx = (int)(t % u.tilesX), ty = (int)(t / u.tilesX);
    auto cnt = [&](int cx, int cy) {
        cx = min(max(cx, 0), (int)u.tilesX - 1);
        cy = min(max(cy, 0), (int)u.tilesY - 1);
        const uint32_t k = (uint32_t)cy * u.tilesX + (uint32_t)cx;
        return (float)(to[k + 1] - to[k]);
    };
    x[0] = log1pf(cnt(tx, ty)) * 0.1f;
    x[1] = log1pf(cnt(tx - 1, ty)) * 0.1f;
    x[2] = log1pf(cnt(tx + 1, ty)) * 0.1f;
    x[3] = log1pf(cnt(tx, ty - 1)) * 0.1f;
    x[4] = log1pf(cnt(tx, ty + 1)) * 0.1f;
    x[5] = ((float)tx + 0.5f) / (float)u.tilesX;
    x[6] = ((float)ty + 0.5f) / (float)u.tilesY;
    x[7] = ty == 0 ? 1.0f : 0.0f;
    x[8] = tx == 0 ? 1.0f : 0.0f;
    x[9] = logf((float)u.W * (float)u.H) * (1.0f / 16.0f);
    x[10] = log1pf((float)to[u.numTiles] / (float)u.numTiles) * 0.1f;
    const float tw = (float)u.tileW, th = (float)u.tileH;
    const float wx = fminf(tw, (float)u.W - tw * tx), wy = fminf(th, (float)u.H - th * ty);
    x[11] = wx * wy / (tw * th);
}

// Per global tile features (cost logging).
__global__ void tile_features_k(const DlView* views, uint32_t V, const uint32_t* tile_base, const uint32_t* tile_off,
                                uint32_t tile_stride, uint32_t total, float* __restrict__ X) {
    const uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x;
    if (gt >= total) return;
    uint32_t lo = 0, hi = V;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (tile_base[mid] <= gt) lo = mid; else hi = mid;
    }
    tile_features(views[lo], tile_off + (uint64_t)lo * tile_stride, gt - tile_base[lo], X + (uint64_t)gt * 12);
}

// The learned order.  sched_pred_k: per tile (all views in parallel) the
// features, the MLP's prediction and an 8-bit bucket that decreases with the
// predicted cost, counted per view; sched_scan_k: per view, bucket offsets
// after the view's first tile; sched_scatter_k: tiles into the work list by
// bucket.  Views keep their launch order (their tiles share splat records in
// L2).  Only the view that ends a rasterizer launch (every `tail_every`-th
// view, and the last) is reordered: its tiles end the launch's queue, where
// the most expensive ones go first so that no long tile is left for the end;
// inside a bucket they go in whatever order the atomics give.  Every other
// view keeps its natural order (identity entries), which keeps neighbouring
// tiles, and the splat records they share, together in L2.  Any order yields
// the same pixels.
constexpr int kSchedThreads = 128;
constexpr uint32_t kSchedKeep = 0xffffffffu;     // bucket word of a tile in natural order
__device__ __forceinline__ bool sched_reordered(uint32_t v, uint32_t V, uint32_t tail_every) {
    return v + 1 == V || (v + 1) % tail_every == 0;
}
__global__ void __launch_bounds__(kSchedThreads) sched_pred_k(const DlView* views, uint32_t V, const uint32_t* tile_base,
                                                              const uint32_t* tile_off, uint32_t tile_stride,
                                                              uint32_t total, const __nv_bfloat16* w,
                                                              uint32_t* __restrict__ bucket, uint32_t* __restrict__ vhist,
                                                              uint32_t tail_every, uint32_t* __restrict__ work) {
    __shared__ float P[dlmlp::kParams];
    dlmlp::load_params(w, P);
    for (uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x; gt < total; gt += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = V;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (tile_base[mid] <= gt) lo = mid; else hi = mid;
        }
        if (!sched_reordered(lo, V, tail_every)) {
            bucket[gt] = kSchedKeep;
            work[gt] = gt;
            continue;
        }
        float x[12];
        tile_features(views[lo], tile_off + (uint64_t)lo * tile_stride, gt - tile_base[lo], x);
        const float y = dlmlp::forward(P, x, nullptr, nullptr);
        const float q = (y == y) ? fminf(fmaxf((y + 4.0f) * 32.0f, 0.0f), 255.0f) : 0.0f;  // standardised log cost
        const uint32_t b = 255u - (uint32_t)q;                                               // 0 = most expensive
        bucket[gt] = (lo << 8) | b;
        atomicAdd(&vhist[lo * 256 + b], 1u);
    }
}

__global__ void sched_scan_k(const uint32_t* tile_base, uint32_t* vhist) {
    const uint32_t v = blockIdx.x;
    if (threadIdx.x == 0) {
        uint32_t acc = tile_base[v];
        for (int b = 0; b < 256; b++) { const uint32_t c = vhist[v * 256 + b]; vhist[v * 256 + b] = acc; acc += c; }
    }
}

__global__ void sched_scatter_k(const uint32_t* __restrict__ bucket, uint32_t total, uint32_t* vhist,
                                uint32_t* __restrict__ work) {
    for (uint32_t gt = blockIdx.x * blockDim.x + threadIdx.x; gt < total; gt += gridDim.x * blockDim.x) {
        const uint32_t vb = bucket[gt];
        if (vb == kSchedKeep) continue;
        work[atomicAdd(&vhist[(vb >> 8) * 256 + (vb & 255u)], 1u)] = gt;
    }
}

// ------------------------------------------------------------------ rasterize
// Persistent, warp-granular rasterizer.  A work item is one 32-pixel
// sub-tile (8x4 by default; 16x2 or 4x8 as tuned) of one 16x16 tile of one view; each warp pulls
// items from a queue (natural order, or the cost order of a work list) and
// owns the item's 32 pixels, one per lane.  It walks its tile's slice 32 pairs
// at a time: every lane loads one pair's screen record, keeps it if the
// splat's box widened by one pixel reaches a pixel centre of the sub-tile (no
// pixel whose per-pixel box test could pass is dropped), and the kept splats,
// in slice order, are staged in warp-private shared memory and composited by
// all 32 lanes with rasterize.ts:62-79 verbatim.  Pairs whose value has
// kPhantomBit (a splat box wholly left of / above the image) are skipped
// without reading their record: no pixel's box test can pass for them.  No CTA barrier: a warp
// leaves as soon as its own pixels saturate.  finalize.ts:30-43 is fused as
// the epilogue.
struct RasterArgs {
    const DlView* views;
    uint32_t num_views;
    const uint32_t* tile_base;     // [V+1] first global tile of each view
    const uint32_t* tile_off;      // [V][tile_stride]
    uint32_t tile_stride;
    const uint32_t* pair_vals;     // sorted by tile, rank order within a tile
    const uint64_t* pair_base;     // [V]
    const float4* recA;            // [V][view_stride]
    const float4* recBC;           // f32 records, or
    const uint4* recH;             // f16 records
    uint64_t view_stride;
    uint32_t* const* outs;         // [V] packed RGBA8 per pixel
    float4* accum;                 // optional [W*H] (single view debug)
    const uint32_t* work;          // optional tile order (global tile ids); NULL: natural order
    uint32_t item_base;            // this launch takes items [item_base, num_items)
    uint32_t num_items;            // 8 x total tiles (4 with two pixels per lane), or a view range's end
    uint32_t* work_counter;
    unsigned long long* eval_count;   // optional: total evaluated (pixel, splat) pairs
    uint32_t* tile_evals;          // optional [total tiles] evaluated pairs per tile
    uint32_t* tile_cycles;         // optional [total tiles] SM cycles / 16 spent per tile
    int sub_lw;                    // log2 of a work item's width: 3 (8x4), 4 (16x2) or 2 (4x8) pixels
    int ipt_lg;                    // log2 of the work items per tile
    int rec_box;                   // 1: recA.zw are the half-extents to test (cull mode), else (radius, depth)
    float stage_pad;               // a splat is staged for a sub-tile when its box, widened by this many
                                   // pixels, reaches one of the sub-tile's pixel centres
};

constexpr int kRasterThreads = 256;
constexpr int kRasterWarps = kRasterThreads / 32;
// dl_expf(p) <= DL_GAUSS_FLOOR exactly when p <= -4.5f (dl_expf is monotone
// there), so alpha = opacity * max(0, exp(p) - floor) is 0 and the splat is
// skipped by the MIN_ALPHA test; skipping before the exp is result-identical.
#define DL_POWER_CUT (-4.5f)

template <bool kExactExp>
__device__ __forceinline__ float raster_exp(float p) {
    if (kExactExp) return dl_expf(p);
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(p * 1.4426950408889634f));
    return y;
}

// Half-extents of the box outside which every pixel of a splat has alpha = 0.
// The rasterizer's quadratic form q(d) = A dx^2 + 2B dx dy + C dy^2 (power =
// -q/2) exceeds 9 outside the axis-aligned box of the ellipse q <= 9, whose
// half-extents are sqrt(9 C / det), sqrt(9 A / det) with det = A C - B^2; and
// q > 8.4 already gives opacity * (exp(-q/2) - exp(-4.5)) < 1/255, the skip of
// rasterize.ts:74.  With A C <= 1024 det the f32 evaluation of q and of the
// box is accurate to well under that margin (9.01 adds 0.05% to the extents),
// so skipping pixels outside the box changes no result.  Worse-conditioned
// conics keep the square box of the radius.
__device__ __forceinline__ void tight_extent(float A, float B, float C, float r, float& ex, float& ey) {
    ex = r;
    ey = r;
    const float ac = A * C;
    const float det = ac - B * B;
    if (det > 0.0f && ac <= 1024.0f * det) {
        const float s = 9.01f / det;
        ex = fminf(r, sqrtf(C * s));
        ey = fminf(r, sqrtf(A * s));
    }
}

__device__ __forceinline__ uint32_t view_of_tile(const RasterArgs& a, uint32_t gt) {
    uint32_t lo = 0, hi = a.num_views;        // last view with tile_base <= gt
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.tile_base[mid] <= gt) lo = mid; else hi = mid;
    }
    return lo;
}

// Stage the next 64 pairs of a tile's slice [b, end) that can reach the
// rectangle [rx0, rx1] x [ry0, ry1] into the warp's shared arrays, in slice
// order; returns how many (warp-uniform).
template <bool kExactExp>
__device__ __forceinline__ uint32_t stage_chunk(const RasterArgs& a, const uint32_t* vals, uint32_t b, uint32_t end,
                                                uint64_t vo, float rx0, float rx1, float ry0, float ry1,
                                                uint32_t lmask, float4* s_a, float4* s_b, float4* s_c) {
    const int lane = threadIdx.x & 31;
    // two chunks of 32 pairs per step: independent load chains in flight
    const uint32_t e0 = b + lane, e1 = b + 32 + lane;
    const uint32_t g0 = e0 < end ? __ldg(vals + e0) : kPhantomBit;
    const uint32_t g1 = e1 < end ? __ldg(vals + e1) : kPhantomBit;
    bool hit0 = false, hit1 = false;
    float4 ra0 = make_float4(0, 0, 0, 0), ra1 = make_float4(0, 0, 0, 0);
    if (!(g0 & kPhantomBit)) {
        ra0 = __ldg(a.recA + vo + g0);
        const float rx = ra0.z, ry = a.rec_box ? ra0.w : ra0.z;
        hit0 = rx > 0.0f && !(ra0.x - rx > rx1) && !(ra0.x + rx < rx0) && !(ra0.y - ry > ry1) && !(ra0.y + ry < ry0);
    }
    if (!(g1 & kPhantomBit)) {
        ra1 = __ldg(a.recA + vo + g1);
        const float rx = ra1.z, ry = a.rec_box ? ra1.w : ra1.z;
        hit1 = rx > 0.0f && !(ra1.x - rx > rx1) && !(ra1.x + rx < rx0) && !(ra1.y - ry > ry1) && !(ra1.y + ry < ry0);
    }
    if (__ballot_sync(0xffffffffu, hit0 || hit1) == 0u) return 0u;
    // square-box hits load their record; the ellipse's box then decides
    // (with eval counting on, the square box alone: the reference's count)
    uint32_t n = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        bool hit = h ? hit1 : hit0;
        const uint32_t g = h ? g1 : g0;
        const float4 ra = h ? ra1 : ra0;
        float A = 0.0f, B = 0.0f, C = 0.0f, al = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
        float ex = ra.z, ey = a.rec_box ? ra.w : ra.z;
        if (hit) {
            if (a.recBC) {
                const float4 p = __ldg(a.recBC + 2 * (vo + g));
                const float4 q = __ldg(a.recBC + 2 * (vo + g) + 1);
                A = p.x; B = p.y; C = p.z; al = p.w; cr = q.x; cg = q.y; cb = q.z;
            } else {
                const uint4 hv = __ldg(a.recH + vo + g);
                const float2 ab = __half22float2(*reinterpret_cast<const __half2*>(&hv.x));
                const float2 ca = __half22float2(*reinterpret_cast<const __half2*>(&hv.y));
                const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&hv.z));
                const float2 bz = __half22float2(*reinterpret_cast<const __half2*>(&hv.w));
                A = ab.x; B = ab.y; C = ca.x; al = ca.y; cr = rg.x; cg = rg.y; cb = bz.x;
            }
            if (!a.eval_count && !a.rec_box) {
                tight_extent(A, B, C, ra.z, ex, ey);
                hit = !(ra.x - ex > rx1) && !(ra.x + ex < rx0) && !(ra.y - ey > ry1) && !(ra.y + ey < ry0);
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) {
            const uint32_t slot = n + __popc(m & lmask);
            // s_b: conic and opacity (read for every pixel inside the box),
            // s_c: colour (read only by pixels that composite the splat)
            s_a[slot] = make_float4(ra.x, ra.y, ex, ey);
            if (kExactExp) {
                s_b[slot] = make_float4(A, 2.0f * B, C, al);
            } else {
                // conic pre-scaled by -0.5*log2(e): the quadratic form is ex2's argument
                s_b[slot] = make_float4(-0.72134752044448170f * A, -1.4426950408889634f * B,
                                        -0.72134752044448170f * C, al);
            }
            s_c[slot] = make_float4(cr, cg, cb, 0.0f);
        }
        n += __popc(m);
    }
    return n;
}

// kCount: count the evaluated (pixel, splat) pairs (eval_count / tile_evals).
template <bool kExactExp, bool kCount>
__device__ __forceinline__ void raster_subtile(const RasterArgs& a, uint32_t v, uint32_t tile, uint32_t sub,
                                               uint32_t gt, float4* s_a, float4* s_b, float4* s_c) {
    const DlView& u = a.views[v];
    const int lane = threadIdx.x & 31;
    const uint32_t tx = tile % u.tilesX, ty = tile / u.tilesX;
    // a work item is sw x sh pixels (sw * sh = 32), 8 items per 16x16 tile
    const uint32_t lw = (uint32_t)a.sub_lw, sw = 1u << lw, sh = 32u >> lw, perRow = u.tileW >> lw;
    const uint32_t sx0 = tx * u.tileW + (sub % perRow) * sw, sy0 = ty * u.tileH + (sub / perRow) * sh;
    const uint32_t x = sx0 + (lane & (sw - 1)), y = sy0 + (lane >> lw);
    const bool inImage = x < u.W && y < u.H;
    if (__all_sync(0xffffffffu, !inImage)) return;       // sub-tile entirely outside the image
    const long long t0 = a.tile_cycles ? clock64() : 0;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const float rx0 = (float)sx0 + 0.5f - a.stage_pad, rx1 = (float)(sx0 + sw) - 0.5f + a.stage_pad;
    const float ry0 = (float)sy0 + 0.5f - a.stage_pad, ry1 = (float)(sy0 + sh) - 0.5f + a.stage_pad;
    const uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    const uint32_t start = to[tile], end = to[tile + 1];
    const uint32_t* vals = a.pair_vals + a.pair_base[v];
    const uint64_t vo = (uint64_t)v * a.view_stride;
    const uint32_t lmask = dl_lanemask_lt();

    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, T = 1.0f;
    bool done = !inImage;
    uint32_t evals = 0;
    for (uint32_t b = start; b < end; b += 64) {
        const uint32_t n = stage_chunk<kExactExp>(a, vals, b, end, vo, rx0, rx1, ry0, ry1, lmask, s_a, s_b, s_c);
        if (n == 0u) continue;
        __syncwarp();
        if (!done && kExactExp) {
            for (uint32_t j = 0; j < n; j++) {
                const float4 sa = s_a[j];
                const float dx = px - sa.x;
                const float dy = py - sa.y;
                if (fabsf(dx) > sa.z || fabsf(dy) > sa.w) continue;
                const float4 sb = s_b[j];
                if (kCount) evals++;
                const float power = -0.5f * ((((sb.x * dx) * dx) + ((sb.y * dx) * dy)) + ((sb.z * dy) * dy));
                if (power > 0.0f || power <= DL_POWER_CUT) continue;
                // the 0.999 cap of rasterize.ts:73 never binds: alpha <= opacity *
                // (1 - exp(-4.5)) < 0.99 for opacity <= 1
                const float alpha = sb.w * fmaxf(0.0f, raster_exp<kExactExp>(power) - DL_GAUSS_FLOOR);
                if (alpha < DL_MIN_ALPHA) continue;
                const float w = T * alpha;
                const float4 sc = s_c[j];
                c0 = c0 + w * sc.x;
                c1 = c1 + w * sc.y;
                c2 = c2 + w * sc.z;
                T = T * (1.0f - alpha);
                if (T < DL_MIN_T) { done = true; break; }
            }
        } else if (!done) {
            // +-1 LSB variant: fused multiply-adds and the hardware ex2 on the
            // pre-scaled quadratic form (same skips, same order of splats)
            for (uint32_t j = 0; j < n; j++) {
                const float4 sa = s_a[j];
                const float dx = px - sa.x;
                const float dy = py - sa.y;
                if (fabsf(dx) > sa.z || fabsf(dy) > sa.w) continue;
                const float4 sb = s_b[j];
                if (kCount) evals++;
                const float p2 = __fmaf_rn(dx, __fmaf_rn(sb.x, dx, sb.y * dy), sb.z * dy * dy);
                // p2 <= -4.5 log2(e) needs no test of its own: there ex2 gives at
                // most exp(-4.5) (to 2^-22), so alpha < 1/255 skips the splat below
                if (p2 > 0.0f) continue;
                float e;
                asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(p2));
                // e - floor < 0 near the cut gives alpha < 0: skipped like alpha = 0
                const float alpha = sb.w * (e - DL_GAUSS_FLOOR);
                if (alpha < DL_MIN_ALPHA) continue;
                const float w = T * alpha;
                const float4 sc = s_c[j];
                c0 = __fmaf_rn(w, sc.x, c0);
                c1 = __fmaf_rn(w, sc.y, c1);
                c2 = __fmaf_rn(w, sc.z, c2);
                T = __fmaf_rn(-T, alpha, T);
                if (T < DL_MIN_T) { done = true; break; }
            }
        }
        if (__all_sync(0xffffffffu, done)) break;
        __syncwarp();                                   // staging area is reused by the next step
    }
    if (kCount) {
        uint32_t s = evals;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && s) {
            if (a.tile_evals) atomicAdd(&a.tile_evals[gt], s);
            if (a.eval_count) atomicAdd(a.eval_count, (unsigned long long)s);
        }
    }
    if (inImage) {
        // finalize.ts:30-43
        const float rr = fminf(fmaxf(c0 + T * u.bg[0], 0.0f), 1.0f);
        const float gg = fminf(fmaxf(c1 + T * u.bg[1], 0.0f), 1.0f);
        const float bb = fminf(fmaxf(c2 + T * u.bg[2], 0.0f), 1.0f);
        const float aa = fminf(fmaxf((1.0f - T) + T * u.bg[3], 0.0f), 1.0f);
        const uint32_t out = dl_sat_u32(rr * 255.0f + 0.5f) | (dl_sat_u32(gg * 255.0f + 0.5f) << 8) |
                             (dl_sat_u32(bb * 255.0f + 0.5f) << 16) | (dl_sat_u32(aa * 255.0f + 0.5f) << 24);
        a.outs[v][(uint64_t)y * u.W + x] = out;
        if (a.accum) a.accum[(uint64_t)y * u.W + x] = make_float4(c0, c1, c2, T);
    }
    if (a.tile_cycles && lane == 0) atomicAdd(&a.tile_cycles[gt], (uint32_t)((clock64() - t0) >> 4));
}

// Two pixels per lane: a work item is an 8x8-pixel quarter of a 16x16 tile;
// lane l owns pixels (l % 8, l / 8) and (l % 8, l / 8 + 4) of it.  The two
// pixels share each staged record's shared-memory reads, and a tile's slice is
// scanned by 4 warps instead of 8.  Per pixel, the same arithmetic in the same
// splat order as raster_subtile.
template <bool kExactExp, bool kCount>
__device__ __forceinline__ void raster_subtile2(const RasterArgs& a, uint32_t v, uint32_t tile, uint32_t sub,
                                                uint32_t gt, float4* s_a, float4* s_b, float4* s_c) {
    const DlView& u = a.views[v];
    const int lane = threadIdx.x & 31;
    const uint32_t tx = tile % u.tilesX, ty = tile / u.tilesX;
    const uint32_t perRow = u.tileW >> 3;       // 8x8 work items
    const uint32_t sx0 = tx * u.tileW + (sub % perRow) * 8u, sy0 = ty * u.tileH + (sub / perRow) * 8u;
    const uint32_t x = sx0 + (lane & 7), y0 = sy0 + (lane >> 3), y1 = y0 + 4u;
    const bool in0 = x < u.W && y0 < u.H, in1 = x < u.W && y1 < u.H;
    if (__all_sync(0xffffffffu, !in0)) return;            // y1 > y0: no pixel of the item is inside
    const long long t0 = a.tile_cycles ? clock64() : 0;
    const float px = (float)x + 0.5f, py0 = (float)y0 + 0.5f, py1 = (float)y1 + 0.5f;
    const float rx0 = (float)sx0 + 0.5f - a.stage_pad, rx1 = (float)(sx0 + 8u) - 0.5f + a.stage_pad;
    const float ry0 = (float)sy0 + 0.5f - a.stage_pad, ry1 = (float)(sy0 + 8u) - 0.5f + a.stage_pad;
    const uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    const uint32_t start = to[tile], end = to[tile + 1];
    const uint32_t* vals = a.pair_vals + a.pair_base[v];
    const uint64_t vo = (uint64_t)v * a.view_stride;
    const uint32_t lmask = dl_lanemask_lt();

    float c[2][3] = {{0.0f, 0.0f, 0.0f}, {0.0f, 0.0f, 0.0f}}, T[2] = {1.0f, 1.0f};
    bool done[2] = {!in0, !in1};
    const float py[2] = {py0, py1};
    uint32_t evals = 0;
    for (uint32_t b = start; b < end; b += 64) {
        const uint32_t n = stage_chunk<kExactExp>(a, vals, b, end, vo, rx0, rx1, ry0, ry1, lmask, s_a, s_b, s_c);
        if (n == 0u) continue;
        __syncwarp();
        if (!(done[0] && done[1])) {
            for (uint32_t j = 0; j < n; j++) {
                const float4 sa = s_a[j];
                const float dx = px - sa.x;
                if (fabsf(dx) > sa.z) continue;
                float dy[2];
                bool box[2];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    dy[k] = py[k] - sa.y;
                    box[k] = !done[k] && !(fabsf(dy[k]) > sa.w);
                }
                if (!(box[0] || box[1])) continue;
                const float4 sb = s_b[j];
                float alpha[2];
                bool use[2];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    use[k] = false;
                    alpha[k] = 0.0f;
                    if (box[k]) {
                        if (kCount) evals++;
                        if (kExactExp) {
                            const float power = -0.5f * ((((sb.x * dx) * dx) + ((sb.y * dx) * dy[k])) +
                                                         ((sb.z * dy[k]) * dy[k]));
                            if (!(power > 0.0f || power <= DL_POWER_CUT)) {
                                alpha[k] = sb.w * fmaxf(0.0f, raster_exp<kExactExp>(power) - DL_GAUSS_FLOOR);
                                use[k] = !(alpha[k] < DL_MIN_ALPHA);
                            }
                        } else {
                            const float p2 = __fmaf_rn(dx, __fmaf_rn(sb.x, dx, sb.y * dy[k]), sb.z * dy[k] * dy[k]);
                            if (!(p2 > 0.0f)) {                 // the cut falls to the alpha test
                                float e;
                                asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e) : "f"(p2));
                                alpha[k] = sb.w * (e - DL_GAUSS_FLOOR);
                                use[k] = !(alpha[k] < DL_MIN_ALPHA);
                            }
                        }
                    }
                }
                if (!(use[0] || use[1])) continue;
                const float4 sc = s_c[j];
#pragma unroll
                for (int k = 0; k < 2; k++) {
                    if (use[k]) {
                        const float w = T[k] * alpha[k];
                        if (kExactExp) {
                            c[k][0] = c[k][0] + w * sc.x;
                            c[k][1] = c[k][1] + w * sc.y;
                            c[k][2] = c[k][2] + w * sc.z;
                            T[k] = T[k] * (1.0f - alpha[k]);
                        } else {
                            c[k][0] = __fmaf_rn(w, sc.x, c[k][0]);
                            c[k][1] = __fmaf_rn(w, sc.y, c[k][1]);
                            c[k][2] = __fmaf_rn(w, sc.z, c[k][2]);
                            T[k] = __fmaf_rn(-T[k], alpha[k], T[k]);
                        }
                        if (T[k] < DL_MIN_T) done[k] = true;
                    }
                }
                if (done[0] && done[1]) break;
            }
        }
        if (__all_sync(0xffffffffu, done[0] && done[1])) break;
        __syncwarp();                                   // staging area is reused by the next step
    }
    if (kCount) {
        uint32_t s = evals;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && s) {
            if (a.tile_evals) atomicAdd(&a.tile_evals[gt], s);
            if (a.eval_count) atomicAdd(a.eval_count, (unsigned long long)s);
        }
    }
#pragma unroll
    for (int k = 0; k < 2; k++) {
        const uint32_t y = k ? y1 : y0;
        if (k ? in1 : in0) {
            // finalize.ts:30-43
            const float rr = fminf(fmaxf(c[k][0] + T[k] * u.bg[0], 0.0f), 1.0f);
            const float gg = fminf(fmaxf(c[k][1] + T[k] * u.bg[1], 0.0f), 1.0f);
            const float bb = fminf(fmaxf(c[k][2] + T[k] * u.bg[2], 0.0f), 1.0f);
            const float aa = fminf(fmaxf((1.0f - T[k]) + T[k] * u.bg[3], 0.0f), 1.0f);
            const uint32_t out = dl_sat_u32(rr * 255.0f + 0.5f) | (dl_sat_u32(gg * 255.0f + 0.5f) << 8) |
                                 (dl_sat_u32(bb * 255.0f + 0.5f) << 16) | (dl_sat_u32(aa * 255.0f + 0.5f) << 24);
            a.outs[v][(uint64_t)y * u.W + x] = out;
            if (a.accum) a.accum[(uint64_t)y * u.W + x] = make_float4(c[k][0], c[k][1], c[k][2], T[k]);
        }
    }
    if (a.tile_cycles && lane == 0) atomicAdd(&a.tile_cycles[gt], (uint32_t)((clock64() - t0) >> 4));
}

// ---- two splats per step in packed f32x2 arithmetic (fast variant only)
// Same work item, staging and per-pixel arithmetic as raster_subtile's fast
// loop, but the staged splats are taken two at a time: the quadratic form,
// exponent and alpha of splats j and j+1 at the lane's pixel are evaluated
// together with sm_100's two-wide FP32 instructions (__fadd2_rn, __fmul2_rn,
// __ffma2_rn: per component the same IEEE operation as the scalar
// instruction), then composited one after the other in depth order.  There
// is no per-pixel box test: a staged splat reaches the sub-tile, and at
// pixels outside its box the alpha test skips it (alpha < 1/255 there, see
// tight_extent), so every pixel gets the same splats, values and order as in
// raster_subtile.  Staged values are stored negated where that saves an
// instruction: with na = -alpha, T*na*(-colour) = T*alpha*colour and
// fma(T, na, T) = fma(-T, alpha, T) exactly.
//
// Shared memory per warp: 32 pairs of staged splats, 20 floats a pair:
//   {-x0, -x1, -y0, -y1}, {A0, A1, B0, B1}, {C0, C1, -o0, -o1},
//   {-r0, -g0, -r1, -g1}, {-b0, -b1, unused, unused}
// (A, B, C: the conic scaled by -0.5 log2 e as in stage_chunk's fast path;
// red and green of a splat side by side, so one f32x2 FMA blends both.)
constexpr int kPairFloats = 20;

// Composites the n staged splats of a warp's packed pair buffer sp (layout
// above) at the lane's pixel, two splats per step, in staging order; sets done
// once T < 1e-4 (the shader's early out) and stops there.  Skipped splats go
// through the blend with alpha 0 (no branch): fma(T, 0, T) = T and
// fma(T * 0, -colour, c) = c for a finite colour.  The second splat of a step
// also blends with alpha 0 when the first one ended the pixel, so one test of
// T per step serves both.
__device__ __forceinline__ void composite_x2(const float* sp, uint32_t n, float2 px2, float2 py2, float& c0,
                                             float& c1, float& c2, float& T, bool& done) {
    const float2 nfloor2 = make_float2(-DL_GAUSS_FLOOR, -DL_GAUSS_FLOOR);
    for (uint32_t j = 0; j < n; j += 2) {
        const float4* P = reinterpret_cast<const float4*>(sp + (j >> 1) * kPairFloats);
        const float4 q0 = P[0], q1 = P[1], q2 = P[2];
        const float2 dx = __fadd2_rn(px2, make_float2(q0.x, q0.y));
        const float2 dy = __fadd2_rn(py2, make_float2(q0.z, q0.w));
        const float2 t = __fmul2_rn(make_float2(q1.z, q1.w), dy);
        const float2 qq = __ffma2_rn(make_float2(q1.x, q1.y), dx, t);
        const float2 uu = __fmul2_rn(__fmul2_rn(make_float2(q2.x, q2.y), dy), dy);
        const float2 pw = __ffma2_rn(dx, qq, uu);
        float e0, e1;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e0) : "f"(pw.x));
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e1) : "f"(pw.y));
        const float2 na = __fmul2_rn(make_float2(q2.z, q2.w), __fadd2_rn(make_float2(e0, e1), nfloor2));
        // the shader's skips: power > 0, alpha < 1/255
        const bool ok0 = !(pw.x > 0.0f) && !(na.x > -DL_MIN_ALPHA);
        const bool ok1 = !(pw.y > 0.0f) && !(na.y > -DL_MIN_ALPHA);
        {
            const float4 q3 = P[3], q4 = P[4];
            const float a0 = ok0 ? na.x : 0.0f;
            float w = T * a0;
            float2 rg = make_float2(c0, c1);
            rg = __ffma2_rn(make_float2(w, w), make_float2(q3.x, q3.y), rg);
            c2 = __fmaf_rn(w, q4.x, c2);
            T = __fmaf_rn(T, a0, T);
            const bool d0 = T < DL_MIN_T;
            const float a1 = (ok1 && !d0) ? na.y : 0.0f;
            w = T * a1;
            rg = __ffma2_rn(make_float2(w, w), make_float2(q3.z, q3.w), rg);
            c2 = __fmaf_rn(w, q4.y, c2);
            T = __fmaf_rn(T, a1, T);
            c0 = rg.x; c1 = rg.y;
            if (T < DL_MIN_T) { done = true; return; }
        }
    }
}

// Writes a staged splat into slot `slot` of a packed pair buffer.
__device__ __forceinline__ void put_pair_slot(float* sp, uint32_t slot, float x, float y, float A, float B, float C,
                                              float al, float cr, float cg, float cb) {
    float* P = sp + (slot >> 1) * kPairFloats;
    const uint32_t c = slot & 1u;
    P[0 + c] = -x;
    P[2 + c] = -y;
    P[4 + c] = -0.72134752044448170f * A;
    P[6 + c] = -1.4426950408889634f * B;
    P[8 + c] = -0.72134752044448170f * C;
    P[10 + c] = -al;
    // colours are >= 0 (project.ts clamps at 0, no upper clamp); an infinite
    // one is held as FLT_MAX, so that alpha 0 times it is 0 and a composited
    // one still saturates its channel: the final bytes are the same
    P[12 + 2 * c] = -fminf(cr, 3.402823466e38f);
    P[13 + 2 * c] = -fminf(cg, 3.402823466e38f);
    P[16 + c] = -fminf(cb, 3.402823466e38f);
}

// An odd count: a splat of opacity 0 fills the last pair (alpha 0 is skipped).
__device__ __forceinline__ void pad_pair_slot(float* sp, uint32_t n) {
    float* P = sp + (n >> 1) * kPairFloats;
    P[1] = 0.0f; P[3] = 0.0f; P[5] = 0.0f; P[7] = 0.0f; P[9] = 0.0f; P[11] = -0.0f;
    P[14] = 0.0f; P[15] = 0.0f; P[17] = 0.0f;
}

// Writes a splat already in the packed form (negated, conic pre-scaled, colours
// held finite: the values put_pair_slot computes) into slot `slot`.
__device__ __forceinline__ void put_pair_slot_raw(float* sp, uint32_t slot, const float4& fa, const float4& fb,
                                                  float fc) {
    float* P = sp + (slot >> 1) * kPairFloats;
    const uint32_t c = slot & 1u;
    P[0 + c] = fa.x; P[2 + c] = fa.y; P[4 + c] = fa.z; P[6 + c] = fa.w;
    P[8 + c] = fb.x; P[10 + c] = fb.y; P[12 + 2 * c] = fb.z; P[13 + 2 * c] = fb.w;
    P[16 + c] = fc;
}

__device__ __forceinline__ uint32_t stage_chunk_x2(const RasterArgs& a, const uint32_t* vals, uint32_t b,
                                                   uint32_t end, uint64_t vo, float rx0, float rx1, float ry0,
                                                   float ry1, uint32_t lmask, float* sp) {
    const int lane = threadIdx.x & 31;
    const uint32_t e0 = b + lane, e1 = b + 32 + lane;
    const uint32_t g0 = e0 < end ? __ldg(vals + e0) : kPhantomBit;
    const uint32_t g1 = e1 < end ? __ldg(vals + e1) : kPhantomBit;
    bool hit0 = false, hit1 = false;
    float4 ra0 = make_float4(0, 0, 0, 0), ra1 = make_float4(0, 0, 0, 0);
    if (!(g0 & kPhantomBit)) {
        ra0 = __ldg(a.recA + vo + g0);
        const float rx = ra0.z, ry = a.rec_box ? ra0.w : ra0.z;
        hit0 = rx > 0.0f && !(ra0.x - rx > rx1) && !(ra0.x + rx < rx0) && !(ra0.y - ry > ry1) && !(ra0.y + ry < ry0);
    }
    if (!(g1 & kPhantomBit)) {
        ra1 = __ldg(a.recA + vo + g1);
        const float rx = ra1.z, ry = a.rec_box ? ra1.w : ra1.z;
        hit1 = rx > 0.0f && !(ra1.x - rx > rx1) && !(ra1.x + rx < rx0) && !(ra1.y - ry > ry1) && !(ra1.y + ry < ry0);
    }
    if (__ballot_sync(0xffffffffu, hit0 || hit1) == 0u) return 0u;
    uint32_t n = 0;
#pragma unroll
    for (int h = 0; h < 2; h++) {
        bool hit = h ? hit1 : hit0;
        const uint32_t g = h ? g1 : g0;
        const float4 ra = h ? ra1 : ra0;
        float A = 0.0f, B = 0.0f, C = 0.0f, al = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
        if (hit) {
            if (a.recBC) {
                const float4 p = __ldg(a.recBC + 2 * (vo + g));
                const float4 q = __ldg(a.recBC + 2 * (vo + g) + 1);
                A = p.x; B = p.y; C = p.z; al = p.w; cr = q.x; cg = q.y; cb = q.z;
            } else {
                const uint4 hv = __ldg(a.recH + vo + g);
                const float2 ab = __half22float2(*reinterpret_cast<const __half2*>(&hv.x));
                const float2 ca = __half22float2(*reinterpret_cast<const __half2*>(&hv.y));
                const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&hv.z));
                const float2 bz = __half22float2(*reinterpret_cast<const __half2*>(&hv.w));
                A = ab.x; B = ab.y; C = ca.x; al = ca.y; cr = rg.x; cg = rg.y; cb = bz.x;
            }
            if (!a.rec_box) {
                float ex, ey;
                tight_extent(A, B, C, ra.z, ex, ey);
                hit = !(ra.x - ex > rx1) && !(ra.x + ex < rx0) && !(ra.y - ey > ry1) && !(ra.y + ey < ry0);
            }
        }
        const uint32_t m = __ballot_sync(0xffffffffu, hit);
        if (hit) put_pair_slot(sp, n + __popc(m & lmask), ra.x, ra.y, A, B, C, al, cr, cg, cb);
        n += __popc(m);
    }
    if ((n & 1u) && lane == 0) pad_pair_slot(sp, n);
    return n;
}

template <bool kCycles>
__device__ __forceinline__ void raster_subtile_x2(const RasterArgs& a, uint32_t v, uint32_t tile, uint32_t sub,
                                                  uint32_t gt, float* sp) {
    const DlView& u = a.views[v];
    const int lane = threadIdx.x & 31;
    const uint32_t tx = tile % u.tilesX, ty = tile / u.tilesX;
    const uint32_t lw = (uint32_t)a.sub_lw, sw = 1u << lw, sh = 32u >> lw, perRow = u.tileW >> lw;
    const uint32_t sx0 = tx * u.tileW + (sub % perRow) * sw, sy0 = ty * u.tileH + (sub / perRow) * sh;
    const uint32_t x = sx0 + (lane & (sw - 1)), y = sy0 + (lane >> lw);
    const bool inImage = x < u.W && y < u.H;
    if (__all_sync(0xffffffffu, !inImage)) return;
    const long long t0 = kCycles ? clock64() : 0;
    const float px = (float)x + 0.5f, py = (float)y + 0.5f;
    const float pad = a.stage_pad;
    const float rx0 = (float)sx0 + 0.5f - pad, rx1 = (float)(sx0 + sw) - 0.5f + pad;
    const float ry0 = (float)sy0 + 0.5f - pad, ry1 = (float)(sy0 + sh) - 0.5f + pad;
    const uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
    const uint32_t start = to[tile], end = to[tile + 1];
    const uint32_t* vals = a.pair_vals + a.pair_base[v];
    const uint64_t vo = (uint64_t)v * a.view_stride;
    const uint32_t lmask = dl_lanemask_lt();
    const float2 px2 = make_float2(px, px), py2 = make_float2(py, py);

    float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, T = 1.0f;
    bool done = !inImage;
    for (uint32_t b = start; b < end; b += 64) {
        const uint32_t n = stage_chunk_x2(a, vals, b, end, vo, rx0, rx1, ry0, ry1, lmask, sp);
        if (n == 0u) continue;
        __syncwarp();
        if (!done) composite_x2(sp, n, px2, py2, c0, c1, c2, T, done);
        if (__all_sync(0xffffffffu, done)) break;
        __syncwarp();                                   // staging area is reused by the next step
    }
    if (inImage) {
        // finalize.ts:30-43
        const float rr = fminf(fmaxf(c0 + T * u.bg[0], 0.0f), 1.0f);
        const float gg = fminf(fmaxf(c1 + T * u.bg[1], 0.0f), 1.0f);
        const float bb = fminf(fmaxf(c2 + T * u.bg[2], 0.0f), 1.0f);
        const float aa = fminf(fmaxf((1.0f - T) + T * u.bg[3], 0.0f), 1.0f);
        const uint32_t out = dl_sat_u32(rr * 255.0f + 0.5f) | (dl_sat_u32(gg * 255.0f + 0.5f) << 8) |
                             (dl_sat_u32(bb * 255.0f + 0.5f) << 16) | (dl_sat_u32(aa * 255.0f + 0.5f) << 24);
        a.outs[v][(uint64_t)y * u.W + x] = out;
        if (a.accum) a.accum[(uint64_t)y * u.W + x] = make_float4(c0, c1, c2, T);
    }
    if (kCycles && lane == 0) atomicAdd(&a.tile_cycles[gt], (uint32_t)((clock64() - t0) >> 4));
}

// The two-pixels-per-lane rasterizer: 8x8-pixel work items (4 per 16x16 tile).
template <bool kExactExp, bool kCount = false>
__global__ void __launch_bounds__(kRasterThreads, 5) rasterize2_k(RasterArgs a) {
    __shared__ float4 s_a[kRasterWarps][64];
    __shared__ float4 s_b[kRasterWarps][64];
    __shared__ float4 s_c[kRasterWarps][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    while (true) {
        uint32_t item = 0;
        if (lane == 0) item = a.item_base + atomicAdd(a.work_counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.num_items) return;
        const uint32_t gt = a.work ? a.work[item >> a.ipt_lg] : (item >> a.ipt_lg);
        const uint32_t v = view_of_tile(a, gt);
        raster_subtile2<kExactExp, kCount>(a, v, gt - a.tile_base[v], item & ((1u << a.ipt_lg) - 1u), gt, s_a[warp],
                                           s_b[warp], s_c[warp]);
        __syncwarp();
    }
}

template <bool kExactExp, bool kCount = false>
__global__ void __launch_bounds__(kRasterThreads, 6) rasterize_k(RasterArgs a) {
    __shared__ float4 s_a[kRasterWarps][64];
    __shared__ float4 s_b[kRasterWarps][64];
    __shared__ float4 s_c[kRasterWarps][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    while (true) {
        uint32_t item = 0;
        if (lane == 0) item = a.item_base + atomicAdd(a.work_counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.num_items) return;
        const uint32_t gt = a.work ? a.work[item >> a.ipt_lg] : (item >> a.ipt_lg);
        const uint32_t v = view_of_tile(a, gt);
        raster_subtile<kExactExp, kCount>(a, v, gt - a.tile_base[v], item & ((1u << a.ipt_lg) - 1u), gt, s_a[warp],
                                          s_b[warp], s_c[warp]);
        __syncwarp();
    }
}

// The packed two-splat rasterizer (fast variant): 32-pixel work items (8 per 16x16 tile).
template <bool kCycles = false>
__global__ void __launch_bounds__(kRasterThreads, 6) rasterize_x2_k(RasterArgs a) {
    __shared__ __align__(16) float s_p[kRasterWarps][32 * kPairFloats];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    while (true) {
        uint32_t item = 0;
        if (lane == 0) item = a.item_base + atomicAdd(a.work_counter, 1u);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= a.num_items) return;
        const uint32_t gt = a.work ? a.work[item >> a.ipt_lg] : (item >> a.ipt_lg);
        const uint32_t v = view_of_tile(a, gt);
        raster_subtile_x2<kCycles>(a, v, gt - a.tile_base[v], item & ((1u << a.ipt_lg) - 1u), gt, s_p[warp]);
        __syncwarp();
    }
}

// ---- one CTA per tile: the tile's slice is read once (fast variant)
// A persistent CTA of 8 warps takes whole 256-pixel tiles (16x16, or 32x8 when
// tuned); warp w owns the 8x4 work item w of the tile.  The slice is read in
// batches of 256 pairs, one pair per thread: the thread loads the pair value
// and screen record, tests the splat's box (staging margin as in stage_chunk)
// against the 8 items' pixel-centre rectangles, and for a splat that reaches
// any of them loads its record and stages it in shared memory with an 8-bit
// mask of the items it reaches.  Each warp then takes, in slice order, the
// staged splats of its own item (ballots over the masks), packs them into its
// pair buffer 64 at a time and composites them with composite_x2 — the same
// splats, values and order as raster_subtile_x2.  The CTA stops reading the
// slice once all 8 warps' pixels are done.  Reads per pair: one pair value and
// one screen record per tile (not per work item), and one record per splat
// that reaches the tile.
constexpr int kTileStage = kRasterThreads;     // pairs staged per batch

template <bool kCycles>
__global__ void __launch_bounds__(kRasterThreads, 5) rasterize_tile_x2_k(RasterArgs a) {
    // each staged pair in the packed form of the pair buffers (put_pair_slot's
    // values, computed once here instead of once per work item it reaches)
    __shared__ float4 s_fa[kTileStage];        // -x, -y, -A log2(e)/2, -B log2(e)
    __shared__ float4 s_fb[kTileStage];        // -C log2(e)/2, -alpha, -r, -g
    __shared__ float s_fc[kTileStage];         // -b
    __shared__ uint8_t s_m[kTileStage];        // items the staged splat reaches (bit w: item w)
    __shared__ __align__(16) float s_p[kRasterWarps][32 * kPairFloats];
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t lmask = dl_lanemask_lt();
    float* sp = s_p[warp];
    while (true) {
        if (tid == 0) s_tile = a.item_base + atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t item = s_tile;
        if (item >= a.num_items) return;
        const uint32_t gt = a.work ? a.work[item] : item;
        const uint32_t v = view_of_tile(a, gt);
        const uint32_t tile = gt - a.tile_base[v];
        const DlView& u = a.views[v];
        const long long t0 = kCycles ? clock64() : 0;
        const uint32_t tx = tile % u.tilesX, ty = tile / u.tilesX;
        const uint32_t perRow = u.tileW >> 3;              // 8x4 items per tile row
        const uint32_t ox = tx * u.tileW, oy = ty * u.tileH;
        const uint32_t sx0 = ox + (warp % perRow) * 8u, sy0 = oy + (warp / perRow) * 4u;
        const uint32_t x = sx0 + (lane & 7), y = sy0 + (lane >> 3);
        const bool inImage = x < u.W && y < u.H;
        const float2 px2 = make_float2((float)x + 0.5f, (float)x + 0.5f);
        const float2 py2 = make_float2((float)y + 0.5f, (float)y + 0.5f);
        const uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
        const uint32_t start = to[tile], end = to[tile + 1];
        const uint32_t* vals = a.pair_vals + a.pair_base[v];
        const uint64_t vo = (uint64_t)v * a.view_stride;
        const float pad = a.stage_pad;
        float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, T = 1.0f;
        bool done = !inImage;
        // the thread's pair value of the next batch is loaded while this batch
        // is composited (one dependent load fewer before the staging barrier)
        uint32_t gNext = start + (uint32_t)tid < end ? __ldg(vals + start + tid) : 0u;
        for (uint32_t b = start; b < end; b += kTileStage) {
            // ---- stage one pair per thread
            uint32_t mask = 0;
            const uint32_t e = b + (uint32_t)tid;
            const uint32_t g = gNext;
            if (e + kTileStage < end) gNext = __ldg(vals + e + kTileStage);
            if (e < end) {
                if (!(g & kPhantomBit)) {
                    const float4 ra = __ldg(a.recA + vo + g);
                    float ex = ra.z, ey = a.rec_box ? ra.w : ra.z;
                    float A = 0.0f, B = 0.0f, C = 0.0f, al = 0.0f, cr = 0.0f, cg = 0.0f, cb = 0.0f;
                    if (ex > 0.0f) {
                        // the box against the tile's pixel-centre rectangle first
                        const float tx0 = (float)ox + 0.5f - pad, tx1 = (float)(ox + u.tileW) - 0.5f + pad;
                        const float ty0 = (float)oy + 0.5f - pad, ty1 = (float)(oy + u.tileH) - 0.5f + pad;
                        if (!(ra.x - ex > tx1) && !(ra.x + ex < tx0) && !(ra.y - ey > ty1) && !(ra.y + ey < ty0)) {
                            if (a.recBC) {
                                const float4 p = __ldg(a.recBC + 2 * (vo + g));
                                const float4 q = __ldg(a.recBC + 2 * (vo + g) + 1);
                                A = p.x; B = p.y; C = p.z; al = p.w; cr = q.x; cg = q.y; cb = q.z;
                            } else {
                                const uint4 hv = __ldg(a.recH + vo + g);
                                const float2 ab = __half22float2(*reinterpret_cast<const __half2*>(&hv.x));
                                const float2 ca = __half22float2(*reinterpret_cast<const __half2*>(&hv.y));
                                const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&hv.z));
                                const float2 bz = __half22float2(*reinterpret_cast<const __half2*>(&hv.w));
                                A = ab.x; B = ab.y; C = ca.x; al = ca.y; cr = rg.x; cg = rg.y; cb = bz.x;
                            }
                            if (!a.rec_box) tight_extent(A, B, C, ra.z, ex, ey);
                            // items: 8x4 pixels, perRow per tile row; item column c covers
                            // pixel centres ox + 8c + 0.5 .. + 7.5, item row r oy + 4r + 0.5 .. + 3.5
                            const float lx = ra.x - ex - pad - (float)ox, hx = ra.x + ex + pad - (float)ox;
                            const float ly = ra.y - ey - pad - (float)oy, hy = ra.y + ey + pad - (float)oy;
                            if (ex == ex && ey == ey) {
                                const int cA = max(0, (int)ceilf((lx - 7.5f) * 0.125f));
                                const int cB = min((int)perRow - 1, (int)floorf((hx - 0.5f) * 0.125f));
                                const int rA = max(0, (int)ceilf((ly - 3.5f) * 0.25f));
                                const int rB = min(kRasterWarps / (int)perRow - 1, (int)floorf((hy - 0.5f) * 0.25f));
                                if (cA <= cB && rA <= rB) {
                                    const uint32_t cm = ((2u << cB) - 1u) & ~((1u << cA) - 1u);
                                    for (int r = rA; r <= rB; r++) mask |= cm << (r * (int)perRow);
                                }
                            } else {
                                mask = (1u << kRasterWarps) - 1u;   // a NaN extent reaches every item, as
                            }                                       // the comparisons it fails would say
                            if (mask) {
                                s_fa[tid] = make_float4(-ra.x, -ra.y, -0.72134752044448170f * A,
                                                        -1.4426950408889634f * B);
                                s_fb[tid] = make_float4(-0.72134752044448170f * C, -al, -fminf(cr, 3.402823466e38f),
                                                        -fminf(cg, 3.402823466e38f));
                                s_fc[tid] = -fminf(cb, 3.402823466e38f);
                            }
                        }
                    }
                }
            }
            s_m[tid] = (uint8_t)mask;
            __syncthreads();
            // ---- this warp's splats, 64 at a time, in slice order
            const uint32_t nb = min((uint32_t)kTileStage, end - b);
            if (!__all_sync(0xffffffffu, done)) {
                for (uint32_t c = 0; c < nb; c += 64) {
                    uint32_t n = 0;
#pragma unroll
                    for (int h = 0; h < 2; h++) {
                        const uint32_t i = c + (uint32_t)h * 32u + (uint32_t)lane;
                        const bool hit = i < nb && ((s_m[i] >> warp) & 1u);
                        const uint32_t m = __ballot_sync(0xffffffffu, hit);
                        if (hit) put_pair_slot_raw(sp, n + __popc(m & lmask), s_fa[i], s_fb[i], s_fc[i]);
                        n += __popc(m);
                    }
                    if (n == 0u) continue;
                    if ((n & 1u) && lane == 0) pad_pair_slot(sp, n);
                    __syncwarp();
                    if (!done) composite_x2(sp, n, px2, py2, c0, c1, c2, T, done);
                    __syncwarp();                           // the pair buffer is refilled next
                    if (__all_sync(0xffffffffu, done)) break;
                }
            }
            // every warp is past this batch's staging area; stop once all pixels are done
            if (__syncthreads_and(done)) break;
        }
        if (inImage) {
            // finalize.ts:30-43
            const float rr = fminf(fmaxf(c0 + T * u.bg[0], 0.0f), 1.0f);
            const float gg = fminf(fmaxf(c1 + T * u.bg[1], 0.0f), 1.0f);
            const float bb = fminf(fmaxf(c2 + T * u.bg[2], 0.0f), 1.0f);
            const float aa = fminf(fmaxf((1.0f - T) + T * u.bg[3], 0.0f), 1.0f);
            const uint32_t out = dl_sat_u32(rr * 255.0f + 0.5f) | (dl_sat_u32(gg * 255.0f + 0.5f) << 8) |
                                 (dl_sat_u32(bb * 255.0f + 0.5f) << 16) | (dl_sat_u32(aa * 255.0f + 0.5f) << 24);
            a.outs[v][(uint64_t)y * u.W + x] = out;
            if (a.accum) a.accum[(uint64_t)y * u.W + x] = make_float4(c0, c1, c2, T);
        }
        if (kCycles && tid == 0) atomicAdd(&a.tile_cycles[gt], (uint32_t)((clock64() - t0) >> 4));
        __syncthreads();                                    // s_tile is rewritten next
    }
}

// ---- one CTA per tile, staged records read in place (both arithmetic variants)
// As rasterize_tile_x2_k, a persistent CTA of 8 warps takes whole 256-pixel
// tiles and reads the slice once, 256 pairs per batch, one pair per thread.
// The work is split into 4x4-pixel cells, 16 per tile: each half-warp owns
// one cell (lanes 0-15 the left half of warp w's 8x4 block, lanes 16-31 the
// right half) and composites its own list of splats, so a splat that reaches
// only one half of the block costs the other half nothing.  The staging
// thread computes the cells its splat's box reaches from the box's column and
// row ranges (pixel-centre rectangles widened by the staging margin) and
// stores the record once, in the form the compositing loop reads it (x, y and
// the conic, opacity, colour).  Each half-warp then lists the batch slots of
// its cell in slice order (ballots, one byte per slot) and composites straight
// from the staged records with rasterize.ts:62-79 per pixel in slice order:
// the exact arithmetic of raster_subtile (kExactExp) or its fast loop.  There
// is no per-pixel box test: at pixels outside the box alpha < 1/255 is skipped.
template <bool kExactExp, bool kCycles>
__global__ void __launch_bounds__(kRasterThreads, 5) rasterize_tile_k(RasterArgs a) {
    __shared__ float4 s_r[2][kTileStage];      // staged records: (x, y, A, B), (C, alpha, r, g)
    __shared__ float s_b[kTileStage];          // staged blue
    __shared__ uint16_t s_m[kTileStage];       // cells the staged splat reaches (bit c: cell c, row-major)
    __shared__ uint8_t s_l[kRasterWarps][2][kTileStage];   // per half-warp: its batch slots in order
    __shared__ uint32_t s_tile;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, half = lane >> 4;
    const uint32_t lmask = dl_lanemask_lt();
    while (true) {
        if (tid == 0) s_tile = a.item_base + atomicAdd(a.work_counter, 1u);
        __syncthreads();
        const uint32_t item = s_tile;
        if (item >= a.num_items) return;
        const uint32_t gt = a.work ? a.work[item] : item;
        const uint32_t v = view_of_tile(a, gt);
        const uint32_t tile = gt - a.tile_base[v];
        const DlView& u = a.views[v];
        const long long t0 = kCycles ? clock64() : 0;
        const uint32_t tx = tile % u.tilesX, ty = tile / u.tilesX;
        const uint32_t perRow = u.tileW >> 3;               // 8x4 blocks (one per warp) per tile row
        const uint32_t cols = u.tileW >> 2, rows = u.tileH >> 2;   // 4x4 cells
        const uint32_t ox = tx * u.tileW, oy = ty * u.tileH;
        const uint32_t cx = (warp % perRow) * 2u + (uint32_t)half, cy = warp / perRow;
        const uint32_t x = ox + cx * 4u + (lane & 3), y = oy + cy * 4u + ((lane >> 2) & 3);
        const bool inImage = x < u.W && y < u.H;
        const float px = (float)x + 0.5f, py = (float)y + 0.5f;
        const uint32_t* to = a.tile_off + (uint64_t)v * a.tile_stride;
        const uint32_t start = to[tile], end = to[tile + 1];
        const uint32_t* vals = a.pair_vals + a.pair_base[v];
        const uint64_t vo = (uint64_t)v * a.view_stride;
        const float pad = a.stage_pad;
        float c0 = 0.0f, c1 = 0.0f, c2 = 0.0f, T = 1.0f;
        bool done = !inImage;
        // the thread's pair value of the next batch is loaded while this batch
        // is composited (one dependent load fewer before the staging barrier)
        uint32_t gNext = start + (uint32_t)tid < end ? __ldg(vals + start + tid) : 0u;
        for (uint32_t b = start; b < end; b += kTileStage) {
            // ---- stage one pair per thread
            uint32_t mask = 0;
            const uint32_t e = b + (uint32_t)tid;
            const uint32_t g = gNext;
            if (e + kTileStage < end) gNext = __ldg(vals + e + kTileStage);
            if (e < end) {
                if (!(g & kPhantomBit)) {
                    const float4 ra = __ldg(a.recA + vo + g);
                    float ex = ra.z, ey = a.rec_box ? ra.w : ra.z;
                    if (ex > 0.0f) {
                        float A, B, C, al, cr, cg, cb;
                        if (a.recBC) {
                            const float4 p = __ldg(a.recBC + 2 * (vo + g));
                            const float4 q = __ldg(a.recBC + 2 * (vo + g) + 1);
                            A = p.x; B = p.y; C = p.z; al = p.w; cr = q.x; cg = q.y; cb = q.z;
                        } else {
                            const uint4 hv = __ldg(a.recH + vo + g);
                            const float2 ab = __half22float2(*reinterpret_cast<const __half2*>(&hv.x));
                            const float2 ca = __half22float2(*reinterpret_cast<const __half2*>(&hv.y));
                            const float2 rg = __half22float2(*reinterpret_cast<const __half2*>(&hv.z));
                            const float2 bz = __half22float2(*reinterpret_cast<const __half2*>(&hv.w));
                            A = ab.x; B = ab.y; C = ca.x; al = ca.y; cr = rg.x; cg = rg.y; cb = bz.x;
                        }
                        if (!a.rec_box) tight_extent(A, B, C, ra.z, ex, ey);
                        // cell column c covers pixel centres ox + 4c + 0.5 .. ox + 4c + 3.5,
                        // cell row r covers oy + 4r + 0.5 .. oy + 4r + 3.5
                        const float lx = ra.x - ex - pad - (float)ox, hx = ra.x + ex + pad - (float)ox;
                        const float ly = ra.y - ey - pad - (float)oy, hy = ra.y + ey + pad - (float)oy;
                        const int cA = max(0, (int)ceilf((lx - 3.5f) * 0.25f));
                        const int cB = min((int)cols - 1, (int)floorf((hx - 0.5f) * 0.25f));
                        const int rA = max(0, (int)ceilf((ly - 3.5f) * 0.25f));
                        const int rB = min((int)rows - 1, (int)floorf((hy - 0.5f) * 0.25f));
                        if (cA <= cB && rA <= rB) {
                            const uint32_t cm = ((1u << (cB + 1)) - 1u) & ~((1u << cA) - 1u);
                            for (int r = rA; r <= rB; r++) mask |= cm << (r * (int)cols);
                            if (kExactExp) {
                                s_r[0][tid] = make_float4(ra.x, ra.y, A, 2.0f * B);
                            } else {
                                // conic pre-scaled by -0.5*log2(e): the quadratic form is ex2's argument
                                s_r[0][tid] = make_float4(ra.x, ra.y, -0.72134752044448170f * A,
                                                          -1.4426950408889634f * B);
                                C = -0.72134752044448170f * C;
                            }
                            s_r[1][tid] = make_float4(C, al, cr, cg);
                            s_b[tid] = cb;
                        }
                    }
                }
            }
            s_m[tid] = (uint16_t)mask;
            __syncthreads();
            const uint32_t nb = min((uint32_t)kTileStage, end - b);
            if (!__all_sync(0xffffffffu, done)) {
                // ---- the slots of both cells of this warp, in slice order
                const uint32_t c0bit = (warp % perRow) * 2u + cy * cols;   // the left cell's bit
                uint32_t n0 = 0, n1 = 0;
                for (uint32_t c = 0; c < nb; c += 32) {
                    const uint32_t i = c + (uint32_t)lane;
                    const uint32_t mm = i < nb ? (uint32_t)s_m[i] >> c0bit : 0u;
                    const uint32_t m0 = __ballot_sync(0xffffffffu, mm & 1u);
                    const uint32_t m1 = __ballot_sync(0xffffffffu, mm & 2u);
                    if (mm & 1u) s_l[warp][0][n0 + __popc(m0 & lmask)] = (uint8_t)i;
                    if (mm & 2u) s_l[warp][1][n1 + __popc(m1 & lmask)] = (uint8_t)i;
                    n0 += __popc(m0);
                    n1 += __popc(m1);
                }
                __syncwarp();
                const uint32_t n = half ? n1 : n0;
                const uint8_t* lst = s_l[warp][half];
                if (!done) {
                    for (uint32_t j = 0; j < n; j++) {
                        const uint32_t i = lst[j];
                        const float4 r0 = s_r[0][i], r1 = s_r[1][i];
                        const float dx = px - r0.x, dy = py - r0.y;
                        float alpha;
                        if (kExactExp) {
                            const float power = -0.5f * ((((r0.z * dx) * dx) + ((r0.w * dx) * dy)) + ((r1.x * dy) * dy));
                            if (power > 0.0f || power <= DL_POWER_CUT) continue;
                            alpha = r1.y * fmaxf(0.0f, dl_expf(power) - DL_GAUSS_FLOOR);
                        } else {
                            const float p2 = __fmaf_rn(dx, __fmaf_rn(r0.z, dx, r0.w * dy), r1.x * dy * dy);
                            if (p2 > 0.0f) continue;
                            float ev;
                            asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ev) : "f"(p2));
                            alpha = r1.y * (ev - DL_GAUSS_FLOOR);
                        }
                        if (alpha < DL_MIN_ALPHA) continue;
                        const float w = T * alpha;
                        const float cbl = s_b[i];
                        if (kExactExp) {
                            c0 = c0 + w * r1.z;
                            c1 = c1 + w * r1.w;
                            c2 = c2 + w * cbl;
                            T = T * (1.0f - alpha);
                        } else {
                            c0 = __fmaf_rn(w, r1.z, c0);
                            c1 = __fmaf_rn(w, r1.w, c1);
                            c2 = __fmaf_rn(w, cbl, c2);
                            T = __fmaf_rn(-T, alpha, T);
                        }
                        if (T < DL_MIN_T) { done = true; break; }
                    }
                }
            }
            // every warp is past this batch's staging area; stop once all pixels are done
            if (__syncthreads_and(done)) break;
        }
        if (inImage) {
            // finalize.ts:30-43
            const float rr = fminf(fmaxf(c0 + T * u.bg[0], 0.0f), 1.0f);
            const float gg = fminf(fmaxf(c1 + T * u.bg[1], 0.0f), 1.0f);
            const float bb = fminf(fmaxf(c2 + T * u.bg[2], 0.0f), 1.0f);
            const float aa = fminf(fmaxf((1.0f - T) + T * u.bg[3], 0.0f), 1.0f);
            const uint32_t out = dl_sat_u32(rr * 255.0f + 0.5f) | (dl_sat_u32(gg * 255.0f + 0.5f) << 8) |
                                 (dl_sat_u32(bb * 255.0f + 0.5f) << 16) | (dl_sat_u32(aa * 255.0f + 0.5f) << 24);
            a.outs[v][(uint64_t)y * u.W + x] = out;
            if (a.accum) a.accum[(uint64_t)y * u.W + x] = make_float4(c0, c1, c2, T);
        }
        if (kCycles && tid == 0) atomicAdd(&a.tile_cycles[gt], (uint32_t)((clock64() - t0) >> 4));
        __syncthreads();                                    // s_tile is rewritten next
    }
}

}  // namespace dlr

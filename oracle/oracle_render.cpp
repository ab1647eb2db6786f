// ORACLE — test infrastructure only.  CPU restatement of droplet's forward
// renderer (TypeScript CPU stages + WGSL compute shaders), used by tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker.
// Nothing in the product (droplet_b200/) links, loads or calls this file.
//
// Every function follows the reference file:line it cites, statement by
// statement, in IEEE f32 (f64 where the TypeScript computes in JS numbers),
// left-to-right evaluation, no FMA contraction (built with -ffp-contract=off).
// The only shared code with the product is dl_math.h (exp / atan2 / asin),
// which the WGSL leaves implementation-defined.
//
// Parity unpinned: the reference pins no numeric outputs (its only tests are
// qualitative browser checks, examples/browser/test.ts:114-273) and cannot run
// here (WebGPU), so no reference output exists to pin this oracle against.  It
// is checked by those ported qualitative checks plus hand-derived closed-form
// known answers (tests/golden/kat.json).
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

// src/render/shaders/constants.ts:19-26,37-38 — WGSL literals parsed as f32.
constexpr uint32_t TILE_SIZE = 16;
constexpr float SIGMA_CUTOFF = 3.0f;
constexpr float AA_DILATION_COV = 0.3f;
constexpr float OPACITY_CAP = 0.999f;
constexpr float MIN_TRANSMITTANCE = 0.0001f;
constexpr float MIN_ALPHA = 0.00392156862745098f;          // 1/255 printed by JS
constexpr float GAUSSIAN_FLOOR = 1.1108996538e-2f;         // exp(-4.5).toExponential(10)
constexpr float RADIUS_FADE_START_FRAC = 0.9481481481481482f;   // 1024/1080
constexpr float RADIUS_FADE_END_FRAC = 1.8962962962962964f;     // 2048/1080

struct Vec3f { float x, y, z; };

inline Vec3f cross(Vec3f a, Vec3f b) {            // WGSL cross()
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// project.ts:50-53  quatRot(q, v): t = 2*cross(q.yzw, v); v + q.x*t + cross(q.yzw, t)
inline Vec3f quatRot(const float q[4], Vec3f v) {
    const Vec3f qv{q[1], q[2], q[3]};
    Vec3f c = cross(qv, v);
    Vec3f t{2.0f * c.x, 2.0f * c.y, 2.0f * c.z};
    Vec3f c2 = cross(qv, t);
    return {(v.x + q[0] * t.x) + c2.x, (v.y + q[0] * t.y) + c2.y, (v.z + q[0] * t.z) + c2.z};
}

// types.ts:35-37
inline int shCoeffs(int bands) { return bands == 0 ? 0 : bands == 1 ? 3 : bands == 2 ? 8 : 15; }

// ---------------------------------------------------------------- camera.ts
struct Basis {
    int projection;  // 0 pinhole, 1 equirect
    float view[16];
    uint32_t width, height;
    double near_, far_;
    double focal, cx, cy;
};

// camera.ts:32-46 (f64 JS numbers)
Basis buildCameraBasis(const orc_camera& c) {
    Basis b;
    b.projection = c.projection;
    std::memcpy(b.view, c.view, sizeof(b.view));
    b.width = c.width;
    b.height = c.height;
    b.near_ = c.near_plane;
    b.far_ = c.far_plane;
    b.focal = (double)c.height / (2.0 * std::tan(c.fov_y / 2.0));
    b.cx = (double)c.width / 2.0;
    b.cy = (double)c.height / 2.0;
    return b;
}

// camera.ts:56-99 — f32 inputs promoted to f64, evaluated left to right; the
// depth is stored into a Float32Array (one rounding).
uint32_t cullToVisible(const float* positions, uint64_t n, const Basis& basis,
                       std::vector<uint32_t>& outIdx, std::vector<float>& outDepth) {
    const float* m = basis.view;
    uint32_t count = 0;
    if (basis.projection == 0) {
        for (uint64_t i = 0; i < n; i++) {
            const double x = positions[i * 3 + 0], y = positions[i * 3 + 1], z = positions[i * 3 + 2];
            const double cz = (double)m[2] * x + (double)m[6] * y + (double)m[10] * z + (double)m[14];
            const double depth = -cz;
            if (depth > basis.near_ && depth < basis.far_) {
                outIdx[count] = (uint32_t)i;
                outDepth[count] = (float)depth;
                count++;
            }
        }
    } else {
        const double nearSq = basis.near_ * basis.near_;
        for (uint64_t i = 0; i < n; i++) {
            const double x = positions[i * 3 + 0], y = positions[i * 3 + 1], z = positions[i * 3 + 2];
            const double cx = (double)m[0] * x + (double)m[4] * y + (double)m[8] * z + (double)m[12];
            const double cy = (double)m[1] * x + (double)m[5] * y + (double)m[9] * z + (double)m[13];
            const double cz = (double)m[2] * x + (double)m[6] * y + (double)m[10] * z + (double)m[14];
            const double r2 = cx * cx + cy * cy + cz * cz;
            if (r2 > nearSq) {
                outIdx[count] = (uint32_t)i;
                outDepth[count] = (float)std::sqrt(r2);
                count++;
            }
        }
    }
    return count;
}

// spatial/radix-sort.ts:65-117 — stable LSD radix sort, 4 passes of 8 bits.
void radixSortIndicesByFloat(std::vector<uint32_t>& indices, const std::vector<float>& depths,
                             uint32_t n, std::vector<uint32_t>& keysOut) {
    keysOut.assign(n, 0);
    if (n <= 1) {
        for (uint32_t i = 0; i < n; i++) keysOut[i] = dl_sortable_key(depths[i]);
        return;
    }
    std::vector<uint32_t> keys(n), idxTmp(n), keyTmp(n);
    for (uint32_t i = 0; i < n; i++) keys[i] = dl_sortable_key(depths[i]);
    uint32_t hist[4 * 256] = {0};
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t k = keys[i];
        hist[k & 0xff]++;
        hist[256 + ((k >> 8) & 0xff)]++;
        hist[512 + ((k >> 16) & 0xff)]++;
        hist[768 + ((k >> 24) & 0xff)]++;
    }
    for (int p = 0; p < 4; p++) {
        uint32_t sum = 0;
        for (int b = 0; b < 256; b++) {
            const uint32_t c = hist[p * 256 + b];
            hist[p * 256 + b] = sum;
            sum += c;
        }
    }
    uint32_t *inIdx = indices.data(), *inKey = keys.data();
    uint32_t *outIdx = idxTmp.data(), *outKey = keyTmp.data();
    for (int p = 0; p < 4; p++) {
        const int shift = p * 8;
        for (uint32_t i = 0; i < n; i++) {
            const uint32_t k = inKey[i];
            const uint32_t b = (k >> shift) & 0xff;
            const uint32_t dst = hist[p * 256 + b]++;
            outIdx[dst] = inIdx[i];
            outKey[dst] = k;
        }
        std::swap(inIdx, outIdx);
        std::swap(inKey, outKey);
    }
    // 4 passes: the result is back in the caller's buffers.
    for (uint32_t i = 0; i < n; i++) keysOut[i] = inKey[i];
}

// preprocess.ts:90-138 — gather into stride 14+3M records.
void packChunkInput(const orc_splats& d, const uint32_t* sortedIdx, uint32_t chunkStart,
                    uint32_t chunkCount, std::vector<float>& out) {
    const int m = shCoeffs(d.sh_bands);
    const int stride = 14 + 3 * m;
    for (uint32_t i = 0; i < chunkCount; i++) {
        const uint64_t g = sortedIdx[chunkStart + i];
        float* o = &out[(size_t)i * stride];
        o[0] = d.positions[g * 3 + 0]; o[1] = d.positions[g * 3 + 1]; o[2] = d.positions[g * 3 + 2];
        o[3] = d.rotations[g * 4 + 0]; o[4] = d.rotations[g * 4 + 1];
        o[5] = d.rotations[g * 4 + 2]; o[6] = d.rotations[g * 4 + 3];
        o[7] = d.log_scales[g * 3 + 0]; o[8] = d.log_scales[g * 3 + 1]; o[9] = d.log_scales[g * 3 + 2];
        o[10] = d.opacity_logits[g];
        o[11] = d.colors_dc[g * 3 + 0]; o[12] = d.colors_dc[g * 3 + 1]; o[13] = d.colors_dc[g * 3 + 2];
        if (d.sh_bands > 0 && d.colors_sh) {
            const uint64_t src = g * 3 * m;
            for (int k = 0; k < 3 * m; k++) o[14 + k] = d.colors_sh[src + k];
        }
    }
}

// project.ts:264-331 evalSH — camera-space direction, channel-major coefficients.
Vec3f evalSH(const float* c, int M, int bands, Vec3f dir) {
    const float x = dir.x, y = dir.y, z = dir.z;
    float r = 0.0f, g = 0.0f, b = 0.0f;
    const float SH1 = 0.4886025119029199f;
    const float nSH1 = -SH1;
    r = r + (nSH1 * y) * c[0];
    r = r + (SH1 * z) * c[1];
    r = r + (nSH1 * x) * c[2];
    g = g + (nSH1 * y) * c[M + 0];
    g = g + (SH1 * z) * c[M + 1];
    g = g + (nSH1 * x) * c[M + 2];
    b = b + (nSH1 * y) * c[2 * M + 0];
    b = b + (SH1 * z) * c[2 * M + 1];
    b = b + (nSH1 * x) * c[2 * M + 2];
    if (bands >= 2) {
        const float xx = x * x, yy = y * y, zz = z * z;
        const float xy = x * y, yz = y * z, xz = x * z;
        const float SH2_0 = 1.0925484305920792f, SH2_1 = -1.0925484305920792f;
        const float SH2_2 = 0.31539156525252005f, SH2_3 = -1.0925484305920792f;
        const float SH2_4 = 0.5462742152960396f;
        const float band2[5] = {SH2_0 * xy, SH2_1 * yz, SH2_2 * (((2.0f * zz) - xx) - yy),
                                SH2_3 * xz, SH2_4 * (xx - yy)};
        for (int k = 0; k < 5; k++) {
            r = r + band2[k] * c[3 + k];
            g = g + band2[k] * c[M + 3 + k];
            b = b + band2[k] * c[2 * M + 3 + k];
        }
        if (bands >= 3) {
            const float SH3_0 = -0.5900435899266435f, SH3_1 = 2.890611442640554f;
            const float SH3_2 = -0.4570457994644658f, SH3_3 = 0.3731763325901154f;
            const float SH3_4 = -0.4570457994644658f, SH3_5 = 1.445305721320277f;
            const float SH3_6 = -0.5900435899266435f;
            const float band3[7] = {
                (SH3_0 * y) * ((3.0f * xx) - yy),
                (SH3_1 * xy) * z,
                (SH3_2 * y) * (((4.0f * zz) - xx) - yy),
                (SH3_3 * z) * (((2.0f * zz) - (3.0f * xx)) - (3.0f * yy)),
                (SH3_4 * x) * (((4.0f * zz) - xx) - yy),
                (SH3_5 * z) * (xx - yy),
                (SH3_6 * x) * (xx - (3.0f * yy))};
            for (int k = 0; k < 7; k++) {
                r = r + band3[k] * c[8 + k];
                g = g + band3[k] * c[M + 8 + k];
                b = b + band3[k] * c[2 * M + 8 + k];
            }
        }
    }
    return {r, g, b};
}

struct ProjUniforms {
    float view[16];
    float width, height, focal, cx, cy, near_, far_;
    uint32_t tilesX, tilesY, maxCoverage;
    int bands, projection;
};

// project.ts:59-234 (+ pinhole :237-249, equirect :251-262) for one splat.
// Writes 12 floats (3 vec4) and returns the tile count.
uint32_t projectOne(const ProjUniforms& u, const float* in, int M, float* proj) {
    const float* V = u.view;
    const float pos[3] = {in[0], in[1], in[2]};
    const float rot[4] = {in[3], in[4], in[5], in[6]};
    const float logScale[3] = {in[7], in[8], in[9]};
    const float opacityLogit = in[10];
    const float dc[3] = {in[11], in[12], in[13]};
    const float scale[3] = {dl_expf(logScale[0]), dl_expf(logScale[1]), dl_expf(logScale[2])};

    // posCam4 = viewMatrix * vec4(pos, 1)  (column-major, columns summed in order)
    Vec3f posCam;
    posCam.x = ((V[0] * pos[0] + V[4] * pos[1]) + V[8] * pos[2]) + V[12] * 1.0f;
    posCam.y = ((V[1] * pos[0] + V[5] * pos[1]) + V[9] * pos[2]) + V[13] * 1.0f;
    posCam.z = ((V[2] * pos[0] + V[6] * pos[1]) + V[10] * pos[2]) + V[14] * 1.0f;
    const float depth = -posCam.z;

    auto cull = [&]() -> uint32_t {
        proj[0] = 0.0f; proj[1] = 0.0f; proj[2] = -1.0f; proj[3] = 0.0f;
        return 0u;
    };

    float screenX, screenY;
    if (u.projection == 0) {
        if (depth <= u.near_ || depth >= u.far_) return cull();
        const float projX = (posCam.x * u.focal) / -posCam.z;
        const float projY = (-posCam.y * u.focal) / -posCam.z;
        screenX = projX + u.cx;
        screenY = projY + u.cy;
    } else {
        const float r = std::sqrt((posCam.x * posCam.x + posCam.y * posCam.y) + posCam.z * posCam.z);
        if (r <= u.near_) return cull();
        const float lon = dl_atan2f(posCam.x, -posCam.z);
        const float lat = dl_asinf(posCam.y / r);
        screenX = (lon / (3.14159265f * 2.0f) + 0.5f) * u.width;
        screenY = (0.5f - lat / 3.14159265f) * u.height;
    }

    const float* s = scale;
    Vec3f rx = quatRot(rot, {1.0f, 0.0f, 0.0f}); rx = {rx.x * s[0], rx.y * s[0], rx.z * s[0]};
    Vec3f ry = quatRot(rot, {0.0f, 1.0f, 0.0f}); ry = {ry.x * s[1], ry.y * s[1], ry.z * s[1]};
    Vec3f rz = quatRot(rot, {0.0f, 0.0f, 1.0f}); rz = {rz.x * s[2], rz.y * s[2], rz.z * s[2]};
    const float cov3_00 = (rx.x * rx.x + ry.x * ry.x) + rz.x * rz.x;
    const float cov3_01 = (rx.x * rx.y + ry.x * ry.y) + rz.x * rz.y;
    const float cov3_02 = (rx.x * rx.z + ry.x * ry.z) + rz.x * rz.z;
    const float cov3_11 = (rx.y * rx.y + ry.y * ry.y) + rz.y * rz.y;
    const float cov3_12 = (rx.y * rx.z + ry.y * ry.z) + rz.y * rz.z;
    const float cov3_22 = (rx.z * rx.z + ry.z * ry.z) + rz.z * rz.z;

    const float v00 = V[0], v01 = V[4], v02 = V[8];
    const float v10 = V[1], v11 = V[5], v12 = V[9];
    const float v20 = V[2], v21 = V[6], v22 = V[10];
    const float a00 = (v00 * cov3_00 + v01 * cov3_01) + v02 * cov3_02;
    const float a01 = (v00 * cov3_01 + v01 * cov3_11) + v02 * cov3_12;
    const float a02 = (v00 * cov3_02 + v01 * cov3_12) + v02 * cov3_22;
    const float a10 = (v10 * cov3_00 + v11 * cov3_01) + v12 * cov3_02;
    const float a11 = (v10 * cov3_01 + v11 * cov3_11) + v12 * cov3_12;
    const float a12 = (v10 * cov3_02 + v11 * cov3_12) + v12 * cov3_22;
    const float a20 = (v20 * cov3_00 + v21 * cov3_01) + v22 * cov3_02;
    const float a21 = (v20 * cov3_01 + v21 * cov3_11) + v22 * cov3_12;
    const float a22 = (v20 * cov3_02 + v21 * cov3_12) + v22 * cov3_22;
    const float cc00 = (a00 * v00 + a01 * v01) + a02 * v02;
    const float cc01 = (a00 * v10 + a01 * v11) + a02 * v12;
    const float cc02 = (a00 * v20 + a01 * v21) + a02 * v22;
    const float cc11 = (a10 * v10 + a11 * v11) + a12 * v12;
    const float cc12 = (a10 * v20 + a11 * v21) + a12 * v22;
    const float cc22 = (a20 * v20 + a21 * v21) + a22 * v22;

    // project.ts:128-149 — J uses invZ = 1/z with z = posCam.z (kept as written).
    const float z = posCam.z;
    const float invZ = 1.0f / z;
    const float j00 = u.focal * invZ;
    const float j02 = ((-u.focal * posCam.x) * invZ) * invZ;
    const float j11 = u.focal * invZ;
    const float j12 = ((-u.focal * posCam.y) * invZ) * invZ;
    const float b00 = j00 * cc00 + j02 * cc02;
    const float b01 = j00 * cc01 + j02 * cc12;
    const float b02 = j00 * cc02 + j02 * cc22;
    const float b10 = j11 * cc01 + j12 * cc02;   // computed but unused, as in the shader
    const float b11 = j11 * cc11 + j12 * cc12;
    const float b12 = j11 * cc12 + j12 * cc22;
    (void)b10;
    float cov2_00 = b00 * j00 + b02 * j02;
    float cov2_01 = b01 * j11 + b02 * j12;
    float cov2_11 = b11 * j11 + b12 * j12;

    // project.ts:157-173
    const float detOrig = cov2_00 * cov2_11 - cov2_01 * cov2_01;
    cov2_00 = cov2_00 + AA_DILATION_COV;
    cov2_11 = cov2_11 + AA_DILATION_COV;
    const float detBlur = cov2_00 * cov2_11 - cov2_01 * cov2_01;
    const float aaFactor = std::sqrt(std::max(detOrig / detBlur, 0.0f));
    const float det = detBlur;
    if (det <= 1.0e-6f) return cull();
    const float invDet = 1.0f / det;
    const float conicA = cov2_11 * invDet;
    const float conicB = -cov2_01 * invDet;
    const float conicC = cov2_00 * invDet;

    // project.ts:180-201
    const float mid = 0.5f * (cov2_00 + cov2_11);
    const float radiusEig = std::sqrt(std::max(0.1f, mid * mid - det));
    const float lambda1 = mid + radiusEig;
    const float radiusRaw = SIGMA_CUTOFF * std::sqrt(lambda1);
    const float fadeStart = RADIUS_FADE_START_FRAC * u.height;
    const float fadeEnd = RADIUS_FADE_END_FRAC * u.height;
    const float radiusFade = std::min(std::max((fadeEnd - radiusRaw) / (fadeEnd - fadeStart), 0.0f), 1.0f);
    if (radiusFade <= 0.0f) return cull();
    const float radius = std::ceil(std::min(radiusRaw, fadeEnd));

    // project.ts:204-217
    float color[3] = {dc[0], dc[1], dc[2]};
    if (u.bands > 0) {
        const float len = std::sqrt((posCam.x * posCam.x + posCam.y * posCam.y) + posCam.z * posCam.z);
        const Vec3f viewDir{posCam.x / len, posCam.y / len, posCam.z / len};
        const Vec3f sh = evalSH(in + 14, M, u.bands, viewDir);
        color[0] = color[0] + sh.x; color[1] = color[1] + sh.y; color[2] = color[2] + sh.z;
    }
    for (int k = 0; k < 3; k++) color[k] = std::max(color[k] + 0.5f, 0.0f);
    const float alpha = (dl_sigmoidf(opacityLogit) * radiusFade) * aaFactor;

    proj[0] = screenX; proj[1] = screenY; proj[2] = radius; proj[3] = depth;
    proj[4] = conicA; proj[5] = conicB; proj[6] = conicC; proj[7] = alpha;
    proj[8] = color[0]; proj[9] = color[1]; proj[10] = color[2]; proj[11] = 0.0f;

    // project.ts:224-233
    const uint32_t minTileX = dl_sat_u32(std::max(0.0f, std::floor((screenX - radius) / 16.0f)));
    const uint32_t minTileY = dl_sat_u32(std::max(0.0f, std::floor((screenY - radius) / 16.0f)));
    const uint32_t maxTileX = dl_sat_u32(std::min((float)u.tilesX - 1.0f, std::floor((screenX + radius) / 16.0f)));
    const uint32_t maxTileY = dl_sat_u32(std::min((float)u.tilesY - 1.0f, std::floor((screenY + radius) / 16.0f)));
    uint32_t count = 0;
    if (maxTileX >= minTileX && maxTileY >= minTileY) {
        count = (maxTileX - minTileX + 1u) * (maxTileY - minTileY + 1u);
        if (count > u.maxCoverage) count = u.maxCoverage;
    }
    return count;
}

// emit-pairs.ts:28-57
void emitPairs(const float* projected, const uint32_t* offsets, uint32_t n, uint32_t tilesX,
               uint32_t tilesY, uint32_t maxCoverage, uint32_t* pairTiles, uint32_t* pairSplats) {
    for (uint32_t idx = 0; idx < n; idx++) {
        const float* v0 = projected + (size_t)idx * 12;
        const float screenX = v0[0], screenY = v0[1], radius = v0[2];
        if (radius <= 0.0f) continue;
        const uint32_t minTileX = dl_sat_u32(std::max(0.0f, std::floor((screenX - radius) / 16.0f)));
        const uint32_t minTileY = dl_sat_u32(std::max(0.0f, std::floor((screenY - radius) / 16.0f)));
        const uint32_t maxTileX = dl_sat_u32(std::min((float)tilesX - 1.0f, std::floor((screenX + radius) / 16.0f)));
        const uint32_t maxTileY = dl_sat_u32(std::min((float)tilesY - 1.0f, std::floor((screenY + radius) / 16.0f)));
        if (maxTileX < minTileX || maxTileY < minTileY) continue;
        uint32_t offset = offsets[idx];
        uint32_t written = 0;
        for (uint32_t ty = minTileY; ty <= maxTileY; ty++) {
            for (uint32_t tx = minTileX; tx <= maxTileX; tx++) {
                if (written >= maxCoverage) goto done;
                pairTiles[offset] = ty * tilesX + tx;
                pairSplats[offset] = idx;
                offset++;
                written++;
            }
        }
    done:;
    }
}

// pipeline.ts:544-578 cpuSortPairs — stable counting sort by tile id.
void cpuSortPairs(std::vector<uint32_t>& tiles, std::vector<uint32_t>& splats, uint32_t n) {
    if (n <= 1) return;
    uint32_t maxT = 0;
    for (uint32_t i = 0; i < n; i++) maxT = std::max(maxT, tiles[i]);
    std::vector<uint32_t> counts((size_t)maxT + 1, 0);
    for (uint32_t i = 0; i < n; i++) counts[tiles[i]]++;
    uint32_t sum = 0;
    for (auto& c : counts) { const uint32_t v = c; c = sum; sum += v; }
    std::vector<uint32_t> tOut(n), sOut(n);
    for (uint32_t i = 0; i < n; i++) {
        const uint32_t t = tiles[i];
        const uint32_t dst = counts[t]++;
        tOut[dst] = t;
        sOut[dst] = splats[i];
    }
    tiles.swap(tOut);
    splats.swap(sOut);
}

// find-boundaries.ts:17-99 — init to 0xffffffff, atomicMin at run starts,
// then the right-to-left fill.  (Sequential equivalent of the three kernels.)
void findBoundaries(const uint32_t* pairTiles, uint32_t numPairs, uint32_t numTiles, uint32_t* off) {
    for (uint32_t i = 0; i <= numTiles; i++) off[i] = 0xffffffffu;
    for (uint32_t i = 0; i < numPairs; i++) {
        const uint32_t cur = pairTiles[i];
        if (i == 0) {
            off[cur] = std::min(off[cur], 0u);
        } else {
            const uint32_t prev = pairTiles[i - 1];
            if (cur != prev)
                for (uint32_t t = prev + 1; t <= cur; t++) off[t] = std::min(off[t], i);
        }
    }
    off[numTiles] = numPairs;
    uint32_t fill = numPairs;
    uint32_t i = numTiles;
    while (i != 0) {
        i--;
        if (off[i] == 0xffffffffu) off[i] = fill; else fill = off[i];
    }
}

// rasterize.ts:36-82 — one pixel; accum is (r, g, b, T) resumed across chunks.
// Returns the number of slice entries examined (up to the T-break).
template <typename T>
uint32_t rasterPixel(const T* projected, const uint32_t* pairSplats, uint32_t sliceStart,
                     uint32_t sliceEnd, uint32_t pixelX, uint32_t pixelY, T* accum, uint32_t* evals) {
    const T px = (T)pixelX + (T)0.5;
    const T py = (T)pixelY + (T)0.5;
    T color[3] = {accum[0], accum[1], accum[2]};
    T Tr = accum[3];
    uint32_t examined = 0, evaluated = 0;
    if (Tr < (T)MIN_TRANSMITTANCE) return 0;
    for (uint32_t i = sliceStart; i < sliceEnd; i++) {
        if (Tr < (T)MIN_TRANSMITTANCE) break;
        examined++;
        const uint32_t s = pairSplats[i];
        const T* v0 = projected + (size_t)s * 12;
        const T dx = px - v0[0];
        const T dy = py - v0[1];
        const T r = v0[2];
        if (r <= (T)0 || std::abs(dx) > r || std::abs(dy) > r) continue;
        evaluated++;
        const T* v1 = v0 + 4;
        const T power = (T)-0.5 * (((v1[0] * dx) * dx + (((T)2.0 * v1[1]) * dx) * dy) + (v1[2] * dy) * dy);
        if (power > (T)0) continue;
        T e;
        if constexpr (sizeof(T) == 4) e = dl_expf(power); else e = dl_exp(power);
        const T alpha = std::min((T)OPACITY_CAP, v1[3] * std::max((T)0, e - (T)GAUSSIAN_FLOOR));
        if (alpha < (T)MIN_ALPHA) continue;
        const T weight = Tr * alpha;
        const T* v2 = v0 + 8;
        color[0] = color[0] + weight * v2[0];
        color[1] = color[1] + weight * v2[1];
        color[2] = color[2] + weight * v2[2];
        Tr = Tr * ((T)1 - alpha);
    }
    accum[0] = color[0]; accum[1] = color[1]; accum[2] = color[2]; accum[3] = Tr;
    if (evals) *evals += evaluated;
    return examined;
}

// finalize.ts:30-43
inline uint32_t finalizePixel(const float* v, const float bg[4]) {
    float rgb[3];
    for (int k = 0; k < 3; k++) rgb[k] = std::min(std::max(v[k] + v[3] * bg[k], 0.0f), 1.0f);
    const float aOut = std::min(std::max((1.0f - v[3]) + v[3] * bg[3], 0.0f), 1.0f);
    const uint32_t r = dl_sat_u32(rgb[0] * 255.0f + 0.5f);
    const uint32_t g = dl_sat_u32(rgb[1] * 255.0f + 0.5f);
    const uint32_t b = dl_sat_u32(rgb[2] * 255.0f + 0.5f);
    const uint32_t a = dl_sat_u32(aOut * 255.0f + 0.5f);
    return r | (g << 8) | (b << 16) | (a << 24);
}

// f64 restatement of projectOne's float outputs for the error reference.  The
// integer decisions (cull, radius, tile ranges) are taken from the f32 pass;
// only conic, alpha and colour are recomputed in double.
void projectOneF64(const ProjUniforms& u, const orc_camera& cam, const float* in, int M, double* out) {
    const double V[16] = {cam.view[0], cam.view[1], cam.view[2], cam.view[3], cam.view[4], cam.view[5],
                          cam.view[6], cam.view[7], cam.view[8], cam.view[9], cam.view[10], cam.view[11],
                          cam.view[12], cam.view[13], cam.view[14], cam.view[15]};
    const double focal = (double)cam.height / (2.0 * std::tan(cam.fov_y / 2.0));
    const double p[3] = {in[0], in[1], in[2]};
    const double w = in[3], qx = in[4], qy = in[5], qz = in[6];
    const double s[3] = {dl_exp(in[7]), dl_exp(in[8]), dl_exp(in[9])};
    const double pc[3] = {V[0] * p[0] + V[4] * p[1] + V[8] * p[2] + V[12],
                          V[1] * p[0] + V[5] * p[1] + V[9] * p[2] + V[13],
                          V[2] * p[0] + V[6] * p[1] + V[10] * p[2] + V[14]};
    // rotation matrix columns R e_j (Rodrigues, exact algebra)
    double R[3][3];
    for (int j = 0; j < 3; j++) {
        double v[3] = {0, 0, 0}; v[j] = 1;
        const double c[3] = {qy * v[2] - qz * v[1], qz * v[0] - qx * v[2], qx * v[1] - qy * v[0]};
        const double t[3] = {2 * c[0], 2 * c[1], 2 * c[2]};
        const double c2[3] = {qy * t[2] - qz * t[1], qz * t[0] - qx * t[2], qx * t[1] - qy * t[0]};
        for (int i = 0; i < 3; i++) R[i][j] = (v[i] + w * t[i] + c2[i]) * s[j];
    }
    double S[3][3];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) S[i][k] = R[i][0] * R[k][0] + R[i][1] * R[k][1] + R[i][2] * R[k][2];
    double W[3][3] = {{V[0], V[4], V[8]}, {V[1], V[5], V[9]}, {V[2], V[6], V[10]}};
    double A[3][3], C[3][3];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) A[i][k] = W[i][0] * S[0][k] + W[i][1] * S[1][k] + W[i][2] * S[2][k];
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) C[i][k] = A[i][0] * W[k][0] + A[i][1] * W[k][1] + A[i][2] * W[k][2];
    const double invZ = 1.0 / pc[2];
    const double j00 = focal * invZ, j02 = -focal * pc[0] * invZ * invZ;
    const double j11 = focal * invZ, j12 = -focal * pc[1] * invZ * invZ;
    const double b00 = j00 * C[0][0] + j02 * C[0][2], b01 = j00 * C[0][1] + j02 * C[1][2];
    const double b02 = j00 * C[0][2] + j02 * C[2][2];
    const double b11 = j11 * C[1][1] + j12 * C[1][2], b12 = j11 * C[1][2] + j12 * C[2][2];
    double c00 = b00 * j00 + b02 * j02, c01 = b01 * j11 + b02 * j12, c11 = b11 * j11 + b12 * j12;
    const double detOrig = c00 * c11 - c01 * c01;
    c00 += 0.3; c11 += 0.3;
    const double det = c00 * c11 - c01 * c01;
    const double aa = std::sqrt(std::max(detOrig / det, 0.0));
    const double mid = 0.5 * (c00 + c11);
    const double lam = mid + std::sqrt(std::max(0.1, mid * mid - det));
    const double rr = 3.0 * std::sqrt(lam);
    const double fs = (1024.0 / 1080.0) * cam.height, fe = (2048.0 / 1080.0) * cam.height;
    const double fade = std::min(std::max((fe - rr) / (fe - fs), 0.0), 1.0);
    double col[3] = {in[11], in[12], in[13]};
    if (u.bands > 0) {
        const double len = std::sqrt(pc[0] * pc[0] + pc[1] * pc[1] + pc[2] * pc[2]);
        const double x = pc[0] / len, y = pc[1] / len, z = pc[2] / len;
        const float* c = in + 14;
        const double SH1 = 0.4886025119029199;
        double basis[15];
        basis[0] = -SH1 * y; basis[1] = SH1 * z; basis[2] = -SH1 * x;
        const double xx = x * x, yy = y * y, zz = z * z;
        basis[3] = 1.0925484305920792 * x * y; basis[4] = -1.0925484305920792 * y * z;
        basis[5] = 0.31539156525252005 * (2 * zz - xx - yy); basis[6] = -1.0925484305920792 * x * z;
        basis[7] = 0.5462742152960396 * (xx - yy);
        basis[8] = -0.5900435899266435 * y * (3 * xx - yy); basis[9] = 2.890611442640554 * x * y * z;
        basis[10] = -0.4570457994644658 * y * (4 * zz - xx - yy);
        basis[11] = 0.3731763325901154 * z * (2 * zz - 3 * xx - 3 * yy);
        basis[12] = -0.4570457994644658 * x * (4 * zz - xx - yy);
        basis[13] = 1.445305721320277 * z * (xx - yy); basis[14] = -0.5900435899266435 * x * (xx - 3 * yy);
        for (int k = 0; k < M; k++) {
            col[0] += basis[k] * c[k]; col[1] += basis[k] * c[M + k]; col[2] += basis[k] * c[2 * M + k];
        }
    }
    for (int k = 0; k < 3; k++) col[k] = std::max(col[k] + 0.5, 0.0);
    const double alpha = (1.0 / (1.0 + dl_exp(-(double)in[10]))) * fade * aa;
    out[4] = c11 / det; out[5] = -c01 / det; out[6] = c00 / det; out[7] = alpha;
    out[8] = col[0]; out[9] = col[1]; out[10] = col[2]; out[11] = 0;
}

}  // namespace

// ---------------------------------------------------------------- driver
// pipeline.ts:181-473 (Renderer.render + composite), chunk loop included.
struct OrcRender {
    uint32_t width = 0, height = 0, tilesX = 0, tilesY = 0, numTiles = 0;
    uint32_t numVisible = 0;
    uint64_t numPairsTotal = 0;
    std::vector<uint32_t> sortedIdx, depthKeys;   // rank order
    std::vector<float> records;                   // rank order, 12 floats
    std::vector<uint32_t> counts, offsets;        // rank order (offsets chunk-local)
    std::vector<uint32_t> tileListOff, tileListVal;   // canonical per-tile rank lists
    std::vector<uint32_t> chunkTileOffsets;       // last chunk's tileOffsets (T+1)
    std::vector<float> accum;                     // W*H*4
    std::vector<double> accum64;                  // f64 error reference (optional)
    std::vector<uint32_t> rgba;                   // W*H packed
    std::vector<uint32_t> tileExamined, tileEvaluated;   // per tile, summed over pixels
};

extern "C" void* orc_render_run(const orc_splats* data, const orc_camera* cam, uint32_t maxCoverage,
                                uint32_t chunkCap, const float bg[4], int withF64) {
    OrcRender* R = new OrcRender();
    const Basis basis = buildCameraBasis(*cam);
    const int bands = data->sh_bands;
    const int M = shCoeffs(bands);
    const int stride = 14 + 3 * M;
    R->width = cam->width; R->height = cam->height;
    R->tilesX = (cam->width + TILE_SIZE - 1) / TILE_SIZE;
    R->tilesY = (cam->height + TILE_SIZE - 1) / TILE_SIZE;
    R->numTiles = R->tilesX * R->tilesY;
    const size_t pixels = (size_t)cam->width * cam->height;
    const uint64_t n = data->count;

    // 1. CPU cull + sort (preprocess.ts:60-78)
    std::vector<uint32_t> idx(n);
    std::vector<float> depths(n);
    const uint32_t numVisible = cullToVisible(data->positions, n, basis, idx, depths);
    R->numVisible = numVisible;
    radixSortIndicesByFloat(idx, depths, numVisible, R->depthKeys);
    R->sortedIdx.assign(idx.begin(), idx.begin() + numVisible);

    // accum init (0,0,0,1) — pipeline.ts:203-208
    R->accum.assign(pixels * 4, 0.0f);
    for (size_t p = 0; p < pixels; p++) R->accum[p * 4 + 3] = 1.0f;
    if (withF64) {
        R->accum64.assign(pixels * 4, 0.0);
        for (size_t p = 0; p < pixels; p++) R->accum64[p * 4 + 3] = 1.0;
    }
    R->records.assign((size_t)numVisible * 12, 0.0f);
    R->counts.assign(numVisible, 0);
    R->offsets.assign(numVisible, 0);
    R->tileExamined.assign(R->numTiles, 0);
    R->tileEvaluated.assign(R->numTiles, 0);
    std::vector<std::vector<uint32_t>> tileLists(R->numTiles);

    if (numVisible > 0) {
        const uint32_t cap = std::min(chunkCap == 0 ? 200000u : chunkCap, numVisible);
        ProjUniforms u;
        std::memcpy(u.view, cam->view, sizeof(u.view));
        u.width = (float)cam->width; u.height = (float)cam->height;
        u.focal = (float)basis.focal; u.cx = (float)basis.cx; u.cy = (float)basis.cy;
        u.near_ = (float)cam->near_plane; u.far_ = (float)cam->far_plane;
        u.tilesX = R->tilesX; u.tilesY = R->tilesY; u.maxCoverage = maxCoverage;
        u.bands = bands; u.projection = cam->projection;
        std::vector<float> staging((size_t)stride * cap);
        std::vector<double> proj64;
        for (uint32_t chunkStart = 0; chunkStart < numVisible; chunkStart += cap) {
            const uint32_t chunkCount = std::min(cap, numVisible - chunkStart);
            packChunkInput(*data, R->sortedIdx.data(), chunkStart, chunkCount, staging);
            float* proj = &R->records[(size_t)chunkStart * 12];
            uint32_t* tc = &R->counts[chunkStart];
            #pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < (int64_t)chunkCount; i++)
                tc[i] = projectOne(u, &staging[(size_t)i * stride], M, proj + (size_t)i * 12);
            // prefix-sum.ts + pipeline.ts:277-286: exclusive scan, numPairs = total
            uint32_t* off = &R->offsets[chunkStart];
            uint32_t sum = 0;
            for (uint32_t i = 0; i < chunkCount; i++) { off[i] = sum; sum += tc[i]; }
            const uint32_t numPairs = sum;
            R->numPairsTotal += numPairs;
            if (numPairs == 0) continue;
            std::vector<uint32_t> pairTiles(numPairs), pairSplats(numPairs);
            emitPairs(proj, off, chunkCount, R->tilesX, R->tilesY, maxCoverage, pairTiles.data(), pairSplats.data());
            cpuSortPairs(pairTiles, pairSplats, numPairs);
            R->chunkTileOffsets.assign(R->numTiles + 1, 0);
            findBoundaries(pairTiles.data(), numPairs, R->numTiles, R->chunkTileOffsets.data());
            const uint32_t* to = R->chunkTileOffsets.data();
            for (uint32_t t = 0; t < R->numTiles; t++)
                for (uint32_t i = to[t]; i < to[t + 1]; i++) tileLists[t].push_back(pairSplats[i] + chunkStart);
            if (withF64) {
                proj64.assign((size_t)chunkCount * 12, 0.0);
                #pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < (int64_t)chunkCount; i++) {
                    double* o = &proj64[(size_t)i * 12];
                    const float* p32 = proj + (size_t)i * 12;
                    for (int k = 0; k < 4; k++) o[k] = p32[k];
                    if (p32[2] > 0.0f) projectOneF64(u, *cam, &staging[(size_t)i * stride], M, o);
                }
            }
            // rasterize.ts — workgroup per tile, thread per pixel
            #pragma omp parallel for schedule(dynamic, 4)
            for (int64_t t = 0; t < (int64_t)R->numTiles; t++) {
                const uint32_t tx = (uint32_t)t % R->tilesX, ty = (uint32_t)t / R->tilesX;
                uint32_t ex = 0, ev = 0;
                for (uint32_t ly = 0; ly < TILE_SIZE; ly++) {
                    for (uint32_t lx = 0; lx < TILE_SIZE; lx++) {
                        const uint32_t x = tx * TILE_SIZE + lx, y = ty * TILE_SIZE + ly;
                        if (x >= cam->width || y >= cam->height) continue;
                        const size_t p = (size_t)y * cam->width + x;
                        ex += rasterPixel<float>(proj, pairSplats.data(), to[t], to[t + 1], x, y, &R->accum[p * 4], &ev);
                        if (withF64)
                            rasterPixel<double>(proj64.data(), pairSplats.data(), to[t], to[t + 1], x, y,
                                                &R->accum64[p * 4], nullptr);
                    }
                }
                R->tileExamined[t] += ex;
                R->tileEvaluated[t] += ev;
            }
        }
    }
    // canonical per-tile rank lists
    R->tileListOff.assign(R->numTiles + 1, 0);
    for (uint32_t t = 0; t < R->numTiles; t++) R->tileListOff[t + 1] = R->tileListOff[t] + (uint32_t)tileLists[t].size();
    R->tileListVal.reserve(R->tileListOff[R->numTiles]);
    for (auto& l : tileLists) R->tileListVal.insert(R->tileListVal.end(), l.begin(), l.end());
    // composite (pipeline.ts:428-473, finalize.ts)
    R->rgba.assign(pixels, 0);
    #pragma omp parallel for schedule(static)
    for (int64_t p = 0; p < (int64_t)pixels; p++) R->rgba[p] = finalizePixel(&R->accum[p * 4], bg);
    return R;
}

// Copy a named result into dst (capacity cap bytes).  Returns the byte size of
// the result, or -1 for an unknown name.  Nothing is copied when cap is too small.
extern "C" int64_t orc_render_get(void* h, const char* name, void* dst, int64_t cap) {
    OrcRender* R = (OrcRender*)h;
    const void* src = nullptr;
    int64_t bytes = -1;
    uint64_t scalar = 0;
    auto vec = [&](const auto& v) { src = v.data(); bytes = (int64_t)(v.size() * sizeof(v[0])); };
    const std::string s(name);
    if (s == "rgba") vec(R->rgba);
    else if (s == "accum") vec(R->accum);
    else if (s == "accum64") vec(R->accum64);
    else if (s == "sorted_idx") vec(R->sortedIdx);
    else if (s == "depth_keys") vec(R->depthKeys);
    else if (s == "records") vec(R->records);
    else if (s == "counts") vec(R->counts);
    else if (s == "offsets") vec(R->offsets);
    else if (s == "tile_list_off") vec(R->tileListOff);
    else if (s == "tile_list_val") vec(R->tileListVal);
    else if (s == "chunk_tile_offsets") vec(R->chunkTileOffsets);
    else if (s == "tile_examined") vec(R->tileExamined);
    else if (s == "tile_evaluated") vec(R->tileEvaluated);
    else if (s == "n_visible") { scalar = R->numVisible; src = &scalar; bytes = 8; }
    else if (s == "n_pairs") { scalar = R->numPairsTotal; src = &scalar; bytes = 8; }
    else return -1;
    if (dst && cap >= bytes && bytes > 0) std::memcpy(dst, src, (size_t)bytes);
    return bytes;
}

extern "C" void orc_render_free(void* h) { delete (OrcRender*)h; }

// Elementwise access to dl_math.h for the CPU tests (op: 0 expf, 1 atan2f(y=in, x=in2), 2 asinf,
// 3 sortable key (bits out), 4 exp f64 on in (as f64 array)).
extern "C" void orc_math(int op, const void* in, const void* in2, void* out, int64_t n) {
    for (int64_t i = 0; i < n; i++) {
        if (op == 0) ((float*)out)[i] = dl_expf(((const float*)in)[i]);
        else if (op == 1) ((float*)out)[i] = dl_atan2f(((const float*)in)[i], ((const float*)in2)[i]);
        else if (op == 2) ((float*)out)[i] = dl_asinf(((const float*)in)[i]);
        else if (op == 3) ((uint32_t*)out)[i] = dl_sortable_key(((const float*)in)[i]);
        else if (op == 4) ((double*)out)[i] = dl_exp(((const double*)in)[i]);
    }
}

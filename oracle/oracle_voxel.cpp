// ORACLE — test infrastructure only.  CPU restatement of droplet's voxelizer
// (src/voxel/voxelize.ts, src/spatial/aabb.ts, src/spatial/bvh.ts,
// src/voxel/shaders/voxelize.ts, src/voxel/block-mask-buffer.ts).  Used by
// tests/ and bench.py's cpu_baseline leg as the checker; the product never
// links or calls it.
//
// Parity unpinned: the reference publishes no numeric voxel outputs and cannot
// run here (WebGPU); the restatement is checked by the ported qualitative
// checks and by closed-form known answers (tests/golden/kat.json).
//
// Two summation orders are offered for the per-voxel density sum:
//   order 0 (canonical): the Gaussians of a batch list in ascending index;
//   order 1 (reference): the batch list in the reference's BVH query order
//            (a statement-by-statement port of bvh.ts).
// The list MEMBERSHIP is the reference's in both (a Gaussian belongs to a
// 16^3-block batch iff its f64 AABB overlaps the batch box, bvh.ts:153-168),
// so the two orders differ only by floating-point summation order.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {

// JS Math.round: round half toward +infinity.
double jsRound(double x) {
    if (!std::isfinite(x)) return x;
    const double f = std::floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

// aabb.ts:22-62 — f64 arithmetic on f32 inputs, result stored as f32.
void computeAabbExtents(const orc_splats& d, std::vector<float>& out) {
    const uint64_t n = d.count;
    out.assign(n * 3, 0.0f);
    for (uint64_t i = 0; i < n; i++) {
        const double qw = d.rotations[i * 4 + 0], qx = d.rotations[i * 4 + 1];
        const double qy = d.rotations[i * 4 + 2], qz = d.rotations[i * 4 + 3];
        const double sx = dl_exp(d.log_scales[i * 3 + 0]);
        const double sy = dl_exp(d.log_scales[i * 3 + 1]);
        const double sz = dl_exp(d.log_scales[i * 3 + 2]);
        const double xx = qx * qx, yy = qy * qy, zz = qz * qz;
        const double xy = qx * qy, xz = qx * qz, yz = qy * qz;
        const double wx = qw * qx, wy = qw * qy, wz = qw * qz;
        const double r00 = 1 - 2 * (yy + zz), r01 = 2 * (xy - wz), r02 = 2 * (xz + wy);
        const double r10 = 2 * (xy + wz), r11 = 1 - 2 * (xx + zz), r12 = 2 * (yz - wx);
        const double r20 = 2 * (xz - wy), r21 = 2 * (yz + wx), r22 = 1 - 2 * (xx + yy);
        auto sq = [](double v) { return v * v; };
        const double ex = std::sqrt(sq(r00 * sx) + sq(r01 * sy) + sq(r02 * sz)) * 3.0;
        const double ey = std::sqrt(sq(r10 * sx) + sq(r11 * sy) + sq(r12 * sz)) * 3.0;
        const double ez = std::sqrt(sq(r20 * sx) + sq(r21 * sy) + sq(r22 * sz)) * 3.0;
        out[i * 3 + 0] = (float)ex;
        out[i * 3 + 1] = (float)ey;
        out[i * 3 + 2] = (float)ez;
    }
}

// voxelize.ts:278-306
void computeBlockAlignedBounds(const orc_splats& d, const std::vector<float>& e, double bs, double b[6]) {
    const double inf = INFINITY;
    double mn[3] = {inf, inf, inf}, mx[3] = {-inf, -inf, -inf};
    for (uint64_t i = 0; i < d.count; i++) {
        for (int a = 0; a < 3; a++) {
            const double p = d.positions[i * 3 + a], ex = e[i * 3 + a];
            if (p - ex < mn[a]) mn[a] = p - ex;
            if (p + ex > mx[a]) mx[a] = p + ex;
        }
    }
    for (int a = 0; a < 3; a++) {
        b[a] = std::floor(mn[a] / bs) * bs;
        b[3 + a] = std::ceil(mx[a] / bs) * bs;
    }
}

// bvh.ts:33-183 — median-split BVH, statement by statement.
struct BVH {
    struct Node { double mn[3], mx[3]; int start, end, left, right; };
    std::vector<Node> nodes;
    std::vector<uint32_t> idx;
    const float* c;
    const float* e;

    BVH(const float* centers, const float* ext, uint32_t n) : c(centers), e(ext) {
        idx.resize(n);
        for (uint32_t i = 0; i < n; i++) idx[i] = i;
        if (n > 0) build(0, (int)n);
    }
    int build(int start, int end) {
        Node node;
        for (int a = 0; a < 3; a++) { node.mn[a] = INFINITY; node.mx[a] = -INFINITY; }
        node.start = start; node.end = end; node.left = -1; node.right = -1;
        const int ni = (int)nodes.size();
        nodes.push_back(node);
        for (int i = start; i < end; i++) {
            const uint32_t g = idx[i];
            for (int a = 0; a < 3; a++) {
                const double cc = c[g * 3 + a], ee = e[g * 3 + a];
                if (cc - ee < nodes[ni].mn[a]) nodes[ni].mn[a] = cc - ee;
                if (cc + ee > nodes[ni].mx[a]) nodes[ni].mx[a] = cc + ee;
            }
        }
        const int count = end - start;
        if (count <= 8) return ni;
        const double dx = nodes[ni].mx[0] - nodes[ni].mn[0];
        const double dy = nodes[ni].mx[1] - nodes[ni].mn[1];
        const double dz = nodes[ni].mx[2] - nodes[ni].mn[2];
        const int axis = dx > dy ? (dx > dz ? 0 : 2) : (dy > dz ? 1 : 2);
        const int mid = start + (count >> 1);
        nth(start, end, mid, axis);
        const int l = build(start, mid);
        const int r = build(mid, end);
        nodes[ni].left = l;
        nodes[ni].right = r;
        return ni;
    }
    void nth(int lo, int hi, int k, int axis) {
        uint32_t* ix = idx.data();
        while (hi - lo > 1) {
            const int m = (lo + hi) >> 1;
            const float a = c[ix[lo] * 3 + axis], b = c[ix[m] * 3 + axis], d = c[ix[hi - 1] * 3 + axis];
            const int pivotIdx = (a < b) ? (b < d ? m : (a < d ? hi - 1 : lo)) : (a < d ? lo : (b < d ? hi - 1 : m));
            std::swap(ix[lo + 1], ix[pivotIdx]);
            const float pivot = c[ix[lo + 1] * 3 + axis];
            int i = lo + 1, j = hi - 1;
            while (true) {
                while (++i < hi && c[ix[i] * 3 + axis] < pivot) {}
                while (--j > lo && c[ix[j] * 3 + axis] > pivot) {}
                if (i >= j) break;
                std::swap(ix[i], ix[j]);
            }
            std::swap(ix[lo + 1], ix[j]);
            if (j == k) return;
            if (j < k) lo = j + 1; else hi = j;
        }
    }
    void query(const double qmn[3], const double qmx[3], std::vector<uint32_t>& out) const {
        out.clear();
        if (nodes.empty()) return;
        std::vector<int> stack{0};
        while (!stack.empty()) {
            const int ni = stack.back();
            stack.pop_back();
            const Node& n = nodes[ni];
            bool skip = false;
            for (int a = 0; a < 3; a++) if (n.mx[a] < qmn[a] || n.mn[a] > qmx[a]) skip = true;
            if (skip) continue;
            if (n.left < 0) {
                for (int i = n.start; i < n.end; i++) {
                    const uint32_t g = idx[i];
                    bool ok = true;
                    for (int a = 0; a < 3 && ok; a++) {
                        const double gmn = (double)c[g * 3 + a] - (double)e[g * 3 + a];
                        const double gmx = (double)c[g * 3 + a] + (double)e[g * 3 + a];
                        if (gmx < qmn[a] || gmn > qmx[a]) ok = false;
                    }
                    if (ok) out.push_back(g);
                }
            } else {
                stack.push_back(n.left);
                stack.push_back(n.right);
            }
        }
    }
};

struct Gauss {   // voxelize.ts:250-276 record (logScale stored in the scale* slots)
    float pos[3], opLogit, rot[4], logScale[3], ext[3];
};

inline void crossf(const float a[3], const float b[3], float o[3]) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// shaders/voxelize.ts:62-84
float evalGaussian(const float vc[3], float half, const Gauss& g) {
    float diff[3];
    for (int a = 0; a < 3; a++) diff[a] = vc[a] - g.pos[a];
    for (int a = 0; a < 3; a++) if (std::abs(diff[a]) > (g.ext[a] + half)) return 0.0f;
    float cd[3];
    for (int a = 0; a < 3; a++) {
        const float closest = std::min(std::max(g.pos[a], vc[a] - half), vc[a] + half);
        cd[a] = closest - g.pos[a];
    }
    const float q[3] = {-g.rot[1], -g.rot[2], -g.rot[3]};
    float c1[3]; crossf(q, cd, c1);
    const float t[3] = {2.0f * c1[0], 2.0f * c1[1], 2.0f * c1[2]};
    float c2[3]; crossf(q, t, c2);
    float ld[3];
    for (int a = 0; a < 3; a++) ld[a] = (cd[a] + g.rot[0] * t[a]) + c2[a];
    const float inv[3] = {dl_expf(-g.logScale[0]), dl_expf(-g.logScale[1]), dl_expf(-g.logScale[2])};
    float s[3];
    for (int a = 0; a < 3; a++) s[a] = ld[a] * inv[a];
    const float d2 = (s[0] * s[0] + s[1] * s[1]) + s[2] * s[2];
    const float opacity = 1.0f / (1.0f + dl_expf(-g.opLogit));
    return opacity * dl_expf(-0.5f * d2);
}

struct BatchOut {
    std::vector<uint32_t> idx, lo, hi, nlo, nhi;   // blocks with solid or near bits
    uint64_t evals = 0;
};

}  // namespace

struct OrcVoxel {
    double bounds[6];
    double dims[3];
    std::vector<float> extents;
    std::vector<uint32_t> blockIdx, maskLo, maskHi;          // BlockMaskBuffer.blocks, in order
    std::vector<uint32_t> nearIdx, nearLo, nearHi, nearSolidLo, nearSolidHi;   // blocks with any |a-c|<eps bit
    uint64_t nearBits = 0, evals = 0, listEntries = 0;
};

// zrow_lo / zrow_hi: when zrow_hi > zrow_lo, only the batches of 16^3 blocks
// whose z row (bz / 16) lies in [zrow_lo, zrow_hi) are voxelized (bounds and
// dims still come from the whole input), so a full-size grid can be checked
// a few rows at a time; the block list keeps the batch order.
extern "C" void* orc_voxelize_run(const orc_splats* data, double voxelRes, double opacityCutoff,
                                  const double* bounds6, int order, float eps, int64_t zrow_lo, int64_t zrow_hi) {
    OrcVoxel* V = new OrcVoxel();
    const double blockSize = 4 * voxelRes;
    computeAabbExtents(*data, V->extents);
    const uint64_t n = data->count;
    if (bounds6) std::memcpy(V->bounds, bounds6, sizeof(V->bounds));
    else computeBlockAlignedBounds(*data, V->extents, blockSize, V->bounds);
    for (int a = 0; a < 3; a++) V->dims[a] = jsRound((V->bounds[3 + a] - V->bounds[a]) / blockSize);
    const double nbX = V->dims[0], nbY = V->dims[1], nbZ = V->dims[2];
    if (!(nbX > 0 && nbY > 0 && nbZ > 0) || n == 0) return V;
    const int64_t NX = (int64_t)nbX, NY = (int64_t)nbY, NZ = (int64_t)nbZ;
    const double bStride = nbX * nbY;

    std::vector<Gauss> gs(n);
    for (uint64_t i = 0; i < n; i++) {
        Gauss& g = gs[i];
        for (int a = 0; a < 3; a++) {
            g.pos[a] = data->positions[i * 3 + a];
            g.logScale[a] = data->log_scales[i * 3 + a];
            g.ext[a] = V->extents[i * 3 + a];
        }
        g.opLogit = data->opacity_logits[i];
        for (int a = 0; a < 4; a++) g.rot[a] = data->rotations[i * 4 + a];
    }
    const float res = (float)voxelRes;
    const float cutoff = (float)opacityCutoff;
    const float half = res * 0.5f;

    // batch grid, voxelize.ts:185-233
    struct Batch { int64_t bx, by, bz, cx, cy, cz; double qmn[3], qmx[3]; bool skip; };
    std::vector<Batch> batches;
    const bool rows = zrow_hi > zrow_lo;
    for (int64_t bz = 0; bz < NZ; bz += 16)
        for (int64_t by = 0; by < NY; by += 16)
            for (int64_t bx = 0; bx < NX; bx += 16) {
                Batch b;
                b.bx = bx; b.by = by; b.bz = bz;
                b.cx = std::min<int64_t>(16, NX - bx);
                b.cy = std::min<int64_t>(16, NY - by);
                b.cz = std::min<int64_t>(16, NZ - bz);
                b.skip = rows && (bz / 16 < zrow_lo || bz / 16 >= zrow_hi);
                b.qmn[0] = V->bounds[0] + (double)bx * blockSize;
                b.qmn[1] = V->bounds[1] + (double)by * blockSize;
                b.qmn[2] = V->bounds[2] + (double)bz * blockSize;
                b.qmx[0] = b.qmn[0] + (double)b.cx * blockSize;
                b.qmx[1] = b.qmn[1] + (double)b.cy * blockSize;
                b.qmx[2] = b.qmn[2] + (double)b.cz * blockSize;
                batches.push_back(b);
            }

    // canonical batch lists: ascending Gaussian index over the f64 overlap test
    std::vector<std::vector<uint32_t>> canon;
    BVH* bvh = nullptr;
    if (order == 1) {
        bvh = new BVH(data->positions, V->extents.data(), (uint32_t)n);
    } else {
        canon.resize(batches.size());
        const int64_t nbx = (NX + 15) / 16, nby = (NY + 15) / 16, nbz = (NZ + 15) / 16;
        for (uint64_t g = 0; g < n; g++) {
            int64_t lo[3], hi[3];
            const int64_t nb[3] = {nbx, nby, nbz};
            for (int a = 0; a < 3; a++) {
                const double gmn = (double)gs[g].pos[a] - (double)gs[g].ext[a];
                const double gmx = (double)gs[g].pos[a] + (double)gs[g].ext[a];
                const double span = 16 * blockSize;
                int64_t b0 = (int64_t)std::floor((gmn - V->bounds[a]) / span) - 1;
                int64_t b1 = (int64_t)std::floor((gmx - V->bounds[a]) / span) + 1;
                b0 = std::max<int64_t>(b0, 0); b1 = std::min<int64_t>(b1, nb[a] - 1);
                lo[a] = INT64_MAX; hi[a] = -1;
                const int64_t N_[3] = {NX, NY, NZ};
                for (int64_t b = b0; b <= b1; b++) {
                    const double qmn = V->bounds[a] + (double)(b * 16) * blockSize;
                    const double qmx = qmn + (double)std::min<int64_t>(16, N_[a] - b * 16) * blockSize;
                    if (gmx < qmn || gmn > qmx) continue;
                    lo[a] = std::min(lo[a], b); hi[a] = std::max(hi[a], b);
                }
            }
            if (rows) { lo[2] = std::max<int64_t>(lo[2], zrow_lo); hi[2] = std::min<int64_t>(hi[2], zrow_hi - 1); }
            for (int64_t z = lo[2]; z <= hi[2]; z++)
                for (int64_t y = lo[1]; y <= hi[1]; y++)
                    for (int64_t x = lo[0]; x <= hi[0]; x++)
                        canon[(size_t)((z * nby + y) * nbx + x)].push_back((uint32_t)g);
        }
    }

    std::vector<BatchOut> outs(batches.size());
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t bi_ = 0; bi_ < (int64_t)batches.size(); bi_++) {
        const Batch& B = batches[bi_];
        if (B.skip) continue;
        std::vector<uint32_t> listBuf;
        const std::vector<uint32_t>* list;
        if (order == 1) { bvh->query(B.qmn, B.qmx, listBuf); list = &listBuf; }
        else list = &canon[bi_];
        if (list->empty()) continue;   // voxelize.ts:212
        const float bmin[3] = {(float)B.qmn[0], (float)B.qmn[1], (float)B.qmn[2]};
        const int64_t total = B.cx * B.cy * B.cz;
        // per-block candidate lists (superset of the voxel-level AABB test, order kept)
        std::vector<std::vector<uint32_t>> blk((size_t)total);
        const int64_t cdim[3] = {B.cx, B.cy, B.cz};
        for (uint32_t g : *list) {
            int64_t lo[3], hi[3];
            for (int a = 0; a < 3; a++) {
                const double E = (double)gs[g].ext[a] + (double)half;
                const double tol = 1e-4 * (std::abs((double)bmin[a]) + 64.0 * voxelRes + E) + 1e-6;
                lo[a] = INT64_MAX; hi[a] = -1;
                for (int64_t l = 0; l < cdim[a]; l++) {
                    const double vlo = (double)bmin[a] + (double)l * 4 * voxelRes + 0.5 * voxelRes - tol;
                    const double vhi = (double)bmin[a] + (double)l * 4 * voxelRes + 3.5 * voxelRes + tol;
                    if ((double)gs[g].pos[a] + E < vlo || (double)gs[g].pos[a] - E > vhi) continue;
                    lo[a] = std::min(lo[a], l); hi[a] = std::max(hi[a], l);
                }
            }
            for (int64_t z = lo[2]; z <= hi[2]; z++)
                for (int64_t y = lo[1]; y <= hi[1]; y++)
                    for (int64_t x = lo[0]; x <= hi[0]; x++)
                        blk[(size_t)(x + y * B.cx + z * B.cx * B.cy)].push_back(g);
        }
        BatchOut& O = outs[bi_];
        for (int64_t fb = 0; fb < total; fb++) {
            const int64_t blockX = fb % B.cx, blockY = (fb / B.cx) % B.cy, blockZ = fb / (B.cx * B.cy);
            uint32_t m[2] = {0, 0}, nm[2] = {0, 0};
            const std::vector<uint32_t>& L = blk[(size_t)fb];
            for (uint32_t vi = 0; vi < 64; vi++) {
                // mortonToXYZ (shaders/voxelize.ts:54-60)
                const uint32_t lx = (vi & 1u) | ((vi >> 2) & 2u);
                const uint32_t ly = ((vi >> 1) & 1u) | ((vi >> 3) & 2u);
                const uint32_t lz = ((vi >> 2) & 1u) | ((vi >> 4) & 2u);
                const float boff[3] = {((float)blockX * 4.0f) * res, ((float)blockY * 4.0f) * res,
                                       ((float)blockZ * 4.0f) * res};
                const float lp[3] = {(float)lx, (float)ly, (float)lz};
                float vc[3];
                for (int a = 0; a < 3; a++) vc[a] = (bmin[a] + boff[a]) + ((lp[a] + 0.5f) * res);
                float sigma = 0.0f;
                for (uint32_t g : L) {
                    sigma = sigma + evalGaussian(vc, half, gs[g]);
                    O.evals++;
                    if (sigma >= 7.0f) break;
                }
                const float opacity = 1.0f - dl_expf(-sigma);
                const uint32_t lin = lz * 16 + ly * 4 + lx;
                if (opacity >= cutoff) m[lin >> 5] |= 1u << (lin & 31);
                if (std::abs(opacity - cutoff) < eps) nm[lin >> 5] |= 1u << (lin & 31);
            }
            if ((m[0] | m[1] | nm[0] | nm[1]) == 0) continue;
            const double flat = (double)(B.bx + blockX) + (double)(B.by + blockY) * nbX +
                                (double)(B.bz + blockZ) * bStride;
            O.idx.push_back((uint32_t)flat);
            O.lo.push_back(m[0]); O.hi.push_back(m[1]);
            O.nlo.push_back(nm[0]); O.nhi.push_back(nm[1]);
        }
        if (order != 1) { std::vector<uint32_t>().swap(canon[bi_]); }
    }
    for (auto& O : outs) {
        V->evals += O.evals;
        for (size_t i = 0; i < O.idx.size(); i++) {
            if (O.lo[i] | O.hi[i]) {   // BlockMaskBuffer.addBlock skips zero masks
                V->blockIdx.push_back(O.idx[i]); V->maskLo.push_back(O.lo[i]); V->maskHi.push_back(O.hi[i]);
            }
            if (O.nlo[i] | O.nhi[i]) {
                V->nearIdx.push_back(O.idx[i]); V->nearLo.push_back(O.nlo[i]); V->nearHi.push_back(O.nhi[i]);
                V->nearSolidLo.push_back(O.lo[i]); V->nearSolidHi.push_back(O.hi[i]);
                V->nearBits += __builtin_popcount(O.nlo[i]) + __builtin_popcount(O.nhi[i]);
            }
        }
    }
    delete bvh;
    return V;
}

extern "C" int64_t orc_voxelize_get(void* h, const char* name, void* dst, int64_t cap) {
    OrcVoxel* V = (OrcVoxel*)h;
    const void* src = nullptr;
    int64_t bytes = -1;
    uint64_t scalar = 0;
    auto vec = [&](const auto& v) { src = v.data(); bytes = (int64_t)(v.size() * sizeof(v[0])); };
    const std::string s(name);
    if (s == "block_idx") vec(V->blockIdx);
    else if (s == "mask_lo") vec(V->maskLo);
    else if (s == "mask_hi") vec(V->maskHi);
    else if (s == "near_idx") vec(V->nearIdx);
    else if (s == "near_lo") vec(V->nearLo);
    else if (s == "near_hi") vec(V->nearHi);
    else if (s == "near_solid_lo") vec(V->nearSolidLo);
    else if (s == "near_solid_hi") vec(V->nearSolidHi);
    else if (s == "extents") vec(V->extents);
    else if (s == "bounds") { src = V->bounds; bytes = 48; }
    else if (s == "dims") { src = V->dims; bytes = 24; }
    else if (s == "near_bits") { scalar = V->nearBits; src = &scalar; bytes = 8; }
    else if (s == "evals") { scalar = V->evals; src = &scalar; bytes = 8; }
    else return -1;
    if (dst && cap >= bytes && bytes > 0) std::memcpy(dst, src, (size_t)bytes);
    return bytes;
}

extern "C" void orc_voxelize_free(void* h) { delete (OrcVoxel*)h; }

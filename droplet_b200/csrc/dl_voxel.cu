// dl_voxel.cu — the voxelizer (src/voxel/voxelize.ts:59-248) on the device.
//
// Reference pipeline: CPU AABB extents (aabb.ts), CPU BVH (bvh.ts), 16^3-block
// batches whose BVH lists are uploaded per mega-flush, one 64-thread workgroup
// per 4x4x4 block scanning the WHOLE batch list (shaders/voxelize.ts), CPU
// decode of the masks into a BlockMaskBuffer.
//
// Here:
//   vox_prep_k     per-Gaussian f64 extents (aabb.ts:22-62, same op order),
//                  the 64-byte evaluation record, and partial bounds.
//   vox_bounds_k   final min/max reduction (voxelize.ts:278-306 inputs).
//   vox_emit_k     Gaussian -> block binning: for every block a Gaussian can
//                  touch, one (block key, Gaussian) pair.  A Gaussian is binned
//                  to a block only if it is in the block's 16^3 batch list under
//                  the reference's f64 box test (bvh.ts:153-168), and only if
//                  its box can reach one of the block's voxel centres (a
//                  superset of the shader's per-voxel test, which still runs).
//                  The key orders blocks exactly as the reference appends them
//                  (batch z, y, x; then x-fastest inside the batch).
//   dlsort         stable sort by key: each block's list is in ascending index.
//   vox_heads_k    run heads -> one work item per non-empty block.
//   vox_eval_k     per block, 64 threads = 64 voxels; 64-Gaussian tiles staged
//                  through shared memory; the density sum, the sigma >= 7 early
//                  exit and the Beer-Lambert threshold of shaders/voxelize.ts:
//                  62-147 in the same f32 order; warp ballots build the two
//                  32-bit masks directly (thread = linear bit index).
//   vox_compact_k  drop all-zero masks (BlockMaskBuffer.addBlock skips them).
// The density of a voxel is summed over its batch list in ascending Gaussian
// index; the reference sums in its BVH's DFS order, so the two agree except
// for voxels whose opacity lies within float rounding of the cutoff.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_bf16.h>

#include "dl_internal.h"
#include "dl_mlp.cuh"
#include "dl_sort.cuh"

// Page-locked host memory for the block lists of a call on their way back
// from the device.  A result handle keeps the buffer until dl_vox_result_free,
// which hands it back for the device's next call (or frees it when the pool
// already holds one); so block lists come back at full PCIe rate without
// pinning memory on every call.
struct PinnedPool {
    std::mutex m;
    void* p = nullptr;
    size_t cap = 0;
    ~PinnedPool() { if (p) cudaFreeHost(p); }
    void take(void** q, size_t* c) {
        std::lock_guard<std::mutex> g(m);
        *q = p; *c = cap; p = nullptr; cap = 0;
    }
    void give(void* q, size_t c) {
        if (!q) return;
        std::lock_guard<std::mutex> g(m);
        if (p && cap >= c) { cudaFreeHost(q); return; }
        if (p) cudaFreeHost(p);
        p = q; cap = c;
    }
};

struct dl_vox_result {
    double bmin[3], bmax[3], dims[3];
    std::vector<uint32_t> idx, lo, hi;             // block lists built on the host (cutoff <= 0)
    // block lists read back from the device: per slab, count entries of idx, lo
    // and hi one after the other in the pinned buffer, from word offset off
    std::shared_ptr<PinnedPool> pool;
    uint32_t* pinned = nullptr;
    size_t pinned_cap = 0;                         // bytes
    uint64_t pinned_used = 0;                      // u32 words
    uint64_t pinned_count = 0;                     // blocks
    std::vector<std::pair<uint64_t, uint32_t>> segs;
    ~dl_vox_result() {
        if (!pinned) return;
        if (pool) pool->give(pinned, pinned_cap);
        else cudaFreeHost(pinned);
    }
    std::vector<float> log_feat, log_cost;         // per evaluated block, with log_blocks
    // with DL_VOX_PROFILE: prep, binning, sort, heads, eval, compact, host (slab set-up and result copies)
    double stage_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

namespace {
// Device-time marks of a profiled voxelize call: each interval between two
// marks is charged to the stage of the mark that ends it.
struct VoxMarks {
    bool on = false;
    cudaStream_t st = nullptr;
    std::vector<std::pair<int, cudaEvent_t>> ev;
    void mark(int stage) {
        if (!on) return;
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return;
        cudaEventRecord(e, st);
        ev.emplace_back(stage, e);
    }
    void finish(double* ms) {
        if (on && !ev.empty()) {
            cudaEventSynchronize(ev.back().second);
            for (size_t i = 1; i < ev.size(); i++) {
                float t = 0.0f;
                if (cudaEventElapsedTime(&t, ev[i - 1].second, ev[i].second) == cudaSuccess) ms[ev[i].first] += t;
            }
        }
        for (auto& e : ev) cudaEventDestroy(e.second);
        ev.clear();
    }
    ~VoxMarks() { for (auto& e : ev) cudaEventDestroy(e.second); }
};
}  // namespace

namespace {

constexpr unsigned long long kAgg = 1ull << 62, kPre = 2ull << 62, kMask = (1ull << 62) - 1;

// Decoupled look-back over the CTAs of one chain, by one whole warp: each step
// reads the 32 nearest predecessors not yet added (lane l reads tile q - l),
// adds the aggregates before the first unpublished one, and stops at the
// first inclusive prefix.  At most spin_limit polls of an unpublished
// predecessor, then DL_DEVERR_TIMEOUT and the prefix summed so far (the CTA's
// writes stay inside the chain).  No fence: a status word carries its own
// value and no other data passes between CTAs.  Returns the exclusive prefix
// to every lane.
__device__ unsigned long long lookback_warp(unsigned long long* status, uint32_t tile, unsigned long long total,
                                            uint32_t* err, uint32_t spin_limit) {
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) dl_st_volatile64(&status[0], kPre | total);
        return 0ull;
    }
    if (lane == 0) dl_st_volatile64(&status[tile], kAgg | total);
    unsigned long long excl = 0;
    int64_t q = (int64_t)tile - 1;
    uint32_t spins = 0;
    while (true) {
        // tile 0 always publishes an inclusive prefix, so a walk never passes it
        const unsigned long long w = (q - lane >= 0) ? dl_ld_volatile64(&status[q - lane]) : kPre;
        const unsigned long long f = w & ~kMask;
        const uint32_t notReady = __ballot_sync(0xffffffffu, f == 0ull);
        const uint32_t prefix = __ballot_sync(0xffffffffu, f == kPre);
        const int firstNR = notReady ? __ffs(notReady) - 1 : 32;
        const int firstP = prefix ? __ffs(prefix) - 1 : 32;
        const int take = firstP < firstNR ? firstP + 1 : firstNR;
        unsigned long long add = lane < take ? (w & kMask) : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) add += __shfl_xor_sync(0xffffffffu, add, o);
        excl += add;
        if (firstP < firstNR) break;
        q -= take;
        if (take == 0) {
            if (++spins > spin_limit) { if (lane == 0) atomicOr(err, DL_DEVERR_TIMEOUT); break; }
            __nanosleep(32);
        }
    }
    if (lane == 0) dl_st_volatile64(&status[tile], kPre | ((excl + total) & kMask));
    return excl;
}

// Gaussian record read by vox_eval_k (voxelize.ts:250-276 fields, with the
// per-Gaussian sub-expressions of evalGaussian precomputed in the same f32 ops).
struct __align__(16) VoxRec {
    float px, py, pz, opacity;      // opacity = 1 / (1 + exp(-logit))
    float qw, nqx, nqy, nqz;        // inverse rotation: xyz negated
    float isx, isy, isz, pad0;      // exp(-logScale)
    float ehx, ehy, ehz, pad1;      // extent + voxelHalf
};

struct VoxParams {
    const float* pos;
    const float* rot;
    const float* lsc;
    const float* opl;
    uint32_t n;
    float res, half, cutoff;
    double boundsMin[3];
    double blockSize;
    int64_t NB[3];                  // blocks per axis
    int64_t NBB[3];                 // batches per axis
    const double* qmn[3];           // per-axis batch box (f64)
    const double* qmx[3];
    const float* bmin32[3];         // per-axis f32 batch min (BatchInfo.blockMin*)
    int64_t zlo, zhi;               // block z range of the slab being processed
    int64_t ylo, yhi;               // block y range of the slab being processed
    int64_t xlo, xhi;               // block x range of the slab being processed
};

__global__ void vox_prep_k(VoxParams p, float* __restrict__ ext, VoxRec* __restrict__ rec, double* __restrict__ part) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (g < p.n) {
        // aabb.ts:28-60 (f64)
        const double qw = p.rot[4ull * g], qx = p.rot[4ull * g + 1], qy = p.rot[4ull * g + 2], qz = p.rot[4ull * g + 3];
        const float l0 = p.lsc[3ull * g], l1 = p.lsc[3ull * g + 1], l2 = p.lsc[3ull * g + 2];
        const double sx = dl_exp((double)l0), sy = dl_exp((double)l1), sz = dl_exp((double)l2);
        const double xx = qx * qx, yy = qy * qy, zz = qz * qz;
        const double xy = qx * qy, xz = qx * qz, yz = qy * qz;
        const double wx = qw * qx, wy = qw * qy, wz = qw * qz;
        const double r00 = 1 - 2 * (yy + zz), r01 = 2 * (xy - wz), r02 = 2 * (xz + wy);
        const double r10 = 2 * (xy + wz), r11 = 1 - 2 * (xx + zz), r12 = 2 * (yz - wx);
        const double r20 = 2 * (xz - wy), r21 = 2 * (yz + wx), r22 = 1 - 2 * (xx + yy);
        const double a0 = r00 * sx, a1 = r01 * sy, a2 = r02 * sz;
        const double b0 = r10 * sx, b1 = r11 * sy, b2 = r12 * sz;
        const double c0 = r20 * sx, c1 = r21 * sy, c2 = r22 * sz;
        const float e[3] = {(float)(sqrt((a0 * a0 + a1 * a1) + a2 * a2) * 3.0),
                            (float)(sqrt((b0 * b0 + b1 * b1) + b2 * b2) * 3.0),
                            (float)(sqrt((c0 * c0 + c1 * c1) + c2 * c2) * 3.0)};
        const float ps[3] = {p.pos[3ull * g], p.pos[3ull * g + 1], p.pos[3ull * g + 2]};
        for (int k = 0; k < 3; k++) {
            ext[3ull * g + k] = e[k];
            mn[k] = (double)ps[k] - (double)e[k];
            mx[k] = (double)ps[k] + (double)e[k];
        }
        VoxRec r;
        r.px = ps[0]; r.py = ps[1]; r.pz = ps[2];
        r.opacity = 1.0f / (1.0f + dl_expf(-p.opl[g]));
        r.qw = (float)qw; r.nqx = -(float)qx; r.nqy = -(float)qy; r.nqz = -(float)qz;
        r.isx = dl_expf(-l0); r.isy = dl_expf(-l1); r.isz = dl_expf(-l2); r.pad0 = 0.0f;
        r.ehx = e[0] + p.half; r.ehy = e[1] + p.half; r.ehz = e[2] + p.half; r.pad1 = 0.0f;
        rec[g] = r;
    }
    // block min/max (NaN-ignoring like the reference's `<` comparisons)
    __shared__ double s[6][256];
    for (int k = 0; k < 3; k++) { s[k][threadIdx.x] = mn[k]; s[3 + k][threadIdx.x] = mx[k]; }
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            for (int k = 0; k < 3; k++) {
                const double a = s[k][threadIdx.x + o];
                if (a < s[k][threadIdx.x]) s[k][threadIdx.x] = a;
                const double b = s[3 + k][threadIdx.x + o];
                if (b > s[3 + k][threadIdx.x]) s[3 + k][threadIdx.x] = b;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x < 6) part[6ull * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

__global__ void vox_bounds_k(const double* part, uint32_t nparts, double* out) {
    if (threadIdx.x >= 6) return;
    const int k = threadIdx.x;
    double v = k < 3 ? INFINITY : -INFINITY;
    for (uint32_t i = 0; i < nparts; i++) {
        const double a = part[6ull * i + k];
        if (k < 3 ? (a < v) : (a > v)) v = a;
    }
    out[k] = v;
}

// Batches along axis a whose f64 box the Gaussian's f64 AABB overlaps
// (bvh.ts:162-168); bhi < blo: none.
__device__ void batch_range(const VoxParams& p, int a, float c, float e, int64_t& blo, int64_t& bhi) {
    blo = INT64_MAX; bhi = -1;
    const int64_t NBB = p.NBB[a];
    const double gmn = (double)c - (double)e, gmx = (double)c + (double)e;
    const double span = 16.0 * p.blockSize;
    const double f0 = floor((gmn - p.boundsMin[a]) / span) - 1.0, f1 = floor((gmx - p.boundsMin[a]) / span) + 1.0;
    if (!(f1 >= 0.0) || !(f0 <= (double)(NBB - 1))) return;
    const int64_t b0 = f0 < 0.0 ? 0 : (int64_t)f0, b1 = f1 > (double)(NBB - 1) ? NBB - 1 : (int64_t)f1;
    for (int64_t b = b0; b <= b1; b++) {
        if (gmx < p.qmn[a][b] || gmn > p.qmx[a][b]) continue;
        blo = min(blo, b); bhi = max(bhi, b);
    }
}

// Block range [lo, hi] along one axis for Gaussian centre c, extent e (hi < lo: none).
__device__ void axis_range(const VoxParams& p, int a, float c, float e, float eh, int64_t& lo, int64_t& hi) {
    lo = 0; hi = -1;
    const int64_t NB = p.NB[a];
    int64_t blo, bhi;
    batch_range(p, a, c, e, blo, bhi);
    if (bhi < 0) return;
    // blocks with a voxel centre coordinate (the f32 expression of vox_eval_k)
    // within eh of c on this axis: the shader's per-axis test, evaluated exactly
    const double step = 4.0 * (double)p.res;
    const double u0 = ((double)c - (double)eh - p.boundsMin[a]) / step - 1.0;
    const double u1 = ((double)c + (double)eh - p.boundsMin[a]) / step + 1.0;
    if (!(u1 >= 0.0) || !(u0 <= (double)(NB - 1))) return;
    const int64_t c0 = u0 < 0.0 ? 0 : (int64_t)u0;
    const int64_t c1 = u1 > (double)(NB - 1) ? NB - 1 : (int64_t)u1;
    int64_t v0 = INT64_MAX, v1 = -1;
    for (int64_t l = c0; l <= c1; l++) {
        const float bmin = p.bmin32[a][l >> 4];
        const float boff = ((float)(l & 15) * 4.0f) * p.res;
        bool any = false;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const float vc = (bmin + boff) + (((float)k + 0.5f) * p.res);
            if (!(fabsf(vc - c) > eh)) any = true;
        }
        if (any) { v0 = min(v0, l); v1 = max(v1, l); }
    }
    if (v1 < 0) return;
    lo = max(v0, blo * 16);
    hi = min(v1, min(bhi * 16 + 15, NB - 1));
    if (a == 2) { lo = max(lo, p.zlo); hi = min(hi, p.zhi); }
    if (a == 1) { lo = max(lo, p.ylo); hi = min(hi, p.yhi); }
    if (a == 0) { lo = max(lo, p.xlo); hi = min(hi, p.xhi); }
}

// Batches with a non-empty batch list (the reference dispatches exactly these).
__global__ void vox_batchused_k(VoxParams p, const float* __restrict__ ext, uint32_t* __restrict__ used) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.n) return;
    int64_t lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        batch_range(p, k, p.pos[3ull * g + k], ext[3ull * g + k], lo[k], hi[k]);
        if (hi[k] < 0) return;
    }
    for (int64_t bz = lo[2]; bz <= hi[2]; bz++)
        for (int64_t by = lo[1]; by <= hi[1]; by++)
            for (int64_t bx = lo[0]; bx <= hi[0]; bx++) used[(bz * p.NBB[1] + by) * p.NBB[0] + bx] = 1u;
}

// Gaussian-block pairs per 16^3-block batch (sizes the slabs).
__global__ void vox_batchcount_k(VoxParams p, const float* __restrict__ ext, unsigned long long* __restrict__ cnt) {
    const uint32_t g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.n) return;
    int64_t lo[3], hi[3];
    for (int k = 0; k < 3; k++) {
        const float e = ext[3ull * g + k];
        axis_range(p, k, p.pos[3ull * g + k], e, e + p.half, lo[k], hi[k]);
    }
    if (hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]) return;
    for (int64_t bz = lo[2] >> 4; bz <= (hi[2] >> 4); bz++) {
        const int64_t nz = min(hi[2], bz * 16 + 15) - max(lo[2], bz * 16) + 1;
        for (int64_t by = lo[1] >> 4; by <= (hi[1] >> 4); by++) {
            const int64_t ny = min(hi[1], by * 16 + 15) - max(lo[1], by * 16) + 1;
            for (int64_t bx = lo[0] >> 4; bx <= (hi[0] >> 4); bx++) {
                const int64_t nx = min(hi[0], bx * 16 + 15) - max(lo[0], bx * 16) + 1;
                atomicAdd(&cnt[(bz * p.NBB[1] + by) * p.NBB[0] + bx], (unsigned long long)(nx * ny * nz));
            }
        }
    }
}

constexpr int kVT = 256, kVI = 4, kVR = kVT * kVI;

struct VoxEmitArgs {
    VoxParams p;
    const float* ext;
    uint32_t* keys;
    uint32_t* vals;
    unsigned long long cap;
    unsigned long long* npairs;
    unsigned long long* status;
    uint32_t* counter;
    uint32_t* err;
    uint32_t* ovf;
    uint32_t spin_limit;
};

__global__ void __launch_bounds__(kVT) vox_emit_k(VoxEmitArgs a) {
    __shared__ uint32_t s_excl[kVR + 1];
    __shared__ uint32_t s_g[kVR];
    __shared__ uint32_t s_x0[kVR], s_y0[kVR], s_z0[kVR];
    __shared__ uint16_t s_xs[kVR], s_ys[kVR];
    __shared__ uint32_t s_wsum[kVT / 32];
    __shared__ uint32_t s_tile, s_skip;
    __shared__ unsigned long long s_pre;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t g0 = tile * kVR;
    if (g0 >= a.p.n) return;
    uint32_t cnt[kVI], local = 0;
#pragma unroll
    for (int j = 0; j < kVI; j++) {
        const uint32_t i = tid * kVI + j;
        const uint32_t g = g0 + i;
        cnt[j] = 0;
        s_g[i] = g;
        if (g < a.p.n) {
            int64_t lo[3], hi[3];
            const float c[3] = {a.p.pos[3ull * g], a.p.pos[3ull * g + 1], a.p.pos[3ull * g + 2]};
            for (int k = 0; k < 3; k++) {
                const float e = a.ext[3ull * g + k];
                axis_range(a.p, k, c[k], e, e + a.p.half, lo[k], hi[k]);
            }
            if (hi[0] >= lo[0] && hi[1] >= lo[1] && hi[2] >= lo[2]) {
                const uint64_t c64 = (uint64_t)(hi[0] - lo[0] + 1) * (uint64_t)(hi[1] - lo[1] + 1) *
                                     (uint64_t)(hi[2] - lo[2] + 1);
                if (c64 >= (1ull << 31) || hi[0] - lo[0] >= 65535 || hi[1] - lo[1] >= 65535) {
                    atomicOr(a.ovf, 4u);    // a single Gaussian touching > 2^31 blocks
                } else {
                    cnt[j] = (uint32_t)c64;
                    s_x0[i] = (uint32_t)lo[0]; s_y0[i] = (uint32_t)lo[1]; s_z0[i] = (uint32_t)lo[2];
                    s_xs[i] = (uint16_t)(hi[0] - lo[0] + 1); s_ys[i] = (uint16_t)(hi[1] - lo[1] + 1);
                }
            }
        }
        local += cnt[j];
    }
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
    for (int w = 0; w < kVT / 32; w++) { if (w < warp) wpre += s_wsum[w]; total += s_wsum[w]; }
    uint32_t run = wpre + inc - local;
#pragma unroll
    for (int j = 0; j < kVI; j++) { s_excl[tid * kVI + j] = run; run += cnt[j]; }
    if (warp == 0) {
        const unsigned long long pre = lookback_warp(a.status, tile, total, a.err, a.spin_limit);
        if (lane == 0) {
            s_excl[kVR] = total;
            s_pre = pre;
            if (g0 + kVR >= a.p.n) *a.npairs = pre + total;
            const bool over = pre + total > a.cap;
            if (over) atomicOr(a.ovf, DL_DEVERR_OVERFLOW);
            s_skip = over;
        }
    }
    __syncthreads();
    if (s_skip) return;
    const unsigned long long base = s_pre;
    const int64_t NX = a.p.NB[0], NY = a.p.NB[1], NBX = a.p.NBB[0], NBY = a.p.NBB[1];
    for (uint32_t o = tid; o < total; o += kVT) {
        uint32_t lo = 0, hi = kVR;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_excl[mid] <= o) lo = mid; else hi = mid;
        }
        const uint32_t w = o - s_excl[lo];
        const uint32_t xs = s_xs[lo], ys = s_ys[lo];
        const int64_t ax = s_x0[lo] + w % xs;
        const int64_t ay = s_y0[lo] + (w / xs) % ys;
        const int64_t az = s_z0[lo] + w / (xs * ys);
        const int64_t bx = ax >> 4, by = ay >> 4, bz = az >> 4;
        const int64_t cx = min((int64_t)16, NX - bx * 16), cy = min((int64_t)16, NY - by * 16);
        const int64_t bi = (ax & 15) + (ay & 15) * cx + (az & 15) * cx * cy;
        const int64_t batch = (bz * NBY + by) * NBX + bx;
        a.keys[base + o] = (uint32_t)((batch << 12) | bi);
        a.vals[base + o] = s_g[lo];
    }
}

// Run heads of the sorted keys -> block work items (key, list start); the
// last CTA writes the block count and the final list end.
struct HeadsArgs {
    const uint32_t* keys;
    const unsigned long long* npairs;
    uint32_t* bkey;
    uint32_t* bstart;
    uint32_t* nblocks;
    unsigned long long* status;
    uint32_t* counter;
    uint32_t* err;
    uint32_t spin_limit;
};

constexpr int kHI = 16, kHR = kVT * kHI;      // sorted keys per thread / per CTA of the heads kernel

__global__ void __launch_bounds__(kVT) vox_heads_k(HeadsArgs a) {
    __shared__ uint32_t s_wsum[kVT / 32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_pre;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // after a timed-out sort the keys may hold unwritten slots: no blocks
    if (__syncthreads_or(tid == 0 && (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT))) {
        if (blockIdx.x == 0 && tid == 0) { *a.nblocks = 0; a.bstart[0] = 0; }
        return;
    }
    if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const unsigned long long n = *a.npairs;
    const unsigned long long i0 = (unsigned long long)tile * kHR;
    if (i0 >= n) {
        if (tile == 0 && tid == 0) { *a.nblocks = 0; a.bstart[0] = 0; }
        return;
    }
    // warp-striped: warp w reads keys [i0 + 512 w, i0 + 512 (w + 1)), 32 at a time
    const uint32_t lmask = dl_lanemask_lt();
    const unsigned long long wb = i0 + (unsigned long long)warp * 32 * kHI;
    uint32_t hm[kHI], key[kHI], wcount = 0;
#pragma unroll
    for (int j = 0; j < kHI; j++) {
        const unsigned long long i = wb + (unsigned long long)j * 32 + lane;
        key[j] = i < n ? a.keys[i] : 0u;
        const bool head = i < n && (i == 0 || key[j] != a.keys[i - 1]);
        hm[j] = __ballot_sync(0xffffffffu, head);
        wcount += __popc(hm[j]);
    }
    if (lane == 0) s_wsum[warp] = wcount;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
    for (int w = 0; w < kVT / 32; w++) { if (w < warp) wpre += s_wsum[w]; total += s_wsum[w]; }
    if (warp == 0) {
        const unsigned long long pre = lookback_warp(a.status, tile, total, a.err, a.spin_limit);
        if (lane == 0) {
            s_pre = pre;
            if (i0 + kHR >= n) { *a.nblocks = (uint32_t)(pre + total); a.bstart[pre + total] = (uint32_t)n; }
        }
    }
    __syncthreads();
    uint32_t run = (uint32_t)s_pre + wpre;
#pragma unroll
    for (int j = 0; j < kHI; j++) {
        if ((hm[j] >> lane) & 1u) {
            const uint32_t pos = run + __popc(hm[j] & lmask);
            a.bkey[pos] = key[j];
            a.bstart[pos] = (uint32_t)(wb + (unsigned long long)j * 32 + lane);
        }
        run += __popc(hm[j]);
    }
}

struct EvalArgs {
    VoxParams p;
    const VoxRec* rec;
    const uint32_t* vals;
    const uint32_t* bkey;
    const uint32_t* bstart;
    const uint32_t* nblocks;
    uint2* masks;
    uint32_t* counter;
    const uint32_t* work;          // optional block order (learned); NULL: block order
    uint32_t* cycles;              // optional [block] SM cycles / 16 spent on the block
    const uint32_t* err;           // DL_DEVERR_TIMEOUT: the block lists are not complete
};

template <bool kFast>
__device__ __forceinline__ float vox_exp(float x) {
    if (!kFast) return dl_expf(x);
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x * 1.4426950408889634f));
    return y;
}

template <bool kFast>
__device__ __forceinline__ float eval_gaussian(const float vc[3], float half, const VoxRec& g) {
    // shaders/voxelize.ts:62-84, same f32 operation order
    const float d0 = vc[0] - g.px, d1 = vc[1] - g.py, d2 = vc[2] - g.pz;
    if (fabsf(d0) > g.ehx || fabsf(d1) > g.ehy || fabsf(d2) > g.ehz) return 0.0f;
    const float cd0 = fminf(fmaxf(g.px, vc[0] - half), vc[0] + half) - g.px;
    const float cd1 = fminf(fmaxf(g.py, vc[1] - half), vc[1] + half) - g.py;
    const float cd2 = fminf(fmaxf(g.pz, vc[2] - half), vc[2] + half) - g.pz;
    const float qx = g.nqx, qy = g.nqy, qz = g.nqz;
    const float t0 = 2.0f * (qy * cd2 - qz * cd1);
    const float t1 = 2.0f * (qz * cd0 - qx * cd2);
    const float t2 = 2.0f * (qx * cd1 - qy * cd0);
    const float l0 = (cd0 + g.qw * t0) + (qy * t2 - qz * t1);
    const float l1 = (cd1 + g.qw * t1) + (qz * t0 - qx * t2);
    const float l2 = (cd2 + g.qw * t2) + (qx * t1 - qy * t0);
    const float s0 = l0 * g.isx, s1 = l1 * g.isy, s2 = l2 * g.isz;
    const float d2s = (s0 * s0 + s1 * s1) + s2 * s2;
    return g.opacity * vox_exp<kFast>(-0.5f * d2s);
}

// kFast: hardware ex2 for the density exponentials (DL_VOX_FAST_EXP)
template <bool kFast>
__global__ void __launch_bounds__(64, 32) vox_eval_k(EvalArgs a) {
    __shared__ VoxRec s_g[64];
    __shared__ uint32_t s_b;
    __shared__ uint32_t s_mask[2];
    const int tid = threadIdx.x;
    // the heads kernel before this one is complete: a timed-out wait there
    // (partial block lists) leaves nothing to evaluate
    const uint32_t nb = (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT) ? 0u : *a.nblocks;
    // linear bit index = z*16 + y*4 + x (shaders/voxelize.ts:137)
    const uint32_t lx = tid & 3, ly = (tid >> 2) & 3, lz = tid >> 4;
    const int64_t NX = a.p.NB[0], NY = a.p.NB[1], NBX = a.p.NBB[0], NBY = a.p.NBB[1];
    while (true) {
        if (tid == 0) {
            const uint32_t k = atomicAdd(a.counter, 1u);
            s_b = (k < nb && a.work) ? a.work[k] : k;
        }
        __syncthreads();
        const uint32_t b = s_b;
        __syncthreads();
        if (b >= nb) break;
        const long long t0 = a.cycles ? clock64() : 0;
        const uint32_t key = a.bkey[b];
        const uint32_t batch = key >> 12, bi = key & 4095u;
        const int64_t bxI = batch % NBX, byI = (batch / NBX) % NBY, bzI = batch / (NBX * NBY);
        const int64_t cx = min((int64_t)16, NX - bxI * 16), cy = min((int64_t)16, NY - byI * 16);
        const uint32_t blockX = bi % cx, blockY = (bi / cx) % cy, blockZ = bi / (cx * cy);
        // voxel centre exactly as shaders/voxelize.ts:103-106
        const float res = a.p.res;
        const float bmin[3] = {a.p.bmin32[0][bxI], a.p.bmin32[1][byI], a.p.bmin32[2][bzI]};
        const float boff[3] = {((float)blockX * 4.0f) * res, ((float)blockY * 4.0f) * res, ((float)blockZ * 4.0f) * res};
        const float lp[3] = {(float)lx, (float)ly, (float)lz};
        float vc[3];
        for (int k = 0; k < 3; k++) vc[k] = (bmin[k] + boff[k]) + ((lp[k] + 0.5f) * res);
        const uint32_t start = a.bstart[b], end = a.bstart[b + 1];
        float sigma = 0.0f;
        for (uint32_t c = start; c < end; c += 64) {
            const uint32_t i = c + tid;
            if (i < end) s_g[tid] = a.rec[a.vals[i]];
            __syncthreads();
            const uint32_t m = min(64u, end - c);
            if (sigma < 7.0f) {
                for (uint32_t j = 0; j < m; j++) {
                    sigma = sigma + eval_gaussian<kFast>(vc, a.p.half, s_g[j]);
                    if (sigma >= 7.0f) break;
                }
            }
            if (__syncthreads_count(sigma < 7.0f) == 0) break;
        }
        const float opacity = 1.0f - vox_exp<kFast>(-sigma);
        const bool solid = opacity >= a.p.cutoff;
        const uint32_t bal = __ballot_sync(0xffffffffu, solid);
        if ((tid & 31) == 0) s_mask[tid >> 5] = bal;
        __syncthreads();
        if (tid == 0) {
            a.masks[b] = make_uint2(s_mask[0], s_mask[1]);
            if (a.cycles) a.cycles[b] = (uint32_t)((clock64() - t0) >> 4);
        }
    }
}

// ---- learned block order.  The 12 inputs of the block-cost model: the list
// lengths of the block and its neighbours in list order, a sample of up to 8
// of its Gaussians (mean and max opacity, mean and min extent in voxels: dense
// opaque lists reach sigma >= 7 early), the block's place in its batch and
// the cutoff.  vox_sched_pred_k: features, prediction, 8-bit bucket that
// decreases with the predicted cost; vox_sched_scan_k: bucket offsets;
// vox_sched_scatter_k: blocks into the work list.  Every block writes its own
// mask, so any order gives the same result.
struct VoxSchedArgs {
    VoxParams p;
    const VoxRec* rec;
    const uint32_t* vals;
    const uint32_t* bkey;
    const uint32_t* bstart;
    const uint32_t* nblocks;
    const __nv_bfloat16* w;        // model parameters (NULL: features only)
    float* feat;                   // optional [block][12]
    uint32_t* bucket;              // [block]
    uint32_t* hist;                // [256] (zeroed)
    uint32_t* work;                // [block]
    const uint32_t* err;           // DL_DEVERR_TIMEOUT: the block lists are not complete
};

__device__ __forceinline__ void vox_block_features(const VoxSchedArgs& a, uint32_t b, uint32_t nb, float* x) {
    const uint32_t s0 = a.bstart[b], s1 = a.bstart[b + 1];
    const uint32_t L = s1 - s0;
    const uint32_t Lp = b > 0 ? s0 - a.bstart[b - 1] : L;
    const uint32_t Ln = b + 1 < nb ? a.bstart[b + 2] - s1 : L;
    float om = 0.0f, ox = 0.0f, em = 0.0f, en = 1e30f;
    const uint32_t k = L < 8u ? L : 8u;
    const float inv = 1.0f / a.p.res;
    for (uint32_t i = 0; i < k; i++) {
        const VoxRec g = a.rec[a.vals[s0 + (uint32_t)(((uint64_t)i * L) / k)]];
        om += g.opacity;
        ox = fmaxf(ox, g.opacity);
        const float e = log1pf(((g.ehx + g.ehy) + g.ehz) * (1.0f / 3.0f) * inv);
        em += e;
        en = fminf(en, e);
    }
    const float ik = k ? 1.0f / (float)k : 0.0f;
    const uint32_t key = a.bkey[b];
    const uint32_t batch = key >> 12, bi = key & 4095u;
    const int64_t NBX = a.p.NBB[0], NBY = a.p.NBB[1];
    const int64_t bxI = batch % NBX, byI = (batch / NBX) % NBY;
    const int64_t cx = min((int64_t)16, a.p.NB[0] - bxI * 16), cy = min((int64_t)16, a.p.NB[1] - byI * 16);
    x[0] = log1pf((float)L) * 0.1f;
    x[1] = log1pf((float)Lp) * 0.1f;
    x[2] = log1pf((float)Ln) * 0.1f;
    x[3] = om * ik;
    x[4] = ox;
    x[5] = em * ik;
    x[6] = k ? en : 0.0f;
    x[7] = log1pf((float)L / 64.0f);
    x[8] = (float)(bi % cx) * (1.0f / 16.0f);
    x[9] = (float)((bi / cx) % cy) * (1.0f / 16.0f);
    x[10] = (float)(bi / (cx * cy)) * (1.0f / 16.0f);
    x[11] = a.p.cutoff;
}

constexpr int kVSchedThreads = 128;
__global__ void __launch_bounds__(kVSchedThreads) vox_sched_pred_k(VoxSchedArgs a) {
    __shared__ float P[dlmlp::kParams];
    if (a.w) dlmlp::load_params(a.w, P);
    const uint32_t nb = (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT) ? 0u : *a.nblocks;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        float x[12];
        vox_block_features(a, b, nb, x);
        if (a.feat)
            for (int i = 0; i < 12; i++) a.feat[(uint64_t)b * 12 + i] = x[i];
        if (a.w) {
            const float y = dlmlp::forward(P, x, nullptr, nullptr);
            const float q = (y == y) ? fminf(fmaxf((y + 4.0f) * 32.0f, 0.0f), 255.0f) : 0.0f;
            const uint32_t bk = 255u - (uint32_t)q;                  // 0 = most expensive
            a.bucket[b] = bk;
            atomicAdd(&a.hist[bk], 1u);
        }
    }
}

__global__ void vox_sched_scan_k(uint32_t* hist) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < 256; i++) { const uint32_t c = hist[i]; hist[i] = acc; acc += c; }
    }
}

__global__ void vox_sched_scatter_k(VoxSchedArgs a) {
    const uint32_t nb = (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT) ? 0u : *a.nblocks;
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
        a.work[atomicAdd(&a.hist[a.bucket[b]], 1u)] = b;
}

// Keep non-zero masks, in block order; write flat indices (voxelize.ts:170-177).
struct CompactArgs {
    VoxParams p;
    const uint32_t* bkey;
    const uint2* masks;
    const uint32_t* nblocks;
    uint32_t* out_idx;
    uint32_t* out_lo;
    uint32_t* out_hi;
    uint32_t* nout;
    unsigned long long* status;
    uint32_t* counter;
    uint32_t* err;
    uint32_t spin_limit;
};

__global__ void __launch_bounds__(kVT) vox_compact_k(CompactArgs a) {
    __shared__ uint32_t s_wsum[kVT / 32];
    __shared__ uint32_t s_tile;
    __shared__ unsigned long long s_pre;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (__syncthreads_or(tid == 0 && (dl_ld_volatile(a.err) & DL_DEVERR_TIMEOUT))) {
        if (blockIdx.x == 0 && tid == 0) *a.nout = 0;
        return;
    }
    if (tid == 0) s_tile = atomicAdd(a.counter, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    const uint32_t n = *a.nblocks;
    const uint32_t i0 = tile * kVR;
    if (i0 >= n) {
        if (tile == 0 && tid == 0) *a.nout = 0;
        return;
    }
    uint32_t keep[kVI], local = 0;
    uint2 m[kVI];
#pragma unroll
    for (int j = 0; j < kVI; j++) {
        const uint32_t i = i0 + tid * kVI + j;
        m[j] = i < n ? a.masks[i] : make_uint2(0, 0);
        keep[j] = (m[j].x | m[j].y) ? 1u : 0u;
        local += keep[j];
    }
    uint32_t inc = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) s_wsum[warp] = inc;
    __syncthreads();
    uint32_t wpre = 0, total = 0;
    for (int w = 0; w < kVT / 32; w++) { if (w < warp) wpre += s_wsum[w]; total += s_wsum[w]; }
    if (warp == 0) {
        const unsigned long long pre = lookback_warp(a.status, tile, total, a.err, a.spin_limit);
        if (lane == 0) {
            s_pre = pre;
            if (i0 + kVR >= n) *a.nout = (uint32_t)(pre + total);
        }
    }
    __syncthreads();
    uint32_t run = (uint32_t)s_pre + wpre + inc - local;
    const int64_t NX = a.p.NB[0], NY = a.p.NB[1], NBX = a.p.NBB[0], NBY = a.p.NBB[1];
#pragma unroll
    for (int j = 0; j < kVI; j++) {
        if (keep[j]) {
            const uint32_t key = a.bkey[i0 + tid * kVI + j];
            const uint32_t batch = key >> 12, bi = key & 4095u;
            const int64_t bxI = batch % NBX, byI = (batch / NBX) % NBY, bzI = batch / (NBX * NBY);
            const int64_t cx = min((int64_t)16, NX - bxI * 16), cy = min((int64_t)16, NY - byI * 16);
            const int64_t ax = bxI * 16 + bi % cx, ay = byI * 16 + (bi / cx) % cy, az = bzI * 16 + bi / (cx * cy);
            a.out_idx[run] = (uint32_t)(ax + ay * NX + az * NX * NY);
            a.out_lo[run] = m[j].x;
            a.out_hi[run] = m[j].y;
            run++;
        }
    }
}

double js_round(double x) {
    if (!std::isfinite(x)) return x;
    const double f = std::floor(x);
    return (x - f >= 0.5) ? f + 1.0 : f;
}

}  // namespace

// The voxelizer's grow-only device buffers, kept on the device between calls.
struct VoxBufs {
    std::shared_ptr<PinnedPool> pinned = std::make_shared<PinnedPool>();
    std::vector<DevBuf*> all;
    DevBuf scene, ext, rec, part, bounds, axes, scratch, keys0, keys1, vals0, vals1, status, hist, segs, bkey, bstart,
        masks, oidx, olo, ohi, used, bcount, sfeat, sbucket, shist, swork, scycles;
    VoxBufs() {
        DevBuf* l[] = {&scene, &ext, &rec, &part, &bounds, &axes, &scratch, &keys0, &keys1, &vals0, &vals1, &status,
                       &hist, &segs, &bkey, &bstart, &masks, &oidx, &olo, &ohi, &used, &bcount, &sfeat, &sbucket,
                       &shist, &swork, &scycles};
        all.assign(l, l + sizeof(l) / sizeof(l[0]));
    }
    ~VoxBufs() { for (DevBuf* b : all) b->release(); }
};

void dl_vox_release(dl_device* dev) {
    delete dev->vox;
    dev->vox = nullptr;
}

namespace {

enum { VS_EMIT = 0, VS_SORT = 1, VS_HEADS = 5, VS_EVAL = 6, VS_COMPACT = 7, VS_ERR = 8, VS_OVF = 9, VS_TILES = 10,
       VS_NBLK = 11, VS_NOUT = 12, VS_WORDS = 16 };

}  // namespace

extern "C" int dl_voxelize(dl_device* dev, const dl_splats* data, const dl_vox_opts* opts, dl_vox_result** out) {
    if (!dev || !data || !out) { dl_set_error("dl_voxelize: NULL argument"); return DL_E_INVALID_ARG; }
    *out = nullptr;
    const double voxelRes = (opts && !opts->use_defaults) ? opts->voxel_resolution : 0.05;
    const double cutoffD = (opts && !opts->use_defaults) ? opts->opacity_cutoff : 0.1;
    if (!(voxelRes > 0.0) || !std::isfinite(voxelRes)) { dl_set_error("voxelResolution must be > 0"); return DL_E_INVALID_ARG; }
    const uint64_t n = data->count;
    if (n >= (1ull << 30)) { dl_set_error("at most 2^30 - 1 Gaussians"); return DL_E_CAPACITY; }
    if (n && (!data->positions || !data->rotations || !data->log_scales || !data->opacity_logits)) {
        dl_set_error("splats: a required array is NULL");
        return DL_E_INVALID_ARG;
    }
    DL_CK(cudaSetDevice(dev->ordinal));
    cudaStream_t st = dev->stream;
    dl_vox_result* R = new dl_vox_result();
    if (!dev->vox) dev->vox = new VoxBufs();
    VoxBufs& B = *dev->vox;
    const bool logBlocks = opts && opts->log_blocks;
    const bool fastExp = opts && (opts->flags & DL_VOX_FAST_EXP);
    VoxMarks marks;
    marks.on = opts && (opts->flags & DL_VOX_PROFILE);
    marks.st = st;
    marks.mark(0);
    const double blockSize = 4 * voxelRes;
    VoxParams p;
    std::memset(&p, 0, sizeof(p));
    p.n = (uint32_t)n;
    p.res = (float)voxelRes;
    p.half = p.res * 0.5f;
    p.cutoff = (float)cutoffD;
    p.blockSize = blockSize;
    // (a failed call waits for copies still in flight into R's buffer first)
    auto fail = [&](int code) { cudaStreamSynchronize(st); delete R; return code; };
    R->pool = B.pinned;
    {
        void* q = nullptr;
        B.pinned->take(&q, &R->pinned_cap);
        R->pinned = static_cast<uint32_t*>(q);
    }

    // ---- upload + per-Gaussian prep + bounds
    const uint64_t oRot = (12 * n + 255) / 256 * 256, oLsc = oRot + (16 * n + 255) / 256 * 256;
    const uint64_t oOpl = oLsc + (12 * n + 255) / 256 * 256, total = oOpl + (4 * n + 255) / 256 * 256;
    int s;
    if ((s = B.scene.ensure(total + 256)) != DL_OK) return fail(s);
    char* sb = B.scene.as<char>();
    double bnd[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
    const uint32_t prepGrid = (uint32_t)std::max<uint64_t>(1, (n + 255) / 256);
    if (n) {
        if (cudaMemcpyAsync(sb, data->positions, 12 * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(sb + oRot, data->rotations, 16 * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(sb + oLsc, data->log_scales, 12 * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(sb + oOpl, data->opacity_logits, 4 * n, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            dl_set_error("voxelize: upload failed");
            return fail(DL_E_CUDA);
        }
        p.pos = (const float*)sb; p.rot = (const float*)(sb + oRot);
        p.lsc = (const float*)(sb + oLsc); p.opl = (const float*)(sb + oOpl);
        if ((s = B.ext.ensure(12 * n)) != DL_OK || (s = B.rec.ensure(sizeof(VoxRec) * n)) != DL_OK ||
            (s = B.part.ensure(48ull * prepGrid)) != DL_OK || (s = B.bounds.ensure(64)) != DL_OK)
            return fail(s);
        vox_prep_k<<<prepGrid, 256, 0, st>>>(p, B.ext.as<float>(), B.rec.as<VoxRec>(), B.part.as<double>());
        vox_bounds_k<<<1, 32, 0, st>>>(B.part.as<double>(), prepGrid, B.bounds.as<double>());
        if (cudaMemcpyAsync(bnd, B.bounds.p, 48, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            dl_set_error(std::string("voxelize prep: ") + cudaGetErrorString(cudaGetLastError()));
            return fail(DL_E_CUDA);
        }
    }
    // voxelize.ts:73-76 and computeBlockAlignedBounds (:278-306)
    if (opts && opts->has_bounds) {
        for (int k = 0; k < 3; k++) { R->bmin[k] = opts->bounds_min[k]; R->bmax[k] = opts->bounds_max[k]; }
    } else {
        for (int k = 0; k < 3; k++) {
            R->bmin[k] = std::floor(bnd[k] / blockSize) * blockSize;
            R->bmax[k] = std::ceil(bnd[3 + k] / blockSize) * blockSize;
        }
    }
    for (int k = 0; k < 3; k++) R->dims[k] = js_round((R->bmax[k] - R->bmin[k]) / blockSize);
    const int shardCount = (opts && opts->shard_count > 1) ? opts->shard_count : 1;
    const int shardIndex = shardCount > 1 ? opts->shard_index : 0;
    if (shardIndex < 0 || shardIndex >= shardCount) { dl_set_error("voxelize: shard_index out of range"); return fail(DL_E_INVALID_ARG); }
    const bool anyBlocks = n > 0 && R->dims[0] > 0 && R->dims[1] > 0 && R->dims[2] > 0;
    if (!anyBlocks) { *out = R; return DL_OK; }
    for (int k = 0; k < 3; k++) {
        if (R->dims[k] > 4.0e6) { dl_set_error("voxel grid too large"); return fail(DL_E_CAPACITY); }
        p.NB[k] = (int64_t)R->dims[k];
        p.NBB[k] = (p.NB[k] + 15) / 16;
        p.boundsMin[k] = R->bmin[k];
    }
    const uint64_t numBatches = (uint64_t)p.NBB[0] * p.NBB[1] * p.NBB[2];
    if (numBatches >= (1ull << 20) || (double)p.NB[0] * p.NB[1] * p.NB[2] >= 4294967296.0) {
        dl_set_error("voxel grid too large: at most 2^20 16^3-block batches and 2^32 blocks");
        return fail(DL_E_CAPACITY);
    }
    // per-axis batch boxes (voxelize.ts:193-198) and f32 batch minima (BatchInfo)
    {
        const uint64_t na = p.NBB[0] + p.NBB[1] + p.NBB[2];
        std::vector<double> hq(2 * na);
        std::vector<float> hf(na);
        uint64_t o = 0;
        for (int k = 0; k < 3; k++) {
            for (int64_t b = 0; b < p.NBB[k]; b++) {
                const double mn = R->bmin[k] + (double)(b * 16) * blockSize;
                const double cnt = (double)std::min<int64_t>(16, p.NB[k] - b * 16);
                hq[o + b] = mn;
                hq[na + o + b] = mn + cnt * blockSize;
                hf[o + b] = (float)mn;
            }
            o += p.NBB[k];
        }
        if ((s = B.axes.ensure(2 * na * 8 + na * 4 + 256)) != DL_OK) return fail(s);
        double* dq = B.axes.as<double>();
        float* df = (float*)(dq + 2 * na);
        if (cudaMemcpyAsync(dq, hq.data(), 2 * na * 8, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(df, hf.data(), na * 4, cudaMemcpyHostToDevice, st) != cudaSuccess) {
            dl_set_error("voxelize: upload failed");
            return fail(DL_E_CUDA);
        }
        o = 0;
        for (int k = 0; k < 3; k++) {
            p.qmn[k] = dq + o; p.qmx[k] = dq + na + o; p.bmin32[k] = df + o;
            o += p.NBB[k];
        }
    }
    if ((s = B.scratch.ensure(4 * VS_WORDS)) != DL_OK) return fail(s);
    uint32_t* scr = B.scratch.as<uint32_t>();

    // ---- slabs of 16-block z rows of batches, each within the pair capacity.
    // Blocks are appended in batch order (z rows outermost), so processing the
    // rows in order and concatenating reproduces the reference's block order.
    // (DL_VOX_SLAB_PAIRS lowers the capacity, to exercise the slab loop on small inputs.)
    unsigned long long kSlabCap = (1ull << 30) - 1;
    if (const char* env = std::getenv("DL_VOX_SLAB_PAIRS")) {
        const unsigned long long e = std::strtoull(env, nullptr, 10);
        if (e > 0 && e < kSlabCap) kSlabCap = e;
    }
    // ---- cutoff <= 0: 1 - exp(-sigma) >= cutoff holds for every voxel, so every
    // voxel of every batch with a non-empty batch list is solid
    if (!(p.cutoff > 0.0f) && p.cutoff <= 0.0f) {
        DevBuf& usedD = B.used;
        if ((s = usedD.ensure(4ull * numBatches)) != DL_OK) return fail(s);
        cudaMemsetAsync(usedD.p, 0, 4ull * numBatches, st);
        vox_batchused_k<<<prepGrid, 256, 0, st>>>(p, B.ext.as<float>(), usedD.as<uint32_t>());
        std::vector<uint32_t> used(numBatches, 0);
        if (cudaMemcpyAsync(used.data(), usedD.p, 4ull * numBatches, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            dl_set_error(std::string("voxelize: ") + cudaGetErrorString(cudaGetLastError()));
            return fail(DL_E_CUDA);
        }
        // shards: z rows split evenly by count
        const int64_t zr0 = p.NBB[2] * shardIndex / shardCount, zr1 = p.NBB[2] * (shardIndex + 1) / shardCount;
        for (uint64_t b = 0; b < numBatches; b++) {
            if (!used[b]) continue;
            const int64_t bxI = b % p.NBB[0], byI = (b / p.NBB[0]) % p.NBB[1], bzI = b / (p.NBB[0] * p.NBB[1]);
            if (bzI < zr0 || bzI >= zr1) continue;
            const int64_t cx = std::min<int64_t>(16, p.NB[0] - bxI * 16), cy = std::min<int64_t>(16, p.NB[1] - byI * 16);
            const int64_t cz = std::min<int64_t>(16, p.NB[2] - bzI * 16);
            for (int64_t bi = 0; bi < cx * cy * cz; bi++) {
                const int64_t ax = bxI * 16 + bi % cx, ay = byI * 16 + (bi / cx) % cy, az = bzI * 16 + bi / (cx * cy);
                R->idx.push_back((uint32_t)(ax + ay * p.NB[0] + az * p.NB[0] * p.NB[1]));
                R->lo.push_back(0xffffffffu);
                R->hi.push_back(0xffffffffu);
            }
        }
        *out = R;
        return DL_OK;
    }
    const int64_t NBX_ = p.NBB[0], NBY_ = p.NBB[1], NBZ_ = p.NBB[2];
    std::vector<unsigned long long> bc((size_t)(NBX_ * NBY_ * NBZ_), 0ull);     // pairs per batch
    {
        DevBuf& cnt = B.bcount;
        if ((s = cnt.ensure(8ull * bc.size())) != DL_OK) return fail(s);
        cudaMemsetAsync(cnt.p, 0, 8ull * bc.size(), st);
        p.zlo = 0; p.zhi = p.NB[2] - 1;
        p.ylo = 0; p.yhi = p.NB[1] - 1;
        p.xlo = 0; p.xhi = p.NB[0] - 1;
        vox_batchcount_k<<<prepGrid, 256, 0, st>>>(p, B.ext.as<float>(), cnt.as<unsigned long long>());
        if (cudaMemcpyAsync(bc.data(), cnt.p, 8ull * bc.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            dl_set_error(std::string("voxelize count: ") + cudaGetErrorString(cudaGetLastError()));
            return fail(DL_E_CUDA);
        }
    }
    marks.mark(0);
    // A slab is a box of batches contiguous in batch order: whole z rows, or
    // whole y rows of one z row, or a range of batches of one (z, y) row.
    struct Slab { int64_t z0, z1, y0, y1, x0, x1; unsigned long long pairs; };
    std::vector<Slab> slabs;
    {
        auto rowSum = [&](int64_t z, int64_t y) {
            unsigned long long a = 0;
            for (int64_t x = 0; x < NBX_; x++) a += bc[(z * NBY_ + y) * NBX_ + x];
            return a;
        };
        // this shard's z rows: contiguous, about 1/shardCount of all pairs each
        int64_t zr0 = 0, zr1 = NBZ_;
        if (shardCount > 1) {
            std::vector<unsigned long long> before((size_t)NBZ_ + 1, 0ull);
            for (int64_t z = 0; z < NBZ_; z++) {
                unsigned long long zs = 0;
                for (int64_t y = 0; y < NBY_; y++) zs += rowSum(z, y);
                before[z + 1] = before[z] + zs;
            }
            auto boundary = [&](int i) -> int64_t {
                if (i <= 0) return 0;
                if (i >= shardCount) return NBZ_;
                const unsigned long long target = (unsigned long long)((double)before[NBZ_] * i / shardCount);
                int64_t z = 0;
                while (z < NBZ_ && before[z] < target) z++;
                return z;
            };
            zr0 = boundary(shardIndex);
            zr1 = std::max(zr0, boundary(shardIndex + 1));
        }
        Slab cur{zr0, zr0, 0, NBY_, 0, NBX_, 0};                 // whole z rows being merged
        for (int64_t z = zr0; z < zr1; z++) {
            unsigned long long zs = 0;
            for (int64_t y = 0; y < NBY_; y++) zs += rowSum(z, y);
            if (zs <= kSlabCap) {
                if (cur.z1 > cur.z0 && cur.pairs + zs > kSlabCap) { slabs.push_back(cur); cur = {z, z, 0, NBY_, 0, NBX_, 0}; }
                if (cur.z1 == cur.z0) cur.z0 = z;
                cur.z1 = z + 1;
                cur.pairs += zs;
                continue;
            }
            if (cur.z1 > cur.z0) slabs.push_back(cur);
            Slab yr{z, z + 1, 0, 0, 0, NBX_, 0};                  // whole y rows of this z row
            for (int64_t y = 0; y < NBY_; y++) {
                const unsigned long long ys = rowSum(z, y);
                if (ys <= kSlabCap) {
                    if (yr.y1 > yr.y0 && yr.pairs + ys > kSlabCap) { slabs.push_back(yr); yr = {z, z + 1, y, y, 0, NBX_, 0}; }
                    if (yr.y1 == yr.y0) yr.y0 = y;
                    yr.y1 = y + 1;
                    yr.pairs += ys;
                    continue;
                }
                if (yr.y1 > yr.y0) slabs.push_back(yr);
                Slab xr{z, z + 1, y, y + 1, 0, 0, 0};             // batches of this (z, y) row
                for (int64_t x = 0; x < NBX_; x++) {
                    const unsigned long long c = bc[(z * NBY_ + y) * NBX_ + x];
                    if (c > (1ull << 30) - 1) {
                        dl_set_error("one 16^3-block batch needs 2^30 or more Gaussian-block pairs");
                        return fail(DL_E_CAPACITY);
                    }
                    if (xr.x1 > xr.x0 && xr.pairs + c > kSlabCap) { slabs.push_back(xr); xr = {z, z + 1, y, y + 1, x, x, 0}; }
                    xr.x1 = x + 1;
                    xr.pairs += c;
                }
                slabs.push_back(xr);
                yr = {z, z + 1, y + 1, y + 1, 0, NBX_, 0};
            }
            if (yr.y1 > yr.y0) slabs.push_back(yr);
            cur = {z + 1, z + 1, 0, NBY_, 0, NBX_, 0};
        }
        if (cur.z1 > cur.z0) slabs.push_back(cur);
    }
    const uint32_t emitTiles = (uint32_t)((n + kVR - 1) / kVR);
    int keyBits = 12;
    while ((1ull << (keyBits - 12)) < numBatches) keyBits++;
    const int passes = (keyBits + 7) / 8;
    for (const Slab& slab : slabs) {
        const unsigned long long cap = slab.pairs;
        if (cap == 0) continue;
        marks.mark(6);
        p.zlo = slab.z0 * 16;
        p.zhi = std::min<int64_t>(slab.z1 * 16, p.NB[2]) - 1;
        p.ylo = slab.y0 * 16;
        p.yhi = std::min<int64_t>(slab.y1 * 16, p.NB[1]) - 1;
        p.xlo = slab.x0 * 16;
        p.xhi = std::min<int64_t>(slab.x1 * 16, p.NB[0]) - 1;
        // ---- binning (exactly `cap` pairs)
        if ((s = B.keys0.ensure(4 * cap)) != DL_OK || (s = B.vals0.ensure(4 * cap)) != DL_OK ||
            (s = B.status.ensure(8ull * std::max<uint64_t>(emitTiles, 1))) != DL_OK)
            return fail(s);
        cudaMemsetAsync(scr, 0, 4 * VS_WORDS, st);
        cudaMemsetAsync(B.status.p, 0, 8ull * emitTiles, st);
        VoxEmitArgs ea;
        ea.p = p; ea.ext = B.ext.as<float>(); ea.keys = B.keys0.as<uint32_t>(); ea.vals = B.vals0.as<uint32_t>();
        ea.cap = cap; ea.npairs = (unsigned long long*)(scr + 14); ea.status = B.status.as<unsigned long long>();
        ea.counter = scr + VS_EMIT; ea.err = scr + VS_ERR; ea.ovf = scr + VS_OVF;
        ea.spin_limit = g_dl_wait.spin_limit;
        vox_emit_k<<<emitTiles, kVT, 0, st>>>(ea);
        marks.mark(1);
        unsigned long long npairs = 0;
        {
            uint32_t h[16];
            if (cudaMemcpyAsync(h, scr, 64, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaStreamSynchronize(st) != cudaSuccess) {
                dl_set_error(std::string("voxelize binning: ") + cudaGetErrorString(cudaGetLastError()));
                return fail(DL_E_CUDA);
            }
            if (h[VS_ERR] & DL_DEVERR_TIMEOUT) { dl_set_error("a bounded device-side wait timed out"); return fail(DL_E_TIMEOUT); }
            if (h[VS_OVF] & 4u) { dl_set_error("a Gaussian overlaps more than 2^31 blocks"); return fail(DL_E_CAPACITY); }
            if (h[VS_OVF] & DL_DEVERR_OVERFLOW) { dl_set_error("voxelize: binning disagrees with its count"); return fail(DL_E_CAPACITY); }
            std::memcpy(&npairs, &h[14], 8);
        }

        // ---- stable sort by block key
        const uint32_t sortTiles = (uint32_t)std::max<unsigned long long>(1, (npairs + dlsort::kTile - 1) / dlsort::kTile);
        if ((s = B.keys1.ensure(4 * std::max<unsigned long long>(npairs, 1))) != DL_OK ||
            (s = B.vals1.ensure(4 * std::max<unsigned long long>(npairs, 1))) != DL_OK ||
            (s = B.status.ensure(std::max<uint64_t>(4ull * 256 * sortTiles, 8ull * ((npairs + kVR - 1) / kVR + 1)))) != DL_OK ||
            (s = B.hist.ensure(4ull * 4 * 256)) != DL_OK || (s = B.segs.ensure(64)) != DL_OK)
            return fail(s);
        uint32_t* keysF = B.keys0.as<uint32_t>();
        uint32_t* valsF = B.vals0.as<uint32_t>();
        if (npairs > 0) {
            uint64_t* segStart = B.segs.as<uint64_t>();
            uint32_t* segLen = (uint32_t*)(segStart + 1);
            uint32_t* segTileBase = segLen + 1;
            cudaMemsetAsync(segStart, 0, 8, st);
            const uint32_t len32 = (uint32_t)npairs;
            cudaMemcpyAsync(segLen, &len32, 4, cudaMemcpyHostToDevice, st);
            dlsort::Segs sg;
            sg.start = segStart; sg.len = segLen; sg.tile_base = segTileBase; sg.total_tiles = scr + VS_TILES; sg.num = 1;
            dlsort::prepare_k<<<1, 32, 0, st>>>(sg);
            cudaMemsetAsync(B.hist.p, 0, 4ull * 4 * 256, st);
            dlsort::hist_k<8><<<std::min<uint32_t>(sortTiles, 4096), dlsort::kThreads, 0, st>>>(keysF, sg, passes, 0, B.hist.as<uint32_t>());
            dlsort::scan_hist_k<8><<<passes, 256, 0, st>>>(B.hist.as<uint32_t>(), passes);
            uint32_t *kin = keysF, *kout = B.keys1.as<uint32_t>(), *vin = valsF, *vout = B.vals1.as<uint32_t>();
            for (int ps = 0; ps < passes; ps++) {
                cudaMemsetAsync(B.status.p, 0, 4ull * 256 * sortTiles, st);
                dlsort::Pass sp;
                sp.keys_in = kin; sp.vals_in = vin; sp.keys_out = kout; sp.vals_out = vout; sp.segs = sg;
                sp.glob_off = B.hist.as<uint32_t>(); sp.status = B.status.as<uint32_t>(); sp.counter = scr + VS_SORT + ps;
                sp.err = scr + VS_ERR; sp.shift = 8 * ps; sp.pass = ps; sp.passes = passes;
                sp.spin_limit = g_dl_wait.spin_limit;
                dlsort::pass_k<8><<<dlsort::pass_grid(sortTiles), dlsort::kThreads, 0, st>>>(sp);
                std::swap(kin, kout);
                std::swap(vin, vout);
            }
            keysF = kin;
            valsF = vin;
        }
        marks.mark(2);
        // ---- blocks, evaluation, compaction
        const uint64_t maxBlocks = std::max<unsigned long long>(npairs, 1);
        if ((s = B.bkey.ensure(4 * maxBlocks)) != DL_OK || (s = B.bstart.ensure(4 * (maxBlocks + 1))) != DL_OK ||
            (s = B.masks.ensure(8 * maxBlocks)) != DL_OK)
            return fail(s);
        const uint32_t headTiles = (uint32_t)std::max<unsigned long long>(1, (npairs + kHR - 1) / kHR);
        cudaMemsetAsync(B.status.p, 0, 8ull * headTiles, st);
        HeadsArgs ha;
        ha.keys = keysF; ha.npairs = (const unsigned long long*)(scr + 14); ha.bkey = B.bkey.as<uint32_t>();
        ha.bstart = B.bstart.as<uint32_t>(); ha.nblocks = scr + VS_NBLK; ha.status = B.status.as<unsigned long long>();
        ha.counter = scr + VS_HEADS; ha.err = scr + VS_ERR; ha.spin_limit = g_dl_wait.spin_limit;
        vox_heads_k<<<headTiles, kVT, 0, st>>>(ha);

        // learned block order (and per-block features for cost logging)
        const uint32_t* work = nullptr;
        if (dev->vox_sched || logBlocks) {
            if ((s = B.sbucket.ensure(4 * maxBlocks)) != DL_OK || (s = B.swork.ensure(4 * maxBlocks)) != DL_OK ||
                (s = B.shist.ensure(1024)) != DL_OK ||
                (logBlocks && ((s = B.sfeat.ensure(48 * maxBlocks)) != DL_OK || (s = B.scycles.ensure(4 * maxBlocks)) != DL_OK)))
                return fail(s);
            VoxSchedArgs sa;
            sa.p = p; sa.rec = B.rec.as<VoxRec>(); sa.vals = valsF; sa.bkey = B.bkey.as<uint32_t>();
            sa.bstart = B.bstart.as<uint32_t>(); sa.nblocks = scr + VS_NBLK;
            sa.w = dev->vox_sched ? (const __nv_bfloat16*)dl_mlp_weights(dev->vox_sched) : nullptr;
            sa.feat = logBlocks ? B.sfeat.as<float>() : nullptr;
            sa.bucket = B.sbucket.as<uint32_t>(); sa.hist = B.shist.as<uint32_t>(); sa.work = B.swork.as<uint32_t>();
            sa.err = scr + VS_ERR;
            const uint32_t sg = (uint32_t)std::min<uint64_t>((maxBlocks + kVSchedThreads - 1) / kVSchedThreads, 4096);
            if (sa.w) cudaMemsetAsync(B.shist.p, 0, 1024, st);
            vox_sched_pred_k<<<sg, kVSchedThreads, 0, st>>>(sa);
            if (sa.w) {
                vox_sched_scan_k<<<1, 32, 0, st>>>(sa.hist);
                vox_sched_scatter_k<<<sg, kVSchedThreads, 0, st>>>(sa);
                work = sa.work;
            }
        }
        marks.mark(3);
        EvalArgs va;
        va.p = p; va.rec = B.rec.as<VoxRec>(); va.vals = valsF; va.bkey = B.bkey.as<uint32_t>();
        va.bstart = B.bstart.as<uint32_t>(); va.nblocks = scr + VS_NBLK; va.masks = B.masks.as<uint2>();
        va.counter = scr + VS_EVAL;
        va.work = work; va.cycles = logBlocks ? B.scycles.as<uint32_t>() : nullptr; va.err = scr + VS_ERR;
        if (fastExp) vox_eval_k<true><<<dev->sm_count * 32, 64, 0, st>>>(va);
        else vox_eval_k<false><<<dev->sm_count * 32, 64, 0, st>>>(va);

        marks.mark(4);
        uint32_t hn[2] = {0, 0};
        if (cudaMemcpyAsync(hn, scr + VS_NBLK, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            dl_set_error(std::string("voxelize eval: ") + cudaGetErrorString(cudaGetLastError()));
            return fail(DL_E_CUDA);
        }
        const uint32_t nblk = hn[0];
        if (logBlocks && nblk) {
            const size_t f0 = R->log_cost.size();
            R->log_feat.resize((f0 + nblk) * 12);
            R->log_cost.resize(f0 + nblk);
            std::vector<uint32_t> cyc(nblk);
            if (cudaMemcpy(R->log_feat.data() + f0 * 12, B.sfeat.p, 48ull * nblk, cudaMemcpyDeviceToHost) != cudaSuccess ||
                cudaMemcpy(cyc.data(), B.scycles.p, 4ull * nblk, cudaMemcpyDeviceToHost) != cudaSuccess) {
                dl_set_error("voxelize: block log copy failed");
                return fail(DL_E_CUDA);
            }
            for (uint32_t i = 0; i < nblk; i++) R->log_cost[f0 + i] = (float)cyc[i];
        }
        if ((s = B.oidx.ensure(4ull * std::max<uint32_t>(nblk, 1))) != DL_OK ||
            (s = B.olo.ensure(4ull * std::max<uint32_t>(nblk, 1))) != DL_OK ||
            (s = B.ohi.ensure(4ull * std::max<uint32_t>(nblk, 1))) != DL_OK)
            return fail(s);
        const uint32_t compTiles = std::max<uint32_t>(1, (nblk + kVR - 1) / kVR);
        cudaMemsetAsync(B.status.p, 0, 8ull * compTiles, st);
        CompactArgs ca;
        ca.p = p; ca.bkey = B.bkey.as<uint32_t>(); ca.masks = B.masks.as<uint2>(); ca.nblocks = scr + VS_NBLK;
        ca.out_idx = B.oidx.as<uint32_t>(); ca.out_lo = B.olo.as<uint32_t>(); ca.out_hi = B.ohi.as<uint32_t>();
        ca.nout = scr + VS_NOUT; ca.status = B.status.as<unsigned long long>(); ca.counter = scr + VS_COMPACT;
        ca.err = scr + VS_ERR; ca.spin_limit = g_dl_wait.spin_limit;
        vox_compact_k<<<compTiles, kVT, 0, st>>>(ca);
        marks.mark(5);
        uint32_t h2[16];
        if (cudaMemcpyAsync(h2, scr, 64, cudaMemcpyDeviceToHost, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
            dl_set_error(std::string("voxelize compact: ") + cudaGetErrorString(cudaGetLastError()));
            return fail(DL_E_CUDA);
        }
        if (h2[VS_ERR] & DL_DEVERR_TIMEOUT) { dl_set_error("a bounded device-side wait timed out"); return fail(DL_E_TIMEOUT); }
        const uint32_t nout = h2[VS_NOUT];
        if (nout) {
            // this slab's lists go to the pinned buffer behind the earlier
            // slabs' (asynchronously: the next slab's kernels queue behind the
            // copies on the same stream, so B.oidx/olo/ohi are not overwritten early)
            const uint64_t need = 4ull * (R->pinned_used + 3ull * nout);
            if (need > R->pinned_cap) {
                if (cudaStreamSynchronize(st) != cudaSuccess) {
                    dl_set_error(std::string("voxelize: ") + cudaGetErrorString(cudaGetLastError()));
                    return fail(DL_E_CUDA);
                }
                const size_t nc = std::max<size_t>(need + need / 2, 16u << 20);
                void* q = nullptr;
                if (cudaHostAlloc(&q, nc, cudaHostAllocDefault) != cudaSuccess) {
                    dl_set_error("voxelize: cudaHostAlloc(" + std::to_string(nc) + ") for the block lists failed");
                    return fail(DL_E_OOM);
                }
                if (R->pinned_used) std::memcpy(q, R->pinned, 4ull * R->pinned_used);
                if (R->pinned) cudaFreeHost(R->pinned);
                R->pinned = static_cast<uint32_t*>(q);
                R->pinned_cap = nc;
            }
            uint32_t* dst = R->pinned + R->pinned_used;
            if (cudaMemcpyAsync(dst, B.oidx.p, 4ull * nout, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaMemcpyAsync(dst + nout, B.olo.p, 4ull * nout, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaMemcpyAsync(dst + 2ull * nout, B.ohi.p, 4ull * nout, cudaMemcpyDeviceToHost, st) != cudaSuccess) {
                dl_set_error("voxelize: result copy failed");
                return fail(DL_E_CUDA);
            }
            R->segs.emplace_back(R->pinned_used, nout);
            R->pinned_used += 3ull * nout;
            R->pinned_count += nout;
        }
    }
    marks.mark(6);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        dl_set_error(std::string("voxelize: ") + cudaGetErrorString(cudaGetLastError()));
        return fail(DL_E_CUDA);
    }
    marks.finish(R->stage_ms);
    *out = R;
    return DL_OK;
}

extern "C" int dl_vox_result_stage_times(const dl_vox_result* r, double* ms, int n) {
    if (!r || !ms) { dl_set_error("dl_vox_result_stage_times: NULL argument"); return DL_E_INVALID_ARG; }
    for (int i = 0; i < n && i < 7; i++) ms[i] = r->stage_ms[i];
    return DL_OK;
}

extern "C" int dl_vox_result_info(const dl_vox_result* r, double bmin[3], double bmax[3], double dims[3],
                                  uint64_t* count) {
    if (!r) { dl_set_error("result is NULL"); return DL_E_INVALID_ARG; }
    for (int k = 0; k < 3; k++) {
        if (bmin) bmin[k] = r->bmin[k];
        if (bmax) bmax[k] = r->bmax[k];
        if (dims) dims[k] = r->dims[k];
    }
    if (count) *count = r->idx.size() + r->pinned_count;
    return DL_OK;
}

extern "C" int dl_vox_result_copy(const dl_vox_result* r, uint32_t* idx, uint32_t* lo, uint32_t* hi) {
    if (!r) { dl_set_error("result is NULL"); return DL_E_INVALID_ARG; }
    const size_t n = r->idx.size();
    if (n && idx) std::memcpy(idx, r->idx.data(), 4 * n);
    if (n && lo) std::memcpy(lo, r->lo.data(), 4 * n);
    if (n && hi) std::memcpy(hi, r->hi.data(), 4 * n);
    if (!r->pinned_count) return DL_OK;
    // the device's lists, slab by slab after the host-built ones; the three
    // arrays are gathered by three threads when they are large
    auto gather = [r, n](uint32_t* dst, int which) {
        if (!dst) return;
        uint64_t o = n;
        for (const auto& sg : r->segs) {
            std::memcpy(dst + o, r->pinned + sg.first + (uint64_t)which * sg.second, 4ull * sg.second);
            o += sg.second;
        }
    };
    if (r->pinned_count < (1u << 20)) {
        gather(idx, 0); gather(lo, 1); gather(hi, 2);
    } else {
        std::thread t1(gather, lo, 1), t2(gather, hi, 2);
        gather(idx, 0);
        t1.join();
        t2.join();
    }
    return DL_OK;
}

extern "C" int dl_vox_result_free(dl_vox_result* r) {
    delete r;
    return DL_OK;
}

extern "C" int dl_device_set_voxel_scheduler(dl_device* dev, dl_mlp* mlp) {
    if (!dev) { dl_set_error("device is NULL"); return DL_E_INVALID_ARG; }
    dev->vox_sched = mlp;
    return DL_OK;
}

extern "C" int dl_vox_result_block_log(const dl_vox_result* r, float* features, float* cost, uint64_t cap,
                                       uint64_t* n) {
    if (!r) { dl_set_error("result is NULL"); return DL_E_INVALID_ARG; }
    const uint64_t T = r->log_cost.size();
    if (n) *n = T;
    if (T == 0 || (!features && !cost)) return DL_OK;
    if (cap < T) { dl_set_error("dl_vox_result_block_log: capacity smaller than the block count"); return DL_E_INVALID_ARG; }
    if (features) std::memcpy(features, r->log_feat.data(), 48ull * T);
    if (cost) std::memcpy(cost, r->log_cost.data(), 4ull * T);
    return DL_OK;
}

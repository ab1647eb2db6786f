// dl_query.cu — point occupancy against a sparse block-mask buffer, and one
// buffer carved out of another, on the device.
//
// A downstream stage of the voxelizer (collision tests against its output), with
// no counterpart in the reference, whose BlockMaskBuffer answers one block at a
// time on the CPU (src/voxel/block-mask-buffer.ts:41-58).  Semantics follow that
// buffer and the voxelizer's grid (src/voxel/voxelize.ts:160-179 and
// src/voxel/shaders/voxelize.ts:103-137):
//   * a point p lies in voxel v = floor((p - boundsMin) / voxelResolution) per
//     axis (in f64), valid when 0 <= v < 4 * numBlocks on every axis;
//   * its block is v >> 2, flat index bx + by * nX + bz * nX * nY, and its bit in
//     the block's 64-bit mask (lo = bits 0-31, hi = bits 32-63) is
//     (v.z & 3) * 16 + (v.y & 3) * 4 + (v.x & 3);
//   * blocks listed more than once are OR-merged (BlockMaskBuffer.addBlock).
// Points outside the grid, non-finite points and points in absent blocks are 0.
//
// The blocks go into an open-addressing hash table in device memory (a power
// of two at least twice the block count, linear probing, masks OR-merged with
// atomics, so the table is the same whatever the insertion order); each point
// is one thread that probes it.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dl_internal.h"

namespace {

constexpr uint32_t kEmpty = 0xffffffffu;

__device__ __forceinline__ uint32_t slot_of(uint32_t key, uint32_t mask) {
    // multiplicative hash (Knuth): spreads consecutive block indices
    return (key * 2654435761u) & mask;
}

__global__ void query_insert_k(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ lo,
                               const uint32_t* __restrict__ hi, uint64_t n, uint32_t* keys, uint32_t* tlo,
                               uint32_t* thi, uint32_t mask) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = idx[i];
        uint32_t s = slot_of(k, mask);
        // at most mask + 1 probes: the table is at most half full
        for (uint32_t probe = 0; probe <= mask; probe++) {
            const uint32_t prev = atomicCAS(&keys[s], kEmpty, k);
            if (prev == kEmpty || prev == k) {
                atomicOr(&tlo[s], lo[i]);
                atomicOr(&thi[s], hi[i]);
                break;
            }
            s = (s + 1u) & mask;
        }
    }
}

struct QueryGrid {
    double bmin[3];
    double res;
    int64_t nvox[3];      // voxels per axis (4 per block)
    int64_t nbx, nby;     // blocks per axis (x, y) of the flat index
};

__global__ void query_points_k(const float* __restrict__ pts, uint64_t n, QueryGrid q, const uint32_t* __restrict__ keys,
                               const uint32_t* __restrict__ tlo, const uint32_t* __restrict__ thi, uint32_t mask,
                               uint8_t* __restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        int64_t v[3];
        bool inside = true;
        for (int a = 0; a < 3; a++) {
            const double f = floor(((double)pts[3 * i + a] - q.bmin[a]) / q.res);
            inside = inside && f >= 0.0 && f < (double)q.nvox[a];     // false for NaN
            v[a] = inside ? (int64_t)f : 0;
        }
        uint8_t r = 0;
        if (inside) {
            const int64_t flat = (v[0] >> 2) + (v[1] >> 2) * q.nbx + (v[2] >> 2) * q.nbx * q.nby;
            if (flat >= 0 && flat < (int64_t)kEmpty) {
                const uint32_t key = (uint32_t)flat;
                const uint32_t bit = (uint32_t)((v[2] & 3) * 16 + (v[1] & 3) * 4 + (v[0] & 3));
                uint32_t s = slot_of(key, mask);
                for (uint32_t probe = 0; probe <= mask; probe++) {
                    const uint32_t k = keys[s];
                    if (k == key) {
                        r = (uint8_t)(((bit < 32 ? tlo[s] >> bit : thi[s] >> (bit - 32)) & 1u));
                        break;
                    }
                    if (k == kEmpty) break;
                    s = (s + 1u) & mask;
                }
            }
        }
        out[i] = r;
    }
}

}  // namespace

extern "C" int dl_vox_query(dl_device* dev, const uint32_t* block_idx, const uint32_t* mask_lo, const uint32_t* mask_hi,
                            uint64_t nblocks, const double bounds_min[3], double voxel_resolution,
                            const double dims[3], const float* points, uint64_t npoints, uint8_t* out) {
    if (!dev || !bounds_min || !dims || (npoints && (!points || !out)) ||
        (nblocks && (!block_idx || !mask_lo || !mask_hi))) {
        dl_set_error("dl_vox_query: NULL argument");
        return DL_E_INVALID_ARG;
    }
    if (npoints == 0) return DL_OK;
    if (nblocks >= (1ull << 30)) { dl_set_error("dl_vox_query: at most 2^30 - 1 blocks"); return DL_E_CAPACITY; }
    // an empty grid (dims -Infinity, bounds +-Infinity) or no blocks: nothing is solid
    bool grid = nblocks > 0 && voxel_resolution > 0.0 && std::isfinite(voxel_resolution);
    QueryGrid q{};
    for (int a = 0; a < 3 && grid; a++) {
        if (!std::isfinite(bounds_min[a]) || !std::isfinite(dims[a]) || dims[a] < 1.0 || dims[a] > 1e9) grid = false;
        else {
            q.bmin[a] = bounds_min[a];
            q.nvox[a] = 4 * (int64_t)dims[a];
        }
    }
    if (!grid) {
        std::memset(out, 0, npoints);
        return DL_OK;
    }
    q.res = voxel_resolution;
    q.nbx = (int64_t)dims[0];
    q.nby = (int64_t)dims[1];
    DL_CK(cudaSetDevice(dev->ordinal));
    cudaStream_t st = dev->stream;
    uint32_t cap = 1;
    while (cap < 2 * nblocks) cap <<= 1;
    DevBuf dIdx, dLo, dHi, dKeys, dTlo, dThi, dPts, dOut;
    auto cleanup = [&]() {
        for (DevBuf* b : {&dIdx, &dLo, &dHi, &dKeys, &dTlo, &dThi, &dPts, &dOut}) b->release();
    };
    int rc = DL_OK;
    if ((rc = dIdx.ensure(4 * nblocks)) != DL_OK || (rc = dLo.ensure(4 * nblocks)) != DL_OK ||
        (rc = dHi.ensure(4 * nblocks)) != DL_OK || (rc = dKeys.ensure(4ull * cap)) != DL_OK ||
        (rc = dTlo.ensure(4ull * cap)) != DL_OK || (rc = dThi.ensure(4ull * cap)) != DL_OK ||
        (rc = dPts.ensure(12 * npoints)) != DL_OK || (rc = dOut.ensure(npoints)) != DL_OK) {
        cleanup();
        return rc;
    }
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ck(cudaMemcpyAsync(dIdx.p, block_idx, 4 * nblocks, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dLo.p, mask_lo, 4 * nblocks, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dHi.p, mask_hi, 4 * nblocks, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dPts.p, points, 12 * npoints, cudaMemcpyHostToDevice, st));
    ck(cudaMemsetAsync(dKeys.p, 0xff, 4ull * cap, st));
    ck(cudaMemsetAsync(dTlo.p, 0, 4ull * cap, st));
    ck(cudaMemsetAsync(dThi.p, 0, 4ull * cap, st));
    const uint32_t gi = (uint32_t)std::min<uint64_t>((nblocks + 255) / 256, 8ull * dev->sm_count * 8);
    query_insert_k<<<gi, 256, 0, st>>>(dIdx.as<uint32_t>(), dLo.as<uint32_t>(), dHi.as<uint32_t>(), nblocks,
                                       dKeys.as<uint32_t>(), dTlo.as<uint32_t>(), dThi.as<uint32_t>(), cap - 1);
    ck(cudaGetLastError());
    const uint32_t gq = (uint32_t)std::min<uint64_t>((npoints + 255) / 256, 8ull * dev->sm_count * 8);
    query_points_k<<<gq, 256, 0, st>>>(dPts.as<float>(), npoints, q, dKeys.as<uint32_t>(), dTlo.as<uint32_t>(),
                                       dThi.as<uint32_t>(), cap - 1, dOut.as<uint8_t>());
    ck(cudaGetLastError());
    ck(cudaMemcpyAsync(out, dOut.p, npoints, cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    cleanup();
    if (e != cudaSuccess) {
        dl_set_error(std::string("dl_vox_query: ") + cudaGetErrorString(e));
        return DL_E_CUDA;
    }
    return DL_OK;
}

// ---- carve: A minus B, block by block
// Each listed block of A keeps the bits that B's blocks (OR-merged) do not
// set; blocks left empty are dropped and the others keep A's order (the order
// voxelize returns), so carving an empty B returns A's non-empty blocks as they
// are.  Two kernels around one host scan of per-CTA counts: the first computes
// every entry's carved masks and its CTA's count of non-empty entries, the
// second writes the kept entries at their CTA's offset plus their rank in it.
namespace {

constexpr int kCarveThreads = 256;

__device__ __forceinline__ void lookup_masks(uint32_t key, const uint32_t* keys, const uint32_t* tlo,
                                             const uint32_t* thi, uint32_t mask, uint32_t& lo, uint32_t& hi) {
    lo = 0u;
    hi = 0u;
    uint32_t s = slot_of(key, mask);
    for (uint32_t probe = 0; probe <= mask; probe++) {
        const uint32_t k = keys[s];
        if (k == key) { lo = tlo[s]; hi = thi[s]; return; }
        if (k == kEmpty) return;
        s = (s + 1u) & mask;
    }
}

__global__ void __launch_bounds__(kCarveThreads) carve_count_k(const uint32_t* __restrict__ idx,
                                                               uint32_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                                               uint64_t n, const uint32_t* keys, const uint32_t* tlo,
                                                               const uint32_t* thi, uint32_t mask, uint32_t* counts) {
    const uint64_t i = blockIdx.x * (uint64_t)kCarveThreads + threadIdx.x;
    bool keep = false;
    if (i < n) {
        uint32_t bl, bh;
        lookup_masks(idx[i], keys, tlo, thi, mask, bl, bh);
        const uint32_t l = lo[i] & ~bl, h = hi[i] & ~bh;
        lo[i] = l;
        hi[i] = h;
        keep = (l | h) != 0u;
    }
    const int c = __syncthreads_count(keep);
    if (threadIdx.x == 0) counts[blockIdx.x] = (uint32_t)c;
}

__global__ void __launch_bounds__(kCarveThreads) carve_write_k(const uint32_t* __restrict__ idx,
                                                               const uint32_t* __restrict__ lo,
                                                               const uint32_t* __restrict__ hi, uint64_t n,
                                                               const uint64_t* __restrict__ offs, uint32_t* oidx,
                                                               uint32_t* olo, uint32_t* ohi) {
    __shared__ uint32_t s_w[kCarveThreads / 32];
    const uint64_t i = blockIdx.x * (uint64_t)kCarveThreads + threadIdx.x;
    const bool keep = i < n && (lo[i] | hi[i]) != 0u;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t b = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_w[warp] = (uint32_t)__popc(b);
    __syncthreads();
    uint32_t before = 0;
    for (int w = 0; w < warp; w++) before += s_w[w];
    if (keep) {
        const uint64_t o = offs[blockIdx.x] + before + (uint32_t)__popc(b & dl_lanemask_lt());
        oidx[o] = idx[i];
        olo[o] = lo[i];
        ohi[o] = hi[i];
    }
}

}  // namespace

extern "C" int dl_vox_carve(dl_device* dev, const uint32_t* a_idx, const uint32_t* a_lo, const uint32_t* a_hi,
                            uint64_t na, const uint32_t* b_idx, const uint32_t* b_lo, const uint32_t* b_hi,
                            uint64_t nb, uint32_t* out_idx, uint32_t* out_lo, uint32_t* out_hi, uint64_t* out_n) {
    if (!dev || !out_n || (na && (!a_idx || !a_lo || !a_hi || !out_idx || !out_lo || !out_hi)) ||
        (nb && (!b_idx || !b_lo || !b_hi))) {
        dl_set_error("dl_vox_carve: NULL argument");
        return DL_E_INVALID_ARG;
    }
    *out_n = 0;
    if (na == 0) return DL_OK;
    if (na >= (1ull << 30) || nb >= (1ull << 30)) { dl_set_error("dl_vox_carve: at most 2^30 - 1 blocks"); return DL_E_CAPACITY; }
    DL_CK(cudaSetDevice(dev->ordinal));
    cudaStream_t st = dev->stream;
    uint32_t cap = 1;
    while (cap < 2 * std::max<uint64_t>(nb, 1)) cap <<= 1;
    const uint64_t ctas = (na + kCarveThreads - 1) / kCarveThreads;
    DevBuf dAi, dAl, dAh, dBi, dBl, dBh, dKeys, dTlo, dThi, dCnt, dOff, dOi, dOl, dOh;
    auto cleanup = [&]() {
        for (DevBuf* b : {&dAi, &dAl, &dAh, &dBi, &dBl, &dBh, &dKeys, &dTlo, &dThi, &dCnt, &dOff, &dOi, &dOl, &dOh})
            b->release();
    };
    int rc = DL_OK;
    if ((rc = dAi.ensure(4 * na)) != DL_OK || (rc = dAl.ensure(4 * na)) != DL_OK || (rc = dAh.ensure(4 * na)) != DL_OK ||
        (rc = dBi.ensure(4 * std::max<uint64_t>(nb, 1))) != DL_OK || (rc = dBl.ensure(4 * std::max<uint64_t>(nb, 1))) != DL_OK ||
        (rc = dBh.ensure(4 * std::max<uint64_t>(nb, 1))) != DL_OK || (rc = dKeys.ensure(4ull * cap)) != DL_OK ||
        (rc = dTlo.ensure(4ull * cap)) != DL_OK || (rc = dThi.ensure(4ull * cap)) != DL_OK ||
        (rc = dCnt.ensure(4 * ctas)) != DL_OK || (rc = dOff.ensure(8 * ctas)) != DL_OK ||
        (rc = dOi.ensure(4 * na)) != DL_OK || (rc = dOl.ensure(4 * na)) != DL_OK || (rc = dOh.ensure(4 * na)) != DL_OK) {
        cleanup();
        return rc;
    }
    cudaError_t e = cudaSuccess;
    auto ck = [&](cudaError_t x) { if (e == cudaSuccess) e = x; };
    ck(cudaMemcpyAsync(dAi.p, a_idx, 4 * na, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dAl.p, a_lo, 4 * na, cudaMemcpyHostToDevice, st));
    ck(cudaMemcpyAsync(dAh.p, a_hi, 4 * na, cudaMemcpyHostToDevice, st));
    if (nb) {
        ck(cudaMemcpyAsync(dBi.p, b_idx, 4 * nb, cudaMemcpyHostToDevice, st));
        ck(cudaMemcpyAsync(dBl.p, b_lo, 4 * nb, cudaMemcpyHostToDevice, st));
        ck(cudaMemcpyAsync(dBh.p, b_hi, 4 * nb, cudaMemcpyHostToDevice, st));
    }
    ck(cudaMemsetAsync(dKeys.p, 0xff, 4ull * cap, st));
    ck(cudaMemsetAsync(dTlo.p, 0, 4ull * cap, st));
    ck(cudaMemsetAsync(dThi.p, 0, 4ull * cap, st));
    if (nb) {
        const uint32_t gi = (uint32_t)std::min<uint64_t>((nb + 255) / 256, 64ull * dev->sm_count);
        query_insert_k<<<gi, 256, 0, st>>>(dBi.as<uint32_t>(), dBl.as<uint32_t>(), dBh.as<uint32_t>(), nb,
                                           dKeys.as<uint32_t>(), dTlo.as<uint32_t>(), dThi.as<uint32_t>(), cap - 1);
        ck(cudaGetLastError());
    }
    carve_count_k<<<(uint32_t)ctas, kCarveThreads, 0, st>>>(dAi.as<uint32_t>(), dAl.as<uint32_t>(), dAh.as<uint32_t>(),
                                                           na, dKeys.as<uint32_t>(), dTlo.as<uint32_t>(),
                                                           dThi.as<uint32_t>(), cap - 1, dCnt.as<uint32_t>());
    ck(cudaGetLastError());
    std::vector<uint32_t> cnt(ctas);
    std::vector<uint64_t> off(ctas);
    ck(cudaMemcpyAsync(cnt.data(), dCnt.p, 4 * ctas, cudaMemcpyDeviceToHost, st));
    ck(cudaStreamSynchronize(st));
    uint64_t total = 0;
    for (uint64_t c = 0; c < ctas; c++) { off[c] = total; total += cnt[c]; }
    if (e == cudaSuccess && total) {
        ck(cudaMemcpyAsync(dOff.p, off.data(), 8 * ctas, cudaMemcpyHostToDevice, st));
        carve_write_k<<<(uint32_t)ctas, kCarveThreads, 0, st>>>(dAi.as<uint32_t>(), dAl.as<uint32_t>(),
                                                               dAh.as<uint32_t>(), na, dOff.as<uint64_t>(),
                                                               dOi.as<uint32_t>(), dOl.as<uint32_t>(), dOh.as<uint32_t>());
        ck(cudaGetLastError());
        ck(cudaMemcpyAsync(out_idx, dOi.p, 4 * total, cudaMemcpyDeviceToHost, st));
        ck(cudaMemcpyAsync(out_lo, dOl.p, 4 * total, cudaMemcpyDeviceToHost, st));
        ck(cudaMemcpyAsync(out_hi, dOh.p, 4 * total, cudaMemcpyDeviceToHost, st));
        ck(cudaStreamSynchronize(st));
    }
    cleanup();
    if (e != cudaSuccess) {
        dl_set_error(std::string("dl_vox_carve: ") + cudaGetErrorString(e));
        return DL_E_CUDA;
    }
    *out_n = total;
    return DL_OK;
}

// dl_sort.cuh — stable LSD radix sort of u32 keys with u32 values
// ("onesweep": one histogram pass, then one scatter pass per digit whose
// tile offsets come from a decoupled look-back; Adinets & Merrill, 2022).
//
// Replaces two reference stages with one device primitive:
//   * the CPU depth sort (src/spatial/radix-sort.ts:65-117: stable LSD,
//     4 x 8-bit digits over the order-preserving u32 depth key);
//   * the CPU stable counting sort of tile pairs (src/render/pipeline.ts:544-578),
//     itself a replacement for the unstable GPU sorter (src/gpu/radix-sort.ts).
// Stability is what both callers rely on: ties keep input order, so equal
// depths stay in index order and each tile's pairs stay in depth-rank order.
//
// Batched use: the key array holds S independent segments (one per view);
// every pass sorts each segment separately in the same launch.  Segment
// lengths live in device memory so a whole frame can run without a host sync.
//
// Every look-back wait is bounded (Pass::spin_limit polls, DL_SPIN_LIMIT by
// default); on expiry the CTA sets DL_DEVERR_TIMEOUT in the error word, keeps
// the prefix it has summed so far (so its writes stay inside its segment) and
// finishes, so the host reports an error instead of the GPU hanging.  A pass
// that starts with the timeout bit already set does nothing: its input may
// hold slots that an earlier pass never wrote; a CTA that sees the bit after a
// tile stops there.
//
// The pass is persistent (at most 4 resident CTAs per SM, pass_grid): a CTA
// claims its next tile from the counter when it starts a tile and loads the
// next tile's keys and values into registers while it waits in the current
// tile's look-back and writes it out.  Tiles are claimed in increasing order
// and a tile's aggregate never waits on anything, so the smallest tile whose
// aggregate is unpublished always belongs to a CTA that can publish it: the
// look-backs cannot wait on one another in a cycle.
//
// Pass kernel choices (measured on B200, 64M random keys, 4 passes, and 256M
// 14-bit keys in 64 segments, 2 passes; 16 B per key per pass): the warp
// match uses shared-memory atomicOr masks instead of __match_any_sync, whose
// cost grows with the number of distinct digits in a warp (1.22 -> 1.86 TB/s);
// the look-back reads four predecessor tiles per step and publishes without a
// fence, because a status word carries its own value (+12% and +5%); 4 CTAs
// per SM (64 registers) instead of 3.  Persistence with the next tile's loads
// in flight: the headline batch's pair sort 4.78 -> 4.08 ms, depth sort
// 4.54 -> 4.36 ms (large single sorts within +-4%).
#pragma once
#include "dl_common.cuh"

namespace dlsort {

constexpr int kThreads = 256;
constexpr int kItems = 15;
constexpr int kTile = kThreads * kItems;     // 3840 keys per CTA tile
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagPrefix = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;

struct Segs {
    const uint64_t* start;       // element offset of each segment
    const uint32_t* len;         // element count of each segment (device)
    uint32_t* tile_base;         // first global tile of each segment (filled by prepare_k)
    uint32_t* total_tiles;       // sum of tiles (filled by prepare_k)
    uint32_t num;
};

// Global tile -> segment (tile_base is ascending; few segments).
__device__ __forceinline__ uint32_t seg_of_tile(const Segs& s, uint32_t tile) {
    uint32_t lo = 0, hi = s.num;            // find last seg with tile_base <= tile
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s.tile_base[mid] <= tile) lo = mid; else hi = mid;
    }
    return lo;
}

static __global__ void prepare_k(Segs s) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t acc = 0;
    for (uint32_t i = 0; i < s.num; i++) {
        s.tile_base[i] = acc;
        acc += (s.len[i] + kTile - 1) / kTile;
    }
    *s.total_tiles = acc;
}

// Digit histograms of all passes: hist[seg][pass][radix] (must be zeroed).
// drop_max: keys equal to 0xffffffff are left out (see Pass::drop_max).
template <int BITS>
__global__ void __launch_bounds__(kThreads) hist_k(const uint32_t* __restrict__ keys, Segs s, int passes,
                                                   int first_shift, uint32_t* __restrict__ hist, int drop_max = 0) {
    constexpr int RADIX = 1 << BITS;
    __shared__ uint32_t sh[4 * RADIX];
    const uint32_t total = *s.total_tiles;
    for (uint32_t tile = blockIdx.x; tile < total; tile += gridDim.x) {
        for (int i = threadIdx.x; i < passes * RADIX; i += kThreads) sh[i] = 0;
        __syncthreads();
        const uint32_t seg = seg_of_tile(s, tile);
        const uint32_t lt = tile - s.tile_base[seg];
        const uint32_t len = s.len[seg];
        const uint64_t base = s.start[seg];
        // all of the thread's keys are loaded before the first count, so that
        // the loads are in flight together rather than one per shared atomic
        uint32_t kk[kItems];
#pragma unroll
        for (int j = 0; j < kItems; j++) {
            const uint32_t e = lt * kTile + j * kThreads + threadIdx.x;
            kk[j] = e < len ? __ldg(keys + base + e) : 0u;
        }
#pragma unroll
        for (int j = 0; j < kItems; j++) {
            const uint32_t e = lt * kTile + j * kThreads + threadIdx.x;
            const uint32_t k = kk[j];
            if (e >= len || (drop_max && k == 0xffffffffu)) continue;
            for (int p = 0; p < passes; p++)
                atomicAdd(&sh[p * RADIX + ((k >> (first_shift + p * BITS)) & (RADIX - 1))], 1u);
        }
        __syncthreads();
        for (int i = threadIdx.x; i < passes * RADIX; i += kThreads)
            if (sh[i]) atomicAdd(&hist[(size_t)seg * passes * RADIX + i], sh[i]);
        __syncthreads();
    }
}

// Exclusive scan of each (segment, pass) histogram row in place.
template <int BITS>
__global__ void scan_hist_k(uint32_t* hist, uint32_t rows) {
    constexpr int RADIX = 1 << BITS;
    __shared__ uint32_t sh[RADIX];
    for (uint32_t row = blockIdx.x; row < rows; row += gridDim.x) {
        uint32_t* h = hist + (size_t)row * RADIX;
        for (int i = threadIdx.x; i < RADIX; i += blockDim.x) sh[i] = h[i];
        __syncthreads();
        if (threadIdx.x == 0) {
            uint32_t acc = 0;
            for (int i = 0; i < RADIX; i++) { const uint32_t v = sh[i]; sh[i] = acc; acc += v; }
        }
        __syncthreads();
        for (int i = threadIdx.x; i < RADIX; i += blockDim.x) h[i] = sh[i];
        __syncthreads();
    }
}

struct Pass {
    const uint32_t* keys_in;
    const uint32_t* vals_in;     // NULL: values are the element index within the segment
    uint32_t* keys_out;          // NULL on a last pass whose keys nobody reads
    uint32_t* vals_out;
    Segs segs;
    const uint32_t* glob_off;    // [seg][passes][radix] exclusive digit offsets
    uint32_t* status;            // [tile][radix] look-back words, zeroed before the pass
    uint32_t* counter;           // dynamic tile counter, zeroed before the pass
    uint32_t* err;
    int shift, pass, passes;
    // 1: elements whose key is 0xffffffff are dropped (neither ranked nor
    // written); the others keep their relative order, so the output is the
    // stable pass over the remaining elements, compacted to the segment start.
    // Launch pass_k<BITS, true> for such a pass; it ignores vals_in and takes
    // the implicit values (each element's index in its segment).
    int drop_max = 0;
    uint32_t spin_limit = DL_SPIN_LIMIT;   // look-back polls before giving up
    uint32_t withhold_tile = 0xffffffffu;  // test hook: this global tile publishes no status
};

// Optional table of the last pass of a sort whose keys index a table: the
// first element of each run of equal keys in a CTA's tile lowers
// bound[seg * stride + key] (atomicMin) to its position in the segment, so the
// table ends with each present key's first position; the caller presets the
// table, and keys_out is not written.  Launch pass_k<BITS, false, true> with it.
struct Bound {
    uint32_t* bound = nullptr;
    uint32_t stride = 0;
};

constexpr int kLookback = 4;

// Persistent passes: at most 4 resident CTAs per SM loop over the tiles.
inline uint32_t pass_grid(uint32_t tiles) {
    static int sms = 0;
    if (sms <= 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0) sms = 148;
    }
    return tiles < (uint32_t)sms * 4u ? tiles : (uint32_t)sms * 4u;
}                 // predecessor tiles read per look-back step

// DROP: compiled in only for passes with Pass::drop_max set; BOUND: only for
// a pass with Pass::bound set (either adds registers that other passes would
// pay for in spills).
template <int BITS, bool DROP = false, bool BOUND = false>
__global__ void __launch_bounds__(kThreads, 4) pass_k(Pass p, Bound bd = Bound()) {
    constexpr int RADIX = 1 << BITS;
    constexpr int WARPS = kThreads / 32;
    constexpr uint32_t MASK = RADIX - 1;
    __shared__ uint32_t s_keys[kTile];
    __shared__ uint32_t s_vals[kTile];
    __shared__ uint32_t s_hist[WARPS][RADIX];
    __shared__ uint32_t s_toff[RADIX];
    __shared__ uint32_t s_glob[RADIX];          // per digit: segment position of local slot i, minus i (mod 2^32)
    __shared__ uint32_t s_wsum[WARPS];
    __shared__ uint32_t s_tile, s_next;
    __shared__ uint32_t s_nkeep;                 // elements of the tile that are written

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (__syncthreads_or(tid == 0 && (dl_ld_volatile(p.err) & DL_DEVERR_TIMEOUT))) return;
    if (tid == 0) s_tile = atomicAdd(p.counter, 1u);
    __syncthreads();
    const uint32_t total = *p.segs.total_tiles;
    uint32_t tile = s_tile;
    if (tile >= total) return;
    const uint32_t lmask = dl_lanemask_lt();
    // per-warp digit -> lane-mask scratch; s_vals is free until the scatter
    uint32_t (*s_match)[RADIX] = reinterpret_cast<uint32_t (*)[RADIX]>(s_vals);

    uint32_t seg = seg_of_tile(p.segs, tile);
    uint32_t lt = tile - p.segs.tile_base[seg];
    uint64_t base = p.segs.start[seg];
    uint32_t t0 = lt * kTile;
    uint32_t nValid = min((uint32_t)kTile, p.segs.len[seg] - t0);
    uint32_t key[kItems], val[kItems], rank[kItems];
#pragma unroll
    for (int j = 0; j < kItems; j++) {
        const uint32_t e = warp * 32 * kItems + j * 32 + lane;
        const bool ok = e < nValid;
        key[j] = ok ? p.keys_in[base + t0 + e] : 0u;
        if (!DROP) val[j] = ok ? (p.vals_in ? p.vals_in[base + t0 + e] : t0 + e) : 0u;
    }

    while (true) {
        const bool publish = tile != p.withhold_tile;
        if (tid == 0) s_next = atomicAdd(p.counter, 1u);     // claimed now, loaded during this tile's look-back
        for (int i = lane; i < RADIX; i += 32) s_hist[warp][i] = 0;
        __syncwarp();
        int dig[kItems];
#pragma unroll
        for (int j = 0; j < kItems; j++) {
            const uint32_t e = warp * 32 * kItems + j * 32 + lane;
            const bool keep = e < nValid && !(DROP && key[j] == 0xffffffffu);
            dig[j] = keep ? (int)((key[j] >> p.shift) & MASK) : RADIX;
        }
        // rank within the warp, in element order
#pragma unroll
        for (int j = 0; j < kItems; j++) {
            const bool valid = dig[j] < RADIX;
            if (valid) s_match[warp][dig[j]] = 0u;
            __syncwarp();
            if (valid) atomicOr(&s_match[warp][dig[j]], 1u << lane);
            __syncwarp();
            const uint32_t peers = valid ? s_match[warp][dig[j]] : 0u;
            const uint32_t before = valid ? s_hist[warp][dig[j]] : 0u;
            __syncwarp();
            const int leader = 31 - __clz(peers);
            if (lane == leader && valid) s_hist[warp][dig[j]] = before + __popc(peers);
            __syncwarp();
            rank[j] = before + __popc(peers & lmask);
        }
        __syncthreads();

        // per digit: warp-exclusive offsets and the tile count; publish the aggregate
        uint32_t cnt = 0;
        if (tid < RADIX) {
            for (int w = 0; w < WARPS; w++) { const uint32_t c = s_hist[w][tid]; s_hist[w][tid] = cnt; cnt += c; }
            if (publish) dl_st_volatile(p.status + (size_t)tile * RADIX + tid, (lt == 0 ? kFlagPrefix : kFlagAgg) | cnt);
        }
        {
            uint32_t v = (tid < RADIX) ? cnt : 0u, inc = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            if (lane == 31) s_wsum[warp] = inc;
            __syncthreads();
            uint32_t wpre = 0;
            for (int w = 0; w < warp; w++) wpre += s_wsum[w];
            if (tid < RADIX) s_toff[tid] = wpre + inc - v;
            if (DROP && tid == RADIX - 1) s_nkeep = wpre + inc;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kItems; j++) {
            if (dig[j] < RADIX) {
                const uint32_t pos = s_toff[dig[j]] + s_hist[warp][dig[j]] + rank[j];
                s_keys[pos] = key[j];
                s_vals[pos] = DROP ? t0 + (uint32_t)(warp * 32 * kItems + j * 32 + lane) : val[j];
            }
        }
        // the next tile's elements: in flight during the look-back and the write-out
        const uint32_t next = s_next;
        uint32_t nseg = 0, nlt = 0, nt0 = 0, nnv = 0;
        uint64_t nbase = 0;
        if (next < total) {
            nseg = seg_of_tile(p.segs, next);
            nlt = next - p.segs.tile_base[nseg];
            nbase = p.segs.start[nseg];
            nt0 = nlt * kTile;
            nnv = min((uint32_t)kTile, p.segs.len[nseg] - nt0);
#pragma unroll
            for (int j = 0; j < kItems; j++) {
                const uint32_t e = warp * 32 * kItems + j * 32 + lane;
                const bool ok = e < nnv;
                key[j] = ok ? p.keys_in[nbase + nt0 + e] : 0u;
                if (!DROP) val[j] = ok ? (p.vals_in ? p.vals_in[nbase + nt0 + e] : nt0 + e) : 0u;
            }
        }
        // decoupled look-back for this digit's prefix over earlier tiles of the segment
        if (tid < RADIX) {
            uint32_t excl = 0;
            if (lt > 0) {
                int64_t q = (int64_t)tile - 1;
                const int64_t first = (int64_t)p.segs.tile_base[seg];
                uint32_t spins = 0;
                while (true) {
                    uint32_t w[kLookback];
#pragma unroll
                    for (int k = 0; k < kLookback; k++)
                        w[k] = (q - k >= first) ? dl_ld_volatile(p.status + (size_t)(q - k) * RADIX + tid) : 0u;
                    bool done = false, stall = false;
                    int used = 0;
#pragma unroll
                    for (int k = 0; k < kLookback; k++) {
                        if (!done && !stall) {
                            const uint32_t flag = w[k] & ~kValMask;
                            if (flag == 0u) {
                                stall = true;
                            } else {
                                excl += w[k] & kValMask;
                                used++;
                                done = flag == kFlagPrefix;
                            }
                        }
                    }
                    if (done) break;
                    q -= used;
                    if (stall) {
                        if (++spins > p.spin_limit) { atomicOr(p.err, DL_DEVERR_TIMEOUT); break; }
                        __nanosleep(32);
                    }
                }
                if (publish) dl_st_volatile(p.status + (size_t)tile * RADIX + tid, kFlagPrefix | ((excl + cnt) & kValMask));
            }
            s_glob[tid] = p.glob_off[((size_t)seg * p.passes + p.pass) * RADIX + tid] + excl - s_toff[tid];
        }
        __syncthreads();
        const uint32_t nKeep = DROP ? s_nkeep : nValid;
        if constexpr (BOUND) {
            uint32_t* const bnd = bd.bound + (size_t)seg * bd.stride;
            for (uint32_t i = tid; i < nKeep; i += kThreads) {
                const uint32_t k = s_keys[i];
                const uint32_t pos = s_glob[(k >> p.shift) & MASK] + i;
                p.vals_out[base + pos] = s_vals[i];
                // the tile is sorted by the whole key here (the earlier passes
                // sorted the lower digits): a run's first slot is its smallest position
                if (i == 0 || s_keys[i - 1] != k) atomicMin(bnd + k, pos);
            }
        } else {
            for (uint32_t i = tid; i < nKeep; i += kThreads) {
                const uint32_t k = s_keys[i];
                const uint32_t d = (k >> p.shift) & MASK;
                const uint64_t dst = base + (uint32_t)(s_glob[d] + i);
                if (p.keys_out) p.keys_out[dst] = k;
                p.vals_out[dst] = s_vals[i];
            }
        }
        // shared memory is reused by the next tile; a timed-out wait ends the CTA
        if (__syncthreads_or(tid == 0 && (dl_ld_volatile(p.err) & DL_DEVERR_TIMEOUT))) return;
        if (next >= total) return;
        tile = next; seg = nseg; lt = nlt; base = nbase; t0 = nt0; nValid = nnv;
    }
}

}  // namespace dlsort

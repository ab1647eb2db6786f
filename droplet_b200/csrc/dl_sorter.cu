// dl_sorter.cu — the GpuRadixSorter contract (src/gpu/radix-sort.ts:91-216)
// on the onesweep sort of dl_sort.cuh.
//
// The reference sorts u32 keys with u32 values in 4-bit passes, reading each
// pass's histogram back to the CPU for the scan, and is not stable.  Here the
// whole sort stays on the device (one histogram kernel for all digits, one
// scan, then one look-back scatter pass per digit) and is stable, which the
// reference's callers may rely on without loss: a stable order is one of the
// orders an unstable sort may return.  As in the reference, sort() returns the
// pair of arrays holding the result — the inputs or the sorter's own pong
// buffers, depending on the number of passes.
#include <algorithm>
#include <cstring>

#include "dl_internal.h"
#include "dl_sort.cuh"

struct dl_sorter {
    dl_device* dev = nullptr;
    cudaStream_t stream = nullptr;
    int bits = 8;
    DevBuf pongKeys, pongVals, idxVals, status, hist, meta;
    uint32_t* h_meta = nullptr;           // pinned: error word read-back
};

namespace {

// meta layout (u32 words): [0] total tiles, [1] tile base, [2] length,
// [3] error word, [4..11] pass counters, then the u64 segment start at 16.
constexpr int kMetaTot = 0, kMetaBase = 1, kMetaLen = 2, kMetaErr = 3, kMetaCtr = 4, kMetaStart64 = 8;

template <int BITS>
void sort_bits(dl_sorter* s, uint32_t* keys, uint32_t* vals, uint64_t n, int passes, uint32_t** ok,
               uint32_t** ov) {
    constexpr int RADIX = 1 << BITS;
    cudaStream_t st = s->stream;
    uint32_t* meta = s->meta.as<uint32_t>();
    dlsort::Segs sg;
    sg.start = reinterpret_cast<const uint64_t*>(meta + 2 * kMetaStart64);
    sg.len = meta + kMetaLen;
    sg.tile_base = meta + kMetaBase;
    sg.total_tiles = meta + kMetaTot;
    sg.num = 1;
    const uint32_t tiles = (uint32_t)((n + dlsort::kTile - 1) / dlsort::kTile);
    dlsort::prepare_k<<<1, 32, 0, st>>>(sg);
    cudaMemsetAsync(s->hist.p, 0, (size_t)passes * RADIX * 4, st);
    dlsort::hist_k<BITS><<<std::min<uint32_t>(tiles, 4096), dlsort::kThreads, 0, st>>>(keys, sg, passes, 0,
                                                                                       s->hist.as<uint32_t>());
    dlsort::scan_hist_k<BITS><<<passes, 256, 0, st>>>(s->hist.as<uint32_t>(), passes);
    uint32_t *kin = keys, *kout = s->pongKeys.as<uint32_t>();
    uint32_t *vin = vals, *vout = vals ? s->pongVals.as<uint32_t>() : s->idxVals.as<uint32_t>();
    uint32_t* vspare = vals ? vals : s->pongVals.as<uint32_t>();
    for (int p = 0; p < passes; p++) {
        cudaMemsetAsync(s->status.p, 0, (size_t)tiles * RADIX * 4, st);
        dlsort::Pass sp;
        sp.keys_in = kin; sp.vals_in = vin; sp.keys_out = kout; sp.vals_out = vout;
        sp.segs = sg; sp.glob_off = s->hist.as<uint32_t>();
        sp.status = s->status.as<uint32_t>(); sp.counter = meta + kMetaCtr + p; sp.err = meta + kMetaErr;
        sp.shift = BITS * p; sp.pass = p; sp.passes = passes;
        sp.spin_limit = g_dl_wait.spin_limit;
        dlsort::pass_k<BITS><<<dlsort::pass_grid(tiles), dlsort::kThreads, 0, st>>>(sp);
        std::swap(kin, kout);
        // values: the pass's output becomes the next input; the other buffer of
        // the pair (or, after an implicit-index first pass, the spare) is next
        uint32_t* nv = vin ? vin : vspare;
        vin = vout;
        vout = nv;
    }
    *ok = kin;
    *ov = vin;
}

}  // namespace

extern "C" int dl_sorter_create(dl_device* dev, dl_sorter** out) {
    if (!dev || !out) { dl_set_error("dl_sorter_create: NULL argument"); return DL_E_INVALID_ARG; }
    *out = nullptr;
    DL_CK(cudaSetDevice(dev->ordinal));
    dl_sorter* s = new dl_sorter();
    s->dev = dev;
    s->stream = dev->stream;
    if (cudaMallocHost(&s->h_meta, 64) != cudaSuccess) {
        delete s;
        dl_set_error("dl_sorter_create: cudaMallocHost failed");
        return DL_E_OOM;
    }
    const int rc = s->meta.ensure(256);
    if (rc != DL_OK) { cudaFreeHost(s->h_meta); delete s; return rc; }
    *out = s;
    return DL_OK;
}

extern "C" int dl_sorter_destroy(dl_sorter* s) {
    if (!s) return DL_OK;
    cudaSetDevice(s->dev->ordinal);
    cudaStreamSynchronize(s->stream);
    s->pongKeys.release(); s->pongVals.release(); s->idxVals.release();
    s->status.release(); s->hist.release(); s->meta.release();
    if (s->h_meta) cudaFreeHost(s->h_meta);
    delete s;
    return DL_OK;
}

extern "C" int dl_sorter_set_stream(dl_sorter* s, void* cuda_stream) {
    if (!s) { dl_set_error("sorter is NULL"); return DL_E_INVALID_ARG; }
    s->stream = cuda_stream ? (cudaStream_t)cuda_stream : s->dev->stream;
    return DL_OK;
}

extern "C" int dl_sorter_set_digit_bits(dl_sorter* s, int bits) {
    if (!s) { dl_set_error("sorter is NULL"); return DL_E_INVALID_ARG; }
    if (bits < 6 || bits > 8) { dl_set_error("dl_sorter_set_digit_bits: bits must be 6, 7 or 8"); return DL_E_INVALID_ARG; }
    s->bits = bits;
    return DL_OK;
}

extern "C" int dl_sorter_sort(dl_sorter* s, uint32_t* keys, uint32_t* vals, uint64_t n, uint32_t key_bits,
                              uint32_t** out_keys, uint32_t** out_vals) {
    if (!s || !out_keys || !out_vals) { dl_set_error("dl_sorter_sort: NULL argument"); return DL_E_INVALID_ARG; }
    if (key_bits == 0) key_bits = 32;
    if (key_bits > 32) { dl_set_error("dl_sorter_sort: key_bits must be 1..32"); return DL_E_INVALID_ARG; }
    if (n > 0xffffffffull) { dl_set_error("dl_sorter_sort: n must be below 2^32"); return DL_E_CAPACITY; }
    *out_keys = keys;
    *out_vals = vals;
    if (n == 0) return DL_OK;
    if (!keys) { dl_set_error("dl_sorter_sort: keys is NULL"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(s->dev->ordinal));
    const int bits = s->bits;
    const int passes = (int)((key_bits + bits - 1) / bits);
    const uint32_t tiles = (uint32_t)((n + dlsort::kTile - 1) / dlsort::kTile);
    DL_TRY(s->pongKeys.ensure(n * 4));
    DL_TRY(s->pongVals.ensure(n * 4));
    if (!vals) DL_TRY(s->idxVals.ensure(n * 4));
    DL_TRY(s->status.ensure((size_t)tiles * 256 * 4));
    DL_TRY(s->hist.ensure((size_t)passes * 256 * 4));
    // one segment [0, n); zero counters and the error word
    uint32_t hm[32];
    std::memset(hm, 0, sizeof(hm));
    hm[kMetaLen] = (uint32_t)n;
    const uint64_t start = 0;
    std::memcpy(&hm[2 * kMetaStart64], &start, 8);
    DL_CK(cudaMemcpyAsync(s->meta.p, hm, sizeof(hm), cudaMemcpyHostToDevice, s->stream));
    if (bits == 8) sort_bits<8>(s, keys, vals, n, passes, out_keys, out_vals);
    else if (bits == 7) sort_bits<7>(s, keys, vals, n, passes, out_keys, out_vals);
    else sort_bits<6>(s, keys, vals, n, passes, out_keys, out_vals);
    DL_CK(cudaGetLastError());
    DL_CK(cudaMemcpyAsync(s->h_meta, s->meta.as<uint32_t>() + kMetaErr, 4, cudaMemcpyDeviceToHost, s->stream));
    DL_CK(cudaStreamSynchronize(s->stream));
    if (s->h_meta[0] & DL_DEVERR_TIMEOUT) {
        dl_set_error("dl_sorter_sort: a look-back wait gave up");
        return DL_E_TIMEOUT;
    }
    return DL_OK;
}

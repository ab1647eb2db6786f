// dl_api.cu — the C ABI (include/droplet_b200.h): devices, renderers, scenes,
// status codes and the thread-local error message.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "dl_internal.h"

static thread_local std::string g_last_error;

void dl_set_error(const std::string& msg) { g_last_error = msg; }

extern "C" const char* dl_last_error(void) { return g_last_error.c_str(); }

// ---------------------------------------------------------------- bounded waits (test hooks)
DlWaitPlan g_dl_wait;

extern "C" int dl_test_set_wait_limit(uint32_t polls) {
    g_dl_wait.spin_limit = polls ? polls : DL_SPIN_LIMIT;
    return DL_OK;
}

int g_dl_alloc_budget = -1;

extern "C" int dl_test_fail_allocation(int after) {
    g_dl_alloc_budget = after < 0 ? -1 : after;
    return DL_OK;
}

extern "C" int dl_test_withhold_status(int stage, uint32_t tile) {
    if (stage < DL_WAIT_STAGE_NONE || stage > DL_WAIT_STAGE_PAIR_SORT) {
        dl_set_error("dl_test_withhold_status: stage must be 0..3");
        return DL_E_INVALID_ARG;
    }
    g_dl_wait.withhold_stage = stage;
    g_dl_wait.withhold_tile = stage == DL_WAIT_STAGE_NONE ? 0xffffffffu : tile;
    return DL_OK;
}

// ---------------------------------------------------------------- device
extern "C" int dl_device_open(int ordinal, dl_device** out) {
    if (!out) { dl_set_error("dl_device_open: out is NULL"); return DL_E_INVALID_ARG; }
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
        cudaGetLastError();
        dl_set_error("no CUDA device available");
        return DL_E_NO_DEVICE;
    }
    if (ordinal < 0 || ordinal >= count) { dl_set_error("device ordinal out of range"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(ordinal));
    cudaDeviceProp prop;
    DL_CK(cudaGetDeviceProperties(&prop, ordinal));
    if (prop.major < 10) {
        dl_set_error(std::string("device ") + prop.name + " is not sm_100 (B200); this library is built for sm_100a only");
        return DL_E_NO_DEVICE;
    }
    dl_device* d = new dl_device();
    d->ordinal = ordinal;
    d->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete d;
        dl_set_error("cudaStreamCreate failed");
        return DL_E_CUDA;
    }
    *out = d;
    return DL_OK;
}

extern "C" int dl_device_close(dl_device* d) {
    if (!d) return DL_OK;
    cudaSetDevice(d->ordinal);
    if (d->stream) cudaStreamSynchronize(d->stream);
    dl_vox_release(d);
    if (d->stream) cudaStreamDestroy(d->stream);
    delete d;
    return DL_OK;
}

// ---------------------------------------------------------------- renderer
extern "C" int dl_renderer_create(dl_device* dev, const dl_renderer_opts* opts, dl_renderer** out) {
    if (!dev || !out) { dl_set_error("dl_renderer_create: NULL argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(dev->ordinal));
    dl_renderer* r = new dl_renderer();
    r->dev = dev;
    // src/render/pipeline.ts:76-81 defaults
    r->chunk_cap = (opts && opts->chunk_cap) ? opts->chunk_cap : 200000u;
    r->max_cov = (opts && opts->max_coverage_per_splat) ? opts->max_coverage_per_splat : 16384u;
    r->stream = dev->stream;
    r->own_scene.dev = dev;
    for (auto& e : r->ev) cudaEventCreate(&e);
    *out = r;
    return DL_OK;
}

extern "C" int dl_renderer_destroy(dl_renderer* r) {
    if (!r) return DL_OK;
    cudaSetDevice(r->dev->ordinal);
    cudaStreamSynchronize(r->stream);
    if (r->copy_stream) cudaStreamSynchronize(r->copy_stream);
    DevBuf* bufs[] = {&r->views, &r->tileBase, &r->segStart, &r->segLen, &r->segTileBase, &r->scratch, &r->keys0, &r->keys1,
                      &r->vals0, &r->vals1, &r->recA, &r->recBC, &r->recH, &r->bbox, &r->nvis, &r->depthHist,
                      &r->sortStatus, &r->pairBase, &r->pairCap, &r->pkeys0, &r->pkeys1, &r->pvals0, &r->pvals1,
                      &r->npairs, &r->emitStatus, &r->tileCount, &r->tileOff, &r->pairSegLen, &r->pairSegTileBase,
                      &r->pairGlob, &r->outs, &r->accum, &r->tileEvals, &r->work, &r->rgba, &r->evalCount, &r->own_scene.mem, &r->feat, &r->pred,
                      &r->skeys0, &r->skeys1, &r->svals0, &r->svals1, &r->sseg, &r->sstatus, &r->shist, &r->tileCycles,
                      &r->visMask};
    for (DevBuf* b : bufs) b->release();
    r->tuneOut.release();
    if (r->copy_stream) { cudaStreamSynchronize(r->copy_stream); cudaStreamDestroy(r->copy_stream); }
    if (r->copy_event) cudaEventDestroy(r->copy_event);
    if (r->raster_stream) { cudaStreamSynchronize(r->raster_stream); cudaStreamDestroy(r->raster_stream); }
    for (auto& e : r->raster_ev) if (e) cudaEventDestroy(e);
    for (auto& e : r->upload_events) if (e) cudaEventDestroy(e);
    if (r->h_views) cudaFreeHost(r->h_views);
    if (r->h_u64) cudaFreeHost(r->h_u64);
    for (auto& e : r->ev) if (e) cudaEventDestroy(e);
    if (r->graph_exec) cudaGraphExecDestroy(r->graph_exec);
    delete r;
    return DL_OK;
}

extern "C" int dl_renderer_set_stream(dl_renderer* r, void* s) {
    if (!r) { dl_set_error("renderer is NULL"); return DL_E_INVALID_ARG; }
    r->stream = s ? (cudaStream_t)s : r->dev->stream;
    return DL_OK;
}

extern "C" int dl_renderer_set_profiling(dl_renderer* r, int on) {
    if (!r) { dl_set_error("renderer is NULL"); return DL_E_INVALID_ARG; }
    r->profiling = on != 0;
    for (double& m : r->stage_ms) m = 0.0;
    return DL_OK;
}

extern "C" int dl_renderer_stage_times(dl_renderer* r, double* ms, int n) {
    if (!r || !ms) { dl_set_error("NULL argument"); return DL_E_INVALID_ARG; }
    for (int i = 0; i < n && i < 6; i++) ms[i] = r->stage_ms[i];
    return DL_OK;
}

extern "C" int dl_renderer_launch_count(dl_renderer* r, uint64_t* count) {
    if (!r || !count) { dl_set_error("NULL argument"); return DL_E_INVALID_ARG; }
    *count = r->launches;
    return DL_OK;
}

extern "C" int dl_renderer_set_debug(dl_renderer* r, int keep_intermediates) {
    if (!r) { dl_set_error("renderer is NULL"); return DL_E_INVALID_ARG; }
    r->keep_accum = keep_intermediates != 0;
    return DL_OK;
}

static int check_camera(const dl_camera* cam) {
    if (!cam) { dl_set_error("camera is NULL"); return DL_E_INVALID_ARG; }
    return DL_OK;
}

// src/render/pipeline.ts:181-426 + composite :428-473
extern "C" int dl_render(dl_renderer* r, const dl_splats* data, const dl_camera* cam, const float bg[4],
                         uint8_t* out_rgba, size_t out_len) {
    if (!r || !data) { dl_set_error("dl_render: NULL argument"); return DL_E_INVALID_ARG; }
    DL_TRY(check_camera(cam));
    const uint64_t pixels = (uint64_t)cam->width * cam->height;
    if (pixels == 0) return DL_OK;
    if (!out_rgba || out_len < pixels * 4) { dl_set_error("dl_render: output buffer smaller than width*height*4"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(r->dev->ordinal));
    DlView v;
    DL_TRY(dl_make_view(cam, bg, r->max_cov, &v));
    DL_TRY(dl_upload_scene(&r->own_scene, data, DL_PREC_F32, r->stream));
    DL_TRY(r->rgba.ensure(pixels * 4));
    uint32_t* outs[1] = {r->rgba.as<uint32_t>()};
    DL_TRY(dl_render_views(r, r->own_scene.d, &v, 1, outs, 0));
    DL_CK(cudaMemcpyAsync(out_rgba, r->rgba.p, pixels * 4, cudaMemcpyDeviceToHost, r->stream));
    DL_CK(cudaStreamSynchronize(r->stream));
    return DL_OK;
}

extern "C" int dl_scene_upload(dl_renderer* r, const dl_splats* data, int precision, dl_scene** out) {
    if (!r || !data || !out) { dl_set_error("dl_scene_upload: NULL argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(r->dev->ordinal));
    dl_scene* s = new dl_scene();
    s->dev = r->dev;
    const int st = dl_upload_scene(s, data, precision, r->stream);
    if (st != DL_OK) { s->mem.release(); delete s; return st; }
    if (cudaStreamSynchronize(r->stream) != cudaSuccess) {
        s->mem.release();
        delete s;
        dl_set_error("scene upload failed");
        return DL_E_CUDA;
    }
    *out = s;
    return DL_OK;
}

extern "C" int dl_scene_free(dl_scene* s) {
    if (!s) return DL_OK;
    cudaSetDevice(s->dev->ordinal);
    s->mem.release();
    delete s;
    return DL_OK;
}

namespace {

int ensure_copy_stream(dl_renderer* r) {
    if (!r->copy_stream) DL_CK(cudaStreamCreateWithFlags(&r->copy_stream, cudaStreamNonBlocking));
    if (!r->copy_event) DL_CK(cudaEventCreateWithFlags(&r->copy_event, cudaEventDisableTiming));
    return DL_OK;
}

// Multi-view render of a scene; `upload` (NULL: the scene is resident) is an
// upload still running on the copy stream.
int render_batch(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4], uint8_t* const* outs,
                 uint32_t flags, const DlUploadChunks* upload);

}  // namespace

extern "C" int dl_render_batch(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4],
                               uint8_t* const* outs, uint32_t flags) {
    return render_batch(r, s, cams, n, bg, outs, flags, nullptr);
}

extern "C" int dl_render_many(dl_renderer* r, const dl_splats* data, const dl_camera* cams, int n, const float bg[4],
                              uint8_t* const* outs, uint32_t flags) {
    if (!r || !data) { dl_set_error("dl_render_many: NULL argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(r->dev->ordinal));
    const int prec = ((flags & DL_BATCH_SH16) && !(flags & DL_BATCH_PLAIN)) ? DL_PREC_F16 : DL_PREC_F32;
    flags &= ~(uint32_t)DL_BATCH_OUT_DEVICE;
    if (n < 8 || r->profiling || (flags & DL_BATCH_PLAIN)) {
        DL_TRY(dl_upload_scene(&r->own_scene, data, prec, r->stream));
        return render_batch(r, &r->own_scene, cams, n, bg, outs, flags, nullptr);
    }
    // the upload runs in splat ranges on the copy stream and projection of
    // each range starts when it has arrived
    DL_TRY(ensure_copy_stream(r));
    DlUploadChunks up;
    for (auto& e : r->upload_events)
        if (!e) DL_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (int k = 0; k < kUploadChunks; k++) {
        up.events[k] = r->upload_events[k];
        up.sh_events[k] = r->upload_events[kUploadChunks + 1 + k];
    }
    up.sh_event = r->upload_events[kUploadChunks];
    // the previous frame's kernels may still read the scene buffer
    DL_CK(cudaEventRecord(r->copy_event, r->stream));
    DL_CK(cudaStreamWaitEvent(r->copy_stream, r->copy_event, 0));
    // lays the scene out; the frame issues the copies (up.issue)
    int rc = dl_upload_scene(&r->own_scene, data, prec, r->copy_stream, &up);
    if (rc == DL_OK) rc = render_batch(r, &r->own_scene, cams, n, bg, outs, flags, &up);
    // every return path leaves no copy running
    const cudaError_t ce = cudaStreamSynchronize(r->copy_stream);
    if (rc != DL_OK) return rc;
    DL_CK(ce);
    return DL_OK;
}

namespace {

int render_batch(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4], uint8_t* const* outs,
                 uint32_t flags, const DlUploadChunks* upload) {
    if (!r || !s || !cams || !outs || n < 0) { dl_set_error("dl_render_batch: bad argument"); return DL_E_INVALID_ARG; }
    if (n == 0) return DL_OK;
    if (n > 4096) { dl_set_error("at most 4096 views per batch"); return DL_E_CAPACITY; }
    DL_CK(cudaSetDevice(r->dev->ordinal));
    std::vector<DlView> views((size_t)n);
    uint64_t totalPix = 0;
    for (int i = 0; i < n; i++) {
        DL_TRY(dl_make_view(&cams[i], bg, r->max_cov, &views[i]));
        if (!outs[i]) { dl_set_error("dl_render_batch: NULL output"); return DL_E_INVALID_ARG; }
        totalPix += (uint64_t)views[i].W * views[i].H;
    }
    const bool outDev = (flags & DL_BATCH_OUT_DEVICE) != 0;
    std::vector<uint32_t*> dOuts((size_t)n);
    if (outDev) {
        for (int i = 0; i < n; i++) dOuts[i] = (uint32_t*)outs[i];
    } else {
        DL_TRY(r->rgba.ensure(totalPix * 4));
        uint64_t off = 0;
        for (int i = 0; i < n; i++) { dOuts[i] = r->rgba.as<uint32_t>() + off; off += (uint64_t)views[i].W * views[i].H; }
    }
    uint64_t launches = 0;
    const bool overlapped = !outDev && n >= 8 && !r->profiling && !(flags & DL_BATCH_PLAIN);
    // an upload still in flight: frames that do not overlap it wait for all of it
    if (upload && !overlapped) {
        if (!upload->issued) DL_TRY(upload->issue());
        DL_CK(cudaStreamWaitEvent(r->stream, upload->events[upload->count - 1], 0));
        if (upload->sh_separate) {
            DL_CK(cudaStreamWaitEvent(r->stream, upload->sh_event, 0));
            DL_TRY(dl_upload_convert_sh(upload, 0, upload->bounds[upload->count], r->stream, nullptr));
        }
    }
    if (flags & DL_BATCH_PLAIN) {
        for (int i = 0; i < n; i++) {
            if ((uint64_t)views[i].W * views[i].H == 0) continue;
            DL_TRY(dl_render_views(r, s->d, &views[i], 1, &dOuts[i], flags & ~DL_BATCH_F16_RECORDS));
            launches += r->launches;
        }
    } else if (overlapped) {
        // host outputs: one frame whose rasterizer runs as kReadBackGroups view
        // ranges; each range is copied back on a second stream while the next
        // rasterizes
        DL_TRY(ensure_copy_stream(r));
        // the frame takes the views largest first, so that the last range,
        // whose read-back nothing overlaps, holds the smallest images (each
        // view is rendered on its own: the order changes no pixel)
        std::vector<int> ord((size_t)n);
        for (int i = 0; i < n; i++) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
            return (uint64_t)views[x].W * views[x].H > (uint64_t)views[y].W * views[y].H;
        });
        std::vector<DlView> pv((size_t)n);
        std::vector<uint32_t*> pdOuts((size_t)n);
        std::vector<uint8_t*> pOuts((size_t)n);
        for (int i = 0; i < n; i++) {
            pv[i] = views[ord[i]];
            pdOuts[i] = dOuts[ord[i]];
            pOuts[i] = outs[ord[i]];
        }
        const DlOverlap ov = {kReadBackGroups, pOuts.data(), r->copy_stream, r->copy_event, upload};
        const int rc = dl_render_views(r, s->d, pv.data(), (uint32_t)n, pdOuts.data(), flags, &ov);
        const cudaError_t ce = cudaStreamSynchronize(r->copy_stream);
        if (rc != DL_OK) return rc;
        DL_CK(ce);
        return DL_OK;
    } else {
        DL_TRY(dl_render_views(r, s->d, views.data(), (uint32_t)n, dOuts.data(), flags));
        launches = r->launches;
    }
    r->launches = launches;
    if (!outDev) {
        for (int i = 0; i < n; i++)
            DL_CK(cudaMemcpyAsync(outs[i], dOuts[i], (uint64_t)views[i].W * views[i].H * 4, cudaMemcpyDeviceToHost, r->stream));
    }
    DL_CK(cudaStreamSynchronize(r->stream));
    return DL_OK;
}

}  // namespace

extern "C" int dl_renderer_set_scheduler(dl_renderer* r, dl_mlp* mlp) {
    if (!r) { dl_set_error("renderer is NULL"); return DL_E_INVALID_ARG; }
    r->sched = mlp;
    return DL_OK;
}

extern "C" int dl_renderer_tile_log(dl_renderer* r, float* features, float* cost, uint64_t cap, uint64_t* n) {
    if (!r) { dl_set_error("renderer is NULL"); return DL_E_INVALID_ARG; }
    const uint64_t T = r->log_tiles;
    if (n) *n = T;
    if (T == 0 || (!features && !cost)) return DL_OK;
    if (cap < T) { dl_set_error("dl_renderer_tile_log: capacity smaller than the tile count"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(r->dev->ordinal));
    if (features) DL_CK(cudaMemcpy(features, r->feat.p, 48ull * T, cudaMemcpyDeviceToHost));
    if (cost) {
        std::vector<uint32_t> c(T);
        DL_CK(cudaMemcpy(c.data(), r->tileCycles.p, 4ull * T, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < T; i++) cost[i] = (float)c[i];
    }
    return DL_OK;
}

// ---------------------------------------------------------------- debug copies
extern "C" int dl_renderer_debug_get(dl_renderer* r, const char* name, void* dst, size_t cap, size_t* bytes) {
    if (!r || !name) { dl_set_error("NULL argument"); return DL_E_INVALID_ARG; }
    const std::string s(name);
    const void* src = nullptr;
    size_t n = 0;
    uint64_t scalar = 0;
    bool host = false;
    DL_CK(cudaSetDevice(r->dev->ordinal));
    if (s == "nvis") {
        uint32_t v = 0;
        DL_CK(cudaMemcpy(&v, r->nvis.p, 4, cudaMemcpyDeviceToHost));
        scalar = v;
        src = &scalar; n = 8; host = true;
    } else if (s == "evals") {
        if (r->evalCount.p) DL_CK(cudaMemcpy(&scalar, r->evalCount.p, 8, cudaMemcpyDeviceToHost));
        src = &scalar; n = 8; host = true;
    } else if (s == "npairs") { src = r->npairs.p; n = 8ull * r->last_V;    } else if (s == "depth_keys") { src = r->keys0.p; n = 4ull * r->last_n; }
    else if (s == "sorted_idx") { src = r->vals0.p; n = 4ull * r->last_n; }
    else if (s == "recA") { src = r->recA.p; n = 16ull * r->last_n; }
    else if (s == "recBC") { src = r->recBC.p; n = 32ull * r->last_n; }
    else if (s == "recH") { src = r->recH.p; n = 16ull * r->last_n; }
    else if (s == "bbox") { src = r->bbox.p; n = 8ull * r->last_n; }
    else if (s == "tile_off") { src = r->tileOff.p; n = 4ull * (r->last_T + 1); }
    else if (s == "pair_vals") { src = r->last_final_vals; n = 4ull * r->last_pairs_final; }
    else if (s == "accum") { src = r->keep_accum ? r->accum.p : nullptr; n = src ? 16ull * r->last_W * r->last_H : 0; }
    else { dl_set_error("unknown debug array: " + s); return DL_E_INVALID_ARG; }
    if (bytes) *bytes = n;
    if (!dst || n == 0) return DL_OK;
    if (cap < n) { dl_set_error("debug_get: destination too small"); return DL_E_INVALID_ARG; }
    if (host) std::memcpy(dst, src, n);
    else DL_CK(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
    return DL_OK;
}

extern "C" int dl_renderer_set_tuning(dl_renderer* r, const dl_tuning* t) {
    if (!r || !t) { dl_set_error("dl_renderer_set_tuning: NULL argument"); return DL_E_INVALID_ARG; }
    if (t->pair_sort_bits < 6 || t->pair_sort_bits > 8 || t->raster_shape < 0 || t->raster_shape > 6 ||
        t->raster_ctas_per_sm < 0 || t->raster_ctas_per_sm > 5 || t->bin_tile < 0 || t->bin_tile > 2) {
        dl_set_error("dl_renderer_set_tuning: knob out of range");
        return DL_E_INVALID_ARG;
    }
    r->tune.pair_bits = t->pair_sort_bits;
    r->tune.shape = t->raster_shape;
    r->tune.ctas_per_sm = t->raster_ctas_per_sm;
    r->tune.bin_tile = t->bin_tile;
    return DL_OK;
}

extern "C" int dl_renderer_get_tuning(dl_renderer* r, dl_tuning* t) {
    if (!r || !t) { dl_set_error("dl_renderer_get_tuning: NULL argument"); return DL_E_INVALID_ARG; }
    t->pair_sort_bits = r->tune.pair_bits;
    t->raster_shape = r->tune.shape;
    t->raster_ctas_per_sm = r->tune.ctas_per_sm;
    t->bin_tile = r->tune.bin_tile;
    return DL_OK;
}

extern "C" int dl_renderer_autotune(dl_renderer* r, dl_scene* s, const dl_camera* cams, int n, const float bg[4],
                                    uint32_t flags, int reps, dl_tuning* best, double* best_ms) {
    if (!r || !s || !cams || n <= 0) { dl_set_error("dl_renderer_autotune: bad argument"); return DL_E_INVALID_ARG; }
    if (flags & DL_BATCH_PLAIN) { dl_set_error("dl_renderer_autotune: the plain path is not tuned"); return DL_E_INVALID_ARG; }
    reps = std::max(1, std::min(reps, 50));
    DL_CK(cudaSetDevice(r->dev->ordinal));
    uint64_t total = 0;
    std::vector<uint64_t> offs((size_t)n);
    for (int i = 0; i < n; i++) { offs[i] = total; total += (uint64_t)cams[i].width * cams[i].height * 4; }
    DL_TRY(r->tuneOut.ensure(std::max<uint64_t>(total, 256)));
    std::vector<uint8_t*> outs((size_t)n);
    for (int i = 0; i < n; i++) outs[i] = r->tuneOut.as<uint8_t>() + offs[i];
    cudaEvent_t e0, e1;
    DL_CK(cudaEventCreate(&e0));
    DL_CK(cudaEventCreate(&e1));
    const uint32_t fl = flags | DL_BATCH_OUT_DEVICE;
    auto timeOne = [&](const DlTuning& t, double* ms) -> int {
        r->tune = t;
        DL_TRY(dl_render_batch(r, s, cams, n, bg, outs.data(), fl));          // warm-up (and graph capture)
        std::vector<double> v;
        for (int k = 0; k < reps; k++) {
            cudaEventRecord(e0, r->stream);
            DL_TRY(dl_render_batch(r, s, cams, n, bg, outs.data(), fl));
            cudaEventRecord(e1, r->stream);
            DL_CK(cudaEventSynchronize(e1));
            float f = 0.0f;
            cudaEventElapsedTime(&f, e0, e1);
            v.push_back(f);
        }
        std::sort(v.begin(), v.end());
        *ms = v[v.size() / 2];
        return DL_OK;
    };
    DlTuning cur = r->tune;
    double curMs = 0.0;
    int rc = timeOne(cur, &curMs);
    // shapes 4 and 5 (two splats per step in f32x2) exist for the fast arithmetic only
    const int bitsC[7] = {8, 7, 6, 8, 8, 8, 8}, shapeC[7] = {6, 5, 4, 0, 1, 2, 3}, ctasC[7] = {0, 4, 3, 0, 0, 0, 0};
    const int tileC[7] = {0, 1, 2, 0, 0, 0, 0};
    const bool fast = (flags & DL_BATCH_FAST_EXP) != 0;
    const int nC[4] = {3, 7, 3, 3};
    for (int knob = 0; knob < 4 && rc == DL_OK; knob++) {
        for (int c = 0; c < nC[knob] && rc == DL_OK; c++) {
            DlTuning t = cur;
            if (knob == 0) { if (t.pair_bits == bitsC[c]) continue; t.pair_bits = bitsC[c]; }
            if (knob == 1) {
                if (t.shape == shapeC[c] || ((shapeC[c] == 4 || shapeC[c] == 5) && !fast)) continue;
                t.shape = shapeC[c];
            }
            if (knob == 2) { if (t.ctas_per_sm == ctasC[c]) continue; t.ctas_per_sm = ctasC[c]; }
            if (knob == 3) { if (t.bin_tile == tileC[c]) continue; t.bin_tile = tileC[c]; }
            double ms = 0.0;
            rc = timeOne(t, &ms);
            // a candidate that cannot render this batch (e.g. finer binning
            // tiles pushing a view past the pair capacity) is skipped
            if (rc == DL_E_CAPACITY) { rc = DL_OK; continue; }
            if (rc == DL_OK && ms < curMs) { cur = t; curMs = ms; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    r->tune = cur;
    if (rc != DL_OK) return rc;
    // a finer binning candidate may have grown the per-view pair capacity far
    // past what the chosen knobs need, and views then sit further apart in
    // the pair buffers than they have to; one more frame with the chosen
    // knobs sizes the capacity for them.
    DL_TRY(dl_render_batch(r, s, cams, n, bg, outs.data(), fl));
    const uint64_t need = r->last_max_pairs + r->last_max_pairs / 4 + 4096;
    if (need < r->pair_cap_per_view) r->pair_cap_per_view = need;
    if (best) {
        best->pair_sort_bits = cur.pair_bits;
        best->raster_shape = cur.shape;
        best->raster_ctas_per_sm = cur.ctas_per_sm;
        best->bin_tile = cur.bin_tile;
    }
    if (best_ms) *best_ms = curMs;
    return DL_OK;
}

// dl_mlp.cu — the learned tile-cost model: a 12 -> 64 -> 64 -> 1 MLP with
// ReLU hidden layers, BF16 weights and FP32 accumulation, trained and
// evaluated by the kernels in this file.  It predicts (a monotone transform
// of) the rasterizer time of a tile from 12 features the renderer computes
// per tile (dl_render_kernels.cuh, tile_features_k); the renderer uses the
// prediction only to order the rasterizer's work queue (longest first), so
// it can change the schedule but never a pixel.  No reference counterpart:
// the reference rasterizes tiles in dispatch order (rasterize.ts).
//
// Training: mini-batch MSE on standardised targets, Adam.  One step =
//   mlp_fwd_bwd_k (per sample: forward with BF16 weights, output and hidden
//                  gradients, stored per sample),
//   mlp_wgrad_k   (per parameter: batch sum of the outer products),
//   mlp_adam_k    (FP32 master weights -> BF16 copies).
// The gradients are those of the BF16 forward pass with respect to the FP32
// master weights (straight-through rounding), which is what the CPU check in
// the tests recomputes in float64.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "dl_internal.h"
#include "dl_mlp.cuh"

namespace {

using namespace dlmlp;

__global__ void __launch_bounds__(128) mlp_infer_k(const __nv_bfloat16* w, const float* __restrict__ X, uint32_t n,
                                                   float* __restrict__ out) {
    __shared__ float P[kParams];
    load_params(w, P);
    for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < n; s += gridDim.x * blockDim.x) {
        float x[kIn];
#pragma unroll
        for (int i = 0; i < kIn; i++) x[i] = X[(uint64_t)s * kIn + i];
        out[s] = forward(P, x, nullptr, nullptr);
    }
}

// Per sample of the batch (indices idx[0..B)): forward, loss, and the
// gradients w.r.t. the output and the two hidden pre-activations.
__global__ void __launch_bounds__(128) mlp_fwd_bwd_k(const __nv_bfloat16* w, const float* __restrict__ X,
                                                     const float* __restrict__ Y, const uint32_t* __restrict__ idx,
                                                     uint32_t B, float* __restrict__ xs, float* __restrict__ h1s,
                                                     float* __restrict__ h2s, float* __restrict__ g1s,
                                                     float* __restrict__ g2s, float* __restrict__ gy,
                                                     float* __restrict__ loss) {
    __shared__ float P[kParams];
    load_params(w, P);
    const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= B) return;
    const uint32_t s = idx ? idx[b] : b;
    float x[kIn];
    for (int i = 0; i < kIn; i++) { x[i] = X[(uint64_t)s * kIn + i]; xs[(uint64_t)b * kIn + i] = x[i]; }
    float* h1 = h1s + (uint64_t)b * kH;
    float* h2 = h2s + (uint64_t)b * kH;
    const float y = forward(P, x, h1, h2);
    const float e = y - Y[s];
    atomicAdd(loss, e * e / (float)B);
    const float dy = 2.0f * e / (float)B;
    gy[b] = dy;
    float g2[kH];
    for (int j = 0; j < kH; j++) {
        g2[j] = h2[j] > 0.0f ? dy * P[oW3 + j] : 0.0f;
        g2s[(uint64_t)b * kH + j] = g2[j];
    }
    for (int k = 0; k < kH; k++) {
        float a = 0.0f;
#pragma unroll
        for (int j = 0; j < kH; j++) a += P[oW2 + k * kH + j] * g2[j];
        g1s[(uint64_t)b * kH + k] = h1[k] > 0.0f ? a : 0.0f;
    }
}

// One thread per parameter: sum over the batch.
__global__ void mlp_wgrad_k(uint32_t B, const float* __restrict__ xs, const float* __restrict__ h1s,
                            const float* __restrict__ h2s, const float* __restrict__ g1s,
                            const float* __restrict__ g2s, const float* __restrict__ gy, float* __restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    float acc = 0.0f;
    if (p < oB1) {                                  // W1[i][j] = sum g1[j] x[i]
        const int i = p / kH, j = p % kH;
        for (uint32_t b = 0; b < B; b++) acc += g1s[(uint64_t)b * kH + j] * xs[(uint64_t)b * kIn + i];
    } else if (p < oW2) {
        const int j = p - oB1;
        for (uint32_t b = 0; b < B; b++) acc += g1s[(uint64_t)b * kH + j];
    } else if (p < oB2) {                           // W2[k][j] = sum g2[j] h1[k]
        const int k = (p - oW2) / kH, j = (p - oW2) % kH;
        for (uint32_t b = 0; b < B; b++) acc += g2s[(uint64_t)b * kH + j] * h1s[(uint64_t)b * kH + k];
    } else if (p < oW3) {
        const int j = p - oB2;
        for (uint32_t b = 0; b < B; b++) acc += g2s[(uint64_t)b * kH + j];
    } else if (p < oB3) {                           // W3[j] = sum gy h2[j]
        const int j = p - oW3;
        for (uint32_t b = 0; b < B; b++) acc += gy[b] * h2s[(uint64_t)b * kH + j];
    } else {
        for (uint32_t b = 0; b < B; b++) acc += gy[b];
    }
    grad[p] = acc;
}

__global__ void mlp_adam_k(float* master, __nv_bfloat16* w, const float* grad, float* m, float* v, float lr,
                           float b1, float b2, float b1t, float b2t) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams) return;
    const float g = grad[p];
    m[p] = b1 * m[p] + (1.0f - b1) * g;
    v[p] = b2 * v[p] + (1.0f - b2) * g * g;
    const float mh = m[p] / (1.0f - b1t), vh = v[p] / (1.0f - b2t);
    master[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
    w[p] = __float2bfloat16_rn(master[p]);
}

__global__ void mlp_round_k(const float* master, __nv_bfloat16* w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) w[p] = __float2bfloat16_rn(master[p]);
}

}  // namespace

struct dl_mlp {
    dl_device* dev = nullptr;
    DevBuf master, w, m, v, grad, loss;
    DevBuf X, Y, idx, xs, h1s, h2s, g1s, g2s, gy;
    uint64_t steps = 0;
};

const void* dl_mlp_weights(const dl_mlp* mlp) { return mlp->w.p; }

int dl_mlp_infer_launch(const dl_mlp* mlp, const float* X, uint32_t n, float* out, cudaStream_t st) {
    if (n == 0) return DL_OK;
    const uint32_t grid = std::min<uint32_t>((n + 127) / 128, 4096);
    mlp_infer_k<<<grid, 128, 0, st>>>(mlp->w.as<__nv_bfloat16>(), X, n, out);
    DL_CK(cudaGetLastError());
    return DL_OK;
}

static int mlp_upload_master(dl_mlp* M, const float* p) {
    DL_CK(cudaMemcpy(M->master.p, p, 4 * kParams, cudaMemcpyHostToDevice));
    mlp_round_k<<<(kParams + 255) / 256, 256, 0, M->dev->stream>>>(M->master.as<float>(), M->w.as<__nv_bfloat16>());
    DL_CK(cudaMemsetAsync(M->m.p, 0, 4 * kParams, M->dev->stream));
    DL_CK(cudaMemsetAsync(M->v.p, 0, 4 * kParams, M->dev->stream));
    DL_CK(cudaStreamSynchronize(M->dev->stream));
    M->steps = 0;
    return DL_OK;
}

extern "C" int dl_mlp_create(dl_device* dev, uint64_t seed, dl_mlp** out) {
    if (!dev || !out) { dl_set_error("dl_mlp_create: NULL argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(dev->ordinal));
    dl_mlp* M = new dl_mlp();
    M->dev = dev;
    int s = DL_OK;
    if ((s = M->master.ensure(4 * kParams)) || (s = M->w.ensure(2 * kParams)) || (s = M->m.ensure(4 * kParams)) ||
        (s = M->v.ensure(4 * kParams)) || (s = M->grad.ensure(4 * kParams)) || (s = M->loss.ensure(8))) {
        delete M;
        return s;
    }
    // He-uniform initialisation from a seeded generator
    std::mt19937_64 rng(seed);
    std::vector<float> p(kParams, 0.0f);
    auto fill = [&](int off, int n, int fan_in) {
        std::uniform_real_distribution<float> u(-std::sqrt(6.0f / fan_in), std::sqrt(6.0f / fan_in));
        for (int i = 0; i < n; i++) p[off + i] = u(rng);
    };
    fill(oW1, kIn * kH, kIn);
    fill(oW2, kH * kH, kH);
    fill(oW3, kH, kH);
    if ((s = mlp_upload_master(M, p.data()))) { delete M; return s; }
    *out = M;
    return DL_OK;
}

extern "C" int dl_mlp_destroy(dl_mlp* M) {
    if (!M) return DL_OK;
    cudaSetDevice(M->dev->ordinal);
    DevBuf* b[] = {&M->master, &M->w, &M->m, &M->v, &M->grad, &M->loss, &M->X, &M->Y, &M->idx, &M->xs, &M->h1s,
                   &M->h2s, &M->g1s, &M->g2s, &M->gy};
    for (DevBuf* x : b) x->release();
    delete M;
    return DL_OK;
}

extern "C" int dl_mlp_get_params(dl_mlp* M, float* out, size_t n) {
    if (!M || !out || n < (size_t)kParams) { dl_set_error("dl_mlp_get_params: bad argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(M->dev->ordinal));
    DL_CK(cudaMemcpy(out, M->master.p, 4 * kParams, cudaMemcpyDeviceToHost));
    return DL_OK;
}

extern "C" int dl_mlp_set_params(dl_mlp* M, const float* in, size_t n) {
    if (!M || !in || n < (size_t)kParams) { dl_set_error("dl_mlp_set_params: bad argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(M->dev->ordinal));
    return mlp_upload_master(M, in);
}

static int mlp_stage_data(dl_mlp* M, const float* X, const float* Y, uint64_t n) {
    DL_TRY(M->X.ensure(4ull * kIn * n));
    DL_CK(cudaMemcpy(M->X.p, X, 4ull * kIn * n, cudaMemcpyHostToDevice));
    if (Y) {
        DL_TRY(M->Y.ensure(4ull * n));
        DL_CK(cudaMemcpy(M->Y.p, Y, 4ull * n, cudaMemcpyHostToDevice));
    }
    return DL_OK;
}

static int mlp_batch_bufs(dl_mlp* M, uint32_t B) {
    DL_TRY(M->idx.ensure(4ull * B));
    DL_TRY(M->xs.ensure(4ull * kIn * B));
    DL_TRY(M->h1s.ensure(4ull * kH * B));
    DL_TRY(M->h2s.ensure(4ull * kH * B));
    DL_TRY(M->g1s.ensure(4ull * kH * B));
    DL_TRY(M->g2s.ensure(4ull * kH * B));
    DL_TRY(M->gy.ensure(4ull * B));
    return DL_OK;
}

// forward + backward of one batch; leaves the gradient in M->grad and the loss in M->loss
static int mlp_grad_batch(dl_mlp* M, const uint32_t* d_idx, uint32_t B, cudaStream_t st) {
    DL_CK(cudaMemsetAsync(M->loss.p, 0, 4, st));
    mlp_fwd_bwd_k<<<(B + 127) / 128, 128, 0, st>>>(M->w.as<__nv_bfloat16>(), M->X.as<float>(), M->Y.as<float>(), d_idx,
                                                   B, M->xs.as<float>(), M->h1s.as<float>(), M->h2s.as<float>(),
                                                   M->g1s.as<float>(), M->g2s.as<float>(), M->gy.as<float>(),
                                                   M->loss.as<float>());
    mlp_wgrad_k<<<(kParams + 127) / 128, 128, 0, st>>>(B, M->xs.as<float>(), M->h1s.as<float>(), M->h2s.as<float>(),
                                                       M->g1s.as<float>(), M->g2s.as<float>(), M->gy.as<float>(),
                                                       M->grad.as<float>());
    DL_CK(cudaGetLastError());
    return DL_OK;
}

extern "C" int dl_mlp_grad(dl_mlp* M, const float* X, const float* Y, uint64_t n, float* grad_out, float* loss_out) {
    if (!M || !X || !Y || !grad_out || n == 0 || n > (1u << 24)) { dl_set_error("dl_mlp_grad: bad argument"); return DL_E_INVALID_ARG; }
    DL_CK(cudaSetDevice(M->dev->ordinal));
    cudaStream_t st = M->dev->stream;
    DL_TRY(mlp_stage_data(M, X, Y, n));
    DL_TRY(mlp_batch_bufs(M, (uint32_t)n));
    DL_TRY(mlp_grad_batch(M, nullptr, (uint32_t)n, st));
    DL_CK(cudaMemcpyAsync(grad_out, M->grad.p, 4 * kParams, cudaMemcpyDeviceToHost, st));
    float loss = 0.0f;
    DL_CK(cudaMemcpyAsync(&loss, M->loss.p, 4, cudaMemcpyDeviceToHost, st));
    DL_CK(cudaStreamSynchronize(st));
    if (loss_out) *loss_out = loss;
    return DL_OK;
}

extern "C" int dl_mlp_train(dl_mlp* M, const float* X, const float* Y, uint64_t n, int epochs, int batch, float lr,
                            uint64_t seed, float* loss_out) {
    if (!M || !X || !Y || n == 0 || epochs < 0 || batch <= 0 || n >= (1ull << 32)) {
        dl_set_error("dl_mlp_train: bad argument");
        return DL_E_INVALID_ARG;
    }
    DL_CK(cudaSetDevice(M->dev->ordinal));
    cudaStream_t st = M->dev->stream;
    DL_TRY(mlp_stage_data(M, X, Y, n));
    const uint32_t B = (uint32_t)std::min<uint64_t>((uint64_t)batch, n);
    DL_TRY(mlp_batch_bufs(M, B));
    DevBuf perm;
    DL_TRY(perm.ensure(4ull * n));
    std::vector<uint32_t> hp(n);
    for (uint64_t i = 0; i < n; i++) hp[i] = (uint32_t)i;
    std::mt19937_64 rng(seed);
    const float b1 = 0.9f, b2 = 0.999f;
    double last = 0.0;
    for (int e = 0; e < epochs; e++) {
        std::shuffle(hp.begin(), hp.end(), rng);
        if (cudaMemcpyAsync(perm.p, hp.data(), 4ull * n, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            perm.release();
            dl_set_error("dl_mlp_train: upload failed");
            return DL_E_CUDA;
        }
        double sum = 0.0;
        uint64_t nb = 0;
        for (uint64_t off = 0; off + B <= n; off += B) {
            const int s = mlp_grad_batch(M, perm.as<uint32_t>() + off, B, st);
            if (s != DL_OK) { perm.release(); return s; }
            M->steps++;
            mlp_adam_k<<<(kParams + 255) / 256, 256, 0, st>>>(M->master.as<float>(), M->w.as<__nv_bfloat16>(),
                                                              M->grad.as<float>(), M->m.as<float>(), M->v.as<float>(),
                                                              lr, b1, b2, std::pow(b1, (float)M->steps),
                                                              std::pow(b2, (float)M->steps));
            if ((nb & 63) == 63 || off + 2 * B > n) {
                float l = 0.0f;
                cudaMemcpyAsync(&l, M->loss.p, 4, cudaMemcpyDeviceToHost, st);
                cudaStreamSynchronize(st);
                sum += l;
                last = l;
            }
            nb++;
        }
        (void)sum;
    }
    perm.release();
    DL_CK(cudaStreamSynchronize(st));
    if (loss_out) *loss_out = (float)last;
    return DL_OK;
}

extern "C" int dl_mlp_predict(dl_mlp* M, const float* X, uint64_t n, float* out) {
    if (!M || !X || !out || n >= (1ull << 32)) { dl_set_error("dl_mlp_predict: bad argument"); return DL_E_INVALID_ARG; }
    if (n == 0) return DL_OK;
    DL_CK(cudaSetDevice(M->dev->ordinal));
    cudaStream_t st = M->dev->stream;
    DL_TRY(mlp_stage_data(M, X, nullptr, n));
    DL_TRY(M->Y.ensure(4ull * n));
    DL_TRY(dl_mlp_infer_launch(M, M->X.as<float>(), (uint32_t)n, M->Y.as<float>(), st));
    DL_CK(cudaMemcpyAsync(out, M->Y.p, 4ull * n, cudaMemcpyDeviceToHost, st));
    DL_CK(cudaStreamSynchronize(st));
    return DL_OK;
}

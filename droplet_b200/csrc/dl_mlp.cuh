// dl_mlp.cuh — device-side forward pass of the tile-cost MLP, shared by the
// training kernels (dl_mlp.cu) and the renderer's scheduling kernel.
#pragma once
#include <cuda_bf16.h>

#include "../../include/droplet_b200.h"

namespace dlmlp {

constexpr int kIn = DL_MLP_IN, kH = DL_MLP_HIDDEN;
// parameter layout (f32 count): W1 [kIn][kH], b1 [kH], W2 [kH][kH], b2 [kH], W3 [kH], b3
constexpr int oW1 = 0, oB1 = oW1 + kIn * kH, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH, kParams = oB3 + 1;
static_assert(kParams == DL_MLP_PARAMS, "parameter count");

// BF16 parameters into shared memory as f32 (all threads of the block).
__device__ __forceinline__ void load_params(const __nv_bfloat16* w, float* s) {
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) s[i] = __bfloat162float(w[i]);
    __syncthreads();
}

// One sample; writes the hidden activations when h1/h2 are given.
__device__ __forceinline__ float forward(const float* P, const float* x, float* h1, float* h2) {
    float a1[kH];
#pragma unroll
    for (int j = 0; j < kH; j++) a1[j] = P[oB1 + j];
#pragma unroll
    for (int i = 0; i < kIn; i++) {
        const float xi = x[i];
#pragma unroll
        for (int j = 0; j < kH; j++) a1[j] += xi * P[oW1 + i * kH + j];
    }
#pragma unroll
    for (int j = 0; j < kH; j++) a1[j] = fmaxf(a1[j], 0.0f);
    if (h1) {
#pragma unroll
        for (int j = 0; j < kH; j++) h1[j] = a1[j];
    }
    float y = P[oB3];
    for (int j = 0; j < kH; j++) {
        float a = P[oB2 + j];
#pragma unroll
        for (int k = 0; k < kH; k++) a += a1[k] * P[oW2 + k * kH + j];
        a = fmaxf(a, 0.0f);
        if (h2) h2[j] = a;
        y += a * P[oW3 + j];
    }
    return y;
}

}  // namespace dlmlp

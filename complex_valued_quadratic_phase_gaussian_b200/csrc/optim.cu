// Fused gradient-norm clip + Adan update over all parameter tensors.
//
// Reference (paths inside the reference project):
//   train_2d_gaussian_rgb.py:205-211  nan_to_num (done by the preprocess adjoint),
//                                     clip_grad_norm_(params, 1.0), optimizer.step()
//   utils/optimizer.py:104-204        Adan.step: per-group step counter (incremented even for a
//                                     group whose parameters have no gradient), bias corrections,
//                                     neg_pre_grad initialised to -grad on the first step a tensor
//                                     has a gradient
//   utils/optimizer.py:207-262        _single_tensor_adan (foreach=False, as the fit uses)
//   train_2d_gaussian_rgb.py:58-86    per-group learning rates; cosine schedule of the means group
// The global norm is recomputed by every CTA from the fixed-order per-CTA
// partial sums of the adjoint (deterministic, no second pass over the gradients).
#include <math.h>

#include "preprocess.cuh"

namespace cvqpg {

__global__ void __launch_bounds__(256) adan_kernel(AdanDev A, const int32_t* __restrict__ iteration) {
    const int t = blockIdx.y;
    if (A.frozen_always[t]) return;
    const int it = iteration ? iteration[0] : 0;
    if (it < A.first_iter[t]) return;  // no gradient yet (frozen during warm-up)
    const int n = A.numel[t];
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x >= n) return;

    // global gradient norm and clip coefficient (torch clip_grad_norm_)
    __shared__ float s_clip;
    if (threadIdx.x < 32) {
        double s = 0.0;
        for (int k = threadIdx.x; k < A.num_partials; k += 32) s += (double)A.norm_partials[k];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) {
            float clip = 1.0f;
            if (A.max_grad_norm > 0.0) {
                const float total = (float)sqrt(s);
                const float coef = (float)A.max_grad_norm / (total + 1e-6f);
                clip = fminf(coef, 1.0f);
            }
            s_clip = clip;
        }
    }
    __syncthreads();
    const float clip = s_clip;

    const int grp = A.group[t];
    const int step = it + 1;  // every group steps every iteration
    const double lr = (grp == 0 && A.lr_table) ? A.lr_table[min(it, A.lr_table_len - 1)] : A.lr[grp];
    const double bc1 = 1.0 - pow(A.beta1, (double)step);
    const double bc2 = 1.0 - pow(A.beta2, (double)step);
    const double bc3s = sqrt(1.0 - pow(A.beta3, (double)step));
    const float b1 = (float)A.beta1, b2 = (float)A.beta2, b3 = (float)A.beta3;
    const float ob1 = (float)(1.0 - A.beta1), ob2 = (float)(1.0 - A.beta2), ob3 = (float)(1.0 - A.beta3);
    const float step_size = (float)(lr / bc1);
    const float step_size_diff = (float)(lr * A.beta2 / bc2);
    const float bc3f = (float)bc3s;
    const float eps = (float)A.eps;
    const float wd = (float)(lr * A.weight_decay);
    const bool fresh = (it == A.first_iter[t]);  // state created now: zeros, neg_pre_grad = -grad*clip

    float* P = A.param[t];
    float* G = A.grad[t];
    float* M = A.exp_avg[t];
    float* V = A.exp_avg_sq[t];
    float* D = A.exp_avg_diff[t];
    float* NG = A.neg_pre_grad[t];
    for (int i = i0; i < n; i += gridDim.x * blockDim.x) {
        float g = G[i] * clip;  // clip_grad_norm_ scales the stored gradient
        float m = fresh ? 0.f : M[i], v = fresh ? 0.f : V[i], d = fresh ? 0.f : D[i];
        float ng = fresh ? -g : NG[i];
        // _single_tensor_adan with Adan's own clip = 1 (max_grad_norm = 0)
        ng = ng + g;
        m = m * b1 + ob1 * g;
        d = d * b2 + ob2 * ng;
        ng = ng * b2 + g;
        v = v * b3 + ob3 * ng * ng;
        const float denom = sqrtf(v) / bc3f + eps;
        float p = P[i];
        if (A.no_prox) {
            p = p * (1.0f - wd);
            p = p + (-step_size) * (m / denom);
            p = p + (-step_size_diff) * (d / denom);
        } else {
            p = p + (-step_size) * (m / denom);
            p = p + (-step_size_diff) * (d / denom);
            p = p / (1.0f + wd);
        }
        P[i] = p;
        M[i] = m;
        V[i] = v;
        D[i] = d;
        NG[i] = -g;
        G[i] = g;
    }
}

void launch_adan(const AdanDev& A, const int32_t* iteration, cudaStream_t s) {
    int maxn = 1;
    for (int t = 0; t < kParamTensors; t++) maxn = max(maxn, A.numel[t]);
    const unsigned bx = min(ceil_div(maxn, 256), 4096u);
    dim3 grid(bx, kParamTensors);
    adan_kernel<<<grid, 256, 0, s>>>(A, iteration);
}

}  // namespace cvqpg

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

// The step's scalars, once per launch (one warp): the clip_grad_norm_ factor
// from the norm partials (fixed-order double sum) and, per tensor t at
// scalars[8 + 8 t]: active, fresh (state created now), step size, step size of
// the difference term, sqrt(bias correction 3), lr * weight decay.
__global__ void adan_scalars_kernel(AdanDev A, const int32_t* __restrict__ iteration) {
    const int lane = threadIdx.x;
    double s = 0.0;
    for (int k = lane; k < A.num_partials; k += 32) s += (double)A.norm_partials[k];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const int it = iteration ? iteration[0] : 0;
    if (lane == 0) {
        float clip = 1.0f;
        if (A.max_grad_norm > 0.0) {
            const float total = (float)sqrt(s);
            const float coef = (float)A.max_grad_norm / (total + 1e-6f);
            clip = fminf(coef, 1.0f);
        }
        A.scalars[0] = clip;
    }
    if (lane < kParamTensors) {
        const int t = lane;
        const int grp = A.group[t];
        const int step = it + 1;  // every group steps every iteration
        const double lr = (grp == 0 && A.lr_table) ? A.lr_table[min(it, A.lr_table_len - 1)] : A.lr[grp];
        const double bc1 = 1.0 - pow(A.beta1, (double)step);
        const double bc2 = 1.0 - pow(A.beta2, (double)step);
        const double bc3s = sqrt(1.0 - pow(A.beta3, (double)step));
        float* o = A.scalars + 8 + 8 * t;
        const bool skip = A.skip && A.skip[0] != 0;
        // frozen during warm-up: no gradient; skipped step: nothing changes
        o[0] = (!skip && !A.frozen_always[t] && it >= A.first_iter[t]) ? 1.0f : 0.0f;
        o[1] = (it == A.first_iter[t]) ? 1.0f : 0.0f;  // state created now: zeros, neg_pre_grad = -grad*clip
        o[2] = (float)(lr / bc1);
        o[3] = (float)(lr * A.beta2 / bc2);
        o[4] = (float)bc3s;
        o[5] = (float)(lr * A.weight_decay);
    }
}

__global__ void __launch_bounds__(256) adan_kernel(AdanDev A) {
    const int t = blockIdx.y;
    const float* sc = A.scalars + 8 + 8 * t;
    if (sc[0] == 0.0f) return;
    const int n = A.numel[t];
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x * blockDim.x >= n) return;
    const float clip = A.scalars[0];
    const bool fresh = sc[1] != 0.0f;
    const float step_size = sc[2], step_size_diff = sc[3], bc3f = sc[4], wd = sc[5];
    const float b1 = (float)A.beta1, b2 = (float)A.beta2, b3 = (float)A.beta3;
    const float ob1 = (float)(1.0 - A.beta1), ob2 = (float)(1.0 - A.beta2), ob3 = (float)(1.0 - A.beta3);
    const float eps = (float)A.eps;

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

// The same update in one pass over all tensors, four elements per thread with float4 accesses,
// for the fit's layout: every array (parameters, gradients, each state vector) holds the tensors
// back to back at the same offsets. end[t] = the flat index one past tensor t. Elements of a
// tensor that does not step this iteration are written back unchanged; the per-element arithmetic
// and its order are those of adan_kernel.
struct AdanFlat {
    int end[kParamTensors];
    int total;
};
__global__ void __launch_bounds__(256) adan_flat4_kernel(AdanDev A, AdanFlat F) {
    const int i0 = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
    if (i0 >= F.total) return;
    const float clip = A.scalars[0];
    const float b1 = (float)A.beta1, b2 = (float)A.beta2, b3 = (float)A.beta3;
    const float ob1 = (float)(1.0 - A.beta1), ob2 = (float)(1.0 - A.beta2), ob3 = (float)(1.0 - A.beta3);
    const float eps = (float)A.eps;
    float4 G4 = *reinterpret_cast<const float4*>(A.grad[0] + i0);
    float4 M4 = *reinterpret_cast<const float4*>(A.exp_avg[0] + i0);
    float4 V4 = *reinterpret_cast<const float4*>(A.exp_avg_sq[0] + i0);
    float4 D4 = *reinterpret_cast<const float4*>(A.exp_avg_diff[0] + i0);
    float4 N4 = *reinterpret_cast<const float4*>(A.neg_pre_grad[0] + i0);
    float4 P4 = *reinterpret_cast<const float4*>(A.param[0] + i0);
    float* Gv = &G4.x;
    float* Mv = &M4.x;
    float* Vv = &V4.x;
    float* Dv = &D4.x;
    float* Nv = &N4.x;
    float* Pv = &P4.x;
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int i = i0 + e;
        int t = 0;
#pragma unroll
        for (int k = 0; k < kParamTensors - 1; k++) t += i >= F.end[k] ? 1 : 0;
        const float* sc = A.scalars + 8 + 8 * t;
        if (sc[0] == 0.0f) continue;
        const bool fresh = sc[1] != 0.0f;
        const float step_size = sc[2], step_size_diff = sc[3], bc3f = sc[4], wd = sc[5];
        float g = Gv[e] * clip;
        float m = fresh ? 0.f : Mv[e], v = fresh ? 0.f : Vv[e], d = fresh ? 0.f : Dv[e];
        float ng = fresh ? -g : Nv[e];
        ng = ng + g;
        m = m * b1 + ob1 * g;
        d = d * b2 + ob2 * ng;
        ng = ng * b2 + g;
        v = v * b3 + ob3 * ng * ng;
        const float denom = sqrtf(v) / bc3f + eps;
        float p = Pv[e];
        if (A.no_prox) {
            p = p * (1.0f - wd);
            p = p + (-step_size) * (m / denom);
            p = p + (-step_size_diff) * (d / denom);
        } else {
            p = p + (-step_size) * (m / denom);
            p = p + (-step_size_diff) * (d / denom);
            p = p / (1.0f + wd);
        }
        Pv[e] = p;
        Mv[e] = m;
        Vv[e] = v;
        Dv[e] = d;
        Nv[e] = -g;
        Gv[e] = g;
    }
    *reinterpret_cast<float4*>(A.grad[0] + i0) = G4;
    *reinterpret_cast<float4*>(A.exp_avg[0] + i0) = M4;
    *reinterpret_cast<float4*>(A.exp_avg_sq[0] + i0) = V4;
    *reinterpret_cast<float4*>(A.exp_avg_diff[0] + i0) = D4;
    *reinterpret_cast<float4*>(A.neg_pre_grad[0] + i0) = N4;
    *reinterpret_cast<float4*>(A.param[0] + i0) = P4;
}

// True when the tensors are back to back in every array and the flat arrays allow float4 access.
static bool adan_flat_layout(const AdanDev& A, AdanFlat* F) {
    long long off = 0;
    for (int t = 0; t < kParamTensors; t++) {
        float* const arrs[6] = {A.param[t], A.grad[t], A.exp_avg[t], A.exp_avg_sq[t], A.exp_avg_diff[t],
                                A.neg_pre_grad[t]};
        float* const bases[6] = {A.param[0], A.grad[0], A.exp_avg[0], A.exp_avg_sq[0], A.exp_avg_diff[0],
                                 A.neg_pre_grad[0]};
        for (int k = 0; k < 6; k++)
            if (arrs[k] != bases[k] + off) return false;
        off += A.numel[t];
        F->end[t] = (int)off;
    }
    if (off % 4 != 0 || off > 0x7fffffffLL) return false;
    F->total = (int)off;
    float* const bases[6] = {A.param[0], A.grad[0], A.exp_avg[0], A.exp_avg_sq[0], A.exp_avg_diff[0],
                             A.neg_pre_grad[0]};
    for (int k = 0; k < 6; k++)
        if ((uintptr_t)bases[k] & 15) return false;
    return true;
}

void launch_adan(const AdanDev& A, const int32_t* iteration, cudaStream_t s) {
    int maxn = 1;
    for (int t = 0; t < kParamTensors; t++) maxn = max(maxn, A.numel[t]);
    const unsigned bx = min(ceil_div(maxn, 256), 4096u);
    dim3 grid(bx, kParamTensors);
    adan_scalars_kernel<<<1, 32, 0, s>>>(A, iteration);
    AdanFlat F;
    if (adan_flat_layout(A, &F)) {
        adan_flat4_kernel<<<ceil_div((size_t)F.total / 4, 256), 256, 0, s>>>(A, F);
        return;
    }
    adan_kernel<<<grid, 256, 0, s>>>(A);
}

}  // namespace cvqpg

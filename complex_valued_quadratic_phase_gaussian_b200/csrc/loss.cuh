// Internal interface of the fused multi-plane loss (loss.cu).
#pragma once

#include "common.cuh"

namespace cvqpg {

constexpr int kMaxLossPlanes = 8;

struct LossDev {
    int C, P, H, W;
    float w0, w1, w2;      // L2, masked L2, correlation L2 weights
    float ssim_weight;     // 0.025 * 0.2 in the reference
    float noise_ratio;     // 1e-3 in the reference
    int inject_noise;
    unsigned long long seed;
    float c1, c2;          // (K1 L)^2, (K2 L)^2 with L = 1
    float inv_n, inv_nmap; // 1/(C H W), 1/(C (H-10) (W-10))
    const float2* tmom;    // optional target moments (mu_T, E_w[T^2]) [P*C][H-10][W-10]
};

int loss_make_dev(const cvqpg_loss_params* q, LossDev* L);
size_t loss_partials_floats(const LossDev& L);
void launch_loss(const LossDev& L, const float* pred, const float* targets, const uint8_t* depth_plane,
                 const float* noise_scale, const int* iteration, float* grad_pred, float* partials, float* out,
                 cudaStream_t stream);
size_t target_moments_bytes(const LossDev& L);
void launch_target_moments(const LossDev& L, const float* targets, float2* mom, cudaStream_t stream);
void launch_target_range(const float* targets, int planes, size_t plane_elems, float* range_out, void* scratch,
                         cudaStream_t stream);

}  // namespace cvqpg

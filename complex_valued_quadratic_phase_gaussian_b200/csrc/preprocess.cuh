// Internal interface of the preprocessing kernels and the fused Adan step.
#pragma once

#include "raster.cuh"

namespace cvqpg {

// Raw (pre-activation) parameters, the Gaussians2D tensors
// (model_2d_gaussian_rgb.py:18-26): means_2d [N,2], pre_act_scales [N,2],
// pre_act_rotation [N], colours [N,C], pre_act_phase [N,C],
// pre_act_opacities [N], curvature [N].
struct RawParams {
    const float* means;
    const float* scales;
    const float* rotation;
    const float* colours;
    const float* phase;
    const float* opac;
    const float* curv;
};

struct RawGrads {
    float* means;
    float* scales;
    float* rotation;
    float* colours;
    float* phase;
    float* opac;
    float* curv;
};

struct SplatGradsIn {
    const float* d_means;
    const float* d_inv;
    const float* d_col;
    const float* d_ph;
    const float* d_op;
    const float* d_cv;
    const float* d_ar;
};

struct PreDev {
    int n;
    int W, H;              // image size (means scale)
    int curv_mode;         // 0 off, 1 constant, 2 scale_aware
    float curv_const;      // 200 in the reference ('constant' mode)
    float eta_lambda;      // curv_nyquist * lambda (min wavelength for RGB, wavelengths[0] for grayscale)
    float dxy_sq;          // pixel_pitch^2
    int curv_trainable;    // 0 for the 'flat' primitive
    int curv_warmup;       // iterations with frozen curvature
};

void launch_preprocess_forward(int channels, const PreDev& P, const RawParams& raw, float* rec, int32_t* radii,
                               float* radius3, uint32_t* tiles_touched, const BinRule& rule, cudaStream_t s);
int preprocess_backward_blocks(int n);
void launch_preprocess_backward(int channels, const PreDev& P, const RawParams& raw, const SplatGradsIn& gin,
                                const RawGrads& out, const int32_t* iteration, float* partials, cudaStream_t s);

// ---- Adan (utils/optimizer.py:104-262) -------------------------------------
constexpr int kParamTensors = 7;  // means, scales, rotation, colours, phase, opacities, curvature

struct AdanDev {
    float* param[kParamTensors];
    float* grad[kParamTensors];
    float* exp_avg[kParamTensors];
    float* exp_avg_sq[kParamTensors];
    float* exp_avg_diff[kParamTensors];
    float* neg_pre_grad[kParamTensors];
    int numel[kParamTensors];
    int group[kParamTensors];        // param group of each tensor
    int first_iter[kParamTensors];   // iteration at which the tensor first has a gradient
    int frozen_always[kParamTensors];
    double lr[8];                    // constant lr per group (group 0 may use lr_table)
    const double* lr_table;          // per-iteration lr of group 0 (means cosine schedule), or null
    int lr_table_len;
    double beta1, beta2, beta3, eps, weight_decay;
    int no_prox;
    double max_grad_norm;            // clip_grad_norm_ max_norm applied before the step (<= 0: none)
    const float* norm_partials;      // per-CTA sums of squares from the preprocess adjoint
    int num_partials;
    float* scalars;                  // kAdanScalars floats of scratch: the step's clip factor and step sizes
    const int32_t* skip;             // nullable: when *skip != 0 the step leaves every tensor unchanged
                                     // (the tile-pair list overflowed, so this step's gradient is incomplete)
};

constexpr int kAdanScalars = 8 + 8 * kParamTensors;

void launch_adan(const AdanDev& A, const int32_t* iteration, cudaStream_t s);

}  // namespace cvqpg

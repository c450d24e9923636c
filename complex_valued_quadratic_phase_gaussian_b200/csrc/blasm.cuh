// Internal interface of the BLASM propagation kernels (blasm.cu), shared with
// the fused fit iteration.
#pragma once

#include "fft.cuh"

namespace cvqpg {

constexpr int kMaxPlanes = 8;
constexpr int kMaxPC = kMaxPlanes * kMaxChannels;

// Per (plane, channel) transfer-function constants (in the table blob).
struct PCParam {
    float K;        // 2 pi z / lambda (float)
    float theta0;   // (2 pi z / lambda) mod 2 pi, reduced in double
    int j0, j1;     // centred row-frequency band [j0, j1)
    int i0, i1;     // centred column-frequency band [i0, i1)
    int pad0, pad1;
};

// Everything the kernels need, by value (kernel parameter).
struct BlasmDev {
    int C, P;
    int H, W;          // splat field / output crop (centred)
    int pH, pW;        // padded field
    int NH, NW;        // FFT grid = 2 pH x 2 pW
    int pad_h, pad_w;  // (pH - H)/2, (pW - W)/2
    int out_h, out_w;  // output crop (H, W in the fit; pH, pW for the full reconstruction)
    int input_mode;    // 0: splat field [C,H,W] (+pad, window, amplitude clamp); 1: padded field [C,pH,pW]
    int G;             // columns per column-pass CTA (tiled layout width)
    int col_radix;     // radix the column kernels keep in registers (0 = automatic)
    float scale;       // 1 / (NH * NW)
    FftPlan row, col;  // NW and NH plans
    const float* wy;   // Tukey window [pH]
    const float* wx;   // [pW]
    const float* a_row;  // [C][NH] lambda_c^2 * fr_j^2 (centred index j)
    const float* b_col;  // [C][NW] lambda_c^2 * fc_i^2
    const int2* aperture;  // [NH] allowed centred column interval per centred row
    const PCParam* pcp;    // [P*C]
};

// Build BlasmDev from the public parameters and a device table blob prepared
// by cvqpg_blasm_setup. Returns a CVQPG_* status.
int blasm_make_dev(const cvqpg_blasm_params* prm, const void* tables, size_t table_bytes, BlasmDev* d);

size_t blasm_workspace_bytes(const BlasmDev& d);

// Optional CUDA-event marks between kernels (bench-time stage timing).
struct StageMarks {
    cudaEvent_t* ev = nullptr;
    int n = 0;
    int idx = 0;
    void mark(cudaStream_t s) {
        if (ev && idx < n) cudaEventRecord(ev[idx++], s);
    }
};

// pred (nullable): also write clamp(|V|^2, 0, 1) [P*C][out_h][out_w].
void blasm_forward(const BlasmDev& d, const float2* in, float2* out, float* pred, void* workspace,
                   cudaStream_t stream, StageMarks* marks = nullptr);
// Either grad_out = dL/dV, or (grad_pred = dL/dpred, vfield = V) with dL/dV formed on load.
void blasm_backward(const BlasmDev& d, const float2* in_field, const float2* grad_out, const float* grad_pred,
                    const float2* vfield, float2* grad_in, void* workspace, cudaStream_t stream,
                    StageMarks* marks = nullptr);

}  // namespace cvqpg

// Per-Gaussian preprocessing (activations, covariance, inverse, culling radius,
// tile count) and its adjoint, fused with the gradient sanitation of the fit loop.
//
// Reference (paths inside the reference project):
//   model_2d_gaussian_rgb.py:83-112    apply_activations (tanh means, exp scales + 0.1, phase mod 2pi,
//                                      sigmoid opacity, curvature bound modes off/constant/scale_aware)
//   model_2d_gaussian_grayscale.py:96  grayscale binds the bound to wavelengths[0]
//   model_2d_gaussian_rgb.py:114-153   covariance + 0.1 I, inverse with det clamped >= 1e-10
//   model_2d_gaussian_rgb.py:429-436   area = |sx sy|, radius = ceil(5 sqrt(lambda_max))
//   train_2d_gaussian_rgb.py:205-209   nan_to_num on every gradient, then clip_grad_norm_(1.0)
// The adjoint is derived by hand from the same formulas (max over the two
// scales routes the curvature-bound gradient to the first maximal entry, the
// det clamp passes gradient only where det >= 1e-10, the phase modulo has slope 1).
#include "preprocess.cuh"

namespace cvqpg {

__device__ __forceinline__ float torch_remainder(float a, float b) {
    float r = fmodf(a, b);
    if (r != 0.0f && ((r < 0.0f) != (b < 0.0f))) r += b;
    return r;
}

template <int C>
__global__ void preprocess_forward_kernel(PreDev P, RawParams raw, float* __restrict__ rec,
                                          int32_t* __restrict__ radii, float* __restrict__ radius3,
                                          uint32_t* __restrict__ tiles_touched, BinRule rule) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P.n) return;
    const float t0 = tanhf(raw.means[2 * g]), t1 = tanhf(raw.means[2 * g + 1]);
    const float mx = (t0 + 1.0f) * 0.5f * (float)P.W;
    const float my = (t1 + 1.0f) * 0.5f * (float)P.H;
    const float sx = expf(raw.scales[2 * g]) + 0.1f, sy = expf(raw.scales[2 * g + 1]) + 0.1f;
    const float rot = raw.rotation[g];
    const float opac = 1.0f / (1.0f + expf(-raw.opac[g]));
    const float sigma = fmaxf(sx, sy);
    float curv = 0.0f;
    if (P.curv_mode == 1) {
        curv = P.curv_const * tanhf(raw.curv[g]);
    } else if (P.curv_mode == 2) {
        const float cmax = P.eta_lambda / (6.0f * sigma * P.dxy_sq + 1e-20f);
        curv = cmax * tanhf(raw.curv[g]);
    }
    float sn, cs;
    sincosf(rot, &sn, &cs);
    const float sx2 = sx * sx, sy2 = sy * sy, cs2 = cs * cs, sn2 = sn * sn, csn = cs * sn;
    const float c00 = sx2 * cs2 + sy2 * sn2 + 0.1f;
    const float c01 = (sx2 - sy2) * csn;
    const float c11 = sx2 * sn2 + sy2 * cs2 + 0.1f;
    const float det = fmaxf(c00 * c11 - c01 * c01, 1e-10f);
    const float idet = 1.0f / det;
    const float area = fabsf(sx * sy);

    float v[kRecordFloats];
    v[0] = mx;
    v[1] = my;
    v[2] = c11 * idet;
    v[3] = -c01 * idet;
    v[4] = c00 * idet;
    v[5] = opac;
    v[6] = curv;
    v[7] = area;
    const float two_pi = 6.28318530717958648f;
#pragma unroll
    for (int c = 0; c < C; c++) {
        v[8 + c] = raw.colours[g * C + c];
        v[8 + C + c] = torch_remainder(raw.phase[g * C + c], two_pi);
    }
#pragma unroll
    for (int i = 8 + 2 * C; i < kRecordFloats; i++) v[i] = 0.0f;
    float4* dst = reinterpret_cast<float4*>(rec + (size_t)g * kRecordFloats);
#pragma unroll
    for (int q = 0; q < 4; q++) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);

    const float mid = 0.5f * (c00 + c11);
    const float disc = sqrtf(((c00 - c11) * 0.5f) * ((c00 - c11) * 0.5f) + c01 * c01);
    const float lmax = sqrtf(mid + disc);
    radii[g] = (int32_t)ceilf(5.0f * lmax);
    if (radius3) radius3[g] = 3.0f * lmax;
    uint32_t cnt = 0;
    for_each_list_tile(rule, mx, my, g, [&](int) { cnt++; });
    tiles_touched[g] = cnt;
}

// Adjoint. Writes the raw-parameter gradients (nan/inf -> 0) into `out`, and the
// per-CTA sum of squares of the trainable gradients into partials[blockIdx.x].
template <int C>
__global__ void __launch_bounds__(256) preprocess_backward_kernel(PreDev P, RawParams raw, SplatGradsIn gin,
                                                                  RawGrads out, const int32_t* __restrict__ iteration,
                                                                  float* __restrict__ partials) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int it = iteration ? iteration[0] : 0;
    const bool curv_trainable = P.curv_trainable && it >= P.curv_warmup;
    float ss = 0.0f;
    if (g < P.n) {
        // recompute the activations
        const float t0 = tanhf(raw.means[2 * g]), t1 = tanhf(raw.means[2 * g + 1]);
        const float es0 = expf(raw.scales[2 * g]), es1 = expf(raw.scales[2 * g + 1]);
        const float sx = es0 + 0.1f, sy = es1 + 0.1f;
        const float rot = raw.rotation[g];
        const float opac = 1.0f / (1.0f + expf(-raw.opac[g]));
        const float tc = tanhf(raw.curv[g]);
        const bool sx_is_max = sx >= sy;  // torch.max(dim) picks the first maximal entry
        const float sigma = sx_is_max ? sx : sy;
        float sn, cs;
        sincosf(rot, &sn, &cs);
        const float sx2 = sx * sx, sy2 = sy * sy;
        const float c00 = sx2 * cs * cs + sy2 * sn * sn + 0.1f;
        const float c01 = (sx2 - sy2) * cs * sn;
        const float c11 = sx2 * sn * sn + sy2 * cs * cs + 0.1f;
        const float det_raw = c00 * c11 - c01 * c01;
        const float det = fmaxf(det_raw, 1e-10f);

        const float gmx = gin.d_means[2 * g], gmy = gin.d_means[2 * g + 1];
        const float gi00 = gin.d_inv[3 * g], gi01 = gin.d_inv[3 * g + 1], gi11 = gin.d_inv[3 * g + 2];
        const float gop = gin.d_op[g], gcv = gin.d_cv[g], gar = gin.d_ar[g];

        // means
        float d_m0 = gmx * 0.5f * (float)P.W * (1.0f - t0 * t0);
        float d_m1 = gmy * 0.5f * (float)P.H * (1.0f - t1 * t1);
        // opacity
        float d_o = gop * opac * (1.0f - opac);
        // curvature and its bound
        float d_c = 0.0f, g_sigma = 0.0f;
        if (P.curv_mode == 1) {
            d_c = gcv * P.curv_const * (1.0f - tc * tc);
        } else if (P.curv_mode == 2) {
            const float den = 6.0f * sigma * P.dxy_sq + 1e-20f;
            const float cmax = P.eta_lambda / den;
            d_c = gcv * cmax * (1.0f - tc * tc);
            g_sigma = gcv * tc * (-P.eta_lambda * 6.0f * P.dxy_sq / (den * den));
        }
        // inverse covariance
        const float idet2 = 1.0f / (det * det);
        float g_det = -(gi00 * c11 - gi01 * c01 + gi11 * c00) * idet2;
        if (!(det_raw >= 1e-10f)) g_det = 0.0f;
        const float g_c00 = gi11 / det + g_det * c11;
        const float g_c11 = gi00 / det + g_det * c00;
        const float g_c01 = -gi01 / det - 2.0f * c01 * g_det;
        // covariance -> scales, rotation; area -> scales
        float g_sx = g_c00 * 2.f * sx * cs * cs + g_c01 * 2.f * sx * cs * sn + g_c11 * 2.f * sx * sn * sn + gar * sy;
        float g_sy = g_c00 * 2.f * sy * sn * sn - g_c01 * 2.f * sy * cs * sn + g_c11 * 2.f * sy * cs * cs + gar * sx;
        float d_rot = g_c00 * 2.f * cs * sn * (sy2 - sx2) + g_c01 * (sx2 - sy2) * (cs * cs - sn * sn) +
                      g_c11 * 2.f * sn * cs * (sx2 - sy2);
        if (sx_is_max) g_sx += g_sigma; else g_sy += g_sigma;
        float d_s0 = g_sx * es0, d_s1 = g_sy * es1;

        auto clean = [](float x) { return isfinite(x) ? x : 0.0f; };  // torch.nan_to_num(nan=0, posinf=0, neginf=0)
        d_m0 = clean(d_m0);
        d_m1 = clean(d_m1);
        d_s0 = clean(d_s0);
        d_s1 = clean(d_s1);
        d_rot = clean(d_rot);
        d_o = clean(d_o);
        d_c = curv_trainable ? clean(d_c) : 0.0f;
        out.means[2 * g] = d_m0;
        out.means[2 * g + 1] = d_m1;
        out.scales[2 * g] = d_s0;
        out.scales[2 * g + 1] = d_s1;
        out.rotation[g] = d_rot;
        out.opac[g] = d_o;
        out.curv[g] = d_c;
        ss = d_m0 * d_m0 + d_m1 * d_m1 + d_s0 * d_s0 + d_s1 * d_s1 + d_rot * d_rot + d_o * d_o + d_c * d_c;
#pragma unroll
        for (int c = 0; c < C; c++) {
            const float a = clean(gin.d_col[g * C + c]);
            const float b = clean(gin.d_ph[g * C + c]);
            out.colours[g * C + c] = a;
            out.phase[g * C + c] = b;
            ss += a * a + b * b;
        }
    }
    // deterministic block reduction
    __shared__ float red[8];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += red[k];
        partials[blockIdx.x] = s;
    }
}

void launch_preprocess_forward(int channels, const PreDev& P, const RawParams& raw, float* rec, int32_t* radii,
                               float* radius3, uint32_t* tiles_touched, const BinRule& rule, cudaStream_t s) {
    if (P.n <= 0) return;
    const unsigned blocks = ceil_div(P.n, 256);
    if (channels == 1)
        preprocess_forward_kernel<1><<<blocks, 256, 0, s>>>(P, raw, rec, radii, radius3, tiles_touched, rule);
    else
        preprocess_forward_kernel<3><<<blocks, 256, 0, s>>>(P, raw, rec, radii, radius3, tiles_touched, rule);
}

int preprocess_backward_blocks(int n) { return (int)ceil_div(n > 0 ? n : 1, 256); }

void launch_preprocess_backward(int channels, const PreDev& P, const RawParams& raw, const SplatGradsIn& gin,
                                const RawGrads& out, const int32_t* iteration, float* partials, cudaStream_t s) {
    const int blocks = preprocess_backward_blocks(P.n);
    if (channels == 1)
        preprocess_backward_kernel<1><<<blocks, 256, 0, s>>>(P, raw, gin, out, iteration, partials);
    else
        preprocess_backward_kernel<3><<<blocks, 256, 0, s>>>(P, raw, gin, out, iteration, partials);
}

}  // namespace cvqpg

using namespace cvqpg;

static int preprocess_dev(const cvqpg_preprocess_params* q, PreDev* P) {
    if (!q) return CVQPG_ERR_ARG;
    if (q->channels != 1 && q->channels != 3) return CVQPG_ERR_CHANNELS;
    if (q->num_gaussians < 0 || q->width <= 0 || q->height <= 0 || q->curv_mode < 0 || q->curv_mode > 2)
        return CVQPG_ERR_ARG;
    P->n = q->num_gaussians;
    P->W = q->width;
    P->H = q->height;
    P->curv_mode = q->curv_mode;
    P->curv_const = (float)q->curv_const;
    double lam = q->wavelengths[0];
    if (q->channels == 3)
        for (int c = 1; c < 3; c++) lam = q->wavelengths[c] < lam ? q->wavelengths[c] : lam;
    P->eta_lambda = (float)(q->curv_nyquist * lam);
    P->dxy_sq = (float)(q->pixel_pitch * q->pixel_pitch);
    P->curv_trainable = q->curv_trainable;
    P->curv_warmup = q->curv_trainable ? q->warmup_iters : 0;
    return CVQPG_OK;
}

static RawParams raw_views(const float* params, int N, int C) {
    return RawParams{params, params + 2 * N, params + 4 * N, params + 5 * N, params + (5 + C) * N,
                     params + (5 + 2 * C) * N, params + (6 + 2 * C) * N};
}

extern "C" int cvqpg_preprocess_forward(const cvqpg_preprocess_params* q, const float* params, float* records,
                                        int32_t* radii, float* radius3, uint32_t* tiles_touched, void* stream) {
    PreDev P;
    const int st = preprocess_dev(q, &P);
    if (st != CVQPG_OK) return st;
    if (P.n > 0 && (!params || !records || !radii || !tiles_touched)) return CVQPG_ERR_ARG;
    const int C = q->channels;
    const BinRule rule = make_bin_rule(CVQPG_CULL_CUDA16_5SIGMA, q->width, q->height, radii, nullptr);
    launch_preprocess_forward(C, P, raw_views(params, P.n, C), records, radii, radius3, tiles_touched, rule,
                              (cudaStream_t)stream);
    return launch_status();
}

extern "C" int cvqpg_preprocess_partials(int num_gaussians) { return preprocess_backward_blocks(num_gaussians); }

extern "C" int cvqpg_preprocess_backward(const cvqpg_preprocess_params* q, const float* params,
                                         const float* splat_grads, float* grads, const int32_t* iteration,
                                         float* partials, void* stream) {
    PreDev P;
    const int st = preprocess_dev(q, &P);
    if (st != CVQPG_OK) return st;
    if (!partials || (P.n > 0 && (!params || !splat_grads || !grads))) return CVQPG_ERR_ARG;
    const int N = P.n, C = q->channels;
    const float* sg = splat_grads;
    const SplatGradsIn gin{sg, sg + 2 * N, sg + 5 * N, sg + (5 + C) * N, sg + (5 + 2 * C) * N,
                           sg + (6 + 2 * C) * N, sg + (7 + 2 * C) * N};
    float* g = grads;
    const RawGrads out{g, g + 2 * N, g + 4 * N, g + 5 * N, g + (5 + C) * N, g + (5 + 2 * C) * N,
                       g + (6 + 2 * C) * N};
    launch_preprocess_backward(C, P, raw_views(params, N, C), gin, out, iteration, partials, (cudaStream_t)stream);
    return launch_status();
}


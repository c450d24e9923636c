// Fused multi-plane loss: L2 + masked L2 + correlation L2 + SSIM, with the
// fresh target noise of every iteration, and dL/d(pred) in the same pass.
//
// Reference (paths inside the reference project):
//   utils/propagator.py:417-449   multiplane_loss_odak.__call__ (weights [1,1,1], inject_noise=True)
//   utils/data_utils.py:22-63     GaussianLoss: 0.025 * 0.2 * (1 - SSIM), pytorch_msssim defaults
//   utils/data_utils.py:66-82     loss factory (weights, blur settings)
//   train_2d_gaussian_rgb.py:192-199  per plane: crop, clamp to [0,1], loss + SSIM, PSNR of plane 0
//
// For plane p with pred = clamp(|V_p|^2, 0, 1), target T, mask M = [depth == p]
// and noisy target N = T + (z * ratio) * (max T - min T), z ~ N(0,1) fresh:
//   L_p = w0 mean((pred-T)^2) + w1 mean((pred M - N M)^2) + w2 mean((pred N - N N)^2)
//         + ssim_w (1 - SSIM(pred, T))
// One CTA owns a 32x32 tile of one (plane, channel) image. SSIM needs the
// windowed moments of a 10-pixel halo on each side: the CTA stages a 52x52
// block, filters it separably (11 taps, sigma 1.5, valid), forms the SSIM map
// and its three partial-derivative maps on the 42x42 map positions that touch
// the tile, then applies the transposed filter to get dSSIM/dpred on the tile.
// Per-CTA partial sums (weighted L2, plain MSE, SSIM map sum) go to a fixed
// slot; a finalize kernel reduces them in a fixed order (deterministic).
#include "loss.cuh"

namespace cvqpg {

constexpr int kLT = 32;              // owned tile edge
constexpr int kLH = kLT + 20;        // staged block edge (52)
constexpr int kLM = kLT + 10;        // map positions touching the tile (42)
constexpr int kLossThreads = 256;

// Gaussian window, 11 taps, sigma 1.5, normalised (computed in double, rounded once).
__device__ __forceinline__ float ssim_w(int k) {
    constexpr float w[11] = {1.028380082e-03f, 7.598758612e-03f, 3.600077721e-02f, 1.093606895e-01f,
                             2.130055428e-01f, 2.660117810e-01f, 2.130055428e-01f, 1.093606895e-01f,
                             3.600077721e-02f, 7.598758612e-03f, 1.028380082e-03f};
    return w[k];
}

__global__ void __launch_bounds__(kLossThreads) loss_kernel(LossDev L, const float* __restrict__ pred,
                                                             const float* __restrict__ target,
                                                             const uint8_t* __restrict__ depth_plane,
                                                             const float* __restrict__ noise_scale,
                                                             const int* __restrict__ iteration,
                                                             float* __restrict__ grad_pred,
                                                             float* __restrict__ partials) {
    extern __shared__ float lsm[];
    float* sX = lsm;                       // [52][52]
    float* sY = sX + kLH * kLH;            // [52][52]
    float* hM = sY + kLH * kLH;            // 5 maps [52][42]
    float* dM = hM + 5 * kLH * kLM;        // 3 maps [42][42]
    float* tM = sX;                        // 3 maps [42][32], reuses sX/sY/hM space after use
    __shared__ float red[3][kLossThreads / 32];

    const int H = L.H, W = L.W;
    const int tiles_x = (W + kLT - 1) / kLT, tiles_y = (H + kLT - 1) / kLT;
    const int tiles = tiles_x * tiles_y;
    const int pc = blockIdx.x / tiles, tile = blockIdx.x - pc * tiles;
    const int p = pc / L.C;
    const int y0 = (tile / tiles_x) * kLT, x0 = (tile % tiles_x) * kLT;
    const size_t plane_off = (size_t)pc * H * W;
    const float* X = pred + plane_off;
    const float* Y = target + plane_off;

    // 1. stage the 52x52 block (zeros outside the image; never used by valid map entries)
    for (int i = threadIdx.x; i < kLH * kLH; i += blockDim.x) {
        const int r = i / kLH, q = i - r * kLH;
        const int y = y0 - 10 + r, x = x0 - 10 + q;
        const bool in = (unsigned)y < (unsigned)H && (unsigned)x < (unsigned)W;
        sX[i] = in ? __ldg(&X[(size_t)y * W + x]) : 0.f;
        sY[i] = in ? __ldg(&Y[(size_t)y * W + x]) : 0.f;
    }
    __syncthreads();
    // 2. horizontal filter -> 5 moment maps on [52][42]
    for (int i = threadIdx.x; i < kLH * kLM; i += blockDim.x) {
        const int r = i / kLM, q = i - r * kLM;
        float a = 0.f, b = 0.f, aa = 0.f, bb = 0.f, ab = 0.f;
#pragma unroll
        for (int k = 0; k < 11; k++) {
            const float w = ssim_w(k), x = sX[r * kLH + q + k], y = sY[r * kLH + q + k];
            a = fmaf(w, x, a);
            b = fmaf(w, y, b);
            aa = fmaf(w, x * x, aa);
            bb = fmaf(w, y * y, bb);
            ab = fmaf(w, x * y, ab);
        }
        hM[0 * kLH * kLM + i] = a;
        hM[1 * kLH * kLM + i] = b;
        hM[2 * kLH * kLM + i] = aa;
        hM[3 * kLH * kLM + i] = bb;
        hM[4 * kLH * kLM + i] = ab;
    }
    __syncthreads();
    // 3. vertical filter -> SSIM map and its partials on the valid map positions
    const float C1 = L.c1, C2 = L.c2;
    float ssim_sum = 0.f;
    for (int i = threadIdx.x; i < kLM * kLM; i += blockDim.x) {
        const int ii = i / kLM, jj = i - ii * kLM;
        const int mi = y0 - 10 + ii, mj = x0 - 10 + jj;
        float dm = 0.f, dxx = 0.f, dxy = 0.f;
        if ((unsigned)mi < (unsigned)(H - 10) && (unsigned)mj < (unsigned)(W - 10)) {
            float mu1 = 0.f, mu2 = 0.f, exx = 0.f, eyy = 0.f, exy = 0.f;
#pragma unroll
            for (int k = 0; k < 11; k++) {
                const float w = ssim_w(k);
                const int o = (ii + k) * kLM + jj;
                mu1 = fmaf(w, hM[0 * kLH * kLM + o], mu1);
                mu2 = fmaf(w, hM[1 * kLH * kLM + o], mu2);
                exx = fmaf(w, hM[2 * kLH * kLM + o], exx);
                eyy = fmaf(w, hM[3 * kLH * kLM + o], eyy);
                exy = fmaf(w, hM[4 * kLH * kLM + o], exy);
            }
            const float s11 = exx - mu1 * mu1, s22 = eyy - mu2 * mu2, s12 = exy - mu1 * mu2;
            const float A1 = 2.f * mu1 * mu2 + C1, A2 = 2.f * s12 + C2;
            const float B1 = mu1 * mu1 + mu2 * mu2 + C1, B2 = s11 + s22 + C2;
            const float iB1 = 1.f / B1, iB2 = 1.f / B2;
            const float smap = A1 * A2 * iB1 * iB2;
            if (ii >= 10 && jj >= 10) ssim_sum += smap;  // owned map position
            dm = 2.f * mu2 * A2 * iB1 * iB2 - 2.f * mu1 * smap * iB1 + A1 * iB1 * (-2.f * mu2 * iB2 + 2.f * mu1 * A2 * iB2 * iB2);
            dxx = -smap * iB2;
            dxy = 2.f * A1 * iB1 * iB2;
        }
        dM[0 * kLM * kLM + i] = dm;
        dM[1 * kLM * kLM + i] = dxx;
        dM[2 * kLM * kLM + i] = dxy;
    }
    __syncthreads();
    // 4. transposed horizontal filter -> [42][32]
    for (int i = threadIdx.x; i < kLM * kLT; i += blockDim.x) {
        const int ii = i / kLT, xx = i - ii * kLT;
        float a = 0.f, b = 0.f, c = 0.f;
#pragma unroll
        for (int k = 0; k < 11; k++) {
            const float w = ssim_w(k);
            const int o = ii * kLM + xx + 10 - k;
            a = fmaf(w, dM[0 * kLM * kLM + o], a);
            b = fmaf(w, dM[1 * kLM * kLM + o], b);
            c = fmaf(w, dM[2 * kLM * kLM + o], c);
        }
        tM[0 * kLM * kLT + i] = a;
        tM[1 * kLM * kLT + i] = b;
        tM[2 * kLM * kLT + i] = c;
    }
    __syncthreads();
    // 5. transposed vertical filter + L2 terms on the owned tile
    const float inv_n = L.inv_n, ssim_scale = -L.ssim_weight * L.inv_nmap;
    const float nscale = noise_scale[p];
    const uint64_t it = iteration ? (uint64_t)(uint32_t)iteration[0] : 0ull;
    float l2_sum = 0.f, mse_sum = 0.f;
    for (int i = threadIdx.x; i < kLT * kLT; i += blockDim.x) {
        const int yy = i / kLT, xx = i - yy * kLT;
        const int y = y0 + yy, x = x0 + xx;
        if (y >= H || x >= W) continue;
        float gm = 0.f, gxx = 0.f, gxy = 0.f;
#pragma unroll
        for (int k = 0; k < 11; k++) {
            const float w = ssim_w(k);
            const int o = (yy + 10 - k) * kLT + xx;
            gm = fmaf(w, tM[0 * kLM * kLT + o], gm);
            gxx = fmaf(w, tM[1 * kLM * kLT + o], gxx);
            gxy = fmaf(w, tM[2 * kLM * kLT + o], gxy);
        }
        const size_t e = (size_t)y * W + x;
        const float xv = __ldg(&X[e]), tv = __ldg(&Y[e]);
        const float m = (__ldg(&depth_plane[e]) == p) ? 1.f : 0.f;
        float nv = tv;
        if (L.inject_noise) {
            const float z = normal_at(L.seed, it, plane_off + e);
            nv = tv + (z * L.noise_ratio) * nscale;
        }
        const float d0 = xv - tv, d1 = (xv * m - nv * m), d2 = (xv * nv - nv * nv);
        l2_sum += L.w0 * d0 * d0 + L.w1 * d1 * d1 + L.w2 * d2 * d2;
        mse_sum += d0 * d0;
        const float g_l2 = 2.f * inv_n * (L.w0 * d0 + L.w1 * d1 * m + L.w2 * d2 * nv);
        const float g_ssim = ssim_scale * (gm + 2.f * xv * gxx + tv * gxy);
        grad_pred[plane_off + e] = g_l2 + g_ssim;
    }
    // 6. block reduction of the three partial sums
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l2_sum += __shfl_xor_sync(0xffffffffu, l2_sum, o);
        mse_sum += __shfl_xor_sync(0xffffffffu, mse_sum, o);
        ssim_sum += __shfl_xor_sync(0xffffffffu, ssim_sum, o);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][w] = l2_sum;
        red[1][w] = mse_sum;
        red[2][w] = ssim_sum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float a = 0.f, b = 0.f, c = 0.f;
        for (int k = 0; k < kLossThreads / 32; k++) {
            a += red[0][k];
            b += red[1][k];
            c += red[2][k];
        }
        float* dst = partials + (size_t)blockIdx.x * 3;
        dst[0] = a;
        dst[1] = b;
        dst[2] = c;
    }
}

// out[0] = total loss, out[1 + p] = MSE of plane p, out[1 + P + p] = SSIM of plane p,
// out[1 + 2P + p] = loss of plane p. Fixed-order double accumulation.
__global__ void loss_finalize_kernel(LossDev L, const float* __restrict__ partials, float* __restrict__ out) {
    const int tiles = ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    __shared__ double acc[kMaxLossPlanes][3];
    const int p = threadIdx.x;
    if (p < L.P) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int ch = 0; ch < L.C; ch++)
            for (int t = 0; t < tiles; t++) {
                const float* s = partials + ((size_t)(p * L.C + ch) * tiles + t) * 3;
                a += s[0];
                b += s[1];
                c += s[2];
            }
        acc[p][0] = a;
        acc[p][1] = b;
        acc[p][2] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double total = 0.0;
        for (int q = 0; q < L.P; q++) {
            const double mse = acc[q][1] * L.inv_n;
            const double ssim = acc[q][2] * L.inv_nmap;
            const double lp = acc[q][0] * L.inv_n + L.ssim_weight * (1.0 - ssim);
            out[1 + q] = (float)mse;
            out[1 + L.P + q] = (float)ssim;
            out[1 + 2 * L.P + q] = (float)lp;
            total += lp;
        }
        out[0] = (float)total;
    }
}

// per-plane noise scale: ratio applied later; here max(T_p) - min(T_p)
__global__ void target_range_kernel(const float* __restrict__ targets, size_t plane_elems,
                                     float* __restrict__ range_out) {
    const int p = blockIdx.x;
    const float* t = targets + (size_t)p * plane_elems;
    float mx = -INFINITY, mn = INFINITY;
    for (size_t i = threadIdx.x; i < plane_elems; i += blockDim.x) {
        const float v = t[i];
        mx = fmaxf(mx, v);
        mn = fminf(mn, v);
    }
    __shared__ float smx[32], smn[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        smx[threadIdx.x >> 5] = mx;
        smn[threadIdx.x >> 5] = mn;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) {
            mx = fmaxf(mx, smx[k]);
            mn = fminf(mn, smn[k]);
        }
        range_out[p] = fmaxf(mx, smx[0]) - fminf(mn, smn[0]);
    }
}

int loss_make_dev(const cvqpg_loss_params* q, LossDev* L) {
    if (!q) return CVQPG_ERR_ARG;
    if (q->channels != 1 && q->channels != 3) return CVQPG_ERR_CHANNELS;
    if (q->planes < 1 || q->planes > kMaxLossPlanes) return CVQPG_ERR_UNSUPPORTED;
    if (q->height < 11 || q->width < 11) return CVQPG_ERR_UNSUPPORTED;  // SSIM window must fit
    L->C = q->channels;
    L->P = q->planes;
    L->H = q->height;
    L->W = q->width;
    L->w0 = q->w_l2;
    L->w1 = q->w_mask;
    L->w2 = q->w_cor;
    L->ssim_weight = q->ssim_weight;
    L->noise_ratio = q->noise_ratio;
    L->inject_noise = q->inject_noise;
    L->seed = q->seed;
    L->c1 = (float)((0.01 * 1.0) * (0.01 * 1.0));
    L->c2 = (float)((0.03 * 1.0) * (0.03 * 1.0));
    L->inv_n = (float)(1.0 / ((double)L->C * L->H * L->W));
    L->inv_nmap = (float)(1.0 / ((double)L->C * (L->H - 10) * (L->W - 10)));
    return CVQPG_OK;
}

size_t loss_partials_floats(const LossDev& L) {
    const int tiles = ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    return (size_t)L.P * L.C * tiles * 3;
}

static size_t loss_smem() {
    const size_t a = (size_t)(2 * kLH * kLH + 5 * kLH * kLM + 3 * kLM * kLM) * sizeof(float);
    return a;
}

void launch_loss(const LossDev& L, const float* pred, const float* targets, const uint8_t* depth_plane,
                 const float* noise_scale, const int* iteration, float* grad_pred, float* partials, float* out,
                 cudaStream_t stream) {
    const int tiles = ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    const size_t sm = loss_smem();
    cudaFuncSetAttribute(loss_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    loss_kernel<<<L.P * L.C * tiles, kLossThreads, sm, stream>>>(L, pred, targets, depth_plane, noise_scale,
                                                                 iteration, grad_pred, partials);
    loss_finalize_kernel<<<1, 32, 0, stream>>>(L, partials, out);
}

void launch_target_range(const float* targets, int planes, size_t plane_elems, float* range_out,
                         cudaStream_t stream) {
    target_range_kernel<<<planes, 1024, 0, stream>>>(targets, plane_elems, range_out);
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

extern "C" int cvqpg_loss_workspace_size(const cvqpg_loss_params* q, size_t* bytes) {
    if (!bytes) return CVQPG_ERR_ARG;
    LossDev L;
    const int st = loss_make_dev(q, &L);
    if (st != CVQPG_OK) return st;
    *bytes = loss_partials_floats(L) * sizeof(float) + 256;
    return CVQPG_OK;
}

extern "C" int cvqpg_loss_target_range(const float* targets, int planes, int channels, int height, int width,
                                       float* range_out, void* stream) {
    if (!targets || !range_out || planes < 1 || channels < 1 || height < 1 || width < 1) return CVQPG_ERR_ARG;
    launch_target_range(targets, planes, (size_t)channels * height * width, range_out, (cudaStream_t)stream);
    return launch_status();
}

extern "C" int cvqpg_loss_forward_backward(const cvqpg_loss_params* q, const float* pred, const float* targets,
                                           const uint8_t* depth_plane, const float* target_range,
                                           const int32_t* iteration, float* grad_pred, float* out,
                                           void* workspace, size_t workspace_bytes, void* stream) {
    LossDev L;
    const int st = loss_make_dev(q, &L);
    if (st != CVQPG_OK) return st;
    if (!pred || !targets || !depth_plane || !target_range || !grad_pred || !out || !workspace)
        return CVQPG_ERR_ARG;
    if (workspace_bytes < loss_partials_floats(L) * sizeof(float)) return CVQPG_ERR_WORKSPACE;
    launch_loss(L, pred, targets, depth_plane, target_range, iteration, grad_pred, (float*)workspace, out,
                (cudaStream_t)stream);
    return launch_status();
}

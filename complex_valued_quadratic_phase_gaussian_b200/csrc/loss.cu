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
// Every filter pass is register-blocked: a thread produces a run of 4-8
// consecutive outputs along the filter direction from one sliding window of
// inputs, so shared-memory reads per output drop from 11 to about 2.5.
// Per-CTA partial sums (weighted L2, plain MSE, SSIM map sum) go to a fixed
// slot; a finalize kernel reduces them in a fixed order (deterministic).
#include "loss.cuh"

namespace cvqpg {

constexpr int kLT = 32;              // owned tile edge
constexpr int kLH = kLT + 20;        // staged block edge (52)
constexpr int kLM = kLT + 10;        // map positions touching the tile (42)
constexpr int kLossThreads = 256;
// shared-memory row strides, odd so that threads walking down a column hit distinct banks
constexpr int kSXLd = kLH + 1;       // staged pred / target [52][53]
constexpr int kHMLd = kLM + 1;       // horizontal moments [52][43] and SSIM partial maps [42][43]
constexpr int kTMLd = kLT + 1;       // transposed-horizontal results [42][33]
// outputs per thread in each pass
constexpr int kHSeg = 7;             // horizontal moments: 52 rows x (42 = 6 x 7) columns
constexpr int kVSeg = 7;             // vertical moments + SSIM: 42 columns x (42 = 6 x 7) rows
constexpr int kTHSeg = 8;            // transposed horizontal: 42 rows x (32 = 4 x 8) columns
constexpr int kTVSeg = 4;            // transposed vertical: 32 columns x (32 = 8 x 4) rows, one Philox call
constexpr int kRegionA = 2 * kLH * kSXLd;  // sX, sY; later the three SSIM partial maps
// NM moment maps filtered per call: 5 (pred, target, pred^2, target^2, pred*target), or 3
// (pred, pred^2, pred*target) when the target moments are precomputed; later the
// transposed-horizontal maps
constexpr int region_b(int nm) { return nm * kLH * kHMLd; }
static_assert(3 * kLM * kHMLd <= kRegionA, "SSIM partial maps must fit in the staging region");
static_assert(3 * kLM * kTMLd <= region_b(3), "transposed maps must fit in the moment region");
static_assert((kLM / kVSeg) * kLM <= kLossThreads, "one vertical item per thread");
static_assert((kLT / kTHSeg) * kLM <= kLossThreads, "one transposed-horizontal item per thread");
static_assert((kLT / kTVSeg) * kLT == kLossThreads, "one transposed-vertical item per thread");

// Gaussian window, 11 taps, sigma 1.5, normalised (computed in double, rounded once).
__device__ __forceinline__ float ssim_w(int k) {
    constexpr float w[11] = {1.028380082e-03f, 7.598758612e-03f, 3.600077721e-02f, 1.093606895e-01f,
                             2.130055428e-01f, 2.660117810e-01f, 2.130055428e-01f, 1.093606895e-01f,
                             3.600077721e-02f, 7.598758612e-03f, 1.028380082e-03f};
    return w[k];
}

template <int NM>
__global__ void __launch_bounds__(kLossThreads, NM == 3 ? 4 : 3) loss_kernel(LossDev L, const float* __restrict__ pred,
                                                                const float* __restrict__ target,
                                                                const uint8_t* __restrict__ depth_plane,
                                                                const float* __restrict__ noise_scale,
                                                                const int* __restrict__ iteration,
                                                                float* __restrict__ grad_pred,
                                                                float* __restrict__ partials) {
    extern __shared__ float lsm[];
    float* sX = lsm;                       // [52][53]
    float* sY = sX + kLH * kSXLd;          // [52][53]
    float* dM = lsm;                       // 3 x [42][43], written once sX/sY are dead
    float* hM = lsm + kRegionA;            // 5 x [52][43]
    float* tM = hM;                        // 3 x [42][33], written once hM is dead
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
    const int tid = threadIdx.x;

    // 1. stage the 52x52 block (zeros outside the image; never used by valid map entries);
    //    all loads of a thread are issued before its stores
    {
        constexpr int kStageIt = (kLH * kLH + kLossThreads - 1) / kLossThreads;
        float vx[kStageIt], vy[kStageIt];
#pragma unroll
        for (int u = 0; u < kStageIt; u++) {
            const int i = tid + u * kLossThreads;
            const int r = i / kLH, q = i - r * kLH;
            const int y = y0 - 10 + r, x = x0 - 10 + q;
            const bool in = i < kLH * kLH && (unsigned)y < (unsigned)H && (unsigned)x < (unsigned)W;
            const size_t e = in ? (size_t)y * W + x : 0;
            vx[u] = in ? __ldg(&X[e]) : 0.f;
            vy[u] = in ? __ldg(&Y[e]) : 0.f;
        }
#pragma unroll
        for (int u = 0; u < kStageIt; u++) {
            const int i = tid + u * kLossThreads;
            if (i < kLH * kLH) {
                const int r = i / kLH, q = i - r * kLH;
                sX[r * kSXLd + q] = vx[u];
                sY[r * kSXLd + q] = vy[u];
            }
        }
    }
    __syncthreads();

    // 2. horizontal filter -> moments on [52][42]; item = (row, 7 columns).
    //    NM = 5: x, y, xx, yy, xy.  NM = 3: x, xx, xy (target moments precomputed).
    for (int item = tid; item < kLH * (kLM / kHSeg); item += kLossThreads) {
        const int r = item % kLH, c0 = (item / kLH) * kHSeg;
        float acc[NM][kHSeg];
#pragma unroll
        for (int o = 0; o < kHSeg; o++)
#pragma unroll
            for (int m = 0; m < NM; m++) acc[m][o] = 0.f;
        const float* px = sX + r * kSXLd + c0;
        const float* py = sY + r * kSXLd + c0;
#pragma unroll
        for (int k = 0; k < kHSeg + 10; k++) {
            const float x = px[k], y = py[k];
            const float xx = x * x, xy = x * y;
#pragma unroll
            for (int o = 0; o < kHSeg; o++) {
                const int t = k - o;
                if (t < 0 || t > 10) continue;
                const float w = ssim_w(t);
                if (NM == 5) {
                    acc[0][o] = fmaf(w, x, acc[0][o]);
                    acc[1][o] = fmaf(w, y, acc[1][o]);
                    acc[2][o] = fmaf(w, xx, acc[2][o]);
                    acc[3 % NM][o] = fmaf(w, y * y, acc[3 % NM][o]);
                    acc[4 % NM][o] = fmaf(w, xy, acc[4 % NM][o]);
                } else {
                    acc[0][o] = fmaf(w, x, acc[0][o]);
                    acc[1][o] = fmaf(w, xx, acc[1][o]);
                    acc[2][o] = fmaf(w, xy, acc[2][o]);
                }
            }
        }
#pragma unroll
        for (int m = 0; m < NM; m++)
#pragma unroll
            for (int o = 0; o < kHSeg; o++) hM[m * kLH * kHMLd + r * kHMLd + c0 + o] = acc[m][o];
    }
    __syncthreads();

    // 3. vertical filter -> SSIM map and its partials on [42][42]; item = (column, 7 rows)
    const float C1 = L.c1, C2 = L.c2;
    float ssim_sum = 0.f;
    if (tid < kLM * (kLM / kVSeg)) {
        const int jj = tid % kLM, i0 = (tid / kLM) * kVSeg;
        const int mj = x0 - 10 + jj;
        const bool col_ok = (unsigned)mj < (unsigned)(W - 10);
        float2 tmv[NM == 3 ? kVSeg : 1];
        if (NM == 3) {  // the target moments of the 7 map positions, loads issued together
#pragma unroll
            for (int o = 0; o < (NM == 3 ? kVSeg : 1); o++) {
                const int mi = y0 - 10 + i0 + o;
                const bool ok = col_ok && (unsigned)mi < (unsigned)(H - 10);
                tmv[o] = ok ? __ldg(&L.tmom[((size_t)pc * (H - 10) + mi) * (W - 10) + mj]) : make_float2(0.f, 0.f);
            }
        }
        float acc[NM][kVSeg];
#pragma unroll
        for (int o = 0; o < kVSeg; o++)
#pragma unroll
            for (int m = 0; m < NM; m++) acc[m][o] = 0.f;
#pragma unroll
        for (int k = 0; k < kVSeg + 10; k++) {
            float v[NM];
#pragma unroll
            for (int m = 0; m < NM; m++) v[m] = hM[m * kLH * kHMLd + (i0 + k) * kHMLd + jj];
#pragma unroll
            for (int o = 0; o < kVSeg; o++) {
                const int t = k - o;
                if (t < 0 || t > 10) continue;
                const float w = ssim_w(t);
#pragma unroll
                for (int m = 0; m < NM; m++) acc[m][o] = fmaf(w, v[m], acc[m][o]);
            }
        }
#pragma unroll
        for (int o = 0; o < kVSeg; o++) {
            const int ii = i0 + o, mi = y0 - 10 + ii;
            float dm = 0.f, dxx = 0.f, dxy = 0.f;
            if (col_ok && (unsigned)mi < (unsigned)(H - 10)) {
                float mu1, mu2, exx, eyy, exy;
                if (NM == 5) {
                    mu1 = acc[0][o], mu2 = acc[1 % NM][o], exx = acc[2 % NM][o], eyy = acc[3 % NM][o];
                    exy = acc[4 % NM][o];
                } else {
                    const float2 tm = tmv[NM == 3 ? o : 0];
                    mu1 = acc[0][o], exx = acc[1][o], exy = acc[2][o], mu2 = tm.x, eyy = tm.y;
                }
                const float s11 = exx - mu1 * mu1, s22 = eyy - mu2 * mu2, s12 = exy - mu1 * mu2;
                const float A1 = 2.f * mu1 * mu2 + C1, A2 = 2.f * s12 + C2;
                const float B1 = mu1 * mu1 + mu2 * mu2 + C1, B2 = s11 + s22 + C2;
                // B1 >= C1 and B2 >= C2 (positive constants): the SFU reciprocal (within 1 ulp) needs no
                // IEEE special cases
                const float iB1 = rcp_ftz(B1), iB2 = rcp_ftz(B2);
                const float P = iB1 * iB2;
                const float smap = A1 * A2 * P;
                if (ii >= 10 && jj >= 10) ssim_sum += smap;  // owned map position
                // dS/dmu1 with E[x^2], E[xy] held: dA1 = 2 mu2, dA2 = -2 mu2, dB1 = 2 mu1, dB2 = -2 mu1
                dm = 2.f * fmaf(mu2 * P, A2 - A1, mu1 * smap * (iB2 - iB1));
                dxx = -smap * iB2;
                dxy = 2.f * A1 * P;
            }
            dM[0 * kLM * kHMLd + ii * kHMLd + jj] = dm;
            dM[1 * kLM * kHMLd + ii * kHMLd + jj] = dxx;
            dM[2 * kLM * kHMLd + ii * kHMLd + jj] = dxy;
        }
    }
    __syncthreads();

    // 4. transposed horizontal filter -> [42][32]; item = (row, 8 columns)
    if (tid < kLM * (kLT / kTHSeg)) {
        const int ii = tid % kLM, c0 = (tid / kLM) * kTHSeg;
        float acc[3][kTHSeg];
#pragma unroll
        for (int o = 0; o < kTHSeg; o++)
#pragma unroll
            for (int m = 0; m < 3; m++) acc[m][o] = 0.f;
#pragma unroll
        for (int k = 0; k < kTHSeg + 10; k++) {
            float v[3];
#pragma unroll
            for (int m = 0; m < 3; m++) v[m] = dM[m * kLM * kHMLd + ii * kHMLd + c0 + k];
#pragma unroll
            for (int o = 0; o < kTHSeg; o++) {
                const int t = o + 10 - k;  // map column c0+k feeds tile column c0+o with weight w(o+10-k)
                if (t < 0 || t > 10) continue;
                const float w = ssim_w(t);
#pragma unroll
                for (int m = 0; m < 3; m++) acc[m][o] = fmaf(w, v[m], acc[m][o]);
            }
        }
#pragma unroll
        for (int m = 0; m < 3; m++)
#pragma unroll
            for (int o = 0; o < kTHSeg; o++) tM[m * kLM * kTMLd + ii * kTMLd + c0 + o] = acc[m][o];
    }
    __syncthreads();

    // 5. transposed vertical filter + L2 terms on the owned tile; item = (column, 4 rows)
    const float inv_n = L.inv_n, ssim_scale = -L.ssim_weight * L.inv_nmap;
    const float nscale = noise_scale[p];
    const uint64_t it = iteration ? (uint64_t)(uint32_t)iteration[0] : 0ull;
    float l2_sum = 0.f, mse_sum = 0.f;
    {
        const int xx = tid % kLT, r0 = (tid / kLT) * kTVSeg;
        float acc[3][kTVSeg];
#pragma unroll
        for (int o = 0; o < kTVSeg; o++)
#pragma unroll
            for (int m = 0; m < 3; m++) acc[m][o] = 0.f;
#pragma unroll
        for (int k = 0; k < kTVSeg + 10; k++) {
            float v[3];
#pragma unroll
            for (int m = 0; m < 3; m++) v[m] = tM[m * kLM * kTMLd + (r0 + k) * kTMLd + xx];
#pragma unroll
            for (int o = 0; o < kTVSeg; o++) {
                const int t = o + 10 - k;
                if (t < 0 || t > 10) continue;
                const float w = ssim_w(t);
#pragma unroll
                for (int m = 0; m < 3; m++) acc[m][o] = fmaf(w, v[m], acc[m][o]);
            }
        }
        const int x = x0 + xx, yb = y0 + r0;
        if (x < W && yb < H) {
            float z[kTVSeg] = {0.f, 0.f, 0.f, 0.f};
            if (L.inject_noise) {
                // counter of the four rows yb..yb+3 of column x (yb is a multiple of 4)
                const uint64_t q = ((uint64_t)pc * (uint64_t)((H + 3) >> 2) + (uint64_t)(yb >> 2)) * (uint64_t)W + x;
                const float4 n4 = normal4_at(L.seed, it, q);
                z[0] = n4.x;
                z[1] = n4.y;
                z[2] = n4.z;
                z[3] = n4.w;
            }
            float xo[kTVSeg], to[kTVSeg];
            uint8_t qo[kTVSeg];
#pragma unroll
            for (int o = 0; o < kTVSeg; o++) {  // loads first, so they are in flight together
                const bool in = yb + o < H;
                const size_t e = (size_t)(in ? yb + o : yb) * W + x;
                xo[o] = __ldg(&X[e]);
                to[o] = __ldg(&Y[e]);
                qo[o] = __ldg(&depth_plane[e]);
            }
#pragma unroll
            for (int o = 0; o < kTVSeg; o++) {
                const int y = yb + o;
                if (y >= H) break;
                const size_t e = (size_t)y * W + x;
                const float xv = xo[o], tv = to[o];
                const float m = (qo[o] == p) ? 1.f : 0.f;
                const float nv = L.inject_noise ? tv + (z[o] * L.noise_ratio) * nscale : tv;
                const float d0 = xv - tv, d1 = (xv * m - nv * m), d2 = (xv * nv - nv * nv);
                l2_sum += L.w0 * d0 * d0 + L.w1 * d1 * d1 + L.w2 * d2 * d2;
                mse_sum += d0 * d0;
                const float g_l2 = 2.f * inv_n * (L.w0 * d0 + L.w1 * d1 * m + L.w2 * d2 * nv);
                const float g_ssim = ssim_scale * (acc[0][o] + 2.f * xv * acc[1][o] + tv * acc[2][o]);
                grad_pred[plane_off + e] = g_l2 + g_ssim;
            }
        }
    }
    // 6. block reduction of the three partial sums
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        l2_sum += __shfl_xor_sync(0xffffffffu, l2_sum, o);
        mse_sum += __shfl_xor_sync(0xffffffffu, mse_sum, o);
        ssim_sum += __shfl_xor_sync(0xffffffffu, ssim_sum, o);
    }
    const int w = tid >> 5, lane = tid & 31;
    if (lane == 0) {
        red[0][w] = l2_sum;
        red[1][w] = mse_sum;
        red[2][w] = ssim_sum;
    }
    __syncthreads();
    if (tid == 0) {
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

constexpr int kFinalThreads = 1024;  // threads of the one-block finalize
constexpr int kRangeThreads = 512;
constexpr int kRangeBlocks = CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE / 8;  // (max, min) float pairs

// out[0] = total loss, out[1 + p] = MSE of plane p, out[1 + P + p] = SSIM of plane p,
// out[1 + 2P + p] = loss of plane p. One block. Every thread accumulates a fixed
// strided subset of the per-tile partials of all planes in double; a fixed
// xor-shuffle tree adds each warp's lanes and warp 0 adds the 32 warp sums the
// same way, so the result does not depend on scheduling (two barriers in all).
__global__ void __launch_bounds__(kFinalThreads) loss_finalize_kernel(LossDev L, const float* __restrict__ partials,
                                                                      float* __restrict__ out) {
    constexpr int kV = 3 * kMaxLossPlanes;  // (weighted L2, MSE, SSIM map sum) per plane
    __shared__ double sh[kV][kFinalThreads / 32];
    const int per_plane = L.C * ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double v[kV];
#pragma unroll
    for (int i = 0; i < kV; i++) v[i] = 0.0;
#pragma unroll
    for (int q = 0; q < kMaxLossPlanes; q++) {
        if (q < L.P) {
            const float* base = partials + (size_t)q * per_plane * 3;
            for (int t = threadIdx.x; t < per_plane; t += kFinalThreads) {
                v[3 * q + 0] += base[(size_t)t * 3 + 0];
                v[3 * q + 1] += base[(size_t)t * 3 + 1];
                v[3 * q + 2] += base[(size_t)t * 3 + 2];
            }
        }
    }
#pragma unroll
    for (int i = 0; i < kV; i++) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], o);
        if (lane == 0) sh[i][w] = v[i];
    }
    __syncthreads();
    if (w == 0) {
        double total = 0.0;
        for (int q = 0; q < L.P; q++) {
            double r[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                r[k] = sh[3 * q + k][lane];
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) r[k] += __shfl_xor_sync(0xffffffffu, r[k], o);
            }
            const double mse = r[1] * L.inv_n;
            const double ssim = r[2] * L.inv_nmap;
            const double lp = r[0] * L.inv_n + L.ssim_weight * (1.0 - ssim);
            total += lp;
            if (lane == 0) {
                out[1 + q] = (float)mse;
                out[1 + L.P + q] = (float)ssim;
                out[1 + 2 * L.P + q] = (float)lp;
            }
        }
        if (lane == 0) out[0] = (float)total;
    }
}

// Per-plane noise scale max(T_p) - min(T_p) (the ratio is applied later).
// Pass 1, grid (kRangeBlocks, planes): each block reduces a strided slice of
// its plane to (max, min). Pass 2, one warp per plane: combine the slices.
__global__ void __launch_bounds__(kRangeThreads) target_range_slices_kernel(const float* __restrict__ targets,
                                                                            size_t plane_elems,
                                                                            float2* __restrict__ slices) {
    const int p = blockIdx.y;
    const float* t = targets + (size_t)p * plane_elems;
    float mx = -INFINITY, mn = INFINITY;
    for (size_t i = (size_t)blockIdx.x * kRangeThreads + threadIdx.x; i < plane_elems;
         i += (size_t)kRangeBlocks * kRangeThreads) {
        const float v = __ldg(&t[i]);
        mx = fmaxf(mx, v);
        mn = fminf(mn, v);
    }
    __shared__ float smx[kRangeThreads / 32], smn[kRangeThreads / 32];
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
        for (int k = 1; k < kRangeThreads / 32; k++) {
            mx = fmaxf(mx, smx[k]);
            mn = fminf(mn, smn[k]);
        }
        slices[(size_t)p * kRangeBlocks + blockIdx.x] = make_float2(mx, mn);
    }
}

__global__ void target_range_combine_kernel(const float2* __restrict__ slices, float* __restrict__ range_out) {
    const int p = blockIdx.x;
    float mx = -INFINITY, mn = INFINITY;
    for (int k = threadIdx.x; k < kRangeBlocks; k += 32) {
        const float2 v = slices[(size_t)p * kRangeBlocks + k];
        mx = fmaxf(mx, v.x);
        mn = fminf(mn, v.y);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    }
    if (threadIdx.x == 0) range_out[p] = mx - mn;
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
    L->tmom = reinterpret_cast<const float2*>(q->target_moments);
    return CVQPG_OK;
}

size_t loss_partials_floats(const LossDev& L) {
    const int tiles = ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    return (size_t)L.P * L.C * tiles * 3;
}

static size_t loss_smem(int nm) { return (size_t)(kRegionA + region_b(nm)) * sizeof(float); }

// Target moments: one CTA per 32x32 block of map positions of one (plane, channel)
// image; the same two separable passes and fma order as the loss kernel's.
constexpr int kTmIn = kLT + 10;  // 42 staged rows / columns
__global__ void __launch_bounds__(kLossThreads) target_moments_kernel(int H, int W, const float* __restrict__ targets,
                                                                      float2* __restrict__ mom) {
    __shared__ float sT[kTmIn][kTmIn + 1];
    __shared__ float hm[2][kTmIn][kLT + 1];
    const int MH = H - 10, MW = W - 10;
    const int tx = (MW + kLT - 1) / kLT, ty = (MH + kLT - 1) / kLT;
    const int pc = blockIdx.x / (tx * ty), tile = blockIdx.x - pc * tx * ty;
    const int m0y = (tile / tx) * kLT, m0x = (tile % tx) * kLT;
    const float* T = targets + (size_t)pc * H * W;
    for (int i = threadIdx.x; i < kTmIn * kTmIn; i += kLossThreads) {
        const int r = i / kTmIn, c = i - r * kTmIn;
        const int y = m0y + r, x = m0x + c;
        sT[r][c] = (y < H && x < W) ? __ldg(&T[(size_t)y * W + x]) : 0.f;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kTmIn * kLT; i += kLossThreads) {
        const int r = i / kLT, c = i - r * kLT;
        float a = 0.f, b = 0.f;
#pragma unroll
        for (int t = 0; t <= 10; t++) {
            const float y = sT[r][c + t];
            a = fmaf(ssim_w(t), y, a);
            b = fmaf(ssim_w(t), y * y, b);
        }
        hm[0][r][c] = a;
        hm[1][r][c] = b;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kLT * kLT; i += kLossThreads) {
        const int r = i / kLT, c = i - r * kLT;
        float a = 0.f, b = 0.f;
#pragma unroll
        for (int t = 0; t <= 10; t++) {
            a = fmaf(ssim_w(t), hm[0][r + t][c], a);
            b = fmaf(ssim_w(t), hm[1][r + t][c], b);
        }
        const int my = m0y + r, mx = m0x + c;
        if (my < MH && mx < MW) mom[((size_t)pc * MH + my) * MW + mx] = make_float2(a, b);
    }
}

size_t target_moments_bytes(const LossDev& L) {
    return (size_t)L.P * L.C * (L.H - 10) * (L.W - 10) * sizeof(float2);
}

void launch_target_moments(const LossDev& L, const float* targets, float2* mom, cudaStream_t stream) {
    const int tiles = ((L.W - 10 + kLT - 1) / kLT) * ((L.H - 10 + kLT - 1) / kLT);
    target_moments_kernel<<<L.P * L.C * tiles, kLossThreads, 0, stream>>>(L.H, L.W, targets, mom);
}

void launch_loss(const LossDev& L, const float* pred, const float* targets, const uint8_t* depth_plane,
                 const float* noise_scale, const int* iteration, float* grad_pred, float* partials, float* out,
                 cudaStream_t stream) {
    const int tiles = ((L.W + kLT - 1) / kLT) * ((L.H + kLT - 1) / kLT);
    if (L.tmom) {
        const size_t sm = loss_smem(3);
        cudaFuncSetAttribute(loss_kernel<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        loss_kernel<3><<<L.P * L.C * tiles, kLossThreads, sm, stream>>>(L, pred, targets, depth_plane, noise_scale,
                                                                        iteration, grad_pred, partials);
    } else {
        const size_t sm = loss_smem(5);
        cudaFuncSetAttribute(loss_kernel<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        loss_kernel<5><<<L.P * L.C * tiles, kLossThreads, sm, stream>>>(L, pred, targets, depth_plane, noise_scale,
                                                                        iteration, grad_pred, partials);
    }
    loss_finalize_kernel<<<1, kFinalThreads, 0, stream>>>(L, partials, out);
}

void launch_target_range(const float* targets, int planes, size_t plane_elems, float* range_out, void* scratch,
                         cudaStream_t stream) {
    float2* slices = (float2*)scratch;
    target_range_slices_kernel<<<dim3(kRangeBlocks, planes), kRangeThreads, 0, stream>>>(targets, plane_elems,
                                                                                         slices);
    target_range_combine_kernel<<<planes, 32, 0, stream>>>(slices, range_out);
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
    const size_t partials = loss_partials_floats(L) * sizeof(float);
    const size_t range = (size_t)L.P * CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE;
    *bytes = (partials > range ? partials : range) + 256;
    return CVQPG_OK;
}

extern "C" int cvqpg_loss_target_range(const float* targets, int planes, int channels, int height, int width,
                                       float* range_out, void* workspace, size_t workspace_bytes, void* stream) {
    if (!targets || !range_out || !workspace || planes < 1 || channels < 1 || height < 1 || width < 1)
        return CVQPG_ERR_ARG;
    if (workspace_bytes < (size_t)planes * CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE) return CVQPG_ERR_WORKSPACE;
    launch_target_range(targets, planes, (size_t)channels * height * width, range_out, workspace,
                        (cudaStream_t)stream);
    return launch_status();
}

extern "C" int cvqpg_loss_target_moments_size(const cvqpg_loss_params* q, size_t* bytes) {
    if (!bytes) return CVQPG_ERR_ARG;
    LossDev L;
    const int st = loss_make_dev(q, &L);
    if (st != CVQPG_OK) return st;
    *bytes = target_moments_bytes(L);
    return CVQPG_OK;
}

extern "C" int cvqpg_loss_target_moments(const cvqpg_loss_params* q, const float* targets, float* moments,
                                         size_t moments_bytes, void* stream) {
    LossDev L;
    const int st = loss_make_dev(q, &L);
    if (st != CVQPG_OK) return st;
    if (!targets || !moments) return CVQPG_ERR_ARG;
    if (reinterpret_cast<uintptr_t>(moments) % 8 != 0) return CVQPG_ERR_ARG;
    if (moments_bytes < target_moments_bytes(L)) return CVQPG_ERR_WORKSPACE;
    launch_target_moments(L, targets, reinterpret_cast<float2*>(moments), (cudaStream_t)stream);
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

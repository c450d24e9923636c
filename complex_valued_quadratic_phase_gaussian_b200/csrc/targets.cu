// Multi-plane defocus targets on the device: depth slicing and defocus blur of
// the reference loss (utils/propagator.py:361-415, settings of
// utils/data_utils.py:66-82), needed once per scene by every fit.
//
// The reference computes, for plane i and channel c,
//   T_i,c = sum_j [sum(I_c * M_j) > 0] * (K_{s_ij} * I_c) * M_j,   M_j = [q == j],
// with q = round(depth^ratio * (P-1)) (torch.round: half to even), s_ij =
// int(|i-j| * blur_ratio) (s = 0 is an impulse) and K_s the normalised L x L
// Gaussian sampled at linspace(-L/2, L/2, L) (L = blur_size + 1 for even
// sizes), applied as a zero-padded 'same' correlation. Because the masks
// partition the image, T_i,c(p) = flag[q(p)][c] * (K_{s(i, q(p))} * I_c)(p):
// one blurred copy per distinct sigma and a gather. K_s = g (x) g / (sum g)^2
// is separable, so each copy is two 1D passes.
//
// Kernels: plane index + per-block masked sums; fixed-order finalize of the
// sums into flags; horizontal and vertical passes per sigma; gather.
#include <math.h>

#include <vector>

#include "common.cuh"

namespace cvqpg {

constexpr int kTgtThreads = 256;
constexpr int kTgtBlocks = 296;
constexpr int kMaxTgtPlanes = 8;
constexpr int kMaxTaps = 63;

struct TapSet {
    int L;
    float w[kMaxTaps];
};

__global__ void targets_quantise_kernel(const float* __restrict__ image, const float* __restrict__ depth, int C,
                                        size_t HW, int P, float ratio, uint8_t* __restrict__ plane,
                                        double* __restrict__ partial) {
    double local[kMaxTgtPlanes * 3];
    for (int i = 0; i < P * C; i++) local[i] = 0.0;
    for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < HW; p += (size_t)gridDim.x * blockDim.x) {
        const float d = depth[p];
        const float biased = (ratio == 1.0f ? d : powf(d, ratio)) * (float)(P - 1);
        int q = (int)rintf(biased);
        q = q < 0 ? 0 : (q > P - 1 ? P - 1 : q);
        plane[p] = (uint8_t)q;
        for (int c = 0; c < C; c++) local[q * C + c] += (double)image[(size_t)c * HW + p];
    }
    // fixed-shape block tree per (plane, channel): deterministic partial sums
    __shared__ double red[kTgtThreads];
    for (int i = 0; i < P * C; i++) {
        red[threadIdx.x] = local[i];
        __syncthreads();
        for (int s = kTgtThreads / 2; s > 0; s >>= 1) {
            if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
            __syncthreads();
        }
        if (threadIdx.x == 0) partial[(size_t)blockIdx.x * P * C + i] = red[0];
        __syncthreads();
    }
}

__global__ void targets_flags_kernel(const double* __restrict__ partial, int nblocks, int PC, int* __restrict__ flag) {
    const int i = threadIdx.x;
    if (i < PC) {
        double s = 0.0;
        for (int b = 0; b < nblocks; b++) s += partial[(size_t)b * PC + i];
        flag[i] = s > 0.0 ? 1 : 0;
    }
}

// one 1D pass of the separable blur (zero padding): horizontal when `vertical` is 0
__global__ void targets_blur_kernel(const float* __restrict__ src, float* __restrict__ dst, int C, int H, int W,
                                    TapSet taps, int vertical) {
    const size_t n = (size_t)C * H * W;
    const int h = taps.L / 2;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % W);
        const int y = (int)((i / W) % H);
        float s = 0.0f;
        if (vertical) {
            for (int t = 0; t < taps.L; t++) {
                const int yy = y + t - h;
                if ((unsigned)yy < (unsigned)H) s = fmaf(taps.w[t], src[i + (ptrdiff_t)(yy - y) * W], s);
            }
        } else {
            for (int t = 0; t < taps.L; t++) {
                const int xx = x + t - h;
                if ((unsigned)xx < (unsigned)W) s = fmaf(taps.w[t], src[i + (xx - x)], s);
            }
        }
        dst[i] = s;
    }
}

// T[i][c][p] = flag[q][c] ? blurred_{|i-q|}[c][p] : 0 (blurred_0 = the image)
__global__ void targets_gather_kernel(const float* __restrict__ image, const float* __restrict__ blurred,
                                      const uint8_t* __restrict__ plane, const int* __restrict__ flag, int C,
                                      size_t HW, int P, float* __restrict__ targets) {
    const size_t n = (size_t)P * C * HW;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const size_t p = i % HW;
        const int c = (int)((i / HW) % C);
        const int pi = (int)(i / ((size_t)C * HW));
        const int q = plane[p];
        float v = 0.0f;
        if (flag[q * C + c]) {
            const int d = pi > q ? pi - q : q - pi;
            v = d == 0 ? image[(size_t)c * HW + p] : blurred[((size_t)(d - 1) * C + c) * HW + p];
        }
        targets[i] = v;
    }
}

static bool make_taps(int blur_size, int sigma, TapSet* t) {
    const int L = (blur_size % 2 == 0) ? blur_size + 1 : blur_size;
    if (L < 1 || L > kMaxTaps) return false;
    t->L = L;
    const double s = sigma != 0 ? (double)sigma : 1e-5;
    std::vector<double> g(L);
    double sum = 0.0;
    for (int i = 0; i < L; i++) {
        const double x = -L / 2.0 + (double)L * i / (double)(L - 1);  // linspace(-L/2, L/2, L)
        g[i] = exp(-x * x / (2.0 * s * s));
        sum += g[i];
    }
    for (int i = 0; i < L; i++) t->w[i] = (float)(g[i] / sum);
    return true;
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

static size_t targets_ws(int C, int H, int W, int P) {
    const size_t img = (size_t)C * H * W;
    Carver cv(nullptr, 0);
    cv.take<float>(img * (P > 1 ? P - 1 : 1));  // blurred copies
    cv.take<float>(img);                        // horizontal-pass scratch
    cv.take<double>((size_t)kTgtBlocks * P * C);
    cv.take<int>((size_t)P * C);
    return cv.off + 256;
}

extern "C" int cvqpg_targets_workspace_size(int channels, int height, int width, int planes, size_t* bytes) {
    if (!bytes || channels < 1 || channels > 3 || height < 1 || width < 1 || planes < 1) return CVQPG_ERR_ARG;
    if (planes > kMaxTgtPlanes) return CVQPG_ERR_UNSUPPORTED;
    *bytes = targets_ws(channels, height, width, planes);
    return CVQPG_OK;
}

extern "C" int cvqpg_targets_synthesize(const float* image, const float* depth, int channels, int height, int width,
                                        int planes, int blur_size, float blur_ratio, float split_ratio,
                                        float* targets, uint8_t* plane_index, void* workspace,
                                        size_t workspace_bytes, void* stream_) {
    if (!image || !depth || !targets || !plane_index || !workspace) return CVQPG_ERR_ARG;
    if (channels < 1 || channels > 3 || height < 1 || width < 1 || planes < 1) return CVQPG_ERR_ARG;
    if (planes > kMaxTgtPlanes) return CVQPG_ERR_UNSUPPORTED;
    if (workspace_bytes < targets_ws(channels, height, width, planes)) return CVQPG_ERR_WORKSPACE;
    const int C = channels, H = height, W = width, P = planes;
    const size_t HW = (size_t)H * W, img = (size_t)C * HW;
    Carver cv(workspace, workspace_bytes);
    float* blurred = cv.take<float>(img * (P > 1 ? P - 1 : 1));
    float* tmp = cv.take<float>(img);
    double* partial = cv.take<double>((size_t)kTgtBlocks * P * C);
    int* flag = cv.take<int>((size_t)P * C);
    cudaStream_t s = (cudaStream_t)stream_;
    const float ratio = (P == 2) ? split_ratio : 1.0f;
    targets_quantise_kernel<<<kTgtBlocks, kTgtThreads, 0, s>>>(image, depth, C, HW, P, ratio, plane_index, partial);
    targets_flags_kernel<<<1, 32, 0, s>>>(partial, kTgtBlocks, P * C, flag);
    for (int d = 1; d < P; d++) {
        TapSet taps;
        if (!make_taps(blur_size, (int)(d * blur_ratio), &taps)) return CVQPG_ERR_UNSUPPORTED;
        float* out = blurred + (size_t)(d - 1) * img;
        targets_blur_kernel<<<kTgtBlocks * 4, kTgtThreads, 0, s>>>(image, tmp, C, H, W, taps, 0);
        targets_blur_kernel<<<kTgtBlocks * 4, kTgtThreads, 0, s>>>(tmp, out, C, H, W, taps, 1);
    }
    targets_gather_kernel<<<kTgtBlocks * 4, kTgtThreads, 0, s>>>(image, blurred, plane_index, flag, C, HW, P,
                                                                 targets);
    return launch_status();
}

// Band-limited angular-spectrum propagation of the CVQPG hologram to every
// (plane, wavelength) in three pruned FFT passes, and its adjoint.
//
// Reference chain replaced (paths inside the reference project):
//   model_2d_gaussian_rgb.py:186-241   soft_window_pad (replicate guard band, Tukey taper)
//   train_2d_gaussian_rgb.py:89-95     phase = angle(U) mod 2pi, amplitude = clamp(|U|, 0, 1)
//   utils/propagator.py:248-290        per (plane, channel): zero_pad x2, fft2, fftshift,
//                                      aperture, transfer function, ifftshift, ifft2, crop
//   utils/propagator.py:41-64          custom()
//   utils/propagator.py:202-222        transfer-function cache (odak BLASM kernel)
//   train_2d_gaussian_rgb.py:193       crop_center to the image
//
// Grid facts used for pruning (all sizes even): the padded field occupies
// rows [NH/2 - pH/2, NH/2 + pH/2) of the 2x grid, and the kept output rows are
// [NH/2 - out_h/2, NH/2 + out_h/2); for even n, fftshift and ifftshift are the
// same half-length rotation, so the shifted multiply equals an unshifted one
// by M[(k + N/2) mod N].
#include <math.h>

#include <algorithm>
#include <initializer_list>
#include <cstring>
#include <vector>

#include "blasm_cols.cuh"

namespace cvqpg {

// ---------------------------------------------------------------------------
// host: FFT plans
// ---------------------------------------------------------------------------
bool make_fft_plan(int n, FftPlan* plan, int order) {
    plan->n = n;
    plan->npass = 0;
    plan->code = 0;
    plan->tw = nullptr;
    int m = n;
    auto push = [&](int r) {
        if (plan->npass >= kMaxPasses) return false;
        plan->code |= (unsigned long long)r << (5 * plan->npass);
        plan->npass++;
        return true;
    };
    const int odd[] = {3, 5, 7, 11, 13, 17};
    const int odd_desc[] = {17, 13, 11, 7, 5, 3};
    auto push_odd = [&](const int* list) {
        for (int k = 0; k < 6; k++)
            while (m % list[k] == 0) {
                if (!push(list[k])) return false;
                m /= list[k];
            }
        return true;
    };
    auto push_pow2 = [&](bool use16) {
        if (use16)
            while (m % 16 == 0)
                if (!push(16)) return false; else m /= 16;
        while (m % 8 == 0)
            if (!push(8)) return false; else m /= 8;
        if (m % 4 == 0) { if (!push(4)) return false; m /= 4; }
        if (m % 2 == 0) { if (!push(2)) return false; m /= 2; }
        return true;
    };
    bool ok = true;
    switch (order) {
        case 1: ok = push_odd(odd_desc) && push_pow2(true); break;
        case 2: ok = push_pow2(false) && push_odd(odd); break;
        case 3: ok = push_odd(odd_desc) && push_pow2(false); break;
        default: ok = push_pow2(true) && push_odd(odd); break;
    }
    return ok && m == 1;
}

// ---------------------------------------------------------------------------
// forward kernels. Intermediates are row-major: A [C][pH][NW] after the row
// pass, B [P*C][out_h][NW] after the column pass. The column pass reads and
// writes one column per CTA at a stride of NW; neighbouring columns are
// handled by neighbouring CTAs at the same time, so the 32-byte sectors are
// completed in L2.
// ---------------------------------------------------------------------------
// Row FFT policies: RowRuntime runs the plan read at run time; RowCT<NT, MI, MO, N, R...>
// the plan fixed at compile time (CtFft), for the row length of the 1080p fit.
// run_out(src, out, a0, a1, ...): the FFT of one row, then out(a, X_a) for every
// kept output a in [a0, a1).
struct RowRuntime {
    static constexpr int kThreads = kRowThreads;
    template <bool INV, typename Src>
    __device__ static __forceinline__ float2* run(Src src, float2* b0, float2* b1, int ld, const BlasmDev& d) {
        return fft_run(src, b0, b1, ld, 0, d.row, INV);
    }
    template <bool INV, typename Src, typename Out>
    __device__ static __forceinline__ void run_out(Src src, Out out, int a0, int a1, float2* b0, float2* b1, int ld,
                                                   const BlasmDev& d) {
        const float2* res = fft_run(src, b0, b1, ld, 0, d.row, INV);
        for (int a = a0 + threadIdx.x; a < a1; a += blockDim.x) out(a, res[fft_pad(a)]);
    }
};

// MI / MO: the row's input is zero outside its middle half / only the middle
// half of the output is kept (2x zero padding; the crops are at most the padded
// width), so the first / last radix-16 pass is pruned (ct_pass MID_IN / MID_OUT).
template <int NT, bool MI, bool MO, int N, int... R>
struct RowCT {
    static constexpr int kThreads = NT;
    static constexpr int kPasses = (int)sizeof...(R);
    template <bool INV, typename Src>
    __device__ static __forceinline__ float2* run(Src src, float2* b0, float2* b1, int, const BlasmDev& d) {
        float2* res = (kPasses % 2 == 1) ? b0 : b1;  // the buffer the last pass does not read
        CtFft<5, NT, N, INV, 1, MI, MO, true, R...>::run(ElemLoadF<Src>{src}, SmemStoreF<5>{res}, b0, b1, d.row.tw);
        return res;
    }
    // the last pass writes the kept outputs straight to global memory (no closing barrier:
    // the kernel ends there)
    template <bool INV, typename Src, typename Out>
    __device__ static __forceinline__ void run_out(Src src, Out out, int a0, int a1, float2* b0, float2* b1, int,
                                                   const BlasmDev& d) {
        auto sink = [=](int, int a, float2 v) {
            if (a >= a0 && a < a1) out(a, v);
        };
        CtFft<5, NT, N, INV, 1, MI, MO, false, R...>::run(ElemLoadF<Src>{src}, ElemStoreF<decltype(sink)>{sink}, b0,
                                                          b1, d.row.tw);
    }
};

// Compile-time row plans (forward kernels: the pruned radix 16 first; inverse
// kernels: radix 16 last), selected when the run-time plan is the default one
// for that length (its twiddle table serves both orders):
//   1080p    4480 = 16 x 8 x 5 x 7, 320 threads (280, 560, 896, 640 butterflies in 1, 2, 3, 2 rounds)
//   512x512  1664 = 16 x 8 x 13
//   768x1024 2688 = 16 x 8 x 3 x 7
//   256x256  1152 = 16 x 8 x 3 x 3
constexpr int kRow4480Threads = 320;
struct RowsRuntime {
    using F = RowRuntime;
    using I = RowRuntime;
};
struct Rows4480 {
    using F = RowCT<kRow4480Threads, true, false, 4480, 16, 8, 5, 7>;
    using I = RowCT<kRow4480Threads, false, true, 4480, 8, 5, 7, 16>;
};
struct Rows1664 {
    using F = RowCT<kRowThreads, true, false, 1664, 16, 8, 13>;
    using I = RowCT<kRowThreads, false, true, 1664, 8, 13, 16>;
};
struct Rows2688 {
    using F = RowCT<kRowThreads, true, false, 2688, 16, 8, 3, 7>;
    using I = RowCT<kRowThreads, false, true, 2688, 8, 3, 7, 16>;
};
struct Rows1152 {
    using F = RowCT<kRowThreads, true, false, 1152, 16, 8, 3, 3>;
    using I = RowCT<kRowThreads, false, true, 1152, 8, 3, 3, 16>;
};

static bool row_plan_is(const BlasmDev& d, int n, std::initializer_list<int> radices) {
    if (d.NW != n || d.row.npass != (int)radices.size()) return false;
    int p = 0;
    for (int r : radices)
        if ((int)((d.row.code >> (5 * p++)) & 31ull) != r) return false;
    return true;
}

// K1: one padded row per CTA. The first FFT pass reads the splat field directly
// (replicate guard band, Tukey window, amplitude clamp on the fly).
template <class RF = RowRuntime>
__global__ void __launch_bounds__(RF::kThreads, 3) blasm_rows_fwd_kernel(BlasmDev d, const float2* __restrict__ in,
                                                                     float2* __restrict__ A) {
    extern __shared__ float2 sm[];
    const int ld = fft_ld(d.NW);
    float2* b0 = sm;
    float2* b1 = sm + ld;
    const int c = blockIdx.x / d.pH, y = blockIdx.x - c * d.pH;
    const int x0 = (d.NW >> 1) - (d.pW >> 1);
    const int pW = d.pW;
    float2* dst = A + ((size_t)c * d.pH + y) * d.NW;
    auto out = [=](int a, float2 v) { dst[a] = v; };
    if (d.input_mode == 0) {
        const int yy = min(max(y - d.pad_h, 0), d.H - 1);
        const float wyv = __ldg(&d.wy[y]);
        const float2* src = in + ((size_t)c * d.H + yy) * d.W;
        const float* wx = d.wx;
        const int pad_w = d.pad_w, W = d.W;
        RF::template run_out<false>(
            [=](int, int e) {
                const int x = e - x0;
                if (x < 0 || x >= pW) return make_float2(0.f, 0.f);
                const int xx = min(max(x - pad_w, 0), W - 1);
                const float w = wyv * __ldg(&wx[x]);
                const float2 u = __ldg(&src[xx]);
                return clamp_amplitude(make_float2(u.x * w, u.y * w));
            },
            out, 0, d.NW, b0, b1, ld, d);
    } else {
        const float2* src = in + ((size_t)c * d.pH + y) * d.pW;
        RF::template run_out<false>(
            [=](int, int e) {
                const int x = e - x0;
                return (x < 0 || x >= pW) ? make_float2(0.f, 0.f) : __ldg(&src[x]);
            },
            out, 0, d.NW, b0, b1, ld, d);
    }
}

// K2 (generic variant, any plan): the spectrum stays in a third shared buffer.
__global__ void __launch_bounds__(kColThreads, 3) blasm_cols_fwd_kernel(BlasmDev d, const float2* __restrict__ A,
                                                                     float2* __restrict__ B) {
    extern __shared__ float2 sm[];
    const int NH = d.NH, NW = d.NW, ld = fft_ld(NH);
    float2* buf[3] = {sm, sm + ld, sm + 2 * ld};
    const int c = blockIdx.x / NW, kx = blockIdx.x - c * NW;
    const int y0 = (NH >> 1) - (d.pH >> 1), pH = d.pH;
    const float2* src = A + (size_t)c * pH * NW + kx;
    float2* spec = fft_run(
        [=](int, int e) {
            const int y = e - y0;
            return (y < 0 || y >= pH) ? make_float2(0.f, 0.f) : __ldg(&src[(size_t)y * NW]);
        },
        buf[0], buf[1], ld, 0, d.col, false);
    float2* w0 = spec == buf[0] ? buf[1] : buf[0];
    float2* w1 = buf[2];
    const int row0 = (NH >> 1) - (d.out_h >> 1);
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        const PCParam pp = d.pcp[pc];
        const float2* sp = spec;
        float2* res = fft_run([=](int, int e) { return cmul(sp[fft_pad(e)], transfer(d, pp, c, e, kx)); }, w0, w1, ld,
                              0, d.col, true);
        float2* dst = B + (size_t)pc * d.out_h * NW + kx;
        for (int y = threadIdx.x; y < d.out_h; y += blockDim.x) dst[(size_t)y * NW] = res[fft_pad(row0 + y)];
        __syncthreads();
    }
}

// K3: inverse FFT of a kept row (first pass reads global), keep out_w columns
// -> V [P*C][out_h][out_w] and optionally pred = clamp(|V|^2, 0, 1)
template <class RF = RowRuntime>
__global__ void __launch_bounds__(RF::kThreads, 3) blasm_rows_inv_kernel(BlasmDev d, const float2* __restrict__ B,
                                                                     float2* __restrict__ V,
                                                                     float* __restrict__ pred) {
    extern __shared__ float2 sm[];
    const int ld = fft_ld(d.NW);
    const size_t row = blockIdx.x;  // pc * out_h + y
    const float2* src = B + row * d.NW;
    const int col0 = (d.NW >> 1) - (d.out_w >> 1);
    float2* dst = V + row * d.out_w;
    float* pd = pred ? pred + row * d.out_w : nullptr;
    // V and the training prediction clamp(|V|^2, 0, 1) (train_2d_gaussian_rgb.py:193-194)
    RF::template run_out<true>(
        [=](int, int e) { return __ldg(&src[e]); },
        [=](int a, float2 v) {
            dst[a - col0] = v;
            // torch.clamp(I, 0, 1) keeps a NaN (fminf would turn it into 1)
            const float i2 = v.x * v.x + v.y * v.y;
            if (pd) pd[a - col0] = i2 > 1.0f ? 1.0f : i2;
        },
        col0, col0 + d.out_w, sm, sm + ld, ld, d);
}

// ---------------------------------------------------------------------------
// adjoint kernels (same layouts: Bt [P*C][out_h][NW], Ab [C][in_h][NW])
// ---------------------------------------------------------------------------
// K3b: gradient row embedded at the out_w centred columns -> forward FFT
template <class RF = RowRuntime>
__global__ void __launch_bounds__(RF::kThreads, 3) blasm_rows_fwd_adj_kernel(BlasmDev d, const float2* __restrict__ gV,
                                                                         const float* __restrict__ gpred,
                                                                         const float2* __restrict__ Vf,
                                                                         float2* __restrict__ Bt) {
    extern __shared__ float2 sm[];
    const int ld = fft_ld(d.NW);
    const int row = blockIdx.x;
    const int col0 = (d.NW >> 1) - (d.out_w >> 1);
    const int ow = d.out_w;
    float2* dst = Bt + (size_t)row * d.NW;
    auto out = [=](int a, float2 v) { dst[a] = v; };
    if (gpred) {
        // dL/dV = 2 V dL/dpred where 0 <= |V|^2 <= 1 (clamp passes its bounds), else 0
        const float* gp = gpred + (size_t)row * ow;
        const float2* vv = Vf + (size_t)row * ow;
        RF::template run_out<false>(
            [=](int, int e) {
                const int x = e - col0;
                if (x < 0 || x >= ow) return make_float2(0.f, 0.f);
                // both loads issued together (the gate on |V|^2 only selects afterwards)
                const float2 v = __ldg(&vv[x]);
                const float gpx = __ldg(&gp[x]);
                const float g = (v.x * v.x + v.y * v.y <= 1.0f) ? 2.0f * gpx : 0.0f;
                return make_float2(g * v.x, g * v.y);
            },
            out, 0, d.NW, sm, sm + ld, ld, d);
    } else {
        const float2* src = gV + (size_t)row * ow;
        RF::template run_out<false>(
            [=](int, int e) {
                const int x = e - col0;
                return (x < 0 || x >= ow) ? make_float2(0.f, 0.f) : __ldg(&src[x]);
            },
            out, 0, d.NW, sm, sm + ld, ld, d);
    }
}

// K2b (generic variant): accumulator in registers over a fixed element mapping.
template <int E>
__global__ void __launch_bounds__(kColThreads, 3) blasm_cols_adj_kernel(BlasmDev d, const float2* __restrict__ Bt,
                                                                     float2* __restrict__ Ab) {
    extern __shared__ float2 sm[];
    const int NH = d.NH, NW = d.NW, ld = fft_ld(NH);
    float2* b0 = sm;
    float2* b1 = sm + ld;
    const int c = blockIdx.x / NW, kx = blockIdx.x - c * NW;
    const int row0 = (NH >> 1) - (d.out_h >> 1), oh = d.out_h;
    float2 acc[E];
#pragma unroll
    for (int i = 0; i < E; i++) acc[i] = make_float2(0.f, 0.f);
    for (int p = 0; p < d.P; p++) {
        const int pc = p * d.C + c;
        const float2* src = Bt + (size_t)pc * oh * NW + kx;
        float2* res = fft_run(
            [=](int, int e) {
                const int y = e - row0;
                return (y < 0 || y >= oh) ? make_float2(0.f, 0.f) : __ldg(&src[(size_t)y * NW]);
            },
            b0, b1, ld, 0, d.col, false);
        const PCParam pp = d.pcp[pc];
#pragma unroll
        for (int i = 0; i < E; i++) {
            const int ky = threadIdx.x + i * blockDim.x;
            if (ky < NH) acc[i] = cadd(acc[i], cmulc(res[fft_pad(ky)], transfer(d, pp, c, ky, kx)));
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < E; i++) {
        const int ky = threadIdx.x + i * blockDim.x;
        if (ky < NH) b0[fft_pad(ky)] = acc[i];
    }
    __syncthreads();
    float2* res = fft_run([b0](int, int e) { return b0[fft_pad(e)]; }, b1, b0, ld, 0, d.col, true);
    const int in_h = d.input_mode == 0 ? d.H : d.pH;
    const int r0 = (NH >> 1) - (in_h >> 1);
    float2* dst = Ab + (size_t)c * in_h * NW + kx;
    for (int y = threadIdx.x; y < in_h; y += blockDim.x) dst[(size_t)y * NW] = res[fft_pad(r0 + y)];
}

// K1b: inverse row FFT (first pass reads global), keep the input columns,
// apply the amplitude-clamp adjoint against the splat field
template <class RF = RowRuntime>
__global__ void __launch_bounds__(RF::kThreads, 3) blasm_rows_inv_adj_kernel(BlasmDev d, const float2* __restrict__ Ab,
                                                                         const float2* __restrict__ field,
                                                                         float2* __restrict__ gin) {
    extern __shared__ float2 sm[];
    const int ld = fft_ld(d.NW);
    const int row = blockIdx.x;  // c * in_h + y
    const float2* src = Ab + (size_t)row * d.NW;
    const int in_w = d.input_mode == 0 ? d.W : d.pW;
    const int c0 = (d.NW >> 1) - (in_w >> 1);
    float2* dst = gin + (size_t)row * in_w;
    auto load = [=](int, int e) { return __ldg(&src[e]); };
    if (d.input_mode == 0) {
        const float2* u = field + (size_t)row * d.W;  // the window is exactly 1 over the image
        RF::template run_out<true>(
            load, [=](int a, float2 v) { dst[a - c0] = clamp_amplitude_adjoint(u[a - c0], v); }, c0, c0 + in_w, sm,
            sm + ld, ld, d);
    } else {
        RF::template run_out<true>(load, [=](int a, float2 v) { dst[a - c0] = v; }, c0, c0 + in_w, sm, sm + ld, ld,
                                   d);
    }
}

// ---------------------------------------------------------------------------
// host: table blob, device config, launches
// ---------------------------------------------------------------------------
struct TableLayout {
    size_t tw_row, tw_col, wy, wx, a_row, b_col, aperture, pcp, total;
};

static TableLayout table_layout(int C, int P, int pH, int pW) {
    TableLayout L;
    const int NH = 2 * pH, NW = 2 * pW;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~(size_t)255;
        size_t o = off;
        off += bytes;
        return o;
    };
    L.tw_row = take(sizeof(float2) * NW);
    L.tw_col = take(sizeof(float2) * NH);
    L.wy = take(sizeof(float) * pH);
    L.wx = take(sizeof(float) * pW);
    L.a_row = take(sizeof(float) * C * NH);
    L.b_col = take(sizeof(float) * C * NW);
    L.aperture = take(sizeof(int2) * NH);
    L.pcp = take(sizeof(PCParam) * P * C);
    L.total = off;
    return L;
}

static int validate(const cvqpg_blasm_params* p) {
    if (!p) return CVQPG_ERR_ARG;
    if (p->channels != 1 && p->channels != 3) return CVQPG_ERR_CHANNELS;
    if (p->planes < 1 || p->planes > kMaxPlanes) return CVQPG_ERR_UNSUPPORTED;
    const int H = p->height, W = p->width, pH = p->pad_height, pW = p->pad_width;
    if (H <= 0 || W <= 0 || pH < H || pW < W) return CVQPG_ERR_ARG;
    if ((H | W | pH | pW) & 1) return CVQPG_ERR_UNSUPPORTED;
    const int oh = p->out_height > 0 ? p->out_height : H, ow = p->out_width > 0 ? p->out_width : W;
    if (oh > pH || ow > pW || ((oh | ow) & 1)) return CVQPG_ERR_UNSUPPORTED;
    if (p->input_mode != 0 && p->input_mode != 1) return CVQPG_ERR_ARG;
    if (!(p->pixel_pitch > 0)) return CVQPG_ERR_ARG;
    FftPlan a, b;
    if (!make_fft_plan(2 * pH, &a) || !make_fft_plan(2 * pW, &b)) return CVQPG_ERR_UNSUPPORTED;
    return CVQPG_OK;
}

// Tukey taper of the reference soft_window_pad (_taper_1d, model_2d_gaussian_rgb.py:224-235)
static void taper_1d(int total, int inner_start, int inner_size, float* w) {
    for (int t = 0; t < total; t++) w[t] = 0.0f;
    for (int t = inner_start; t < inner_start + inner_size; t++) w[t] = 1.0f;
    for (int t = 0; t < inner_start; t++) w[t] = (float)(0.5 * (1.0 - cos(M_PI * (t + 1.0) / inner_start)));
    const int right = inner_start + inner_size, n_right = total - right;
    for (int t = 0; t < n_right; t++) w[right + t] = (float)(0.5 * (1.0 + cos(M_PI * (t + 1.0) / n_right)));
}

// symmetric frequency sample j of an n-point axis (odak BLASM grid convention, see oracle/odak_restated.py)
static double freq(int j, int n, double dx) {
    const double s = dx * n;
    const double a = -1.0 / (2.0 * dx) + 0.5 / (2.0 * s);
    const double b = 1.0 / (2.0 * dx) - 0.5 / (2.0 * s);
    return a + (b - a) * (double)j / (double)(n - 1);
}

static void band_interval(int n, double dx, double lim, int* lo, int* hi) {
    int a = n, b = 0;
    for (int j = 0; j < n; j++)
        if (fabs(freq(j, n, dx)) < lim) {
            a = std::min(a, j);
            b = std::max(b, j + 1);
        }
    if (a >= b) a = b = 0;
    *lo = a;
    *hi = b;
}

int blasm_make_dev(const cvqpg_blasm_params* p, const void* tables, size_t table_bytes, BlasmDev* d) {
    int st = validate(p);
    if (st != CVQPG_OK) return st;
    const int C = p->channels, P = p->planes;
    TableLayout L = table_layout(C, P, p->pad_height, p->pad_width);
    if (!tables || table_bytes < L.total) return CVQPG_ERR_WORKSPACE;
    std::memset(d, 0, sizeof(*d));
    d->C = C;
    d->P = P;
    d->H = p->height;
    d->W = p->width;
    d->pH = p->pad_height;
    d->pW = p->pad_width;
    d->NH = 2 * d->pH;
    d->NW = 2 * d->pW;
    d->pad_h = (d->pH - d->H) / 2;
    d->pad_w = (d->pW - d->W) / 2;
    d->out_h = p->out_height > 0 ? p->out_height : d->H;
    d->out_w = p->out_width > 0 ? p->out_width : d->W;
    d->input_mode = p->input_mode;
    // adjacent columns per column-pass CTA: four where a four-column kernel exists
    // (blasm_cols4.cuh; row-major intermediates either way), unless the hint asks for one
    d->G = (p->plan_hint & CVQPG_PLAN_COLS1) || (d->NW % 4) != 0 ? 1 : 4;
    if ((size_t)3 * fft_ld(d->NH) * sizeof(float2) > 227 * 1024) return CVQPG_ERR_UNSUPPORTED;
    d->scale = (float)(1.0 / ((double)d->NH * (double)d->NW));
    const int hint = p->plan_hint;
    d->col_radix = hint & 31;
    if (!make_fft_plan(d->NW, &d->row, (hint >> 8) & 7) || !make_fft_plan(d->NH, &d->col, (hint >> 5) & 7))
        return CVQPG_ERR_UNSUPPORTED;
    const char* base = (const char*)tables;
    d->row.tw = (const float2*)(base + L.tw_row);
    d->col.tw = (const float2*)(base + L.tw_col);
    d->wy = (const float*)(base + L.wy);
    d->wx = (const float*)(base + L.wx);
    d->a_row = (const float*)(base + L.a_row);
    d->b_col = (const float*)(base + L.b_col);
    d->aperture = (const int2*)(base + L.aperture);
    d->pcp = (const PCParam*)(base + L.pcp);
    return CVQPG_OK;
}

size_t blasm_workspace_bytes(const BlasmDev& d) {
    const size_t a = (size_t)d.C * d.NW * d.pH;
    const size_t b = (size_t)d.P * d.C * d.out_h * d.NW;
    return ((a * sizeof(float2) + 255) & ~(size_t)255) + b * sizeof(float2) + 256;
}

static void carve(const BlasmDev& d, void* ws, float2** A, float2** B) {
    const size_t a = (size_t)d.C * d.NW * d.pH;
    *A = (float2*)ws;
    *B = (float2*)((char*)ws + ((a * sizeof(float2) + 255) & ~(size_t)255));
}

static size_t row_smem(const BlasmDev& d) { return (size_t)2 * fft_ld(d.NW) * sizeof(float2); }
static size_t col2_smem(const BlasmDev& d) { return (size_t)2 * fft_ld(d.NH) * sizeof(float2); }
static size_t col3_smem(const BlasmDev& d) { return (size_t)3 * fft_ld(d.NH) * sizeof(float2); }
constexpr size_t kSmemMax = 227 * 1024;

#define CVQPG_SMEM_ATTR(kern, bytes) cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(bytes))

// Pick the radix whose butterflies stay in registers between the column FFTs:
// the supported radix of the plan with the smallest register footprint
// (butterflies per thread x radix). Returns false when no variant applies.
static bool column_split(const FftPlan& plan, ColSplit* cs, int radix_hint) {
    static const int kRL[] = {3, 5, 7, 8, 11, 13, 16};
    int best = -1, best_mb = 0, best_score = 1 << 30;
    for (int p = 0; p < plan.npass; p++) {
        const int r = (int)((plan.code >> (5 * p)) & 31ull);
        bool ok = false;
        for (int q : kRL) ok |= (q == r);
        if (!ok || plan.npass < 2) continue;
        const int nb = plan.n / r;
        const int mb = (nb + kColThreads - 1) / kColThreads;
        const int mbr = mb <= 1 ? 1 : (mb <= 2 ? 2 : 0);
        if (!mbr) continue;
        // the hinted radix wins when the plan has it; otherwise the smallest register footprint
        const int score = (radix_hint && r == radix_hint) ? -1 : mbr * r;
        if (score < best_score) {
            best_score = score;
            best = p;
            best_mb = mbr;
        }
    }
    if (best < 0) return false;
    int rmin = plan.n;
    for (int p = 0; p < plan.npass; p++) rmin = std::min(rmin, (int)((plan.code >> (5 * p)) & 31ull));
    cs->ntw = plan.n / rmin;
    if (((size_t)2 * fft_ldT<kColPad>(plan.n) + cs->ntw) * sizeof(float2) + (size_t)plan.n * sizeof(float) > kSmemMax)
        return false;
    cs->rl = (int)((plan.code >> (5 * best)) & 31ull);
    cs->mb = best_mb;
    cs->head_code = 0;
    cs->head_npass = 0;
    for (int p = 0; p < plan.npass; p++) {
        if (p == best) continue;
        const unsigned long long r = (plan.code >> (5 * p)) & 31ull;
        cs->head_code |= r << (5 * cs->head_npass);
        cs->head_npass++;
    }
    return true;
}

static void launch_columns(bool adjoint, const BlasmDev& d, const float2* in, float2* out, cudaStream_t s) {
    ColSplit cs;
    if (column_split(d.col, &cs, d.col_radix)) {
        if (launch_cols_ct(adjoint, d, cs, in, out, s)) return;
        switch (cs.rl) {
            case 3: launch_cols_reg_r3(adjoint, d, cs, in, out, s); return;
            case 5: launch_cols_reg_r5(adjoint, d, cs, in, out, s); return;
            case 7: launch_cols_reg_r7(adjoint, d, cs, in, out, s); return;
            case 8: launch_cols_reg_r8(adjoint, d, cs, in, out, s); return;
            case 11: launch_cols_reg_r11(adjoint, d, cs, in, out, s); return;
            case 13: launch_cols_reg_r13(adjoint, d, cs, in, out, s); return;
            case 16: launch_cols_reg_r16(adjoint, d, cs, in, out, s); return;
            default: break;
        }
    }
    if (!adjoint) {
        const size_t sm = col3_smem(d);
        CVQPG_SMEM_ATTR(blasm_cols_fwd_kernel, sm);
        blasm_cols_fwd_kernel<<<d.C * d.NW, kColThreads, sm, s>>>(d, in, out);
    } else {
        const size_t sm = col2_smem(d);
        const int e = (d.NH + kColThreads - 1) / kColThreads;
        if (e <= 8) {
            CVQPG_SMEM_ATTR(blasm_cols_adj_kernel<8>, sm);
            blasm_cols_adj_kernel<8><<<d.C * d.NW, kColThreads, sm, s>>>(d, in, out);
        } else if (e <= 16) {
            CVQPG_SMEM_ATTR(blasm_cols_adj_kernel<16>, sm);
            blasm_cols_adj_kernel<16><<<d.C * d.NW, kColThreads, sm, s>>>(d, in, out);
        } else {
            CVQPG_SMEM_ATTR(blasm_cols_adj_kernel<32>, sm);
            blasm_cols_adj_kernel<32><<<d.C * d.NW, kColThreads, sm, s>>>(d, in, out);
        }
    }
}

template <class RF>
static void rows_forward(const BlasmDev& d, const float2* in, float2* A, cudaStream_t s) {
    const size_t rs = row_smem(d);
    CVQPG_SMEM_ATTR(blasm_rows_fwd_kernel<RF>, rs);
    blasm_rows_fwd_kernel<RF><<<d.C * d.pH, RF::kThreads, rs, s>>>(d, in, A);
}

template <class RF>
static void rows_inverse(const BlasmDev& d, const float2* B, float2* out, float* pred, cudaStream_t s) {
    const size_t rs = row_smem(d);
    CVQPG_SMEM_ATTR(blasm_rows_inv_kernel<RF>, rs);
    blasm_rows_inv_kernel<RF><<<d.P * d.C * d.out_h, RF::kThreads, rs, s>>>(d, B, out, pred);
}

template <class RF>
static void rows_forward_adjoint(const BlasmDev& d, const float2* grad_out, const float* grad_pred,
                                 const float2* vfield, float2* B, cudaStream_t s) {
    const size_t rs = row_smem(d);
    CVQPG_SMEM_ATTR(blasm_rows_fwd_adj_kernel<RF>, rs);
    blasm_rows_fwd_adj_kernel<RF><<<d.P * d.C * d.out_h, RF::kThreads, rs, s>>>(d, grad_out, grad_pred, vfield, B);
}

template <class RF>
static void rows_inverse_adjoint(const BlasmDev& d, const float2* A, const float2* in_field, float2* grad_in,
                                 cudaStream_t s) {
    const size_t rs = row_smem(d);
    const int in_h = d.input_mode == 0 ? d.H : d.pH;
    CVQPG_SMEM_ATTR(blasm_rows_inv_adj_kernel<RF>, rs);
    blasm_rows_inv_adj_kernel<RF><<<d.C * in_h, RF::kThreads, rs, s>>>(d, A, in_field, grad_in);
}

template <class RP>
static void forward_with(const BlasmDev& d, const float2* in, float2* out, float* pred, float2* A, float2* B,
                         cudaStream_t s, StageMarks* marks) {
    rows_forward<typename RP::F>(d, in, A, s);
    if (marks) marks->mark(s);
    launch_columns(false, d, A, B, s);
    if (marks) marks->mark(s);
    rows_inverse<typename RP::I>(d, B, out, pred, s);
    if (marks) marks->mark(s);
}

template <class RP>
static void backward_with(const BlasmDev& d, const float2* in_field, const float2* grad_out,
                          const float* grad_pred, const float2* vfield, float2* grad_in, float2* A, float2* B,
                          cudaStream_t s, StageMarks* marks) {
    rows_forward_adjoint<typename RP::F>(d, grad_out, grad_pred, vfield, B, s);
    if (marks) marks->mark(s);
    launch_columns(true, d, B, A, s);
    if (marks) marks->mark(s);
    rows_inverse_adjoint<typename RP::I>(d, A, in_field, grad_in, s);
    if (marks) marks->mark(s);
}

// calls f(RowsX{}) for the row plan of d
template <typename F>
static void with_row_plan(const BlasmDev& d, F&& f) {
    if (row_plan_is(d, 4480, {16, 8, 5, 7}))
        f(Rows4480{});
    else if (row_plan_is(d, 1664, {16, 8, 13}))
        f(Rows1664{});
    else if (row_plan_is(d, 2688, {16, 8, 3, 7}))
        f(Rows2688{});
    else if (row_plan_is(d, 1152, {16, 8, 3, 3}))
        f(Rows1152{});
    else
        f(RowsRuntime{});
}

void blasm_forward(const BlasmDev& d, const float2* in, float2* out, float* pred, void* workspace, cudaStream_t s,
                   StageMarks* marks) {
    float2 *A, *B;
    carve(d, workspace, &A, &B);
    with_row_plan(d, [&](auto rp) { forward_with<decltype(rp)>(d, in, out, pred, A, B, s, marks); });
}

void blasm_backward(const BlasmDev& d, const float2* in_field, const float2* grad_out, const float* grad_pred,
                    const float2* vfield, float2* grad_in, void* workspace, cudaStream_t s, StageMarks* marks) {
    float2 *A, *B;
    carve(d, workspace, &A, &B);
    with_row_plan(d, [&](auto rp) {
        backward_with<decltype(rp)>(d, in_field, grad_out, grad_pred, vfield, grad_in, A, B, s, marks);
    });
}

static bool fits(const BlasmDev& d) {
    return row_smem(d) <= kSmemMax && col3_smem(d) <= kSmemMax && (d.NH + kColThreads - 1) / kColThreads <= 32;
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

extern "C" int cvqpg_blasm_tables_size(const cvqpg_blasm_params* p, size_t* bytes) {
    if (!bytes) return CVQPG_ERR_ARG;
    int st = validate(p);
    if (st != CVQPG_OK) return st;
    *bytes = table_layout(p->channels, p->planes, p->pad_height, p->pad_width).total;
    return CVQPG_OK;
}

extern "C" int cvqpg_blasm_setup(const cvqpg_blasm_params* p, void* tables, size_t table_bytes) {
    int st = validate(p);
    if (st != CVQPG_OK) return st;
    const int C = p->channels, P = p->planes, pH = p->pad_height, pW = p->pad_width;
    const int H = p->height, W = p->width, NH = 2 * pH, NW = 2 * pW;
    TableLayout L = table_layout(C, P, pH, pW);
    if (!tables || table_bytes < L.total) return CVQPG_ERR_WORKSPACE;
    std::vector<char> host(L.total, 0);
    char* b = host.data();
    auto twiddles = [](int n, float2* t) {
        for (int m = 0; m < n; m++) {
            const double a = -2.0 * M_PI * (double)m / (double)n;
            t[m] = make_float2((float)cos(a), (float)sin(a));
        }
    };
    twiddles(NW, (float2*)(b + L.tw_row));
    twiddles(NH, (float2*)(b + L.tw_col));
    taper_1d(pH, (pH - H) / 2, H, (float*)(b + L.wy));
    taper_1d(pW, (pW - W) / 2, W, (float*)(b + L.wx));
    const double dx = p->pixel_pitch;
    float* ar = (float*)(b + L.a_row);
    float* bc = (float*)(b + L.b_col);
    for (int c = 0; c < C; c++) {
        const double lam = p->wavelengths[c];
        for (int j = 0; j < NH; j++) {
            const double f = freq(j, NH, dx);
            ar[c * NH + j] = (float)(lam * lam * f * f);
        }
        for (int i = 0; i < NW; i++) {
            const double f = freq(i, NW, dx);
            bc[c * NW + i] = (float)(lam * lam * f * f);
        }
    }
    // circular Fourier aperture (utils/propagator.py:10-38, 179-200): per centred row j the
    // allowed centred columns i satisfy sqrt(X_j^2 + Y_i^2) < r, X = linspace(-NH/2, NH/2, NH)
    int2* ap = (int2*)(b + L.aperture);
    const double r = p->aperture_radius;
    for (int j = 0; j < NH; j++) {
        if (!(r > 0)) {
            ap[j] = make_int2(0, NW);
            continue;
        }
        const double X = -NH / 2.0 + (double)NH * j / (NH - 1.0);
        int lo = NW, hi = 0;
        for (int i = 0; i < NW; i++) {
            const double Y = -NW / 2.0 + (double)NW * i / (NW - 1.0);
            if (sqrt(X * X + Y * Y) < r) {
                lo = std::min(lo, i);
                hi = std::max(hi, i + 1);
            }
        }
        ap[j] = lo < hi ? make_int2(lo, hi) : make_int2(0, 0);
    }
    PCParam* pcp = (PCParam*)(b + L.pcp);
    for (int pl = 0; pl < P; pl++)
        for (int c = 0; c < C; c++) {
            const double lam = p->wavelengths[c], z = p->distances[pl];
            PCParam q;
            std::memset(&q, 0, sizeof(q));
            const double K = 2.0 * M_PI * z / lam;
            q.K = (float)K;
            double t0 = fmod(K, 2.0 * M_PI);
            if (t0 < 0) t0 += 2.0 * M_PI;
            q.theta0 = (float)t0;
            const double lim_r = 1.0 / sqrt(pow(2.0 * z * (1.0 / (dx * NH)), 2) + 1.0) / lam;
            const double lim_c = 1.0 / sqrt(pow(2.0 * z * (1.0 / (dx * NW)), 2) + 1.0) / lam;
            band_interval(NH, dx, lim_r, &q.j0, &q.j1);
            band_interval(NW, dx, lim_c, &q.i0, &q.i1);
            pcp[pl * C + c] = q;
        }
    if (cudaMemcpy(tables, host.data(), L.total, cudaMemcpyHostToDevice) != cudaSuccess) return CVQPG_ERR_CUDA;
    return CVQPG_OK;
}

extern "C" int cvqpg_blasm_workspace_size(const cvqpg_blasm_params* p, size_t* bytes) {
    if (!bytes) return CVQPG_ERR_ARG;
    int st = validate(p);
    if (st != CVQPG_OK) return st;
    BlasmDev d;
    static const char dummy[1] = {0};
    st = blasm_make_dev(p, dummy, (size_t)-1, &d);
    if (st != CVQPG_OK) return st;
    *bytes = blasm_workspace_bytes(d);
    return CVQPG_OK;
}

extern "C" int cvqpg_blasm_forward(const cvqpg_blasm_params* p, const void* tables, size_t table_bytes,
                                   const float* input, float* out_field, void* workspace, size_t workspace_bytes,
                                   void* stream) {
    BlasmDev d;
    int st = blasm_make_dev(p, tables, table_bytes, &d);
    if (st != CVQPG_OK) return st;
    if (!fits(d)) return CVQPG_ERR_UNSUPPORTED;
    if (!input || !out_field || !workspace) return CVQPG_ERR_ARG;
    if (workspace_bytes < blasm_workspace_bytes(d)) return CVQPG_ERR_WORKSPACE;
    blasm_forward(d, (const float2*)input, (float2*)out_field, nullptr, workspace, (cudaStream_t)stream);
    return launch_status();
}

extern "C" int cvqpg_blasm_backward(const cvqpg_blasm_params* p, const void* tables, size_t table_bytes,
                                    const float* input, const float* grad_out, float* grad_input, void* workspace,
                                    size_t workspace_bytes, void* stream) {
    BlasmDev d;
    int st = blasm_make_dev(p, tables, table_bytes, &d);
    if (st != CVQPG_OK) return st;
    if (!fits(d)) return CVQPG_ERR_UNSUPPORTED;
    if (!grad_out || !grad_input || !workspace || (d.input_mode == 0 && !input)) return CVQPG_ERR_ARG;
    if (workspace_bytes < blasm_workspace_bytes(d)) return CVQPG_ERR_WORKSPACE;
    blasm_backward(d, (const float2*)input, (const float2*)grad_out, nullptr, nullptr, (float2*)grad_input,
                   workspace, (cudaStream_t)stream);
    return launch_status();
}

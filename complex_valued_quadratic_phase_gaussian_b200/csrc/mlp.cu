// Per-tile MLP of the learned initialiser: in_dim -> hidden -> hidden -> out_dim,
// GELU (erf form) after the two hidden layers, BF16 operands with FP32
// accumulation on the tensor cores (gemm.cu), FP32 master weights, Adam.
// No reference counterpart: the reference initialises every fit at random.
//
// Weights (FP32, flat): W1 [H][D] | b1 [H] | W2 [H][H] | b2 [H] | W3 [O'][H] | b3 [O']
// with O' = out_dim rounded up to 128; rows >= out_dim of W3/b3 stay zero.
// Derived BF16 copies live in the workspace, both row-major (forward B operand)
// and transposed (backward B operand): W1b, W1t, W2b, W2t, W3b, W3t.
//
// One training step (every launch on `stream`, nothing synchronises the host):
//   X (fp32 [M][D]) -> X0 bf16 [M'][D] + X0t [D][M']   (rows >= M are zero)
//   Z1 = X0 W1^T + b1, H1 = GELU(Z1)     -> Z1 f32, H1 bf16, H1t
//   Z2 = H1 W2^T + b2, H2 = GELU(Z2)     -> Z2 f32, H2 bf16, H2t
//   Y  = H2 W3^T + b3                    -> Y f32 [M'][O']
//   L  = sum_{m<M, j<O} w_j (Y - T)^2 / M;  dY -> dZ3 bf16 [M'][O'] + dZ3t
//   dZ2 = (dZ3 W3) * GELU'(Z2)           -> dZ2 bf16 + dZ2t
//   dZ1 = (dZ2 W2) * GELU'(Z1)           -> dZ1t
//   dW3 = dZ3t H2t^T, dW2 = dZ2t H1t^T, dW1 = dZ1t X0t^T   (split-K slabs, fixed-order sum)
//   db_l = row sums of dZ_l t            (fixed order)
//   Adam (bias-corrected), then refresh the BF16 copies.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>

#include "gemm.cuh"

namespace cvqpg {

struct MlpDims {
    int M, Mp;        // batch, padded to 128
    int D, Hd, O, Op; // in, hidden, out, out padded to 128
    int splits;       // split-K of the weight-gradient GEMMs
    size_t off_w1, off_b1, off_w2, off_b2, off_w3, off_b3, total;
};

static int mlp_dims(const cvqpg_mlp_params* p, MlpDims* d) {
    if (!p || p->batch < 1 || p->in_dim < 1 || p->hidden < 1 || p->out_dim < 1) return CVQPG_ERR_ARG;
    if (p->in_dim % 128 || p->hidden % 128) return CVQPG_ERR_UNSUPPORTED;
    d->M = p->batch;
    d->Mp = (p->batch + 127) / 128 * 128;
    d->D = p->in_dim;
    d->Hd = p->hidden;
    d->O = p->out_dim;
    d->Op = (p->out_dim + 127) / 128 * 128;
    const int kb = d->Mp / 64;
    d->splits = 1;
    for (int s : {8, 4, 2})
        if (kb % s == 0) {
            d->splits = s;
            break;
        }
    size_t o = 0;
    d->off_w1 = o; o += (size_t)d->Hd * d->D;
    d->off_b1 = o; o += d->Hd;
    d->off_w2 = o; o += (size_t)d->Hd * d->Hd;
    d->off_b2 = o; o += d->Hd;
    d->off_w3 = o; o += (size_t)d->Op * d->Hd;
    d->off_b3 = o; o += d->Op;
    d->total = o;
    return CVQPG_OK;
}

struct MlpWs {
    __nv_bfloat16 *x0, *x0t, *h1, *h1t, *h2, *h2t, *dz3, *dz3t, *dz2, *dz2t, *dz1t;
    __nv_bfloat16 *w1b, *w1t, *w2b, *w2t, *w3b, *w3t;
    float *z1, *z2, *y, *slabs, *grads, *loss_part;
};

constexpr int kLossBlocks = 256;

static size_t mlp_carve(const MlpDims& d, void* base, MlpWs* w) {
    Carver c(base, ~(size_t)0);
    typedef __nv_bfloat16 bf;
    const size_t Mp = d.Mp;
    w->x0 = c.take<bf>(Mp * d.D);
    w->x0t = c.take<bf>(Mp * d.D);
    w->h1 = c.take<bf>(Mp * d.Hd);
    w->h1t = c.take<bf>(Mp * d.Hd);
    w->h2 = c.take<bf>(Mp * d.Hd);
    w->h2t = c.take<bf>(Mp * d.Hd);
    w->dz3 = c.take<bf>(Mp * d.Op);
    w->dz3t = c.take<bf>(Mp * d.Op);
    w->dz2 = c.take<bf>(Mp * d.Hd);
    w->dz2t = c.take<bf>(Mp * d.Hd);
    w->dz1t = c.take<bf>(Mp * d.Hd);
    w->w1b = c.take<bf>((size_t)d.Hd * d.D);
    w->w1t = c.take<bf>((size_t)d.Hd * d.D);
    w->w2b = c.take<bf>((size_t)d.Hd * d.Hd);
    w->w2t = c.take<bf>((size_t)d.Hd * d.Hd);
    w->w3b = c.take<bf>((size_t)d.Op * d.Hd);
    w->w3t = c.take<bf>((size_t)d.Op * d.Hd);
    w->z1 = c.take<float>(Mp * d.Hd);
    w->z2 = c.take<float>(Mp * d.Hd);
    w->y = c.take<float>(Mp * d.Op);
    size_t slab = std::max((size_t)d.Hd * d.D, std::max((size_t)d.Hd * d.Hd, (size_t)d.Op * d.Hd));
    w->slabs = c.take<float>(slab * d.splits);
    w->grads = c.take<float>(d.total);
    w->loss_part = c.take<float>(kLossBlocks + 4);
    return c.off + 256;
}

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// X fp32 [M][D] -> X0 bf16 [Mp][D] (zero rows beyond M) and X0t [D][Mp]; 32x32 tiles through shared memory.
__global__ void mlp_prep_input_kernel(const float* __restrict__ X, int M, int Mp, int D, __nv_bfloat16* __restrict__ x0,
                                      __nv_bfloat16* __restrict__ x0t) {
    __shared__ float tile[32][33];
    const int d0 = blockIdx.x * 32, m0 = blockIdx.y * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int r = ty; r < 32; r += 8) {
        const int m = m0 + r, dd = d0 + tx;
        const float v = (m < M) ? __ldg(&X[(size_t)m * D + dd]) : 0.0f;
        tile[r][tx] = v;
        x0[(size_t)m * D + dd] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    for (int r = ty; r < 32; r += 8) x0t[(size_t)(d0 + r) * Mp + m0 + tx] = __float2bfloat16_rn(tile[tx][r]);
}

// Weighted squared error against T over the valid block; dY written as BF16
// row-major and transposed (zero outside the valid block); one partial per block.
__global__ void mlp_loss_kernel(const float* __restrict__ Y, int ldy, const float* __restrict__ T,
                                const float* __restrict__ wout, int M, int Mp, int O, int Op,
                                __nv_bfloat16* __restrict__ dz, __nv_bfloat16* __restrict__ dzt,
                                float* __restrict__ part) {
    __shared__ float red[8];
    float acc = 0.0f;
    const float inv_m = 1.0f / (float)M;
    const size_t total = (size_t)Mp * Op;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(i / Op), j = (int)(i - (size_t)m * Op);
        float g = 0.0f;
        if (m < M && j < O) {
            const float r = Y[(size_t)m * ldy + j] - __ldg(&T[(size_t)m * O + j]);
            const float w = __ldg(&wout[j]);
            acc += w * r * r;
            g = 2.0f * w * r * inv_m;
        }
        const __nv_bfloat16 gb = __float2bfloat16_rn(g);
        dz[(size_t)m * Op + j] = gb;
        dzt[(size_t)j * Mp + m] = gb;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.0f;
        for (int k = 0; k < (int)(blockDim.x >> 5); k++) s += red[k];
        part[blockIdx.x] = s;
    }
}

__global__ void mlp_loss_finalize_kernel(const float* __restrict__ part, int nparts, int M, float* __restrict__ out) {
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < nparts; k++) s += part[k];
        out[0] = (float)(s / M);
    }
}

// out[i] = sum_s slab[s][i], fixed order
__global__ void mlp_reduce_slabs_kernel(const float* __restrict__ slabs, int splits, size_t n, size_t stride,
                                        float* __restrict__ out) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < splits; k++) s += slabs[(size_t)k * stride + i];
        out[i] = s;
    }
}

// db[n] = sum_m dzt[n][m] over the first Mp columns, one block per n, fixed-shape tree.
__global__ void mlp_bias_grad_kernel(const __nv_bfloat16* __restrict__ dzt, int Mp, float* __restrict__ db) {
    __shared__ float red[256];
    const __nv_bfloat16* row = dzt + (size_t)blockIdx.x * Mp;
    float s = 0.0f;
    for (int m = threadIdx.x; m < Mp; m += blockDim.x) s += __bfloat162float(row[m]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) db[blockIdx.x] = red[0];
}

// Adam on one [rows][cols] matrix (or a bias vector with cols = 1 and no copies);
// rows >= valid_rows are kept at zero. Writes the BF16 row-major and transposed copies.
__global__ void mlp_adam_kernel(float* __restrict__ w, float* __restrict__ m1, float* __restrict__ m2,
                                const float* __restrict__ g, int rows, int cols, int valid_rows,
                                const int* __restrict__ step, float lr, float b1, float b2, float eps, float wd,
                                int update, __nv_bfloat16* __restrict__ wb, __nv_bfloat16* __restrict__ wt) {
    const size_t n = (size_t)rows * cols;
    const int t = step ? step[0] + 1 : 1;
    const float bc1 = 1.0f - powf(b1, (float)t), bc2 = 1.0f - powf(b2, (float)t);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / cols), c = (int)(i - (size_t)r * cols);
        float v = w[i];
        if (update) {
            if (r < valid_rows) {
                float gi = g[i];
                if (wd != 0.0f) gi += wd * v;
                const float a = b1 * m1[i] + (1.0f - b1) * gi;
                const float b = b2 * m2[i] + (1.0f - b2) * gi * gi;
                m1[i] = a;
                m2[i] = b;
                v -= lr * (a / bc1) / (sqrtf(b / bc2) + eps);
            } else {
                v = 0.0f;
            }
            w[i] = v;
        }
        if (wb) wb[i] = __float2bfloat16_rn(v);
        if (wt) wt[(size_t)c * rows + r] = __float2bfloat16_rn(v);
    }
}

__global__ void mlp_step_kernel(int* step) {
    if (threadIdx.x == 0) step[0] += 1;
}

// Y f32 [Mp][Op] -> out [M][O]
__global__ void mlp_copy_out_kernel(const float* __restrict__ y, int Op, int M, int O, float* __restrict__ out) {
    const size_t n = (size_t)M * O;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int m = (int)(i / O), j = (int)(i - (size_t)m * O);
        out[i] = y[(size_t)m * Op + j];
    }
}

static unsigned grid_for(size_t n, int threads) {
    size_t b = (n + threads - 1) / threads;
    return (unsigned)std::min<size_t>(std::max<size_t>(b, 1), 148 * 16);
}

static GemmEpi epi_none() {
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    return e;
}

// ---------------------------------------------------------------------------
// host sequences
// ---------------------------------------------------------------------------
static void adam_or_sync(const MlpDims& d, const MlpWs& w, float* weights, float* state, const float* grads,
                         const int* step, const cvqpg_mlp_params* p, int update, cudaStream_t s) {
    const size_t T = d.total;
    float* m1 = state;
    float* m2 = state ? state + T : nullptr;
    struct L {
        size_t off;
        int rows, cols, valid;
        __nv_bfloat16 *wb, *wt;
    } layers[6] = {{d.off_w1, d.Hd, d.D, d.Hd, w.w1b, w.w1t}, {d.off_b1, d.Hd, 1, d.Hd, nullptr, nullptr},
                   {d.off_w2, d.Hd, d.Hd, d.Hd, w.w2b, w.w2t}, {d.off_b2, d.Hd, 1, d.Hd, nullptr, nullptr},
                   {d.off_w3, d.Op, d.Hd, d.O, w.w3b, w.w3t},  {d.off_b3, d.Op, 1, d.O, nullptr, nullptr}};
    for (const L& l : layers) {
        const size_t n = (size_t)l.rows * l.cols;
        mlp_adam_kernel<<<grid_for(n, 256), 256, 0, s>>>(
            weights + l.off, update ? m1 + l.off : nullptr, update ? m2 + l.off : nullptr,
            update ? grads + l.off : nullptr, l.rows, l.cols, l.valid, step, p->lr, p->beta1, p->beta2, p->eps,
            p->weight_decay, update, l.wb, l.wt);
    }
}

static int mlp_forward_impl(const MlpDims& d, const MlpWs& w, const float* weights, const float* X, int* status,
                            cudaStream_t s) {
    dim3 pg(d.D / 32, d.Mp / 32), pb(32, 8);
    mlp_prep_input_kernel<<<pg, pb, 0, s>>>(X, d.M, d.Mp, d.D, w.x0, w.x0t);
    GemmEpi e = epi_none();
    e.mode = CVQPG_GEMM_EPI_BIAS_GELU;
    e.valid_n = d.Hd;
    e.bias = weights + d.off_b1;
    e.out_f32 = w.z1;
    e.ld_f32 = d.Hd;
    e.out_bf16 = w.h1;
    e.ld_bf16 = d.Hd;
    e.out_bf16_t = w.h1t;
    e.ld_t = d.Mp;
    int st = tc_gemm(w.x0, d.D, w.w1b, d.D, d.Mp, d.Hd, d.D, e, 1, status, s);
    if (st) return st;
    e.bias = weights + d.off_b2;
    e.out_f32 = w.z2;
    e.out_bf16 = w.h2;
    e.out_bf16_t = w.h2t;
    st = tc_gemm(w.h1, d.Hd, w.w2b, d.Hd, d.Mp, d.Hd, d.Hd, e, 1, status, s);
    if (st) return st;
    GemmEpi f = epi_none();
    f.mode = CVQPG_GEMM_EPI_BIAS;
    f.bias = weights + d.off_b3;
    f.out_f32 = w.y;
    f.ld_f32 = d.Op;
    f.valid_n = d.Op;
    return tc_gemm(w.h2, d.Hd, w.w3b, d.Hd, d.Mp, d.Op, d.Hd, f, 1, status, s);
}

static int mlp_backward_impl(const MlpDims& d, const MlpWs& w, const float* T, const float* wout, float* grads,
                             float* loss, int* status, cudaStream_t s) {
    mlp_loss_kernel<<<kLossBlocks, 256, 0, s>>>(w.y, d.Op, T, wout, d.M, d.Mp, d.O, d.Op, w.dz3, w.dz3t,
                                                 w.loss_part);
    mlp_loss_finalize_kernel<<<1, 32, 0, s>>>(w.loss_part, kLossBlocks, d.M, loss);
    // data gradients
    GemmEpi e = epi_none();
    e.mode = CVQPG_GEMM_EPI_DGELU;
    e.valid_n = d.Hd;
    e.zin = w.z2;
    e.ld_z = d.Hd;
    e.out_bf16 = w.dz2;
    e.ld_bf16 = d.Hd;
    e.out_bf16_t = w.dz2t;
    e.ld_t = d.Mp;
    int st = tc_gemm(w.dz3, d.Op, w.w3t, d.Op, d.Mp, d.Hd, d.Op, e, 1, status, s);
    if (st) return st;
    e.zin = w.z1;
    e.out_bf16 = nullptr;
    e.out_bf16_t = w.dz1t;
    st = tc_gemm(w.dz2, d.Hd, w.w2t, d.Hd, d.Mp, d.Hd, d.Hd, e, 1, status, s);
    if (st) return st;
    // weight gradients: split-K over the batch into slabs, then a fixed-order sum
    struct G {
        const __nv_bfloat16 *a, *b;
        int rows, cols;
        size_t off;
    } gs[3] = {{w.dz3t, w.h2t, d.Op, d.Hd, d.off_w3}, {w.dz2t, w.h1t, d.Hd, d.Hd, d.off_w2},
               {w.dz1t, w.x0t, d.Hd, d.D, d.off_w1}};
    for (const G& g : gs) {
        GemmEpi f = epi_none();
        f.mode = CVQPG_GEMM_EPI_F32;
        f.out_f32 = w.slabs;
        f.ld_f32 = g.cols;
        f.split_stride = (long long)g.rows * g.cols;
        st = tc_gemm(g.a, d.Mp, g.b, d.Mp, g.rows, g.cols, d.Mp, f, d.splits, status, s);
        if (st) return st;
        const size_t n = (size_t)g.rows * g.cols;
        mlp_reduce_slabs_kernel<<<grid_for(n, 256), 256, 0, s>>>(w.slabs, d.splits, n, n, grads + g.off);
    }
    mlp_bias_grad_kernel<<<d.Op, 256, 0, s>>>(w.dz3t, d.Mp, grads + d.off_b3);
    mlp_bias_grad_kernel<<<d.Hd, 256, 0, s>>>(w.dz2t, d.Mp, grads + d.off_b2);
    mlp_bias_grad_kernel<<<d.Hd, 256, 0, s>>>(w.dz1t, d.Mp, grads + d.off_b1);
    return launch_status();
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

static int mlp_prepare(const cvqpg_mlp_params* p, void* ws, size_t bytes, MlpDims* d, MlpWs* w) {
    int st = mlp_dims(p, d);
    if (st) return st;
    if (!ws) return CVQPG_ERR_ARG;
    if (bytes < mlp_carve(*d, nullptr, w)) return CVQPG_ERR_WORKSPACE;
    mlp_carve(*d, ws, w);
    return CVQPG_OK;
}

extern "C" int cvqpg_mlp_weights_size(const cvqpg_mlp_params* p, size_t* floats) {
    MlpDims d;
    if (!floats) return CVQPG_ERR_ARG;
    const int st = mlp_dims(p, &d);
    if (st) return st;
    *floats = d.total;
    return CVQPG_OK;
}

extern "C" int cvqpg_mlp_workspace_size(const cvqpg_mlp_params* p, size_t* bytes) {
    MlpDims d;
    MlpWs w;
    if (!bytes) return CVQPG_ERR_ARG;
    const int st = mlp_dims(p, &d);
    if (st) return st;
    *bytes = mlp_carve(d, nullptr, &w);
    return CVQPG_OK;
}

extern "C" int cvqpg_mlp_sync_weights(const cvqpg_mlp_params* p, const float* weights, void* ws, size_t bytes,
                                      void* stream) {
    MlpDims d;
    MlpWs w;
    int st = mlp_prepare(p, ws, bytes, &d, &w);
    if (st) return st;
    if (!weights) return CVQPG_ERR_ARG;
    adam_or_sync(d, w, (float*)weights, nullptr, nullptr, nullptr, p, 0, (cudaStream_t)stream);
    return launch_status();
}

extern "C" int cvqpg_mlp_forward(const cvqpg_mlp_params* p, const float* weights, const float* X, float* Y,
                                 void* ws, size_t bytes, int* status, void* stream) {
    MlpDims d;
    MlpWs w;
    int st = mlp_prepare(p, ws, bytes, &d, &w);
    if (st) return st;
    if (!weights || !X || !status) return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    st = mlp_forward_impl(d, w, weights, X, status, s);
    if (st) return st;
    if (Y) mlp_copy_out_kernel<<<grid_for((size_t)d.M * d.O, 256), 256, 0, s>>>(w.y, d.Op, d.M, d.O, Y);
    return launch_status();
}

extern "C" int cvqpg_mlp_gradients(const cvqpg_mlp_params* p, const float* weights, const float* X, const float* T,
                                   const float* out_weight, float* grads, float* loss, void* ws, size_t bytes,
                                   int* status, void* stream) {
    MlpDims d;
    MlpWs w;
    int st = mlp_prepare(p, ws, bytes, &d, &w);
    if (st) return st;
    if (!weights || !X || !T || !out_weight || !grads || !loss || !status) return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    st = mlp_forward_impl(d, w, weights, X, status, s);
    if (st) return st;
    return mlp_backward_impl(d, w, T, out_weight, grads, loss, status, s);
}

extern "C" int cvqpg_mlp_adam_step(const cvqpg_mlp_params* p, float* weights, float* adam_state, int* step,
                                   const float* grads, void* ws, size_t bytes, void* stream) {
    MlpDims d;
    MlpWs w;
    int st = mlp_prepare(p, ws, bytes, &d, &w);
    if (st) return st;
    if (!weights || !adam_state || !step || !grads) return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    adam_or_sync(d, w, weights, adam_state, grads, step, p, 1, s);
    mlp_step_kernel<<<1, 32, 0, s>>>(step);
    return launch_status();
}

extern "C" int cvqpg_mlp_train_step(const cvqpg_mlp_params* p, float* weights, float* adam_state, int* step,
                                    const float* X, const float* T, const float* out_weight, float* loss, void* ws,
                                    size_t bytes, int* status, void* stream) {
    MlpDims d;
    MlpWs w;
    int st = mlp_prepare(p, ws, bytes, &d, &w);
    if (st) return st;
    if (!weights || !adam_state || !step || !X || !T || !out_weight || !loss || !status) return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    st = mlp_forward_impl(d, w, weights, X, status, s);
    if (st) return st;
    st = mlp_backward_impl(d, w, T, out_weight, w.grads, loss, status, s);
    if (st) return st;
    adam_or_sync(d, w, weights, adam_state, w.grads, step, p, 1, s);
    mlp_step_kernel<<<1, 32, 0, s>>>(step);
    return launch_status();
}

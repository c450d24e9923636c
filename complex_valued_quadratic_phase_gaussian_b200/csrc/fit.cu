// The fused fit iteration: every stage of the reference loop body
// (train_2d_gaussian_rgb.py:187-211) as kernels on one stream, with no host
// synchronisation, so that a whole iteration is captured once in a CUDA graph.
#include <cstring>
#include <vector>

#include "blasm.cuh"
#include "loss.cuh"
#include "preprocess.cuh"

namespace cvqpg {

struct FitLayout {
    // constant tables
    void* blasm_tables;
    size_t blasm_tables_bytes;
    double* lr_table;
    float* kvec;        // wavenumbers [C]
    // per-iteration buffers
    float* records;
    int32_t* radii;
    float* radius3;
    BinWorkspace bin;
    int32_t* point_list;
    int32_t* ranges;
    int32_t* pair_count;
    int32_t* tile_order;  // longest-list-first launch order of the splat tiles
    float2* field;      // splat output U [C,H,W]
    float2* vfield;     // V [P,C,H,W]
    float* pred;        // clamp(|V|^2) [P,C,H,W]
    float* gpred;       // dL/dpred [P,C,H,W]
    void* blasm_ws;
    float2* gfield;     // dL/dU [C,H,W]
    float* splat_grads; // SoA (8 + 2C) N
    float* norm_partials;
    float* adan_scalars;  // clip factor and step sizes of the current step
    float* loss_partials;
    float* loss_out;    // 1 + 3P
    size_t total;
};

static int fit_dims(const cvqpg_fit_params* q, cvqpg_blasm_params* bp, cvqpg_loss_params* lp) {
    if (!q) return CVQPG_ERR_ARG;
    if (q->channels != 1 && q->channels != 3) return CVQPG_ERR_CHANNELS;
    const int cull = q->cull_mode & ~CVQPG_PHASE_ISO;
    if (q->num_gaussians < 0 || q->pair_capacity < 0 || cull < 0 || cull > 2) return CVQPG_ERR_ARG;
    if (q->curv_mode < 0 || q->curv_mode > 2 || q->history_len < 1) return CVQPG_ERR_ARG;
    std::memset(bp, 0, sizeof(*bp));
    bp->channels = q->channels;
    bp->planes = q->planes;
    bp->height = q->height;
    bp->width = q->width;
    bp->pad_height = q->pad_height;
    bp->pad_width = q->pad_width;
    bp->input_mode = 0;
    bp->pixel_pitch = q->pixel_pitch;
    for (int i = 0; i < 3; i++) bp->wavelengths[i] = q->wavelengths[i];
    for (int i = 0; i < 8; i++) bp->distances[i] = q->distances[i];
    bp->aperture_radius = q->aperture_radius;
    bp->plan_hint = q->plan_hint;
    std::memset(lp, 0, sizeof(*lp));
    lp->channels = q->channels;
    lp->planes = q->planes;
    lp->height = q->height;
    lp->width = q->width;
    lp->w_l2 = q->loss_weights[0];
    lp->w_mask = q->loss_weights[1];
    lp->w_cor = q->loss_weights[2];
    lp->ssim_weight = q->ssim_weight;
    lp->noise_ratio = q->noise_ratio;
    lp->inject_noise = q->inject_noise;
    lp->seed = q->seed;
    lp->target_moments = q->target_moments;
    return CVQPG_OK;
}

static int fit_layout(const cvqpg_fit_params* q, void* base, size_t cap, FitLayout* L, BlasmDev* bd, LossDev* ld) {
    cvqpg_blasm_params bp;
    cvqpg_loss_params lp;
    int st = fit_dims(q, &bp, &lp);
    if (st != CVQPG_OK) return st;
    size_t tbytes = 0;
    st = cvqpg_blasm_tables_size(&bp, &tbytes);
    if (st != CVQPG_OK) return st;
    st = loss_make_dev(&lp, ld);
    if (st != CVQPG_OK) return st;
    const int N = q->num_gaussians, C = q->channels, P = q->planes, H = q->height, W = q->width;
    const BinRule rule = make_bin_rule(q->cull_mode & ~CVQPG_PHASE_ISO, W, H, nullptr, nullptr);
    Carver cv(base, cap);
    L->blasm_tables = cv.take<char>(tbytes);
    L->blasm_tables_bytes = tbytes;
    L->lr_table = cv.take<double>(q->num_iters > 0 ? q->num_iters : 1);
    L->kvec = cv.take<float>(4);
    const int n1 = N > 0 ? N : 1;
    L->records = cv.take<float>((size_t)n1 * kRecordFloats);
    L->radii = cv.take<int32_t>(n1);
    L->radius3 = cv.take<float>(n1);
    L->bin = carve_bin_workspace(cv, N, q->pair_capacity);
    L->point_list = cv.take<int32_t>(q->pair_capacity > 0 ? q->pair_capacity : 1);
    L->ranges = cv.take<int32_t>((size_t)2 * bin_rule_lists(rule));
    L->pair_count = cv.take<int32_t>(2);
    L->tile_order = cv.take<int32_t>((size_t)((W + kTile - 1) / kTile) * ((H + kTile - 1) / kTile));
    L->field = cv.take<float2>((size_t)C * H * W);
    L->vfield = cv.take<float2>((size_t)P * C * H * W);
    L->pred = cv.take<float>((size_t)P * C * H * W);
    L->gpred = cv.take<float>((size_t)P * C * H * W);
    // BLASM device config (needs the table pointer)
    st = blasm_make_dev(&bp, base ? L->blasm_tables : (const void*)"", base ? tbytes : (size_t)-1, bd);
    if (st != CVQPG_OK) return st;
    L->blasm_ws = cv.take<char>(blasm_workspace_bytes(*bd));
    L->gfield = cv.take<float2>((size_t)C * H * W);
    L->splat_grads = cv.take<float>((size_t)(8 + 2 * C) * n1);
    L->norm_partials = cv.take<float>(preprocess_backward_blocks(N));
    L->adan_scalars = cv.take<float>(kAdanScalars);
    L->loss_partials = cv.take<float>(loss_partials_floats(*ld));
    L->loss_out = cv.take<float>(1 + 3 * P);
    L->total = cv.off + 256;
    if (base && !cv.fits()) return CVQPG_ERR_WORKSPACE;
    return CVQPG_OK;
}

static PreDev make_pre(const cvqpg_fit_params* q) {
    PreDev P;
    P.n = q->num_gaussians;
    P.W = q->width;
    P.H = q->height;
    P.curv_mode = q->curv_mode;
    P.curv_const = (float)q->curv_const;
    double lam = q->wavelengths[0];
    if (q->channels == 3)
        for (int c = 1; c < 3; c++) lam = q->wavelengths[c] < lam ? q->wavelengths[c] : lam;
    P.eta_lambda = (float)(q->curv_nyquist * lam);
    P.dxy_sq = (float)(q->pixel_pitch * q->pixel_pitch);
    P.curv_trainable = q->curv_trainable;
    P.curv_warmup = q->curv_trainable ? q->warmup_iters : 0;
    return P;
}

struct FlatViews {
    RawParams raw;
    RawGrads grads;
    float* t_param[kParamTensors];
    float* t_grad[kParamTensors];
    int numel[kParamTensors];
};

static FlatViews flat_views(const cvqpg_fit_params* q, float* params, float* grads) {
    const int N = q->num_gaussians, C = q->channels;
    const int numel[kParamTensors] = {2 * N, 2 * N, N, C * N, C * N, N, N};
    FlatViews v;
    size_t off = 0;
    for (int t = 0; t < kParamTensors; t++) {
        v.numel[t] = numel[t];
        v.t_param[t] = params ? params + off : nullptr;
        v.t_grad[t] = grads ? grads + off : nullptr;
        off += numel[t];
    }
    v.raw = RawParams{v.t_param[0], v.t_param[1], v.t_param[2], v.t_param[3], v.t_param[4], v.t_param[5],
                      v.t_param[6]};
    v.grads = RawGrads{v.t_grad[0], v.t_grad[1], v.t_grad[2], v.t_grad[3], v.t_grad[4], v.t_grad[5], v.t_grad[6]};
    return v;
}

__global__ void record_step_kernel(const float* __restrict__ loss_out, int nvals, const int32_t* __restrict__ pair_count,
                                   float* __restrict__ history, int history_len, int32_t* __restrict__ status,
                                   int32_t* __restrict__ iteration, int advance) {
    const int it = iteration ? iteration[0] : 0;
    if (history) {
        float* dst = history + (size_t)(it % history_len) * nvals;
        for (int i = threadIdx.x; i < nvals; i += blockDim.x) dst[i] = loss_out[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (status) {
            // bit 0: the tile pairs overflowed the capacity; bit 1: the loss was not finite (a
            // NaN/Inf parameter or target; nan_to_num zeroes the gradients as the reference does)
            const int bits = (pair_count[1] ? 1 : 0) | (nvals > 0 && !isfinite(loss_out[0]) ? 2 : 0);
            if (bits) atomicOr(status, bits);
        }
        // an overflowed step applied no update (AdanDev::skip): the counter stays, so the host
        // can enlarge the pair capacity and run the same iteration again
        if (advance && iteration && !pair_count[1]) iteration[0] = it + 1;
    }
}

// forward half shared by step and evaluate
static void run_forward(const cvqpg_fit_params* q, const FitLayout& L, const BlasmDev& bd, const LossDev& ld,
                        const RawParams& raw, const float* targets, const uint8_t* depth_plane,
                        const float* target_range, const int32_t* iteration, cudaStream_t s,
                        StageMarks* marks = nullptr) {
    const int C = q->channels;
    const PreDev P = make_pre(q);
    const BinRule rule = make_bin_rule(q->cull_mode & ~CVQPG_PHASE_ISO, q->width, q->height, L.radii, L.radius3);
    if (marks) marks->mark(s);
    launch_preprocess_forward(C, P, raw, L.records, L.radii, L.radius3, L.bin.tiles_touched, rule, s);
    if (marks) marks->mark(s);
    launch_binning(rule, L.records, L.bin, L.point_list, L.ranges, L.pair_count, s);
    launch_tile_order(rule, L.ranges, L.tile_order, s);
    if (marks) marks->mark(s);
    const float dxy2 = (float)(q->pixel_pitch * q->pixel_pitch);
    launch_splat_forward(C, rule, L.ranges, L.point_list, L.records, L.kvec, dxy2, L.field, s,
                         (q->cull_mode & CVQPG_PHASE_ISO) != 0, L.tile_order);
    if (marks) marks->mark(s);
    blasm_forward(bd, L.field, L.vfield, L.pred, L.blasm_ws, s, marks);
    launch_loss(ld, L.pred, targets, depth_plane, target_range, iteration, L.gpred, L.loss_partials, L.loss_out, s);
    if (marks) marks->mark(s);
}

}  // namespace cvqpg

using namespace cvqpg;

extern "C" int cvqpg_fit_workspace_size(const cvqpg_fit_params* q, size_t* bytes) {
    if (!bytes) return CVQPG_ERR_ARG;
    FitLayout L;
    BlasmDev bd;
    LossDev ld;
    const int st = fit_layout(q, nullptr, 0, &L, &bd, &ld);
    if (st != CVQPG_OK) return st;
    *bytes = L.total;
    return CVQPG_OK;
}

extern "C" int cvqpg_fit_setup(const cvqpg_fit_params* q, const double* lr_table, void* workspace, size_t bytes) {
    FitLayout L;
    BlasmDev bd;
    LossDev ld;
    if (!workspace) return CVQPG_ERR_ARG;
    int st = fit_layout(q, workspace, bytes, &L, &bd, &ld);
    if (st != CVQPG_OK) return st;
    cvqpg_blasm_params bp;
    cvqpg_loss_params lp;
    fit_dims(q, &bp, &lp);
    st = cvqpg_blasm_setup(&bp, L.blasm_tables, L.blasm_tables_bytes);
    if (st != CVQPG_OK) return st;
    const int n = q->num_iters > 0 ? q->num_iters : 1;
    std::vector<double> t(n, q->lr[0]);
    if (lr_table)
        for (int i = 0; i < q->num_iters; i++) t[i] = lr_table[i];
    if (cudaMemcpy(L.lr_table, t.data(), sizeof(double) * n, cudaMemcpyHostToDevice) != cudaSuccess)
        return CVQPG_ERR_CUDA;
    // k = 2 pi / lambda as the reference computes it: float32 tensor op (model_2d_gaussian_rgb.py:379)
    float k[4] = {0.f, 0.f, 0.f, 0.f};
    for (int c = 0; c < q->channels; c++) k[c] = (float)6.283185307179586 / (float)q->wavelengths[c];
    if (cudaMemcpy(L.kvec, k, sizeof(k), cudaMemcpyHostToDevice) != cudaSuccess) return CVQPG_ERR_CUDA;
    return CVQPG_OK;
}

static int fit_prepare(const cvqpg_fit_params* q, void* workspace, size_t bytes, FitLayout* L, BlasmDev* bd,
                       LossDev* ld) {
    if (!workspace) return CVQPG_ERR_ARG;
    return fit_layout(q, workspace, bytes, L, bd, ld);
}

static int fit_step_impl(const cvqpg_fit_params* q, float* params, float* grads, float* adan_state,
                         const float* targets, const uint8_t* depth_plane, const float* target_range,
                         int32_t* iteration, float* history, int32_t* status, void* workspace, size_t bytes,
                         void* stream_, StageMarks* marks) {
    FitLayout L;
    BlasmDev bd;
    LossDev ld;
    int st = fit_prepare(q, workspace, bytes, &L, &bd, &ld);
    if (st != CVQPG_OK) return st;
    if (!params || !grads || !adan_state || !targets || !depth_plane || !target_range || !iteration)
        return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream_;
    const int N = q->num_gaussians, C = q->channels, P = q->planes;
    FlatViews fv = flat_views(q, params, grads);
    // forward: render, propagate, loss (+ dL/dpred)
    run_forward(q, L, bd, ld, fv.raw, targets, depth_plane, target_range, iteration, s, marks);
    record_step_kernel<<<1, 64, 0, s>>>(L.loss_out, 1 + 3 * P, L.pair_count, history, q->history_len, status,
                                        iteration, 0);
    // adjoint of the propagation (dL/dpred -> dL/dU)
    blasm_backward(bd, L.field, nullptr, L.gpred, L.vfield, L.gfield, L.blasm_ws, s, marks);
    // splat adjoint
    cudaMemsetAsync(L.splat_grads, 0, sizeof(float) * (size_t)(8 + 2 * C) * (N > 0 ? N : 1), s);
    float* sg = L.splat_grads;
    SplatGrads out{sg, sg + 2 * N, sg + 5 * N, sg + (5 + C) * N, sg + (5 + 2 * C) * N, sg + (6 + 2 * C) * N,
                   sg + (7 + 2 * C) * N};
    const BinRule rule = make_bin_rule(q->cull_mode & ~CVQPG_PHASE_ISO, q->width, q->height, L.radii, L.radius3);
    const float dxy2 = (float)(q->pixel_pitch * q->pixel_pitch);
    launch_splat_backward(C, rule, L.ranges, L.point_list, L.records, L.kvec, dxy2, L.gfield, out, s,
                          (q->cull_mode & CVQPG_PHASE_ISO) != 0, L.tile_order);
    if (marks) marks->mark(s);
    // preprocessing adjoint + nan_to_num + norm partials
    SplatGradsIn gin{out.d_means, out.d_inv, out.d_col, out.d_ph, out.d_op, out.d_cv, out.d_ar};
    launch_preprocess_backward(C, make_pre(q), fv.raw, gin, fv.grads, iteration, L.norm_partials, s);
    if (marks) marks->mark(s);
    // clip + Adan
    AdanDev A;
    std::memset(&A, 0, sizeof(A));
    const size_t total = (size_t)(7 + 2 * C) * N;
    static const int kGroup[kParamTensors] = {0, 1, 4, 2, 2, 3, 5};
    size_t off = 0;
    for (int t = 0; t < kParamTensors; t++) {
        A.param[t] = fv.t_param[t];
        A.grad[t] = fv.t_grad[t];
        A.exp_avg[t] = adan_state + off;
        A.exp_avg_sq[t] = adan_state + total + off;
        A.exp_avg_diff[t] = adan_state + 2 * total + off;
        A.neg_pre_grad[t] = adan_state + 3 * total + off;
        A.numel[t] = fv.numel[t];
        A.group[t] = kGroup[t];
        A.first_iter[t] = 0;
        A.frozen_always[t] = 0;
        off += fv.numel[t];
    }
    A.first_iter[6] = q->curv_trainable ? q->warmup_iters : 0;
    A.frozen_always[6] = q->curv_trainable ? 0 : 1;
    for (int g = 0; g < 6; g++) A.lr[g] = q->lr[g];
    A.lr_table = L.lr_table;
    A.lr_table_len = q->num_iters > 0 ? q->num_iters : 1;
    A.beta1 = q->betas[0];
    A.beta2 = q->betas[1];
    A.beta3 = q->betas[2];
    A.eps = q->eps;
    A.weight_decay = q->weight_decay;
    A.no_prox = q->no_prox;
    A.max_grad_norm = q->max_grad_norm;
    A.norm_partials = L.norm_partials;
    A.num_partials = preprocess_backward_blocks(N);
    A.scalars = L.adan_scalars;
    A.skip = L.pair_count + 1;
    if (N > 0) launch_adan(A, iteration, s);
    if (marks) marks->mark(s);
    record_step_kernel<<<1, 32, 0, s>>>(L.loss_out, 0, L.pair_count, nullptr, 1, nullptr, iteration, 1);
    return launch_status();
}

extern "C" int cvqpg_fit_step(const cvqpg_fit_params* q, float* params, float* grads, float* adan_state,
                              const float* targets, const uint8_t* depth_plane, const float* target_range,
                              int32_t* iteration, float* history, int32_t* status, void* workspace, size_t bytes,
                              void* stream) {
    return fit_step_impl(q, params, grads, adan_state, targets, depth_plane, target_range, iteration, history, status,
                         workspace, bytes, stream, nullptr);
}

extern "C" int cvqpg_fit_step_timed(const cvqpg_fit_params* q, float* params, float* grads, float* adan_state,
                                    const float* targets, const uint8_t* depth_plane, const float* target_range,
                                    int32_t* iteration, float* history, int32_t* status, void* workspace,
                                    size_t bytes, void* stream, void** stage_events, int num_events) {
    StageMarks m;
    m.ev = (cudaEvent_t*)stage_events;
    m.n = num_events;
    return fit_step_impl(q, params, grads, adan_state, targets, depth_plane, target_range, iteration, history, status,
                         workspace, bytes, stream, &m);
}

extern "C" int cvqpg_fit_pair_count(const cvqpg_fit_params* q, const void* workspace, size_t bytes,
                                    int32_t* out_device, void* stream) {
    FitLayout L;
    BlasmDev bd;
    LossDev ld;
    if (!out_device) return CVQPG_ERR_ARG;
    const int st = fit_prepare(q, const_cast<void*>(workspace), bytes, &L, &bd, &ld);
    if (st != CVQPG_OK) return st;
    if (cudaMemcpyAsync(out_device, L.pair_count, 2 * sizeof(int32_t), cudaMemcpyDeviceToDevice,
                        (cudaStream_t)stream) != cudaSuccess)
        return CVQPG_ERR_CUDA;
    return CVQPG_OK;
}

extern "C" int cvqpg_fit_evaluate(const cvqpg_fit_params* q, const float* params, const float* targets,
                                  const uint8_t* depth_plane, const float* target_range, float* out,
                                  float* field_out, float* planes_out, int32_t* status, void* workspace,
                                  size_t bytes, void* stream_) {
    cvqpg_fit_params qq = *q;
    qq.inject_noise = 0;
    FitLayout L;
    BlasmDev bd;
    LossDev ld;
    int st = fit_prepare(&qq, workspace, bytes, &L, &bd, &ld);
    if (st != CVQPG_OK) return st;
    if (!params || !targets || !depth_plane || !target_range || !out) return CVQPG_ERR_ARG;
    cudaStream_t s = (cudaStream_t)stream_;
    FlatViews fv = flat_views(&qq, const_cast<float*>(params), nullptr);
    run_forward(&qq, L, bd, ld, fv.raw, targets, depth_plane, target_range, nullptr, s);
    const int P = qq.planes, C = qq.channels, H = qq.height, W = qq.width;
    cudaMemcpyAsync(out, L.loss_out, sizeof(float) * (1 + 3 * P), cudaMemcpyDeviceToDevice, s);
    if (field_out)
        cudaMemcpyAsync(field_out, L.field, sizeof(float2) * (size_t)C * H * W, cudaMemcpyDeviceToDevice, s);
    if (planes_out)
        cudaMemcpyAsync(planes_out, L.vfield, sizeof(float2) * (size_t)P * C * H * W, cudaMemcpyDeviceToDevice, s);
    record_step_kernel<<<1, 32, 0, s>>>(L.loss_out, 0, L.pair_count, nullptr, 1, status, nullptr, 0);
    return launch_status();
}

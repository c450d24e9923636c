/*
 * cvqpg.h - C ABI of the B200 (sm_100a) CVQPG hologram-fitting kernels.
 *
 * Every entry point takes plain device pointers, sizes and a CUDA stream
 * (passed as void*, a cudaStream_t; NULL = legacy default stream), enqueues its
 * kernels on that stream and returns a status code (CVQPG_OK = 0). Nothing in
 * this header allocates device memory: scratch space is a caller-provided
 * workspace whose size is reported by the matching *_workspace_size query.
 * No entry point synchronises the host, so every one of them can be recorded
 * into a CUDA graph.
 *
 * Layouts (all little-endian, C-contiguous):
 *   complex fields  float2 (re, im) interleaved = torch.complex64 storage
 *   per-Gaussian    SoA rows exactly as the reference tensors ([N,2], [N,3], [N,C], [N])
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   cuda/raster.cu:30-105   qpf_render_forward   -> cvqpg_render_forward
 *   cuda/raster.cu:107-143  qpf_render_backward  -> cvqpg_render_backward
 *   cuda/qpf_rasterizer.h:30-57 (declarations of the two above)
 */
#ifndef CVQPG_H_
#define CVQPG_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CVQPG_API __attribute__((visibility("default")))
#else
#define CVQPG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
#define CVQPG_OK 0
#define CVQPG_ERR_ARG 1        /* invalid argument (null pointer, bad size)          */
#define CVQPG_ERR_CHANNELS 2   /* channel count not 1 or 3 (cuda/forward.cu:173)     */
#define CVQPG_ERR_WORKSPACE 3  /* workspace smaller than the size query reported     */
#define CVQPG_ERR_CUDA 4       /* a kernel launch failed (cudaGetLastError)          */
#define CVQPG_ERR_UNSUPPORTED 5 /* size/shape outside what the kernels were built for */

/* ---- culling rules (which Gaussians enter which tile list) --------------- */
#define CVQPG_CULL_CUDA16_5SIGMA 0  /* reference CUDA renderer: 16-px tiles, int radius rect */
#define CVQPG_CULL_TORCH64_3SIGMA 1 /* reference torch renderer: 64-px tiles, 3-sigma circle */
#define CVQPG_CULL_NONE 2           /* every Gaussian at every pixel                          */
/* OR-ed into a cull mode: the isotropic quadratic phase 0.5*c*|r-mu|^2*dxy2 of the
 * torch renderer's --phase_iso (model_2d_gaussian_rgb.py:356-359) instead of the
 * Mahalanobis form 0.5*c*m*area*dxy2 (:360-363); the reference CUDA renderer
 * rejects --phase_iso (model_2d_gaussian_rgb.py:263-265), this one supports it. */
#define CVQPG_PHASE_ISO 0x100

/* Human-readable text of a status code. */
CVQPG_API const char* cvqpg_status_string(int status);

/* Library version as 10000*major + 100*minor + patch. */
CVQPG_API int cvqpg_version(void);

/* ---- drop-in rasterizer ---------------------------------------------------
 *
 * cvqpg_render_forward replaces qpf_render_forward (cuda/raster.cu:30-105,
 * declared at cuda/qpf_rasterizer.h:30-41). Same inputs and meaning:
 *   means_2d [N,2] pixel coords, inv_cov [N,3] (inv00, inv01, inv11),
 *   colours [N,C], phase [N,C], opacities [N], curvature [N], area [N] = |sx*sy|,
 *   radii [N] int32 culling radius in px, k [C] wavenumbers, dxy2 = pitch^2.
 * Outputs:
 *   out_field  [C,H,W] complex64, fully written (no pre-zeroing needed)
 *   point_list [pair_capacity] int32, Gaussian ids sorted by (tile, id)
 *   ranges     [T,2] int32, T = ceil(W/16)*ceil(H/16), [start,end) per tile
 *   pair_count [2] int32 (device): [0] = pairs required (the reference's
 *              total_pairs), [1] = 1 if that exceeded pair_capacity (then only
 *              the first pair_capacity pairs were binned, the field is
 *              incomplete and the caller must retry with a larger capacity)
 * The tile lists are bit-identical to the reference's 64-bit (tile<<32 | id)
 * CUB sort: the pairs are generated in id order and a stable LSD radix sort on
 * the tile bits keeps that order inside each tile.
 * Errors: CVQPG_ERR_CHANNELS for C not in {1,3} (cuda/forward.cu:173),
 * CVQPG_ERR_ARG for null pointers / negative sizes (cuda/raster.cu:22-28).
 */
CVQPG_API int cvqpg_render_workspace_size(int n, int width, int height, int pair_capacity, size_t* bytes);

CVQPG_API int cvqpg_render_forward(const float* means_2d, const float* inv_cov, const float* colours,
                         const float* phase, const float* opacities, const float* curvature,
                         const float* area, const int32_t* radii, const float* k, float dxy2,
                         int n, int width, int height, int channels,
                         float* out_field, int32_t* point_list, int pair_capacity, int32_t* ranges,
                         int32_t* pair_count, void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free render forward. No counterpart in the reference: the
 * reference allocates its scratch with torch on every call.
 * Same inputs, outputs and status codes as cvqpg_render_forward, without the
 * workspace argument, for callers that cannot allocate device memory where
 * they render (a host that owns every allocation and passes only its own
 * buffers, a process running under a fixed device-memory budget, or code that
 * must not call cudaMalloc because it would synchronise the device). The
 * scratch is a fixed device array inside the library (about 5.5 MiB, held by
 * every GPU that loads the library until exit), so:
 *   - n <= 16384 Gaussians and pair_capacity <= 262144, else CVQPG_ERR_UNSUPPORTED;
 *   - the first call on a device looks the array up (cudaGetSymbolAddress) for
 *     the device that is current; make that first call before any stream capture;
 *   - all calls share the array: calls that can overlap on the GPU (different
 *     streams, or different host threads) race and must be serialised;
 *   - nothing in the array needs clearing between calls (every buffer is
 *     written before it is read);
 *   - the looked-up address is kept for the life of the process: do not call
 *     this entry point on a device after cudaDeviceReset on it.
 * It calls no cudaMalloc, cudaFree or allocating library routine. */
CVQPG_API int cvqpg_render_forward_noalloc(const float* means_2d, const float* inv_cov, const float* colours,
                                           const float* phase, const float* opacities, const float* curvature,
                                           const float* area, const int32_t* radii, const float* k, float dxy2,
                                           int n, int width, int height, int channels,
                                           float* out_field, int32_t* point_list, int pair_capacity,
                                           int32_t* ranges, int32_t* pair_count, void* stream);

/* Number of tile lists (rows of `ranges`) a culling rule produces. */
CVQPG_API int cvqpg_render_num_lists(int cull_mode, int width, int height);

/* Forward with an explicit culling rule, so that each parity check compares
 * like with like: CVQPG_CULL_CUDA16_5SIGMA uses `radii` (as
 * cvqpg_render_forward), CVQPG_CULL_TORCH64_3SIGMA uses `radius3` = the
 * torch renderer's float 3-sigma radius (model_2d_gaussian_rgb.py:400-403)
 * and 64-px lists (model_2d_gaussian_rgb.py:311-314), CVQPG_CULL_NONE sums
 * every Gaussian at every pixel (cuda/rasterizer.py:74-91). `ranges` has
 * cvqpg_render_num_lists(cull_mode, W, H) rows.
 */
CVQPG_API int cvqpg_render_forward_cull(const float* means_2d, const float* inv_cov, const float* colours,
                                        const float* phase, const float* opacities, const float* curvature,
                                        const float* area, int cull_mode, const int32_t* radii,
                                        const float* radius3, const float* k, float dxy2, int n, int width,
                                        int height, int channels, float* out_field, int32_t* point_list,
                                        int pair_capacity, int32_t* ranges, int32_t* pair_count,
                                        void* workspace, size_t workspace_bytes, void* stream);

/* cvqpg_render_backward replaces qpf_render_backward (cuda/raster.cu:107-143,
 * declared at cuda/qpf_rasterizer.h:43-57). grad_field is dL/d(field) as a
 * complex64 [C,H,W] tensor (real part = dL/dRe, imaginary part = dL/dIm, the
 * torch convention). point_list/ranges come from the forward.
 * Outputs (overwritten, not accumulated): d_means [N,2], d_inv_cov [N,3],
 * d_colours [N,C], d_phase [N,C], d_opacities [N], d_curvature [N], d_area [N].
 * The workspace (size from cvqpg_render_backward_workspace_size) holds the
 * packed per-Gaussian records.
 */
CVQPG_API int cvqpg_render_backward_workspace_size(int n, size_t* bytes);

CVQPG_API int cvqpg_render_backward(const float* grad_field, const float* means_2d, const float* inv_cov,
                          const float* colours, const float* phase, const float* opacities,
                          const float* curvature, const float* area, const float* k,
                          const int32_t* point_list, const int32_t* ranges, float dxy2,
                          int n, int width, int height, int channels,
                          float* d_means, float* d_inv_cov, float* d_colours, float* d_phase,
                          float* d_opacities, float* d_curvature, float* d_area,
                          void* workspace, size_t workspace_bytes, void* stream);

/* Backward matching cvqpg_render_forward_cull (same cull_mode, lists, ranges). */
CVQPG_API int cvqpg_render_backward_cull(const float* grad_field, const float* means_2d, const float* inv_cov,
                                         const float* colours, const float* phase, const float* opacities,
                                         const float* curvature, const float* area, const float* k,
                                         int cull_mode, const int32_t* point_list, const int32_t* ranges,
                                         float dxy2, int n, int width, int height, int channels,
                                         float* d_means, float* d_inv_cov, float* d_colours, float* d_phase,
                                         float* d_opacities, float* d_curvature, float* d_area,
                                         void* workspace, size_t workspace_bytes, void* stream);

/* ---- band-limited angular-spectrum propagation (BLASM) --------------------
 *
 * Replaces, for one hologram, the reference chain
 *   soft_window_pad                (model_2d_gaussian_rgb.py:186-241)
 *   angle % 2pi, clamp(|U|, 0, 1)  (train_2d_gaussian_rgb.py:89-95)
 *   propagator._reconstruct_impl   (utils/propagator.py:248-290; custom() :41-64;
 *                                   transfer functions :202-222, aperture :179-200)
 *   crop_center to the image       (train_2d_gaussian_rgb.py:193)
 * with every plane and wavelength in one sequence of three kernels:
 *   rows   : pad/window/clamp + forward FFT of the pH nonzero rows (length 2pW)
 *   columns: forward FFT (length 2pH) once, then per plane the transfer-function
 *            multiply (computed on the fly) and the inverse FFT, keeping only
 *            the output rows
 *   rows   : inverse FFT of the kept rows, keeping only the output columns.
 * Output: the complex field V [P, C, out_h, out_w] (the reference intensity is
 * |V|^2). The adjoint applies the same kernels with the conjugate transfer
 * function, summed over planes.
 *
 * input_mode 0: input = splat field [C, H, W] (complex64); the kernel applies
 *               the replicate guard band, Tukey window and amplitude clamp.
 *               The adjoint returns dL/d(splat field) [C, H, W] (the guard band
 *               carries no gradient, as in the reference).
 * input_mode 1: input = already-padded complex field [C, pH, pW]; the adjoint
 *               returns dL/d(input) [C, pH, pW].
 * Requirements: even H, W, pH, pW with pH >= H, pW >= W; 2pH and 2pW products
 * of primes <= 17; planes <= 8; channels 1 or 3.
 */
/* plan_hint: which FFT plan the propagation uses (the autotuner's knob; no
 * reference counterpart, cuFFT picks its own plans). 0 everywhere = defaults.
 *   bits [0,5)  radix kept in registers by the column kernels (0 = automatic);
 *   bits [5,8)  radix order of the column FFTs, bits [8,11) of the row FFTs:
 *               0 radix 16 first then 8/4/2 then odd, 1 odd first then 16/8/4/2,
 *               2 radix 8 first then 4/2 then odd, 3 odd first then 8/4/2;
 *   bit 11      one column per CTA in the column kernels (CVQPG_PLAN_COLS1)
 *               instead of four adjacent columns where the grid has a four-
 *               column kernel (column length 16 x 11 x 16 = 2816). */
#define CVQPG_PLAN_HINT(col_radix, col_order, row_order) \
    ((col_radix) | ((col_order) << 5) | ((row_order) << 8))
#define CVQPG_PLAN_COLS1 (1 << 11)

typedef struct cvqpg_blasm_params {
    int channels;
    int planes;
    int height, width;          /* image H, W                                  */
    int pad_height, pad_width;  /* pH, pW (the reference pad_size)             */
    int out_height, out_width;  /* output crop; 0 = (H, W)                     */
    int input_mode;             /* 0 or 1, see above                           */
    int plan_hint;              /* FFT plan choice, 0 = default (CVQPG_PLAN_*)  */
    double pixel_pitch;         /* metres                                      */
    double wavelengths[3];      /* metres, one per channel                     */
    double distances[8];        /* metres, one per plane                       */
    double aperture_radius;     /* Fourier aperture radius on the 2x grid (px);
                                   <= 0 disables it                            */
} cvqpg_blasm_params;

/* Device table blob (twiddles, windows, frequency tables, band limits):
 * size query, then a synchronous host-side fill of a caller buffer. */
CVQPG_API int cvqpg_blasm_tables_size(const cvqpg_blasm_params* prm, size_t* bytes);
CVQPG_API int cvqpg_blasm_setup(const cvqpg_blasm_params* prm, void* tables, size_t table_bytes);
CVQPG_API int cvqpg_blasm_workspace_size(const cvqpg_blasm_params* prm, size_t* bytes);
CVQPG_API int cvqpg_blasm_forward(const cvqpg_blasm_params* prm, const void* tables, size_t table_bytes,
                                  const float* input, float* out_field, void* workspace,
                                  size_t workspace_bytes, void* stream);
CVQPG_API int cvqpg_blasm_backward(const cvqpg_blasm_params* prm, const void* tables, size_t table_bytes,
                                   const float* input, const float* grad_out, float* grad_input,
                                   void* workspace, size_t workspace_bytes, void* stream);

/* ---- fused multi-plane loss ---------------------------------------------
 *
 * Replaces, per plane p of the fit loop (train_2d_gaussian_rgb.py:192-199),
 *   multiplane_loss_odak.__call__(pred, target, p, inject_noise=True)
 *                                       (utils/propagator.py:417-449)
 *   + GaussianLoss(pred, target)        (utils/data_utils.py:22-41)
 * for all planes in one launch, with pred = clamp(|V_p|^2, 0, 1):
 *   L = sum_p  w_l2 mean((pred-T)^2) + w_mask mean((pred M - N M)^2)
 *            + w_cor mean((pred N - N N)^2) + ssim_weight (1 - SSIM(pred, T))
 * M = [depth_plane == p]; N = T + (z * noise_ratio) * target_range[p] with a
 * fresh standard normal z per element and iteration (Philox4x32-10 keyed by
 * `seed`, counter = (element, *iteration)); SSIM with the pytorch_msssim
 * defaults (11-tap Gaussian, sigma 1.5, K = 0.01/0.03, data range 1, valid).
 * Writes grad_pred = dL/dpred [P,C,H,W] and out[1 + 3P]:
 *   out[0] loss, out[1+p] MSE(pred_p, T_p) (PSNR = -10 log10 MSE),
 *   out[1+P+p] SSIM_p, out[1+2P+p] loss of plane p.
 */
typedef struct cvqpg_loss_params {
    int channels;
    int planes;
    int height, width;
    float w_l2, w_mask, w_cor;  /* reference weights [1, 1, 1] (utils/data_utils.py:75) */
    float ssim_weight;          /* reference 0.025 * 0.2 = 0.005 (utils/data_utils.py:22-41) */
    float noise_ratio;          /* reference 1e-3 (utils/propagator.py:417) */
    int inject_noise;           /* 1 in the fit loop (train_2d_gaussian_rgb.py:195) */
    unsigned long long seed;
    /* Optional: SSIM moments of these targets from cvqpg_loss_target_moments, or NULL
     * to filter the targets on every call. The targets are constant during a fit,
     * so precomputing them leaves three of the five windowed moments per call. */
    const float* target_moments;
} cvqpg_loss_params;

CVQPG_API int cvqpg_loss_workspace_size(const cvqpg_loss_params* prm, size_t* bytes);
/* target_range[p] = max(T_p) - min(T_p), once per fit (targets are constant).
 * workspace: at least planes * CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE bytes
 * (the cvqpg_loss_workspace_size workspace of the same planes is enough). */
#define CVQPG_TARGET_RANGE_WORKSPACE_PER_PLANE 512
CVQPG_API int cvqpg_loss_target_range(const float* targets, int planes, int channels, int height, int width,
                                      float* target_range, void* workspace, size_t workspace_bytes, void* stream);
/* Windowed SSIM moments of the targets (same 11-tap window as the loss):
 * float2 (mu_T, E_w[T^2]) per valid map position, [P*C][H-10][W-10]. Summed in the
 * loss kernel's order, so the loss gives the same result with or without them. */
CVQPG_API int cvqpg_loss_target_moments_size(const cvqpg_loss_params* prm, size_t* bytes);
CVQPG_API int cvqpg_loss_target_moments(const cvqpg_loss_params* prm, const float* targets, float* moments,
                                        size_t moments_bytes, void* stream);
CVQPG_API int cvqpg_loss_forward_backward(const cvqpg_loss_params* prm, const float* pred, const float* targets,
                                          const uint8_t* depth_plane, const float* target_range,
                                          const int32_t* iteration, float* grad_pred, float* out,
                                          void* workspace, size_t workspace_bytes, void* stream);

/* ---- fused fit iteration ---------------------------------------------------
 *
 * One call = one iteration of the reference fit loop body
 * (train_2d_gaussian_rgb.py:187-211): render (preprocess, bin, splat) ->
 * pad/clamp + BLASM to every plane -> multi-plane loss + SSIM -> adjoint of
 * all of it -> nan_to_num -> clip_grad_norm_(max_grad_norm) -> Adan step,
 * plus the means cosine schedule and the curvature warm-up. Every stage is a
 * kernel on `stream`; nothing synchronises the host, so the call can be
 * captured once in a CUDA graph and replayed. The iteration counter lives in
 * device memory (`iteration`, incremented at the end of each step) and drives
 * the learning-rate table, the warm-up and the per-iteration target noise.
 *
 * Parameter layout (one flat float buffer, reference tensor order and shapes,
 * model_2d_gaussian_rgb.py:18-26), with N = num_gaussians, C = channels:
 *   means_2d [N,2] | pre_act_scales [N,2] | pre_act_rotation [N] | colours [N,C]
 *   | pre_act_phase [N,C] | pre_act_opacities [N] | curvature [N]
 * `grads` has the same layout; `adan_state` holds exp_avg, exp_avg_sq,
 * exp_avg_diff, neg_pre_grad, each in that layout (utils/optimizer.py:161-169).
 * Param groups (train_2d_gaussian_rgb.py:73-86): lr[0] means (optionally a
 * per-iteration table), lr[1] scales, lr[2] colours + phase, lr[3] opacities,
 * lr[4] rotation, lr[5] curvature.
 * history: ring of history_len records of 1 + 3P floats (cvqpg_loss_forward_backward
 * `out` layout), record (iteration % history_len) written each step.
 * status[0] bit 0 is set (and stays) if a step's tile pairs exceeded pair_capacity;
 * bit 1 if a step's loss was not finite (NaN/Inf in a parameter or target: the
 * gradients are zeroed by nan_to_num, as in the reference, and the step goes on).
 * A step whose pairs overflowed applies no parameter update and does not advance `iteration`: the
 * caller enlarges pair_capacity (cvqpg_fit_pair_count gives the total needed),
 * sets up a new workspace and runs the same iteration again. The reference never
 * drops pairs because it sizes its sort buffers on the host every forward.
 */
typedef struct cvqpg_fit_params {
    int channels, planes;
    int height, width;
    int pad_height, pad_width;
    int num_gaussians;
    int pair_capacity;
    int cull_mode;          /* CVQPG_CULL_*; the CUDA renderer's rule by default */
    int curv_mode;          /* 0 off ('flat'), 1 constant, 2 scale_aware */
    int curv_trainable;     /* 0 for --primitive flat */
    int warmup_iters;       /* curvature frozen for the first warmup_iters iterations */
    int num_iters;          /* length of the means learning-rate table */
    int history_len;
    int no_prox;
    int inject_noise;
    double pixel_pitch;
    double wavelengths[3];
    double distances[8];
    double aperture_radius;
    double curv_nyquist;    /* 0.9 */
    double curv_const;      /* 200 */
    double lr[6];
    double betas[3];        /* (0.98, 0.92, 0.99) */
    double eps;             /* 1e-8 */
    double weight_decay;    /* 0 */
    double max_grad_norm;   /* 1.0 */
    float loss_weights[3];  /* [1, 1, 1] */
    float ssim_weight;      /* 0.005 */
    float noise_ratio;      /* 1e-3 */
    int plan_hint;          /* FFT plan choice of the propagation, 0 = default (CVQPG_PLAN_*) */
    unsigned long long seed;
    const float* target_moments; /* optional, as in cvqpg_loss_params (same targets) */
} cvqpg_fit_params;

CVQPG_API int cvqpg_fit_workspace_size(const cvqpg_fit_params* prm, size_t* bytes);
/* Synchronous: fills the workspace's constant tables (BLASM tables, lr table of
 * num_iters doubles for the means group, or NULL for a constant lr[0]). */
CVQPG_API int cvqpg_fit_setup(const cvqpg_fit_params* prm, const double* means_lr_table, void* workspace,
                              size_t workspace_bytes);
CVQPG_API int cvqpg_fit_step(const cvqpg_fit_params* prm, float* params, float* grads, float* adan_state,
                             const float* targets, const uint8_t* depth_plane, const float* target_range,
                             int32_t* iteration, float* history, int32_t* status, void* workspace,
                             size_t workspace_bytes, void* stream);
/* cvqpg_fit_step with CUDA events recorded on `stream` at the stage
 * boundaries (for timing; not for graph capture). Stage order, 14 events:
 *  0 start | 1 preprocess | 2 binning | 3 splat | 4 BLASM rows | 5 BLASM columns
 *  6 BLASM inverse rows | 7 loss | 8 adjoint rows | 9 adjoint columns
 * 10 adjoint inverse rows | 11 splat adjoint | 12 preprocess adjoint | 13 clip + Adan
 * (event i marks the end of the stage named at i; event 0 the start). */
CVQPG_API int cvqpg_fit_step_timed(const cvqpg_fit_params* prm, float* params, float* grads, float* adan_state,
                                   const float* targets, const uint8_t* depth_plane, const float* target_range,
                                   int32_t* iteration, float* history, int32_t* status, void* workspace,
                                   size_t workspace_bytes, void* stream, void** stage_events, int num_events);
/* Tile pairs of the last step or evaluation that used this workspace: out_device[0] =
 * the true pair total (saturated at INT32_MAX), out_device[1] = 1 if it exceeded
 * pair_capacity. Two int32 copied device to device on `stream`. It replaces the
 * reference's host read total_pairs = point_offsets[N-1].item() (cuda/raster.cu:71),
 * which sizes its sort buffers every forward; here the host reads it only when a
 * step reports an overflow. */
CVQPG_API int cvqpg_fit_pair_count(const cvqpg_fit_params* prm, const void* workspace, size_t workspace_bytes,
                                   int32_t* out_device, void* stream);
/* Forward only (no noise, no update): out = 1 + 3P floats as in the loss; optionally
 * the splat field [C,H,W] and the plane fields V [P,C,H,W] (complex64) when non-null. */
CVQPG_API int cvqpg_fit_evaluate(const cvqpg_fit_params* prm, const float* params, const float* targets,
                                 const uint8_t* depth_plane, const float* target_range, float* out,
                                 float* field_out, float* planes_out, int32_t* status, void* workspace,
                                 size_t workspace_bytes, void* stream);

/* ---- per-Gaussian preprocessing -------------------------------------------
 *
 * The activations, covariance, inverse and culling radii of the fit's first
 * stage and their adjoint, as separate calls (the fit step runs the same
 * kernels). Reference: Gaussians2D.apply_activations (model_2d_gaussian_rgb.py:83-112;
 * grayscale binds the curvature bound to wavelengths[0], model_2d_gaussian_grayscale.py:96),
 * compute_2d_covariance_elements + invert_cov_2D (:114-153), the radii of
 * Scene2D._render_cuda (:429-436) and the torch renderer's 3-sigma radius
 * (:400-403), with the adjoint autograd would form through them plus the
 * nan_to_num of train_2d_gaussian_rgb.py:205-208.
 *
 * params: the flat raw-parameter layout of cvqpg_fit_step. records [N][16]:
 *   mx, my, inv00, inv01, inv11, opacity, curvature (activated c), area |sx sy|,
 *   colours[C], phase mod 2 pi [C], zeros.
 * radii [N] = ceil(5 sqrt(lambda_max)) (int32); radius3 [N] = 3 sqrt(lambda_max)
 * (nullable); tiles_touched [N] = 16-px tiles of the CUDA renderer's rect.
 * Backward: splat_grads = (8 + 2C) N floats, d_means [N,2] | d_inv_cov [N,3] |
 * d_colours [N,C] | d_phase [N,C] | d_opacity [N] | d_curvature [N] | d_area [N]
 * (the gradients of cvqpg_render_backward); grads = the raw-parameter gradients
 * (flat layout) with nan/inf set to 0; partials [cvqpg_preprocess_partials(N)] =
 * per-CTA sums of squares (for clip_grad_norm_). iteration (device int, nullable =
 * 0) gates the curvature gradient during the warm-up. */
typedef struct cvqpg_preprocess_params {
    int channels;
    int num_gaussians;
    int width, height;
    int curv_mode;          /* 0 off, 1 constant, 2 scale_aware */
    int curv_trainable;
    int warmup_iters;
    double pixel_pitch;
    double wavelengths[3];
    double curv_nyquist;    /* 0.9 */
    double curv_const;      /* 200 */
} cvqpg_preprocess_params;

CVQPG_API int cvqpg_preprocess_forward(const cvqpg_preprocess_params* prm, const float* params, float* records,
                                       int32_t* radii, float* radius3, uint32_t* tiles_touched, void* stream);
CVQPG_API int cvqpg_preprocess_partials(int num_gaussians);
CVQPG_API int cvqpg_preprocess_backward(const cvqpg_preprocess_params* prm, const float* params,
                                        const float* splat_grads, float* grads, const int32_t* iteration,
                                        float* partials, void* stream);

/* Self-check of the bounded mbarrier wait that every tcgen05 kernel here uses
 * (no counterpart in the reference, which has no tensor-core code). One thread
 * waits on a shared-memory mbarrier; with arrive = 0 nothing arrives, so the
 * wait gives up after spin_limit polls and *status (device int) = 4; with
 * arrive = 1 the phase completes and *status = 0. The kernel returns either way:
 * the failure path of a timed-out pipeline wait, exercised without a fault. */
CVQPG_API int cvqpg_wait_probe(int arrive, unsigned spin_limit, int* status, void* stream);

/* ---- BF16 tensor-core GEMM (learned initialiser) ---------------------------
 *
 * No reference counterpart: the reference has no learned part. C[M,N] =
 * A[M,K] * B[N,K]^T with A and B BF16 row-major (K contiguous), FP32
 * accumulation in tensor memory (tcgen05, sm_100a), and a fused epilogue:
 *   F32        out_f32[m][n] = C (split-K: slab `split` at out_f32 + split*split_stride)
 *   BIAS       out_f32 = C + bias[n]
 *   BIAS_GELU  Z = C + bias[n] -> out_f32 (if non-null); H = GELU(Z) (erf form) ->
 *              out_bf16 [M][ld_bf16] and/or out_bf16_t [N][ld_t] (transposed)
 *   DGELU      dZ = C * GELU'(zin[m][n]) -> out_bf16 and/or out_bf16_t
 * Columns n >= valid_n are written as 0 in the BF16 outputs (padding).
 * M and N multiples of 128, K a multiple of 64*splits, lda/ldb multiples of 8,
 * 16-byte aligned operands; splits > 1 only with F32. status[0] (device int) is
 * set non-zero if a pipeline wait timed out; the kernel then writes nothing. */
#define CVQPG_GEMM_EPI_F32 0
#define CVQPG_GEMM_EPI_BIAS 1
#define CVQPG_GEMM_EPI_BIAS_GELU 2
#define CVQPG_GEMM_EPI_DGELU 3
typedef struct cvqpg_gemm_epilogue {
    int mode;
    int valid_n;
    const float* bias;
    const float* zin;
    int ld_z;
    int ld_f32;
    float* out_f32;
    long long split_stride;
    void* out_bf16;
    void* out_bf16_t;
    int ld_bf16;
    int ld_t;
} cvqpg_gemm_epilogue;

CVQPG_API int cvqpg_gemm_bf16_tn(const void* A, int lda, const void* B, int ldb, int M, int N, int K,
                                 const cvqpg_gemm_epilogue* epilogue, int splits, int* status, void* stream);

/* ---- per-tile MLP of the learned initialiser --------------------------------
 *
 * No reference counterpart: the reference starts every fit from random
 * Gaussians. in_dim -> hidden -> hidden -> out_dim with GELU after the hidden
 * layers; GEMMs on the tensor cores (cvqpg_gemm_bf16_tn, BF16 operands, FP32
 * accumulation); FP32 master weights and Adam. in_dim and hidden must be
 * multiples of 128. Weights are one FP32 vector (cvqpg_mlp_weights_size floats):
 *   W1 [hidden][in_dim] | b1 [hidden] | W2 [hidden][hidden] | b2 [hidden] |
 *   W3 [out_pad][hidden] | b3 [out_pad],  out_pad = out_dim rounded up to 128
 * (rows >= out_dim of W3 and b3 are kept at zero). The workspace holds the
 * activations and the BF16 weight copies; call cvqpg_mlp_sync_weights after
 * writing the FP32 weights from outside (cvqpg_mlp_train_step keeps them in step).
 * Loss: sum over rows m < batch and outputs j < out_dim of
 * out_weight[j] * (Y[m][j] - T[m][j])^2, divided by batch. */
typedef struct cvqpg_mlp_params {
    int batch;
    int in_dim;
    int hidden;
    int out_dim;
    float lr, beta1, beta2, eps, weight_decay;
    int reserved;
} cvqpg_mlp_params;

CVQPG_API int cvqpg_mlp_weights_size(const cvqpg_mlp_params* prm, size_t* floats);
CVQPG_API int cvqpg_mlp_workspace_size(const cvqpg_mlp_params* prm, size_t* bytes);
CVQPG_API int cvqpg_mlp_sync_weights(const cvqpg_mlp_params* prm, const float* weights, void* workspace,
                                     size_t workspace_bytes, void* stream);
/* Y [batch][out_dim] (may be null: the output then stays in the workspace). */
CVQPG_API int cvqpg_mlp_forward(const cvqpg_mlp_params* prm, const float* weights, const float* X, float* Y,
                                void* workspace, size_t workspace_bytes, int* status, void* stream);
/* Forward, loss and dL/dweights (same layout as the weights), no update. */
CVQPG_API int cvqpg_mlp_gradients(const cvqpg_mlp_params* prm, const float* weights, const float* X, const float* T,
                                  const float* out_weight, float* grads, float* loss, void* workspace,
                                  size_t workspace_bytes, int* status, void* stream);
/* Adam step from given gradients (e.g. after an all-reduce across data-parallel ranks). */
CVQPG_API int cvqpg_mlp_adam_step(const cvqpg_mlp_params* prm, float* weights, float* adam_state, int* step,
                                  const float* grads, void* workspace, size_t workspace_bytes, void* stream);
/* One Adam step (state = 2 x weights: first and second moments; step = device int,
 * incremented; bias correction uses step + 1). Graph-capturable. */
CVQPG_API int cvqpg_mlp_train_step(const cvqpg_mlp_params* prm, float* weights, float* adam_state, int* step,
                                   const float* X, const float* T, const float* out_weight, float* loss,
                                   void* workspace, size_t workspace_bytes, int* status, void* stream);

/* ---- multi-plane defocus targets (once per scene) --------------------------
 *
 * Replaces set_targets + add_defocus_blur (utils/propagator.py:361-415) with
 * the factory settings of utils/data_utils.py:66-82 (blur_size 20, blur_ratio 8):
 * plane_index = round(depth^r * (P-1)) (r = split_ratio when P == 2, else 1),
 * targets[i][c] = sum_j [sum(image_c * M_j) > 0] * (K_{int(|i-j| blur_ratio)} * image_c) * M_j,
 * M_j = [plane_index == j], K_s the normalised (blur_size+1)^2 Gaussian (an
 * impulse for s = 0), zero-padded 'same'. image [C,H,W], depth [H,W] in [0,1],
 * targets [P,C,H,W], plane_index [H,W]; planes <= 8. */
CVQPG_API int cvqpg_targets_workspace_size(int channels, int height, int width, int planes, size_t* bytes);
CVQPG_API int cvqpg_targets_synthesize(const float* image, const float* depth, int channels, int height, int width,
                                       int planes, int blur_size, float blur_ratio, float split_ratio,
                                       float* targets, uint8_t* plane_index, void* workspace,
                                       size_t workspace_bytes, void* stream);

/* ---- phase-only hologram export (export_poh.py:110-119, 175-194) -----------
 *
 * From the splat field [C,H,W] (prm->input_mode 0, tables of cvqpg_blasm_setup):
 * soft window pad + amplitude clamp -> DPAC (phase -/+ arccos(amplitude) on a
 * checkerboard, minus where y + x is even) -> 8-bit levels [C,pH,pW]
 * (round(poh / 2pi * 256) mod 256). phase_field (nullable, complex [C,pH,pW]):
 * exp(i 2 pi level / 256), ready for cvqpg_blasm_forward with input_mode 1. */
CVQPG_API int cvqpg_poh_encode(const cvqpg_blasm_params* prm, const void* tables, size_t table_bytes,
                               const float* field, uint8_t* levels, float* phase_field, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CVQPG_H_ */

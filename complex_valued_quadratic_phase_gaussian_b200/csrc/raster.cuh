// Internal interface of the rasterizer stages (binning + splat), shared by the
// drop-in C-ABI (raster.cu) and the fused fit iteration (fit.cu).
#pragma once

#include "common.cuh"

namespace cvqpg {

// One Gaussian as the splat reads it: 16 floats (64 B, four float4 loads).
//   [0] mean x  [1] mean y  [2] inv00 [3] inv01 [4] inv11 [5] opacity
//   [6] curvature (activated) [7] area = |sx*sy| [8..8+C) colour [8+C..8+2C) phase
constexpr int kRecordFloats = 16;

// Gaussians beyond this Mahalanobis distance from every pixel of a warp are
// skipped by that warp (contribution below exp(-20) ~ 2e-9 of the amplitude,
// under the float32 resolution of the per-pixel sum).
constexpr float kMahalCut = 40.0f;

struct BinWorkspace {
    uint32_t* tiles_touched;  // [N]
    uint32_t* offsets;        // [N] inclusive scan of tiles_touched
    uint32_t* scan_partials;  // [ceil(N/1024)]
    uint32_t* keys_a;         // [cap]
    uint32_t* keys_b;         // [cap]
    uint32_t* vals_a;         // [cap]
    uint32_t* vals_b;         // [cap]
    uint32_t* hist;           // [256 * sort_ctas] per-CTA digit counts, then in-row exclusive offsets
    uint32_t* digit_base;     // [256] exclusive scan of the digit totals
    int n;
    int cap;
    int sort_ctas;
};

// Carve the binning scratch out of a workspace (pass base=nullptr to size it).
BinWorkspace carve_bin_workspace(Carver& cv, int n, int cap);

// Culling rule that decides which Gaussians enter which tile list.
//   CVQPG_CULL_CUDA16_5SIGMA : 16-px lists, integer-radius rectangle
//                              (reference cuda/forward.cu:8-13, radii from
//                              model_2d_gaussian_rgb.py:432-436)
//   CVQPG_CULL_TORCH64_3SIGMA: 64-px lists, |mu - tile centre| < r3 + 32*sqrt(2)
//                              (reference model_2d_gaussian_rgb.py:311-314, 400-406)
//   CVQPG_CULL_NONE          : one list holding every Gaussian (uncut sum)
struct BinRule {
    int mode;
    int list_tile;            // list tile edge in px (16, 64, or 0 for the single list)
    int lgx, lgy;             // list grid
    int width, height;
    const int32_t* radii;     // mode CUDA16
    const float* radius_f;    // mode TORCH64 (3-sigma radius, float)
};

BinRule make_bin_rule(int mode, int width, int height, const int32_t* radii, const float* radius_f);
inline int bin_rule_lists(const BinRule& r) { return r.lgx * r.lgy; }

// Pack the reference SoA tensors into records (drop-in path).
void launch_pack_records(int channels, int n, const float* means, const float* inv_cov, const float* colours,
                         const float* phase, const float* opac, const float* curv, const float* area, float* rec,
                         cudaStream_t stream);

// Count kernel for the drop-in path (records already packed).
void launch_tile_count(const BinRule& rule, const float* records, int n, uint32_t* tiles_touched,
                       cudaStream_t stream);

// tiles_touched must already be filled. Produces point_list, ranges and
// pair_count (see cvqpg_render_forward); ranges has one row per list tile.
void launch_binning(const BinRule& rule, const float* records, const BinWorkspace& ws, int32_t* point_list,
                    int32_t* ranges, int32_t* pair_count, cudaStream_t stream);

// tile_order (optional, launch_tile_order): CTA i renders tile tile_order[i].
void launch_splat_forward(int channels, const BinRule& rule, const int32_t* ranges, const int32_t* point_list,
                          const float* records, const float* k, float dxy2, float2* out, cudaStream_t stream,
                          bool iso = false, const int32_t* tile_order = nullptr);

// Longest-list-first launch order of the 16-px tiles ([tiles] int32) from the ranges.
void launch_tile_order(const BinRule& rule, const int32_t* ranges, int32_t* order, cudaStream_t stream);

// Gradient outputs in the reference SoA layout; they are accumulated with
// atomics and must be zeroed beforehand.
struct SplatGrads {
    float* d_means;   // [N,2]
    float* d_inv;     // [N,3]
    float* d_col;     // [N,C]
    float* d_ph;      // [N,C]
    float* d_op;      // [N]
    float* d_cv;      // [N]
    float* d_ar;      // [N]
};

void launch_splat_backward(int channels, const BinRule& rule, const int32_t* ranges, const int32_t* point_list,
                           const float* records, const float* k, float dxy2, const float2* grad,
                           const SplatGrads& out, cudaStream_t stream, bool iso = false,
                           const int32_t* tile_order = nullptr);

// Tile rectangle of a Gaussian, written with the exact float operation order
// of the reference getRect (cuda/forward.cu:8-13) so that the per-tile lists
// are bit-identical to the reference's.
__device__ __forceinline__ void tile_rect(float px, float py, int r, int gx, int gy, int& x0, int& y0, int& x1,
                                          int& y1) {
    const float fr = (float)r;
    x0 = min(gx, max(0, (int)((px - fr) / 16.0f)));
    y0 = min(gy, max(0, (int)((py - fr) / 16.0f)));
    x1 = min(gx, max(0, (int)((((px + fr) + 16.0f) - 1.0f) / 16.0f)));
    y1 = min(gy, max(0, (int)((((py + fr) + 16.0f) - 1.0f) / 16.0f)));
}


// Number of tile lists a Gaussian enters and the visitor over them, shared by
// the counting and the emitting kernels so that both agree exactly.
template <typename F>
__device__ __forceinline__ void for_each_list_tile(const BinRule& R, float mx, float my, int g, F&& f) {
    if (R.mode == CVQPG_CULL_CUDA16_5SIGMA) {
        const int r = R.radii[g];
        if (r <= 0) return;
        int x0, y0, x1, y1;
        tile_rect(mx, my, r, R.lgx, R.lgy, x0, y0, x1, y1);
        for (int y = y0; y < y1; y++)
            for (int x = x0; x < x1; x++) f(y * R.lgx + x);
    } else if (R.mode == CVQPG_CULL_TORCH64_3SIGMA) {
        // fp32 with the reference torch op order, no contraction:
        // dist = (mx-cx)^2 + (my-cy)^2 ; thr = r3 + 45.254833995939045 ; keep dist < thr^2
        const float thr = __fadd_rn(R.radius_f[g], 45.254833995939045f);
        const float thr2 = __fmul_rn(thr, thr);
        if (!(thr > 0.0f) || !(mx == mx) || !(my == my)) return;
        const float lo_x = floorf((mx - thr) / 64.0f) - 1.0f, hi_x = floorf((mx + thr) / 64.0f) + 1.0f;
        const float lo_y = floorf((my - thr) / 64.0f) - 1.0f, hi_y = floorf((my + thr) / 64.0f) + 1.0f;
        const int tx0 = (int)fmaxf(0.0f, lo_x), tx1 = (int)fminf((float)(R.lgx - 1), hi_x);
        const int ty0 = (int)fmaxf(0.0f, lo_y), ty1 = (int)fminf((float)(R.lgy - 1), hi_y);
        for (int ty = ty0; ty <= ty1; ty++) {
            const int y0 = ty * 64, y1 = min(y0 + 64, R.height);
            const float cy = (float)(y0 + y1) * 0.5f;
            const float dy = __fsub_rn(my, cy);
            const float dy2 = __fmul_rn(dy, dy);
            for (int tx = tx0; tx <= tx1; tx++) {
                const int x0 = tx * 64, x1 = min(x0 + 64, R.width);
                const float cx = (float)(x0 + x1) * 0.5f;
                const float dx = __fsub_rn(mx, cx);
                const float d2 = __fadd_rn(__fmul_rn(dx, dx), dy2);
                if (d2 < thr2) f(ty * R.lgx + tx);
            }
        }
    } else {
        f(0);
    }
}

}  // namespace cvqpg

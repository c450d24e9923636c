// Tile binning and the complex quadratic-phase splat (forward and adjoint).
//
// Binning (reference: cuda/forward.cu:8-60, cuda/raster.cu:60-95):
//   tiles_touched -> inclusive scan -> (tile, id) pairs in id order -> stable
//   LSD radix sort on the tile bits only -> per-tile [start, end) ranges.
// The reference sorts 64-bit (tile<<32 | id) keys over all 64 bits; because the
// pairs are emitted in ascending id and an LSD radix sort is stable, sorting
// the ceil(log2 T) tile bits gives the identical permutation with 1-2 passes
// instead of 8. The pair count stays on the device (no host round trip), so
// every stage can be captured in a CUDA graph; buffers are sized by a caller
// capacity and an overflow flag reports when it was too small.
//
// Splat (reference: cuda/forward.cu:63-162 forward, cuda/backward.cu:22-168
// adjoint): linear coherent sum
//   U_c(p) = sum_g A_gc * o_g * G_g(p) * exp(i (phi_gc + k_c * 0.5 * c_g * m_g(p) * area_g * dxy2))
// with m = Mahalanobis distance and G = exp(max(-m/2, -50)).
#include "raster.cuh"

namespace cvqpg {

// ---------------------------------------------------------------------------
// record packing for the drop-in entry point (reference SoA tensors -> records)
// ---------------------------------------------------------------------------
template <int C>
__global__ void pack_records_kernel(int n, const float* __restrict__ means, const float* __restrict__ inv_cov,
                                    const float* __restrict__ colours, const float* __restrict__ phase,
                                    const float* __restrict__ opac, const float* __restrict__ curv,
                                    const float* __restrict__ area, float* __restrict__ rec) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    float v[kRecordFloats];
    v[0] = means[2 * g];
    v[1] = means[2 * g + 1];
    v[2] = inv_cov[3 * g];
    v[3] = inv_cov[3 * g + 1];
    v[4] = inv_cov[3 * g + 2];
    v[5] = opac[g];
    v[6] = curv[g];
    v[7] = area[g];
#pragma unroll
    for (int c = 0; c < C; c++) {
        v[8 + c] = colours[g * C + c];
        v[8 + C + c] = phase[g * C + c];
    }
#pragma unroll
    for (int i = 8 + 2 * C; i < kRecordFloats; i++) v[i] = 0.0f;
    float4* dst = reinterpret_cast<float4*>(rec + (size_t)g * kRecordFloats);
#pragma unroll
    for (int q = 0; q < 4; q++) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
}

void launch_pack_records(int channels, int n, const float* means, const float* inv_cov, const float* colours,
                                const float* phase, const float* opac, const float* curv, const float* area,
                                float* rec, cudaStream_t stream) {
    if (n <= 0) return;
    if (channels == 1)
        pack_records_kernel<1><<<ceil_div(n, 256), 256, 0, stream>>>(n, means, inv_cov, colours, phase, opac, curv,
                                                                     area, rec);
    else
        pack_records_kernel<3><<<ceil_div(n, 256), 256, 0, stream>>>(n, means, inv_cov, colours, phase, opac, curv,
                                                                     area, rec);
}

// reference preprocessKernel (cuda/forward.cu:15-26), generalised to the rule
__global__ void tile_count_kernel(BinRule rule, const float* __restrict__ rec, int n,
                                  uint32_t* __restrict__ tiles_touched) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const float2 m = *reinterpret_cast<const float2*>(rec + (size_t)g * kRecordFloats);
    uint32_t cnt = 0;
    for_each_list_tile(rule, m.x, m.y, g, [&](int) { cnt++; });
    tiles_touched[g] = cnt;
}

BinRule make_bin_rule(int mode, int width, int height, const int32_t* radii, const float* radius_f) {
    BinRule r;
    r.mode = mode;
    r.width = width;
    r.height = height;
    r.radii = radii;
    r.radius_f = radius_f;
    if (mode == CVQPG_CULL_CUDA16_5SIGMA) {
        r.list_tile = kTile;
    } else if (mode == CVQPG_CULL_TORCH64_3SIGMA) {
        r.list_tile = 64;
    } else {
        r.list_tile = 0;
    }
    if (r.list_tile > 0) {
        r.lgx = (width + r.list_tile - 1) / r.list_tile;
        r.lgy = (height + r.list_tile - 1) / r.list_tile;
    } else {
        r.lgx = 1;
        r.lgy = 1;
    }
    return r;
}

void launch_tile_count(const BinRule& rule, const float* records, int n, uint32_t* tiles_touched,
                       cudaStream_t stream) {
    if (n <= 0) return;
    tile_count_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(rule, records, n, tiles_touched);
}

// ---------------------------------------------------------------------------
// inclusive scan of tiles_touched (reduce, scan of block sums, downsweep)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanBlock = kScanThreads * kScanItems;  // 1024

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t s = lane < nw ? warp_sums[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        warp_sums[lane] = s;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t warp_prefix = w > 0 ? warp_sums[w - 1] : 0;
    if (total) *total = warp_sums[nw - 1];
    const uint32_t excl = warp_prefix + x - v;
    __syncthreads();
    return excl;
}

__global__ void scan_reduce_kernel(int n, const uint32_t* __restrict__ in, uint32_t* __restrict__ partials) {
    const int base = blockIdx.x * kScanBlock;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        const int idx = base + i * kScanThreads + threadIdx.x;
        if (idx < n) s += in[idx];
    }
    uint32_t total;
    block_exclusive_scan(s, &total);
    if (threadIdx.x == 0) partials[blockIdx.x] = total;
}

// Single block: exclusive scan of the block sums; writes the pair count and the
// overflow flag. pair_count[0] is the true pair total (saturated at INT32_MAX);
// the kernels that read the pairs clamp it to the capacity themselves.
__global__ void scan_partials_kernel(int nblocks, uint32_t* __restrict__ partials, int cap,
                                     int32_t* __restrict__ pair_count) {
    // each thread handles a contiguous chunk of ceil(nblocks/blockDim) partials
    const int per = (nblocks + blockDim.x - 1) / blockDim.x;
    const int b0 = threadIdx.x * per;
    uint32_t local = 0;
    for (int i = 0; i < per; i++)
        if (b0 + i < nblocks) local += partials[b0 + i];
    uint32_t total;
    uint32_t run = block_exclusive_scan(local, &total);
    for (int i = 0; i < per; i++)
        if (b0 + i < nblocks) {
            const uint32_t t = partials[b0 + i];
            partials[b0 + i] = run;
            run += t;
        }
    if (threadIdx.x == 0) {
        const bool over = total > (uint32_t)cap;
        pair_count[0] = total > 0x7fffffffu ? 0x7fffffff : (int32_t)total;
        pair_count[1] = over ? 1 : 0;
    }
}

__global__ void scan_downsweep_kernel(int n, const uint32_t* __restrict__ in, const uint32_t* __restrict__ partials,
                                      uint32_t* __restrict__ out) {
    const int base = blockIdx.x * kScanBlock + threadIdx.x * kScanItems;  // blocked arrangement
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        v[i] = (base + i < n) ? in[base + i] : 0;
        s += v[i];
    }
    uint32_t run = block_exclusive_scan(s, nullptr) + partials[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        run += v[i];
        if (base + i < n) out[base + i] = run;
    }
}

// ---------------------------------------------------------------------------
// emit (tile, id) pairs in id order (reference duplicateWithKeysKernel,
// cuda/forward.cu:28-47; the key keeps only the tile, the order is implied)
// ---------------------------------------------------------------------------
__global__ void duplicate_kernel(BinRule rule, int n, const float* __restrict__ rec,
                                 const uint32_t* __restrict__ tiles_touched, const uint32_t* __restrict__ offsets,
                                 uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, int cap) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= n) return;
    const uint32_t cnt = tiles_touched[g];
    if (cnt == 0) return;
    uint32_t off = offsets[g] - cnt;
    const float2 m = *reinterpret_cast<const float2*>(rec + (size_t)g * kRecordFloats);
    for_each_list_tile(rule, m.x, m.y, g, [&](int tile) {
        if (off < (uint32_t)cap) {
            keys[off] = (uint32_t)tile;
            vals[off] = (uint32_t)g;
        }
        off++;
    });
}

// ---------------------------------------------------------------------------
// stable LSD radix sort, 8-bit digits, keys = tile ids
// ---------------------------------------------------------------------------
constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 keys per CTA
constexpr int kSortWarpSpan = 32 * kSortItems;        // 512 keys per warp

__global__ void __launch_bounds__(kSortThreads) sort_upsweep_kernel(const uint32_t* __restrict__ keys,
                                                                    const int32_t* __restrict__ pair_count, int cap,
                                                                    int shift, uint32_t* __restrict__ hist,
                                                                    int sort_ctas) {
    __shared__ uint32_t h[256];
    const int n = min(pair_count[0], cap);
    const int base = blockIdx.x * kSortTile;
    if (base >= n) return;  // columns past the active range are never read
    h[threadIdx.x] = 0;
    __syncthreads();
#pragma unroll 4
    for (int i = 0; i < kSortItems; i++) {
        const int idx = base + i * kSortThreads + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * sort_ctas + blockIdx.x] = h[threadIdx.x];
}

// Digit-major exclusive scan of hist in two steps: one CTA per digit scans its
// row of per-CTA counts in place (coalesced) and records the row total; then one
// warp-group scans the 256 totals into digit_base. The downsweep adds both.
__global__ void __launch_bounds__(256) sort_scan_rows_kernel(uint32_t* __restrict__ hist,
                                                             const int32_t* __restrict__ pair_count, int cap,
                                                             int sort_ctas, uint32_t* __restrict__ digit_total) {
    const int n = min(pair_count[0], cap);
    const int active = (n + kSortTile - 1) / kSortTile;
    uint32_t* row = hist + (size_t)blockIdx.x * sort_ctas;
    uint32_t carry = 0;
    for (int c0 = 0; c0 < active; c0 += 256) {
        const int c = c0 + threadIdx.x;
        const uint32_t v = c < active ? row[c] : 0u;
        uint32_t total = 0;
        const uint32_t ex = block_exclusive_scan(v, &total);
        if (c < active) row[c] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) digit_total[blockIdx.x] = carry;
}

__global__ void __launch_bounds__(256) sort_scan_digits_kernel(uint32_t* __restrict__ digit_base) {
    const uint32_t v = digit_base[threadIdx.x];  // the totals, replaced by their exclusive scan
    const uint32_t ex = block_exclusive_scan(v, nullptr);
    digit_base[threadIdx.x] = ex;
}

__global__ void __launch_bounds__(kSortThreads) sort_downsweep_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
    uint32_t* __restrict__ vals_out, const int32_t* __restrict__ pair_count, int cap, int shift,
    const uint32_t* __restrict__ hist, const uint32_t* __restrict__ digit_base, int sort_ctas) {
    __shared__ uint32_t wc[kSortWarps][257];  // slot 256 absorbs invalid lanes
    const int n = min(pair_count[0], cap);
    const int base = blockIdx.x * kSortTile;
    if (base >= n) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = threadIdx.x; i < kSortWarps * 257; i += kSortThreads) (&wc[0][0])[i] = 0;
    __syncthreads();

    const uint32_t lt_mask = (1u << lane) - 1u;
    uint32_t key[kSortItems], val[kSortItems], rank[kSortItems];
    const int wbase = base + w * kSortWarpSpan;
#pragma unroll
    for (int i = 0; i < kSortItems; i++) {
        const int idx = wbase + i * 32 + lane;
        const bool valid = idx < n;
        key[i] = valid ? keys_in[idx] : 0u;
        val[i] = valid ? vals_in[idx] : 0u;
        const uint32_t d = valid ? ((key[i] >> shift) & 255u) : 256u;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t before = wc[w][d];
        rank[i] = before + __popc(peers & lt_mask);
        __syncwarp();
        if (lane == __ffs(peers) - 1) wc[w][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive scan over warps for each digit
    {
        const int d = threadIdx.x;  // 256 threads = 256 digits
        uint32_t run = 0;
#pragma unroll
        for (int ww = 0; ww < kSortWarps; ww++) {
            const uint32_t c = wc[ww][d];
            wc[ww][d] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kSortItems; i++) {
        const int idx = wbase + i * 32 + lane;
        if (idx < n) {
            const uint32_t d = (key[i] >> shift) & 255u;
            const uint32_t pos = digit_base[d] + hist[d * sort_ctas + blockIdx.x] + wc[w][d] + rank[i];
            keys_out[pos] = key[i];
            vals_out[pos] = val[i];
        }
    }
}

__global__ void zero_ranges_kernel(int32_t* __restrict__ ranges, int num_tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < num_tiles) reinterpret_cast<int2*>(ranges)[i] = make_int2(0, 0);
}

// reference identifyTileRangesKernel (cuda/forward.cu:49-60)
__global__ void ranges_kernel(const uint32_t* __restrict__ keys, const int32_t* __restrict__ pair_count, int cap,
                              int32_t* __restrict__ ranges) {
    const int n = min(pair_count[0], cap);
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= n) return;
    const uint32_t tile = keys[idx];
    if (idx == 0) {
        ranges[2 * tile] = 0;
    } else {
        const uint32_t prev = keys[idx - 1];
        if (prev != tile) {
            ranges[2 * prev + 1] = idx;
            ranges[2 * tile] = idx;
        }
    }
    if (idx == n - 1) ranges[2 * tile + 1] = n;
}

BinWorkspace carve_bin_workspace(Carver& cv, int n, int cap) {
    BinWorkspace ws;
    ws.n = n;
    ws.cap = cap;
    ws.sort_ctas = (int)ceil_div((size_t)(cap > 0 ? cap : 1), kSortTile);
    const int nscan = (int)ceil_div((size_t)(n > 0 ? n : 1), kScanBlock);
    ws.tiles_touched = cv.take<uint32_t>(n > 0 ? n : 1);
    ws.offsets = cv.take<uint32_t>(n > 0 ? n : 1);
    ws.scan_partials = cv.take<uint32_t>(nscan);
    ws.keys_a = cv.take<uint32_t>(cap > 0 ? cap : 1);
    ws.keys_b = cv.take<uint32_t>(cap > 0 ? cap : 1);
    ws.vals_a = cv.take<uint32_t>(cap > 0 ? cap : 1);
    ws.vals_b = cv.take<uint32_t>(cap > 0 ? cap : 1);
    ws.hist = cv.take<uint32_t>((size_t)256 * ws.sort_ctas);
    ws.digit_base = cv.take<uint32_t>(256);
    return ws;
}

void launch_binning(const BinRule& rule, const float* records, const BinWorkspace& ws, int32_t* point_list,
                    int32_t* ranges, int32_t* pair_count, cudaStream_t stream) {
    const int num_lists = bin_rule_lists(rule);
    const int n = ws.n;
    zero_ranges_kernel<<<ceil_div(num_lists, 256), 256, 0, stream>>>(ranges, num_lists);
    if (n <= 0) {
        cudaMemsetAsync(pair_count, 0, 2 * sizeof(int32_t), stream);
        return;
    }
    const int nscan = (int)ceil_div(n, kScanBlock);
    scan_reduce_kernel<<<nscan, kScanThreads, 0, stream>>>(n, ws.tiles_touched, ws.scan_partials);
    scan_partials_kernel<<<1, 1024, 0, stream>>>(nscan, ws.scan_partials, ws.cap, pair_count);
    scan_downsweep_kernel<<<nscan, kScanThreads, 0, stream>>>(n, ws.tiles_touched, ws.scan_partials, ws.offsets);
    if (ws.cap <= 0) return;
    duplicate_kernel<<<ceil_div(n, 256), 256, 0, stream>>>(rule, n, records, ws.tiles_touched, ws.offsets,
                                                           ws.keys_a, ws.vals_a, ws.cap);
    int bits = 0;
    while ((1 << bits) < num_lists) bits++;
    const int passes = bits <= 8 ? 1 : (bits + 7) / 8;
    const uint32_t* kin = ws.keys_a;
    const uint32_t* vin = ws.vals_a;
    for (int p = 0; p < passes; p++) {
        uint32_t* kout = (p % 2 == 0) ? ws.keys_b : ws.keys_a;
        uint32_t* vout = (p == passes - 1) ? reinterpret_cast<uint32_t*>(point_list)
                                           : ((p % 2 == 0) ? ws.vals_b : ws.vals_a);
        sort_upsweep_kernel<<<ws.sort_ctas, kSortThreads, 0, stream>>>(kin, pair_count, ws.cap, 8 * p, ws.hist,
                                                                        ws.sort_ctas);
        sort_scan_rows_kernel<<<256, 256, 0, stream>>>(ws.hist, pair_count, ws.cap, ws.sort_ctas, ws.digit_base);
        sort_scan_digits_kernel<<<1, 256, 0, stream>>>(ws.digit_base);
        sort_downsweep_kernel<<<ws.sort_ctas, kSortThreads, 0, stream>>>(kin, vin, kout, vout, pair_count, ws.cap,
                                                                          8 * p, ws.hist, ws.digit_base,
                                                                          ws.sort_ctas);
        kin = kout;
        vin = vout;
    }
    ranges_kernel<<<ceil_div(ws.cap, 256), 256, 0, stream>>>(kin, pair_count, ws.cap, ranges);
}

// Index of the list a 16-px splat tile reads.
__device__ __forceinline__ int list_of_tile(const BinRule& R, int tx, int ty) {
    if (R.list_tile == kTile) return ty * R.lgx + tx;
    if (R.list_tile == 64) return (ty >> 2) * R.lgx + (tx >> 2);
    return 0;
}

// Launch order of the 16-px splat tiles, longest list first (a counting sort on
// list length / 4, lengths above 4095 sharing the first bucket): the block
// scheduler then hands the heaviest tiles out first and the last wave holds
// short ones (longest-processing-time-first list scheduling). One CTA.
constexpr int kOrderThreads = 1024;
__global__ void __launch_bounds__(kOrderThreads) tile_order_kernel(BinRule rule, const int32_t* __restrict__ ranges,
                                                                 int gx, int ntiles, int32_t* __restrict__ order) {
    __shared__ int cnt[kOrderThreads];
    __shared__ int wsum[kOrderThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int2* r2 = reinterpret_cast<const int2*>(ranges);
    cnt[t] = 0;
    __syncthreads();
    for (int i = t; i < ntiles; i += kOrderThreads) {
        const int2 r = r2[list_of_tile(rule, i % gx, i / gx)];
        atomicAdd(&cnt[kOrderThreads - 1 - min(max(r.y - r.x, 0), 4 * kOrderThreads - 1) / 4], 1);
    }
    __syncthreads();
    const int v = cnt[t];
    int incl = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[w] = incl;
    __syncthreads();
    if (w == 0) {
        const int x = wsum[lane];
        int ix = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, ix, o);
            if (lane >= o) ix += y;
        }
        wsum[lane] = ix - x;
    }
    __syncthreads();
    cnt[t] = wsum[w] + incl - v;
    __syncthreads();
    for (int i = t; i < ntiles; i += kOrderThreads) {
        const int2 r = r2[list_of_tile(rule, i % gx, i / gx)];
        const int pos = atomicAdd(&cnt[kOrderThreads - 1 - min(max(r.y - r.x, 0), 4 * kOrderThreads - 1) / 4], 1);
        order[pos] = i;
    }
}

void launch_tile_order(const BinRule& rule, const int32_t* ranges, int32_t* order, cudaStream_t stream) {
    const int gx = (rule.width + kTile - 1) / kTile, gy = (rule.height + kTile - 1) / kTile;
    tile_order_kernel<<<1, kOrderThreads, 0, stream>>>(rule, ranges, gx, gx * gy, order);
}


// ---------------------------------------------------------------------------
// splat forward: one CTA per 16x16 tile, one pixel per thread, each warp an
// 8x4 pixel block; Gaussian batches of 256 records staged in shared memory.
// ---------------------------------------------------------------------------
template <int C, bool ISO>
__global__ void __launch_bounds__(kTilePixels) splat_forward_kernel(
    BinRule rule, const int32_t* __restrict__ ranges, const int32_t* __restrict__ point_list,
    const float4* __restrict__ rec, const float* __restrict__ k, float dxy2, float2* __restrict__ out, int W, int H,
    int gx, const int32_t* __restrict__ order) {
    constexpr int NV = (8 + 2 * C + 3) / 4;  // float4 words used per record
    __shared__ float4 s_rec[kTilePixels][NV];
    const int tile = order ? order[blockIdx.x] : blockIdx.x;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    const int px = (tile % gx) * kTile + (w & 1) * 8 + (lane & 7);
    const int py = (tile / gx) * kTile + (w >> 1) * 4 + (lane >> 3);
    const float fx = (float)px, fy = (float)py;
    const int2 range = reinterpret_cast<const int2*>(ranges)[list_of_tile(rule, tile % gx, tile / gx)];

    float kc[C], acc_r[C], acc_i[C];
#pragma unroll
    for (int c = 0; c < C; c++) {
        kc[c] = k[c];
        acc_r[c] = 0.0f;
        acc_i[c] = 0.0f;
    }

    for (int b = range.x; b < range.y; b += kTilePixels) {
        __syncthreads();
        if (b + t < range.y) {
            const int g = point_list[b + t];
            float4 v[NV];
#pragma unroll
            for (int q = 0; q < NV; q++) v[q] = __ldg(&rec[(size_t)g * 4 + q]);
            const float op = v[1].y;  // colours staged pre-multiplied by the opacity
            v[2].x *= op;
            if (C > 1) {
                v[2].y *= op;
                v[2].z *= op;
            }
#pragma unroll
            for (int q = 0; q < NV; q++) s_rec[t][q] = v[q];
        }
        __syncthreads();
        const int cnt = min(kTilePixels, range.y - b);
        for (int j = 0; j < cnt; j++) {
            const float4 r0 = s_rec[j][0];  // mx my i00 i01
            const float4 r1 = s_rec[j][1];  // i11 opac curv area
            const float dx = r0.x - fx, dy = r0.y - fy;
            const float mahal = dx * (r0.z * dx + r0.w * dy) + dy * (r0.w * dx + r1.x * dy);
            if (!__any_sync(0xffffffffu, mahal < kMahalCut)) continue;
            const float power = fmaxf(-0.5f * mahal, -50.0f);
            const float G = ex2_ftz(power * 1.44269504088896341f);  // exp(power)
            // Mahalanobis QPF (c m area) or, with ISO, the isotropic form (c |r - mu|^2)
            const float base = ISO ? 0.5f * r1.z * (dx * dx + dy * dy) * dxy2 : 0.5f * r1.z * mahal * r1.w * dxy2;
            const float4 r2 = s_rec[j][2];
            float col[C], ph[C];
            if (C == 1) {
                col[0] = r2.x;
                ph[0] = r2.y;
            } else {
                const float4 r3 = s_rec[j][NV - 1];
                col[0] = r2.x;
                col[C > 1 ? 1 : 0] = r2.y;
                col[C > 2 ? 2 : 0] = r2.z;
                ph[0] = r2.w;
                ph[C > 1 ? 1 : 0] = r3.x;
                ph[C > 2 ? 2 : 0] = r3.y;
            }
#pragma unroll
            for (int c = 0; c < C; c++) {
                float s, co;
                sincos_reduced_ftz(ph[c] + kc[c] * base, &s, &co);
                const float amp = col[c] * G;  // colour x opacity (folded at staging) x G
                acc_r[c] = fmaf(amp, co, acc_r[c]);
                acc_i[c] = fmaf(amp, s, acc_i[c]);
            }
        }
    }
    if (px < W && py < H) {
        const size_t pid = (size_t)py * W + px;
#pragma unroll
        for (int c = 0; c < C; c++) out[(size_t)c * H * W + pid] = make_float2(acc_r[c], acc_i[c]);
    }
}

void launch_splat_forward(int channels, const BinRule& rule, const int32_t* ranges, const int32_t* point_list,
                          const float* records, const float* k, float dxy2, float2* out, cudaStream_t stream,
                          bool iso, const int32_t* tile_order) {
    const int width = rule.width, height = rule.height;
    const int gx = (width + kTile - 1) / kTile, gy = (height + kTile - 1) / kTile;
    const float4* rec = reinterpret_cast<const float4*>(records);
    const dim3 grid(gx * gy);
    if (channels == 1) {
        if (iso)
            splat_forward_kernel<1, true><<<grid, kTilePixels, 0, stream>>>(rule, ranges, point_list, rec, k, dxy2,
                                                                            out, width, height, gx, tile_order);
        else
            splat_forward_kernel<1, false><<<grid, kTilePixels, 0, stream>>>(rule, ranges, point_list, rec, k, dxy2,
                                                                             out, width, height, gx, tile_order);
    } else {
        if (iso)
            splat_forward_kernel<3, true><<<grid, kTilePixels, 0, stream>>>(rule, ranges, point_list, rec, k, dxy2,
                                                                            out, width, height, gx, tile_order);
        else
            splat_forward_kernel<3, false><<<grid, kTilePixels, 0, stream>>>(rule, ranges, point_list, rec, k, dxy2,
                                                                             out, width, height, gx, tile_order);
    }
}

// Columns [x0, x0 + n) of tile row `fy` (tile origin tx0, xmax columns) where
// the Gaussian (mx, my, inverse covariance i00 i01 i11) may be under the cut.
__device__ __forceinline__ void cut_row_span(float mx, float my, float i00, float i01, float i11, float fy, int tx0,
                                             int xmax, int* x0, int* n) {
    const float cut = kMahalCut * 1.001f;
    const float dy = my - fy;
    // i00 dx^2 + 2 i01 dy dx + i11 dy^2 < cut, dx = mx - x
    const float q = fmaf(i01 * dy, i01 * dy, -i00 * fmaf(i11 * dy, dy, -cut));
    if (!(i00 > 0.0f) || !(q < 3.0e38f) || !(i00 < 3.0e38f)) {  // degenerate: scan the whole row
        *x0 = 0;
        *n = xmax;
        return;
    }
    if (q < 0.0f) {
        *x0 = 0;
        *n = 0;
        return;
    }
    const float centre = mx + i01 * dy / i00 - (float)tx0;  // x of the minimum, tile-relative
    const float hw = sqrtf(q) / i00 + 1.0e-3f;
    const float lo = fmaxf(ceilf(centre - hw), 0.0f);
    const float hi = fminf(floorf(centre + hw), (float)(xmax - 1));
    if (!(hi >= lo)) {
        *x0 = 0;
        *n = 0;
        return;
    }
    *x0 = (int)lo;
    *n = (int)hi - (int)lo + 1;
}

// ---------------------------------------------------------------------------
// splat adjoint over row segments ("items"): one CTA per tile. For a batch of
// list entries the CTA cuts every entry's rows to the span under the
// Mahalanobis cut (cut_row_span), and each non-empty (entry, row, span) is one
// item. Items are counting-sorted by (span length descending, row), and thread
// t takes items t, t + NT, ...: the 32 items of a warp step have (nearly) the
// same length, and items of the same row read the same dL/dU pixels
// (shared-memory broadcast). Each warp adds its items' sums into its own
// per-entry sums in shared memory; one global atomic per parameter per
// (Gaussian, tile) follows at the end of the batch.
//
// Along a row segment dy is fixed and dx steps by -1, so the Mahalanobis
// distance is m = (i00 dx + 2 i01 dy) dx + i11 dy^2 and the per-pixel terms of
// the reference adjoint (cuda/backward.cu:101-147) regroup into sums whose row
// totals give every parameter. With (P_c + i Q_c) = conj(exp(i theta_c)) dL/dU_c:
//   Acol_c = sum G P_c, Aph_c = sum G Q_c,
//   M = G (-(1/2) sum_c col_c P_c + kq sum_c k_c col_c Q_c)   (= dL/dm / opacity,
//       kq = c area dxy2 / 2),
//   R0 = sum M, R1 = sum M dx, R2 = sum M dx^2, T = sum G (sum_c k_c col_c Q_c) m;
// per row: d inv00 = o R2, d inv01 = 2 o dy R1, d inv11 = o dy^2 R0,
// d mx = 2 o (i00 R1 + i01 dy R0), d my = 2 o (i11 dy R0 + i01 R1); per entry:
// d opacity = sum_c col_c Acol_c, d colour_c = o Acol_c, d phase_c = o col_c Aph_c,
// d curvature = o (area dxy2 / 2) T, d area = o (c dxy2 / 2) T (o = opacity).
// The isotropic form (theta = phi + k (c dxy2 / 2)(dx^2 + dy^2)) has no phase
// term in dL/dm and adds the phase's own dependence on the mean
// (U0 = sum G K, U1 = sum G K dx, U2 = sum G K dx^2, K = sum_c k_c col_c Q_c).
// The phase is evaluated per pixel (Cody-Waite reduction + SFU sin/cos), as in
// the forward: a rotation recurrence along the row would save no issue slots
// and its rounding drifts with the segment length.
// ---------------------------------------------------------------------------
constexpr int kRowThreads = 128;
constexpr int kRowBatch = 96;                  // list entries per batch (one per thread when staging)
constexpr int kRowWarps = kRowThreads / 32;
constexpr int kRowItems = kRowBatch * kTile;   // at most one item per entry and tile row
constexpr int kRowKeys = kTile * kTile;        // sort keys: (16 - length) * 16 + row
constexpr int kGRow = kTile + 1;               // padded row of the staged dL/dU tile

template <int C, bool ISO>
__global__ void __launch_bounds__(kRowThreads) splat_backward_rows_kernel(
    BinRule rule, const int32_t* __restrict__ ranges, const int32_t* __restrict__ point_list,
    const float4* __restrict__ rec, const float* __restrict__ k, float dxy2, const float2* __restrict__ grad, int W,
    int H, int gx, SplatGrads out, const int32_t* __restrict__ order) {
    constexpr int NV = (8 + 2 * C + 3) / 4;  // float4 words used per record
    constexpr int NE = 6 + 2 * C;            // per-entry sums: mx my d00 d01 d11 T Acol[C] Aph[C]
    __shared__ float2 s_g[C][kTile * kGRow];  // rows padded to 17: rows at one column hit distinct banks
    __shared__ float4 s_rec[NV][kRowBatch];  // word-major: lanes of different entries hit distinct banks
    __shared__ int s_gid[kRowBatch];
    __shared__ uint32_t s_item[kRowItems];         // entry | row word << 8
    // per-warp sums of each entry ([warp][entry][NE], NE a multiple of 4: one lane's sums are three
    // float4 words at a 48-byte stride, eight bank groups); before the items are processed the same
    // memory holds the entries' row spans and the sort-key counts
    __shared__ __align__(16) float s_acc[kRowWarps * NE * kRowBatch];
    static_assert(NE % 4 == 0, "per-entry sums in float4 words");
    // row word: 0 (empty) or 0x8000 | y | x0 << 4 | (n - 1) << 8
    uint16_t(*s_rows)[kTile] = reinterpret_cast<uint16_t(*)[kTile]>(s_acc);
    int* s_key = reinterpret_cast<int*>(s_acc) + kRowBatch * kTile / 2;
    static_assert(kRowBatch * kTile / 2 + kRowKeys <= kRowWarps * NE * kRowBatch, "span and key scratch fit");
    static_assert(kRowBatch <= kRowThreads, "one entry per thread when staging the records");

    const int tile = order ? order[blockIdx.x] : blockIdx.x;
    const int2 range = reinterpret_cast<const int2*>(ranges)[list_of_tile(rule, tile % gx, tile / gx)];
    if (range.y <= range.x) return;
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    const int tx0 = (tile % gx) * kTile, ty0 = (tile / gx) * kTile;
    {  // the tile's dL/dU, all loads of a thread issued before its stores
        constexpr int kIt = kTilePixels / kRowThreads;
        float2 gv[kIt][C];
#pragma unroll
        for (int u = 0; u < kIt; u++) {
            const int p = t + u * kRowThreads;
            const int px = tx0 + (p & 15), py = ty0 + (p >> 4);
            const bool inside = px < W && py < H;
            const size_t e = inside ? (size_t)py * W + px : 0;
#pragma unroll
            for (int c = 0; c < C; c++) gv[u][c] = inside ? grad[(size_t)c * H * W + e] : make_float2(0.0f, 0.0f);
        }
#pragma unroll
        for (int u = 0; u < kIt; u++)
#pragma unroll
            for (int c = 0; c < C; c++) s_g[c][((t + u * kRowThreads) >> 4) * kGRow + ((t + u * kRowThreads) & 15)] = gv[u][c];
        for (int i = t; i < C * kTile; i += kRowThreads) s_g[i / kTile][(i % kTile) * kGRow + kTile] = make_float2(0.f, 0.f);
    }
    static_assert(kTilePixels % kRowThreads == 0, "whole pixel rounds");
    const int xmax = min(kTile, W - tx0), ymax = min(kTile, H - ty0);

    float kc[C];
#pragma unroll
    for (int c = 0; c < C; c++) kc[c] = k[c];

    for (int b0 = range.x; b0 < range.y; b0 += kRowBatch) {
        const int nb = min(kRowBatch, range.y - b0);
        // 1. stage the entry's record and its row spans; count the sort keys
        for (int i = t; i < kRowKeys; i += kRowThreads) s_key[i] = 0;
        __syncthreads();
        if (t < nb) {
            const int g = point_list[b0 + t];
            s_gid[t] = g;
#pragma unroll
            for (int q = 0; q < NV; q++) s_rec[q][t] = __ldg(&rec[(size_t)g * 4 + q]);
        }
        __syncthreads();
        // spans, one (entry, row) per thread step (16 lanes share an entry: broadcast reads)
        for (int idx = t; idx < nb * kTile; idx += kRowThreads) {
            const int e = idx >> 4, yy = idx & 15;
            const float4 r0 = s_rec[0][e];
            const float i11 = s_rec[1][e].x;
            int x0 = 0, n = 0;
            // a Gaussian whose mean or inverse covariance is not finite reaches no pixel under the cut
            const bool finite = fabsf(r0.x) + fabsf(r0.y) + fabsf(r0.z) + fabsf(r0.w) + fabsf(i11) < INFINITY;
            if (finite && yy < ymax) cut_row_span(r0.x, r0.y, r0.z, r0.w, i11, (float)(ty0 + yy), tx0, xmax, &x0, &n);
            s_rows[e][yy] = n > 0 ? (uint16_t)(0x8000 | yy | (x0 << 4) | ((n - 1) << 8)) : (uint16_t)0;
            if (n > 0) atomicAdd(&s_key[(kTile - n) * kTile + yy], 1);
        }
        __syncthreads();
        // 2. exclusive scan of the key counts (warp 0; 8 keys per lane)
        if (wid == 0) {
            constexpr int kPerLane = kRowKeys / 32;
            int cnt[kPerLane], sum = 0;
#pragma unroll
            for (int u = 0; u < kPerLane; u++) {
                cnt[u] = s_key[lane * kPerLane + u];
                sum += cnt[u];
            }
            int incl = sum;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += y;
            }
            int run = incl - sum;
#pragma unroll
            for (int u = 0; u < kPerLane; u++) {
                s_key[lane * kPerLane + u] = run;
                run += cnt[u];
            }
        }
        __syncthreads();
        // 3. scatter the items into key order
        for (int idx = t; idx < nb * kTile; idx += kRowThreads) {
            const int w = s_rows[idx >> 4][idx & 15];
            if (w & 0x8000) {
                const int n = ((w >> 8) & 15) + 1, yy = w & 15;
                const int pos = atomicAdd(&s_key[(kTile - n) * kTile + yy], 1);
                s_item[pos] = (uint32_t)(idx >> 4) | ((uint32_t)(w & 0xfff) << 8);
            }
        }
        __syncthreads();
        const int nitems = s_key[kRowKeys - 1];  // the last key's cursor ends at the item total
        __syncthreads();  // every thread holds the total before the scratch becomes the sums
        for (int i = t; i < kRowWarps * NE * kRowBatch; i += kRowThreads) s_acc[i] = 0.0f;
        __syncthreads();

        // 4. the items, 32 per warp step (warp-uniform loop: the flush below needs the whole warp)
        float* acc = s_acc + wid * (NE * kRowBatch);
        for (int base = wid * 32; base < nitems; base += kRowThreads) {
            const int i = base + lane;
            const bool valid = i < nitems;
            const uint32_t word = s_item[valid ? i : 0];
            const int e = word & 0xff;
            const int yy = (word >> 8) & 15, x0 = (word >> 12) & 15;
            const int n = valid ? ((word >> 16) & 15) + 1 : 0;
            const float4 r0 = s_rec[0][e], r1 = s_rec[1][e], r2 = s_rec[2][e];
            const float mx = r0.x, my = r0.y, i00 = r0.z, i01 = r0.w, i11 = r1.x;
            const float curv = r1.z, ar = r1.w;
            float col[C], ph[C];
            if (C == 1) {
                col[0] = r2.x;
                ph[0] = r2.y;
            } else {
                const float4 r3 = s_rec[NV - 1][e];
                col[0] = r2.x;
                col[C > 1 ? 1 : 0] = r2.y;
                col[C > 2 ? 2 : 0] = r2.z;
                ph[0] = r2.w;
                ph[C > 1 ? 1 : 0] = r3.x;
                ph[C > 2 ? 2 : 0] = r3.y;
            }
            const float fy = (float)(ty0 + yy);
            const float dy = my - fy;
            float dx = mx - (float)(tx0 + x0);
            const float lin = 2.0f * i01 * dy, cst = i11 * dy * dy;  // m = (i00 dx + lin) dx + cst
            // phase = phi_c + k_c base, base = kq m (isotropic form: kq (dx^2 + dy^2))
            const float kq = ISO ? 0.5f * curv * dxy2 : 0.5f * curv * ar * dxy2;
            const float dy2 = dy * dy;
            float kcol[C], colh[C];
#pragma unroll
            for (int c = 0; c < C; c++) {
                kcol[c] = kc[c] * col[c];
                colh[c] = -0.5f * col[c];
            }
            float acol[C], aph[C];
#pragma unroll
            for (int c = 0; c < C; c++) acol[c] = aph[c] = 0.0f;
            float R0 = 0.f, R1 = 0.f, R2 = 0.f, T = 0.f, U0 = 0.f, U1 = 0.f, U2 = 0.f;
            int p = yy * kGRow + x0;
#pragma unroll 1  // measured: 2- and 4-way unrolled forms of this loop were 2-3 % slower
            for (int j = 0; j < n; j++, p++) {
                const float mahal = fmaf(fmaf(i00, dx, lin), dx, cst);
                {
                    // a pixel beyond the cut adds nothing (G = 0; its terms are finite). Under the cut
                    // mahal < 40, so the forward's clamp of the exponent at -50 never applies.
                    const float G = mahal < kMahalCut ? ex2_ftz(mahal * kNegHalfLog2e) : 0.0f;
                    const float base = kq * (ISO ? fmaf(dx, dx, dy2) : mahal);
                    float sp = 0.f, kqs = 0.f;
#pragma unroll
                    for (int c = 0; c < C; c++) {
                        float zs, zc;
                        sincos_reduced_ftz(fmaf(kc[c], base, ph[c]), &zs, &zc);
                        const float2 gp = s_g[c][p];
                        const float P = fmaf(gp.x, zc, gp.y * zs);
                        const float Q = fmaf(gp.y, zc, -gp.x * zs);
                        acol[c] = fmaf(G, P, acol[c]);
                        aph[c] = fmaf(G, Q, aph[c]);
                        sp = fmaf(colh[c], P, sp);
                        kqs = fmaf(kcol[c], Q, kqs);
                    }
                    const float gk = G * kqs;
                    if (ISO) {
                        const float M = G * sp;
                        const float tm = M * dx;
                        R0 += M;
                        R1 += tm;
                        R2 = fmaf(tm, dx, R2);
                        const float tu = gk * dx;
                        U0 += gk;
                        U1 += tu;
                        U2 = fmaf(tu, dx, U2);
                    } else {
                        const float M = fmaf(kq, gk, G * sp);
                        const float tm = M * dx;
                        R0 += M;
                        R1 += tm;
                        R2 = fmaf(tm, dx, R2);
                        T = fmaf(gk, mahal, T);
                    }
                }
                dx -= 1.0f;
            }
            // the row's totals into the entry's sums (opacity factors applied per entry)
            float v[NE];
            v[0] = 2.0f * fmaf(i00, R1, i01 * dy * R0);
            v[1] = 2.0f * fmaf(i11 * dy, R0, i01 * R1);
            v[2] = R2;
            v[3] = 2.0f * dy * R1;
            v[4] = dy2 * R0;
            if (ISO) {
                const float hc = curv * dxy2;
                v[0] = fmaf(hc, U1, v[0]);
                v[1] = fmaf(hc * dy, U0, v[1]);
                v[5] = 0.5f * dxy2 * fmaf(dy2, U0, U2);
            } else {
                v[5] = T;
            }
#pragma unroll
            for (int c = 0; c < C; c++) {
                v[6 + c] = acol[c];
                v[6 + C + c] = aph[c];
            }
            // Into this warp's sums: a float atomicAdd on shared memory is a compare-and-swap loop,
            // so lanes that share an entry add in turn instead (rank among the lanes with that entry).
            __syncwarp();
            const unsigned peers = __match_any_sync(0xffffffffu, valid ? (unsigned)e : 0x100u + (unsigned)lane);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            const int rounds = (int)__reduce_max_sync(0xffffffffu, (unsigned)__popc(peers));
            for (int r = 0; r < rounds; r++) {
                if (valid && rank == r) {
#pragma unroll
                    for (int q = 0; q < NE / 4; q++) {
                        float4* a4 = reinterpret_cast<float4*>(acc + e * NE) + q;
                        float4 x = *a4;
                        x.x += v[4 * q];
                        x.y += v[4 * q + 1];
                        x.z += v[4 * q + 2];
                        x.w += v[4 * q + 3];
                        *a4 = x;
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
        // 5. one global atomic per parameter per (Gaussian, tile)
        if (t < nb) {
            const int g = s_gid[t];
            const float4 r1 = s_rec[1][t], r2 = s_rec[2][t];
            const float opac = r1.y, curv = r1.z, ar = r1.w;
            float col[C];
            col[0] = r2.x;
            if (C > 1) {
                col[C > 1 ? 1 : 0] = r2.y;
                col[C > 2 ? 2 : 0] = r2.z;
            }
            float a[NE];
#pragma unroll
            for (int q = 0; q < NE; q++) a[q] = 0.0f;
#pragma unroll
            for (int w = 0; w < kRowWarps; w++)
#pragma unroll
                for (int q = 0; q < NE / 4; q++) {
                    const float4 x = reinterpret_cast<const float4*>(s_acc + (w * kRowBatch + t) * NE)[q];
                    a[4 * q] += x.x;
                    a[4 * q + 1] += x.y;
                    a[4 * q + 2] += x.z;
                    a[4 * q + 3] += x.w;
                }
            float dop = 0.0f;
#pragma unroll
            for (int c = 0; c < C; c++) dop = fmaf(col[c], a[6 + c], dop);
            const float vm0 = opac * a[0], vm1 = opac * a[1];
            const float v00 = opac * a[2], v01 = opac * a[3], v11 = opac * a[4];
            const float vcv = ISO ? opac * a[5] : opac * (0.5f * ar * dxy2) * a[5];
            const float var = ISO ? 0.0f : opac * (0.5f * curv * dxy2) * a[5];
            if (vm0 != 0.f) atomicAdd(&out.d_means[2 * g], vm0);
            if (vm1 != 0.f) atomicAdd(&out.d_means[2 * g + 1], vm1);
            if (v00 != 0.f) atomicAdd(&out.d_inv[3 * g], v00);
            if (v01 != 0.f) atomicAdd(&out.d_inv[3 * g + 1], v01);
            if (v11 != 0.f) atomicAdd(&out.d_inv[3 * g + 2], v11);
            if (dop != 0.f) atomicAdd(&out.d_op[g], dop);
            if (vcv != 0.f) atomicAdd(&out.d_cv[g], vcv);
            if (var != 0.f) atomicAdd(&out.d_ar[g], var);
#pragma unroll
            for (int c = 0; c < C; c++) {
                const float vc = opac * a[6 + c], vp = opac * col[c] * a[6 + C + c];
                if (vc != 0.f) atomicAdd(&out.d_col[g * C + c], vc);
                if (vp != 0.f) atomicAdd(&out.d_ph[g * C + c], vp);
            }
        }
        __syncthreads();
    }
}

template <int C, bool ISO>
static void launch_splat_backward_t(const BinRule& rule, const int32_t* ranges, const int32_t* point_list,
                                    const float4* rec, const float* k, float dxy2, const float2* grad,
                                    const SplatGrads& out, cudaStream_t stream, const int32_t* tile_order) {
    const int gx = (rule.width + kTile - 1) / kTile, gy = (rule.height + kTile - 1) / kTile;
    splat_backward_rows_kernel<C, ISO><<<gx * gy, kRowThreads, 0, stream>>>(
        rule, ranges, point_list, rec, k, dxy2, grad, rule.width, rule.height, gx, out, tile_order);
}

void launch_splat_backward(int channels, const BinRule& rule, const int32_t* ranges, const int32_t* point_list,
                           const float* records, const float* k, float dxy2, const float2* grad,
                           const SplatGrads& out, cudaStream_t stream, bool iso, const int32_t* tile_order) {
    const float4* rec = reinterpret_cast<const float4*>(records);
    if (channels == 1) {
        if (iso)
            launch_splat_backward_t<1, true>(rule, ranges, point_list, rec, k, dxy2, grad, out, stream, tile_order);
        else
            launch_splat_backward_t<1, false>(rule, ranges, point_list, rec, k, dxy2, grad, out, stream, tile_order);
    } else {
        if (iso)
            launch_splat_backward_t<3, true>(rule, ranges, point_list, rec, k, dxy2, grad, out, stream, tile_order);
        else
            launch_splat_backward_t<3, false>(rule, ranges, point_list, rec, k, dxy2, grad, out, stream, tile_order);
    }
}

}  // namespace cvqpg

// ===========================================================================
// C ABI
// ===========================================================================
using namespace cvqpg;

extern "C" const char* cvqpg_status_string(int status) {
    switch (status) {
        case CVQPG_OK: return "ok";
        case CVQPG_ERR_ARG: return "invalid argument";
        case CVQPG_ERR_CHANNELS: return "qpf rasterizer supports 1 or 3 channels";
        case CVQPG_ERR_WORKSPACE: return "workspace too small";
        case CVQPG_ERR_CUDA: return "CUDA launch failed";
        case CVQPG_ERR_UNSUPPORTED: return "unsupported size";
        default: return "unknown status";
    }
}

extern "C" int cvqpg_version(void) { return 100; }

static size_t render_ws_bytes(int n, int cap) {
    Carver cv(nullptr, 0);
    cv.take<float>((size_t)(n > 0 ? n : 1) * kRecordFloats);
    carve_bin_workspace(cv, n, cap);
    return cv.off + 256;
}

extern "C" int cvqpg_render_workspace_size(int n, int width, int height, int pair_capacity, size_t* bytes) {
    if (n < 0 || width <= 0 || height <= 0 || pair_capacity < 0 || !bytes) return CVQPG_ERR_ARG;
    *bytes = render_ws_bytes(n, pair_capacity);
    return CVQPG_OK;
}

extern "C" int cvqpg_render_num_lists(int cull_mode, int width, int height) {
    cull_mode &= ~CVQPG_PHASE_ISO;
    if (cull_mode < 0 || cull_mode > 2 || width <= 0 || height <= 0) return -1;
    BinRule r = make_bin_rule(cull_mode, width, height, nullptr, nullptr);
    return bin_rule_lists(r);
}

extern "C" int cvqpg_render_forward_cull(const float* means_2d, const float* inv_cov, const float* colours,
                                         const float* phase, const float* opacities, const float* curvature,
                                         const float* area, int cull_mode, const int32_t* radii,
                                         const float* radius3, const float* k, float dxy2, int n, int width,
                                         int height, int channels, float* out_field, int32_t* point_list,
                                         int pair_capacity, int32_t* ranges, int32_t* pair_count, void* workspace,
                                         size_t workspace_bytes, void* stream_) {
    if (channels != 1 && channels != 3) return CVQPG_ERR_CHANNELS;
    const bool iso = (cull_mode & CVQPG_PHASE_ISO) != 0;
    cull_mode &= ~CVQPG_PHASE_ISO;
    if (n < 0 || width <= 0 || height <= 0 || pair_capacity < 0 || cull_mode < 0 || cull_mode > 2)
        return CVQPG_ERR_ARG;
    if (!k || !out_field || !ranges || !pair_count) return CVQPG_ERR_ARG;
    if (n > 0 && (!means_2d || !inv_cov || !colours || !phase || !opacities || !curvature || !area ||
                  !workspace || (pair_capacity > 0 && !point_list)))
        return CVQPG_ERR_ARG;
    if (n > 0 && cull_mode == CVQPG_CULL_CUDA16_5SIGMA && !radii) return CVQPG_ERR_ARG;
    if (n > 0 && cull_mode == CVQPG_CULL_TORCH64_3SIGMA && !radius3) return CVQPG_ERR_ARG;
    if (workspace_bytes < render_ws_bytes(n, pair_capacity)) return CVQPG_ERR_WORKSPACE;
    cudaStream_t stream = (cudaStream_t)stream_;
    Carver cv(workspace, workspace_bytes);
    float* rec = cv.take<float>((size_t)(n > 0 ? n : 1) * kRecordFloats);
    BinWorkspace ws = carve_bin_workspace(cv, n, pair_capacity);
    BinRule rule = make_bin_rule(cull_mode, width, height, radii, radius3);
    launch_pack_records(channels, n, means_2d, inv_cov, colours, phase, opacities, curvature, area, rec, stream);
    launch_tile_count(rule, rec, n, ws.tiles_touched, stream);
    launch_binning(rule, rec, ws, point_list, ranges, pair_count, stream);
    launch_splat_forward(channels, rule, ranges, point_list, rec, k, dxy2, reinterpret_cast<float2*>(out_field),
                         stream, iso);
    return launch_status();
}

extern "C" int cvqpg_render_forward(const float* means_2d, const float* inv_cov, const float* colours,
                                    const float* phase, const float* opacities, const float* curvature,
                                    const float* area, const int32_t* radii, const float* k, float dxy2, int n,
                                    int width, int height, int channels, float* out_field, int32_t* point_list,
                                    int pair_capacity, int32_t* ranges, int32_t* pair_count, void* workspace,
                                    size_t workspace_bytes, void* stream) {
    return cvqpg_render_forward_cull(means_2d, inv_cov, colours, phase, opacities, curvature, area,
                                     CVQPG_CULL_CUDA16_5SIGMA, radii, nullptr, k, dxy2, n, width, height, channels,
                                     out_field, point_list, pair_capacity, ranges, pair_count, workspace,
                                     workspace_bytes, stream);
}

extern "C" int cvqpg_render_backward_workspace_size(int n, size_t* bytes) {
    if (n < 0 || !bytes) return CVQPG_ERR_ARG;
    *bytes = (size_t)(n > 0 ? n : 1) * kRecordFloats * sizeof(float) + 256;
    return CVQPG_OK;
}

extern "C" int cvqpg_render_backward_cull(const float* grad_field, const float* means_2d, const float* inv_cov,
                                          const float* colours, const float* phase, const float* opacities,
                                          const float* curvature, const float* area, const float* k,
                                          int cull_mode, const int32_t* point_list, const int32_t* ranges,
                                          float dxy2, int n, int width, int height, int channels, float* d_means,
                                          float* d_inv_cov, float* d_colours, float* d_phase, float* d_opacities,
                                          float* d_curvature, float* d_area, void* workspace,
                                          size_t workspace_bytes, void* stream_) {
    if (channels != 1 && channels != 3) return CVQPG_ERR_CHANNELS;
    const bool iso = (cull_mode & CVQPG_PHASE_ISO) != 0;
    cull_mode &= ~CVQPG_PHASE_ISO;
    if (n < 0 || width <= 0 || height <= 0 || cull_mode < 0 || cull_mode > 2) return CVQPG_ERR_ARG;
    if (n == 0) return CVQPG_OK;
    if (!grad_field || !means_2d || !inv_cov || !colours || !phase || !opacities || !curvature || !area || !k ||
        !point_list || !ranges || !d_means || !d_inv_cov || !d_colours || !d_phase || !d_opacities ||
        !d_curvature || !d_area || !workspace)
        return CVQPG_ERR_ARG;
    size_t need = 0;
    cvqpg_render_backward_workspace_size(n, &need);
    if (workspace_bytes < need) return CVQPG_ERR_WORKSPACE;
    cudaStream_t stream = (cudaStream_t)stream_;
    Carver cv(workspace, workspace_bytes);
    float* rec = cv.take<float>((size_t)n * kRecordFloats);
    const int C = channels;
    cudaMemsetAsync(d_means, 0, sizeof(float) * 2 * n, stream);
    cudaMemsetAsync(d_inv_cov, 0, sizeof(float) * 3 * n, stream);
    cudaMemsetAsync(d_colours, 0, sizeof(float) * C * n, stream);
    cudaMemsetAsync(d_phase, 0, sizeof(float) * C * n, stream);
    cudaMemsetAsync(d_opacities, 0, sizeof(float) * n, stream);
    cudaMemsetAsync(d_curvature, 0, sizeof(float) * n, stream);
    cudaMemsetAsync(d_area, 0, sizeof(float) * n, stream);
    launch_pack_records(C, n, means_2d, inv_cov, colours, phase, opacities, curvature, area, rec, stream);
    BinRule rule = make_bin_rule(cull_mode, width, height, nullptr, nullptr);
    SplatGrads out{d_means, d_inv_cov, d_colours, d_phase, d_opacities, d_curvature, d_area};
    launch_splat_backward(C, rule, ranges, point_list, rec, k, dxy2, reinterpret_cast<const float2*>(grad_field),
                          out, stream, iso);
    return launch_status();
}

extern "C" int cvqpg_render_backward(const float* grad_field, const float* means_2d, const float* inv_cov,
                                     const float* colours, const float* phase, const float* opacities,
                                     const float* curvature, const float* area, const float* k,
                                     const int32_t* point_list, const int32_t* ranges, float dxy2, int n, int width,
                                     int height, int channels, float* d_means, float* d_inv_cov, float* d_colours,
                                     float* d_phase, float* d_opacities, float* d_curvature, float* d_area,
                                     void* workspace, size_t workspace_bytes, void* stream) {
    return cvqpg_render_backward_cull(grad_field, means_2d, inv_cov, colours, phase, opacities, curvature, area, k,
                                      CVQPG_CULL_CUDA16_5SIGMA, point_list, ranges, dxy2, n, width, height,
                                      channels, d_means, d_inv_cov, d_colours, d_phase, d_opacities, d_curvature,
                                      d_area, workspace, workspace_bytes, stream);
}

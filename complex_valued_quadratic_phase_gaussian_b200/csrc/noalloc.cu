// Allocation-free variant of cvqpg_render_forward.
//
// Some callers cannot allocate device memory at the point where they render:
// code that runs inside a fixed memory budget reserved up front (for example a
// serving process whose allocator is capped, or a plugin host that owns every
// allocation and hands out only its own buffers), or code that must not call
// cudaMalloc because it would synchronise the device or fragment a pool the
// host manages. For them this entry point takes only the inputs and outputs of
// cvqpg_render_forward and keeps its scratch (packed records, tile counts,
// scan sums, sort keys and values, radix histograms) in one file-scope device
// array of fixed size. That array is part of the library image: every GPU that
// loads the library holds it until the process exits.
#include <mutex>

#include "raster.cuh"

namespace cvqpg {

// Limits of the allocation-free path (scratch sized for them, ~5.4 MiB).
constexpr int kNoAllocMaxGaussians = 16384;
constexpr int kNoAllocMaxPairs = 262144;

// Bytes the render scratch needs at the limits above (same carving as the
// workspace path: records, then the binning buffers).
static size_t noalloc_scratch_bytes(int n, int cap) {
    Carver cv(nullptr, 0);
    cv.take<float>((size_t)(n > 0 ? n : 1) * kRecordFloats);
    carve_bin_workspace(cv, n, cap);
    return cv.off + 256;
}

constexpr size_t kNoAllocScratchBytes = 5u * 1024u * 1024u + 512u * 1024u;

// The scratch. In host code this name is only a stand-in for the symbol; the
// device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_render_scratch[kNoAllocScratchBytes];

static std::mutex g_scratch_mutex;
static void* g_scratch_addr[64] = {nullptr};

// Device address of the scratch on the current device, looked up once per
// device (the first call on a device does this set-up). The address is kept
// for the life of the process, so the entry point must not be used on a device
// after cudaDeviceReset on it (the reset ends the context the address belongs to).
static int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return CVQPG_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_render_scratch) != cudaSuccess || !p) return CVQPG_ERR_CUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return CVQPG_OK;
}

}  // namespace cvqpg

using namespace cvqpg;

extern "C" int cvqpg_render_forward_noalloc(const float* means_2d, const float* inv_cov, const float* colours,
                                            const float* phase, const float* opacities, const float* curvature,
                                            const float* area, const int32_t* radii, const float* k, float dxy2,
                                            int n, int width, int height, int channels, float* out_field,
                                            int32_t* point_list, int pair_capacity, int32_t* ranges,
                                            int32_t* pair_count, void* stream_) {
    if (channels != 1 && channels != 3) return CVQPG_ERR_CHANNELS;
    if (n < 0 || width <= 0 || height <= 0 || pair_capacity < 0) return CVQPG_ERR_ARG;
    if (n > kNoAllocMaxGaussians || pair_capacity > kNoAllocMaxPairs) return CVQPG_ERR_UNSUPPORTED;
    if (!k || !out_field || !ranges || !pair_count) return CVQPG_ERR_ARG;
    if (n > 0 && (!means_2d || !inv_cov || !colours || !phase || !opacities || !curvature || !area || !radii ||
                  (pair_capacity > 0 && !point_list)))
        return CVQPG_ERR_ARG;
    const size_t need = noalloc_scratch_bytes(n, pair_capacity);
    if (need > kNoAllocScratchBytes) return CVQPG_ERR_UNSUPPORTED;
    void* scratch = nullptr;
    const int st = scratch_address(&scratch);
    if (st != CVQPG_OK) return st;
    cudaStream_t stream = (cudaStream_t)stream_;
    // Every scratch buffer below is written before it is read (tile counts by
    // the count kernel, sums by the scan, keys/values by the pair emission,
    // histograms by the upsweep), so nothing has to be cleared between calls.
    Carver cv(scratch, kNoAllocScratchBytes);
    float* rec = cv.take<float>((size_t)(n > 0 ? n : 1) * kRecordFloats);
    BinWorkspace ws = carve_bin_workspace(cv, n, pair_capacity);
    BinRule rule = make_bin_rule(CVQPG_CULL_CUDA16_5SIGMA, width, height, radii, nullptr);
    launch_pack_records(channels, n, means_2d, inv_cov, colours, phase, opacities, curvature, area, rec, stream);
    launch_tile_count(rule, rec, n, ws.tiles_touched, stream);
    launch_binning(rule, rec, ws, point_list, ranges, pair_count, stream);
    launch_splat_forward(channels, rule, ranges, point_list, rec, k, dxy2, reinterpret_cast<float2*>(out_field),
                         stream);
    return launch_status();
}

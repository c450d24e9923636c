// Phase-only hologram (POH) export: the product step after a fit
// (export_poh.py:110-119, 175-194). From the splat field [C,H,W]:
//   padded field = soft window pad + amplitude clamp (as the propagation's first pass),
//   phase = angle mod 2 pi, amplitude = |.| (<= 1 after the clamp),
//   DPAC (double-phase amplitude coding): phase -/+ arccos(amplitude) on a
//   checkerboard (minus where y + x is even), wrapped to [0, 2 pi),
//   level = round(poh / (2 pi) * 256) mod 256 (8-bit, round half to even).
// Optionally also writes the phase-only field exp(i 2 pi level / 256) that the
// reference reconstructs through a Fourier aperture (input_mode 1 of the
// propagation), so the 8-bit hologram's reconstruction needs no host round trip.
#include <algorithm>

#include "blasm_cols.cuh"

namespace cvqpg {

__global__ void poh_encode_kernel(BlasmDev d, const float2* __restrict__ field, uint8_t* __restrict__ levels,
                                  float2* __restrict__ phase_field) {
    const int pH = d.pH, pW = d.pW;
    const size_t n = (size_t)d.C * pH * pW;
    const float two_pi = 6.28318530717958647692f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % pW);
        const int y = (int)((i / pW) % pH);
        const int c = (int)(i / ((size_t)pH * pW));
        const int yy = min(max(y - d.pad_h, 0), d.H - 1);
        const int xx = min(max(x - d.pad_w, 0), d.W - 1);
        const float w = __ldg(&d.wy[y]) * __ldg(&d.wx[x]);
        const float2 u0 = __ldg(&field[((size_t)c * d.H + yy) * d.W + xx]);
        // complex-times-real as torch evaluates it, (a w - b 0, a 0 + b w): where the taper is exactly 0
        // the signed zeros (and so the angle, 0 or pi) match the reference's
        const float2 u = clamp_amplitude(make_float2(u0.x * w - u0.y * 0.0f, u0.x * 0.0f + u0.y * w));
        float phase = atan2f(u.y, u.x);
        phase = phase - floorf(phase / two_pi) * two_pi;  // torch '%': result in [0, 2 pi)
        const float amp = fminf(sqrtf(u.x * u.x + u.y * u.y), 1.0f);
        const float offset = acosf(amp);
        float v = ((y ^ x) & 1) == 0 ? phase - offset : phase + offset;
        v = v - floorf(v / two_pi) * two_pi;
        const int g = ((int)rintf(v / two_pi * 256.0f)) & 255;
        levels[i] = (uint8_t)g;
        if (phase_field) {
            float s, co;
            sincospif((float)g / 128.0f, &s, &co);
            phase_field[i] = make_float2(co, s);
        }
    }
}

}  // namespace cvqpg

using namespace cvqpg;

extern "C" int cvqpg_poh_encode(const cvqpg_blasm_params* prm, const void* tables, size_t table_bytes,
                                const float* field, uint8_t* levels, float* phase_field, void* stream) {
    BlasmDev d;
    const int st = blasm_make_dev(prm, tables, table_bytes, &d);
    if (st != CVQPG_OK) return st;
    if (!field || !levels) return CVQPG_ERR_ARG;
    if (d.input_mode != 0) return CVQPG_ERR_ARG;  // needs the splat field [C,H,W]
    const size_t n = (size_t)d.C * d.pH * d.pW;
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
    poh_encode_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(d, (const float2*)field, levels,
                                                               (float2*)phase_field);
    return launch_status();
}

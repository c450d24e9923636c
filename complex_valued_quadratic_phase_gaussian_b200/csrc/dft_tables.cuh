// cos/sin(2*pi*q/R) for the small odd DFTs and radix-8/16 internal twiddles.
// Values computed in double precision and rounded once to float. Indices are
// compile-time constants at every call site (fully unrolled loops), so the
// lookups fold into immediates.
#pragma once

namespace cvqpg {

template <int R> struct DftTab;

template <> struct DftTab<3> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[3] = {1.000000000e+00f, -5.000000000e-01f, -5.000000000e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[3] = {0.000000000e+00f, 8.660254038e-01f, -8.660254038e-01f};
        return t[q];
    }
};
template <> struct DftTab<5> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[5] = {1.000000000e+00f, 3.090169944e-01f, -8.090169944e-01f, -8.090169944e-01f, 3.090169944e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[5] = {0.000000000e+00f, 9.510565163e-01f, 5.877852523e-01f, -5.877852523e-01f, -9.510565163e-01f};
        return t[q];
    }
};
template <> struct DftTab<7> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[7] = {1.000000000e+00f, 6.234898019e-01f, -2.225209340e-01f, -9.009688679e-01f, -9.009688679e-01f, -2.225209340e-01f, 6.234898019e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[7] = {0.000000000e+00f, 7.818314825e-01f, 9.749279122e-01f, 4.338837391e-01f, -4.338837391e-01f, -9.749279122e-01f, -7.818314825e-01f};
        return t[q];
    }
};
template <> struct DftTab<8> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[8] = {1.000000000e+00f, 7.071067812e-01f, 6.123233996e-17f, -7.071067812e-01f, -1.000000000e+00f, -7.071067812e-01f, -1.836970199e-16f, 7.071067812e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[8] = {0.000000000e+00f, 7.071067812e-01f, 1.000000000e+00f, 7.071067812e-01f, 1.224646799e-16f, -7.071067812e-01f, -1.000000000e+00f, -7.071067812e-01f};
        return t[q];
    }
};
template <> struct DftTab<11> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[11] = {1.000000000e+00f, 8.412535328e-01f, 4.154150130e-01f, -1.423148383e-01f, -6.548607339e-01f, -9.594929736e-01f, -9.594929736e-01f, -6.548607339e-01f, -1.423148383e-01f, 4.154150130e-01f, 8.412535328e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[11] = {0.000000000e+00f, 5.406408175e-01f, 9.096319954e-01f, 9.898214419e-01f, 7.557495744e-01f, 2.817325568e-01f, -2.817325568e-01f, -7.557495744e-01f, -9.898214419e-01f, -9.096319954e-01f, -5.406408175e-01f};
        return t[q];
    }
};
template <> struct DftTab<13> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[13] = {1.000000000e+00f, 8.854560257e-01f, 5.680647467e-01f, 1.205366803e-01f, -3.546048870e-01f, -7.485107482e-01f, -9.709418174e-01f, -9.709418174e-01f, -7.485107482e-01f, -3.546048870e-01f, 1.205366803e-01f, 5.680647467e-01f, 8.854560257e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[13] = {0.000000000e+00f, 4.647231720e-01f, 8.229838659e-01f, 9.927088741e-01f, 9.350162427e-01f, 6.631226582e-01f, 2.393156643e-01f, -2.393156643e-01f, -6.631226582e-01f, -9.350162427e-01f, -9.927088741e-01f, -8.229838659e-01f, -4.647231720e-01f};
        return t[q];
    }
};
template <> struct DftTab<16> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[16] = {1.000000000e+00f, 9.238795325e-01f, 7.071067812e-01f, 3.826834324e-01f, 6.123233996e-17f, -3.826834324e-01f, -7.071067812e-01f, -9.238795325e-01f, -1.000000000e+00f, -9.238795325e-01f, -7.071067812e-01f, -3.826834324e-01f, -1.836970199e-16f, 3.826834324e-01f, 7.071067812e-01f, 9.238795325e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[16] = {0.000000000e+00f, 3.826834324e-01f, 7.071067812e-01f, 9.238795325e-01f, 1.000000000e+00f, 9.238795325e-01f, 7.071067812e-01f, 3.826834324e-01f, 1.224646799e-16f, -3.826834324e-01f, -7.071067812e-01f, -9.238795325e-01f, -1.000000000e+00f, -9.238795325e-01f, -7.071067812e-01f, -3.826834324e-01f};
        return t[q];
    }
};
template <> struct DftTab<17> {
    __host__ __device__ __forceinline__ static constexpr float c(int q) {
        constexpr float t[17] = {1.000000000e+00f, 9.324722294e-01f, 7.390089172e-01f, 4.457383558e-01f, 9.226835946e-02f, -2.736629901e-01f, -6.026346364e-01f, -8.502171357e-01f, -9.829730997e-01f, -9.829730997e-01f, -8.502171357e-01f, -6.026346364e-01f, -2.736629901e-01f, 9.226835946e-02f, 4.457383558e-01f, 7.390089172e-01f, 9.324722294e-01f};
        return t[q];
    }
    __host__ __device__ __forceinline__ static constexpr float s(int q) {
        constexpr float t[17] = {0.000000000e+00f, 3.612416662e-01f, 6.736956436e-01f, 8.951632914e-01f, 9.957341763e-01f, 9.618256432e-01f, 7.980172273e-01f, 5.264321629e-01f, 1.837495178e-01f, -1.837495178e-01f, -5.264321629e-01f, -7.980172273e-01f, -9.618256432e-01f, -9.957341763e-01f, -8.951632914e-01f, -6.736956436e-01f, -3.612416662e-01f};
        return t[q];
    }
};

}  // namespace cvqpg

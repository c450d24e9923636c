// Column kernels of the BLASM passes with the FFT plan fixed at compile time
// (HeadCT, and the four-column kernels of blasm_cols4.cuh): the strides, index
// splits and padded addresses of every pass are constants. This unit holds the
// dispatcher and the column length of the 1920x1080 fit with the default guard
// band: 2 x 1408 = 2816 = 16 x 16 x 11.
#include "blasm_cols4.cuh"

namespace cvqpg {

bool launch_cols_ct(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                    cudaStream_t s) {
    if (d.NH == 2816 && col_split_is(cs, 11, 1, {16, 16})) {
        if (d.G == 4)
            launch_cols4_t<11>(adjoint, d, in, out, s);  // four adjacent columns per CTA, plan 16 x 11 x 16
        else
            launch_cols_reg_t<11, 1, HeadCT<2816, 16, 16>>(adjoint, d, cs, in, out, s);
        return true;
    }
    if (d.NH == 1664) return launch_cols_ct_1664(adjoint, d, cs, in, out, s);
    if (d.NH == 2176) return launch_cols_ct_2176(adjoint, d, cs, in, out, s);
    if (d.NH == 1152) return launch_cols_ct_1152(adjoint, d, cs, in, out, s);
    return false;
}

}  // namespace cvqpg

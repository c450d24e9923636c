// Column kernels of the BLASM passes with the FFT plan fixed at compile time
// (HeadCT2): the strides, index splits and padded addresses of every pass are
// constants. Instantiated for the column length of the 1920x1080 fit with the
// default guard band: 2 x 1408 = 2816 = 16 x 16 x 11 (radix 11 in registers).
#include "blasm_cols.cuh"

namespace cvqpg {

bool launch_cols_ct(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                    cudaStream_t s) {
    if (cs.head_npass != 2 || cs.mb != 1) return false;
    const int ra = (int)(cs.head_code & 31ull), rb = (int)((cs.head_code >> 5) & 31ull);
    if (d.NH == 2816 && cs.rl == 11 && ra == 16 && rb == 16) {
        launch_cols_reg_t<11, 1, HeadCT2<2816, 16, 16>>(adjoint, d, cs, in, out, s);
        return true;
    }
    return false;
}

}  // namespace cvqpg

// Compile-time column plan (HeadCT) for the column length of 256x256 images (pad 576).
#include "blasm_cols.cuh"

namespace cvqpg {

bool launch_cols_ct_1152(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                       cudaStream_t s) {
    if (!col_split_is(cs, 3, 2, {16, 8, 3})) return false;
    launch_cols_reg_t<3, 2, HeadCT<1152, 16, 8, 3>>(adjoint, d, cs, in, out, s);
    return true;
}

}  // namespace cvqpg

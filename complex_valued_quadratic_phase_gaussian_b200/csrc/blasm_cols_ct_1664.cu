// Compile-time column plan (HeadCT) for the column length of 512x512 images (pad 832).
#include "blasm_cols.cuh"

namespace cvqpg {

bool launch_cols_ct_1664(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                       cudaStream_t s) {
    if (!col_split_is(cs, 8, 1, {16, 13})) return false;
    launch_cols_reg_t<8, 1, HeadCT<1664, 16, 13>>(adjoint, d, cs, in, out, s);
    return true;
}

}  // namespace cvqpg

// Compile-time column plan (HeadCT) for the column length of 768-row images (pad 1088).
#include "blasm_cols.cuh"

namespace cvqpg {

bool launch_cols_ct_2176(bool adjoint, const BlasmDev& d, const ColSplit& cs, const float2* in, float2* out,
                       cudaStream_t s) {
    if (!col_split_is(cs, 16, 1, {8, 17})) return false;
    launch_cols_reg_t<16, 1, HeadCT<2176, 8, 17>>(adjoint, d, cs, in, out, s);
    return true;
}

}  // namespace cvqpg

// Register-spectrum column kernels of the BLASM passes for last radix 11
// (one translation unit per radix so the variants compile in parallel).
#include "blasm_cols.cuh"

namespace cvqpg {
CVQPG_DEFINE_COLS_REG(11)
}  // namespace cvqpg

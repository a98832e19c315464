// Line-pass kernels for lines of 384 points (radices 24, 4, 4; see line_kernels.cuh).
#include "line_kernels.cuh"

namespace mtb {
template void rows_dispatch_mode<384>(RowMode, const RowArgs&, int, cudaStream_t);
template void cols_dispatch_flags<384>(int, const ColArgs&, int, cudaStream_t);
template int cols_det_width<384>();
}  // namespace mtb

// Line-pass kernels for lines of 2048 points (see line_kernels.cuh).
#include "line_kernels.cuh"

namespace mtb {
template void rows_dispatch_mode<2048>(RowMode, const RowArgs&, int, cudaStream_t);
template void cols_dispatch_flags<2048>(int, const ColArgs&, int, cudaStream_t);
template int cols_det_width<2048>();
}  // namespace mtb

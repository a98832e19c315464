// Line-pass kernels for lines of 1024 points (see line_kernels.cuh).
#include "line_kernels.cuh"

namespace mtb {
template void rows_dispatch_mode<1024>(RowMode, const RowArgs&, int, cudaStream_t);
template void cols_dispatch_flags<1024>(int, const ColArgs&, int, cudaStream_t);
template int cols_det_width<1024>();
}  // namespace mtb

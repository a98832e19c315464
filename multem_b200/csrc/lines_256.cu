// Line-pass kernels for lines of 256 points (see line_kernels.cuh).
#include "line_kernels.cuh"

namespace mtb {
template void rows_dispatch_mode<256>(RowMode, const RowArgs&, int, cudaStream_t);
template void cols_dispatch_flags<256>(int, const ColArgs&, int, cudaStream_t);
template int cols_det_width<256>();
}  // namespace mtb

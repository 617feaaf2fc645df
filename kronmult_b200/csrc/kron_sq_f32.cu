// FP32 storage / FP32 accumulation square-shape kernels (batched layout).
#include "kron_sq_table.cuh"

namespace kron {
SqKernelInfo sq_kernel_f32(int D, int N) { return sq_pick<float, PREC_F32, false>(D, N); }
} // namespace kron

// Split hi+lo FP32 arithmetic on FP64 storage, square shapes (batched layout).
#include "kron_sq_table.cuh"

namespace kron {
SqKernelInfo sq_kernel_split(int D, int N) { return sq_pick<double, PREC_SPLIT, false>(D, N); }
} // namespace kron

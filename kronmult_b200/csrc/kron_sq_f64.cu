// FP64 square-shape kernels (distinct outputs and merging/atomic outputs).
#include "kron_sq_table.cuh"

namespace kron {
SqKernelInfo sq_kernel_f64(int D, int N, bool merge)
{
  return merge ? sq_pick<double, PREC_F64, true>(D, N) : sq_pick<double, PREC_F64, false>(D, N);
}
} // namespace kron

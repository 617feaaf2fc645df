// Compile-time (d, n) kernel tables for the square layouts.
#pragma once

#include "kron_kernels.cuh"

namespace kron {

struct SqKernelInfo
{
  const void *fn;     // kernel entry (nullptr: (d, n) not instantiated / does not fit)
  int GS;             // threads per entry group
  size_t group_bytes; // shared memory per group
};

constexpr size_t SMEM_OPTIN_MAX = 232448; // 227 KB per block on sm_100

SqKernelInfo sq_kernel_f64(int D, int N, bool merge);
SqKernelInfo sq_kernel_f32(int D, int N);
SqKernelInfo sq_kernel_split(int D, int N);

template <typename T, int PREC, bool MERGE, int D, int N>
SqKernelInfo sq_make()
{
  using S = SqShape<T, D, N, PREC, MERGE>;
  if constexpr (S::GROUP_BYTES <= SMEM_OPTIN_MAX)
    return {reinterpret_cast<const void *>(&kron_sq_kernel<T, D, N, PREC, MERGE>), S::GS,
            S::GROUP_BYTES};
  else
    return {nullptr, 0, 0};
}

template <typename T, int PREC, bool MERGE, int D>
SqKernelInfo sq_pick_n(int N)
{
  switch (N)
  {
  case 2: return sq_make<T, PREC, MERGE, D, 2>();
  case 3: return sq_make<T, PREC, MERGE, D, 3>();
  case 4: return sq_make<T, PREC, MERGE, D, 4>();
  case 5: return sq_make<T, PREC, MERGE, D, 5>();
  case 6: return sq_make<T, PREC, MERGE, D, 6>();
  case 7: return sq_make<T, PREC, MERGE, D, 7>();
  case 8: return sq_make<T, PREC, MERGE, D, 8>();
  default: return {nullptr, 0, 0};
  }
}

template <typename T, int PREC, bool MERGE>
SqKernelInfo sq_pick(int D, int N)
{
  switch (D)
  {
  case 1: return sq_pick_n<T, PREC, MERGE, 1>(N);
  case 2: return sq_pick_n<T, PREC, MERGE, 2>(N);
  case 3: return sq_pick_n<T, PREC, MERGE, 3>(N);
  case 4: return sq_pick_n<T, PREC, MERGE, 4>(N);
  case 5: return sq_pick_n<T, PREC, MERGE, 5>(N);
  case 6: return sq_pick_n<T, PREC, MERGE, 6>(N);
  default: return {nullptr, 0, 0};
  }
}

} // namespace kron

// Device-side pointer arrays from integer lists (no reference counterpart:
// the reference's tests build Aparray / pdXarray / pdYarray on the host and
// copy them over, test_kronmult6_xbatched.cpp:231-271).  A caller that holds
// an element grid as index lists (output element i, input element j, pool
// matrix per dimension) uploads the integers once and gets the pointer
// arrays of the xbatched / pbatched layouts built on the device:
//   pX[k]         = X + xlist[k] * xstride          (xlist NULL: k)
//   pY[k]         = Y + ylist[k] * ystride          (ylist NULL: k)
//   pA[l + k * d] = A + alist[l + k * d] * astride  (alist NULL: l + k * d)
#include "kron_launch.h"
#include "kronmult.h"

namespace {

__global__ void kron_pointers_kernel(int d, int batch, const double *A, long long astride,
                                     const int *alist, const double *X, long long xstride,
                                     const int *xlist, double *Y, long long ystride,
                                     const int *ylist, const double **pA, double **pX,
                                     double **pY)
{
  const long long na = (long long)batch * d;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < na;
       i += (long long)gridDim.x * blockDim.x)
  {
    if (pA)
      pA[i] = A + (alist ? (long long)alist[i] : i) * astride;
    if (i < batch)
    {
      if (pX)
        pX[i] = const_cast<double *>(X) + (xlist ? (long long)xlist[i] : i) * xstride;
      if (pY)
        pY[i] = Y + (ylist ? (long long)ylist[i] : i) * ystride;
    }
  }
}

} // namespace

extern "C" int kron_build_pointers_async(int d, int batchCount, double const *A, long long astride,
                                         int const alist[], double const *X, long long xstride,
                                         int const xlist[], double *Y, long long ystride,
                                         int const ylist[], double const *Aarray_out[],
                                         double *Xarray_out[], double *Yarray_out[],
                                         kron_stream_t stream)
{
  if (d < 1 || d > kron::MAXD || batchCount < 0 || astride < 0 || xstride < 0 || ystride < 0)
    return KRON_ERROR_INVALID_VALUE;
  if ((Aarray_out && !A) || (Xarray_out && !X) || (Yarray_out && !Y))
    return KRON_ERROR_INVALID_VALUE;
  if (batchCount == 0 || (!Aarray_out && !Xarray_out && !Yarray_out))
    return KRON_SUCCESS;
  const long long na = (long long)batchCount * d;
  const int block    = 256;
  const long long grid =
      std::min<long long>((na + block - 1) / block, (long long)kron::device_info().sms * 8);
  kron_pointers_kernel<<<(unsigned)grid, block, 0, (cudaStream_t)stream>>>(
      d, batchCount, A, astride, alist, X, xstride, xlist, Y, ystride, ylist, Aarray_out,
      Xarray_out, Yarray_out);
  return cudaGetLastError() == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

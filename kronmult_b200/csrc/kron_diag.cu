// Diagnostics: live measurement of this GPU's FP64 throughput, the
// denominator of the compute roofline for the FP64 kernels (the driver's
// peak file only has HBM and bf16 figures).
//
//   kron_measure_fp64_peak(&tensor, &cuda_core)
//
// times independent chains of mma.sync.m16n8k8.f64 (FP64 tensor path) and of
// FP64 fma (CUDA cores) over every SM, 8 blocks of 256 threads per SM, and
// returns TFLOP/s.  It allocates a small device buffer for the kernels'
// (never taken) result store.
#include <cuda_runtime.h>

#include "kron_internal.cuh"

namespace {

__global__ void probe_dmma(double *out, int iters)
{
  double a0 = threadIdx.x * 1e-3, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, b0 = 1.0, b1 = 0.5;
  double c[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
      c[i][j] = 0;
  for (int it = 0; it < iters; it++)
  {
#pragma unroll
    for (int i = 0; i < 4; i++)
      asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
                   "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                   : "+d"(c[i][0]), "+d"(c[i][1]), "+d"(c[i][2]), "+d"(c[i][3])
                   : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
      s += c[i][j];
  if (s == 123.456)
    out[threadIdx.x] = s;
}

__global__ void probe_dfma(double *out, int iters, double a, double b)
{
  double acc[8];
#pragma unroll
  for (int i = 0; i < 8; i++)
    acc[i] = threadIdx.x * 1e-9 + i;
  for (int it = 0; it < iters; it++)
  {
#pragma unroll
    for (int i = 0; i < 8; i++)
      acc[i] = fma(acc[i], a, b);
  }
  double s = 0;
#pragma unroll
  for (int i = 0; i < 8; i++)
    s += acc[i];
  if (s == 123.456)
    out[threadIdx.x] = s;
}

} // namespace

extern "C" int kron_measure_fp64_peak(double *tensor_tflops, double *cuda_core_tflops)
{
  if (!tensor_tflops || !cuda_core_tflops)
    return KRON_ERROR_INVALID_VALUE;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  double *out = nullptr;
  if (kron::dev_malloc((void **)&out, 256 * sizeof(double)) != cudaSuccess)
    return KRON_ERROR_ALLOC;
  cudaEvent_t s = nullptr, e = nullptr;
  cudaEventCreate(&s);
  cudaEventCreate(&e);
  const int grid = sms * 8, block = 256, iters = 4000;
  float ms = 0.f;
  double best_t = 0.0, best_c = 0.0;
  for (int rep = 0; rep < 3; rep++)
  {
    cudaEventRecord(s);
    probe_dmma<<<grid, block>>>(out, iters);
    cudaEventRecord(e);
    cudaEventSynchronize(e);
    cudaEventElapsedTime(&ms, s, e);
    double fl = 2.0 * 16 * 8 * 8 * 4 * (double)iters * grid * (block / 32);
    if (ms > 0 && rep > 0)
      best_t = std::max(best_t, fl / ms / 1e9);
    cudaEventRecord(s);
    probe_dfma<<<grid, block>>>(out, iters * 4, 1.0000001, 1e-9);
    cudaEventRecord(e);
    cudaEventSynchronize(e);
    cudaEventElapsedTime(&ms, s, e);
    fl = 2.0 * 8 * (double)iters * 4 * grid * block;
    if (ms > 0 && rep > 0)
      best_c = std::max(best_c, fl / ms / 1e9);
  }
  cudaError_t err = cudaGetLastError();
  cudaEventDestroy(s);
  cudaEventDestroy(e);
  kron::dev_free(out);
  *tensor_tflops    = best_t;
  *cuda_core_tflops = best_c;
  return err == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

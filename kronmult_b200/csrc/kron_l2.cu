// Repeated application with the same operator (no reference counterpart):
// an iterative solver applies kron(A_1..A_d) to a new X every iteration, so
// the factors (and any other fixed operand) can stay in L2 between calls.
// kron_l2_persist_async marks a byte range persisting for the kernels this
// library launches on `stream` (a CUDA access-policy window on the stream,
// captured into graphs with the kernels) and sets this context's persisting
// L2 carve-out to the range (capped at the device maximum).  Both settings
// belong to this process's context; kron_l2_persist_reset removes the window,
// returns the lines to normal and sets the carve-out back to 0.
#include "kron_launch.h"
#include "kronmult.h"

extern "C" int kron_l2_persist_async(const void *ptr, size_t bytes, kron_stream_t stream)
{
  if (!ptr || bytes == 0)
    return KRON_ERROR_INVALID_VALUE;
  int dev = 0, maxwin = 0, maxpersist = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&maxpersist, cudaDevAttrMaxPersistingL2CacheSize, dev) !=
          cudaSuccess)
    return KRON_ERROR_LAUNCH;
  if (maxwin <= 0 || maxpersist <= 0)
    return KRON_ERROR_NOT_SUPPORTED;
  const size_t win   = bytes < (size_t)maxwin ? bytes : (size_t)maxwin;
  const size_t carve = win < (size_t)maxpersist ? win : (size_t)maxpersist;
  if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, carve) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  cudaStreamAttrValue a = {};
  a.accessPolicyWindow.base_ptr  = const_cast<void *>(ptr);
  a.accessPolicyWindow.num_bytes = win;
  // lines beyond the carve-out are fetched as normal (streaming) lines
  a.accessPolicyWindow.hitRatio  = (float)((double)carve / (double)win);
  a.accessPolicyWindow.hitProp   = cudaAccessPropertyPersisting;
  a.accessPolicyWindow.missProp  = cudaAccessPropertyStreaming;
  return cudaStreamSetAttribute((cudaStream_t)stream, cudaStreamAttributeAccessPolicyWindow, &a) ==
                 cudaSuccess
             ? KRON_SUCCESS
             : KRON_ERROR_LAUNCH;
}

extern "C" int kron_l2_persist_reset(kron_stream_t stream)
{
  cudaStreamAttrValue a = {};
  a.accessPolicyWindow.num_bytes = 0;
  a.accessPolicyWindow.hitRatio  = 0.f;
  a.accessPolicyWindow.hitProp   = cudaAccessPropertyNormal;
  a.accessPolicyWindow.missProp  = cudaAccessPropertyNormal;
  if (cudaStreamSetAttribute((cudaStream_t)stream, cudaStreamAttributeAccessPolicyWindow, &a) !=
          cudaSuccess ||
      cudaCtxResetPersistingL2Cache() != cudaSuccess ||
      cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  return KRON_SUCCESS;
}

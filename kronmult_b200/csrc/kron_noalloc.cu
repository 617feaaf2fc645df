// kronmult_batched_noalloc_async: the batched product for callers that
// cannot allocate device memory.
//
// Who needs it: code that must not call cudaMalloc at the point where it
// applies the operator, for example
//   - a solver that enqueues its iteration inside a CUDA stream capture in
//     global capture mode (cudaMalloc is not permitted during such a capture),
//   - an application whose memory pool reserved all of HBM at start-up, so a
//     separate cudaMalloc for W fails or fragments the pool,
//   - a matrix-free operator callback that is handed only A, X and Y and has
//     no place to pass a workspace.
// The reference entry points need a caller-provided W (n^d doubles per
// entry); vectors larger than shared memory need that scratch here too.  This
// entry point instead uses one file-scope device array of
// KRON_NOALLOC_SCRATCH_BYTES (16 MiB), which every GPU that loads the library
// holds until the process exits.  It calls no cudaMalloc/cudaFree and no
// allocating library routine.
//
// Contract:
//   - vectors of more than 16 MiB / 8 = 2,097,152 doubles (n^d) are rejected
//     with KRON_ERROR_WORKSPACE before anything is launched;
//   - larger batches are processed in chunks that fit the array;
//   - nothing in the array needs to start at zero: phase 1 of the two-phase
//     path writes every element that phase 2 later reads;
//   - every call shares the array, so calls whose work overlaps on the GPU
//     (different streams without ordering, or different host threads) race
//     and give wrong results; calls on one stream are ordered and safe;
//   - every call looks up the array's device address (cudaGetSymbolAddress)
//     on the current device, whatever the shape, so the address stays right
//     after a context reset; while `stream` is capturing, the address that
//     the last call outside capture found on this device is used instead.
//     So the first call on a device should come before any stream capture.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "kron_launch.h"

using namespace kron;

namespace {

constexpr size_t KRON_NOALLOC_SCRATCH_BYTES = 16u << 20;

__device__ __align__(256) double g_noalloc_scratch[KRON_NOALLOC_SCRATCH_BYTES / sizeof(double)];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_scratch_addr[MAX_DEVICES] = {};

// Device address of the scratch array for the current device (host code
// must not use the symbol itself as a device pointer).  Looked up afresh
// unless `stream` is capturing (a context reset may move the array); during
// a capture the address cached by the last lookup on this device is used.
int scratch_address(cudaStream_t stream, void **out)
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
    return KRON_ERROR_LAUNCH;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  // an error here (the legacy stream while another stream captures) counts
  // as capturing
  const bool capturing =
      cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!capturing || !g_scratch_addr[dev])
  {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
    {
      cudaGetLastError();
      return KRON_ERROR_LAUNCH;
    }
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return KRON_SUCCESS;
}

} // namespace

extern "C" int kronmult_batched_noalloc_async(int d, int n, double const A[], double const X[],
                                              double Y[], int batchCount, kron_stream_t stream)
{
  if (d < 1 || d > MAXD || n < 0 || batchCount < 0)
    return KRON_ERROR_INVALID_VALUE;
  // the size limit comes first: nothing is touched for oversize requests
  constexpr long long max_elems = (long long)(KRON_NOALLOC_SCRATCH_BYTES / sizeof(double));
  long long L = 1;
  for (int l = 0; l < d; l++)
  {
    L *= n;
    if (L > max_elems)
      return KRON_ERROR_WORKSPACE;
  }
  if (batchCount == 0 || n == 0)
    return KRON_SUCCESS;
  if (!A || !X || !Y)
    return KRON_ERROR_INVALID_VALUE;

  Params p;
  std::memset(&p, 0, sizeof(p));
  p.layout = LAYOUT_BATCHED;
  p.accum  = ACC_DISTINCT;
  p.d      = d;
  p.batch  = batchCount;
  for (int l = 0; l < MAXD; l++)
  {
    p.m[l] = l < d ? n : 1;
    p.n[l] = l < d ? n : 1;
  }
  p.lda     = n;
  p.A       = A;
  p.X       = X;
  p.Y       = Y;
  p.xstride = p.ystride = L;
  cudaStream_t s        = (cudaStream_t)stream;

  // the address lookup comes first, whatever the shape, so that a first
  // call with a small shape caches it for later calls under capture
  void *scratch = nullptr;
  int rc        = scratch_address(s, &scratch);
  if (rc != KRON_SUCCESS)
    return rc;

  if (fits_on_chip(d, p.m, p.n, PREC_F64, false))
  {
    p.ebase = 0;
    p.eend  = batchCount;
    Workspace ws{};
    rc = launch_kron(p, PREC_F64, ws, s);
    if (rc != KRON_SUCCESS)
      return rc;
    return cudaGetLastError() == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
  }
  // the batched two-phase path keeps entry k's intermediate at slot
  // (k - chunk start) * n^d
  const long long per_chunk = (long long)(KRON_NOALLOC_SCRATCH_BYTES / sizeof(double)) / L;
  for (long long k0 = 0; k0 < batchCount; k0 += per_chunk)
  {
    p.ebase = (int)k0;
    p.eend  = (int)std::min<long long>(batchCount, k0 + per_chunk);
    Workspace ws{};
    ws.W       = scratch;
    ws.wstride = L;
    rc         = launch_kron(p, PREC_F64, ws, s);
    if (rc != KRON_SUCCESS)
      return rc;
  }
  return cudaGetLastError() == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

// The C ABI of libkronmult_b200.so (declared in include/kronmult.h).
//
// Every entry point validates its arguments on the host, fills a
// kron::Params describing where entry k's operands live, and hands it to
// kron::launch_kron.  The reference-signature (C++ linkage, void) functions
// forward to their _async twins on stream 0 and record the status.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <new>
#include <numeric>
#include <vector>

#include "kron_launch.h"

using namespace kron;

namespace {

thread_local int g_last_status = KRON_SUCCESS;

int record(int rc)
{
  if (rc != KRON_SUCCESS)
    g_last_status = rc;
  return rc;
}

Params base_params(int layout, int accum, int d, int batch)
{
  Params p;
  std::memset(&p, 0, sizeof(p));
  p.layout = layout;
  p.accum  = accum;
  p.d      = d;
  p.batch  = batch;
  p.ebase  = 0;
  p.eend   = batch;
  for (int l = 0; l < MAXD; l++)
  {
    p.m[l] = 1;
    p.n[l] = 1;
  }
  return p;
}

long long ipow_ll(int b, int e)
{
  long long r = 1;
  for (int i = 0; i < e; i++)
    r *= b;
  return r;
}

bool bad_common(int d, int n, int batch)
{
  return d < 1 || d > MAXD || n < 0 || batch < 0;
}

int finish(int rc)
{
  if (rc != KRON_SUCCESS)
    return rc;
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

void set_square(Params &p, int d, int n)
{
  for (int l = 0; l < d; l++)
  {
    p.m[l] = n;
    p.n[l] = n;
  }
  p.lda = n;
}

int do_batched(int d, int n, int prec, const void *A, const void *X, void *Y, void *W, int batch,
               cudaStream_t s)
{
  if (bad_common(d, n, batch))
    return KRON_ERROR_INVALID_VALUE;
  if (batch == 0 || n == 0)
    return KRON_SUCCESS;
  if (!A || !X || !Y)
    return KRON_ERROR_INVALID_VALUE;
  Params p = base_params(LAYOUT_BATCHED, ACC_DISTINCT, d, batch);
  set_square(p, d, n);
  p.A       = A;
  p.X       = X;
  p.Y       = Y;
  p.xstride = p.ystride = ipow_ll(n, d);
  Workspace ws{};
  ws.W       = W;
  ws.wstride = p.xstride;
  return finish(launch_kron(p, prec, ws, s));
}

int do_pbatched(int d, int n, const double *A, double **pX, double **pY, double **pW, int batch,
                int accum, const int *perm, const int *seg_off, const int *seg_host, int nseg,
                cudaStream_t s)
{
  if (bad_common(d, n, batch))
    return KRON_ERROR_INVALID_VALUE;
  if (batch == 0 || n == 0)
    return KRON_SUCCESS;
  if (!A || !pX || !pY)
    return KRON_ERROR_INVALID_VALUE;
  Params p = base_params(LAYOUT_PBATCHED, accum, d, batch);
  set_square(p, d, n);
  p.A       = A;
  p.pX      = reinterpret_cast<const void *const *>(pX);
  p.pY      = reinterpret_cast<void *const *>(pY);
  p.perm    = perm;
  p.seg_off = seg_off;
  Workspace ws{};
  ws.pW       = reinterpret_cast<void *const *>(pW);
  ws.npW      = pW ? batch : 0;
  ws.pw_elems = ipow_ll(n, d);
  ws.seg_host = seg_host;
  ws.nseg     = nseg;
  return finish(launch_kron(p, PREC_F64, ws, s));
}

int do_xbatched(int d, int n, const double *const *pA, int lda, double **pX, double **pY,
                double **pW, int batch, int subbatch, int accum, const int *perm,
                const int *seg_off, const int *seg_host, int nseg, cudaStream_t s)
{
  if (bad_common(d, n, batch) || lda < std::max(1, n))
    return KRON_ERROR_INVALID_VALUE;
  if (batch == 0 || n == 0)
    return KRON_SUCCESS;
  if (!pA || !pX || !pY)
    return KRON_ERROR_INVALID_VALUE;
  if (subbatch <= 0)
    subbatch = std::max(1, batch / 2); // kronmult_xbatched.hpp:60-63
  Params p = base_params(LAYOUT_XBATCHED, accum, d, batch);
  set_square(p, d, n);
  p.lda     = lda;
  p.apk     = d;
  p.pA      = reinterpret_cast<const void *const *>(pA);
  p.pX      = reinterpret_cast<const void *const *>(pX);
  p.pY      = reinterpret_cast<void *const *>(pY);
  p.perm    = perm;
  p.seg_off = seg_off;
  Workspace ws{};
  ws.pW       = reinterpret_cast<void *const *>(pW);
  // the reference needs 2*subbatchCount W pointers (kronmult_xbatched.hpp:110-113)
  ws.npW      = pW ? (batch > 1 ? 2 * std::min(subbatch, batch) : 1) : 0;
  ws.pw_elems = ipow_ll(n, d);
  ws.seg_host = seg_host;
  ws.nseg     = nseg;
  return finish(launch_kron(p, PREC_F64, ws, s));
}

int do_vbatched(int d, const int *m, const int *n, const double *const *pA, double **pX,
                double **pY, double *W, size_t Wbytes, int batch, cudaStream_t s)
{
  if (d < 1 || d > MAXD || batch < 0)
    return KRON_ERROR_INVALID_VALUE;
  for (int l = 0; l < d; l++)
    if (m[l] < 0 || n[l] < 0)
      return KRON_ERROR_INVALID_VALUE;
  if (batch == 0)
    return KRON_SUCCESS;
  for (int l = 0; l < d; l++)
    if (m[l] == 0 || n[l] == 0)
      return KRON_SUCCESS;
  if (!pA || !pX || !pY)
    return KRON_ERROR_INVALID_VALUE;
  Params p = base_params(LAYOUT_VBATCHED, ACC_ATOMIC, d, batch);
  for (int l = 0; l < d; l++)
  {
    p.m[l] = m[l];
    p.n[l] = n[l];
  }
  p.apk = d;
  p.pA  = reinterpret_cast<const void *const *>(pA);
  p.pX  = reinterpret_cast<const void *const *>(pX);
  p.pY  = reinterpret_cast<void *const *>(pY);
  Workspace ws{};
  ws.W      = W;
  ws.Wbytes = W ? Wbytes : 0;
  return finish(launch_kron(p, PREC_F64, ws, s));
}

int do_kgemm(int op, int mm, int nn, int kk, double alpha, double *const *A, const int *ldA,
             double *const *B, const int *ldB, double beta, double *const *C, const int *ldC,
             int batch, cudaStream_t s)
{
  if (mm < 0 || nn < 0 || kk < 0 || batch < 0)
    return KRON_ERROR_INVALID_VALUE;
  if (batch == 0 || mm == 0 || nn == 0)
    return KRON_SUCCESS;
  if (!A || !ldA || !B || !ldB || !C || !ldC)
    return KRON_ERROR_INVALID_VALUE;
  return finish(launch_kgemm(op, mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, s));
}

} // namespace

// ========================================================================
// extern "C"
// ========================================================================
extern "C" {

const char *kron_status_string(int status)
{
  switch (status)
  {
  case KRON_SUCCESS: return "KRON_SUCCESS";
  case KRON_ERROR_INVALID_VALUE: return "KRON_ERROR_INVALID_VALUE";
  case KRON_ERROR_WORKSPACE: return "KRON_ERROR_WORKSPACE";
  case KRON_ERROR_LAUNCH: return "KRON_ERROR_LAUNCH";
  case KRON_ERROR_NOT_SUPPORTED: return "KRON_ERROR_NOT_SUPPORTED";
  case KRON_ERROR_ALLOC: return "KRON_ERROR_ALLOC";
  case KRON_ERROR_INTERNAL: return "KRON_ERROR_INTERNAL";
  default: return "KRON_ERROR_UNKNOWN";
  }
}

int kron_get_last_status(void) { return g_last_status; }
void kron_clear_last_status(void) { g_last_status = KRON_SUCCESS; }
const char *kron_version(void) { return "0.1.0"; }

#define KRON_DEFINE_D(D)                                                                        \
  int kronmult##D##_batched_async(int n, double const Aarray_[], double Xarray_[],             \
                                  double Yarray_[], double Warray_[], int batchCount,          \
                                  kron_stream_t stream)                                        \
  {                                                                                            \
    return do_batched(D, n, PREC_F64, Aarray_, Xarray_, Yarray_, Warray_, batchCount,          \
                      (cudaStream_t)stream);                                                   \
  }                                                                                            \
  int kronmult##D##_pbatched_async(int n, double const Aarray_[], double *Xarray_[],           \
                                   double *Yarray_[], double *Warray_[], int batchCount,       \
                                   kron_stream_t stream)                                       \
  {                                                                                            \
    return do_pbatched(D, n, Aarray_, Xarray_, Yarray_, Warray_, batchCount, ACC_ATOMIC,       \
                       nullptr, nullptr, nullptr, 0, (cudaStream_t)stream);                    \
  }                                                                                            \
  int kronmult##D##_xbatched_async(int n, double const *const Aarray_[], int lda,              \
                                   double *Xarray_[], double *Yarray_[], double *Warray_[],    \
                                   int batchCount, int subbatchCount, kron_stream_t stream)    \
  {                                                                                            \
    return do_xbatched(D, n, Aarray_, lda, Xarray_, Yarray_, Warray_, batchCount,              \
                       subbatchCount, ACC_ATOMIC, nullptr, nullptr, nullptr, 0,                \
                       (cudaStream_t)stream);                                                  \
  }

KRON_DEFINE_D(1)
KRON_DEFINE_D(2)
KRON_DEFINE_D(3)
KRON_DEFINE_D(4)
KRON_DEFINE_D(5)
KRON_DEFINE_D(6)
#undef KRON_DEFINE_D

int kronmult1_vbatched_async(int m1, int n1, double const *const Aarray_[], double *pX_[],
                             double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream)
{
  int m[] = {m1}, n[] = {n1};
  return do_vbatched(1, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}
int kronmult2_vbatched_async(int m1, int n1, int m2, int n2, double const *const Aarray_[],
                             double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                             int batchCount, kron_stream_t stream)
{
  int m[] = {m1, m2}, n[] = {n1, n2};
  return do_vbatched(2, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}
int kronmult3_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3,
                             double const *const Aarray_[], double *pX_[], double *pY_[],
                             double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream)
{
  int m[] = {m1, m2, m3}, n[] = {n1, n2, n3};
  return do_vbatched(3, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}
int kronmult4_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             double const *const Aarray_[], double *pX_[], double *pY_[],
                             double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream)
{
  int m[] = {m1, m2, m3, m4}, n[] = {n1, n2, n3, n4};
  return do_vbatched(4, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}
int kronmult5_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             int m5, int n5, double const *const Aarray_[], double *pX_[],
                             double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream)
{
  int m[] = {m1, m2, m3, m4, m5}, n[] = {n1, n2, n3, n4, n5};
  return do_vbatched(5, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}
int kronmult6_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             int m5, int n5, int m6, int n6, double const *const Aarray_[],
                             double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                             int batchCount, kron_stream_t stream)
{
  int m[] = {m1, m2, m3, m4, m5, m6}, n[] = {n1, n2, n3, n4, n5, n6};
  return do_vbatched(6, m, n, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                     (cudaStream_t)stream);
}

int kgemm_nn_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream)
{
  return do_kgemm(0, mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta, Carray_,
                  ldCarray_, batchCount, (cudaStream_t)stream);
}
int kgemm_nt_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream)
{
  return do_kgemm(1, mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta, Carray_,
                  ldCarray_, batchCount, (cudaStream_t)stream);
}
int kgemm_tt_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream)
{
  return do_kgemm(2, mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta, Carray_,
                  ldCarray_, batchCount, (cudaStream_t)stream);
}

size_t kron_batched_workspace_bytes(int d, int n, int batchCount)
{
  if (d < 1 || d > MAXD || n < 1 || batchCount < 1)
    return 0;
  int m[MAXD], nv[MAXD];
  for (int l = 0; l < d; l++)
    m[l] = nv[l] = n;
  if (fits_on_chip(d, m, nv, PREC_F64, false))
    return 0;
  return (size_t)ipow_ll(n, d) * batchCount * sizeof(double);
}

size_t kron_vbatched_workspace_bytes(int d, int const m[], int const n[], int batchCount)
{
  if (d < 1 || d > MAXD || batchCount < 1 || !m || !n)
    return 0;
  if (fits_on_chip(d, m, n, PREC_F64, true) || fits_on_chip(d, m, n, PREC_F64, false))
    return 0;
  return large_workspace_elems(d, m, n) * (size_t)batchCount * sizeof(double);
}

int kronmult_batched_f32_async(int d, int n, float const A[], float X[], float Y[], float W[],
                               int batchCount, kron_stream_t stream)
{
  return do_batched(d, n, PREC_F32, A, X, Y, W, batchCount, (cudaStream_t)stream);
}

int kronmult_batched_split_async(int d, int n, double const A[], double X[], double Y[],
                                 double W[], int batchCount, kron_stream_t stream)
{
  return do_batched(d, n, PREC_SPLIT, A, X, Y, W, batchCount, (cudaStream_t)stream);
}

double kron_flops_c(int d, int const m[], int const n[])
{
  // kroncommon.hpp:154-185
  if (d <= 0 || !m || !n)
    return 0.0;
  if (d == 1)
    return 2.0 * m[0] * n[0];
  double rest = 1.0;
  for (int l = 1; l < d; l++)
    rest *= n[l];
  return 2.0 * rest * n[0] * m[0] + (double)m[0] * kron_flops_c(d - 1, m + 1, n + 1);
}

} // extern "C"

// ========================================================================
// Segment plans (deterministic accumulation)
// ========================================================================
struct kron_segments_st
{
  int batch;
  int nseg;
  int *d_perm;    // device: position -> entry
  int *d_seg;     // device: nseg + 1 offsets
  std::vector<int> h_seg;
};

extern "C" int kron_segments_create(kron_segments_t *plan, double *const Yarray_[],
                                    int batchCount, kron_stream_t stream)
{
  if (!plan || batchCount < 0 || (batchCount > 0 && !Yarray_))
    return KRON_ERROR_INVALID_VALUE;
  *plan = nullptr;
  std::vector<uintptr_t> ys(batchCount);
  if (batchCount > 0)
  {
    if (cudaMemcpyAsync(ys.data(), Yarray_, sizeof(uintptr_t) * batchCount,
                        cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess ||
        cudaStreamSynchronize((cudaStream_t)stream) != cudaSuccess)
      return KRON_ERROR_LAUNCH;
  }
  // stable grouping by output pointer: keeps every group's entries in order
  std::vector<int> perm(batchCount);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return ys[a] < ys[b]; });
  std::vector<int> seg;
  for (int e = 0; e < batchCount; e++)
    if (e == 0 || ys[perm[e]] != ys[perm[e - 1]])
      seg.push_back(e);
  seg.push_back(batchCount);

  kron_segments_st *pl = new (std::nothrow) kron_segments_st();
  if (!pl)
    return KRON_ERROR_ALLOC;
  pl->batch = batchCount;
  pl->nseg  = (int)seg.size() - 1;
  pl->h_seg = seg;
  pl->d_perm = nullptr;
  pl->d_seg  = nullptr;
  if (kron::dev_malloc((void **)&pl->d_perm, sizeof(int) * std::max(1, batchCount)) != cudaSuccess ||
      kron::dev_malloc((void **)&pl->d_seg, sizeof(int) * seg.size()) != cudaSuccess)
  {
    kron::dev_free(pl->d_perm);
    kron::dev_free(pl->d_seg);
    delete pl;
    return KRON_ERROR_ALLOC;
  }
  if ((batchCount > 0 &&
       cudaMemcpy(pl->d_perm, perm.data(), sizeof(int) * batchCount, cudaMemcpyHostToDevice) !=
           cudaSuccess) ||
      cudaMemcpy(pl->d_seg, seg.data(), sizeof(int) * seg.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess)
  {
    kron::dev_free(pl->d_perm);
    kron::dev_free(pl->d_seg);
    delete pl;
    return KRON_ERROR_LAUNCH;
  }
  *plan = pl;
  return KRON_SUCCESS;
}

extern "C" int kron_segments_destroy(kron_segments_t plan)
{
  if (!plan)
    return KRON_SUCCESS;
  kron::dev_free(plan->d_perm);
  kron::dev_free(plan->d_seg);
  delete plan;
  return KRON_SUCCESS;
}

extern "C" int kron_segments_count(kron_segments_t plan) { return plan ? plan->nseg : 0; }

extern "C" int kronmult_xbatched_segmented_async(int d, int n, double const *const Aarray_[],
                                                 int lda, double *Xarray_[], double *Yarray_[],
                                                 double *Warray_[], int batchCount,
                                                 kron_segments_t plan, kron_stream_t stream)
{
  if (!plan || plan->batch != batchCount)
    return KRON_ERROR_INVALID_VALUE;
  return do_xbatched(d, n, Aarray_, lda, Xarray_, Yarray_, Warray_, batchCount, 0,
                     ACC_SEGMENTED, plan->d_perm, plan->d_seg, plan->h_seg.data(), plan->nseg,
                     (cudaStream_t)stream);
}

extern "C" int kronmult_pbatched_segmented_async(int d, int n, double const Aarray_[],
                                                 double *Xarray_[], double *Yarray_[],
                                                 double *Warray_[], int batchCount,
                                                 kron_segments_t plan, kron_stream_t stream)
{
  if (!plan || plan->batch != batchCount)
    return KRON_ERROR_INVALID_VALUE;
  return do_pbatched(d, n, Aarray_, Xarray_, Yarray_, Warray_, batchCount, ACC_SEGMENTED,
                     plan->d_perm, plan->d_seg, plan->h_seg.data(), plan->nseg,
                     (cudaStream_t)stream);
}

// ========================================================================
// The reference signatures (C++ linkage)
// ========================================================================
#define KRON_REF_D(D)                                                                           \
  void kronmult##D##_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[], \
                             double Warray_[], int batchCount)                                 \
  {                                                                                            \
    record(kronmult##D##_batched_async(n, Aarray_, Xarray_, Yarray_, Warray_, batchCount,      \
                                       nullptr));                                              \
  }                                                                                            \
  void kronmult##D##_pbatched(int n, double const Aarray_[], double *Xarray_[],                \
                              double *Yarray_[], double *Warray_[], int batchCount)            \
  {                                                                                            \
    record(kronmult##D##_pbatched_async(n, Aarray_, Xarray_, Yarray_, Warray_, batchCount,     \
                                        nullptr));                                             \
  }                                                                                            \
  void kronmult##D##_xbatched(int n, double const *const Aarray_[], int lda,                   \
                              double *Xarray_[], double *Yarray_[], double *Warray_[],         \
                              int batchCount, int subbatchCount)                               \
  {                                                                                            \
    record(kronmult##D##_xbatched_async(n, Aarray_, lda, Xarray_, Yarray_, Warray_,            \
                                        batchCount, subbatchCount, nullptr));                  \
  }

KRON_REF_D(1)
KRON_REF_D(2)
KRON_REF_D(3)
KRON_REF_D(4)
KRON_REF_D(5)
KRON_REF_D(6)
#undef KRON_REF_D

void kronmult1_vbatched(int m1, int n1, double const *const Aarray_[], double *pX_[],
                        double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount)
{
  record(kronmult1_vbatched_async(m1, n1, Aarray_, pX_, pY_, W_, Wcapacity_bytes, batchCount,
                                  nullptr));
}
void kronmult2_vbatched(int m1, int n1, int m2, int n2, double const *const Aarray_[],
                        double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                        int batchCount)
{
  record(kronmult2_vbatched_async(m1, n1, m2, n2, Aarray_, pX_, pY_, W_, Wcapacity_bytes,
                                  batchCount, nullptr));
}
void kronmult3_vbatched(int m1, int n1, int m2, int n2, int m3, int n3,
                        double const *const Aarray_[], double *pX_[], double *pY_[], double *W_,
                        size_t Wcapacity_bytes, int batchCount)
{
  record(kronmult3_vbatched_async(m1, n1, m2, n2, m3, n3, Aarray_, pX_, pY_, W_,
                                  Wcapacity_bytes, batchCount, nullptr));
}
void kronmult4_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                        double const *const Aarray_[], double *pX_[], double *pY_[], double *W_,
                        size_t Wcapacity_bytes, int batchCount)
{
  record(kronmult4_vbatched_async(m1, n1, m2, n2, m3, n3, m4, n4, Aarray_, pX_, pY_, W_,
                                  Wcapacity_bytes, batchCount, nullptr));
}
void kronmult5_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4, int m5,
                        int n5, double const *const Aarray_[], double *pX_[], double *pY_[],
                        double *W_, size_t Wcapacity_bytes, int batchCount)
{
  record(kronmult5_vbatched_async(m1, n1, m2, n2, m3, n3, m4, n4, m5, n5, Aarray_, pX_, pY_,
                                  W_, Wcapacity_bytes, batchCount, nullptr));
}
void kronmult6_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4, int m5,
                        int n5, int m6, int n6, double const *const Aarray_[], double *pX_[],
                        double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount)
{
  record(kronmult6_vbatched_async(m1, n1, m2, n2, m3, n3, m4, n4, m5, n5, m6, n6, Aarray_, pX_,
                                  pY_, W_, Wcapacity_bytes, batchCount, nullptr));
}

void kgemm_nn_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount)
{
  record(kgemm_nn_batched_async(mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta,
                                Carray_, ldCarray_, batchCount, nullptr));
}
void kgemm_nt_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount)
{
  record(kgemm_nt_batched_async(mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta,
                                Carray_, ldCarray_, batchCount, nullptr));
}
void kgemm_tt_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount)
{
  record(kgemm_tt_batched_async(mm, nn, kk, alpha, Aarray_, ldAarray_, Barray_, ldBarray_, beta,
                                Carray_, ldCarray_, batchCount, nullptr));
}

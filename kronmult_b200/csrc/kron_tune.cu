// Autotuner: which kernel variant (and its tile / cluster / entries-per-block
// parameter) runs square shapes of a given (d, n, precision).
//
// kron_autotune times every variant that can run the shape on a synthetic
// batched problem (one warm-up launch, then the fastest of three CUDA-event
// timings on the caller's stream) and records the winner; launch_kron tries
// the recorded variant before its built-in order.  Choices can also be set,
// read, cleared, saved to and loaded from a text file (one
// "d n precision variant param" line per shape).  The table is process-wide
// and guarded by a mutex; it is empty until a caller fills it, so nothing
// changes for callers that never tune.
#include <cstdio>
#include <map>
#include <mutex>
#include <vector>

#include "kron_launch.h"
#include "kronmult.h"

namespace kron {

namespace {

struct TuneKey
{
  int d, n, prec;
  bool operator<(const TuneKey &o) const
  {
    if (d != o.d)
      return d < o.d;
    if (n != o.n)
      return n < o.n;
    return prec < o.prec;
  }
};

struct TuneChoice
{
  int variant, param;
};

std::mutex g_tune_mu;
std::map<TuneKey, TuneChoice> g_tune;

bool valid_variant(int v) { return v >= VAR_MMA8 && v <= VAR_SPLIT_TC; }

} // namespace

bool tune_lookup(int d, int n, int prec, int &variant, int &param)
{
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (g_tune.empty())
    return false;
  auto it = g_tune.find(TuneKey{d, n, prec});
  if (it == g_tune.end())
    return false;
  variant = it->second.variant;
  param   = it->second.param;
  return true;
}

} // namespace kron

using namespace kron;

static_assert(KRON_PREC_F64 == PREC_F64 && KRON_PREC_F32 == PREC_F32 &&
                  KRON_PREC_SPLIT == PREC_SPLIT,
              "precision codes");
static_assert(KRON_VARIANT_MMA8 == VAR_MMA8 && KRON_VARIANT_PIPE == VAR_PIPE &&
                  KRON_VARIANT_SQ == VAR_SQ && KRON_VARIANT_GEN == VAR_GEN &&
                  KRON_VARIANT_BIG == VAR_BIG && KRON_VARIANT_LARGE == VAR_LARGE &&
                  KRON_VARIANT_SLAB == VAR_SLAB && KRON_VARIANT_SPLIT_TC == VAR_SPLIT_TC,
              "variant codes");

extern "C" int kron_tune_set(int d, int n, int precision, int variant, int param)
{
  if (d < 1 || d > MAXD || n < 1 || precision < PREC_F64 || precision > PREC_SPLIT ||
      (variant != 0 && !valid_variant(variant)) || param < 0)
    return KRON_ERROR_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  if (variant == 0)
    g_tune.erase(TuneKey{d, n, precision});
  else
    g_tune[TuneKey{d, n, precision}] = TuneChoice{variant, param};
  return KRON_SUCCESS;
}

extern "C" int kron_tune_get(int d, int n, int precision, int *variant, int *param)
{
  if (!variant || !param)
    return KRON_ERROR_INVALID_VALUE;
  int v = 0, q = 0;
  if (!tune_lookup(d, n, precision, v, q))
    v = q = 0;
  *variant = v;
  *param   = q;
  return KRON_SUCCESS;
}

extern "C" void kron_tune_clear(void)
{
  std::lock_guard<std::mutex> lock(g_tune_mu);
  g_tune.clear();
}

extern "C" int kron_tune_save(const char *path)
{
  if (!path)
    return KRON_ERROR_INVALID_VALUE;
  std::lock_guard<std::mutex> lock(g_tune_mu);
  FILE *f = std::fopen(path, "w");
  if (!f)
    return KRON_ERROR_INVALID_VALUE;
  for (const auto &kv : g_tune)
    std::fprintf(f, "%d %d %d %d %d\n", kv.first.d, kv.first.n, kv.first.prec,
                 kv.second.variant, kv.second.param);
  return std::fclose(f) == 0 ? KRON_SUCCESS : KRON_ERROR_INVALID_VALUE;
}

extern "C" int kron_tune_load(const char *path)
{
  if (!path)
    return KRON_ERROR_INVALID_VALUE;
  FILE *f = std::fopen(path, "r");
  if (!f)
    return KRON_ERROR_INVALID_VALUE;
  int d, n, pr, v, q, rc = KRON_SUCCESS;
  while (std::fscanf(f, "%d %d %d %d %d", &d, &n, &pr, &v, &q) == 5)
    if (kron_tune_set(d, n, pr, v, q) != KRON_SUCCESS)
      rc = KRON_ERROR_INVALID_VALUE;
  std::fclose(f);
  return rc;
}

namespace {

struct DevBuf
{
  void *p = nullptr;
  ~DevBuf()
  {
    if (p)
      kron::dev_free(p);
  }
  bool alloc(size_t bytes) { return bytes == 0 || dev_malloc(&p, bytes) == cudaSuccess; }
};

} // namespace

extern "C" int kron_autotune(int d, int n, int precision, int batch, int *variant, int *param,
                             double *best_us, kron_stream_t stream_)
{
  if (d < 1 || d > MAXD || n < 1 || batch < 1 || precision < PREC_F64 ||
      precision > PREC_SPLIT)
    return KRON_ERROR_INVALID_VALUE;
  cudaStream_t stream = (cudaStream_t)stream_;
  const size_t esize  = precision == PREC_F32 ? 4 : 8;
  long long L = 1;
  for (int l = 0; l < d; l++)
    L *= n;
  // keep the synthetic problem under 1 GiB (x, y, A and a workspace slot
  // per entry)
  const long long per_entry = (3 * L + (long long)d * n * n) * (long long)esize;
  const long long cap       = std::max<long long>(1, (1LL << 30) / per_entry);
  const int B               = (int)std::min<long long>(batch, cap);

  DevBuf A, X, Y, W;
  if (!A.alloc((size_t)d * n * n * B * esize) || !X.alloc((size_t)L * B * esize) ||
      !Y.alloc((size_t)L * B * esize) || !W.alloc((size_t)L * B * esize))
    return KRON_ERROR_ALLOC;
  cudaMemsetAsync(A.p, 0, (size_t)d * n * n * B * esize, stream);
  cudaMemsetAsync(X.p, 0, (size_t)L * B * esize, stream);
  cudaMemsetAsync(Y.p, 0, (size_t)L * B * esize, stream);

  Params p{};
  p.layout = LAYOUT_BATCHED;
  p.accum  = ACC_DISTINCT;
  p.d      = d;
  for (int l = 0; l < MAXD; l++)
    p.m[l] = p.n[l] = (l < d) ? n : 1;
  p.batch   = B;
  p.A       = A.p;
  p.X       = X.p;
  p.Y       = Y.p;
  p.apk     = d;
  p.lda     = n;
  p.xstride = p.ystride = L;
  p.ebase   = 0;
  p.eend    = B;
  Workspace ws{};
  ws.W       = W.p;
  ws.wstride = L;

  // candidates: every variant, the square kernel at 1, 2, 4, ... entries
  // per block, the cluster kernel at cluster sizes 1, 2, 4 (FP64 n = 8: on
  // the tensor cores and on CUDA cores; FP64 n = 6: W in the workspace or
  // on chip)
  std::vector<std::pair<int, int>> cand = {{VAR_MMA8, 0}, {VAR_PIPE, 0}, {VAR_SLAB, 0}};
  const int ngmax = sq_entries_max(precision, d, n, false);
  for (int ng = 1; ng <= ngmax; ng *= 2)
    cand.push_back({VAR_SQ, ng});
  if (ngmax > 0 && (ngmax & (ngmax - 1)))
    cand.push_back({VAR_SQ, ngmax});
  cand.push_back({VAR_GEN, 0});
  // FP64 d = 6, n = 6 can also keep W in the cluster's shared memory
  // (fixed cluster of 2)
  if (precision == PREC_F64 && d == 6 && n == 6)
    cand.push_back({VAR_BIG, KRON_BIG_SMEM_W});
  for (int cs : {1, 2, 4})
  {
    cand.push_back({VAR_BIG, cs});
    if (precision == PREC_F64 && d == 6 && n == 8)
      cand.push_back({VAR_BIG, cs | KRON_BIG_CUDA_CORES});
  }
  cand.push_back({VAR_LARGE, 0});

  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess)
  {
    if (e0)
      cudaEventDestroy(e0);
    return KRON_ERROR_ALLOC;
  }
  int best_v = 0, best_p = 0;
  float best = 0.f;
  for (const auto &c : cand)
  {
    Params q = p;
    launch_setup(q, ws);
    int rc = launch_variant(q, precision, ws, c.first, c.second, stream); // warm-up
    if (rc != KRON_SUCCESS)
      continue;
    float t = -1.f;
    for (int rep = 0; rep < 3 && rc == KRON_SUCCESS; rep++)
    {
      cudaEventRecord(e0, stream);
      rc = launch_variant(q, precision, ws, c.first, c.second, stream);
      cudaEventRecord(e1, stream);
      if (cudaEventSynchronize(e1) != cudaSuccess)
        rc = KRON_ERROR_LAUNCH;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (rc == KRON_SUCCESS && (t < 0.f || ms < t))
        t = ms;
    }
    if (rc == KRON_SUCCESS && t >= 0.f && (best_v == 0 || t < best))
    {
      best_v = c.first;
      best_p = c.second;
      best   = t;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (cudaStreamSynchronize(stream) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  if (best_v == 0)
    return KRON_ERROR_NOT_SUPPORTED;
  kron_tune_set(d, n, precision, best_v, best_p);
  if (variant)
    *variant = best_v;
  if (param)
    *param = best_p;
  if (best_us)
    *best_us = 1e3 * best;
  return KRON_SUCCESS;
}

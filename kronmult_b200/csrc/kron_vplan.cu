// Uneven-batch plans: every entry has its own d and rectangular shapes
// (no reference counterpart; the reference's vbatched needs one launch per
// (d, shape) group, kronmult_vbatched.hpp:17-228).
//
// The plan (built once on the host from the shape table) orders entries by
// cost, largest first, and groups entries of identical shape so each group
// runs the compile-time or runtime on-chip kernel; entries too large for
// shared memory take the two-phase workspace path.  Alg. 993 forward or
// backward order is chosen per shape by flop count (kronm.hpp:39-89).
// Executions on a non-default stream are captured once into a CUDA graph
// and replayed while the operand arrays stay the same.
#include <algorithm>
#include <cstring>
#include <map>
#include <new>
#include <vector>

#include "kron_launch.h"

using namespace kron;

namespace {

struct ShapeKey
{
  int d;
  int m[MAXD], n[MAXD];
  bool operator<(const ShapeKey &o) const
  {
    if (d != o.d)
      return d < o.d;
    for (int l = 0; l < d; l++)
    {
      if (m[l] != o.m[l])
        return m[l] < o.m[l];
      if (n[l] != o.n[l])
        return n[l] < o.n[l];
    }
    return false;
  }
};

struct Group
{
  ShapeKey key;
  int begin, end;   // positions in perm
  double cost;      // flops per entry of the chosen variant
  bool on_chip;
  long long slot_elems;
};

} // namespace

struct kron_vplan_st
{
  int batch;
  std::vector<Group> groups;
  int *d_perm;
  double flops;
  size_t ws_bytes;
  // graph cache
  cudaGraphExec_t exec;
  const void *gA, *gX, *gY, *gW;
  size_t gWcap;
  cudaStream_t gstream;
};

extern "C" int kron_vplan_create(kron_vplan_t *plan, int batchCount, int const shapes[])
{
  if (!plan || batchCount < 0 || (batchCount > 0 && !shapes))
    return KRON_ERROR_INVALID_VALUE;
  *plan = nullptr;
  std::map<ShapeKey, std::vector<int>> by_shape;
  for (int k = 0; k < batchCount; k++)
  {
    const int *s = shapes + 13LL * k;
    ShapeKey key;
    std::memset(&key, 0, sizeof(key));
    key.d = s[0];
    if (key.d < 1 || key.d > MAXD)
      return KRON_ERROR_INVALID_VALUE;
    for (int l = 0; l < key.d; l++)
    {
      key.m[l] = s[1 + 2 * l];
      key.n[l] = s[2 + 2 * l];
      if (key.m[l] < 1 || key.n[l] < 1)
        return KRON_ERROR_INVALID_VALUE;
    }
    by_shape[key].push_back(k);
  }
  kron_vplan_st *pl = new (std::nothrow) kron_vplan_st();
  if (!pl)
    return KRON_ERROR_ALLOC;
  pl->batch  = batchCount;
  pl->d_perm = nullptr;
  pl->flops  = 0.0;
  pl->ws_bytes = 0;
  pl->exec   = nullptr;
  std::vector<Group> groups;
  for (auto &kv : by_shape)
  {
    Group g;
    g.key = kv.first;
    const ShapeKey &k = kv.first;
    g.cost = std::min(flops_forward(k.d, k.m, k.n), flops_backward(k.d, k.m, k.n));
    g.on_chip = fits_on_chip(k.d, k.m, k.n, PREC_F64, true) ||
                fits_on_chip(k.d, k.m, k.n, PREC_F64, false);
    g.slot_elems = g.on_chip ? 0 : (long long)large_workspace_elems(k.d, k.m, k.n);
    if (!g.on_chip && g.slot_elems <= 0)
    {
      delete pl;
      return KRON_ERROR_NOT_SUPPORTED;
    }
    g.begin = 0;
    g.end   = (int)kv.second.size();
    groups.push_back(g);
    pl->flops += g.cost * kv.second.size();
  }
  // largest per-entry cost first
  std::vector<int> order(groups.size());
  for (size_t i = 0; i < order.size(); i++)
    order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return groups[a].cost > groups[b].cost; });
  std::vector<int> perm;
  perm.reserve(batchCount);
  for (int gi : order)
  {
    Group g   = groups[gi];
    auto &ids = by_shape[g.key];
    g.begin   = (int)perm.size();
    perm.insert(perm.end(), ids.begin(), ids.end());
    g.end = (int)perm.size();
    if (!g.on_chip)
      pl->ws_bytes = std::max(pl->ws_bytes, (size_t)g.slot_elems * (g.end - g.begin) * 8);
    pl->groups.push_back(g);
  }
  if (batchCount > 0)
  {
    if (cudaMalloc(&pl->d_perm, sizeof(int) * batchCount) != cudaSuccess)
    {
      delete pl;
      return KRON_ERROR_ALLOC;
    }
    if (cudaMemcpy(pl->d_perm, perm.data(), sizeof(int) * batchCount, cudaMemcpyHostToDevice) !=
        cudaSuccess)
    {
      cudaFree(pl->d_perm);
      delete pl;
      return KRON_ERROR_LAUNCH;
    }
  }
  *plan = pl;
  return KRON_SUCCESS;
}

extern "C" int kron_vplan_destroy(kron_vplan_t plan)
{
  if (!plan)
    return KRON_SUCCESS;
  if (plan->exec)
    cudaGraphExecDestroy(plan->exec);
  cudaFree(plan->d_perm);
  delete plan;
  return KRON_SUCCESS;
}

extern "C" size_t kron_vplan_workspace_bytes(kron_vplan_t plan) { return plan ? plan->ws_bytes : 0; }
extern "C" double kron_vplan_flops(kron_vplan_t plan) { return plan ? plan->flops : 0.0; }

static int vplan_launch_all(kron_vplan_t pl, double const *const *A, double **X, double **Y,
                            void *W, size_t Wcap, cudaStream_t s)
{
  for (const Group &g : pl->groups)
  {
    Params p;
    std::memset(&p, 0, sizeof(p));
    p.layout = LAYOUT_VBATCHED;
    p.accum  = ACC_ATOMIC;
    p.d      = g.key.d;
    for (int l = 0; l < MAXD; l++)
    {
      p.m[l] = l < p.d ? g.key.m[l] : 1;
      p.n[l] = l < p.d ? g.key.n[l] : 1;
    }
    p.apk   = MAXD;
    p.batch = pl->batch;
    p.pA    = reinterpret_cast<const void *const *>(A);
    p.pX    = reinterpret_cast<const void *const *>(X);
    p.pY    = reinterpret_cast<void *const *>(Y);
    p.perm  = pl->d_perm;
    p.ebase = g.begin;
    p.eend  = g.end;
    Workspace ws{};
    ws.W      = W;
    ws.Wbytes = W ? Wcap : 0;
    int rc    = launch_kron(p, PREC_F64, ws, s);
    if (rc != KRON_SUCCESS)
      return rc;
  }
  return KRON_SUCCESS;
}

extern "C" int kron_vplan_execute_async(kron_vplan_t plan, double const *const Aarray_[],
                                        double *pX_[], double *pY_[], void *W,
                                        size_t Wcapacity_bytes, kron_stream_t stream)
{
  if (!plan)
    return KRON_ERROR_INVALID_VALUE;
  if (plan->batch == 0)
    return KRON_SUCCESS;
  if (!Aarray_ || !pX_ || !pY_)
    return KRON_ERROR_INVALID_VALUE;
  cudaStream_t s = (cudaStream_t)stream;
  if (plan->ws_bytes > 0 && (!W || Wcapacity_bytes == 0))
    return KRON_ERROR_WORKSPACE;

  // Graphs only on explicit streams that are not already capturing.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  bool use_graph             = (s != nullptr) && cudaStreamIsCapturing(s, &cs) == cudaSuccess &&
                   cs == cudaStreamCaptureStatusNone;
  if (!use_graph)
  {
    int rc = vplan_launch_all(plan, Aarray_, pX_, pY_, W, Wcapacity_bytes, s);
    if (rc != KRON_SUCCESS)
      return rc;
    return cudaGetLastError() == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
  }
  const bool same = plan->exec && plan->gA == Aarray_ && plan->gX == pX_ && plan->gY == pY_ &&
                    plan->gW == W && plan->gWcap == Wcapacity_bytes;
  if (!same)
  {
    if (plan->exec)
    {
      cudaGraphExecDestroy(plan->exec);
      plan->exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return KRON_ERROR_LAUNCH;
    int rc = vplan_launch_all(plan, Aarray_, pX_, pY_, W, Wcapacity_bytes, s);
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (rc != KRON_SUCCESS)
    {
      if (graph)
        cudaGraphDestroy(graph);
      return rc;
    }
    if (ce != cudaSuccess || !graph)
      return KRON_ERROR_LAUNCH;
    cudaGraphExec_t exec = nullptr;
    ce                   = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess)
      return KRON_ERROR_LAUNCH;
    plan->exec  = exec;
    plan->gA    = Aarray_;
    plan->gX    = pX_;
    plan->gY    = pY_;
    plan->gW    = W;
    plan->gWcap = Wcapacity_bytes;
  }
  return cudaGraphLaunch(plan->exec, s) == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

// Host-side dispatch: picks the kernel family for a problem and launches it.
//
//  * square n in 2..8 whose n^d vector (and merge buffer) fits a block's
//    shared memory            -> kron_sq_kernel<T, d, n>   (compile-time shape)
//  * any other shape that fits -> kron_gen_kernel<T>        (runtime shape)
//  * vectors too large for shared memory -> two launches of kron_gen_kernel
//    through the caller's workspace W: phase 1 applies the trailing modes to
//    every contiguous block of x (writing W), phase 2 applies the leading
//    modes to column tiles of W and accumulates into y.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <map>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

#include "kron_launch.h"
#include "kron_sq_table.cuh"

namespace kron {

const DeviceInfo &device_info()
{
  static std::mutex mu;
  static std::vector<DeviceInfo> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  for (auto &d : cache)
    if (d.device == dev)
      return d;
  DeviceInfo info{};
  info.device = dev;
  cudaDeviceGetAttribute(&info.sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&info.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&info.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
  if (info.sms <= 0)
    info.sms = 148;
  if (info.max_smem_optin <= 0)
    info.max_smem_optin = (int)SMEM_OPTIN_MAX;
  cache.push_back(info);
  return cache.back();
}

// Per (kernel, device) launch facts, computed once: the dynamic shared
// memory attribute is raised to the device maximum and the occupancy for a
// (block, smem) pair is cached (host-side launch cost matters for the
// microsecond-scale kernels of small batches).
struct FnKey
{
  const void *fn;
  int dev, block;
  size_t smem;
  bool operator<(const FnKey &o) const
  {
    if (fn != o.fn)
      return fn < o.fn;
    if (dev != o.dev)
      return dev < o.dev;
    if (block != o.block)
      return block < o.block;
    return smem < o.smem;
  }
};

int cached_occupancy(const void *fn, int block, size_t smem, int *per_sm)
{
  static std::mutex mu;
  static std::map<FnKey, int> occ;
  static std::set<std::pair<const void *, int>> attr;
  int dev = 0;
  cudaGetDevice(&dev);
  FnKey key{fn, dev, block, smem};
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = occ.find(key);
    if (it != occ.end())
    {
      *per_sm = it->second;
      return KRON_SUCCESS;
    }
  }
  if (!attr.count({fn, dev}))
  {
    // dynamic + static shared memory may not exceed the opt-in maximum
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, fn) != cudaSuccess)
      return KRON_ERROR_LAUNCH;
    const int dyn_max = device_info().max_smem_optin - (int)fa.sharedSizeBytes;
    if ((long long)smem > dyn_max ||
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn_max) !=
            cudaSuccess)
      return KRON_ERROR_LAUNCH;
  }
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, block, smem) != cudaSuccess || n < 1)
    n = 1;
  std::lock_guard<std::mutex> lock(mu);
  attr.insert({fn, dev});
  occ[key] = n;
  *per_sm  = n;
  return KRON_SUCCESS;
}

static int launch_blocks(const void *fn, int nitems_groups, int ng, int block, size_t smem,
                         void **args, cudaStream_t stream)
{
  int per_sm = 1;
  int rc     = cached_occupancy(fn, block, smem, &per_sm);
  if (rc != KRON_SUCCESS)
    return rc;
  const DeviceInfo &di = device_info();
  long long want = ((long long)nitems_groups + ng - 1) / ng;
  long long grid = std::min<long long>(want, (long long)di.sms * per_sm);
  if (grid < 1)
    grid = 1;
  cudaError_t e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(block), args, smem, stream);
  return e == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

static long long prodl(int d, const int *v)
{
  long long p = 1;
  for (int i = 0; i < d; i++)
    p *= v[i];
  return p;
}

double flops_forward(int d, const int *m, const int *n)
{
  double size = (double)prodl(d, n), total = 0.0;
  for (int l = 0; l < d; l++)
  {
    double cols = size / n[l];
    total += 2.0 * m[l] * cols * n[l];
    size = m[l] * cols;
  }
  return total;
}

double flops_backward(int d, const int *m, const int *n)
{
  double size = (double)prodl(d, n), total = 0.0;
  for (int l = d - 1; l >= 0; l--)
  {
    double rows = size / n[l];
    total += 2.0 * rows * m[l] * n[l];
    size = rows * m[l];
  }
  return total;
}

// kronm.hpp:83-89: forward only when strictly cheaper.
bool choose_forward(int d, const int *m, const int *n)
{
  return flops_forward(d, m, n) < flops_backward(d, m, n);
}

// Largest intermediate (elements) along the chosen order, input included.
long long max_intermediate(int d, const int *m, const int *n, bool forward)
{
  int dims[MAXD];
  for (int l = 0; l < d; l++)
    dims[l] = n[l];
  long long best = prodl(d, dims);
  for (int s = 0; s < d; s++)
  {
    int l   = forward ? s : d - 1 - s;
    dims[l] = m[l];
    best    = std::max(best, prodl(d, dims));
  }
  return best;
}

static int round_up(long long v, int q) { return (int)((v + q - 1) / q * q); }

static int pick_gs(long long work)
{
  if (work >= 2048)
    return 256;
  if (work >= 512)
    return 128;
  if (work >= 128)
    return 64;
  return 32;
}

// Per-group shared-memory elements of a whole-vector runtime launch.
static bool gen_whole_view(int d, const int *m, const int *n, bool merge, int esize, GenView &v)
{
  v       = GenView{};
  v.dd    = d;
  v.mode0 = 0;
  for (int l = 0; l < d; l++)
  {
    v.mm[l] = m[l];
    v.nn[l] = n[l];
  }
  v.forward      = choose_forward(d, m, n) ? 1 : 0;
  v.subs         = 1;
  v.C            = 1;
  v.total_cols   = 0;
  v.in_row       = 1;
  v.out_row      = 1;
  const int q    = 16 / esize;
  long long mi   = max_intermediate(d, m, n, v.forward != 0);
  v.max_inter    = round_up(mi, q);
  v.out_elems    = round_up(prodl(d, m), q);
  long long asz  = 0;
  for (int l = 0; l < d; l++)
    asz += (long long)m[l] * n[l];
  v.asz          = (int)asz;
  v.merge        = merge ? 1 : 0;
  long long ge   = 2LL * v.max_inter + (merge ? v.out_elems : 0) + round_up(asz, q);
  v.group_elems  = (int)std::min<long long>(ge, 1LL << 30);
  v.GS           = pick_gs(mi);
  return ge * esize <= (long long)device_info().max_smem_optin;
}

template <typename T, int PREC>
static int launch_gen(Params p, const GenView &v, cudaStream_t stream)
{
  const void *fn   = reinterpret_cast<const void *>(&kron_gen_kernel<T, PREC>);
  size_t gbytes    = (size_t)v.group_elems * sizeof(T);
  const int maxsm  = device_info().max_smem_optin;
  int ng           = std::max(1, std::min(256 / v.GS, (int)(maxsm / std::max<size_t>(gbytes, 1))));
  int block        = ng * v.GS;
  size_t smem      = (size_t)ng * gbytes;
  void *args[]     = {&p, const_cast<GenView *>(&v)};
  long long groups = (long long)p.nitems * v.subs;
  if (groups <= 0)
    return KRON_SUCCESS;
  return launch_blocks(fn, (int)std::min<long long>(groups, 1LL << 30), ng, block, smem, args,
                       stream);
}

static int launch_gen_prec(int prec, Params p, const GenView &v, cudaStream_t stream)
{
  switch (prec)
  {
  case PREC_F64: return launch_gen<double, PREC_F64>(p, v, stream);
  case PREC_F32: return launch_gen<float, PREC_F32>(p, v, stream);
  case PREC_SPLIT: return launch_gen<double, PREC_SPLIT>(p, v, stream);
  default: return KRON_ERROR_NOT_SUPPORTED;
  }
}

static SqKernelInfo pick_sq(int prec, int d, int n, bool merge)
{
  switch (prec)
  {
  case PREC_F64: return sq_kernel_f64(d, n, merge);
  case PREC_F32: return merge ? SqKernelInfo{nullptr, 0, 0} : sq_kernel_f32(d, n);
  case PREC_SPLIT: return merge ? SqKernelInfo{nullptr, 0, 0} : sq_kernel_split(d, n);
  default: return {nullptr, 0, 0};
  }
}

static bool is_square(const Params &p)
{
  for (int l = 0; l < p.d; l++)
    if (p.m[l] != p.n[0] || p.n[l] != p.n[0])
      return false;
  return true;
}

// Work-item setup for whole-entry launches.
static void setup_items(Params &p, const Workspace &ws)
{
  // positions [ebase, eend) are set by the caller (0..batch for whole calls)
  p.ibase = 0;
  if (p.seg_off)
  {
    p.nitems = ws.nseg;
    p.chunk  = 0;
    return;
  }
  if (p.accum == ACC_ATOMIC)
  {
    // short runs of consecutive entries per item so equal outputs merge
    p.chunk = 8;
  }
  else
    p.chunk = 1;
  p.nitems = (p.eend - p.ebase + p.chunk - 1) / p.chunk;
}

void launch_setup(Params &p, const Workspace &ws) { setup_items(p, ws); }

size_t large_workspace_elems(int d, const int *m, const int *n)
{
  LargePlan lp;
  if (!plan_large(d, m, n, 8, true, lp))
    return 0;
  return (size_t)lp.slot_elems;
}

bool plan_large(int d, const int *m, const int *n, int esize, bool merge, LargePlan &best)
{
  const int maxsm = device_info().max_smem_optin;
  bool found      = false;
  for (int q = 1; q < d; q++)
  {
    // phase 1: modes [q, d) on contiguous blocks; phase 2: modes [0, q) on column tiles
    GenView v1;
    if (!gen_whole_view(d - q, m + q, n + q, false, esize, v1))
      continue;
    const long long Nhead = prodl(q, n), Mtail = prodl(d - q, m + q);
    for (int C : {32, 16, 8, 4, 2, 1})
    {
      GenView v2;
      gen_whole_view(q, m, n, merge, esize, v2);
      const int qv   = 16 / esize;
      long long mi   = max_intermediate(q, m, n, v2.forward != 0) * C;
      v2.max_inter   = round_up(mi, qv);
      v2.out_elems   = round_up(prodl(q, m) * C, qv);
      long long ge   = 2LL * v2.max_inter + (merge ? v2.out_elems : 0) + round_up(v2.asz, qv);
      if (ge * esize > maxsm)
        continue;
      v2.group_elems = (int)ge;
      v2.GS          = pick_gs(mi);
      // prefer the most balanced split, then the widest tile
      long long score = std::abs((long long)(v1.max_inter) - (long long)(v2.max_inter / C)) -
                        (long long)C * 1000;
      if (!found || score < best.score)
      {
        best.q          = q;
        best.v1         = v1;
        best.v2         = v2;
        best.C          = C;
        best.slot_elems = Nhead * Mtail;
        best.score      = score;
        found           = true;
      }
      break;
    }
  }
  return found;
}

template <typename T>
static int launch_large_t(int prec, Params p, const Workspace &ws, cudaStream_t stream)
{
  const bool merge = (p.accum == ACC_ATOMIC || p.accum == ACC_SEGMENTED);
  LargePlan lp;
  if (!plan_large(p.d, p.m, p.n, sizeof(T), merge, lp))
    return KRON_ERROR_NOT_SUPPORTED;
  const int d = p.d, q = lp.q;
  const long long Ntail = prodl(d - q, p.n + q), Mtail = prodl(d - q, p.m + q);
  const long long Nhead = prodl(q, p.n);

  // workspace slots
  long long nslots = 0;
  GenView v1 = lp.v1, v2 = lp.v2;
  v1.ws_ptrs = v2.ws_ptrs = nullptr;
  v1.ws_ptr_step = v2.ws_ptr_step = 1;
  if (p.layout == LAYOUT_BATCHED)
  {
    if (!ws.W || ws.wstride < lp.slot_elems)
      return KRON_ERROR_WORKSPACE;
    nslots     = p.eend - p.ebase;
    v1.ws_base = v2.ws_base = ws.W;
    v1.ws_stride = v2.ws_stride = ws.wstride;
  }
  else if (ws.pW)
  {
    if (ws.pw_elems < lp.slot_elems || ws.npW < 1)
      return KRON_ERROR_WORKSPACE;
    nslots     = ws.npW;
    v1.ws_ptrs = v2.ws_ptrs = ws.pW;
  }
  else
  {
    nslots = (ws.W ? (long long)(ws.Wbytes / (sizeof(T) * (size_t)lp.slot_elems)) : 0);
    if (nslots < 1)
      return KRON_ERROR_WORKSPACE;
    v1.ws_base = v2.ws_base = ws.W;
    v1.ws_stride = v2.ws_stride = lp.slot_elems;
  }

  // phase views
  v1.mode0       = q;
  v1.subs        = (int)Nhead;
  v1.C           = 1;
  v1.in_sub_off  = Ntail;
  v1.out_sub_off = Mtail;
  v1.in_ws       = 0;
  v1.out_ws      = 1;
  v1.merge       = 0;
  v2.mode0       = 0;
  v2.C           = lp.C;
  v2.subs        = (int)((Mtail + lp.C - 1) / lp.C);
  v2.total_cols  = Mtail;
  v2.in_sub_off  = lp.C;
  v2.out_sub_off = lp.C;
  v2.in_row      = Mtail;
  v2.out_row     = Mtail;
  v2.in_ws       = 1;
  v2.out_ws      = 0;

  // chunks of positions that fit the slots (segment-aligned when segmented)
  int pos = p.ebase, seg = 0;
  const int pend = p.eend;
  while (pos < pend)
  {
    int end  = (int)std::min<long long>(pend, pos + nslots);
    int seg1 = seg;
    if (p.seg_off)
    {
      // advance whole segments
      while (seg1 < ws.nseg && ws.seg_host[seg1 + 1] <= pos + nslots)
        seg1++;
      if (seg1 == seg)
        return KRON_ERROR_WORKSPACE; // one output group needs more slots than provided
      end = ws.seg_host[seg1];
    }
    Params p1  = p;
    p1.seg_off = nullptr;
    p1.ebase   = pos;
    p1.eend    = end;
    p1.chunk   = 1;
    p1.nitems  = end - pos;
    v1.slot0   = pos;
    int rc     = launch_gen_prec(prec, p1, v1, stream);
    if (rc != KRON_SUCCESS)
      return rc;
    Params p2 = p;
    v2.slot0  = pos;
    if (p.seg_off)
    {
      p2.ibase  = seg;
      p2.nitems = seg1 - seg;
    }
    else
    {
      p2.ebase  = pos;
      p2.eend   = end;
      p2.chunk  = (p.accum == ACC_ATOMIC) ? 8 : 1;
      p2.nitems = (end - pos + p2.chunk - 1) / p2.chunk;
    }
    rc = launch_gen_prec(prec, p2, v2, stream);
    if (rc != KRON_SUCCESS)
      return rc;
    pos = end;
    seg = seg1;
  }
  return KRON_SUCCESS;
}

bool fits_on_chip(int d, const int *m, const int *n, int precision, bool merge)
{
  GenView v;
  return gen_whole_view(d, m, n, merge, precision == PREC_F32 ? 4 : 8, v);
}

int sq_entries_max(int prec, int d, int n, bool merge)
{
  if (n < 2 || n > 8)
    return 0;
  SqKernelInfo ki = pick_sq(prec, d, n, merge);
  if (!ki.fn && merge)
    ki = pick_sq(prec, d, n, false); // atomic without run merging
  if (!ki.fn || ki.group_bytes > (size_t)device_info().max_smem_optin)
    return 0;
  return std::max(1, std::min(256 / ki.GS, (int)(device_info().max_smem_optin / ki.group_bytes)));
}

// ---- slab-cluster kernel with a side kernel on the SMs it leaves idle ----
//
// The slab kernel's clusters of 12 blocks fill whole GPCs only so far: on
// B200 its 21 resident clusters hold 126 of the 148 SMs.  When the caller
// passes a workspace, a share of the entries goes to the cluster two-phase
// kernel (clusters of 2) on a second stream, whose blocks take the idle SMs
// while the slab kernel runs.  The share gives each idle SM SIDE_RATE of a
// slab SM's entries (measured for 4096 entries of d = 6, n = 6: 1.59 ms
// alone; 1.40 ms with 13% of the entries on the side, 1.43 ms with 10%;
// 1.60 ms with 16%, where the side kernel finishes last -- hence the
// cautious rate).  The two launches are joined by events, also inside a
// stream capture (the side stream is created by the first call outside
// one; a call under capture before that runs the slab kernel alone).
namespace {

constexpr double SIDE_RATE         = 0.75;
constexpr long long SIDE_MIN_ENTRIES = 512;

struct SideRes
{
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_side_mu;
SideRes g_side[64];

// the side stream and events of the current device; created outside
// capture only
bool side_resources(bool capturing, SideRes *&out)
{
  const int dev = device_info().device;
  if (dev < 0 || dev >= 64)
    return false;
  SideRes &r = g_side[dev];
  if (!r.stream)
  {
    if (capturing)
      return false;
    if (cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&r.fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&r.join, cudaEventDisableTiming) != cudaSuccess)
    {
      cudaGetLastError();
      if (r.stream)
        cudaStreamDestroy(r.stream);
      if (r.fork)
        cudaEventDestroy(r.fork);
      r = SideRes{};
      return false;
    }
  }
  out = &r;
  return true;
}

bool side_workspace(const Params &p, const Workspace &ws, long long L)
{
  if (p.layout == LAYOUT_BATCHED)
    return ws.W && ws.wstride >= L;
  if (ws.pW)
    return ws.pw_elems >= L && ws.npW >= 1;
  return ws.W && ws.Wbytes >= (size_t)L * sizeof(double);
}

} // namespace

int launch_slab_side(Params p, int prec, const Workspace &ws, int flags, cudaStream_t stream)
{
  const long long work = p.eend - p.ebase;
  long long L = 1;
  for (int l = 0; l < p.d; l++)
    L *= p.n[l];
  int used = 0;
  const int sms = device_info().sms;
  if (prec != PREC_F64 || (flags & KRON_SLAB_NO_SIDE) || work < SIDE_MIN_ENTRIES ||
      !big_supported(p, prec) || !side_workspace(p, ws, L) ||
      slab_sms_used(p.n[0], prec, flags, &used) != KRON_SUCCESS || sms - used < 2)
    return launch_slab(p, prec, flags, stream);
  const int idle       = sms - used;
  const long long side = (long long)((double)work * (idle * SIDE_RATE) / (used + idle * SIDE_RATE));
  if (side < 1)
    return launch_slab(p, prec, flags, stream);
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  // an error here (the legacy stream while another stream captures) counts
  // as capturing
  const bool capturing =
      cudaStreamIsCapturing(stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone;
  cudaGetLastError();
  std::lock_guard<std::mutex> lock(g_side_mu);
  SideRes *r = nullptr;
  if (!side_resources(capturing, r))
    return launch_slab(p, prec, flags, stream);
  Params ps = p, pb = p;
  ps.eend  = (int)(p.eend - side);
  pb.ebase = ps.eend;
  if (cudaEventRecord(r->fork, stream) != cudaSuccess ||
      cudaStreamWaitEvent(r->stream, r->fork, 0) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  // the slab kernel first, so that its clusters take their SMs before the
  // side kernel's blocks are placed
  const int rc1 = launch_slab(ps, prec, flags, stream);
  const int rc2 = launch_big(pb, ws, prec, 0, r->stream);
  if (cudaEventRecord(r->join, r->stream) != cudaSuccess ||
      cudaStreamWaitEvent(stream, r->join, 0) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  return rc1 != KRON_SUCCESS ? rc1 : rc2;
}

int launch_variant(Params p, int prec, const Workspace &ws, int variant, int param,
                   cudaStream_t stream)
{
  const bool merge = (p.accum == ACC_ATOMIC || p.accum == ACC_SEGMENTED);
  const int esize  = (prec == PREC_F32) ? 4 : 8;
  switch (variant)
  {
  case VAR_MMA8:
    return mma8_supported(p, prec) ? launch_mma8(p, stream) : KRON_ERROR_NOT_SUPPORTED;
  case VAR_PIPE:
    return pipe_supported(p, prec) ? launch_pipe(p, prec, stream) : KRON_ERROR_NOT_SUPPORTED;
  case VAR_SQ: {
    if (!is_square(p))
      return KRON_ERROR_NOT_SUPPORTED;
    const int ngmax = sq_entries_max(prec, p.d, p.n[0], merge);
    if (ngmax < 1)
      return KRON_ERROR_NOT_SUPPORTED;
    SqKernelInfo ki = pick_sq(prec, p.d, p.n[0], merge);
    if (!ki.fn)
      ki = pick_sq(prec, p.d, p.n[0], false);
    const int ng   = param > 0 ? std::min(param, ngmax) : ngmax;
    const int block = ng * ki.GS;
    size_t smem     = (size_t)ng * ki.group_bytes;
    void *args[]    = {&p};
    return launch_blocks(ki.fn, p.nitems, ng, block, smem, args, stream);
  }
  case VAR_GEN: {
    GenView v;
    if (gen_whole_view(p.d, p.m, p.n, merge, esize, v))
      return launch_gen_prec(prec, p, v, stream);
    if (merge && gen_whole_view(p.d, p.m, p.n, false, esize, v))
      return launch_gen_prec(prec, p, v, stream);
    return KRON_ERROR_NOT_SUPPORTED;
  }
  case VAR_BIG:
    return big_supported(p, prec) ? launch_big(p, ws, prec, param, stream)
                                  : KRON_ERROR_NOT_SUPPORTED;
  case VAR_SLAB:
    return slab_supported(p, prec) ? launch_slab_side(p, prec, ws, param, stream)
                                    : KRON_ERROR_NOT_SUPPORTED;
  case VAR_SPLIT_TC:
    return splittc_supported(p, prec) ? launch_splittc(p, ws, stream)
                                          : KRON_ERROR_NOT_SUPPORTED;
  case VAR_LARGE:
    if (prec == PREC_F32)
      return launch_large_t<float>(prec, p, ws, stream);
    return launch_large_t<double>(prec, p, ws, stream);
  default: return KRON_ERROR_NOT_SUPPORTED;
  }
}

int launch_kron(Params p, int prec, const Workspace &ws, cudaStream_t stream)
{
  if (p.batch <= 0 || p.eend <= p.ebase)
    return KRON_SUCCESS;
  setup_items(p, ws);
  if (p.nitems <= 0)
    return KRON_SUCCESS;

  // a variant recorded for this (d, n, precision) goes first; one that
  // cannot run this call (layout, accumulation mode, or a workspace the
  // caller did not pass) leaves it to the built-in order
  int tv = 0, tp = 0;
  if (is_square(p) && tune_lookup(p.d, p.n[0], prec, tv, tp))
  {
    const int rc = launch_variant(p, prec, ws, tv, tp, stream);
    if (rc != KRON_ERROR_NOT_SUPPORTED && rc != KRON_ERROR_WORKSPACE)
      return rc;
  }
  // default order: the specialised kernels, then the general ones
  // (VAR_SPLIT_TC: split precision at d = 6, n = 8 on the tcgen05 tensor
  // cores, 3.6 ms for 256 entries against 7.5 ms for the CUDA-core split)
  static const int order[] = {VAR_MMA8, VAR_PIPE,     VAR_SLAB, VAR_SQ,
                              VAR_GEN,  VAR_BIG,      VAR_SPLIT_TC, VAR_LARGE};
  for (int v : order)
  {
    if ((v == VAR_MMA8 && std::getenv("KRON_DISABLE_MMA8")) ||
        (v == VAR_PIPE && std::getenv("KRON_DISABLE_PIPE")) ||
        (v == VAR_SLAB && std::getenv("KRON_DISABLE_SLAB")) ||
        (v == VAR_BIG && std::getenv("KRON_DISABLE_BIG")) ||
        (v == VAR_SPLIT_TC && std::getenv("KRON_DISABLE_SPLIT_TC")))
      continue;
    const int rc = launch_variant(p, prec, ws, v, 0, stream);
    if (rc != KRON_ERROR_NOT_SUPPORTED)
      return rc;
  }
  return KRON_ERROR_NOT_SUPPORTED;
}

} // namespace kron

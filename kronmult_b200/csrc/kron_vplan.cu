// Uneven-batch plans: every entry has its own d and rectangular shapes
// (no reference counterpart; the reference's vbatched needs one launch per
// (d, shape) group, kronmult_vbatched.hpp:17-228, nearly one per entry at
// d >= 3 for random shapes).
//
// kron_vplan_create (host, once) builds a per-entry descriptor table:
//   - Alg. 993 order per entry: forward only when strictly cheaper
//     (kronm.hpp:39-89), and the largest intermediate of that order;
//   - a class by that size: "warp" (<= 512 elements: one warp per entry,
//     eight entries per block), "block" (fits the block's shared memory
//     twice: one block per entry), "huge" (beyond: a two-phase split, head
//     modes [0, q) and tail modes [q, d), sizes chosen like the uniform
//     path);
//   - every huge entry is cut into work items: row items (phase 1: the tail
//     modes on a range of head rows, written to the entry's own region of
//     the workspace) and tile items (phase 2: the head modes on a range of
//     column tiles of that region, added into y), so all SMs share the
//     largest entries;
//   - within each list, items sorted by cost, largest first.
// kron_vplan_execute_async runs one persistent kernel twice: stage 0 takes
// huge row items, then block-class entries, then warp-class entries from
// device work counters; stage 1 (after the launch boundary, the only
// dependency) takes the tile items.  On a non-default stream the counter
// reset and both launches are captured once into a CUDA graph and replayed
// while the operand arrays stay the same.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "kron_launch.h"

using namespace kron;

namespace {

constexpr int VP_THREADS  = 256;
constexpr int VP_WARPS    = VP_THREADS / 32;
constexpr int WARP_MAX    = 512;   // elements of the largest intermediate, warp class
constexpr int CLS_WARP = 0, CLS_QUAD = 1, CLS_HALF = 2, CLS_BLOCK = 3, CLS_HUGE = 4;
constexpr int NCLS     = 5;

struct VDesc
{
  long long woff;       // huge: element offset of the entry's workspace region
  int k;                // entry index (operands at pA[6k + l], pX[k], pY[k])
  unsigned char d, fwd, q, C;  // order; huge: head modes q, tile columns C
  unsigned char m[6], n[6];
  int mi;               // largest intermediate (elements) of the chosen order
  int mi2;              // huge: phase-2 buffer elements (tile rows x C)
  unsigned char fwd1, fwd2;         // huge: order of phase 1 / phase 2
  unsigned char pad[2];             // huge: [0] warp-parallel phase 1, [1] tail factor
                                    // elements / 16 (rounded up)
};

// a range [lo, hi) of head rows (phase 1) or column tiles (phase 2) of the
// huge entry desc[d]
struct VItem
{
  int d, lo, hi, pad;
};

struct VParams
{
  const VDesc *desc;          // [huge | block | half | quad | warp]
  const VItem *items;         // [row items | tile items]
  int nhuge, nblock, nhalf, nquad, nwarp;
  int nrow, ntile;
  int stage;                  // 0: row items, block and warp classes; 1: tile items
  int *counters;              // work counters (zeroed before every execution)
  const double *const *pA;
  const double *const *pX;
  double *const *pY;
  double *ws;                 // huge class: per-entry regions
  int block_elems;            // shared elements per block in block mode
};

// One entry (or one sub-block view of it) computed by a group of GS threads
// in the shared buffers b0/b1 (each >= v.max_inter) with factors in As.
__device__ __forceinline__ void vp_group_entry(const GenView &v, bool strided, const double *x,
                                               double *out, int accum, double *b0, double *b1,
                                               double *As, const double *const *A,
                                               const int *ld, int t, int GS, int g,
                                               bool load_a = true)
{
  if (load_a)
  {
    int o = 0;
    for (int q = 0; q < v.dd; q++)
    {
      const int l = v.mode0 + q, mq = v.mm[q], nq = v.nn[q];
      for (int u = t; u < mq * nq; u += GS)
      {
        const int j = u / mq, i = u - j * mq;
        As[o + u]   = __ldg(A[l] + i + (long long)j * ld[l]);
      }
      o += mq * nq;
    }
  }
  int rows_in = 1, rows_out = 1;
  for (int q = 0; q < v.dd; q++)
  {
    rows_in *= v.nn[q];
    rows_out *= v.mm[q];
  }
  if (!strided)
    group_copy_in(b0, x, rows_in, t, GS);
  else
    group_copy_tile(b0, x, rows_in, v.C, (int)v.total_cols, v.in_row, t, GS);
  group_sync(g, GS);
  double *cur = b0, *nxt = b1;
  gen_apply_modes<double, PREC_F64, true>(v, cur, nxt, As, v.C, t, GS, g);
  if (!strided)
    group_flush(accum, out, cur, cur, false, rows_out, t, GS);
  else
    for (int q = t; q < rows_out * v.C; q += GS)
    {
      const int i = q / v.C, c = q - i * v.C;
      if (c < v.total_cols)
        y_update(accum, out + i * v.out_row, c, cur[q]);
    }
  group_sync(g, GS);
}

__device__ __forceinline__ void vp_view(GenView &v, const VDesc &e, int mode0, int dd)
{
  v.dd    = dd;
  v.mode0 = mode0;
  for (int q = 0; q < dd; q++)
  {
    v.mm[q] = e.m[mode0 + q];
    v.nn[q] = e.n[mode0 + q];
  }
  v.forward = e.fwd;
  v.C       = 1;
  v.in_row = v.out_row = 1;
  v.total_cols         = 1;
}

__device__ __forceinline__ void vp_operands(const VParams &vp, const VDesc &e, const double *A[6],
                                            int ld[6], const double *&x, double *&y)
{
  for (int l = 0; l < 6; l++)
  {
    A[l]  = l < e.d ? vp.pA[6LL * e.k + l] : nullptr;
    ld[l] = l < e.d ? e.m[l] : 1;
  }
  x = vp.pX[e.k];
  y = vp.pY[e.k];
}

// Sizes of a huge entry's split: head inputs Nhead, tail inputs / outputs
// Ntail, Mtail (phase 1 maps each head row of Ntail elements to Mtail).
struct HugeDims
{
  int Nhead, Ntail, Mtail;
};

__device__ __forceinline__ HugeDims huge_dims(const VDesc &e)
{
  HugeDims h{1, 1, 1};
  for (int l = 0; l < e.q; l++)
    h.Nhead *= e.n[l];
  for (int l = e.q; l < e.d; l++)
  {
    h.Ntail *= e.n[l];
    h.Mtail *= e.m[l];
  }
  return h;
}

// next work item of a list for the whole block
__device__ __forceinline__ int block_take(int *counter, int *s_idx, int tid)
{
  if (tid == 0)
    *s_idx = atomicAdd(counter, 1);
  __syncthreads();
  const int idx = *s_idx;
  __syncthreads();
  return idx;
}

// Entries of one class run by groups of GS threads, VP_THREADS / GS per
// block, each group with its own slice of shared memory and named barrier.
template <int GS>
__device__ __forceinline__ void group_class(const VParams &vp, const VDesc *list, int n,
                                            int *counter, double *smem, int *s_gidx, int tid)
{
  constexpr int NG = VP_THREADS / GS;
  const int g = tid / GS, t = tid - (tid / GS) * GS;
  double *b0  = smem + (long long)g * ((vp.block_elems / NG) & ~1);
  const double *A[6];
  int ld[6];
  const double *x;
  double *y;
  while (true)
  {
    if (t == 0)
      s_gidx[g] = atomicAdd(counter, 1);
    group_sync(g, GS);
    const int idx = s_gidx[g];
    group_sync(g, GS);
    if (idx >= n)
      break;
    const VDesc e = list[idx];
    GenView v;
    vp_view(v, e, 0, e.d);
    vp_operands(vp, e, A, ld, x, y);
    const int mi = (e.mi + 1) & ~1;
    vp_group_entry(v, false, x, y, ACC_ATOMIC, b0, b0 + mi, b0 + 2 * mi, A, ld, t, GS, g);
  }
  __syncthreads(); // the next class lays its slices over these
}

// Stage 0: huge row items, then the block, half, quad and warp classes.
// Stage 1: huge tile items.  Counters: [0] row items, [1] block class,
// [2] warp class, [3] tile items, [4] half class, [5] quad class.
__global__ void __launch_bounds__(VP_THREADS, 2) kron_vplan_kernel(const __grid_constant__ VParams vp)
{
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_idx;
  __shared__ int s_gidx[4];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const double *A[6];
  int ld[6];
  const double *x;
  double *y;

  if (vp.stage == 1)
  {
    // ---- phase 2 of huge entries: head modes on column tiles -> y
    while (true)
    {
      const int idx = block_take(&vp.counters[3], &s_idx, tid);
      if (idx >= vp.ntile)
        break;
      const VItem it = vp.items[vp.nrow + idx];
      const VDesc e  = vp.desc[it.d];
      vp_operands(vp, e, A, ld, x, y);
      const HugeDims hd = huge_dims(e);
      const double *wr  = vp.ws + e.woff;
      GenView v2;
      vp_view(v2, e, 0, e.q);
      v2.forward = e.fwd2;
      v2.C       = e.C;
      v2.in_row = v2.out_row = hd.Mtail;
      const int mi2 = e.mi2;
      for (int t = it.lo; t < it.hi; t++)
      {
        const int c0  = t * e.C;
        v2.total_cols = min((int)e.C, hd.Mtail - c0);
        vp_group_entry(v2, true, wr + c0, y + c0, ACC_ATOMIC, smem, smem + mi2, smem + 2 * mi2,
                       A, ld, tid, VP_THREADS, 0);
      }
    }
    return;
  }

  // ---- phase 1 of huge entries: tail modes on head rows -> the entry's region
  while (true)
  {
    const int idx = block_take(&vp.counters[0], &s_idx, tid);
    if (idx >= vp.nrow)
      break;
    const VItem it = vp.items[idx];
    const VDesc e  = vp.desc[it.d];
    vp_operands(vp, e, A, ld, x, y);
    const HugeDims hd = huge_dims(e);
    double *wr        = vp.ws + e.woff;
    GenView v1;
    vp_view(v1, e, e.q, e.d - e.q);
    v1.forward    = e.fwd1;
    const int mi1 = e.mi;
    if (e.pad[0])
    {
      // one head row per warp (the plan checked that eight slices fit)
      const int slice = (2 * mi1 + e.pad[1] * 16 + 1) & ~1;
      double *b0      = smem + warp * slice;
      // the warp's factors stay in its slice from its first row on
      for (int h = it.lo + warp; h < it.hi; h += VP_WARPS)
        vp_group_entry(v1, false, x + (long long)h * hd.Ntail, wr + (long long)h * hd.Mtail,
                       ACC_STORE, b0, b0 + mi1, b0 + 2 * mi1, A, ld, lane, 32, warp,
                       h == it.lo + warp);
    }
    else
      for (int h = it.lo; h < it.hi; h++)
        vp_group_entry(v1, false, x + (long long)h * hd.Ntail, wr + (long long)h * hd.Mtail,
                       ACC_STORE, smem, smem + mi1, smem + 2 * mi1, A, ld, tid, VP_THREADS, 0,
                       h == it.lo);
    __syncthreads();
  }

  // ---- block class: the whole block per entry
  const VDesc *blk = vp.desc + vp.nhuge;
  while (true)
  {
    const int idx = block_take(&vp.counters[1], &s_idx, tid);
    if (idx >= vp.nblock)
      break;
    const VDesc e = blk[idx];
    GenView v;
    vp_view(v, e, 0, e.d);
    vp_operands(vp, e, A, ld, x, y);
    const int mi = (e.mi + 1) & ~1;
    vp_group_entry(v, false, x, y, ACC_ATOMIC, smem, smem + mi, smem + 2 * mi, A, ld, tid,
                   VP_THREADS, 0);
  }

  // ---- half and quad classes: two / four entries per block at a time
  {
    const VDesc *hd = vp.desc + vp.nhuge + vp.nblock;
    group_class<VP_THREADS / 2>(vp, hd, vp.nhalf, &vp.counters[4], smem, s_gidx, tid);
    group_class<VP_THREADS / 4>(vp, hd + vp.nhalf, vp.nquad, &vp.counters[5], smem, s_gidx, tid);
  }

  // ---- warp class: one warp per entry
  const int slice = vp.block_elems / VP_WARPS;
  double *b0      = smem + warp * slice;
  const VDesc *wd = vp.desc + vp.nhuge + vp.nblock + vp.nhalf + vp.nquad;
  while (true)
  {
    int idx = 0;
    if (lane == 0)
      idx = atomicAdd(&vp.counters[2], 1);
    idx = __shfl_sync(0xffffffffu, idx, 0);
    if (idx >= vp.nwarp)
      break;
    const VDesc e = wd[idx];
    GenView v;
    vp_view(v, e, 0, e.d);
    vp_operands(vp, e, A, ld, x, y);
    vp_group_entry(v, false, x, y, ACC_ATOMIC, b0, b0 + WARP_MAX, b0 + 2 * WARP_MAX, A, ld, lane,
                   32, warp);
  }
}

} // namespace

struct kron_vplan_st
{
  int batch;
  int nhuge, nblock, nhalf, nquad, nwarp;
  int nrow, ntile;
  VDesc *d_desc;
  VItem *d_items;
  int *d_counters;
  double flops;
  size_t ws_bytes;
  size_t smem_main, smem_huge, smem_tile;
  int block_elems;
  // graph cache
  cudaGraphExec_t exec;
  const void *gA, *gX, *gY, *gW;
  size_t gWcap;
};

extern "C" int kron_vplan_create(kron_vplan_t *plan, int batchCount, int const shapes[])
{
  if (!plan || batchCount < 0 || (batchCount > 0 && !shapes))
    return KRON_ERROR_INVALID_VALUE;
  *plan = nullptr;
  const DeviceInfo &di = device_info();
  const int maxsm      = di.max_smem_optin;
  // block class: two buffers + factors within the block's shared memory
  const int block_elems = (maxsm - 4096) / 8;
  std::vector<VDesc> cls[NCLS];
  std::vector<double> cost[NCLS];
  double total_flops   = 0.0;
  size_t smem_huge     = 0;
  size_t smem_tile     = 0;
  for (int k = 0; k < batchCount; k++)
  {
    const int *s = shapes + 13LL * k;
    VDesc e;
    std::memset(&e, 0, sizeof(e));
    e.k     = k;
    const int d = s[0];
    if (d < 1 || d > MAXD)
      return KRON_ERROR_INVALID_VALUE;
    int m[MAXD], n[MAXD];
    for (int l = 0; l < d; l++)
    {
      m[l] = s[1 + 2 * l];
      n[l] = s[2 + 2 * l];
      if (m[l] < 1 || n[l] < 1 || m[l] > 255 || n[l] > 255)
        return KRON_ERROR_INVALID_VALUE;
      e.m[l] = (unsigned char)m[l];
      e.n[l] = (unsigned char)n[l];
    }
    e.d              = (unsigned char)d;
    const bool fwd   = choose_forward(d, m, n);
    e.fwd            = fwd ? 1 : 0;
    const long long mi = max_intermediate(d, m, n, fwd);
    const double fl  = std::min(flops_forward(d, m, n), flops_backward(d, m, n));
    total_flops += fl;
    long long asz = 0;
    for (int l = 0; l < d; l++)
      asz += (long long)m[l] * n[l];
    const long long mi2r = (mi + 1) & ~1LL;
    int c;
    const long long need = 2 * mi2r + asz;
    if (mi <= WARP_MAX && 2 * WARP_MAX + asz <= block_elems / VP_WARPS)
      c = CLS_WARP;
    else if (need <= ((block_elems / 4) & ~1))
      c = CLS_QUAD;
    else if (need <= ((block_elems / 2) & ~1))
      c = CLS_HALF;
    else if (need <= block_elems)
      c = CLS_BLOCK;
    else
    {
      c = CLS_HUGE;
      LargePlan lp;
      if (!plan_large(d, m, n, 8, false, lp) || lp.C > 255)
        return KRON_ERROR_NOT_SUPPORTED;
      e.q    = (unsigned char)lp.q;
      e.fwd1 = (unsigned char)lp.v1.forward;
      e.fwd2 = (unsigned char)lp.v2.forward;
      // phase-2 tiles narrowed so that one fits half the shared memory (two
      // blocks per SM run the tile launch)
      {
        const long long rows2 = std::max<long long>(1, lp.v2.max_inter / std::max(1, lp.C));
        const long long budget = (long long)(maxsm / 2 - 1024) / 8 - lp.v2.asz;
        long long C2 = std::min<long long>(lp.C, budget / (2 * rows2));
        if (C2 < 1)
          C2 = lp.C; // keep the plan's width; the tile launch then runs one block per SM
        e.C   = (unsigned char)C2;
        e.mi2 = (int)((rows2 * C2 + 1) & ~1LL);
        smem_tile = std::max(smem_tile, (size_t)(2 * e.mi2 + lp.v2.asz + 2) * 8);
      }
      size_t need = (size_t)std::max(lp.v1.group_elems, lp.v2.group_elems) * 8;
      // phase 1 one block per warp when eight slices fit
      const long long a16   = (lp.v1.asz + 15) / 16;
      const long long slice = (2LL * lp.v1.max_inter + a16 * 16 + 1) & ~1LL;
      if (a16 < 256 && (size_t)(VP_WARPS * slice * 8) <= (size_t)(maxsm - 1024))
      {
        e.pad[0] = 1;
        e.pad[1] = (unsigned char)a16;
        need     = std::max(need, (size_t)(VP_WARPS * slice * 8));
      }
      smem_huge = std::max(smem_huge, need);
    }
    e.mi = (c == CLS_HUGE) ? 0 : (int)mi;
    if (c == CLS_HUGE)
    {
      LargePlan lp;
      plan_large(d, m, n, 8, false, lp);
      e.mi = lp.v1.max_inter; // phase-1 buffer elements, rounded
    }
    cls[c].push_back(e);
    cost[c].push_back(fl);
  }
  kron_vplan_st *pl = new (std::nothrow) kron_vplan_st();
  if (!pl)
    return KRON_ERROR_ALLOC;
  std::vector<VDesc> all;
  all.reserve(batchCount);
  for (int c : {CLS_HUGE, CLS_BLOCK, CLS_HALF, CLS_QUAD, CLS_WARP})
  {
    std::vector<int> order(cls[c].size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return cost[c][a] > cost[c][b]; });
    for (int i : order)
      all.push_back(cls[c][i]);
  }
  pl->batch  = batchCount;
  pl->nhuge  = (int)cls[CLS_HUGE].size();
  pl->nblock = (int)cls[CLS_BLOCK].size();
  pl->nhalf  = (int)cls[CLS_HALF].size();
  pl->nquad  = (int)cls[CLS_QUAD].size();
  pl->nwarp  = (int)cls[CLS_WARP].size();

  // workspace regions and work items of the huge entries: row items of
  // about 32k input elements (whole warps' worth of rows), tile items of one
  // column tile; each list largest first
  std::vector<VItem> rows, tiles;
  std::vector<double> rcost, tcost;
  long long woff = 0;
  for (int i = 0; i < pl->nhuge; i++)
  {
    VDesc &e = all[i];
    e.woff   = woff;
    long long Nhead = 1, Ntail = 1, Mtail = 1, Mhead = 1;
    for (int l = 0; l < e.q; l++)
    {
      Nhead *= e.n[l];
      Mhead *= e.m[l];
    }
    for (int l = e.q; l < e.d; l++)
    {
      Ntail *= e.n[l];
      Mtail *= e.m[l];
    }
    woff += (Nhead * Mtail + 1) & ~1LL;
    long long rpi = std::max<long long>(1, 32768 / std::max<long long>(1, Ntail));
    rpi           = std::max<long long>(VP_WARPS, (rpi + VP_WARPS - 1) / VP_WARPS * VP_WARPS);
    for (long long h0 = 0; h0 < Nhead; h0 += rpi)
    {
      const long long h1 = std::min(Nhead, h0 + rpi);
      rows.push_back(VItem{i, (int)h0, (int)h1, 0});
      rcost.push_back((double)(h1 - h0) * (double)(Ntail + Mtail));
    }
    const long long nt = (Mtail + e.C - 1) / e.C;
    for (long long t = 0; t < nt; t++)
    {
      tiles.push_back(VItem{i, (int)t, (int)t + 1, 0});
      tcost.push_back((double)std::min<long long>(e.C, Mtail - t * e.C) * (double)(Nhead + Mhead));
    }
  }
  auto sorted = [](std::vector<VItem> &v, const std::vector<double> &c) {
    std::vector<int> o(v.size());
    std::iota(o.begin(), o.end(), 0);
    std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return c[a] > c[b]; });
    std::vector<VItem> r;
    r.reserve(v.size());
    for (int i : o)
      r.push_back(v[i]);
    return r;
  };
  std::vector<VItem> items = sorted(rows, rcost);
  {
    std::vector<VItem> t = sorted(tiles, tcost);
    items.insert(items.end(), t.begin(), t.end());
  }
  pl->nrow        = (int)rows.size();
  pl->ntile       = (int)tiles.size();
  pl->flops       = total_flops;
  pl->block_elems = block_elems;
  pl->smem_main   = (size_t)block_elems * 8;
  pl->smem_huge   = std::max<size_t>(smem_huge, 16);
  pl->smem_tile   = std::max<size_t>(smem_tile, 16);
  pl->ws_bytes    = (size_t)woff * 8;
  pl->exec        = nullptr;
  pl->d_desc      = nullptr;
  pl->d_items     = nullptr;
  pl->d_counters  = nullptr;
  if (kron::dev_malloc((void **)&pl->d_counters, 8 * sizeof(int)) != cudaSuccess ||
      (batchCount > 0 && kron::dev_malloc((void **)&pl->d_desc, sizeof(VDesc) * batchCount) != cudaSuccess) ||
      (!items.empty() && kron::dev_malloc((void **)&pl->d_items, sizeof(VItem) * items.size()) != cudaSuccess))
  {
    kron::dev_free(pl->d_items);
    kron::dev_free(pl->d_desc);
    kron::dev_free(pl->d_counters);
    delete pl;
    return KRON_ERROR_ALLOC;
  }
  if ((batchCount > 0 && cudaMemcpy(pl->d_desc, all.data(), sizeof(VDesc) * batchCount,
                                    cudaMemcpyHostToDevice) != cudaSuccess) ||
      (!items.empty() && cudaMemcpy(pl->d_items, items.data(), sizeof(VItem) * items.size(),
                                    cudaMemcpyHostToDevice) != cudaSuccess))
  {
    kron::dev_free(pl->d_items);
    kron::dev_free(pl->d_desc);
    kron::dev_free(pl->d_counters);
    delete pl;
    return KRON_ERROR_LAUNCH;
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
  kron::dev_free(plan->d_items);
  kron::dev_free(plan->d_desc);
  kron::dev_free(plan->d_counters);
  delete plan;
  return KRON_SUCCESS;
}

extern "C" size_t kron_vplan_workspace_bytes(kron_vplan_t plan) { return plan ? plan->ws_bytes : 0; }
extern "C" double kron_vplan_flops(kron_vplan_t plan) { return plan ? plan->flops : 0.0; }

static int vplan_launch_all(kron_vplan_t pl, double const *const *A, double **X, double **Y,
                            void *W, cudaStream_t s)
{
  if (cudaMemsetAsync(pl->d_counters, 0, 8 * sizeof(int), s) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  VParams vp;
  std::memset(&vp, 0, sizeof(vp));
  vp.desc        = pl->d_desc;
  vp.items       = pl->d_items;
  vp.nhuge       = pl->nhuge;
  vp.nblock      = pl->nblock;
  vp.nhalf       = pl->nhalf;
  vp.nquad       = pl->nquad;
  vp.nwarp       = pl->nwarp;
  vp.nrow        = pl->nrow;
  vp.ntile       = pl->ntile;
  vp.counters    = pl->d_counters;
  vp.pA          = A;
  vp.pX          = X;
  vp.pY          = Y;
  vp.ws          = static_cast<double *>(W);
  vp.block_elems = pl->block_elems;
  void *args[]   = {&vp};
  const int sms  = device_info().sms;
  const void *fm = reinterpret_cast<const void *>(&kron_vplan_kernel);
  const size_t smem = std::max(pl->smem_main, pl->smem_huge);
  int occ           = 1;
  if (cached_occupancy(fm, VP_THREADS, smem, &occ) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  const long long work0 = (long long)pl->nrow + pl->nblock + (pl->nhalf + 1) / 2 +
                          (pl->nquad + 3) / 4 + (pl->nwarp + VP_WARPS - 1) / VP_WARPS;
  if (work0 > 0)
  {
    vp.stage       = 0;
    const int grid = (int)std::max<long long>(1, std::min<long long>((long long)sms * occ, work0));
    if (cudaLaunchKernel(fm, dim3(grid), dim3(VP_THREADS), args, smem, s) != cudaSuccess)
      return KRON_ERROR_LAUNCH;
  }
  if (pl->ntile > 0)
  {
    vp.stage   = 1;
    int occ1   = 1;
    if (cached_occupancy(fm, VP_THREADS, pl->smem_tile, &occ1) != KRON_SUCCESS)
      return KRON_ERROR_LAUNCH;
    const int grid = std::max(1, std::min(sms * occ1, pl->ntile));
    if (cudaLaunchKernel(fm, dim3(grid), dim3(VP_THREADS), args, pl->smem_tile, s) !=
        cudaSuccess)
      return KRON_ERROR_LAUNCH;
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
  if (plan->ws_bytes > 0 && (!W || Wcapacity_bytes < plan->ws_bytes))
    return KRON_ERROR_WORKSPACE;

  // Graphs only on explicit streams that are not already capturing.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  bool use_graph             = (s != nullptr) && cudaStreamIsCapturing(s, &cs) == cudaSuccess &&
                   cs == cudaStreamCaptureStatusNone;
  if (!use_graph)
  {
    int rc = vplan_launch_all(plan, Aarray_, pX_, pY_, W, s);
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
    // kernel attributes are set outside the capture
    int rc = vplan_launch_all(plan, Aarray_, pX_, pY_, W, s);
    if (rc != KRON_SUCCESS)
      return rc;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
      return KRON_ERROR_LAUNCH;
    rc             = vplan_launch_all(plan, Aarray_, pX_, pY_, W, s);
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
    return KRON_SUCCESS; // this execution ran directly above
  }
  return cudaGraphLaunch(plan->exec, s) == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

// Uneven-batch plans: every entry has its own d and rectangular shapes
// (no reference counterpart; the reference's vbatched needs one launch per
// (d, shape) group, kronmult_vbatched.hpp:17-228, nearly one per entry at
// d >= 3 for random shapes).
//
// kron_vplan_create (host, once) builds a per-entry descriptor table:
//   - Alg. 993 order per entry: forward only when strictly cheaper
//     (kronm.hpp:39-89), and the largest intermediate of that order;
//   - a class by the shared memory the entry needs (two buffers of that
//     intermediate plus its factors) against the per-block budget, half of
//     an SM so that two blocks share each SM: "warp" (<= 512 elements: one
//     warp per entry), "quad" / "half" / "block" (a quarter, a half or all
//     of a block per entry), "huge" (beyond: a two-phase split, head modes
//     [0, q) and tail modes [q, d));
//   - every huge entry is cut into work items: chunk items (phase 1: the
//     tail modes on as many head rows as one block's buffers hold, written
//     to the entry's own region of the workspace) and tile items (phase 2:
//     the head modes on one column tile of that region, added into y);
//   - one queue of huge items, largest entries first, where each entry's
//     tile items follow its chunk items by a lag (a few hundred items, at
//     most ~40 MB of live regions): a tile item waits (bounded) on its
//     entry's chunk counter, which by then is normally complete, and the
//     region it reads is still in L2.
// kron_vplan_execute_async runs one persistent kernel: the huge queue, then
// the block, half, quad and warp classes, each from its own device work
// counter.  All operands reach shared memory by cp.async, so a block keeps
// every byte of its current item in flight at once.  On a non-default
// stream the counter reset and the launch are captured once into a CUDA
// graph and replayed while the operand arrays stay the same.
#include <algorithm>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "kron_launch.h"
#include "kron_ptx.cuh"

using namespace kron;

namespace {

constexpr int VP_THREADS = 256;
constexpr int VP_WARPS   = VP_THREADS / 32;
constexpr int VP_MINB    = 2;     // blocks per SM the shared-memory budget leaves room for
constexpr int WARP_MAX   = 512;   // elements of the largest intermediate, warp class
constexpr int CLS_WARP = 0, CLS_QUAD = 1, CLS_HALF = 2, CLS_BLOCK = 3, CLS_HUGE = 4;
constexpr int NCLS   = 5;
constexpr int NCOUNT = 8;         // work counters ahead of the per-entry chunk counters

struct VDesc
{
  // fetched as twelve 32-bit words by the kernel's fetch stages
  long long woff;       // huge: element offset of the entry's workspace region
  int k;                // entry index (operands at pA[6k + l], pX[k], pY[k])
  unsigned char d, fwd, q, C;  // order; huge: head modes q, tile columns C
  unsigned char m[6], n[6];
  int mi;               // buffer elements: the largest intermediate of the chosen
                        // order (huge: of one chunk of R head rows)
  int mi2;              // huge: phase-2 buffer elements (tile rows x C)
  unsigned char fwd1, fwd2;   // huge: order of the tail / head modes
  unsigned short R;           // huge: head rows per chunk item
  int nchunk;                 // huge: chunk items (its tile items wait for all)
};

static_assert(sizeof(VDesc) == 48, "VDesc is fetched as 12 words");

// kind 0: chunk item, head rows [lo, hi); kind 1: tile item, column tile lo
// of the huge entry desc[e]
struct VItem
{
  int e, lo, hi, kind;
};

struct VParams
{
  const VDesc *desc;          // [huge | block | half | quad | warp]
  const VItem *items;         // the huge queue
  int nhuge, nblock, nhalf, nquad, nwarp;
  int nitems;
  int *counters;              // [0] huge queue, [1] block, [2] warp, [4] half,
                              // [5] quad; [NCOUNT + i] chunks done of huge entry i
  int *status;                // the library's device status word
  long long spin;             // polls before a chunk wait gives up
  const double *const *pA;
  const double *const *pX;
  double *const *pY;
  double *ws;                 // huge class: per-entry regions
  int budget;                 // shared elements per block
};

// 8-byte global -> shared copy through the LSU's asynchronous path
// (zero-filled when !valid; src must still point into the operand).
__device__ __forceinline__ void cp8(double *dst, const double *src, bool valid = true)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(ptx::smem_addr(dst)),
               "l"(src), "r"(valid ? 8 : 0)
               : "memory");
}

__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ int ld_acquire(const int *p)
{
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// The view's factors (leading dimension m_l: each contiguous) into As.
__device__ __forceinline__ void vp_load_factors(const GenView &v, double *As,
                                                const double *const *A, int t, int GS)
{
  int o = 0;
  for (int q = 0; q < v.dd; q++)
  {
    const int sz    = v.mm[q] * v.nn[q];
    const double *a = A[v.mode0 + q];
    for (int u = t; u < sz; u += GS)
      cp8(As + o + u, a + u);
    o += sz;
  }
}

// rows consecutive vectors of the view (x contiguous) computed by a group
// of GS threads in buffers b0 / b1 (each >= rows x the largest
// intermediate), factors at As; the results go to out (contiguous).
// hook(s) runs the next item's fetch stage s at four points: after the
// copies are issued, after they land, before the results go out, and
// before the closing barrier.
template <typename Hook>
__device__ __forceinline__ void vp_run(const GenView &v, int rows, const double *x, double *out,
                                       int accum, double *b0, double *b1, double *As,
                                       const double *const *A, int t, int GS, int g,
                                       const Hook &hook)
{
  vp_load_factors(v, As, A, t, GS);
  int rin = rows, rout = rows;
  for (int q = 0; q < v.dd; q++)
  {
    rin *= v.nn[q];
    rout *= v.mm[q];
  }
  for (int i = t; i < rin; i += GS)
    cp8(b0 + i, x + i);
  hook(1);
  cp_wait_all();
  group_sync(g, GS);
  hook(2);
  double *cur = b0, *nxt = b1;
  gen_apply_modes<double, PREC_F64, true>(v, cur, nxt, As, 1, t, GS, g, rows);
  hook(3);
  group_flush(accum, out, cur, cur, false, rout, t, GS);
  hook(4);
  group_sync(g, GS);
}

// One column tile of a huge entry's region: rows of C columns at stride
// in_row (the first Cc valid, the rest zero-filled), the head modes, and
// the Cc valid columns added into y (row stride out_row).  Whole block;
// hook as for vp_run.
template <typename Hook>
__device__ __forceinline__ void vp_run_tile(const GenView &v, const double *w, long long in_row,
                                            int C, int Cc, double *y, long long out_row,
                                            double *b0, double *b1, double *As,
                                            const double *const *A, int tid, const Hook &hook)
{
  vp_load_factors(v, As, A, tid, VP_THREADS);
  int rin = 1, rout = 1;
  for (int q = 0; q < v.dd; q++)
  {
    rin *= v.nn[q];
    rout *= v.mm[q];
  }
  const int lane = tid & 31, warp = tid >> 5;
  for (int h = warp; h < rin; h += VP_WARPS)
    for (int c = lane; c < C; c += 32)
      cp8(b0 + h * C + c, w + h * in_row + (c < Cc ? c : 0), c < Cc);
  hook(1);
  cp_wait_all();
  __syncthreads();
  hook(2);
  double *cur = b0, *nxt = b1;
  gen_apply_modes<double, PREC_F64, true>(v, cur, nxt, As, C, tid, VP_THREADS, 0);
  hook(3);
  for (int i = warp; i < rout; i += VP_WARPS)
    for (int c = lane; c < Cc; c += 32)
      red_add(y + i * out_row + c, cur[i * C + c]);
  hook(4);
  __syncthreads();
}

// What a group needs to start its next item, in shared memory.  The
// group's first warp fetches it in stages during the current item, one
// dependent load per stage (queue index, item, descriptor, operand
// pointers), so none of those round trips stalls the group.
struct NextSlot
{
  int idx;               // queue / list position (>= the count: no more work)
  int ready;             // huge tile item: its entry's chunks were complete
  VItem it;              // huge queue only
  VDesc e;
  const double *ptr[8];  // A_1..A_6, x, y
};

// The fetching warp's registers between stages.
struct Fetch
{
  int r;                 // lane 0: the counter's old value; lanes: a word in flight
  int nidx;
  const double *p;       // lanes 0-7: a pointer in flight
};

// Stages of the fetch for the huge queue (kind = true) or a class list.
// Stage 0 takes the next position; 1 loads the item (huge) or the
// descriptor; 2 stores it and loads the descriptor (huge) or the pointers;
// 3 and 4 finish.  Every store to the slot happens after the current item
// has read the slot (the first barrier of the item lies between).
template <bool HUGE>
__device__ __forceinline__ void fetch_stage(int s, Fetch &f, NextSlot &slot, const VParams &vp,
                                            const VDesc *list, int n, int *counter, int lane)
{
  const unsigned FULL = 0xffffffffu;
  if (s == 0)
  {
    if (lane == 0)
      f.r = atomicAdd(counter, 1);
    return;
  }
  if (s == 1)
  {
    f.nidx = __shfl_sync(FULL, f.r, 0);
    if (f.nidx < n)
    {
      if (HUGE && lane < 4)
        f.r = reinterpret_cast<const int *>(vp.items + f.nidx)[lane];
      if (!HUGE && lane < 12)
        f.r = reinterpret_cast<const int *>(list + f.nidx)[lane];
    }
    return;
  }
  const bool more = f.nidx < n;
  if (HUGE)
  {
    if (s == 2)
    {
      if (lane == 0)
        slot.idx = f.nidx;
      if (more && lane < 4)
        reinterpret_cast<int *>(&slot.it)[lane] = f.r;
      __syncwarp();
      if (more && lane < 12)
        f.r = reinterpret_cast<const int *>(vp.desc + slot.it.e)[lane];
    }
    else if (s == 3)
    {
      if (more && lane < 12)
        reinterpret_cast<int *>(&slot.e)[lane] = f.r;
      __syncwarp();
      if (more && lane < 8)
      {
        const int k = slot.e.k, d = slot.e.d;
        f.p = lane < 6 ? (lane < d ? vp.pA[6LL * k + lane] : nullptr)
                       : (lane == 6 ? vp.pX[k] : vp.pY[k]);
      }
      if (more && lane == 8)
        f.r = slot.it.kind == 1 && ld_acquire(vp.counters + NCOUNT + slot.it.e) >= slot.e.nchunk;
    }
    else
    {
      if (more && lane < 8)
        slot.ptr[lane] = f.p;
      if (more && lane == 8)
        slot.ready = f.r;
    }
  }
  else
  {
    if (s == 2)
    {
      if (lane == 0)
        slot.idx = f.nidx;
      if (more && lane < 12)
        reinterpret_cast<int *>(&slot.e)[lane] = f.r;
      __syncwarp();
      if (more && lane < 8)
      {
        const int k = slot.e.k, d = slot.e.d;
        f.p = lane < 6 ? (lane < d ? vp.pA[6LL * k + lane] : nullptr)
                       : (lane == 6 ? vp.pX[k] : vp.pY[k]);
      }
    }
    else if (s == 3)
    {
      if (more && lane < 8)
        slot.ptr[lane] = f.p;
    }
  }
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

// Thread 0 polls the entry's chunk counter (acquire) until `need` chunk
// items are done, at most `spin` polls; on giving up it records 1 in the
// status word.  Returns the outcome to the whole block.
__device__ __forceinline__ bool vp_wait_chunks(const VParams &vp, int e, int need, int *s_flag,
                                               int tid)
{
  if (tid == 0)
  {
    const int *done = vp.counters + NCOUNT + e;
    int ok          = 1;
    long long polls = 0;
    while (ld_acquire(done) < need)
    {
      if (++polls > vp.spin)
      {
        ok = 0;
        if (vp.status)
          atomicExch(vp.status, 1);
        break;
      }
      __nanosleep(64);
    }
    __threadfence();
    *s_flag = ok;
  }
  __syncthreads();
  return *s_flag != 0;
}

// Read the slot into the item's registers (every thread of the group).
__device__ __forceinline__ void slot_read(const NextSlot &slot, VDesc &e, const double *A[6],
                                          const double *&x, double *&y)
{
  e = slot.e;
  for (int l = 0; l < 6; l++)
    A[l] = slot.ptr[l];
  x = slot.ptr[6];
  y = const_cast<double *>(slot.ptr[7]);
}

// Entries of one class run by groups of GS threads, VP_THREADS / GS per
// block, each group with its own slice of shared memory, barrier and slot.
template <int GS>
__device__ __forceinline__ void group_class(const VParams &vp, const VDesc *list, int n,
                                            int *counter, double *smem, NextSlot *slots, int tid)
{
  constexpr int NG = VP_THREADS / GS;
  const int g = tid / GS, t = tid - (tid / GS) * GS, lane = tid & 31;
  double *b0     = smem + (long long)g * ((vp.budget / NG) & ~1);
  NextSlot &slot = slots[g];
  const bool fw  = t < 32; // the group's first warp fetches
  Fetch f{0, 0, nullptr};
  if (fw)
    for (int st = 0; st < 4; st++)
    {
      fetch_stage<false>(st, f, slot, vp, list, n, counter, lane);
      __syncwarp();
    }
  group_sync(g, GS);
  const double *A[6];
  const double *x;
  double *y;
  VDesc e;
  while (true)
  {
    const int idx = slot.idx;
    if (idx >= n)
      break;
    slot_read(slot, e, A, x, y);
    if (fw)
      fetch_stage<false>(0, f, slot, vp, list, n, counter, lane);
    GenView v;
    vp_view(v, e, 0, e.d);
    vp_run(v, 1, x, y, ACC_ATOMIC, b0, b0 + e.mi, b0 + 2 * e.mi, A, t, GS, g, [&](int st) {
      if (fw && st < 4)
        fetch_stage<false>(st, f, slot, vp, list, n, counter, lane);
    });
  }
  __syncthreads(); // the next class lays its slices (and slots) over these
}

// The huge queue, then the block, half, quad and warp classes.
__global__ void __launch_bounds__(VP_THREADS, VP_MINB)
    kron_vplan_kernel(const __grid_constant__ VParams vp)
{
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_flag;
  __shared__ NextSlot s_slot[VP_WARPS];
  const int tid = threadIdx.x, lane = tid & 31;
  const bool fw = tid < 32;
  const double *A[6];
  const double *x;
  double *y;
  VDesc e;
  bool dead = false; // a chunk wait of this block gave up: skip later tile items

  NextSlot &slot = s_slot[0];
  Fetch f{0, 0, nullptr};
  if (fw)
    for (int st = 0; st < 5; st++)
    {
      fetch_stage<true>(st, f, slot, vp, nullptr, vp.nitems, &vp.counters[0], lane);
      __syncwarp();
    }
  __syncthreads();
  auto hook = [&](int st) {
    if (fw)
      fetch_stage<true>(st, f, slot, vp, nullptr, vp.nitems, &vp.counters[0], lane);
  };
  while (true)
  {
    if (slot.idx >= vp.nitems)
      break;
    const VItem it   = slot.it;
    const bool ready = slot.ready != 0;
    slot_read(slot, e, A, x, y);
    if (fw)
      fetch_stage<true>(0, f, slot, vp, nullptr, vp.nitems, &vp.counters[0], lane);
    const HugeDims hd = huge_dims(e);
    double *wr        = vp.ws + e.woff;
    if (it.kind == 0)
    {
      // phase 1: tail modes on head rows [lo, hi) -> the entry's region
      GenView v1;
      vp_view(v1, e, e.q, e.d - e.q);
      v1.forward = e.fwd1;
      vp_run(v1, it.hi - it.lo, x + (long long)it.lo * hd.Ntail,
             wr + (long long)it.lo * hd.Mtail, ACC_STORE, smem, smem + e.mi, smem + 2 * e.mi, A,
             tid, VP_THREADS, 0, hook);
      // vp_run ended with a block barrier: every store of the chunk is issued
      if (tid == 0)
      {
        __threadfence();
        atomicAdd(vp.counters + NCOUNT + it.e, 1);
      }
    }
    else
    {
      // phase 2: head modes on column tile lo of the region -> y
      if (!ready && !dead && !vp_wait_chunks(vp, it.e, e.nchunk, &s_flag, tid))
        dead = true;
      if (dead)
      {
        // keep the fetch going: the stages still run, the tile does not
        for (int st = 1; st < 5; st++)
        {
          hook(st);
          __syncthreads();
        }
        continue;
      }
      GenView v2;
      vp_view(v2, e, 0, e.q);
      v2.forward   = e.fwd2;
      const int c0 = it.lo * e.C;
      vp_run_tile(v2, wr + c0, hd.Mtail, e.C, min((int)e.C, hd.Mtail - c0), y + c0, hd.Mtail,
                  smem, smem + e.mi2, smem + 2 * e.mi2, A, tid, hook);
    }
  }
  __syncthreads();

  const VDesc *blk = vp.desc + vp.nhuge;
  group_class<VP_THREADS>(vp, blk, vp.nblock, &vp.counters[1], smem, s_slot, tid);
  blk += vp.nblock;
  group_class<VP_THREADS / 2>(vp, blk, vp.nhalf, &vp.counters[4], smem, s_slot, tid);
  blk += vp.nhalf;
  group_class<VP_THREADS / 4>(vp, blk, vp.nquad, &vp.counters[5], smem, s_slot, tid);
  blk += vp.nquad;
  group_class<32>(vp, blk, vp.nwarp, &vp.counters[2], smem, s_slot, tid);
}

} // namespace

struct kron_vplan_st
{
  int batch;
  int nhuge, nblock, nhalf, nquad, nwarp;
  int nitems;
  VDesc *d_desc;
  VItem *d_items;
  int *d_counters;            // NCOUNT work counters + one chunk counter per huge entry
  double flops;
  size_t ws_bytes;
  int budget;                 // shared elements per block
  int grid_work;              // work units of the launch (grid upper bound)
  // graph cache
  cudaGraphExec_t exec;
  const void *gA, *gX, *gY, *gW;
  size_t gWcap;
};

namespace {

long long even(long long v) { return (v + 1) & ~1LL; }

// Two-phase split of a huge entry for a block of `budget` shared elements:
// phase 1 applies modes [q, d) to chunks of R head rows, phase 2 modes
// [0, q) to column tiles of C columns.  Prefers tiles of >= 16 columns
// (128-byte row segments), then the smallest region (Nhead x Mtail).
struct HugeSplit
{
  int q, C, R, fwd1, fwd2;
  long long mi1, mi2; // buffer elements: per head row (phase 1), per column (phase 2)
};

bool plan_huge(int d, const int *m, const int *n, long long budget, HugeSplit &best)
{
  bool found = false;
  long long best_w = 0;
  int best_c = 0;
  for (int q = 1; q < d; q++)
  {
    const bool f1    = choose_forward(d - q, m + q, n + q);
    const bool f2    = choose_forward(q, m, n);
    const long long r1 = max_intermediate(d - q, m + q, n + q, f1);
    const long long r2 = max_intermediate(q, m, n, f2);
    long long a1 = 0, a2 = 0, Nhead = 1, Mtail = 1;
    for (int l = 0; l < q; l++)
    {
      a2 += (long long)m[l] * n[l];
      Nhead *= n[l];
    }
    for (int l = q; l < d; l++)
    {
      a1 += (long long)m[l] * n[l];
      Mtail *= m[l];
    }
    const long long R = (budget - even(a1) - 2) / (2 * r1);
    const long long C = std::min<long long>({255, Mtail, (budget - even(a2) - 2) / (2 * r2)});
    if (R < 1 || C < 1)
      continue;
    const int cq        = (int)std::min<long long>(C, 16);
    const long long wsz = Nhead * Mtail;
    if (!found || cq > best_c || (cq == best_c && wsz < best_w))
    {
      best = HugeSplit{q, (int)C, (int)std::min<long long>(R, 65535), f1 ? 1 : 0, f2 ? 1 : 0,
                       r1, r2};
      best_c = cq;
      best_w = wsz;
      found  = true;
    }
  }
  return found;
}

} // namespace

extern "C" int kron_vplan_create(kron_vplan_t *plan, int batchCount, int const shapes[])
{
  if (!plan || batchCount < 0 || (batchCount > 0 && !shapes))
    return KRON_ERROR_INVALID_VALUE;
  *plan = nullptr;
  const DeviceInfo &di = device_info();
  // shared elements per block: two blocks per SM (1 KB of each block's share
  // is reserved by the hardware; 2 KB cover the kernel's own variables)
  const long long budget =
      (std::min<long long>(di.max_smem_optin, di.smem_per_sm / VP_MINB - 1024) - 2048) / 8 & ~1LL;
  std::vector<VDesc> cls[NCLS];
  std::vector<double> cost[NCLS];
  double total_flops = 0.0;
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
    const long long mi = even(max_intermediate(d, m, n, fwd));
    const double fl  = std::min(flops_forward(d, m, n), flops_backward(d, m, n));
    total_flops += fl;
    long long asz = 0;
    for (int l = 0; l < d; l++)
      asz += (long long)m[l] * n[l];
    const long long need = 2 * mi + even(asz);
    int c;
    if (mi <= WARP_MAX && 2 * WARP_MAX + even(asz) <= (budget / VP_WARPS & ~1LL))
      c = CLS_WARP;
    else if (need <= (budget / 4 & ~1LL))
      c = CLS_QUAD;
    else if (need <= (budget / 2 & ~1LL))
      c = CLS_HALF;
    else if (need <= budget)
      c = CLS_BLOCK;
    else
    {
      c = CLS_HUGE;
      HugeSplit hs;
      if (!plan_huge(d, m, n, budget, hs))
        return KRON_ERROR_NOT_SUPPORTED;
      e.q    = (unsigned char)hs.q;
      e.C    = (unsigned char)hs.C;
      e.fwd1 = (unsigned char)hs.fwd1;
      e.fwd2 = (unsigned char)hs.fwd2;
      long long Nhead = 1;
      for (int l = 0; l < hs.q; l++)
        Nhead *= n[l];
      // chunks of equal size, at most R rows each
      const long long nchunk = (Nhead + hs.R - 1) / hs.R;
      const long long R      = (Nhead + nchunk - 1) / nchunk;
      e.R      = (unsigned short)R;
      e.nchunk = (int)nchunk;
      e.mi     = (int)even(R * hs.mi1);
      e.mi2    = (int)even(hs.C * hs.mi2);
    }
    if (c != CLS_HUGE)
      e.mi = (c == CLS_WARP) ? WARP_MAX : (int)mi;
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

  // The huge queue: entries largest first; an entry's tile items enter the
  // queue once `lag_items` items or `lag_elems` elements of live regions
  // separate them from its chunk items (whichever comes first), so a tile
  // item rarely waits and its region is still in L2.  Regions start on
  // 128-byte boundaries.
  std::vector<VItem> items;
  const long long lag_items = 2LL * di.sms * VP_MINB;
  const long long lag_elems = 40LL << 17; // 40 MB of regions
  struct Pending
  {
    int e;
    size_t pos;
    long long elems;
  };
  std::vector<Pending> pend;
  size_t pend_head   = 0;
  long long live     = 0;
  long long woff     = 0;
  auto emit_tiles = [&](const Pending &p) {
    const VDesc &e = all[p.e];
    long long Mtail = 1;
    for (int l = e.q; l < e.d; l++)
      Mtail *= e.m[l];
    const long long nt = (Mtail + e.C - 1) / e.C;
    for (long long t = 0; t < nt; t++)
      items.push_back(VItem{p.e, (int)t, (int)t + 1, 1});
    live -= p.elems;
  };
  for (int i = 0; i < pl->nhuge; i++)
  {
    VDesc &e = all[i];
    e.woff   = woff;
    long long Nhead = 1, Mtail = 1;
    for (int l = 0; l < e.q; l++)
      Nhead *= e.n[l];
    for (int l = e.q; l < e.d; l++)
      Mtail *= e.m[l];
    const long long region = (Nhead * Mtail + 15) & ~15LL;
    woff += region;
    for (long long h0 = 0; h0 < Nhead; h0 += e.R)
      items.push_back(VItem{i, (int)h0, (int)std::min<long long>(Nhead, h0 + e.R), 0});
    pend.push_back(Pending{i, items.size(), region});
    live += region;
    while (pend_head < pend.size() &&
           ((long long)(items.size() - pend[pend_head].pos) >= lag_items || live > lag_elems))
      emit_tiles(pend[pend_head++]);
  }
  while (pend_head < pend.size())
    emit_tiles(pend[pend_head++]);

  pl->nitems     = (int)items.size();
  pl->flops      = total_flops;
  pl->budget     = (int)budget;
  pl->ws_bytes   = (size_t)woff * 8;
  pl->grid_work  = (int)std::min<long long>(
      1LL << 30, (long long)items.size() + pl->nblock + (pl->nhalf + 1) / 2 +
                     (pl->nquad + 3) / 4 + (pl->nwarp + VP_WARPS - 1) / VP_WARPS);
  pl->exec       = nullptr;
  pl->d_desc     = nullptr;
  pl->d_items    = nullptr;
  pl->d_counters = nullptr;
  const size_t ncount = NCOUNT + (size_t)pl->nhuge;
  if (kron::dev_malloc((void **)&pl->d_counters, ncount * sizeof(int)) != cudaSuccess ||
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
  if (cudaMemsetAsync(pl->d_counters, 0, (NCOUNT + (size_t)pl->nhuge) * sizeof(int), s) !=
      cudaSuccess)
    return KRON_ERROR_LAUNCH;
  if (pl->grid_work <= 0)
    return KRON_SUCCESS;
  VParams vp;
  std::memset(&vp, 0, sizeof(vp));
  vp.desc     = pl->d_desc;
  vp.items    = pl->d_items;
  vp.nhuge    = pl->nhuge;
  vp.nblock   = pl->nblock;
  vp.nhalf    = pl->nhalf;
  vp.nquad    = pl->nquad;
  vp.nwarp    = pl->nwarp;
  vp.nitems   = pl->nitems;
  vp.counters = pl->d_counters;
  vp.status   = device_status_ptr();
  vp.spin     = wait_limit();
  vp.pA       = A;
  vp.pX       = X;
  vp.pY       = Y;
  vp.ws       = static_cast<double *>(W);
  vp.budget   = pl->budget;
  void *args[]      = {&vp};
  const void *fm    = reinterpret_cast<const void *>(&kron_vplan_kernel);
  const size_t smem = (size_t)pl->budget * 8;
  int occ           = 1;
  if (cached_occupancy(fm, VP_THREADS, smem, &occ) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  // persistent: every block stays resident until the queues run dry
  const int grid =
      (int)std::max<long long>(1, std::min<long long>((long long)device_info().sms * occ,
                                                      pl->grid_work));
  if (cudaLaunchKernel(fm, dim3(grid), dim3(VP_THREADS), args, smem, s) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
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

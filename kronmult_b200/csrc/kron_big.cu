// Vectors too large for one block's shared memory (d = 5..6 with n = 6..8:
// 373 KB .. 2 MB per entry in FP64): one thread-block cluster per entry.
//
// The d modes split into a head [0, Q) and a tail [Q, d) with
// LH = n^Q head rows and LT = n^(d-Q) tail columns, x = X[h][t] (t fastest).
//   phase 1: every head row h (a contiguous LT block of x) gets the tail
//            modes; a warp per block (for n = 8 in FP64 the 512-element
//            FP64 tensor-core routine of kron_mma8_core.cuh), result -> W;
//   barrier.cluster (hardware, no spinning) -- W is complete;
//   phase 2: every column tile (LH rows x C columns of W, C contiguous
//            doubles per row), fetched by cp.async one tile ahead, gets the
//            head modes in shared memory and is added into y with
//            red.global.add (one rounding, as y += r; no load round trip).
// This is the recursive algorithm's two-level split (kronmultv_recur.hpp:
// 117-145 applies A_1 on X viewed as (n2..nd) x n1, then recurses), with
// the intermediate W kept L2-resident: only one entry per cluster is in
// flight, so the live W is (#clusters x n^d) elements, and W is written with
// an evict-last L2 policy while x, y and W's read-back take evict-first, so
// the streaming operands do not push W out to HBM before phase 2 reads it.  The next entry's x
// and this entry's y are prefetched into L2 while the cluster computes.
#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <type_traits>

#include "kron_launch.h"
#include "kron_mma8_core.cuh"
#include "kronmult.h"

namespace kron {

namespace {

constexpr int BIG_THREADS = 256;
constexpr int BIG_WARPS   = BIG_THREADS / 32;

__device__ __forceinline__ void cluster_sync_all()
{
  asm volatile("barrier.cluster.arrive.release.aligned;\n\t"
               "barrier.cluster.wait.acquire.aligned;" ::
                   : "memory");
}

__device__ __forceinline__ unsigned cluster_rank()
{
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ unsigned cluster_size()
{
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

__device__ __forceinline__ void prefetch_l2(const void *p, long long bytes)
{
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  const uintptr_t b = (a + 15) & ~uintptr_t(15);
  const long long n = (bytes - (long long)(b - a)) & ~15LL;
  if (n >= 16)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b), "r"((unsigned)n)
                 : "memory");
}

// Workspace slot for cluster cid working on entry k at position e of the
// launch range [ebase, eend).
struct BigWS
{
  void *base;
  long long stride;     // elements between slots (base form)
  void *const *ptrs;    // pointer form
  int per_entry;        // 1: a slot per entry; 0: a slot per cluster
  int l2_hints;         // 1: W written evict-last, x and y streamed evict-first
};

// L2 cache policies.  The intermediate W of the clusters in flight (tens of
// MB) fits the 126 MB L2, but x and y stream past it at several TB/s and
// would push it out before phase 2 reads it back; W's stores carry
// evict-last, the streaming x loads, W's read-back and y's adds evict-first.
// Without hints both policies are evict-normal.
struct L2Pol
{
  uint64_t keep, stream;
};

__device__ __forceinline__ L2Pol make_policies(bool hints)
{
  L2Pol p;
  if (hints)
  {
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p.keep));
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p.stream));
  }
  else
  {
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p.keep));
    p.stream = p.keep;
  }
  return p;
}

template <typename T>
__device__ __forceinline__ void st_pol(T *p, T v, uint64_t pol)
{
  if constexpr (sizeof(T) == 8)
    asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol)
                 : "memory");
  else
    asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
                 : "memory");
}

// 16 bytes from shared-memory-resident registers to global
template <typename T>
__device__ __forceinline__ void st16_pol(T *p, const T *v, uint64_t pol)
{
  if constexpr (sizeof(T) == 8)
    asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(v[0]),
                 "d"(v[1]), "l"(pol)
                 : "memory");
  else
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
                 "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "l"(pol)
                 : "memory");
}

__device__ __forceinline__ double2 ld16_pol(const double *p, uint64_t pol)
{
  double2 r;
  asm volatile("ld.global.nc.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
               : "=d"(r.x), "=d"(r.y)
               : "l"(p), "l"(pol));
  return r;
}

__device__ __forceinline__ double ld_pol(const double *p, uint64_t pol)
{
  double r;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(r) : "l"(p), "l"(pol));
  return r;
}

template <typename T>
__device__ __forceinline__ void red_pol(T *p, T v, uint64_t pol)
{
  if constexpr (sizeof(T) == 8)
    asm volatile("red.global.add.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(p), "d"(v), "l"(pol)
                 : "memory");
  else
    asm volatile("red.global.add.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(p), "f"(v), "l"(pol)
                 : "memory");
}

template <typename T>
__device__ __forceinline__ T *big_slot(const BigWS &ws, int k, int e, int ebase, int cid)
{
  if (!ws.per_entry)
    return ws.ptrs ? static_cast<T *>(ws.ptrs[cid])
                   : static_cast<T *>(ws.base) + (long long)cid * ws.stride;
  // pointer form: the caller's W pointer of entry k; base form: slot
  // (e - ebase) of a buffer that covers exactly this launch's range
  return ws.ptrs ? static_cast<T *>(ws.ptrs[k])
                 : static_cast<T *>(ws.base) + (long long)(e - ebase) * ws.stride;
}

// TC: FP64 n = 8 runs its 8x8 mode products on the tensor cores (mma.sync
// f64); TC = false keeps every shape on CUDA-core FMAs (a comparison form)
template <typename T, int D, int N, int Q, int C, bool TC = true>
struct BigShape
{
  static constexpr int LH   = cpow(N, Q);
  static constexpr int LT   = cpow(N, D - Q);
  static constexpr int L    = LH * LT;
  static constexpr int ASZ  = (D * N * N + 15) / 16 * 16;
  static constexpr bool MMA = TC && (sizeof(T) == 8) && (N == 8) && (D - Q == 3);
  // phase 1 without tensor cores: rounds of NB head rows share the block's
  // threads (LT/N fibres per row and mode)
  static constexpr int FPB  = LT / N;
  static constexpr int NB   = (BIG_THREADS / FPB) > 0 ? (BIG_THREADS / FPB) : 1;
  static constexpr int RBUF = ((MMA ? 512 * BIG_WARPS : NB * LT) + 15) / 16 * 16;
  // phase 2 on FP64 tensor cores when the head is three 8x8 modes: tiles are
  // kept transposed, column c at c * PITCH (16-byte aligned columns)
  static constexpr bool MMA2 = TC && (sizeof(T) == 8) && (N == 8) && (Q == 3);
  static constexpr int PITCH = 514;
  static constexpr int TBUF  = ((MMA2 ? C * PITCH : LH * C) + 15) / 16 * 16;
  static constexpr size_t OFF_A    = 0;
  static constexpr size_t OFF_R    = OFF_A + (size_t)ASZ * sizeof(T);           // 2 round buffers
  // the tensor-core phase 1 uses one round buffer, the others two; phase 2
  // double-buffers its tiles
  static constexpr size_t OFF_TILE = OFF_R + (MMA ? 1 : 2) * (size_t)RBUF * sizeof(T);
  static constexpr size_t SMEM     = OFF_TILE + 2 * (size_t)TBUF * sizeof(T);
};

template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(src) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_elem_pol(T *dst, const T *src, uint64_t pol)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 8, %2;" ::"r"(s),
                 "l"(src), "l"(pol)
                 : "memory");
  else
    asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], 4, %2;" ::"r"(s),
                 "l"(src), "l"(pol)
                 : "memory");
}
__device__ __forceinline__ void cp_async16_pol(void *dst, const void *src, uint64_t pol)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;" ::"r"(s),
               "l"(src), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ bool al16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }
template <int Nleft>
__device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(Nleft) : "memory"); }

// One mode pass (mode stride S, N-element fibres) over `nblk` consecutive
// buffers of `blen` elements, fibres spread over the block's threads;
// A_m (N x N, column major in shared memory) in registers.
template <typename T, int N, int S, int FPB>
__device__ __forceinline__ void cta_mode_pass(T *buf, int blen, int nfib, const T *Am, int tid)
{
  T a[N][N];
#pragma unroll
  for (int i = 0; i < N; i++)
#pragma unroll
    for (int j = 0; j < N; j++)
      a[i][j] = Am[i + j * N];
  for (int f = tid; f < nfib; f += BIG_THREADS)
  {
    const int bi = f / FPB, ff = f - (f / FPB) * FPB;
    const int o = ff / S, r = ff - (ff / S) * S;
    T *b = buf + bi * blen + o * N * S + r;
    T x[N];
#pragma unroll
    for (int j = 0; j < N; j++)
      x[j] = b[j * S];
#pragma unroll
    for (int i = 0; i < N; i++)
    {
      T z = T(0);
#pragma unroll
      for (int j = 0; j < N; j++)
        z = fma(a[i][j], x[j], z);
      b[i * S] = z;
    }
  }
}

// tail modes m = Q..D-1 on the round buffer (compile-time strides)
template <typename T, int D, int N, int Q, int m>
__device__ __forceinline__ void round_tail_passes(T *buf, int nrows, const T *As, int tid)
{
  if constexpr (m < D)
  {
    constexpr int LT  = cpow(N, D - Q);
    constexpr int S   = cpow(N, D - 1 - m);
    constexpr int FPB = LT / N;
    cta_mode_pass<T, N, S, FPB>(buf, LT, nrows * FPB, As + m * N * N, tid);
    __syncthreads();
    round_tail_passes<T, D, N, Q, m + 1>(buf, nrows, As, tid);
  }
}

// head modes m = 0..Q-1 on a tile (LH rows x C columns, column fastest)
template <typename T, int N, int Q, int C, int m>
__device__ __forceinline__ void tile_head_passes(T *tile, const T *As, int tid)
{
  if constexpr (m < Q)
  {
    constexpr int LH  = cpow(N, Q);
    constexpr int SR  = cpow(N, Q - 1 - m) * C; // element stride of mode m
    constexpr int FPB = LH * C / N;
    cta_mode_pass<T, N, SR, FPB>(tile, 0, FPB, As + m * N * N, tid);
    __syncthreads();
    tile_head_passes<T, N, Q, C, m + 1>(tile, As, tid);
  }
}

template <typename T, int D, int N, int Q, int C, int MINB, bool TC>
__global__ void __launch_bounds__(BIG_THREADS, MINB)
    kron_big_kernel(const __grid_constant__ Params p, const __grid_constant__ BigWS ws)
{
  using S            = BigShape<T, D, N, Q, C, TC>;
  constexpr int LH   = S::LH;
  constexpr int LT   = S::LT;
  constexpr int L    = S::L;
  extern __shared__ __align__(128) unsigned char smem[];
  T *As    = reinterpret_cast<T *>(smem + S::OFF_A);
  T *rbuf0 = reinterpret_cast<T *>(smem + S::OFF_R);
  T *tbuf0 = reinterpret_cast<T *>(smem + S::OFF_TILE);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const L2Pol pol = make_policies(ws.l2_hints != 0);

  const int cs   = (int)cluster_size();
  const int rank = (int)cluster_rank();
  const int cid  = blockIdx.x / cs;
  const int ncl  = gridDim.x / cs;
  const long long tot = p.eend - p.ebase;
  const int eb = p.ebase + (int)(tot * cid / ncl);
  const int ee = p.ebase + (int)(tot * (cid + 1) / ncl);
  if (eb >= ee)
    return; // the whole cluster leaves together

  const int hb = (int)((long long)LH * rank / cs), he = (int)((long long)LH * (rank + 1) / cs);
  constexpr int NT = (LT + C - 1) / C;
  const int tb = (int)((long long)NT * rank / cs), te = (int)((long long)NT * (rank + 1) / cs);

  for (int e = eb; e < ee; ++e)
  {
    const int k = entry_index(p, e);
    EntryRef<T> en;
    entry_fetch<T>(p, k, D, en);
    T *w = big_slot<T>(ws, k, e, p.ebase, cid);

    if (tid == 0)
    {
      const long long share = (long long)L * sizeof(T) / cs;
      prefetch_l2(reinterpret_cast<const char *>(en.y) + share * rank, share);
      if (e + 1 < ee)
      {
        EntryRef<T> nx;
        entry_fetch<T>(p, entry_index(p, e + 1), D, nx);
        prefetch_l2(reinterpret_cast<const char *>(nx.x) + share * rank, share);
      }
    }
    for (int q = tid; q < D * N * N; q += BIG_THREADS)
    {
      const int l = q / (N * N), ij = q - l * (N * N);
      const int j = ij / N, i = ij - j * N;
      As[q]       = __ldg(en.A[l] + i + (long long)j * en.ld[l]);
    }
    __syncthreads();

    // ---------------- phase 1: tail modes on head rows [hb, he)
    if constexpr (S::MMA)
    {
      const int g = lane >> 2, t = lane & 3;
      double *blk = reinterpret_cast<double *>(rbuf0) + warp * 512;
      AFrag8 f;
      load_afrag8(f, reinterpret_cast<const double *>(en.A[Q]), en.ld[Q],
                  reinterpret_cast<const double *>(en.A[Q + 1]), en.ld[Q + 1],
                  reinterpret_cast<const double *>(en.A[Q + 2]), en.ld[Q + 2], g, t);
      const bool al16 = ((reinterpret_cast<uintptr_t>(en.x) & 15) == 0);
      // this lane's 16 elements of head row h (the next row is loaded while
      // the current one is on the tensor cores)
      auto load_row = [&](int h, double (&v)[8][2]) {
        const double *xb = reinterpret_cast<const double *>(en.x) + (long long)h * LT;
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
          const double *src = xb + q * 64 + g * 8 + 2 * t;
          if (al16)
          {
            const double2 u = ld16_pol(src, pol.stream);
            v[q][0]         = u.x;
            v[q][1]         = u.y;
          }
          else
          {
            v[q][0] = ld_pol(src, pol.stream);
            v[q][1] = ld_pol(src + 1, pol.stream);
          }
        }
      };
      double vn[8][2];
      if (hb + warp < he)
        load_row(hb + warp, vn);
      for (int h = hb + warp; h < he; h += BIG_WARPS)
      {
        double v[8][2], acc[8][2];
#pragma unroll
        for (int q = 0; q < 8; q++)
        {
          v[q][0] = vn[q][0];
          v[q][1] = vn[q][1];
          acc[q][0] = acc[q][1] = 0.0;
        }
        if (h + BIG_WARPS < he)
          load_row(h + BIG_WARPS, vn);
        kron8x3_tile(v, acc, f, blk, g, t);
        double *wb = reinterpret_cast<double *>(w) + (long long)h * LT;
#pragma unroll
        for (int q = 0; q < 8; q++)
#pragma unroll
          for (int pp = 0; pp < 2; pp++)
            st_pol(wb + (2 * t + pp) * 64 + q * 8 + g, acc[q][pp], pol.keep);
      }
    }
    else
    {
      // rounds of NB consecutive head rows, loads double buffered (cp.async)
      constexpr int NB = S::NB;
      constexpr int V = 16 / sizeof(T); // elements per 16-byte copy
      auto issue_round = [&](int h0, T *buf) {
        const int nr  = min(NB, he - h0);
        const T *src = en.x + (long long)h0 * LT;
        if ((LT * sizeof(T)) % 16 == 0 && al16(src))
          for (int q = tid; q < nr * LT / V; q += BIG_THREADS)
            cp_async16_pol(buf + q * V, src + q * V, pol.stream);
        else
          for (int q = tid; q < nr * LT; q += BIG_THREADS)
            cp_async_elem_pol(buf + q, src + q, pol.stream);
        cp_commit();
      };
      int cur = 0;
      if (hb < he)
        issue_round(hb, rbuf0);
      for (int h0 = hb; h0 < he; h0 += NB)
      {
        T *buf = rbuf0 + cur * S::RBUF;
        if (h0 + NB < he)
        {
          issue_round(h0 + NB, rbuf0 + (cur ^ 1) * S::RBUF);
          cp_wait<1>();
        }
        else
          cp_wait<0>();
        __syncthreads();
        const int nr = min(NB, he - h0);
        round_tail_passes<T, D, N, Q, Q>(buf, nr, As, tid);
        T *dst = w + (long long)h0 * LT;
        if ((LT * sizeof(T)) % 16 == 0 && al16(dst))
        {
          for (int q = tid; q < nr * LT / V; q += BIG_THREADS)
            st16_pol(dst + q * V, buf + q * V, pol.keep);
        }
        else
          for (int q = tid; q < nr * LT; q += BIG_THREADS)
            st_pol(dst + q, buf[q], pol.keep);
        __syncthreads();
        cur ^= 1;
      }
    }
    __threadfence();
    __syncthreads();
    cluster_sync_all(); // W of this entry is complete

    // ---------------- phase 2: head modes on column tiles [tb, te)
    if constexpr (S::MMA2)
    {
      constexpr int PITCH = S::PITCH;
      const int g = lane >> 2, t = lane & 3;
      double *tiles = reinterpret_cast<double *>(tbuf0);
      double *xs   = reinterpret_cast<double *>(rbuf0) + warp * 512; // transpose scratch
      AFrag8 f;
      load_afrag8(f, reinterpret_cast<const double *>(en.A[0]), en.ld[0],
                  reinterpret_cast<const double *>(en.A[1]), en.ld[1],
                  reinterpret_cast<const double *>(en.A[2]), en.ld[2], g, t);
      const double *wd = reinterpret_cast<const double *>(w);
      double *yd       = reinterpret_cast<double *>(en.y);
      // W rows -> transposed tile (column c contiguous) by cp.async, one
      // tile ahead of the one being computed
      auto issue_gather = [&](int tt, double *tile) {
        const int c0 = tt * C, cc = min(C, LT - c0);
        for (int q = tid; q < LH * C; q += BIG_THREADS)
        {
          const int h = q / C, c = q - (q / C) * C;
          if (c < cc)
            cp_async_elem_pol(tile + c * PITCH + h, wd + (long long)h * LT + c0 + c, pol.stream);
          else
            tile[c * PITCH + h] = 0.0;
        }
        cp_commit();
      };
      int cur = 0;
      if (tb < te)
        issue_gather(tb, tiles);
      for (int tt = tb; tt < te; ++tt)
      {
        const int c0 = tt * C, cc = min(C, LT - c0);
        double *tile = tiles + cur * S::TBUF;
        if (tt + 1 < te)
        {
          issue_gather(tt + 1, tiles + (cur ^ 1) * S::TBUF);
          cp_wait<1>();
        }
        else
          cp_wait<0>();
        __syncthreads();
        // each warp: kron(A_1, A_2, A_3) on whole columns
        for (int c = warp; c < cc; c += BIG_WARPS)
        {
          double *col = tile + c * PITCH;
          double v[8][2], acc[8][2];
#pragma unroll
          for (int q = 0; q < 8; q++)
          {
            const double2 u = *reinterpret_cast<const double2 *>(col + q * 64 + g * 8 + 2 * t);
            v[q][0]   = u.x;
            v[q][1]   = u.y;
            acc[q][0] = acc[q][1] = 0.0;
          }
          kron8x3_tile(v, acc, f, xs, g, t);
          __syncwarp();
          // result element (i0 = 2t+p, i1 = q, i2 = g) stored at i1*64 + i2*8 + i0
#pragma unroll
          for (int q = 0; q < 8; q++)
            *reinterpret_cast<double2 *>(col + q * 64 + g * 8 + 2 * t) =
                make_double2(acc[q][0], acc[q][1]);
        }
        __syncthreads();
        // tile rows into y by red.global.add (fire and forget; each output
        // element has one writer in this launch unless outputs alias)
        for (int q = tid; q < LH * C; q += BIG_THREADS)
        {
          const int i = q / C, c = q - (q / C) * C;
          if (c < cc)
          {
            const int pos = ((i >> 3) & 7) * 64 + (i & 7) * 8 + (i >> 6);
            red_pol(yd + (long long)i * LT + c0 + c, tile[c * PITCH + pos], pol.stream);
          }
        }
        __syncthreads();
        cur ^= 1;
      }
    }
    else
    {
      constexpr int V = 16 / sizeof(T); // elements per 16-byte copy
      // W rows are 16-byte aligned when the slot is and rows are whole
      // 16-byte multiples (tile starts c0 are multiples of C)
      const bool wvec = (LT * sizeof(T)) % 16 == 0 && (C % V) == 0 && al16(w);
      auto issue_tile = [&](int tt, T *buf) {
        const int c0 = tt * C, cc = min(C, LT - c0);
        if (wvec)
          for (int q = tid; q < LH * C / V; q += BIG_THREADS)
          {
            const int h = (q * V) / C, c = q * V - h * C;
            if (c + V <= cc)
              cp_async16_pol(buf + q * V, w + (long long)h * LT + c0 + c, pol.stream);
            else
#pragma unroll
              for (int u = 0; u < V; u++)
              {
                if (c + u < cc)
                  cp_async_elem_pol(buf + q * V + u, w + (long long)h * LT + c0 + c + u,
                                    pol.stream);
                else
                  buf[q * V + u] = T(0);
              }
          }
        else
          for (int q = tid; q < LH * C; q += BIG_THREADS)
          {
            const int h = q / C, c = q - (q / C) * C;
            if (c < cc)
              cp_async_elem_pol(buf + q, w + (long long)h * LT + c0 + c, pol.stream);
            else
              buf[q] = T(0);
          }
        cp_commit();
      };
      int cur = 0;
      if (tb < te)
        issue_tile(tb, tbuf0);
      for (int tt = tb; tt < te; ++tt)
      {
        T *tile = tbuf0 + cur * S::TBUF;
        if (tt + 1 < te)
        {
          issue_tile(tt + 1, tbuf0 + (cur ^ 1) * S::TBUF);
          cp_wait<1>();
        }
        else
          cp_wait<0>();
        __syncthreads();
        tile_head_passes<T, N, Q, C, 0>(tile, As, tid);
        const int c0 = tt * C, cc = min(C, LT - c0);
        // tile rows into y by red.global.add (fire and forget)
        for (int q = tid; q < LH * C; q += BIG_THREADS)
        {
          const int i = q / C, c = q - (q / C) * C;
          if (c < cc)
            red_pol(en.y + (long long)i * LT + c0 + c, tile[q], pol.stream);
        }
        __syncthreads();
        cur ^= 1;
      }
    }
    cluster_sync_all(); // every block is done with this entry's W
  }
}

// ---------------------------------------------------------------------------
// W in the cluster's shared memory.  When the whole intermediate of one entry
// fits in the shared memory of a CS-block cluster (FP64 d = 6, n = 6: 373 KB
// over two blocks), block r owns the W columns [r LT/CS, (r+1) LT/CS) as an
// LH x NCOL array in its own shared memory:
//   phase 1: head rows [hb, he) of x get the tail modes (cp.async rounds, as
//            above); every result pair goes straight to the block that owns
//            its column (st.shared::cluster through mapa);
//   barrier.cluster -- every block holds its complete W columns;
//   phase 2: the head modes in place on the local LH x NCOL array, then one
//            TMA bulk reduce-add per row segment (NCOL contiguous elements of
//            y) -- or red.global.add when y is not 16-byte aligned;
//   barrier.cluster -- the bulk reads are done before the next entry's
//            phase 1 writes into any block's W.
// No workspace and no W traffic through L2 / HBM: x is read once, y read and
// written once.
template <typename T, int D, int N, int Q, int CS>
struct DsmShape
{
  static constexpr int LH   = cpow(N, Q);
  static constexpr int LT   = cpow(N, D - Q);
  static constexpr int L    = LH * LT;
  static_assert(LT % CS == 0, "W columns split evenly over the cluster");
  static constexpr int NCOL = LT / CS;
  static constexpr int V    = 16 / sizeof(T); // elements per 16-byte store
  static_assert(NCOL % V == 0 && LT % V == 0, "16-byte stores stay inside one block's columns");
  static constexpr int ASZ  = (D * N * N + 15) / 16 * 16;
  static constexpr int FPB  = LT / N;
  static constexpr int NB   = (BIG_THREADS / FPB) > 0 ? (BIG_THREADS / FPB) : 1;
  static constexpr int RBUF = (NB * LT + 15) / 16 * 16;
  static constexpr size_t OFF_A = 0;
  static constexpr size_t OFF_R = OFF_A + (size_t)ASZ * sizeof(T);
  static constexpr int NS       = 3; // round buffers: two rounds load ahead
  static constexpr size_t OFF_W = OFF_R + NS * (size_t)RBUF * sizeof(T);
  static constexpr size_t SMEM  = OFF_W + (size_t)LH * NCOL * sizeof(T);
};

__device__ __forceinline__ unsigned mapa_rank(unsigned saddr, unsigned rank)
{
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}

template <typename T>
__device__ __forceinline__ void st_cluster16(unsigned addr, const T *v)
{
  if constexpr (sizeof(T) == 8)
    asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(addr), "d"(v[0]), "d"(v[1])
                 : "memory");
  else
    asm volatile("st.shared::cluster.v4.f32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v[0]),
                 "f"(v[1]), "f"(v[2]), "f"(v[3])
                 : "memory");
}

template <typename T>
__device__ __forceinline__ void bulk_reduce_row(T *y, const T *src, unsigned bytes)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(src);
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(y),
                 "r"(s), "r"(bytes)
                 : "memory");
  else
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(y),
                 "r"(s), "r"(bytes)
                 : "memory");
}

template <typename T, int D, int N, int Q, int CS>
__global__ void __launch_bounds__(BIG_THREADS, 1)
    kron_bigdsm_kernel(const __grid_constant__ Params p)
{
  using S          = DsmShape<T, D, N, Q, CS>;
  constexpr int LH = S::LH, LT = S::LT, L = S::L, NCOL = S::NCOL, V = S::V;
  extern __shared__ __align__(128) unsigned char smem[];
  T *As    = reinterpret_cast<T *>(smem + S::OFF_A);
  T *rbuf0 = reinterpret_cast<T *>(smem + S::OFF_R);
  T *wloc  = reinterpret_cast<T *>(smem + S::OFF_W);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const int rank = (int)cluster_rank();
  const int cid  = blockIdx.x / CS;
  const int ncl  = gridDim.x / CS;
  const long long tot = p.eend - p.ebase;
  const int eb = p.ebase + (int)(tot * cid / ncl);
  const int ee = p.ebase + (int)(tot * (cid + 1) / ncl);
  if (eb >= ee)
    return; // the whole cluster leaves together
  // every block of the cluster has started before any shared::cluster store
  cluster_sync_all();

  const unsigned wl = (unsigned)__cvta_generic_to_shared(wloc);
  unsigned wr[CS];
#pragma unroll
  for (int r = 0; r < CS; r++)
    wr[r] = mapa_rank(wl, (unsigned)r);
  const int hb = LH * rank / CS, he = LH * (rank + 1) / CS;
  const int t0 = NCOL * rank;
  constexpr int NB = S::NB, NS = S::NS;
  const int nround = (he - hb + NB - 1) / NB;
  // copies of round r (head rows hb + r NB ..) of the entry whose x is `x`
  // into buffer r mod NS: one cp.async group per call, empty past the last
  // round, so a wait for "all but the newest two groups" always covers the
  // round about to be computed
  auto issue_round = [&](const T *x, int r) {
    if (r < nround)
    {
      const int h0  = hb + r * NB;
      const int nr  = min(NB, he - h0);
      T *buf        = rbuf0 + (r % NS) * S::RBUF;
      const T *src  = x + (long long)h0 * LT;
      if ((LT * sizeof(T)) % 16 == 0 && al16(src))
        for (int q = tid; q < nr * LT / V; q += BIG_THREADS)
          cp_async16(buf + q * V, src + q * V);
      else
        for (int q = tid; q < nr * LT; q += BIG_THREADS)
          cp_async_elem(buf + q, src + q);
    }
    cp_commit();
  };
  {
    EntryRef<T> e0;
    entry_fetch<T>(p, entry_index(p, eb), D, e0);
    issue_round(e0.x, 0);
    issue_round(e0.x, 1);
  }

  for (int e = eb; e < ee; ++e)
  {
    const int k = entry_index(p, e);
    EntryRef<T> en;
    entry_fetch<T>(p, k, D, en);
    if (tid == 0)
    {
      const long long share = (long long)L * sizeof(T) / CS;
      prefetch_l2(reinterpret_cast<const char *>(en.y) + share * rank, share);
      if (e + 1 < ee)
      {
        EntryRef<T> nx;
        entry_fetch<T>(p, entry_index(p, e + 1), D, nx);
        prefetch_l2(reinterpret_cast<const char *>(nx.x) + share * rank, share);
      }
    }
    for (int q = tid; q < D * N * N; q += BIG_THREADS)
    {
      const int l = q / (N * N), ij = q - l * (N * N);
      const int j = ij / N, i = ij - j * N;
      As[q]       = __ldg(en.A[l] + i + (long long)j * en.ld[l]);
    }
    __syncthreads();

    // ---------------- phase 1: tail modes on head rows [hb, he) -> owners' W
    // (rounds r and r+1 are in flight when round r starts; r+2 goes into
    // the buffer round r-1 used)
    for (int r = 0; r < nround; ++r)
    {
      issue_round(en.x, r + 2);
      cp_wait<2>();
      __syncthreads();
      const int h0 = hb + r * NB;
      const int nr = min(NB, he - h0);
      T *buf       = rbuf0 + (r % NS) * S::RBUF;
      round_tail_passes<T, D, N, Q, Q>(buf, nr, As, tid);
      // element (row, t) -> block t / NCOL, offset ((h0+row) NCOL + t mod NCOL)
      for (int q = tid; q < nr * LT / V; q += BIG_THREADS)
      {
        const int row = (q * V) / LT, t = q * V - row * LT;
        const int owner = t / NCOL, c = t - owner * NCOL;
        const unsigned off = (unsigned)(((h0 + row) * NCOL + c) * (int)sizeof(T));
        st_cluster16<T>(wr[owner] + off, buf + q * V);
      }
      __syncthreads();
    }
    cluster_sync_all(); // every block holds its complete W columns
    // the next entry's first two rounds load during phase 2
    if (e + 1 < ee)
    {
      EntryRef<T> nx;
      entry_fetch<T>(p, entry_index(p, e + 1), D, nx);
      issue_round(nx.x, 0);
      issue_round(nx.x, 1);
    }

    // ---------------- phase 2: head modes in place on the local columns
    tile_head_passes<T, N, Q, NCOL, 0>(wloc, As, tid);
    T *yb = en.y + t0;
    const bool bulk = al16(yb) && (LT * sizeof(T)) % 16 == 0;
    if (bulk)
    {
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (warp == 0)
      {
        for (int h = lane; h < LH; h += 32)
          bulk_reduce_row<T>(yb + (long long)h * LT, wloc + h * NCOL,
                             (unsigned)(NCOL * sizeof(T)));
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
      }
    }
    else
      for (int q = tid; q < LH * NCOL; q += BIG_THREADS)
      {
        const int h = q / NCOL, c = q - h * NCOL;
        red_add(yb + (long long)h * LT + c, wloc[q]);
      }
    __syncthreads();
    cluster_sync_all(); // W reads done before the next entry's phase 1
  }
  if (warp == 0)
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

template <typename T, int D, int N, int Q, int CS>
int launch_bigdsm_t(Params p, cudaStream_t stream)
{
  using S        = DsmShape<T, D, N, Q, CS>;
  const void *fn = reinterpret_cast<const void *>(&kron_bigdsm_kernel<T, D, N, Q, CS>);
  if (S::SMEM > (size_t)device_info().max_smem_optin)
    return KRON_ERROR_NOT_SUPPORTED;
  int dummy = 1;
  if (cached_occupancy(fn, BIG_THREADS, S::SMEM, &dummy) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id               = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim             = dim3(BIG_THREADS);
  cfg.dynamicSmemBytes     = S::SMEM;
  cfg.stream               = stream;
  cfg.attrs                = attr;
  cfg.numAttrs             = 1;
  cfg.gridDim              = dim3((device_info().sms / CS) * CS);
  int ncl                  = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg) != cudaSuccess || ncl < 1)
    return KRON_ERROR_NOT_SUPPORTED;
  ncl         = (int)std::min<long long>((long long)ncl, p.eend - p.ebase);
  cfg.gridDim = dim3(ncl * CS);
  void *args[] = {&p};
  return cudaLaunchKernelExC(&cfg, fn, args) == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

template <typename T, int D, int N, int Q, int C, int MINB, bool TC = true>
int launch_big_t(Params p, const Workspace &wsp, int prec, int cluster, cudaStream_t stream)
{
  using S        = BigShape<T, D, N, Q, C, TC>;
  const void *fn = reinterpret_cast<const void *>(&kron_big_kernel<T, D, N, Q, C, MINB, TC>);
  if (S::SMEM > (size_t)device_info().max_smem_optin)
    return KRON_ERROR_NOT_SUPPORTED;
  int dummy = 1;
  if (cached_occupancy(fn, BIG_THREADS, S::SMEM, &dummy) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;

  // workspace slots: one per entry when the caller's W has them, else one
  // per cluster
  BigWS ws{};
  ws.l2_hints              = (cluster & KRON_BIG_NO_L2_HINTS) ? 0 : 1;
  long long nslots_cluster = 1LL << 30;
  if (p.layout == LAYOUT_BATCHED)
  {
    if (!wsp.W || wsp.wstride < S::L)
      return KRON_ERROR_WORKSPACE;
    ws.base      = wsp.W;
    ws.stride    = wsp.wstride;
    ws.per_entry = 1;
  }
  else if (wsp.pW)
  {
    if (wsp.pw_elems < S::L || wsp.npW < 1)
      return KRON_ERROR_WORKSPACE;
    ws.ptrs = wsp.pW;
    if (p.layout == LAYOUT_PBATCHED && wsp.npW >= p.batch)
      ws.per_entry = 1;
    else
      nslots_cluster = wsp.npW;
  }
  else
  {
    nslots_cluster = wsp.W ? (long long)(wsp.Wbytes / (sizeof(T) * (size_t)S::L)) : 0;
    if (nslots_cluster < 1)
      return KRON_ERROR_WORKSPACE;
    ws.base   = wsp.W;
    ws.stride = S::L;
  }

  const long long work = p.eend - p.ebase;
  int cs               = 2;
  cluster &= ~(KRON_BIG_CUDA_CORES | KRON_BIG_SMEM_W | KRON_BIG_NO_L2_HINTS);
  if (cluster > 0)
    cs = std::min(8, cluster);
  else if (const char *env = std::getenv("KRON_BIG_CLUSTER"))
    cs = std::max(1, std::min(8, std::atoi(env)));
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id               = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim             = dim3(BIG_THREADS);
  cfg.dynamicSmemBytes     = S::SMEM;
  cfg.stream               = stream;
  cfg.attrs                = attr;
  cfg.numAttrs             = 1;
  int ncl                  = 0;
  cfg.gridDim              = dim3((device_info().sms / cs) * cs);
  if (cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg) != cudaSuccess || ncl < 1)
    ncl = std::max(1, device_info().sms / cs);
  ncl         = (int)std::min<long long>({(long long)ncl, work, nslots_cluster});
  cfg.gridDim = dim3(ncl * cs);
  void *args[] = {&p, &ws};
  return cudaLaunchKernelExC(&cfg, fn, args) == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

} // namespace

bool big_supported(const Params &p, int prec)
{
  if (prec == PREC_SPLIT || p.accum == ACC_SEGMENTED || p.accum == ACC_STORE)
    return false;
  const int n = p.n[0];
  for (int l = 0; l < p.d; l++)
    if (p.m[l] != n || p.n[l] != n)
      return false;
  if (p.d == 6)
    return n >= 6 && n <= 8;
  if (p.d == 5)
    return n == 8;
  return false;
}

int launch_big(Params p, const Workspace &ws, int prec, int cluster, cudaStream_t stream)
{
  if (p.eend <= p.ebase)
    return KRON_SUCCESS;
  const int n = p.n[0];
  // (T, d, n, head modes, tile columns, blocks per SM)
  if (prec == PREC_F32)
  {
    if (p.d == 6 && n == 7)
      return launch_big_t<float, 6, 7, 3, 32, 2>(p, ws, prec, cluster, stream);
    if (p.d == 6 && n == 8)
      return launch_big_t<float, 6, 8, 3, 16, 2>(p, ws, prec, cluster, stream);
    return KRON_ERROR_NOT_SUPPORTED;
  }
  if (p.d == 6 && n == 6)
  {
    // the workspace form (measured faster: 2.12 vs 2.44 ms for 4096
    // entries) when the caller passed W; W in the cluster's shared memory
    // when it did not, or when the tuning table asks for it
    if (!(cluster & KRON_BIG_SMEM_W))
    {
      const int rc = launch_big_t<double, 6, 6, 3, 16, 2>(p, ws, prec, cluster, stream);
      if (rc != KRON_ERROR_WORKSPACE)
        return rc;
    }
    const int rc = launch_bigdsm_t<double, 6, 6, 3, 2>(p, stream);
    if (rc != KRON_ERROR_NOT_SUPPORTED)
      return rc;
    return launch_big_t<double, 6, 6, 3, 16, 2>(p, ws, prec, cluster, stream);
  }
  if (p.d == 6 && n == 7)
    return launch_big_t<double, 6, 7, 3, 8, 2>(p, ws, prec, cluster, stream);
  if (p.d == 6 && n == 8)
    return (cluster & KRON_BIG_CUDA_CORES)
               ? launch_big_t<double, 6, 8, 3, 16, 1, false>(p, ws, prec, cluster, stream)
               : launch_big_t<double, 6, 8, 3, 16, 1>(p, ws, prec, cluster, stream);
  if (p.d == 5 && n == 8)
    return launch_big_t<double, 5, 8, 2, 32, 1>(p, ws, prec, cluster, stream);
  return KRON_ERROR_NOT_SUPPORTED;
}

} // namespace kron

// Kernel templates for the batched Kronecker matvec.
//
// Algorithm (replaces kronmultv_recur.hpp / kronm_forward.hpp /
// kronm_backward.hpp): the reference evaluates one entry as a chain of
// block-cooperative global-memory GEMMs (kgemm_nt / kgemm_tt) through the
// workspace W.  Here an entry's whole vector stays in shared memory and the
// d mode products run on chip:
//
//   Z[o, i, r] = sum_j A_l(i, j) * V[o, j, r]      (mode l, r the faster modes)
//
// which is the same contraction as one kgemm_nt call of the recursive
// algorithm (kronmultv_recur.hpp:117-131, X_i * A1^T) or one kgemm_nt /
// kgemm_tt step of Alg. 993 (kronm_forward.hpp:110-151,
// kronm_backward.hpp:92-124), without the global round trip.  x is read
// once, y read-modified-written once, A read once per entry.
//
// Thread organisation: a block holds NG independent "groups" of GS threads
// (GS a multiple of 32); each group owns one entry at a time and its own
// slice of shared memory, so small vectors are packed several per block.
#pragma once

#include <type_traits>

#include "kron_internal.cuh"

namespace kron {

// ---------------------------------------------------------------- math
// Inner product policies.  F64/F32: fused multiply-add chain in T.
// SPLIT (T = double storage): A and the vector are split into FP32 hi+lo
// parts; each product a*x is formed as hi*hi exactly (TwoProduct by fma)
// plus the two cross products hi*lo + lo*hi, and the terms are summed with
// compensated (TwoSum) FP32 accumulation; the pair is returned as a double.
struct SplitF
{
  float hi, lo;
};

__device__ __forceinline__ SplitF split_double(double v)
{
  float h = __double2float_rn(v);
  float l = __double2float_rn(v - (double)h);
  return {h, l};
}

struct DFAcc
{
  float s, c; // running sum and its compensation
};

__device__ __forceinline__ void df_add_product(DFAcc &acc, SplitF a, SplitF x)
{
  float p  = a.hi * x.hi;
  float pe = fmaf(a.hi, x.hi, -p);          // exact rounding error of hi*hi
  float pl = fmaf(a.hi, x.lo, fmaf(a.lo, x.hi, pe));
  float t  = acc.s + p;                     // TwoSum(acc.s, p)
  float bp = t - acc.s;
  float e  = (acc.s - (t - bp)) + (p - bp);
  acc.s    = t;
  acc.c    = acc.c + (e + pl);
}

__device__ __forceinline__ double df_value(const DFAcc &acc)
{
  return (double)acc.s + (double)acc.c;
}

// ---------------------------------------------------------------- loads
template <typename T>
__device__ __forceinline__ T ldg_stream(const T *p)
{
  return __ldg(p);
}

// Copy `count` elements global -> shared with the group's threads, 16-byte
// vectors when both ends allow it.
template <typename T>
__device__ __forceinline__ void group_copy_in(T *dst, const T *src, int count, int t, int GS)
{
  constexpr int V = 16 / sizeof(T);
  const bool vec  = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && (count % V == 0);
  if (vec)
  {
    using VT     = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    const int nv = count / V;
    const VT *s  = reinterpret_cast<const VT *>(src);
    VT *d        = reinterpret_cast<VT *>(dst);
    for (int i = t; i < nv; i += GS)
      d[i] = __ldg(s + i);
  }
  else
  {
    for (int i = t; i < count; i += GS)
      dst[i] = __ldg(src + i);
  }
}

// A tile of `rows` rows x C columns (row stride in_row, the first Cc columns
// valid, the rest zero-filled) into dst.
template <typename T>
__device__ __forceinline__ void group_copy_tile(T *dst, const T *src, int rows, int C, int Cc,
                                                long long in_row, int t, int GS)
{
  for (int q = t; q < rows * C; q += GS)
  {
    const int h = q / C, c = q - (q / C) * C;
    dst[q]      = (c < Cc) ? __ldg(src + h * in_row + c) : T(0);
  }
}

// y (+)= buf (+ acc) for `count` elements, by the group.  The y loads of a
// batch of iterations are issued before any store (generic pointers would
// otherwise serialise every load behind the previous store).
template <typename T>
__device__ __forceinline__ void group_flush(int accum, T *y, const T *buf, const T *acc,
                                            bool use_acc, int count, int t, int GS)
{
  constexpr int V = 16 / sizeof(T);
  constexpr int B = 4; // vectors in flight per thread
  const bool vec  = (accum != ACC_ATOMIC) && ((reinterpret_cast<uintptr_t>(y) & 15) == 0) &&
                   (count % V == 0);
  if (vec)
  {
    using VT     = typename std::conditional<sizeof(T) == 8, double2, float4>::type;
    const int nv = count / V;
    VT *yv       = reinterpret_cast<VT *>(y);
    const VT *bv = reinterpret_cast<const VT *>(buf);
    const VT *av = reinterpret_cast<const VT *>(acc);
    for (int i0 = t; i0 < nv; i0 += GS * B)
    {
      VT old[B];
      if (accum != ACC_STORE)
#pragma unroll
        for (int b = 0; b < B; b++)
          if (i0 + b * GS < nv)
            old[b] = yv[i0 + b * GS];
#pragma unroll
      for (int b = 0; b < B; b++)
      {
        const int i = i0 + b * GS;
        if (i >= nv)
          continue;
        VT v = bv[i];
        T *pv = reinterpret_cast<T *>(&v);
        if (use_acc)
        {
          VT a        = av[i];
          const T *pa = reinterpret_cast<const T *>(&a);
#pragma unroll
          for (int u = 0; u < V; u++)
            pv[u] += pa[u];
        }
        if (accum != ACC_STORE)
        {
          const T *po = reinterpret_cast<const T *>(&old[b]);
#pragma unroll
          for (int u = 0; u < V; u++)
            pv[u] += po[u];
        }
        yv[i] = v;
      }
    }
  }
  else
  {
    for (int i0 = t; i0 < count; i0 += GS * B)
    {
      T old[B];
      if (accum != ACC_ATOMIC && accum != ACC_STORE)
#pragma unroll
        for (int b = 0; b < B; b++)
          if (i0 + b * GS < count)
            old[b] = y[i0 + b * GS];
#pragma unroll
      for (int b = 0; b < B; b++)
      {
        const int i = i0 + b * GS;
        if (i >= count)
          continue;
        T v = buf[i];
        if (use_acc)
          v += acc[i];
        if (accum == ACC_ATOMIC)
          red_add(y + i, v);
        else if (accum == ACC_STORE)
          y[i] = v;
        else
          y[i] = old[b] + v;
      }
    }
  }
}

// ====================================================================
// Square, compile-time (D, N): in-place mode passes, A_l in registers.
// ====================================================================
template <typename T, int D, int N, int PREC, bool MERGE>
struct SqShape
{
  static constexpr int L   = cpow(N, D);
  static constexpr int F   = L / N; // fibers per mode pass
  static constexpr int ASZ = D * N * N;
  // group size: about >= 2 fibers per thread per pass
  static constexpr int GS = F >= 512 ? 256 : (F >= 256 ? 128 : (F >= 128 ? 64 : 32));
  static constexpr int ELEMS_RAW = L * (MERGE ? 2 : 1) + ASZ;
  static constexpr int ELEMS     = (ELEMS_RAW + (16 / (int)sizeof(T)) - 1) /
                               (16 / (int)sizeof(T)) * (16 / (int)sizeof(T));
  static constexpr size_t GROUP_BYTES = (size_t)ELEMS * sizeof(T);
  static constexpr bool A_IN_REGS     = (N <= 6);
};

// One mode pass over the group's vector (in place: each fiber is read in
// full by one thread before that thread overwrites it).
template <typename T, int D, int N, int PREC, int l>
__device__ __forceinline__ void sq_mode_pass(T *buf, const T *As, int t, int GS)
{
  constexpr int S = cpow(N, D - 1 - l); // stride of mode l
  constexpr int F = cpow(N, D - 1);
  const T *Al     = As + l * N * N;     // Al[i + j*N]

  if constexpr (PREC == PREC_SPLIT)
  {
    SplitF a[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
        a[i][j] = split_double((double)Al[i + j * N]);
    for (int f = t; f < F; f += GS)
    {
      const int o = f / S, r = f - (f / S) * S;
      T *base     = buf + o * (N * S) + r;
      SplitF xv[N];
#pragma unroll
      for (int j = 0; j < N; j++)
        xv[j] = split_double((double)base[j * S]);
#pragma unroll
      for (int i = 0; i < N; i++)
      {
        DFAcc acc{0.f, 0.f};
#pragma unroll
        for (int j = 0; j < N; j++)
          df_add_product(acc, a[i][j], xv[j]);
        base[i * S] = (T)df_value(acc);
      }
    }
  }
  else if constexpr (N <= 6)
  {
    T a[N][N];
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
        a[i][j] = Al[i + j * N];
    for (int f = t; f < F; f += GS)
    {
      const int o = f / S, r = f - (f / S) * S;
      T *base     = buf + o * (N * S) + r;
      T xv[N];
#pragma unroll
      for (int j = 0; j < N; j++)
        xv[j] = base[j * S];
#pragma unroll
      for (int i = 0; i < N; i++)
      {
        T z = T(0);
#pragma unroll
        for (int j = 0; j < N; j++)
          z = fma(a[i][j], xv[j], z);
        base[i * S] = z;
      }
    }
  }
  else
  {
    for (int f = t; f < F; f += GS)
    {
      const int o = f / S, r = f - (f / S) * S;
      T *base     = buf + o * (N * S) + r;
      T xv[N];
#pragma unroll
      for (int j = 0; j < N; j++)
        xv[j] = base[j * S];
#pragma unroll
      for (int i = 0; i < N; i++)
      {
        T z = T(0);
#pragma unroll
        for (int j = 0; j < N; j++)
          z = fma(Al[i + j * N], xv[j], z);
        base[i * S] = z;
      }
    }
  }
}

template <typename T, int D, int N, int PREC, int l>
__device__ __forceinline__ void sq_all_passes(T *buf, const T *As, int t, int GS, int g)
{
  if constexpr (l < D)
  {
    sq_mode_pass<T, D, N, PREC, l>(buf, As, t, GS);
    group_sync(g, GS);
    sq_all_passes<T, D, N, PREC, l + 1>(buf, As, t, GS, g);
  }
}

template <typename T, int D, int N, int PREC, bool MERGE>
__global__ void __launch_bounds__(256) kron_sq_kernel(const __grid_constant__ Params p)
{
  using S             = SqShape<T, D, N, PREC, MERGE>;
  constexpr int L     = S::L;
  constexpr int GS    = S::GS;
  const int ng        = blockDim.x / GS;
  const int g         = threadIdx.x / GS;
  const int t         = threadIdx.x - g * GS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *buf = reinterpret_cast<T *>(smem_raw) + (size_t)g * S::ELEMS;
  T *acc = buf + L;
  T *As  = buf + L * (MERGE ? 2 : 1);

  for (int w = blockIdx.x * ng + g; w < p.nitems; w += gridDim.x * ng)
  {
    int e0, e1;
    item_range(p, w, e0, e1);
    bool have_acc = false;
    for (int e = e0; e < e1; ++e)
    {
      const int k = entry_index(p, e);
      EntryRef<T> en;
      entry_fetch<T>(p, k, D, en);

      group_sync(g, GS); // previous readers of buf / As are done
#pragma unroll
      for (int l = 0; l < D; l++)
        for (int ij = t; ij < N * N; ij += GS)
        {
          const int j = ij / N, i = ij - j * N;
          As[l * N * N + ij] = __ldg(en.A[l] + i + (long long)j * en.ld[l]);
        }
      group_copy_in(buf, en.x, L, t, GS);
      group_sync(g, GS);

      sq_all_passes<T, D, N, PREC, 0>(buf, As, t, GS, g);

      bool same_next = false;
      if constexpr (MERGE)
      {
        if (e + 1 < e1)
          same_next = (entry_y<T>(p, entry_index(p, e + 1)) == en.y);
      }
      if (same_next)
      {
        for (int i = t; i < L; i += GS)
          acc[i] = have_acc ? acc[i] + buf[i] : buf[i];
        have_acc = true;
      }
      else
      {
        group_flush(p.accum, en.y, buf, acc, have_acc, L, t, GS);
        have_acc = false;
      }
    }
  }
}

// ====================================================================
// Runtime shapes: rectangular A_l, any n, optional sub-block views (the
// two-phase path for vectors that exceed shared memory).  Out-of-place
// ping-pong between two buffers; A_l read from shared memory.
// ====================================================================
struct GenView
{
  int dd;           // number of modes applied
  int mode0;        // first applied mode of the entry
  int mm[MAXD];     // their output sizes
  int nn[MAXD];     // their input sizes
  int forward;      // 1: apply modes mode0.. first (Alg. 993 forward); 0: last first
  int subs;         // sub-blocks per entry (1 for whole vectors)
  int C;            // columns per sub-block (1 = plain vector)
  long long total_cols;   // columns overall (clips the last tile); 0 = C exactly
  long long in_sub_off;   // input element offset between consecutive sub-blocks
  long long out_sub_off;  // output element offset between consecutive sub-blocks
  long long in_row;       // input row stride (elements) of a tile
  long long out_row;      // output row stride
  int in_ws;        // 1: input from the workspace slot, 0: from x
  int out_ws;       // 1: output to the workspace slot (store), 0: to y (p.accum)
  // workspace slots: slot s at ws_base + s*ws_stride or ws_ptrs[s]
  void *ws_base;
  long long ws_stride;
  void *const *ws_ptrs;
  int ws_ptr_step;  // xbatched keeps X copies in even pointers: slot s -> ws_ptrs[s*step]
  int slot0;        // entry position e uses slot (e - slot0)
  int max_inter;    // max intermediate elements (rows * C) -- ping-pong buffer size
  int out_elems;    // output tile elements (rows_out * C)
  int asz;          // sum m*n of applied modes
  int group_elems;  // per-group shared elements
  int GS;
  int merge;
};

// One mode on fibres of compile-time length: input sizes NQ, output MQ,
// fibre f = (o, r) reads cur[(o NQ + j) in32 + r], writes
// nxt[(o MQ + i) in32 + r].  Small factors live in registers, larger ones
// are read from shared memory (broadcast) where they are used.
template <typename T, int NQ, int MQ>
__device__ __forceinline__ void gen_mode_fibres(const T *cur, T *nxt, const T *Aq, int in32,
                                                int nfib, int t, int GS)
{
  constexpr bool AREG = NQ * MQ <= 16;
  T a[AREG ? MQ : 1][AREG ? NQ : 1];
  if constexpr (AREG)
  {
#pragma unroll
    for (int i = 0; i < MQ; i++)
#pragma unroll
      for (int j = 0; j < NQ; j++)
        a[i][j] = Aq[i + j * MQ];
  }
  for (int f = t; f < nfib; f += GS)
  {
    const int o = f / in32, r = f - (f / in32) * in32;
    const T *src = cur + (o * NQ) * in32 + r;
    T *dst       = nxt + (o * MQ) * in32 + r;
    T x[NQ];
#pragma unroll
    for (int j = 0; j < NQ; j++)
      x[j] = src[j * in32];
#pragma unroll
    for (int i = 0; i < MQ; i++)
    {
      T z = T(0);
#pragma unroll
      for (int j = 0; j < NQ; j++)
        z = fma(AREG ? a[i][j] : Aq[i + j * MQ], x[j], z);
      dst[i * in32] = z;
    }
  }
}

// dispatch (nq, mq) in 1..8 to the compile-time fibre pass; false when
// out of range
template <typename T>
__device__ __forceinline__ bool gen_mode_sized(int nq, int mq, const T *cur, T *nxt, const T *Aq,
                                               int in32, int nfib, int t, int GS)
{
#define KRON_GM(NQ_, MQ_)                                                                       \
  case NQ_ * 16 + MQ_: gen_mode_fibres<T, NQ_, MQ_>(cur, nxt, Aq, in32, nfib, t, GS); return true;
#define KRON_GM_ROW(NQ_)                                                                        \
  KRON_GM(NQ_, 1) KRON_GM(NQ_, 2) KRON_GM(NQ_, 3) KRON_GM(NQ_, 4) KRON_GM(NQ_, 5)              \
  KRON_GM(NQ_, 6) KRON_GM(NQ_, 7) KRON_GM(NQ_, 8)
  switch (nq * 16 + mq)
  {
    KRON_GM_ROW(1) KRON_GM_ROW(2) KRON_GM_ROW(3) KRON_GM_ROW(4)
    KRON_GM_ROW(5) KRON_GM_ROW(6) KRON_GM_ROW(7) KRON_GM_ROW(8)
  default: return false;
  }
#undef KRON_GM_ROW
#undef KRON_GM
}

// SIZED: dispatch modes with n_l, m_l <= 8 to compile-time-sized fibre
// passes (fewer instructions per product, more registers: used by the
// uneven-batch kernel, whose blocks are limited by shared memory anyway).
// rows: independent vectors stored one after another in the buffer (an
// outer index that no mode touches; 1 for a single vector).
template <typename T, int PREC, bool SIZED = false>
__device__ void gen_apply_modes(const GenView &v, T *&cur, T *&nxt, const T *As, int C, int t,
                                int GS, int g, int rows = 1)
{
  // current dims of the applied modes
  int dims[MAXD];
  for (int q = 0; q < v.dd; q++)
    dims[q] = v.nn[q];
  int aoff[MAXD];
  {
    int o = 0;
    for (int q = 0; q < v.dd; q++)
    {
      aoff[q] = o;
      o += v.mm[q] * v.nn[q];
    }
  }
  for (int step = 0; step < v.dd; step++)
  {
    const int q  = v.forward ? step : (v.dd - 1 - step);
    const int mq = v.mm[q], nq = v.nn[q];
    long long outer = rows, inner = C;
    for (int u = 0; u < q; u++)
      outer *= dims[u];
    for (int u = q + 1; u < v.dd; u++)
      inner *= dims[u];
    const T *Aq         = As + aoff[q]; // Aq[i + j*mq]
    const long long tot = outer * mq * inner;
    if (SIZED && PREC != PREC_SPLIT && nq <= 8 && mq <= 8 && tot < (1LL << 31) &&
        gen_mode_sized<T>(nq, mq, cur, nxt, Aq, (int)inner, (int)(outer * inner), t, GS))
    {
      // fibre per thread with compile-time sizes (done above)
    }
    else if (PREC != PREC_SPLIT && nq <= 8 && tot < (1LL << 31))
    {
      // fibre per thread: its nq inputs are read once, all mq outputs formed
      // from them (A broadcast from shared memory); 32-bit index math
      const int in32 = (int)inner, nfib = (int)(outer * inner);
      for (int f = t; f < nfib; f += GS)
      {
        const int o = f / in32, r = f - (f / in32) * in32;
        const T *src = cur + (o * nq) * in32 + r;
        T *dst       = nxt + (o * mq) * in32 + r;
        T x[8];
#pragma unroll
        for (int j = 0; j < 8; j++)
          x[j] = (j < nq) ? src[j * in32] : T(0);
        for (int i = 0; i < mq; i++)
        {
          T z = T(0);
#pragma unroll
          for (int j = 0; j < 8; j++)
            if (j < nq)
              z = fma(Aq[i + j * mq], x[j], z);
          dst[i * in32] = z;
        }
      }
    }
    else
    for (long long idx = t; idx < tot; idx += GS)
    {
      const long long r  = idx % inner;
      const long long oi = idx / inner;
      const int i        = (int)(oi % mq);
      const long long o  = oi / mq;
      const T *src       = cur + o * nq * inner + r;
      if constexpr (PREC == PREC_SPLIT)
      {
        DFAcc acc{0.f, 0.f};
        for (int j = 0; j < nq; j++)
          df_add_product(acc, split_double((double)Aq[i + j * mq]),
                         split_double((double)src[j * inner]));
        nxt[idx] = (T)df_value(acc);
      }
      else
      {
        T z = T(0);
        for (int j = 0; j < nq; j++)
          z = fma(Aq[i + j * mq], src[j * inner], z);
        nxt[idx] = z;
      }
    }
    dims[q] = mq;
    T *tmp  = cur;
    cur     = nxt;
    nxt     = tmp;
    group_sync(g, GS);
  }
}

template <typename T, int PREC>
__global__ void __launch_bounds__(256) kron_gen_kernel(const __grid_constant__ Params p,
                                                       const __grid_constant__ GenView v)
{
  const int GS = v.GS;
  const int ng = blockDim.x / GS;
  const int g  = threadIdx.x / GS;
  const int t  = threadIdx.x - g * GS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *base = reinterpret_cast<T *>(smem_raw) + (size_t)g * v.group_elems;
  T *b0   = base;
  T *b1   = base + v.max_inter;
  T *acc  = base + 2 * v.max_inter;
  T *As   = acc + (v.merge ? v.out_elems : 0);

  int rows_in = 1, rows_out = 1;
  for (int q = 0; q < v.dd; q++)
  {
    rows_in *= v.nn[q];
    rows_out *= v.mm[q];
  }
  const long long total_items = (long long)p.nitems * v.subs;

  for (long long it = blockIdx.x * ng + g; it < total_items; it += (long long)gridDim.x * ng)
  {
    const int w   = (int)(it / v.subs);
    const int sub = (int)(it - (long long)w * v.subs);
    int e0, e1;
    item_range(p, w, e0, e1);
    int Cc = v.C;
    if (v.total_cols > 0)
      Cc = (int)min((long long)v.C, v.total_cols - (long long)sub * v.C);
    bool have_acc = false;
    for (int e = e0; e < e1; ++e)
    {
      const int k = entry_index(p, e);
      EntryRef<T> en;
      entry_fetch<T>(p, k, p.d, en);
      // input / output bases for this sub-block
      T *slot = nullptr;
      if (v.in_ws || v.out_ws)
      {
        const long long s = e - v.slot0;
        slot              = v.ws_ptrs ? static_cast<T *>(v.ws_ptrs[s * v.ws_ptr_step])
                                      : static_cast<T *>(v.ws_base) + s * v.ws_stride;
      }
      const T *in = (v.in_ws ? slot : en.x) + (long long)sub * v.in_sub_off;
      T *out      = (v.out_ws ? slot : en.y) + (long long)sub * v.out_sub_off;

      group_sync(g, GS);
      {
        int o = 0;
        for (int q = 0; q < v.dd; q++)
        {
          const int l   = v.mode0 + q;
          const int mq  = v.mm[q], nq = v.nn[q];
          const T *Asrc = en.A[l];
          const int ld  = en.ld[l];
          for (int u = t; u < mq * nq; u += GS)
          {
            const int j = u / mq, i = u - j * mq;
            As[o + u]   = __ldg(Asrc + i + (long long)j * ld);
          }
          o += mq * nq;
        }
      }
      if (v.C == 1)
        group_copy_in(b0, in, rows_in, t, GS);
      else
        group_copy_tile(b0, in, rows_in, v.C, Cc, v.in_row, t, GS);
      group_sync(g, GS);

      T *cur = b0, *nxt = b1;
      gen_apply_modes<T, PREC>(v, cur, nxt, As, v.C, t, GS, g);

      const int accum = v.out_ws ? (int)ACC_STORE : p.accum;
      bool same_next  = false;
      if (v.merge && !v.out_ws && e + 1 < e1)
        same_next = (entry_y<T>(p, entry_index(p, e + 1)) == en.y);
      if (same_next)
      {
        for (int i = t; i < rows_out * v.C; i += GS)
          acc[i] = have_acc ? acc[i] + cur[i] : cur[i];
        have_acc = true;
      }
      else if (v.C == 1)
      {
        group_flush(accum, out, cur, acc, have_acc, rows_out, t, GS);
        have_acc = false;
      }
      else
      {
        for (int q = t; q < rows_out * v.C; q += GS)
        {
          const int i = q / v.C, c = q - i * v.C;
          if (c < Cc)
          {
            T val = cur[q];
            if (have_acc)
              val += acc[q];
            y_update(accum, out + i * v.out_row, c, val);
          }
        }
        have_acc = false;
      }
    }
  }
}

} // namespace kron

// Pipelined on-chip kernel for square n in {3,4,5} with mid-size vectors
// (4 KB .. 64 KB per entry): the HBM-bound regime of kronmult{d}_batched
// (e.g. d = 6, n = 4, 32 KB vectors in FP64).
//
// Persistent 256-thread blocks (2 per SM in FP64, 4 in FP32) each own a
// balanced contiguous range of entries.  Each entry's x vector and its
// A_1..A_d block are brought into a ring of shared-memory stages by TMA bulk
// copies (cp.async.bulk, one elected thread, mbarrier completion) ahead of
// use, and y is prefetched into L2 at the same time, so HBM streams while the
// block computes.  The d mode products run as ceil(d/k) register-blocked
// passes: a thread loads a fibre of n^k elements spanning k consecutive
// modes, applies those k factors from registers (k = 2, 2, 1 for n = 3, 4, 5)
// and writes the fibre back.  Pass order: group 0 first (reading the stage,
// consecutive lanes on consecutive addresses), the last group next, the
// middle groups last; the final pass writes the result, unswizzled, into the
// entry's stage and one TMA bulk reduce-add adds it into y.  The stage is
// refilled after the next entry's first pass, when the reduce has read it.
//
// For n = 4 the work buffer is XOR-swizzled within 128-byte rows (8-byte
// elements: row r permutes its elements by r & 15; 4-byte elements: whole
// 16-byte chunks by (r & 3) | ((r >> 1) & 4), so contiguous fibres move as
// float4), which a bank model shows conflict free for every pass.  Both
// swizzles are linear over XOR, so a fibre's element addresses are its base
// address XOR compile-time constants.  FP32 with n = 4 computes with packed
// fma.rn.f32x2 / mul.rn.f32x2 from a row-major copy of the factors made once
// per entry: each output is two pair products and one add.  For d = 6,
// n = 4 the last two passes stay inside each warp's slabs and are separated
// by a warp barrier only.
//
// Every mbarrier wait is bounded (wait_limit() polls); on time-out the block
// records 1 in the library's device status word (kron_device_status), lets the
// copies it started land (bounded by the full default limit, whatever the
// wait limit) and leaves.
#include <cstdint>

#include "kron_launch.h"
#include "kron_ptx.cuh"

namespace kron {

namespace {

// FP32 blocks per SM (compile time; 4 measured best for d = 6, n = 4: more
// resident warps hide the shared-memory latency of the passes)
#ifndef KRON_PIPE_F32_BLOCKS
#define KRON_PIPE_F32_BLOCKS 4
#endif

constexpr int PIPE_THREADS = 256;
constexpr int MAX_STAGES   = 6;

template <int N>
struct GroupK
{
  static constexpr int k = (N == 5) ? 1 : 2;
};

template <typename T, int N>
__device__ __forceinline__ int swz(int e)
{
  if constexpr (N == 4)
  {
    if constexpr (sizeof(T) == 8)
    {
      const int row = e >> 4;
      return e ^ (row & 15);
    }
    else
    {
      // 4-byte elements: whole 16-byte chunks are permuted (chunk index XOR
      // row & 3, and XOR 4 for rows with bit 3 set), so contiguous fibres can
      // move as float4 while strided passes stay conflict free
      const int row = e >> 5;
      return e ^ (((row & 3) | ((row >> 1) & 4)) << 2);
    }
  }
  else
    return e;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
  unsigned a = (unsigned)__cvta_generic_to_shared(bar);
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(a), "r"(parity)
               : "memory");
  return ok != 0;
}

__device__ __forceinline__ void tma_load(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
  unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(src), "r"(bytes), "r"(b)
               : "memory");
}

__device__ __forceinline__ void l2_prefetch(const void *src, unsigned bytes)
{
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// y[0..bytes) += smem[0..bytes) by the TMA engine (element-wise atomic adds
// in L2); completion tracked by the issuing thread's bulk group.
template <typename T>
__device__ __forceinline__ void bulk_reduce_add(T *y, const T *src, unsigned bytes)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(src);

  if constexpr (sizeof(T) == 8)
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(y),
                 "r"(s), "r"(bytes)
                 : "memory");
  else
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(y),
                 "r"(s), "r"(bytes)
                 : "memory");
  asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ bool tma_ok(const void *ptr, long long bytes)
{
  return ((reinterpret_cast<uintptr_t>(ptr) & 15) == 0) && (bytes % 16 == 0) && bytes > 0 &&
         bytes < (1LL << 20);
}

// Passes in order: group 0 (reads the stage), then the last group, then the
// middle groups; the final pass writes the result into the stage for one
// bulk reduce-add.
template <typename T, int D, int N>
struct PipePlan
{
  static constexpr int k      = GroupK<N>::k;
  static constexpr int ngroup = (D + k - 1) / k;
  static constexpr int last_a = (ngroup - 1) * k;
  static constexpr int last_k = D - last_a;
  // stride of the pass executed last (a middle group when ngroup >= 3)
  static constexpr int final_a = ngroup >= 3 ? (ngroup - 2) * k : last_a;
  static constexpr int final_k = ngroup >= 3 ? k : last_k;
  static constexpr int final_S = cpow(N, D - final_a - final_k);
  // d = 6 with two-mode groups: the last-group pass (fibre f = n^2
  // contiguous elements, inside slab f / n^2) and the final middle pass
  // (fibre f = o n^2 + r, inside slab o = f / n^2) keep fibre f in the same
  // slab (fixed i_1, i_2) of n^4 elements; with f = thread index and n^2
  // dividing the warp size (n = 4), each warp's fibres cover whole slabs,
  // so a warp reads and writes only its own slabs between the two passes
  static constexpr bool WARP_LOCAL_TAIL =
      D == 6 && k == 2 && ngroup == 3 && 32 % (N * N) == 0 && cpow(N, 4) <= PIPE_THREADS;
};

// Stage layout in shared memory (bytes; every region 16-byte aligned):
//   [0, 64)                     mbarriers (MAX_STAGES x 8)
//   [64, 64 + 4*MAX_STAGES)     per-stage operand flags (META_*)
//   [128, 128 + LB)             work buffer (swizzled)
//   [.., + AREG)                A of the entry being computed, row major
//                               (packed FP32 passes only)
//   then per stage: x (LB bytes) and A (AB bytes); the final pass writes the
//   result over x
template <typename T, int D, int N>
struct PipeLayout
{
  static constexpr int L        = cpow(N, D);
  static constexpr int ASZ      = D * N * N;
  static constexpr bool PACKED  = sizeof(T) == 4 && N == 4;
  static constexpr size_t LB    = ((size_t)L * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t AB    = ((size_t)ASZ * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t AREG  = PACKED ? (size_t)D * 16 * sizeof(float) : 0;
  static constexpr size_t WORK  = 128;
  static constexpr size_t ACUR  = WORK + LB;
  static constexpr size_t STAGE0 = ACUR + AREG;
  static constexpr size_t STAGE_BYTES = LB + AB;
  static size_t bytes(int ns) { return STAGE0 + ns * STAGE_BYTES; }
};

// flags the issuing thread records per stage
constexpr int META_X_TMA  = 1; // x arrived by bulk copy
constexpr int META_A_TMA  = 2; // A_1..A_d arrived by bulk copy (contiguous)
constexpr int META_Y_BULK = 4; // y takes the bulk reduce-add
constexpr int META_Y_PF   = 8; // y's L2 prefetch went out with the copies

// Offset of element base + kk of a fibre.  In a swizzled buffer the XOR
// swizzle is linear over GF(2) and base, kk occupy disjoint bits (n = 4:
// base = o*C*S + r with r < S, kk = c*S < C*S), so
// swz(base + kk) = swz(base) ^ swz(kk) with swz(kk) a compile-time constant.
template <typename T, int N, bool SWZ>
__device__ __forceinline__ int fib_off(int sb, int kk)
{
  if constexpr (SWZ && N == 4)
    return sb ^ swz<T, N>(kk);
  else
    return sb + kk;
}

// the k factors of a group, Ar[m][i][j] = A_{a+m}(i, j), from column-major
// storage (16-byte aligned for n = 4: one vector load per column)
template <typename T, int N, int k>
__device__ __forceinline__ void load_factors(const T *As, T (&Ar)[k][N][N])
{
#pragma unroll
  for (int m = 0; m < k; m++)
#pragma unroll
    for (int j = 0; j < N; j++)
    {
      if constexpr (N == 4 && sizeof(T) == 8)
      {
        const double2 u0 = *reinterpret_cast<const double2 *>(As + m * 16 + 4 * j);
        const double2 u1 = *reinterpret_cast<const double2 *>(As + m * 16 + 4 * j + 2);
        Ar[m][0][j] = u0.x;
        Ar[m][1][j] = u0.y;
        Ar[m][2][j] = u1.x;
        Ar[m][3][j] = u1.y;
      }
      else if constexpr (N == 4 && sizeof(T) == 4)
      {
        const float4 u = *reinterpret_cast<const float4 *>(As + m * 16 + 4 * j);
        Ar[m][0][j] = u.x;
        Ar[m][1][j] = u.y;
        Ar[m][2][j] = u.z;
        Ar[m][3][j] = u.w;
      }
      else
      {
#pragma unroll
        for (int i = 0; i < N; i++)
          Ar[m][i][j] = As[m * N * N + i + j * N];
      }
    }
}

// destinations of a pass
constexpr int DST_WORK  = 0; // work buffer (swizzled)
constexpr int DST_STAGE = 1; // stage buffer (plain layout)

// One register-blocked pass over the modes [a, a+k): the source is the
// stage (plain layout) or the work buffer (swizzled).  As points at A_1
// (column-major, n x n per mode).
template <typename T, int D, int N, int a, int k, bool SRC_STAGE, int DST>
__device__ __forceinline__ void pipe_pass(const T *src, T *dst, const T *As, int tid)
{
  constexpr int S = cpow(N, D - a - k); // stride of the group's last mode
  constexpr int C = cpow(N, k);
  constexpr int F = cpow(N, D) / C;
  T Ar[k][N][N];
  load_factors<T, N, k>(As + a * N * N, Ar);

  for (int f = tid; f < F; f += PIPE_THREADS)
  {
    const int o = f / S, r = f - (f / S) * S;
    const int base = o * (C * S) + r;
    const int sbs  = SRC_STAGE ? base : swz<T, N>(base);
    const int sbd  = DST == DST_WORK ? swz<T, N>(base) : base;
    constexpr bool VEC4 = (sizeof(T) == 4) && (S == 1) && (C % 4 == 0) && (N == 4);
    T v[C];
    if constexpr (VEC4)
    {
#pragma unroll
      for (int c = 0; c < C; c += 4)
      {
        const float4 u = *reinterpret_cast<const float4 *>(src + fib_off<T, N, !SRC_STAGE>(sbs, c));
        v[c] = u.x;
        v[c + 1] = u.y;
        v[c + 2] = u.z;
        v[c + 3] = u.w;
      }
    }
    else
    {
#pragma unroll
      for (int c = 0; c < C; c++)
        v[c] = src[fib_off<T, N, !SRC_STAGE>(sbs, c * S)];
    }
    // apply the group's factors, fastest mode (a+k-1) first
#pragma unroll
    for (int m = k - 1; m >= 0; m--)
    {
      const int inner = cpow(N, k - 1 - m); // stride of mode a+m inside the fibre
      T w[C];
#pragma unroll
      for (int c = 0; c < C; c++)
      {
        const int jm   = (c / inner) % N;
        const int base0 = c - jm * inner;
        T z            = T(0);
#pragma unroll
        for (int j = 0; j < N; j++)
          z = fma(Ar[m][jm][j], v[base0 + j * inner], z);
        w[c] = z;
      }
#pragma unroll
      for (int c = 0; c < C; c++)
        v[c] = w[c];
    }
    if constexpr (VEC4)
    {
#pragma unroll
      for (int c = 0; c < C; c += 4)
        *reinterpret_cast<float4 *>(dst + fib_off<T, N, DST == DST_WORK>(sbd, c)) =
            make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
    }
    else
    {
#pragma unroll
      for (int c = 0; c < C; c++)
        dst[fib_off<T, N, DST == DST_WORK>(sbd, c * S)] = v[c];
    }
  }
}

// ---- packed FP32 (fma.rn.f32x2) passes for n = 4 ----
typedef unsigned long long f2_t; // two floats in one 64-bit register pair

__device__ __forceinline__ f2_t pk2(float x, float y)
{
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
  return r;
}
__device__ __forceinline__ void upk2(f2_t r, float &x, float &y)
{
  asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(r));
}
__device__ __forceinline__ float hsum2(f2_t r)
{
  float x, y;
  upk2(r, x, y);
  return x + y;
}
__device__ __forceinline__ f2_t mul2(f2_t a, f2_t b)
{
  f2_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t fma2(f2_t a, f2_t b, f2_t c)
{
  f2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Factor layout for the packed passes, built once per entry:
//   arow[l*16 + 4i + j] = A_l(i, j)   (row major)
// Both modes of a pass contract horizontally: pairs {A(i,2h), A(i,2h+1)}
// times pairs of the two inputs they multiply, then one add per output.
__device__ __forceinline__ void prep_packed(const float *Acol, float *arow, int D, int tid)
{
  for (int t = tid; t < D * 16; t += PIPE_THREADS)
  {
    const int l = t >> 4, i = t & 3, j = (t >> 2) & 3; // t = l*16 + i + 4j
    arow[l * 16 + 4 * i + j] = Acol[t];
  }
}

// fibre of 4 consecutive-mode elements v[4q + j] (q = slow index, j = fast):
// w[4q + i] = sum_j A(i, j) v[4q + j] with V[2q + h] = {v[4q+2h], v[4q+2h+1]}
template <int Q>
__device__ __forceinline__ void fast_mode(const float *arow, const f2_t (&V)[2 * Q], float (&w)[4 * Q])
{
#pragma unroll
  for (int i = 0; i < 4; i++)
  {
    const ulonglong2 P = *reinterpret_cast<const ulonglong2 *>(arow + 4 * i);
#pragma unroll
    for (int q = 0; q < Q; q++)
      w[4 * q + i] = hsum2(fma2(P.y, V[2 * q + 1], mul2(P.x, V[2 * q])));
  }
}

template <int D, int a, int k, bool SRC_STAGE, int DST>
__device__ __forceinline__ void pipe_pass_packed(const float *src, float *dst, const float *areg,
                                                 int tid)
{
  constexpr int N = 4;
  constexpr int S = cpow(N, D - a - k);
  constexpr int C = cpow(N, k);
  constexpr int F = cpow(N, D) / C;
  static_assert(k == 1 || k == 2, "packed passes cover one or two modes");
  static_assert(k == 2 || S == 1, "a one-mode packed pass is the last (contiguous) group");
  const float *arow = areg + (a + k - 1) * 16; // fast mode a+k-1
  const float *srow = areg + a * 16;           // slow mode a

  for (int f = tid; f < F; f += PIPE_THREADS)
  {
    const int o = f / S, r = f - (f / S) * S;
    const int base = o * (C * S) + r;
    const int sbs  = SRC_STAGE ? base : swz<float, N>(base);
    const int sbd  = DST == DST_WORK ? swz<float, N>(base) : base;
    constexpr int Q = C / 4;
    f2_t V[2 * Q];
    if constexpr (S == 1)
    {
#pragma unroll
      for (int q = 0; q < Q; q++)
      {
        const ulonglong2 u =
            *reinterpret_cast<const ulonglong2 *>(src + fib_off<float, N, !SRC_STAGE>(sbs, 4 * q));
        V[2 * q]     = u.x;
        V[2 * q + 1] = u.y;
      }
    }
    else
    {
#pragma unroll
      for (int c = 0; c < C; c += 2)
        V[c / 2] = pk2(src[fib_off<float, N, !SRC_STAGE>(sbs, c * S)],
                       src[fib_off<float, N, !SRC_STAGE>(sbs, (c + 1) * S)]);
    }
    float w[C];
    fast_mode<Q>(arow, V, w);
    // store 4 results q' (elements 4q' .. 4q'+3 of the fibre)
    auto put4 = [&](int q, float o0, float o1, float o2, float o3) {
      if constexpr (S == 1)
        *reinterpret_cast<float4 *>(dst + fib_off<float, N, DST == DST_WORK>(sbd, 4 * q)) =
            make_float4(o0, o1, o2, o3);
      else
      {
        dst[fib_off<float, N, DST == DST_WORK>(sbd, (4 * q) * S)]     = o0;
        dst[fib_off<float, N, DST == DST_WORK>(sbd, (4 * q + 1) * S)] = o1;
        dst[fib_off<float, N, DST == DST_WORK>(sbd, (4 * q + 2) * S)] = o2;
        dst[fib_off<float, N, DST == DST_WORK>(sbd, (4 * q + 3) * S)] = o3;
      }
    };
    if constexpr (k == 1)
      put4(0, w[0], w[1], w[2], w[3]);
    else
    {
      // slow mode a: out[4q' + t] = sum_j A_a(q', j) w[4j + t], contracted
      // in pairs {w[t], w[4+t]}, {w[8+t], w[12+t]}
      f2_t W[8];
#pragma unroll
      for (int t = 0; t < 4; t++)
      {
        W[2 * t]     = pk2(w[t], w[4 + t]);
        W[2 * t + 1] = pk2(w[8 + t], w[12 + t]);
      }
#pragma unroll
      for (int qq = 0; qq < 4; qq++)
      {
        const ulonglong2 R = *reinterpret_cast<const ulonglong2 *>(srow + 4 * qq);
        float o4[4];
#pragma unroll
        for (int t = 0; t < 4; t++)
          o4[t] = hsum2(fma2(R.y, W[2 * t + 1], mul2(R.x, W[2 * t])));
        put4(qq, o4[0], o4[1], o4[2], o4[3]);
      }
    }
  }
}

// dispatch one pass to the packed or the scalar form
template <typename T, int D, int N, int a, int k, bool SRC_STAGE, int DST>
__device__ __forceinline__ void run_pass(const T *src, T *dst, const T *As, int tid)
{
  if constexpr (PipeLayout<T, D, N>::PACKED)
    pipe_pass_packed<D, a, k, SRC_STAGE, DST>(src, dst, As, tid);
  else
    pipe_pass<T, D, N, a, k, SRC_STAGE, DST>(src, dst, As, tid);
}

template <typename T, int D, int N, int gi>
__device__ __forceinline__ void middle_passes(T *work, const T *As, int tid)
{
  using P = PipePlan<T, D, N>;
  if constexpr (gi < P::ngroup - 1)
  {
    constexpr int a = gi * P::k;
    if constexpr (gi != P::ngroup - 2) // group ngroup-2 is the final pass
    {
      run_pass<T, D, N, a, P::k, false, DST_WORK>(work, work, As, tid);
      __syncthreads();
    }
    middle_passes<T, D, N, gi + 1>(work, As, tid);
  }
}

// blocks per SM the kernel is compiled for: the 4-byte path moves half the
// bytes per entry, so more blocks hide its per-entry fixed costs
template <typename T>
struct PipeOcc
{
  static constexpr int value = sizeof(T) == 4 ? KRON_PIPE_F32_BLOCKS : 2;
};

template <typename T, int D, int N>
__global__ void __launch_bounds__(PIPE_THREADS, PipeOcc<T>::value)
    kron_pipe_kernel(const __grid_constant__ Params p, int nstage, int *status, long long spin,
                     long long drain)
{
  using Lay = PipeLayout<T, D, N>;
  using P   = PipePlan<T, D, N>;
  constexpr int L   = Lay::L;
  constexpr int ASZ = Lay::ASZ;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  int *meta      = reinterpret_cast<int *>(smem + 64);
  T *work        = reinterpret_cast<T *>(smem + Lay::WORK);
  T *areg        = reinterpret_cast<T *>(smem + Lay::ACUR);
  auto stage_x   = [&](int s) { return reinterpret_cast<T *>(smem + Lay::STAGE0 + s * Lay::STAGE_BYTES); };
  auto stage_a   = [&](int s) {
    return reinterpret_cast<T *>(smem + Lay::STAGE0 + s * Lay::STAGE_BYTES + Lay::LB);
  };
  const int tid  = threadIdx.x;

  const long long tot = p.eend - p.ebase;
  const int eb = p.ebase + (int)(tot * blockIdx.x / gridDim.x);
  const int ee = p.ebase + (int)(tot * (blockIdx.x + 1) / gridDim.x);
  if (eb >= ee)
    return;

  if (tid == 0)
  {
    for (int s = 0; s < nstage; s++)
      mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const long long xb = (long long)L * sizeof(T);
  const long long ab = (long long)ASZ * sizeof(T);
  unsigned inflight = 0; // thread 0: stages with copies not yet waited for
  // issue the copies of position e into stage s (thread 0 only) and record
  // which operands the copies carry
  // pf_y: prefetch y into L2 together with the copies (refills, an entry or
  // more ahead); the copies issued at launch leave it to the entry's start so
  // that every block's first x is not queued behind the y lines
  auto issue = [&](int e, int s, bool pf_y) {
    EntryRef<T> en;
    entry_fetch<T>(p, entry_index(p, e), D, en);
    const bool a_contig =
        (p.layout == LAYOUT_BATCHED || p.layout == LAYOUT_PBATCHED) && tma_ok<T>(en.A[0], ab);
    const bool x_ok = tma_ok<T>(en.x, xb);
    const bool y_ok = tma_ok<T>(en.y, xb);
    meta[s] = (x_ok ? META_X_TMA : 0) | (a_contig ? META_A_TMA : 0) | (y_ok ? META_Y_BULK : 0) |
              (y_ok && pf_y ? META_Y_PF : 0);
    unsigned bytes = (x_ok ? (unsigned)xb : 0u) + (a_contig ? (unsigned)ab : 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bars[s], bytes);
    if (x_ok)
      tma_load(stage_x(s), en.x, (unsigned)xb, &bars[s]);
    if (a_contig)
      tma_load(stage_a(s), en.A[0], (unsigned)ab, &bars[s]);
    if (y_ok && pf_y)
      l2_prefetch(en.y, (unsigned)xb);
    inflight |= 1u << s;
  };

  int ahead = min(nstage, ee - eb);
  if (tid == 0)
    for (int i = 0; i < ahead; i++)
      issue(eb + i, i, false);
  unsigned phases = 0; // bit s = parity to wait for on stage s
  int pending_e = -1, pending_s = 0; // stage refill waiting for its reduce to read it

  for (int e = eb; e < ee; ++e)
  {
    const int s = (e - eb) % nstage;
    // wait for stage s (bounded); the outcome is combined at the barrier
    // below, after the A preparation (which reads in-bounds shared memory
    // either way)
    const bool done = ptx::mbar_wait_bounded(&bars[s], (phases >> s) & 1, spin);
    const int fl = meta[s];
    if (tid == 0 && done)
    {
      inflight &= ~(1u << s);
      if ((fl & META_Y_BULK) && !(fl & META_Y_PF))
        l2_prefetch(entry_y<T>(p, entry_index(p, e)), (unsigned)xb);
    }
    T *sx        = stage_x(s);
    T *sa        = stage_a(s);
    // operands the bulk copy could not take (block-uniform): plain loads
    // into the same stage
    if ((fl & (META_X_TMA | META_A_TMA)) != (META_X_TMA | META_A_TMA))
    {
      EntryRef<T> en;
      entry_fetch<T>(p, entry_index(p, e), D, en);
      if (!(fl & META_X_TMA))
        for (int i = tid; i < L; i += PIPE_THREADS)
          sx[i] = __ldg(en.x + i);
      if (!(fl & META_A_TMA))
      {
#pragma unroll
        for (int l = 0; l < D; l++)
          for (int ij = tid; ij < N * N; ij += PIPE_THREADS)
          {
            const int j = ij / N, i = ij - j * N;
            sa[l * N * N + ij] = __ldg(en.A[l] + i + (long long)j * en.ld[l]);
          }
      }
      __syncthreads();
    }
    // A for this entry's passes: straight from the stage, or (packed FP32)
    // in the layouts the packed passes read
    const T *As = sa;
    if constexpr (Lay::PACKED)
    {
      prep_packed(reinterpret_cast<const float *>(sa), reinterpret_cast<float *>(areg), D, tid);
      As = areg;
    }
    if (!__syncthreads_and(done))
    {
      if (tid == 0)
      {
        if (status)
          atomicExch(status, 1);
        // let the copies this block started land before it leaves (bounded)
        for (int s2 = 0; s2 < nstage; s2++)
          if ((inflight >> s2) & 1)
            for (long long it = 0; it < drain; ++it)
              if (mbar_try_wait(&bars[s2], (phases >> s2) & 1))
                break;
        bulk_wait_all();
      }
      return;
    }
    phases ^= 1u << s;

    // pass 1: group 0, stage -> work
    run_pass<T, D, N, 0, P::k, true, DST_WORK>(sx, work, As, tid);
    __syncthreads();
    // the previous entry's reduce was issued a pass ago: refill its stage
    if (tid == 0 && pending_e >= 0)
    {
      bulk_wait_read();
      issue(pending_e, pending_s, true);
      pending_e = -1;
    }

    // remaining passes; the last writes the result, unswizzled, into the
    // (now free) stage buffer
    if constexpr (P::ngroup >= 3)
    {
      run_pass<T, D, N, P::last_a, P::last_k, false, DST_WORK>(work, work, As, tid);
      if constexpr (P::WARP_LOCAL_TAIL)
        __syncwarp(); // both passes keep to this warp's slabs
      else
        __syncthreads();
      middle_passes<T, D, N, 1>(work, As, tid);
      run_pass<T, D, N, P::final_a, P::final_k, false, DST_STAGE>(work, sx, As, tid);
    }
    else
      run_pass<T, D, N, P::last_a, P::last_k, false, DST_STAGE>(work, sx, As, tid);

    // y += result: one bulk reduce-add by the TMA engine when y allows it
    const bool bulk = (fl & META_Y_BULK) != 0;
    if (bulk)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (bulk)
    {
      if (tid == 0)
        bulk_reduce_add(entry_y<T>(p, entry_index(p, e)), sx, (unsigned)xb);
    }
    else
    {
      T *y = entry_y<T>(p, entry_index(p, e));
      constexpr int B = 8;
      for (int i0 = tid; i0 < L; i0 += PIPE_THREADS * B)
      {
        T yv[B];
        if (p.accum != ACC_ATOMIC)
#pragma unroll
          for (int b = 0; b < B; b++)
            if (i0 + b * PIPE_THREADS < L)
              yv[b] = y[i0 + b * PIPE_THREADS];
#pragma unroll
        for (int b = 0; b < B; b++)
        {
          const int i = i0 + b * PIPE_THREADS;
          if (i < L)
          {
            if (p.accum == ACC_ATOMIC)
              red_add(y + i, sx[i]);
            else
              y[i] = yv[b] + sx[i];
          }
        }
      }
      __syncthreads();
    }
    // the stage now holds the result; it is refilled after the next
    // entry's first pass, when the reduce has read it
    if (tid == 0 && e + nstage < ee)
    {
      pending_e = e + nstage;
      pending_s = s;
    }
  }
  if (tid == 0)
    bulk_wait_all();
}

template <typename T, int D, int N>
int launch_pipe_t(Params p, cudaStream_t stream)
{
  using Lay            = PipeLayout<T, D, N>;
  const void *fn       = reinterpret_cast<const void *>(&kron_pipe_kernel<T, D, N>);
  const int maxsm      = device_info().max_smem_optin;
  // PipeOcc blocks per SM when two stages each still fit, else one block
  int per_sm = PipeOcc<T>::value;
  int ns     = 0;
  for (; per_sm >= 2; --per_sm)
  {
    const long long budget = (long long)device_info().smem_per_sm / per_sm - 1024;
    ns = (int)std::min<long long>(MAX_STAGES, (budget - (long long)Lay::STAGE0) /
                                                  (long long)Lay::STAGE_BYTES);
    if (ns >= 2)
      break;
  }
  if (ns < 2)
  {
    per_sm = 1;
    ns     = (int)std::min<long long>(
        MAX_STAGES, (long long)((maxsm - Lay::STAGE0) / Lay::STAGE_BYTES));
  }
  if (ns < 2)
    return KRON_ERROR_NOT_SUPPORTED;
  const size_t smem = Lay::bytes(ns);
  int occ           = 1;
  if (cached_occupancy(fn, PIPE_THREADS, smem, &occ) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  per_sm = std::min(per_sm, occ);
  const long long work = p.eend - p.ebase;
  const long long grid =
      std::max<long long>(1, std::min<long long>(work, (long long)device_info().sms * per_sm));
  int *status          = device_status_ptr();
  long long spin       = wait_limit();
  long long drain      = drain_limit();
  void *args[]         = {&p, &ns, &status, &spin, &drain};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(PIPE_THREADS), args, smem, stream) ==
                 cudaSuccess
             ? KRON_SUCCESS
             : KRON_ERROR_LAUNCH;
}

template <typename T>
int pipe_pick(int d, int n, Params p, cudaStream_t s)
{
  // the (d, n) whose vectors are 4..64 KB in FP64 or FP32
  if (d == 6 && n == 3)
    return launch_pipe_t<T, 6, 3>(p, s);
  if (d == 5 && n == 4)
    return launch_pipe_t<T, 5, 4>(p, s);
  if (d == 6 && n == 4)
    return launch_pipe_t<T, 6, 4>(p, s);
  if (d == 4 && n == 5)
    return launch_pipe_t<T, 4, 5>(p, s);
  if (d == 5 && n == 5)
    return launch_pipe_t<T, 5, 5>(p, s);
  if (d == 6 && n == 5)
    return launch_pipe_t<T, 6, 5>(p, s);
  return KRON_ERROR_NOT_SUPPORTED;
}

} // namespace

bool pipe_supported(const Params &p, int prec)
{
  if (prec == PREC_SPLIT || p.accum == ACC_SEGMENTED || p.accum == ACC_STORE)
    return false;
  if (p.d < 3 || p.d > 6)
    return false;
  const int n = p.n[0];
  if (n < 3 || n > 5)
    return false;
  for (int l = 0; l < p.d; l++)
    if (p.m[l] != n || p.n[l] != n)
      return false;
  long long L = 1;
  for (int l = 0; l < p.d; l++)
    L *= n;
  const long long bytes = L * (prec == PREC_F32 ? 4 : 8);
  return bytes >= 4096 && bytes <= 65536;
}

int launch_pipe(Params p, int prec, cudaStream_t stream)
{
  if (p.eend <= p.ebase)
    return KRON_SUCCESS;
  if (prec == PREC_F32)
    return pipe_pick<float>(p.d, p.n[0], p, stream);
  return pipe_pick<double>(p.d, p.n[0], p, stream);
}

} // namespace kron

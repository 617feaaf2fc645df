// Pipelined on-chip kernel for square n in {3,4,5} with mid-size vectors
// (4 KB .. 64 KB per entry): the HBM-bound regime of kronmult{d}_batched
// (e.g. d = 6, n = 4, 32 KB vectors in FP64).
//
// One persistent 256-thread block per SM owns a balanced contiguous range
// of entries.  Each entry's x vector and its A_1..A_d block are brought into
// a ring of shared-memory stages by TMA bulk copies (cp.async.bulk, one
// elected thread, mbarrier completion) several entries ahead, and y is
// prefetched into L2 at the same time, so HBM streams while the block
// computes.  The d mode products run as ceil(d/k) register-blocked passes:
// a thread loads a fibre of n^k elements spanning k consecutive modes,
// applies those k factors from registers (k = 2, 2, 1 for n = 3, 4, 5)
// and writes the fibre back.  Pass order: the group holding mode 1 first
// (reading the TMA stage, consecutive lanes on consecutive addresses), the
// group holding mode d next, the middle groups last; when the last pass's
// stride is at least 16 elements it adds straight into y with coalesced
// accesses, otherwise a final coalesced sweep does.  For power-of-two n the
// work buffer is XOR-swizzled within 128-byte rows (8-byte elements: row r
// permutes its elements by r & 15; 4-byte elements: whole 16-byte chunks by
// (r & 3) | ((r >> 1) & 4), so contiguous fibres move as float4), which a
// bank model shows conflict free for every pass.
//
// Every mbarrier wait is bounded; on time-out the block records 1 in the
// library's device status word (kron_device_status) and leaves.
#include <cstdint>

#include "kron_launch.h"

namespace kron {

__device__ int g_device_status = 0;

namespace {

constexpr int PIPE_THREADS = 256;
constexpr int MAX_STAGES   = 6;
constexpr long long SPIN_LIMIT = 1LL << 26;

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
// all but the most recent bulk group have finished reading shared memory
__device__ __forceinline__ void bulk_wait_read_but_last() { asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

template <typename T>
__device__ __forceinline__ bool tma_ok(const void *ptr, long long bytes)
{
  return ((reinterpret_cast<uintptr_t>(ptr) & 15) == 0) && (bytes % 16 == 0) && bytes > 0 &&
         bytes < (1LL << 20);
}

// Stage layout in shared memory (bytes):
//   [0, 64)                     mbarriers (MAX_STAGES x 8)
//   [128, 128 + L*sz)           work buffer (swizzled)
//   [.., + ASZ*sz)              A of the entry being computed
//   then per stage: x (L*sz) and A (ASZ*sz), 16-byte aligned
template <typename T, int D, int N>
struct PipeLayout
{
  static constexpr int L        = cpow(N, D);
  static constexpr int ASZ      = D * N * N;
  static constexpr int ASZ_PAD  = (ASZ + 15) / 16 * 16;
  static constexpr size_t WORK  = 128;
  static constexpr size_t ACUR  = WORK + (size_t)L * sizeof(T);
  static constexpr size_t STAGE0 = ACUR + (size_t)ASZ_PAD * sizeof(T);
  static constexpr size_t STAGE_BYTES = ((size_t)L + ASZ_PAD) * sizeof(T);
  static size_t bytes(int ns) { return STAGE0 + ns * STAGE_BYTES; }
};

// One register-blocked pass over the modes [a, a+k): SRC/DST select the
// stage (unswizzled) / work buffer (swizzled) / y (global, DIRECT).
template <typename T, int D, int N, int a, int k, bool SRC_STAGE, bool DIRECT>
__device__ __forceinline__ void pipe_pass(const T *src, T *dst, const T *As, T *y, int accum,
                                          int tid)
{
  constexpr int S = cpow(N, D - a - k); // stride of the group's last mode
  constexpr int C = cpow(N, k);
  constexpr int F = cpow(N, D) / C;
  // factors of the group in registers: Ar[m][i][j] = A_{a+m}(i, j)
  T Ar[k][N][N];
#pragma unroll
  for (int m = 0; m < k; m++)
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
        Ar[m][i][j] = As[(a + m) * N * N + i + j * N];

  for (int f = tid; f < F; f += PIPE_THREADS)
  {
    const int o = f / S, r = f - (f / S) * S;
    const int base = o * (C * S) + r;
    constexpr bool VEC4 = (sizeof(T) == 4) && (S == 1) && (C % 4 == 0) && (N == 4);
    T v[C];
    if constexpr (VEC4)
    {
#pragma unroll
      for (int c = 0; c < C; c += 4)
      {
        const int e = base + c;
        const float4 u = *reinterpret_cast<const float4 *>(src + (SRC_STAGE ? e : swz<T, N>(e)));
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
      {
        const int e = base + c * S;
        v[c]        = SRC_STAGE ? src[e] : src[swz<T, N>(e)];
      }
    }
    // apply the group's factors, fastest mode (a+k-1) first
#pragma unroll
    for (int m = k - 1; m >= 0; m--)
    {
      constexpr int dummy = 0;
      (void)dummy;
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
      {
        const int e = base + c;
        *reinterpret_cast<float4 *>(dst + (DIRECT ? e : swz<T, N>(e))) =
            make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
      }
    }
    else if constexpr (DIRECT)
    {
      // final pass: plain (unswizzled) layout into the output stage
#pragma unroll
      for (int c = 0; c < C; c++)
        dst[base + c * S] = v[c];
    }
    else
    {
#pragma unroll
      for (int c = 0; c < C; c++)
        dst[swz<T, N>(base + c * S)] = v[c];
    }
  }
}

// Passes in order: group 0, then the last group, then the middle groups.
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
};

template <typename T, int D, int N, int gi>
__device__ __forceinline__ void middle_passes(T *work, const T *As, int tid)
{
  using P = PipePlan<T, D, N>;
  if constexpr (gi < P::ngroup - 1)
  {
    constexpr int a = gi * P::k;
    if constexpr (gi != P::ngroup - 2) // group ngroup-2 is the final pass
    {
      pipe_pass<T, D, N, a, P::k, false, false>(work, work, As, nullptr, 0, tid);
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
  static constexpr int value = sizeof(T) == 4 ? 3 : 2;
};

template <typename T, int D, int N>
__global__ void __launch_bounds__(PIPE_THREADS, PipeOcc<T>::value)
    kron_pipe_kernel(const __grid_constant__ Params p, int nstage)
{
  using Lay = PipeLayout<T, D, N>;
  using P   = PipePlan<T, D, N>;
  constexpr int L   = Lay::L;
  constexpr int ASZ = Lay::ASZ;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem);
  T *work        = reinterpret_cast<T *>(smem + Lay::WORK);
  T *acur        = reinterpret_cast<T *>(smem + Lay::ACUR);
  auto stage_x   = [&](int s) { return reinterpret_cast<T *>(smem + Lay::STAGE0 + s * Lay::STAGE_BYTES); };
  auto stage_a   = [&](int s) { return stage_x(s) + L; };
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

  // issue the copies of position e into stage s (thread 0 only)
  auto issue = [&](int e, int s) {
    EntryRef<T> en;
    entry_fetch<T>(p, entry_index(p, e), D, en);
    const long long xb = (long long)L * sizeof(T);
    const long long ab = (long long)ASZ * sizeof(T);
    const bool a_contig =
        (p.layout == LAYOUT_BATCHED || p.layout == LAYOUT_PBATCHED) && tma_ok<T>(en.A[0], ab);
    const bool x_ok = tma_ok<T>(en.x, xb);
    unsigned bytes  = (x_ok ? (unsigned)xb : 0u) + (a_contig ? (unsigned)ab : 0u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    mbar_expect_tx(&bars[s], bytes);
    if (x_ok)
      tma_load(stage_x(s), en.x, (unsigned)xb, &bars[s]);
    if (a_contig)
      tma_load(stage_a(s), en.A[0], (unsigned)ab, &bars[s]);
    if (tma_ok<T>(en.y, xb))
      l2_prefetch(en.y, (unsigned)xb);
  };

  int ahead = min(nstage, ee - eb);
  if (tid == 0)
    for (int i = 0; i < ahead; i++)
      issue(eb + i, i);
  unsigned phases = 0; // bit s = parity to wait for on stage s
  int pending_e = -1, pending_s = 0; // refill deferred to the next iteration

  for (int e = eb; e < ee; ++e)
  {
    const int s = (e - eb) % nstage;
    EntryRef<T> en;
    entry_fetch<T>(p, entry_index(p, e), D, en);
    // wait for stage s (bounded)
    bool done = false;
    for (long long it = 0; it < SPIN_LIMIT; ++it)
      if (mbar_try_wait(&bars[s], (phases >> s) & 1))
      {
        done = true;
        break;
      }
    if (!__syncthreads_and(done))
    {
      if (tid == 0)
        atomicExch(&g_device_status, 1);
      return;
    }
    phases ^= 1u << s;
    // operands the TMA could not take: plain loads
    const long long xb = (long long)L * sizeof(T);
    const long long ab = (long long)ASZ * sizeof(T);
    T *sx = stage_x(s);
    if (!tma_ok<T>(en.x, xb))
      for (int i = tid; i < L; i += PIPE_THREADS)
        sx[i] = __ldg(en.x + i);
    const bool a_contig =
        (p.layout == LAYOUT_BATCHED || p.layout == LAYOUT_PBATCHED) && tma_ok<T>(en.A[0], ab);
    if (a_contig)
    {
      const T *sa = stage_a(s);
      for (int i = tid; i < ASZ; i += PIPE_THREADS)
        acur[i] = sa[i];
    }
    else
    {
#pragma unroll
      for (int l = 0; l < D; l++)
        for (int ij = tid; ij < N * N; ij += PIPE_THREADS)
        {
          const int j = ij / N, i = ij - j * N;
          acur[l * N * N + ij] = __ldg(en.A[l] + i + (long long)j * en.ld[l]);
        }
    }
    __syncthreads();

    // pass 1: group 0, stage -> work
    pipe_pass<T, D, N, 0, P::k, true, false>(sx, work, acur, nullptr, 0, tid);
    __syncthreads();

    // remaining passes; the last writes the result, unswizzled, into the
    // (now free) stage buffer
    if constexpr (P::ngroup >= 3)
    {
      pipe_pass<T, D, N, P::last_a, P::last_k, false, false>(work, work, acur, nullptr, 0, tid);
      __syncthreads();
      middle_passes<T, D, N, 1>(work, acur, tid);
      pipe_pass<T, D, N, P::final_a, P::final_k, false, true>(work, sx, acur, nullptr, 0, tid);
    }
    else
      pipe_pass<T, D, N, P::last_a, P::last_k, false, true>(work, sx, acur, nullptr, 0, tid);

    // y += result: one bulk reduce-add by the TMA engine when y allows it
    const bool bulk = tma_ok<T>(en.y, xb);
    if (bulk)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (bulk)
    {
      if (tid == 0)
        bulk_reduce_add(en.y, sx, (unsigned)xb);
    }
    else
    {
      constexpr int B = 8;
      for (int i0 = tid; i0 < L; i0 += PIPE_THREADS * B)
      {
        T yv[B];
        if (p.accum != ACC_ATOMIC)
#pragma unroll
          for (int b = 0; b < B; b++)
            if (i0 + b * PIPE_THREADS < L)
              yv[b] = en.y[i0 + b * PIPE_THREADS];
#pragma unroll
        for (int b = 0; b < B; b++)
        {
          const int i = i0 + b * PIPE_THREADS;
          if (i < L)
          {
            if (p.accum == ACC_ATOMIC)
              red_add(en.y + i, sx[i]);
            else
              en.y[i] = yv[b] + sx[i];
          }
        }
      }
      __syncthreads();
    }
    // With three or more stages, refill one iteration late: the previous
    // entry's stage is refilled once its reduce has read it (all bulk groups
    // but this entry's), so no thread waits on the reduce just issued.  With
    // two stages that would leave nothing in flight, so refill at once.
    if (tid == 0)
    {
      if (nstage >= 3)
      {
        if (pending_e >= 0)
        {
          if (bulk)
            bulk_wait_read_but_last();
          else
            bulk_wait_read();
          issue(pending_e, pending_s);
        }
        pending_e = (e + nstage < ee) ? e + nstage : -1;
        pending_s = s;
      }
      else if (e + nstage < ee)
      {
        bulk_wait_read();
        issue(e + nstage, s);
      }
    }
  }
  if (tid == 0)
  {
    if (pending_e >= 0) // nothing left to compute; no refill needed
      pending_e = -1;
    bulk_wait_all();
  }
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
  void *args[]         = {&p, &ns};
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

extern "C" int kron_device_status(int clear)
{
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, kron::g_device_status, sizeof(int)) != cudaSuccess)
    return -1;
  if (clear && v != 0)
  {
    int z = 0;
    cudaMemcpyToSymbol(kron::g_device_status, &z, sizeof(int));
  }
  return v;
}

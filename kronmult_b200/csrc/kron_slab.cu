// Slab-cluster kernel: square d = 6 vectors too large for one block's shared
// memory (n = 6: 373 KB per entry in FP64, 187 KB in FP32), with no
// workspace and no intermediate traffic through L2 or HBM.
//
// One thread-block cluster of n blocks works on one entry at a time.  Block r
// owns slab r of x, the n^5 contiguous elements with i_1 = r, brought into its
// shared memory by one TMA bulk copy.  The six mode products run as three
// register-blocked passes of two modes each.  Every thread takes one fibre of
// n^2 elements per pass and holds one factor at a time in registers:
//   pass A  modes 5, 6: fibres of n^2 contiguous slab elements;
//   pass B  modes 3, 4: fibres (i_3, i_4) at slab strides n^3, n^2;
//   pass C  modes 1, 2: block r takes the n^3 tuples t = (i_3..i_6) in
//           [r n^3, (r+1) n^3) and reads the n^2 elements slab_{i_1}[i_2 n^4 +
//           t] from the cluster's shared memory (ld.shared::cluster).
// Pass C's results are added into y straight from registers by
// fire-and-forget reductions in L2 (red.global.add): y is read and written
// once, in L2, outputs that alias add up, and the adds drain while the block
// goes on with the next entry.
//
// Each block keeps a ring of three stages (x slab + factors): the entry being
// computed, the next one (already landed) and the one after it.  A stage is
// refilled as soon as every block has read it, with the entry three places
// ahead, so every copy has more than an iteration to land.  The cluster
// barriers are split so that independent work fills their latency:
//
//   [pass A(e+1)]  wait1(e)  pass C reads(e)  arrive2(e)
//   [pass C math(e), pass B(e+1)]  wait2(e)  arrive1(e+1)
//   refill stage(e) with e+3;  y += results(e) ...
//
// Barrier 1 of entry e: every block has finished pass B(e), so pass C may
// read.  Barrier 2 of entry e: every block has finished reading the others'
// slabs of e, so the stage can be refilled and no block leaves while another
// still reads it.
//
// Every mbarrier wait is bounded (wait_limit() polls).  A block whose copies
// do not arrive in time does four things:
//   - records 1 in the device status word;
//   - marks itself dead in its shared memory;
//   - stops issuing copies and reduce-adds;
//   - before leaving, lets its outstanding copies land (bounded by
//     drain_limit()).
// The other blocks read the dead marks after barrier 1 and stop writing y
// too.  All blocks still take every cluster barrier.
//
// The product is the reference's (kronmult6_batched.hpp:41-75, computed
// there by kronmultv_recur.hpp:117-145): y += (A_1 x ... x A_6) x, with A_6's
// index fastest.  The six mode products run in a different order, which
// changes rounding only.
#include <algorithm>
#include <cstdint>

#include "kron_launch.h"
#include "kron_ptx.cuh"

namespace kron {

namespace {

using namespace ptx;

// H: blocks per slab.  Block r of the cluster holds part r % H of slab
// r / H: i_1 = r / H and the n / H values of i_2 from (r % H) n / H on,
// n^5 / H contiguous elements of x.
template <typename T, int N, int H>
struct SlabShape
{
  static_assert(N % H == 0, "slabs split evenly");
  static constexpr int CS      = N * H; // blocks per cluster
  static constexpr int N2      = N * N;
  static constexpr int N3      = N2 * N;
  static constexpr int N4      = N3 * N;
  static constexpr int N5      = N4 * N;
  static constexpr int NL      = N / H;  // values of i_2 in a block
  static constexpr int PART    = N5 / H; // elements of x in a block
  static constexpr int FIB     = N3 / H; // fibres of every pass (pass C: tuples)
  static constexpr int THREADS = (FIB + 31) / 32 * 32;
  static constexpr int ASZ     = 6 * N2;
  static constexpr size_t XB   = (size_t)PART * sizeof(T);
  static constexpr size_t AB   = ((size_t)ASZ * sizeof(T) + 15) / 16 * 16;
  static constexpr size_t STAGE_BYTES = (XB + AB + 127) / 128 * 128;
  static constexpr int NS      = 3; // stages: computing, landing, being refilled
  // header: NS mbarriers, this block's dead mark, the cluster's dead mark,
  // per-stage copy flags
  static constexpr size_t OFF_BARS      = 0;
  static constexpr size_t OFF_DEAD      = 8 * NS;
  static constexpr size_t OFF_PEER_DEAD = OFF_DEAD + 4;
  static constexpr size_t OFF_FLAGS     = OFF_PEER_DEAD + 4;
  static constexpr size_t OFF_STAGE0    = 128;
  static constexpr size_t SMEM          = OFF_STAGE0 + NS * STAGE_BYTES;
  static_assert(OFF_FLAGS + 4 * NS <= OFF_STAGE0, "header");
  // blocks per SM that the shared memory allows, and the register cap that
  // lets that many blocks of THREADS threads share the 64K registers
  // (at most three: more blocks would leave too few registers per thread)
  static constexpr int SMEMB  = (228 * 1024) / (int)(SMEM + 1024);
  static constexpr int MINB   = SMEMB < 1 ? 1 : (SMEMB > 3 ? 3 : SMEMB);
  static constexpr int RFIT   = 65536 / (MINB * THREADS) / 8 * 8;
  static constexpr int MAXREG = RFIT > 255 ? 255 : RFIT;
  static constexpr bool XTMA   = XB % 16 == 0;
  static_assert(FIB <= 1024, "one fibre per thread");
};

constexpr int FLAG_X_TMA = 1; // slab arrived by bulk copy
constexpr int FLAG_A_TMA = 2; // A_1..A_6 arrived by bulk copy (contiguous)

// factor A (column major, A(i, j) at i + j N) into registers
template <typename T, int N>
__device__ __forceinline__ void load_factor(const T *A, T (&a)[N][N])
{
#pragma unroll
  for (int j = 0; j < N; j++)
  {
    if constexpr (sizeof(T) == 8 && N % 2 == 0)
    {
#pragma unroll
      for (int i = 0; i < N; i += 2)
      {
        const double2 u = *reinterpret_cast<const double2 *>(A + i + j * N);
        a[i][j]         = u.x;
        a[i + 1][j]     = u.y;
      }
    }
    else if constexpr (sizeof(T) == 4 && N % 2 == 0)
    {
#pragma unroll
      for (int i = 0; i < N; i += 2)
      {
        const float2 u = *reinterpret_cast<const float2 *>(A + i + j * N);
        a[i][j]        = u.x;
        a[i + 1][j]    = u.y;
      }
    }
    else
    {
#pragma unroll
      for (int i = 0; i < N; i++)
        a[i][j] = A[i + j * N];
    }
  }
}

// v is an n x n block, v[a N + b]: apply_fast applies A along b (the faster
// mode), apply_slow along a
template <typename T, int N>
__device__ __forceinline__ void apply_fast(T (&v)[N * N], const T *A)
{
  T a[N][N];
  load_factor<T, N>(A, a);
#pragma unroll
  for (int r = 0; r < N; r++)
  {
    T t[N];
#pragma unroll
    for (int i = 0; i < N; i++)
    {
      T z = a[i][0] * v[r * N];
#pragma unroll
      for (int j = 1; j < N; j++)
        z = fma(a[i][j], v[r * N + j], z);
      t[i] = z;
    }
#pragma unroll
    for (int i = 0; i < N; i++)
      v[r * N + i] = t[i];
  }
}

template <typename T, int N>
__device__ __forceinline__ void apply_slow(T (&v)[N * N], const T *A, int rot = 0)
{
  T a[N][N];
  if (rot == 0)
    load_factor<T, N>(A, a);
  else
  {
    // rows of v hold rows (r + rot) mod N: the factor with rows and columns
    // rotated the same way gives the rotated rows of the product
#pragma unroll
    for (int i = 0; i < N; i++)
#pragma unroll
      for (int j = 0; j < N; j++)
      {
        const int ri = i + rot < N ? i + rot : i + rot - N;
        const int rj = j + rot < N ? j + rot : j + rot - N;
        a[i][j]      = A[ri + rj * N];
      }
  }
#pragma unroll
  for (int c = 0; c < N; c++)
  {
    T t[N];
#pragma unroll
    for (int i = 0; i < N; i++)
    {
      T z = a[i][0] * v[c];
#pragma unroll
      for (int j = 1; j < N; j++)
        z = fma(a[i][j], v[j * N + c], z);
      t[i] = z;
    }
#pragma unroll
    for (int i = 0; i < N; i++)
      v[i * N + c] = t[i];
  }
}

// pass A: modes 5 (A_5, slow) and 6 (A_6, fast) on the contiguous fibre f.
// FP64 fibres of n^2 = 36 elements start 18 16-byte units apart, so lanes f
// and f + 4 of a quarter-warp would hit the same banks on every vector
// access; with `rotate`, lanes with bit 2 set walk their rows starting one
// row later (a 3-unit shift, which makes the eight lanes' units distinct)
// and apply A_5 with rotated indices.
template <typename T, int N>
__device__ __forceinline__ void pass_a(T *slab, const T *As, int f, bool rotate)
{
  constexpr int N2 = N * N;
  constexpr int V  = 16 / sizeof(T);
  T *b             = slab + f * N2;
  // rotation by whole rows keeps the 16-byte units inside rows
  const int rot = (sizeof(T) == 8 && N % 2 == 0 && rotate) ? ((f >> 2) & 1) : 0;
  T v[N2];
  if constexpr ((N2 * sizeof(T)) % 16 == 0)
  {
    // 16-byte aligned fibre: vector loads and stores
#pragma unroll
    for (int c = 0; c < N2; c += V)
    {
      if constexpr (sizeof(T) == 8)
      {
        int src = c + rot * N;
        src     = src < N2 ? src : src - N2;
        const double2 u = *reinterpret_cast<const double2 *>(b + src);
        v[c]            = u.x;
        v[c + 1]        = u.y;
      }
      else
      {
        const float4 u = *reinterpret_cast<const float4 *>(b + c);
        v[c]           = u.x;
        v[c + 1]       = u.y;
        v[c + 2]       = u.z;
        v[c + 3]       = u.w;
      }
    }
  }
  else
  {
#pragma unroll
    for (int c = 0; c < N2; c++)
      v[c] = b[c];
  }
  apply_fast<T, N>(v, As + 5 * N2);
  apply_slow<T, N>(v, As + 4 * N2, rot);
  if constexpr ((N2 * sizeof(T)) % 16 == 0)
  {
#pragma unroll
    for (int c = 0; c < N2; c += V)
    {
      if constexpr (sizeof(T) == 8)
      {
        int dst = c + rot * N;
        dst     = dst < N2 ? dst : dst - N2;
        *reinterpret_cast<double2 *>(b + dst) = make_double2(v[c], v[c + 1]);
      }
      else
        *reinterpret_cast<float4 *>(b + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
    }
  }
  else
  {
#pragma unroll
    for (int c = 0; c < N2; c++)
      b[c] = v[c];
  }
}

// pass B: modes 3 (A_3, slow) and 4 (A_4, fast) on fibre f = (i_2, i_5, i_6)
template <typename T, int N>
__device__ __forceinline__ void pass_b(T *slab, const T *As, int f)
{
  constexpr int N2 = N * N, N3 = N2 * N, N4 = N3 * N;
  const int o = f / N2, r = f - o * N2;
  T *b        = slab + o * N4 + r;
  T v[N2];
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int c = 0; c < N; c++)
      v[a * N + c] = b[a * N3 + c * N2];
  apply_fast<T, N>(v, As + 3 * N2);
  apply_slow<T, N>(v, As + 2 * N2);
#pragma unroll
  for (int a = 0; a < N; a++)
#pragma unroll
    for (int c = 0; c < N; c++)
      b[a * N3 + c * N2] = v[a * N + c];
}

template <typename T, int N, int H>
__global__ void __maxnreg__((SlabShape<T, N, H>::MAXREG))
    kron_slab_kernel(const __grid_constant__ Params p, int *status, long long spin,
                     long long drain, int flags)
{
  using S            = SlabShape<T, N, H>;
  constexpr int CS   = S::CS;
  constexpr int NL   = S::NL, PART = S::PART, FIB = S::FIB;
  constexpr int NS   = S::NS;
  constexpr int N2   = S::N2, N3 = S::N3, N4 = S::N4, N5 = S::N5, ASZ = S::ASZ;
  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + S::OFF_BARS);
  int *dead_mark = reinterpret_cast<int *>(smem + S::OFF_DEAD);
  int *peer_dead = reinterpret_cast<int *>(smem + S::OFF_PEER_DEAD);
  int *sflags    = reinterpret_cast<int *>(smem + S::OFF_FLAGS);
  auto stage_x   = [&](int s) {
    return reinterpret_cast<T *>(smem + S::OFF_STAGE0 + s * S::STAGE_BYTES);
  };
  auto stage_a = [&](int s) {
    return reinterpret_cast<T *>(smem + S::OFF_STAGE0 + s * S::STAGE_BYTES + S::XB);
  };
  const int tid     = threadIdx.x;
  const int rank    = (int)cluster_ctarank();
  const bool rotate = !(flags & KRON_SLAB_NO_ROTATE);
  const bool atomic_y = p.accum != ACC_DISTINCT || !(flags & KRON_SLAB_PLAIN_Y);
  // this thread's n^2 elements of position e's y into L2
  auto prefetch_y = [&](const T *yt) {
#pragma unroll
    for (int q = 0; q < N2; q++)
    {
      const int a = q / N, c = q - a * N;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(yt + (long long)a * N5 + (long long)c * N4));
    }
  };
  const int cid     = blockIdx.x / CS;
  const int ncl     = gridDim.x / CS;
  const long long tot = p.eend - p.ebase;
  const int eb = p.ebase + (int)(tot * cid / ncl);
  const int ee = p.ebase + (int)(tot * (cid + 1) / ncl);
  if (eb >= ee)
    return; // the whole cluster leaves together

  if (tid == 0)
  {
    for (int s = 0; s < NS; s++)
      mbar_init(&bars[s], 1);
    *dead_mark = 0;
    *peer_dead = 0;
    fence_mbar_init();
  }
  __syncthreads();
  // every block of the cluster is running before any shared::cluster access
  cluster_sync();

  unsigned inflight = 0; // thread 0: stages whose copies were not waited for
  unsigned phase    = 0; // bit s: parity of stage s's next completion
  bool dead         = false;

  // thread 0: start the copies of position e into stage s
  auto issue = [&](int e, int s) {
    EntryRef<T> en;
    entry_fetch<T>(p, entry_index(p, e), 6, en);
    const T *xs      = en.x + (long long)rank * PART;
    const bool x_tma = S::XTMA && aligned16(xs);
    const bool a_tma = (p.layout == LAYOUT_BATCHED || p.layout == LAYOUT_PBATCHED) &&
                       (ASZ * sizeof(T)) % 16 == 0 && aligned16(en.A[0]);
    sflags[s] = (x_tma ? FLAG_X_TMA : 0) | (a_tma ? FLAG_A_TMA : 0);
    fence_proxy_async();
    const unsigned bytes =
        (x_tma ? (unsigned)S::XB : 0u) + (a_tma ? (unsigned)(ASZ * sizeof(T)) : 0u);
    mbar_expect_tx(&bars[s], bytes);
    if (x_tma)
      tma_load_1d(stage_x(s), xs, (unsigned)S::XB, &bars[s]);
    if (a_tma)
      tma_load_1d(stage_a(s), en.A[0], (unsigned)(ASZ * sizeof(T)), &bars[s]);
    inflight |= 1u << s;
  };

  // every thread: wait for stage s (position e) and load what its copies did
  // not carry; a time-out makes the block dead
  auto acquire = [&](int e, int s) {
    bool ok = true;
    if (!dead)
    {
      ok = mbar_wait_bounded(&bars[s], (phase >> s) & 1, spin);
      if (ok)
      {
        phase ^= 1u << s;
        if (tid == 0)
          inflight &= ~(1u << s);
        const int fl = sflags[s];
        if ((fl & (FLAG_X_TMA | FLAG_A_TMA)) != (FLAG_X_TMA | FLAG_A_TMA))
        {
          EntryRef<T> en;
          entry_fetch<T>(p, entry_index(p, e), 6, en);
          if (!(fl & FLAG_X_TMA))
          {
            const T *xs = en.x + (long long)rank * PART;
            T *sx       = stage_x(s);
            for (int i = tid; i < PART; i += blockDim.x)
              sx[i] = xs[i];
          }
          if (!(fl & FLAG_A_TMA))
          {
            T *sa = stage_a(s);
            for (int q = tid; q < ASZ; q += blockDim.x)
            {
              const int l = q / N2, ij = q - l * N2;
              const int j = ij / N, i = ij - j * N;
              sa[q]       = en.A[l][i + (long long)j * en.ld[l]];
            }
          }
        }
      }
    }
    if (!__syncthreads_and(ok) && !dead)
    {
      dead = true;
      if (tid == 0)
      {
        if (status)
          atomicExch(status, 1);
        *dead_mark = 1;
      }
    }
  };

  if (tid == 0)
    for (int k = 0; k < NS && eb + k < ee; k++)
      issue(eb + k, k);

  if (!atomic_y && tid < FIB)
    prefetch_y(entry_y<T>(p, entry_index(p, eb)) + (long long)rank * FIB + tid);
  // passes A and B of the first position
  acquire(eb, 0);
  if (tid < FIB)
    pass_a<T, N>(stage_x(0), stage_a(0), tid, rotate);
  __syncthreads();
  if (tid < FIB)
    pass_b<T, N>(stage_x(0), stage_a(0), tid);
  cluster_arrive(); // barrier 1 (eb)

  const unsigned dead_addr = smem_addr(dead_mark);
  for (int e = eb; e < ee; ++e)
  {
    const int i     = e - eb;
    const int s     = i % NS;
    const int s1    = (i + 1) % NS;
    const bool more = e + 1 < ee;
    // pass A of the next position while barrier 1 settles
    if (more)
    {
      acquire(e + 1, s1);
      if (tid < FIB)
        pass_a<T, N>(stage_x(s1), stage_a(s1), tid, rotate);
    }
    cluster_wait(); // barrier 1 (e): every block finished pass B(e)
    if (tid == 0)
    {
      int any = 0;
#pragma unroll
      for (int a = 0; a < CS; a++)
        any |= ld_cluster_s32(mapa(dead_addr, (unsigned)a));
      *peer_dead = any;
    }
    // pass C: tuple t of every slab of the cluster
    T v[N2];
    const unsigned sbase = smem_addr(stage_x(s));
    const int t          = rank * FIB + tid;
    if (tid < FIB)
    {
      // element (i_1 = a, i_2 = c, t) is in block a H + c / NL, at
      // (c mod NL) n^4 + t of its part
#pragma unroll
      for (int a = 0; a < N; a++)
#pragma unroll
        for (int h = 0; h < H; h++)
        {
          const unsigned base = mapa(sbase, (unsigned)(a * H + h));
#pragma unroll
          for (int cl = 0; cl < NL; cl++)
            v[a * N + h * NL + cl] =
                ld_cluster<T>(base + (unsigned)((cl * N4 + t) * sizeof(T)));
        }
    }
    cluster_arrive(); // barrier 2 (e): this block's reads of the slabs are done
    if (tid < FIB)
    {
      apply_fast<T, N>(v, stage_a(s) + 1 * N2);
      apply_slow<T, N>(v, stage_a(s) + 0 * N2);
    }
    // this thread is done with stage s (pass B wrote it, pass C read it and
    // its factors): its generic accesses come before the copy that refills it
    fence_proxy_async();
    __syncthreads(); // pass A(e+1) done block-wide; the dead marks are in
    dead = dead || (*peer_dead != 0);
    if (more && tid < FIB)
      pass_b<T, N>(stage_x(s1), stage_a(s1), tid);
    T *y = entry_y<T>(p, entry_index(p, e)) + (long long)rank * FIB;
    cluster_wait(); // barrier 2 (e): no block reads this block's stage s any more
    if (more)
      cluster_arrive(); // barrier 1 (e+1): pass B(e+1) is done
    // stage s is free: it takes position e + 3, more than an iteration ahead
    if (tid == 0 && !dead && e + NS < ee)
      issue(e + NS, s);
    // y += results: fire-and-forget adds in L2 (outputs that alias add up).
    // With KRON_SLAB_PLAIN_Y, distinct outputs take plain loads (the lines
    // were prefetched into L2 an iteration ago) and stores instead; measured
    // slower on B200 (1.62 against 1.53 ms for 4096 entries), so the adds
    // are the default
    if (!dead && tid < FIB)
    {
      if (atomic_y)
      {
#pragma unroll
        for (int q = 0; q < N2; q++)
        {
          const int a = q / N, c = q - a * N;
          red_add(y + (long long)a * N5 + (long long)c * N4 + tid, v[q]);
        }
      }
      else
      {
        T yv[N2];
#pragma unroll
        for (int q = 0; q < N2; q++)
        {
          const int a = q / N, c = q - a * N;
          yv[q]       = y[(long long)a * N5 + (long long)c * N4 + tid];
        }
#pragma unroll
        for (int q = 0; q < N2; q++)
        {
          const int a = q / N, c = q - a * N;
          y[(long long)a * N5 + (long long)c * N4 + tid] = yv[q] + v[q];
        }
      }
    }
    if (!atomic_y && !dead && more && tid < FIB)
      prefetch_y(entry_y<T>(p, entry_index(p, e + 1)) + (long long)rank * FIB + tid);
  }

  if (tid == 0 && dead)
    for (int s = 0; s < NS; s++)
      if ((inflight >> s) & 1)
        mbar_wait_bounded(&bars[s], (phase >> s) & 1, drain);
}

// Launch configuration of the slab kernel and the clusters the device runs
// at once (ncl), with the blocks each SM holds (per_sm).
template <typename T, int N, int H>
int slab_config_t(cudaLaunchConfig_t &cfg, cudaLaunchAttribute *attr, int &ncl, int &per_sm)
{
  using S        = SlabShape<T, N, H>;
  const void *fn = reinterpret_cast<const void *>(&kron_slab_kernel<T, N, H>);
  if (S::SMEM > (size_t)device_info().max_smem_optin)
    return KRON_ERROR_NOT_SUPPORTED;
  per_sm = 1;
  if (cached_occupancy(fn, S::THREADS, S::SMEM, &per_sm) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  if (S::CS > 8)
  {
    // clusters above the portable 8 blocks (B200 runs up to 16); set once
    // per device
    static bool nonportable_set[64] = {};
    const int dev = device_info().device;
    if (dev < 0 || dev >= 64)
      return KRON_ERROR_NOT_SUPPORTED;
    if (!nonportable_set[dev])
    {
      if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
          cudaSuccess)
      {
        cudaGetLastError();
        return KRON_ERROR_NOT_SUPPORTED;
      }
      nonportable_set[dev] = true;
    }
  }
  cfg                      = cudaLaunchConfig_t{};
  attr[0].id               = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = S::CS;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim             = dim3(S::THREADS);
  cfg.dynamicSmemBytes     = S::SMEM;
  cfg.attrs                = attr;
  cfg.numAttrs             = 1;
  cfg.gridDim              = dim3((device_info().sms / S::CS) * S::CS);
  ncl                      = 0;
  if (cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg) != cudaSuccess || ncl < 1)
  {
    cudaGetLastError();
    return KRON_ERROR_NOT_SUPPORTED;
  }
  return KRON_SUCCESS;
}

template <typename T, int N, int H>
int launch_slab_t(Params p, int flags, cudaStream_t stream)
{
  const void *fn = reinterpret_cast<const void *>(&kron_slab_kernel<T, N, H>);
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  int ncl = 0, per_sm = 1;
  const int rc = slab_config_t<T, N, H>(cfg, attr, ncl, per_sm);
  if (rc != KRON_SUCCESS)
    return rc;
  using S      = SlabShape<T, N, H>;
  ncl          = (int)std::min<long long>((long long)ncl, p.eend - p.ebase);
  cfg.gridDim  = dim3(ncl * S::CS);
  cfg.stream   = stream;
  int *status  = device_status_ptr();
  long long sp = wait_limit();
  long long dr = drain_limit();
  void *args[] = {&p, &status, &sp, &dr, &flags};
  return cudaLaunchKernelExC(&cfg, fn, args) == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

template <typename T, int N, int H>
int slab_sms_t(int &used)
{
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute attr[1];
  int ncl = 0, per_sm = 1;
  const int rc = slab_config_t<T, N, H>(cfg, attr, ncl, per_sm);
  if (rc != KRON_SUCCESS)
    return rc;
  using S = SlabShape<T, N, H>;
  used    = std::min(device_info().sms, (ncl * S::CS + per_sm - 1) / std::max(1, per_sm));
  return KRON_SUCCESS;
}

} // namespace

bool slab_supported(const Params &p, int prec)
{
  if ((prec != PREC_F64 && prec != PREC_F32) || p.seg_off ||
      (p.accum != ACC_DISTINCT && p.accum != ACC_ATOMIC) || p.d != 6)
    return false;
  const int n = p.n[0];
  for (int l = 0; l < p.d; l++)
    if (p.m[l] != n || p.n[l] != n)
      return false;
  return n == 6;
}

int slab_sms_used(int n, int prec, int flags, int *used)
{
  *used = 0;
  if (n != 6)
    return KRON_ERROR_NOT_SUPPORTED;
  if (flags & KRON_SLAB_WHOLE)
    return prec == PREC_F32 ? slab_sms_t<float, 6, 1>(*used) : slab_sms_t<double, 6, 1>(*used);
  return prec == PREC_F32 ? slab_sms_t<float, 6, 2>(*used) : slab_sms_t<double, 6, 2>(*used);
}

int launch_slab(Params p, int prec, int flags, cudaStream_t stream)
{
  if (p.eend <= p.ebase)
    return KRON_SUCCESS;
  if (p.n[0] == 6)
  {
    // half slabs (clusters of 12, two or four blocks per SM) by default;
    // whole slabs (clusters of 6) on request
    if (flags & KRON_SLAB_WHOLE)
      return prec == PREC_F32 ? launch_slab_t<float, 6, 1>(p, flags, stream)
                              : launch_slab_t<double, 6, 1>(p, flags, stream);
    return prec == PREC_F32 ? launch_slab_t<float, 6, 2>(p, flags, stream)
                            : launch_slab_t<double, 6, 2>(p, flags, stream);
  }
  return KRON_ERROR_NOT_SUPPORTED;
}

} // namespace kron

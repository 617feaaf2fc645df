// Split-precision d = 6, n = 8 on the 5th-generation tensor cores (tcgen05,
// BF16 operands, FP32 accumulators in tensor memory), FP64 data.
//
// The product runs as the two-level split of the recursive algorithm
// (kronmultv_recur.hpp:117-145): phase 1 applies the tail modes 4..6 to every
// head row of x (512 contiguous elements) and writes W; phase 2 applies the
// head modes 1..3 to every column of W and adds into y.  Both phases work on
// tiles of two 8x8x8 blocks (1024 elements) that share their three factors.
// One mode product over a tile is a GEMM of 128 fibres (M) by the mode's 8
// outputs, contracting 8 elements -- done on the tensor cores exactly, in
// slices:
//   - every fibre r is scaled by its own power of two 2^E_r (max |x| < 2^E_r)
//     and cut into six signed 8-bit integer slices, x = 2^E_r sum_s X_s
//     2^-8(s+1); every row i of the factor likewise, with 2^F_i;
//   - an integer of at most 8 significant bits is exact in BF16, a product of
//     two is exact in FP32, and every accumulator collects only products of
//     one weight w = s_x + s_a (at most 48 integers below 2^17): the FP32 sums
//     are exact, whatever the order the tensor core adds in;
//   - one tcgen05.mma per X slice s_x (M = 128, K = 16 with the upper half
//     zero, N = the factor slices 0 .. 5 - s_x rounded up to 16 rows) adds
//     X_sx * A_sa^T into accumulator columns 8 (s_x + s_a) + i, so column
//     block w holds D_w[r, i] = sum_{s_x + s_a = w} sum_k X_sx[r,k] A_sa[i,k]
//     (weights w > 5, which the truncated triangle drops, land in columns
//     48..55 and are ignored);
//   - y[r, i] = 2^(E_r + F_i) sum_w 2^-8(w+2) D_w[r, i], summed in FP64.
// The dropped weights and the slices' truncation leave a relative error near
// 2^-48 per mode product.  Operands sit in shared memory in the K-major
// layout without swizzle (core matrices of 8 rows x 16 bytes); one thread
// issues the MMAs and a tcgen05.commit arrives on an mbarrier; each warp then
// reads its 32 accumulator lanes with tcgen05.ld.
//
// Every mbarrier wait is bounded (wait_limit() polls).  On a time-out the
// block records 1 in the device status word, waits (bounded by
// drain_limit()) for the MMAs it issued, frees its tensor memory and leaves.
#include <algorithm>
#include <cstdint>

#include "kron_launch.h"
#include "kron_ptx.cuh"

namespace kron {

namespace {

using namespace ptx;

constexpr int TC_THREADS = 128; // warp w reads accumulator lanes 32w .. 32w + 31
// Blocks per SM.  The runtime's occupancy query answers 1 for kernels that
// allocate tensor memory, but five blocks fit: 5 x 64 of the SM's 512
// tensor-memory columns, 5 x 37.5 KB of shared memory, 5 x 128 x 96
// registers.  Measured for 256 entries: 9.65 ms at one block per SM, 3.77 ms
// at four, 3.57 ms at five.  The kernels keep the register budget of four
// blocks (__launch_bounds__ 128 x 4: 92 registers, 96 allocated, so five
// blocks still fit); compiled for five (80 registers) they ran at 4.66 ms.
constexpr int TC_BLOCKS  = 5;
constexpr int NSL        = 6;   // 8-bit slices per operand
constexpr int TMEM_COLS  = 64;  // accumulator columns (56 written)
constexpr int TILE       = 1024;
constexpr int BLK        = 512; // 8 x 8 x 8
constexpr int ITEMS      = 256; // tiles per entry and phase (2^18 / 1024)

// shared memory (bytes)
constexpr int XS_BYTES  = 128 * 32;            // one X slice: 16 row groups x 256 B
constexpr int OFF_XS    = 0;                   // NSL X slices
constexpr int FS_BYTES  = NSL * 8 * 32;        // one factor's slices: 48 rows = 6 groups x 256 B
constexpr int OFF_FS    = OFF_XS + NSL * XS_BYTES;
constexpr int OFF_BUF   = OFF_FS + 3 * FS_BYTES;
constexpr int OFF_FEXP  = OFF_BUF + TILE * 8;  // int F_i, 3 factors x 8 rows
constexpr int OFF_BAR   = OFF_FEXP + 3 * 8 * 4;
constexpr int OFF_TSLOT = OFF_BAR + 8;
constexpr int SMEM      = OFF_TSLOT + 8;
static_assert(OFF_BAR % 8 == 0 && OFF_BUF % 16 == 0 && OFF_FS % 256 == 0, "alignment");

// shared-memory matrix descriptor: K-major, no swizzle, the two 16-byte K
// chunks of a core matrix 128 B apart (leading byte offset), 8-row groups
// 256 B apart (stride byte offset), descriptor version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr)
{
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128 >> 4) << 16) |
         ((uint64_t)(256 >> 4) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> F32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) |
         ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, int accum)
{
  asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
               "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accum)
               : "memory");
}

__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

// 16 accumulator columns of this thread's lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
  uint32_t r[16];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, "
               "%10, %11, %12, %13, %14, %15}, [%16];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
               : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; j++)
    v[j] = __uint_as_float(r[j]);
}

__device__ __forceinline__ void tc_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// The conversions below stay off the XU pipe (which a first version, with
// rint and FP64 <-> FP32 casts, kept 52% busy): rounding by adding and
// subtracting 1.5 * 2^52, BF16 bits and FP64 values put together from the
// operands' bit fields with integer operations.

// nearest integer (ties to even) of |v| < 2^51 by two FP64 adds
__device__ __forceinline__ double round_int(double v)
{
  return __dadd_rn(__dadd_rn(v, 6755399441055744.0), -6755399441055744.0);
}

// BF16 bits of an integer-valued q with |q| <= 256, from q's FP64 fields:
// the exponent rebiased from 1023 to 127, the mantissa's top 7 bits (exact:
// q has at most 8 significant bits); zero of either sign gives +0
__device__ __forceinline__ uint32_t bf16_bits(double q)
{
  const uint32_t h = (uint32_t)__double2hiint(q);
  const uint32_t b = (((h >> 13) & 0x3FFFFu) - (896u << 7)) | ((h >> 16) & 0x8000u);
  return (h & 0x7FFFFFFFu) ? b : 0u;
}

// FP64 value of an integer-valued FP32 d with |d| < 2^22: the integer
// through the FP32 add of 1.5 * 2^23, then the FP64 subtraction of
// 2^52 + 2^31 from the double whose low word is that integer + 2^31
__device__ __forceinline__ double int_float_to_double(float d)
{
  const int i = __float_as_int(__fadd_rn(d, 12582912.0f)) - 0x4B400000;
  return __dsub_rn(__hiloint2double(0x43300000, i ^ (int)0x80000000), 4503601774854144.0);
}

// 2^e for -1000 < e < 1000 from its bit fields (no ldexp)
__device__ __forceinline__ double pow2(int e) { return __hiloint2double((1023 + e) << 20, 0); }

// Cut v[0..7] (one fibre or one factor row) into NSL slices after scaling by
// 2^-E; writes slice s's eight BF16 values as 16 bytes at dst + s * sstride.
// Returns E.
__device__ __forceinline__ int slice8(const double (&v)[8], unsigned char *dst, int sstride)
{
  double mx = 0.0;
#pragma unroll
  for (int k = 0; k < 8; k++)
    mx = fmax(mx, fabs(v[k]));
  // mx = m 2^E with m in [0.5, 1): E from the exponent field when mx is
  // normal, frexp otherwise
  int E = 0;
  if (mx > 0.0)
  {
    const int ex = (__double2hiint(mx) >> 20) & 0x7FF;
    if (ex > 0 && ex < 0x7FF)
      E = ex - 1022;
    else
      frexp(mx, &E);
  }
  const bool fast = E > -1000 && E < 1000;
  const double sc = fast ? pow2(-E) : 0.0;
  double u[8];
#pragma unroll
  for (int k = 0; k < 8; k++)
    u[k] = fast ? v[k] * sc : ldexp(v[k], -E); // |u| < 1, exact
#pragma unroll
  for (int s = 0; s < NSL; s++)
  {
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 8; k += 2)
    {
      const double q0 = round_int(u[k] * 256.0), q1 = round_int(u[k + 1] * 256.0);
      u[k]            = u[k] * 256.0 - q0; // exact
      u[k + 1]        = u[k + 1] * 256.0 - q1;
      w[k / 2]        = bf16_bits(q0) | (bf16_bits(q1) << 16);
    }
    *reinterpret_cast<uint4 *>(dst + s * sstride) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  return E;
}

// Byte offset of row r of a K-major operand (K 0..7 chunk).
__device__ __forceinline__ int row_off(int r) { return (r & 7) * 16 + (r >> 3) * 256; }

struct TcState
{
  uint32_t tmem;   // accumulator base (lane 0, column 0)
  unsigned phase;  // parity of the mbarrier's next completion
  bool dead;
};

// Three mode products on the tile buf[2][8][8][8] (last index fastest) with
// factor slices FS[0] (slowest mode) .. FS[2] (fastest mode).  false when a
// wait timed out (the block must stop).
__device__ bool tile_modes(unsigned char *smem, double *buf, TcState &st, long long spin)
{
  const int t = threadIdx.x, warp = t >> 5;
  const int blk = t >> 6, a = (t >> 3) & 7, b = t & 7;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem + OFF_BAR);
  const int *fexp = reinterpret_cast<const int *>(smem + OFF_FEXP);
  const uint32_t xs0 = smem_addr(smem + OFF_XS);
  const uint32_t fs0 = smem_addr(smem + OFF_FS);
#pragma unroll 1
  for (int f = 2; f >= 0; --f)
  {
    // fibre t of this mode: contract index k at stride 1 (f = 2), 8, 64
    const int stride = f == 2 ? 1 : (f == 1 ? 8 : 64);
    const int base   = blk * BLK + (f == 2 ? a * 64 + b * 8 : (f == 1 ? a * 64 + b : a * 8 + b));
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; k++)
      v[k] = buf[base + k * stride];
    const int E = slice8(v, smem + OFF_XS + row_off(t), XS_BYTES);
    fence_async_smem();
    __syncthreads();
    if (t == 0)
    {
      tc_fence_after();
#pragma unroll
      for (int sx = 0; sx < NSL; sx++)
      {
        const int nrow = ((8 * (NSL - sx)) + 15) / 16 * 16;
        tc_mma(st.tmem + 8 * sx, smem_desc(xs0 + sx * XS_BYTES), smem_desc(fs0 + f * FS_BYTES),
               idesc_bf16(128, nrow), sx > 0);
      }
      tc_commit(bar);
    }
    const bool ok = mbar_wait_bounded(bar, st.phase, spin);
    if (!__syncthreads_and(ok))
      return false;
    st.phase ^= 1u;
    tc_fence_after();
    float D[48];
    {
      const uint32_t ta = st.tmem + ((uint32_t)(32 * warp) << 16);
      float c0[16], c1[16], c2[16];
      tc_ld16(ta, c0);
      tc_ld16(ta + 16, c1);
      tc_ld16(ta + 32, c2);
      tc_wait_ld();
#pragma unroll
      for (int j = 0; j < 16; j++)
      {
        D[j]      = c0[j];
        D[16 + j] = c1[j];
        D[32 + j] = c2[j];
      }
    }
#pragma unroll
    for (int i = 0; i < 8; i++)
    {
      double acc = int_float_to_double(D[8 * (NSL - 1) + i]);
#pragma unroll
      for (int w = NSL - 2; w >= 0; --w)
        acc = fma(acc, 0.00390625, int_float_to_double(D[8 * w + i])); // 2^-8
      const int e = E + fexp[f * 8 + i] - 16;
      buf[base + i * stride] = (e > -1000 && e < 1000) ? acc * pow2(e) : ldexp(acc, e);
    }
    // accumulator reads done before the next MMAs overwrite it; the tile's
    // outputs in place before the next mode reads other fibres
    tc_fence_before();
    __syncthreads();
  }
  return true;
}

// Factor slices of A_l (column major, leading dimension ld) for l = l0 ..
// l0 + 2: threads 0..23, one factor row each
__device__ __forceinline__ void build_factors(unsigned char *smem, const EntryRef<double> &en,
                                              int l0)
{
  const int t = threadIdx.x;
  if (t < 24)
  {
    const int f = t >> 3, i = t & 7;
    const double *A = en.A[l0 + f];
    const long long ld = en.ld[l0 + f];
    double v[8];
#pragma unroll
    for (int k = 0; k < 8; k++)
      v[k] = A[i + k * ld];
    // row (s, i) of factor f: group s, row i of the group
    const int E = slice8(v, smem + OFF_FS + f * FS_BYTES + i * 16, 256);
    reinterpret_cast<int *>(smem + OFF_FEXP)[f * 8 + i] = E;
  }
}

__device__ __forceinline__ void tc_setup(unsigned char *smem, TcState &st)
{
  const int t = threadIdx.x;
  // the upper K halves (K = 8..15) of every operand row stay zero
  for (int q = t; q < (NSL * XS_BYTES + 3 * FS_BYTES) / 256; q += TC_THREADS)
  {
    uint4 *z = reinterpret_cast<uint4 *>(smem + q * 256 + 128);
#pragma unroll
    for (int j = 0; j < 8; j++)
      z[j] = make_uint4(0, 0, 0, 0);
  }
  if (t == 0)
  {
    mbar_init(reinterpret_cast<uint64_t *>(smem + OFF_BAR), 1);
    fence_mbar_init();
  }
  if (t < 32)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(smem + OFF_TSLOT)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  fence_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  st.tmem  = *reinterpret_cast<volatile uint32_t *>(smem + OFF_TSLOT);
  st.phase = 0;
  st.dead  = false;
}

__device__ __forceinline__ void tc_teardown(unsigned char *smem, TcState &st, int *status,
                                            long long drain)
{
  if (st.dead)
  {
    // the MMAs of the timed-out wait may still run: let them finish first
    if (threadIdx.x == 0)
    {
      if (status)
        atomicExch(status, 1);
      mbar_wait_bounded(reinterpret_cast<uint64_t *>(smem + OFF_BAR), st.phase, drain);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32)
  {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(st.tmem),
                 "r"(TMEM_COLS)
                 : "memory");
  }
}

// this block's contiguous range of the launch's items (position, tile)
__device__ __forceinline__ void item_range(const Params &p, long long &ib, long long &ie)
{
  const long long tot = (long long)(p.eend - p.ebase) * ITEMS;
  ib = tot * blockIdx.x / gridDim.x;
  ie = tot * (blockIdx.x + 1) / gridDim.x;
}

// phase 1: tail modes 4..6 on head rows 2q, 2q + 1 of x -> W
__global__ void __launch_bounds__(TC_THREADS, 4)
    kron_splittc_rows_kernel(const __grid_constant__ Params p, double *W, long long wstride,
                             int *status, long long spin, long long drain)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  double *buf = reinterpret_cast<double *>(smem + OFF_BUF);
  TcState st;
  tc_setup(smem, st);
  long long ib, ie;
  item_range(p, ib, ie);
  int cur = -1;
  EntryRef<double> en;
  for (long long it = ib; it < ie && !st.dead; ++it)
  {
    const int e = p.ebase + (int)(it / ITEMS), q = (int)(it % ITEMS);
    if (e != cur)
    {
      entry_fetch<double>(p, entry_index(p, e), 6, en);
      build_factors(smem, en, 3);
      cur = e;
    }
    const double *x = en.x + (long long)q * TILE;
    for (int j = threadIdx.x; j < TILE / 2; j += TC_THREADS)
    {
      const double2 u = reinterpret_cast<const double2 *>(x)[j];
      buf[2 * j]      = u.x;
      buf[2 * j + 1]  = u.y;
    }
    __syncthreads();
    if (!tile_modes(smem, buf, st, spin))
    {
      st.dead = true;
      break;
    }
    double *w = W + (long long)(e - p.ebase) * wstride + (long long)q * TILE;
    for (int j = threadIdx.x; j < TILE / 2; j += TC_THREADS)
      reinterpret_cast<double2 *>(w)[j] = make_double2(buf[2 * j], buf[2 * j + 1]);
    __syncthreads();
  }
  tc_teardown(smem, st, status, drain);
}

// phase 2: head modes 1..3 on columns 2q, 2q + 1 of W (stride 512) -> y +=
__global__ void __launch_bounds__(TC_THREADS, 4)
    kron_splittc_cols_kernel(const __grid_constant__ Params p, const double *W,
                             long long wstride, int *status, long long spin, long long drain)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  double *buf = reinterpret_cast<double *>(smem + OFF_BUF);
  TcState st;
  tc_setup(smem, st);
  long long ib, ie;
  item_range(p, ib, ie);
  int cur = -1;
  EntryRef<double> en;
  for (long long it = ib; it < ie && !st.dead; ++it)
  {
    const int e = p.ebase + (int)(it / ITEMS), q = (int)(it % ITEMS);
    if (e != cur)
    {
      entry_fetch<double>(p, entry_index(p, e), 6, en);
      build_factors(smem, en, 0);
      cur = e;
    }
    const double *w = W + (long long)(e - p.ebase) * wstride + 2 * q;
    for (int h = threadIdx.x; h < BLK; h += TC_THREADS)
    {
      const double2 u = *reinterpret_cast<const double2 *>(w + (long long)h * BLK);
      buf[h]          = u.x;
      buf[BLK + h]    = u.y;
    }
    __syncthreads();
    if (!tile_modes(smem, buf, st, spin))
    {
      st.dead = true;
      break;
    }
    double *y = en.y + 2 * q;
    for (int h = threadIdx.x; h < BLK; h += TC_THREADS)
    {
      red_add(y + (long long)h * BLK, buf[h]);
      red_add(y + (long long)h * BLK + 1, buf[BLK + h]);
    }
    __syncthreads();
  }
  tc_teardown(smem, st, status, drain);
}

} // namespace

bool splittc_supported(const Params &p, int prec)
{
  if (prec != PREC_SPLIT || p.d != 6 || p.layout != LAYOUT_BATCHED || p.seg_off ||
      (p.accum != ACC_DISTINCT && p.accum != ACC_ATOMIC))
    return false;
  for (int l = 0; l < 6; l++)
    if (p.m[l] != 8 || p.n[l] != 8)
      return false;
  return true;
}

int launch_splittc(Params p, const Workspace &ws, cudaStream_t stream)
{
  if (p.eend <= p.ebase)
    return KRON_SUCCESS;
  constexpr long long L = 1LL << 18;
  if (!ws.W || ws.wstride < L || (ws.wstride % 2) != 0)
    return KRON_ERROR_WORKSPACE;
  // tiles are read and written as 16-byte pairs
  if ((reinterpret_cast<uintptr_t>(p.X) | reinterpret_cast<uintptr_t>(p.Y) |
       reinterpret_cast<uintptr_t>(ws.W)) & 15 ||
      (p.xstride | p.ystride) & 1)
    return KRON_ERROR_NOT_SUPPORTED;
  const void *f1 = reinterpret_cast<const void *>(&kron_splittc_rows_kernel);
  const void *f2 = reinterpret_cast<const void *>(&kron_splittc_cols_kernel);
  int unused = 1; // sets the kernels' shared-memory limit once
  if (cached_occupancy(f1, TC_THREADS, SMEM, &unused) != KRON_SUCCESS ||
      cached_occupancy(f2, TC_THREADS, SMEM, &unused) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  const long long work = (long long)(p.eend - p.ebase) * ITEMS;
  const unsigned grid =
      (unsigned)std::min<long long>(work, (long long)device_info().sms * TC_BLOCKS);
  double *W            = static_cast<double *>(ws.W);
  long long wstride    = ws.wstride;
  int *status          = device_status_ptr();
  long long spin = wait_limit(), drain = drain_limit();
  void *a1[] = {&p, &W, &wstride, &status, &spin, &drain};
  if (cudaLaunchKernel(f1, dim3(grid), dim3(TC_THREADS), a1, SMEM, stream) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  const double *Wc = W;
  void *a2[]       = {&p, &Wc, &wstride, &status, &spin, &drain};
  if (cudaLaunchKernel(f2, dim3(grid), dim3(TC_THREADS), a2, SMEM, stream) != cudaSuccess)
    return KRON_ERROR_LAUNCH;
  return KRON_SUCCESS;
}

} // namespace kron

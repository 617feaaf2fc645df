// FP64 tensor-core kernel for square 8x8 factors, d = 3 (512-element vectors).
//
// One warp owns one entry at a time; the entry's vector never leaves the
// warp's registers except for one 4 KB transpose through shared memory.
// The three mode products of kronmultv_recur.hpp / kronm_forward.hpp are
// 8x8-by-8x64 GEMMs done with mma.sync f64 (the sm_100a FP64 tensor path):
//
//   X[j0][j1][j2] (j2 fastest) is held as a warp tile (G, P, Q):
//   lane (g = lane/4, t = lane%4) holds G-index g, P-index pair {2t, 2t+1},
//   and 8 Q-tiles in registers.
//
//   load      : (G=j1, P=j2, Q=j0)       16-byte loads, coalesced
//   mode 3    : m8n8k4, A_3 as the A operand, data as B      -> (G=i2, P=j1, Q=j0)
//   mode 2    : m16n8k8, data as A operand, A_2^T as B        -> (G=i2, P=i1, Q=j0)
//   transpose : P <-> Q inside each quad via shared memory     -> (G=i2, P=j0, Q=i1)
//   mode 1    : m16n8k8, accumulating into the output-group sum -> (G=i2, P=i0, Q=i1)
//
// The accumulator layout of one MMA is reused as the next MMA's operand
// layout; the K index order this implies (k = t holds column 2t, k = t+4
// column 2t+1) is absorbed by permuting the rows of the constant A_l^T
// fragments, so no data moves between modes except the one transpose.
// Consecutive entries with the same output pointer are summed in the MMA
// accumulators and written once (atomic red.global.add, or a plain
// read-modify-write when outputs are exclusive / segmented).
#include <cstdint>

#include "kron_launch.h"

namespace kron {

namespace {

constexpr int WARPS = 8;                  // warps per block
constexpr int XBUF  = 512;                // doubles per X staging buffer
constexpr int SWBUF = 512;                // doubles per transpose buffer
constexpr int WARP_SMEM = 2 * XBUF + SWBUF; // doubles per warp (12 KB)

__device__ __forceinline__ void mma884(double &d0, double &d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void mma1688(double &c0, double &c1, double &c2, double &c3, double a0,
                                        double a1, double a2, double a3, double b0, double b1)
{
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
               "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Stage x (512 doubles) into shared memory asynchronously (whole warp).
__device__ __forceinline__ void stage_x(double *buf, const double *x, int lane)
{
  if ((reinterpret_cast<uintptr_t>(x) & 15) == 0)
  {
#pragma unroll
    for (int i = 0; i < 8; i++)
    {
      const int c = lane + 32 * i; // 16-byte chunk
      cp_async16(buf + 2 * c, x + 2 * c);
    }
  }
  else
  {
#pragma unroll
    for (int i = 0; i < 16; i++)
    {
      const int c = lane + 32 * i;
      cp_async8(buf + c, x + c);
    }
  }
  cp_async_commit();
}

struct AFrag
{
  double a3[2]; // A_3(g, 2t+s), s = 0,1   (A operand of the m8n8k4 steps)
  double b2[2]; // A_2(g, 2t), A_2(g, 2t+1) (B operand, K rows permuted)
  double b1[2]; // A_1(g, 2t), A_1(g, 2t+1)
};

__device__ __forceinline__ void load_afrag(AFrag &f, const EntryRef<double> &en, int g, int t)
{
  const long long c0 = (long long)(2 * t) * en.ld[0], c1 = (long long)(2 * t + 1) * en.ld[0];
  f.b1[0] = __ldg(en.A[0] + g + c0);
  f.b1[1] = __ldg(en.A[0] + g + c1);
  const long long d0 = (long long)(2 * t) * en.ld[1], d1 = (long long)(2 * t + 1) * en.ld[1];
  f.b2[0] = __ldg(en.A[1] + g + d0);
  f.b2[1] = __ldg(en.A[1] + g + d1);
  const long long e0 = (long long)(2 * t) * en.ld[2], e1 = (long long)(2 * t + 1) * en.ld[2];
  f.a3[0] = __ldg(en.A[2] + g + e0);
  f.a3[1] = __ldg(en.A[2] + g + e1);
}

// acc[q][p] holds y(i0 = 2t+p, i1 = q, i2 = g): add it into y.
__device__ __forceinline__ void flush_acc(double (&acc)[8][2], double *y, int accum, int g, int t)
{
#pragma unroll
  for (int q = 0; q < 8; q++)
#pragma unroll
    for (int p = 0; p < 2; p++)
    {
      double *a = y + (2 * t + p) * 64 + q * 8 + g;
      if (accum == ACC_ATOMIC)
        atomicAdd(a, acc[q][p]);
      else
        *a += acc[q][p];
      acc[q][p] = 0.0;
    }
}

__global__ void __launch_bounds__(WARPS * 32) kron_n8d3_mma_kernel(const __grid_constant__ Params p)
{
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  double *xbase = smem + warp * WARP_SMEM; // two X staging buffers
  double *sw    = smem + warp * WARP_SMEM + 2 * XBUF;

  const int gw     = blockIdx.x * WARPS + warp;
  const int nwarps = gridDim.x * WARPS;

  for (int w = gw; w < p.nitems; w += nwarps)
  {
    int e0, e1;
    item_range(p, w, e0, e1);
    if (e0 >= e1)
      continue;
    double acc[8][2];
#pragma unroll
    for (int q = 0; q < 8; q++)
      acc[q][0] = acc[q][1] = 0.0;

    EntryRef<double> cur, nxt;
    entry_fetch<double>(p, entry_index(p, e0), 3, cur);
    AFrag fc, fn;
    load_afrag(fc, cur, g, t);
    int buf = 0;
    stage_x(xbase, cur.x, lane);

    for (int e = e0; e < e1; ++e)
    {
      const bool has_next = (e + 1 < e1);
      if (has_next)
        entry_fetch<double>(p, entry_index(p, e + 1), 3, nxt);
      cp_async_wait_all();
      __syncwarp();
      if (has_next)
      {
        stage_x(xbase + (buf ^ 1) * XBUF, nxt.x, lane); // overlaps this entry's math
        load_afrag(fn, nxt, g, t);
      }

      // ---- load (G=j1, P=j2, Q=j0)
      double v[8][2];
      const double *xs = xbase + buf * XBUF;
#pragma unroll
      for (int q = 0; q < 8; q++)
      {
        double2 u = *reinterpret_cast<const double2 *>(xs + q * 64 + g * 8 + 2 * t);
        v[q][0]   = u.x;
        v[q][1]   = u.y;
      }

      // ---- mode 3 (contract j2): D(i2, j1) = A_3 * X_q, m8n8k4, K = j2 as {2t, 2t+1}
      double r[8][2];
#pragma unroll
      for (int q = 0; q < 8; q++)
      {
        r[q][0] = r[q][1] = 0.0;
        mma884(r[q][0], r[q][1], fc.a3[0], v[q][0]);
        mma884(r[q][0], r[q][1], fc.a3[1], v[q][1]);
      }
      // r[q][p] = T(j0 = q, i2 = g, j1 = 2t+p)

      // ---- mode 2 (contract j1): rows (tile q, i2 = g), K = j1, B = A_2^T
#pragma unroll
      for (int rr = 0; rr < 4; rr++)
      {
        double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
        mma1688(c0, c1, c2, c3, r[2 * rr][0], r[2 * rr + 1][0], r[2 * rr][1],
                r[2 * rr + 1][1], fc.b2[0], fc.b2[1]);
        v[2 * rr][0]     = c0;
        v[2 * rr][1]     = c1;
        v[2 * rr + 1][0] = c2;
        v[2 * rr + 1][1] = c3;
      }
      // v[q][p] = U(j0 = q, i2 = g, i1 = 2t+p)

      // ---- transpose P <-> Q inside each quad: 2x2 blocks (i1 pair a, j0 pair b)
      // block (a, b) of lane-group g at 32-byte slot g*16 + a*4 + (b ^ a); its two
      // 16-byte halves swap places for odd g so both sides are conflict free.
      {
        const int gpar = g & 1;
#pragma unroll
        for (int b = 0; b < 4; b++)
        {
          double *blk = sw + 4 * (g * 16 + t * 4 + (b ^ t));
          // half 0: (i1 = 2t,   j0 = 2b, 2b+1); half 1: (i1 = 2t+1, ...)
          *reinterpret_cast<double2 *>(blk + 2 * gpar)       = make_double2(v[2 * b][0], v[2 * b + 1][0]);
          *reinterpret_cast<double2 *>(blk + 2 * (1 - gpar)) = make_double2(v[2 * b][1], v[2 * b + 1][1]);
        }
        __syncwarp();
#pragma unroll
        for (int a = 0; a < 4; a++)
        {
          const double *blk = sw + 4 * (g * 16 + a * 4 + (t ^ a));
          double2 h0 = *reinterpret_cast<const double2 *>(blk + 2 * gpar);       // i1 = 2a
          double2 h1 = *reinterpret_cast<const double2 *>(blk + 2 * (1 - gpar)); // i1 = 2a+1
          r[2 * a][0]     = h0.x; // (i1 = 2a,   j0 = 2t)
          r[2 * a][1]     = h0.y; // (i1 = 2a,   j0 = 2t+1)
          r[2 * a + 1][0] = h1.x;
          r[2 * a + 1][1] = h1.y;
        }
        __syncwarp();
      }
      // r[q][p] = U(i1 = q, i2 = g, j0 = 2t+p)

      // ---- mode 1 (contract j0), accumulate into the output-group sum
#pragma unroll
      for (int rr = 0; rr < 4; rr++)
        mma1688(acc[2 * rr][0], acc[2 * rr][1], acc[2 * rr + 1][0], acc[2 * rr + 1][1],
                r[2 * rr][0], r[2 * rr + 1][0], r[2 * rr][1], r[2 * rr + 1][1], fc.b1[0],
                fc.b1[1]);
      // acc[q][p] = Y(i0 = 2t+p, i1 = q, i2 = g)

      const bool same_next = has_next && (nxt.y == cur.y);
      if (!same_next)
        flush_acc(acc, cur.y, p.accum, g, t);
      if (has_next)
      {
        cur = nxt;
        fc  = fn;
      }
      buf ^= 1;
    }
  }
}

} // namespace

bool mma8_supported(const Params &p, int prec)
{
  if (prec != PREC_F64 || p.d != 3 || p.accum == ACC_STORE)
    return false;
  for (int l = 0; l < 3; l++)
    if (p.m[l] != 8 || p.n[l] != 8)
      return false;
  return true;
}

int launch_mma8(Params p, cudaStream_t stream)
{
  if (!p.seg_off)
  {
    p.chunk  = 8; // runs of consecutive entries per warp: X prefetch + output merging
    p.nitems = (p.eend - p.ebase + p.chunk - 1) / p.chunk;
  }
  if (p.nitems <= 0)
    return KRON_SUCCESS;
  const void *fn    = reinterpret_cast<const void *>(&kron_n8d3_mma_kernel);
  const size_t smem = (size_t)WARPS * WARP_SMEM * sizeof(double);
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && !attr_set[dev])
  {
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
      return KRON_ERROR_LAUNCH;
    attr_set[dev] = true;
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, WARPS * 32, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  const long long want = ((long long)p.nitems + WARPS - 1) / WARPS;
  const long long grid = std::max<long long>(
      1, std::min<long long>(want, (long long)device_info().sms * per_sm));
  void *args[] = {&p};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(WARPS * 32), args, smem, stream) ==
                 cudaSuccess
             ? KRON_SUCCESS
             : KRON_ERROR_LAUNCH;
}

} // namespace kron

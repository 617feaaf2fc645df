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

constexpr int WARPS     = 8;        // warps per block
constexpr int XBUF      = 512;      // doubles per X staging buffer
constexpr int WARP_SMEM = 2 * XBUF; // doubles per warp (8 KB)

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

// acc[q][p] holds y(i0 = 2t+p, i1 = q, i2 = g): add it into y with
// red.global.add.  With exclusive outputs (distinct or segmented) there is
// exactly one add per element and call, so the result is the plain sum
// y + acc, bitwise reproducible; with aliasing outputs the adds commute as
// the reference's atomicAdd does.
__device__ __forceinline__ void flush_acc(double (&acc)[8][2], double *y, int g, int t)
{
#pragma unroll
  for (int q = 0; q < 8; q++)
#pragma unroll
    for (int p = 0; p < 2; p++)
    {
      atomicAdd(y + (2 * t + p) * 64 + q * 8 + g, acc[q][p]);
      acc[q][p] = 0.0;
    }
}

// Balanced contiguous range of positions for warp gw of nw: positions are
// split evenly; with output groups (seg_off) the split points snap to the
// next group start so a group is never shared between warps.
__device__ __forceinline__ int snap_to_group(const Params &p, long long pos)
{
  int lo = p.ibase, hi = p.ibase + p.nitems; // first s with seg_off[s] >= pos
  while (lo < hi)
  {
    const int mid = (lo + hi) >> 1;
    if (p.seg_off[mid] < pos)
      lo = mid + 1;
    else
      hi = mid;
  }
  return p.seg_off[lo];
}

__device__ __forceinline__ void warp_range(const Params &p, int gw, int nw, int &eb, int &ee)
{
  if (p.seg_off)
  {
    const long long b = p.seg_off[p.ibase], tot = p.seg_off[p.ibase + p.nitems] - b;
    eb = snap_to_group(p, b + tot * gw / nw);
    ee = snap_to_group(p, b + tot * (gw + 1) / nw);
  }
  else
  {
    const long long tot = p.eend - p.ebase;
    eb = p.ebase + (int)(tot * gw / nw);
    ee = p.ebase + (int)(tot * (gw + 1) / nw);
  }
}

__global__ void __launch_bounds__(WARPS * 32) kron_n8d3_mma_kernel(const __grid_constant__ Params p)
{
  extern __shared__ __align__(16) double smem[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  // two X staging buffers per warp; the one just consumed doubles as the
  // transpose buffer
  double *xbase = smem + warp * WARP_SMEM;

  int eb, ee;
  warp_range(p, blockIdx.x * WARPS + warp, gridDim.x * WARPS, eb, ee);
  if (eb >= ee)
    return;
  int e = eb; // position being computed; e+1 has operands in flight, e+2 pointers

  EntryRef<double> cur, nxt, far;
  entry_fetch<double>(p, entry_index(p, e), 3, cur);
  if (e + 1 < ee)
    entry_fetch<double>(p, entry_index(p, e + 1), 3, nxt);
  AFrag fc, fn;
  load_afrag(fc, cur, g, t);
  int buf = 0;
  stage_x(xbase, cur.x, lane);

  double acc[8][2];
#pragma unroll
  for (int q = 0; q < 8; q++)
    acc[q][0] = acc[q][1] = 0.0;

  while (true)
  {
    const bool has_next = (e + 1 < ee);
    const bool has_far  = (e + 2 < ee);
    if (has_far)
      entry_fetch<double>(p, entry_index(p, e + 2), 3, far);
    cp_async_wait_all();
    __syncwarp();
    if (has_next)
    {
      stage_x(xbase + (buf ^ 1) * XBUF, nxt.x, lane); // overlaps this entry's math
      load_afrag(fn, nxt, g, t);
    }

    // ---- load (G=j1, P=j2, Q=j0)
    double v[8][2];
    double *xs = xbase + buf * XBUF;
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
      mma1688(c0, c1, c2, c3, r[2 * rr][0], r[2 * rr + 1][0], r[2 * rr][1], r[2 * rr + 1][1],
              fc.b2[0], fc.b2[1]);
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
      __syncwarp(); // every lane has read its X tile from xs
      const int gpar = g & 1;
#pragma unroll
      for (int b = 0; b < 4; b++)
      {
        double *blk = xs + 4 * (g * 16 + t * 4 + (b ^ t));
        // half 0: (i1 = 2t, j0 = 2b, 2b+1); half 1: (i1 = 2t+1, ...)
        *reinterpret_cast<double2 *>(blk + 2 * gpar) = make_double2(v[2 * b][0], v[2 * b + 1][0]);
        *reinterpret_cast<double2 *>(blk + 2 * (1 - gpar)) =
            make_double2(v[2 * b][1], v[2 * b + 1][1]);
      }
      __syncwarp();
#pragma unroll
      for (int a = 0; a < 4; a++)
      {
        const double *blk = xs + 4 * (g * 16 + a * 4 + (t ^ a));
        double2 h0 = *reinterpret_cast<const double2 *>(blk + 2 * gpar);       // i1 = 2a
        double2 h1 = *reinterpret_cast<const double2 *>(blk + 2 * (1 - gpar)); // i1 = 2a+1
        r[2 * a][0]     = h0.x; // (i1 = 2a,   j0 = 2t)
        r[2 * a][1]     = h0.y; // (i1 = 2a,   j0 = 2t+1)
        r[2 * a + 1][0] = h1.x;
        r[2 * a + 1][1] = h1.y;
      }
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
      flush_acc(acc, cur.y, g, t);
    if (!has_next)
      break;
    cur = nxt;
    fc  = fn;
    nxt = far;
    ++e;
    buf ^= 1;
  }
  cp_async_wait_all();
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
  const long long work = p.seg_off ? p.nitems : (long long)(p.eend - p.ebase);
  if (work <= 0)
    return KRON_SUCCESS;
  const void *fn    = reinterpret_cast<const void *>(&kron_n8d3_mma_kernel);
  const size_t smem = (size_t)WARPS * WARP_SMEM * sizeof(double);
  int per_sm = 1;
  if (cached_occupancy(fn, WARPS * 32, smem, &per_sm) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  // one resident wave; every warp gets a balanced contiguous range
  const long long want = (work + WARPS - 1) / WARPS;
  const long long grid = std::max<long long>(
      1, std::min<long long>(want, (long long)device_info().sms * per_sm));
  void *args[] = {&p};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(WARPS * 32), args, smem, stream) ==
                 cudaSuccess
             ? KRON_SUCCESS
             : KRON_ERROR_LAUNCH;
}

} // namespace kron

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
#include "kron_mma8_core.cuh"

namespace kron {

namespace {

constexpr int WARPS     = 8;        // warps per block
constexpr int XBUF      = 512;      // doubles per X staging buffer
constexpr int WARP_SMEM = 2 * XBUF; // doubles per warp (8 KB)

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

__device__ __forceinline__ void load_afrag(AFrag8 &f, const EntryRef<double> &en, int g, int t)
{
  load_afrag8(f, en.A[0], en.ld[0], en.A[1], en.ld[1], en.A[2], en.ld[2], g, t);
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
  AFrag8 fc, fn;
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

    kron8x3_tile(v, acc, fc, xs, g, t);
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

// Internal definitions shared by the kronmult_b200 CUDA sources.
//
// Data model.  One "entry" k is  y_k += kron(A_1..A_d) x_k  with A_l an
// m_l x n_l column-major matrix (leading dimension ld_l), x_k of length
// N = prod n_l and y_k of length M = prod m_l, A_d's index fastest.  The
// four reference layouts only differ in how entry k's pointers are found
// (EntryFetch below):
//   batched  : A + (k*d + l)*n*n, X + k*N, Y + k*M   (kronmult6_batched.hpp:16-19,41-53)
//   pbatched : A + (k*d + l)*n*n, pX[k], pY[k]       (kronmult6_pbatched.hpp:52-62)
//   xbatched : pA[l + k*d] (lda), pX[k], pY[k]       (kronmult_xbatched.hpp:67-69,121-131)
//   vbatched : pA[l + k*d] (ld = m_l), pX[k], pY[k]  (kronmult_vbatched.hpp:165-189)
//   entries  : pA[l + 6*k] (ld = m_l), per-entry shapes (uneven batch)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kronmult.h"

namespace kron {

constexpr int MAXD = 6;

enum Layout : int
{
  LAYOUT_BATCHED  = 0,
  LAYOUT_PBATCHED = 1,
  LAYOUT_XBATCHED = 2,
  LAYOUT_VBATCHED = 3,
};

// How an entry's result reaches y.
enum Accum : int
{
  ACC_DISTINCT  = 0, // every entry owns its y: plain read-modify-write
  ACC_ATOMIC    = 1, // outputs may alias: red.global.add (runs of equal y merged first)
  ACC_SEGMENTED = 2, // work items are output groups (plan): fixed order, one plain RMW
  ACC_STORE     = 3, // overwrite (intermediate into workspace)
};

enum Precision : int
{
  PREC_F64   = 0,
  PREC_F32   = 1,
  PREC_SPLIT = 2, // FP64 storage, hi+lo FP32 arithmetic
};

// Everything a kernel needs to find entry k and the work items.
struct Params
{
  int layout;
  int accum;
  int d;
  int m[MAXD];
  int n[MAXD];
  int lda; // xbatched common leading dimension (batched/pbatched: n)
  int apk; // A pointers per entry in pA (xbatched/vbatched: d; per-entry plans: 6)
  int batch;
  const void *A;                 // batched / pbatched
  const void *const *pA;         // xbatched / vbatched
  const void *X;                 // batched
  void *Y;                       // batched
  const void *const *pX;         // pointer layouts
  void *const *pY;               // pointer layouts
  long long xstride, ystride;    // batched column strides (elements)
  // Work items.  Without seg_off, item w covers positions
  // [ebase + w*chunk, min(eend, ebase + (w+1)*chunk)); with seg_off it covers
  // [seg_off[ibase + w], seg_off[ibase + w + 1]).  Position e is entry
  // perm[e] (identity when perm is null).
  int nitems;
  int chunk;
  int ebase, eend, ibase;
  const int *perm;
  const int *seg_off;
};

__host__ __device__ constexpr int cpow(int b, int e) { return e == 0 ? 1 : b * cpow(b, e - 1); }

template <typename T>
struct EntryRef
{
  const T *A[MAXD];
  int ld[MAXD];
  const T *x;
  T *y;
};

// Resolve entry k's operands.  D is the number of modes (compile-time or
// p.d for the runtime kernels).
template <typename T>
__device__ __forceinline__ T *entry_y(const Params &p, int k)
{
  if (p.layout == LAYOUT_BATCHED)
    return static_cast<T *>(p.Y) + (long long)k * p.ystride;
  return static_cast<T *>(p.pY[k]);
}

template <typename T>
__device__ __forceinline__ void entry_fetch(const Params &p, int k, int D, EntryRef<T> &e)
{
  switch (p.layout)
  {
  case LAYOUT_BATCHED:
  case LAYOUT_PBATCHED: {
    const T *A = static_cast<const T *>(p.A);
    const long long nn = (long long)p.n[0] * p.n[0];
    for (int l = 0; l < D; l++)
    {
      e.A[l]  = A + ((long long)k * D + l) * nn;
      e.ld[l] = p.n[0];
    }
    if (p.layout == LAYOUT_BATCHED)
    {
      e.x = static_cast<const T *>(p.X) + (long long)k * p.xstride;
      e.y = static_cast<T *>(p.Y) + (long long)k * p.ystride;
    }
    else
    {
      e.x = static_cast<const T *>(p.pX[k]);
      e.y = static_cast<T *>(p.pY[k]);
    }
    break;
  }
  case LAYOUT_XBATCHED:
  default: {
    for (int l = 0; l < D; l++)
    {
      e.A[l]  = static_cast<const T *>(p.pA[(long long)k * p.apk + l]);
      e.ld[l] = (p.layout == LAYOUT_XBATCHED) ? p.lda : p.m[l];
    }
    e.x = static_cast<const T *>(p.pX[k]);
    e.y = static_cast<T *>(p.pY[k]);
    break;
  }
  }
}

__device__ __forceinline__ void item_range(const Params &p, int w, int &e0, int &e1)
{
  if (p.seg_off)
  {
    e0 = p.seg_off[p.ibase + w];
    e1 = p.seg_off[p.ibase + w + 1];
  }
  else
  {
    e0 = p.ebase + w * p.chunk;
    e1 = min(p.eend, e0 + p.chunk);
  }
}

__device__ __forceinline__ int entry_index(const Params &p, int e)
{
  return p.perm ? p.perm[e] : e;
}

// Barrier over one thread group of `nthreads` (a multiple of 32) with a
// group-private id (1..15); the whole block uses __syncthreads().
__device__ __forceinline__ void group_sync(int gid, int nthreads)
{
  if (nthreads == (int)blockDim.x)
    __syncthreads();
  else if (nthreads == 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;" ::"r"(gid + 1), "r"(nthreads) : "memory");
}

template <typename T>
__device__ __forceinline__ void red_add(T *addr, T v)
{
  atomicAdd(addr, v);
}

// Add v into y[i] according to the accumulation mode.
template <typename T>
__device__ __forceinline__ void y_update(int accum, T *y, long long i, T v)
{
  if (accum == ACC_ATOMIC)
    red_add(y + i, v);
  else if (accum == ACC_STORE)
    y[i] = v;
  else
    y[i] += v;
}

// ---- host side ----------------------------------------------------------

// cudaMalloc with the failure injection of kron_test_fail_alloc
// (kron_status.cu); every device allocation of the library goes through it
cudaError_t dev_malloc(void **ptr, size_t bytes);
void dev_free(void *ptr);

struct DeviceInfo
{
  int device;
  int sms;
  int max_smem_optin; // bytes per block
  int smem_per_sm;
};
const DeviceInfo &device_info();

// Launch the full problem described by p (all layouts, uniform shapes).
// W / pW / Wbytes give the caller's workspace for vectors too large to stay
// on chip.  Returns a kron_status_t.
struct Workspace
{
  void *W;                 // flat workspace (batched: column k at W + k*wstride)
  void *const *pW;         // pointer workspace (pbatched/xbatched)
  int npW;                 // number of pW pointers usable
  long long wstride;       // batched: elements per W column
  size_t Wbytes;           // flat capacity (vbatched)
  long long pw_elems;      // elements behind each pW pointer
  const int *seg_host;     // segmented: host copy of the segment offsets
  int nseg;                // segmented: number of segments
};

int launch_kron(Params p, int precision, const Workspace &ws, cudaStream_t stream);
size_t large_workspace_elems(int d, const int *m, const int *n);
bool fits_on_chip(int d, const int *m, const int *n, int precision, bool merge);

int launch_kgemm(int op, int mm, int nn, int kk, double alpha, double *const *A, const int *ldA,
                 double *const *B, const int *ldB, double beta, double *const *C,
                 const int *ldC, int batch, cudaStream_t stream);

} // namespace kron

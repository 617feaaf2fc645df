// Inline-PTX helpers for sm_100a kernels: mbarriers, 1-D TMA bulk copies and
// bulk reduce-adds, thread-block-cluster ranks, barriers and shared::cluster
// (DSMEM) loads.
#pragma once

#include <cstdint>

namespace kron {
namespace ptx {

__device__ __forceinline__ unsigned smem_addr(const void *p)
{
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrive on the barrier and add `bytes` to the transaction count its
// current phase waits for
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// non-blocking test of the phase with the given parity
__device__ __forceinline__ bool mbar_test_wait(uint64_t *bar, unsigned parity)
{
  unsigned ok;
  asm volatile("{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n"
               " selp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}

// wait for the phase with the given parity to complete, at most `limit`
// polls; false when the limit ran out.  The first poll does not block (a
// limit of 1 gives up unless the phase has already completed), the others
// may suspend the thread for a while each.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long long limit)
{
  if (limit < 1)
    return false;
  if (mbar_test_wait(bar, parity))
    return true;
  for (long long it = 1; it < limit; ++it)
    if (mbar_try_wait(bar, parity))
      return true;
  return false;
}

// global -> this block's shared memory, completion counted on `bar`
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, unsigned bytes,
                                            uint64_t *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
               "%2, [%3];" ::"r"(smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// y[0..bytes) += smem[0..bytes), element-wise adds performed in L2
template <typename T>
__device__ __forceinline__ void bulk_reduce_add(T *y, const T *src, unsigned bytes)
{
  if constexpr (sizeof(T) == 8)
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f64 [%0], [%1], %2;" ::"l"(y),
                 "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
  else
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(y),
                 "r"(smem_addr(src)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the sources of every committed bulk group have been read
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// every committed bulk group has completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) accesses
__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ unsigned cluster_ctarank()
{
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// whole-cluster barrier (every thread of every block), split into its two
// halves; arrive releases this thread's prior memory accesses, wait
// acquires every other thread's
__device__ __forceinline__ void cluster_arrive()
{
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait()
{
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_sync()
{
  cluster_arrive();
  cluster_wait();
}

// shared::cluster address of the same offset in block `rank`'s shared memory
__device__ __forceinline__ unsigned mapa(unsigned saddr, unsigned rank)
{
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}

template <typename T>
__device__ __forceinline__ T ld_cluster(unsigned addr)
{
  if constexpr (sizeof(T) == 8)
  {
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
  }
  else
  {
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
  }
}

__device__ __forceinline__ int ld_cluster_s32(unsigned addr)
{
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
  return v;
}

__device__ __forceinline__ bool aligned16(const void *p)
{
  return (reinterpret_cast<uintptr_t>(p) & 15) == 0;
}

} // namespace ptx
} // namespace kron

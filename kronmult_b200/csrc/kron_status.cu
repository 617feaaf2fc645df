// The library's device status word and the bound on its kernels' waits.
//
// Kernels that wait on an mbarrier poll it at most wait_limit() times; when
// the bound runs out they store 1 into the status word (its device address
// comes from device_status_ptr(), passed as a kernel argument), let the
// copies they started land and leave without touching y.  The host reads and
// clears the word with kron_device_status.  kron_set_wait_limit lowers the
// bound for the launches that follow, so a test can make a wait run out on
// purpose without a hung or faulted GPU: the copies still land, only the
// waiting block gives up early.
//
// dev_malloc / dev_free are the library's only route to cudaMalloc and
// cudaFree (plans, the autotuner's synthetic problem, the FP64 peak probe).
// kron_test_fail_alloc makes one of the following allocations fail and
// kron_test_live_allocs counts the allocations not yet freed, so a test can
// check that every caller returns KRON_ERROR_ALLOC and frees what it already
// holds.
#include <atomic>
#include <mutex>

#include "kron_launch.h"

namespace kron {

namespace {

__device__ int g_device_status = 0;

constexpr long long DEFAULT_WAIT_LIMIT = 1LL << 26;
std::atomic<long long> g_wait_limit{DEFAULT_WAIT_LIMIT};

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
int *g_status_addr[MAX_DEVICES] = {};

// allocations left before the injected failure; -1: none injected
std::atomic<int> g_fail_countdown{-1};
// device allocations made through dev_malloc and not yet freed
std::atomic<long long> g_live_allocs{0};

} // namespace

cudaError_t dev_malloc(void **ptr, size_t bytes)
{
  int c = g_fail_countdown.load();
  while (c >= 0 && !g_fail_countdown.compare_exchange_weak(c, c - 1))
  {
  }
  if (c == 0)
  {
    *ptr = nullptr;
    return cudaErrorMemoryAllocation;
  }
  const cudaError_t e = cudaMalloc(ptr, bytes);
  if (e == cudaSuccess)
    g_live_allocs.fetch_add(1);
  return e;
}

void dev_free(void *ptr)
{
  if (ptr && cudaFree(ptr) == cudaSuccess)
    g_live_allocs.fetch_sub(1);
}

int *device_status_ptr()
{
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES)
    return nullptr;
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_status_addr[dev])
  {
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_device_status) != cudaSuccess)
      return nullptr;
    g_status_addr[dev] = static_cast<int *>(p);
  }
  return g_status_addr[dev];
}

long long wait_limit() { return g_wait_limit.load(std::memory_order_relaxed); }

long long drain_limit() { return DEFAULT_WAIT_LIMIT; }

} // namespace kron

extern "C" int kron_device_status(int clear)
{
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, kron::g_device_status, sizeof(int)) != cudaSuccess)
    return -1;
  if (clear && v != 0)
  {
    int z = 0;
    if (cudaMemcpyToSymbol(kron::g_device_status, &z, sizeof(int)) != cudaSuccess)
      return -1;
  }
  return v;
}

extern "C" int kron_set_wait_limit(long long polls)
{
  if (polls < 0)
    return KRON_ERROR_INVALID_VALUE;
  kron::g_wait_limit.store(polls == 0 ? kron::DEFAULT_WAIT_LIMIT : polls,
                           std::memory_order_relaxed);
  return KRON_SUCCESS;
}

extern "C" int kron_test_fail_alloc(int nth)
{
  if (nth < -1)
    return KRON_ERROR_INVALID_VALUE;
  kron::g_fail_countdown.store(nth);
  return KRON_SUCCESS;
}

extern "C" long long kron_test_live_allocs(void) { return kron::g_live_allocs.load(); }

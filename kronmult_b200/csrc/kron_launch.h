// Host-side planning helpers shared by the launcher and the C API.
#pragma once

#include "kron_kernels.cuh"

namespace kron {

// Raises the kernel's dynamic shared-memory limit once and caches the
// resident blocks per SM for (block, smem).
int cached_occupancy(const void *fn, int block, size_t smem, int *per_sm);

double flops_forward(int d, const int *m, const int *n);
double flops_backward(int d, const int *m, const int *n);
bool choose_forward(int d, const int *m, const int *n);
long long max_intermediate(int d, const int *m, const int *n, bool forward);

// Two-phase plan for vectors that exceed shared memory.
struct LargePlan
{
  int q;                 // phase 1 applies modes [q, d), phase 2 modes [0, q)
  GenView v1, v2;
  int C;                 // phase-2 tile columns
  long long slot_elems;  // workspace elements per entry
  long long score;
};
bool plan_large(int d, const int *m, const int *n, int esize, bool merge, LargePlan &lp);

// FP64 tensor-core path for square 8x8 factors, d = 3 (kron_mma8.cu).
bool mma8_supported(const Params &p, int prec);
int launch_mma8(Params p, cudaStream_t stream);

// TMA-pipelined register-blocked kernel for square n in {2..5}, 4-64 KB
// vectors (kron_pipe.cu).
bool pipe_supported(const Params &p, int prec);
int launch_pipe(Params p, int prec, cudaStream_t stream);

// Slab-cluster kernel for square d = 6 vectors beyond one block's shared
// memory whose n slabs of n^5 elements fit (kron_slab.cu).
bool slab_supported(const Params &p, int prec);
int launch_slab(Params p, int prec, int flags, cudaStream_t stream);
// SMs that the slab kernel's resident clusters occupy (the cluster shape can
// leave some SMs of each GPC without a whole cluster).
int slab_sms_used(int n, int prec, int flags, int *used);
// The slab kernel plus a side kernel (cluster two-phase, second stream) on
// the SMs its clusters leave idle, when p and the workspace allow
// (kron_launch.cu).
int launch_slab_side(Params p, int prec, const Workspace &ws, int flags, cudaStream_t stream);

// Device status word (kron_status.cu): its device address for kernel
// arguments, the poll bound of mbarrier waits (kron_set_wait_limit), and the
// bound of the final drain that lets a giving-up block's copies land.
int *device_status_ptr();
long long wait_limit();
long long drain_limit();

// Cluster two-phase kernel for vectors beyond shared memory (kron_big.cu);
// cluster <= 0 picks the default cluster size.
bool big_supported(const Params &p, int prec);
int launch_big(Params p, const Workspace &ws, int prec, int cluster, cudaStream_t stream);

// Split precision (FP64 data, exact BF16 slice products on the tcgen05 tensor
// cores) for square d = 6, n = 8 in the batched layout with a workspace W
// (kron_splittc.cu).
bool splittc_supported(const Params &p, int prec);
int launch_splittc(Params p, const Workspace &ws, cudaStream_t stream);

// Kernel variants the launcher chooses among (values of KRON_VARIANT_* in
// kronmult.h).
enum Variant : int
{
  VAR_NONE  = 0,
  VAR_MMA8  = 1, // FP64 tensor-core d = 3, n = 8 (param unused)
  VAR_PIPE  = 2, // TMA-pipelined register-blocked passes (param unused)
  VAR_SQ    = 3, // square on-chip kernel; param = entries per block (0: most that fit)
  VAR_GEN   = 4, // runtime-shape on-chip kernel (param unused)
  VAR_BIG   = 5, // cluster two-phase kernel; param = cluster size (0: default)
                 // | KRON_BIG_CUDA_CORES (FP64 n = 8 without tensor cores)
                 // | KRON_BIG_SMEM_W (FP64 n = 6: W in the cluster's shared memory)
  VAR_LARGE = 6, // two-phase launches through the workspace (param unused)
  VAR_SLAB  = 7, // slab-cluster kernel, no workspace; param: KRON_SLAB_NO_ROTATE
  VAR_SPLIT_TC = 8, // split precision d = 6, n = 8 on the tcgen05 tensor cores
};

// Work items of a launch (launch_kron does this before any variant).
void launch_setup(Params &p, const Workspace &ws);
// Launch one variant; KRON_ERROR_NOT_SUPPORTED when it cannot run p.
int launch_variant(Params p, int prec, const Workspace &ws, int variant, int param,
                   cudaStream_t stream);
// Most entries per block of the square on-chip kernel for (d, n), 0 when it
// does not apply.
int sq_entries_max(int prec, int d, int n, bool merge);
// Variant recorded for (d, n, prec) by the autotuner or the caller.
bool tune_lookup(int d, int n, int prec, int &variant, int &param);

} // namespace kron

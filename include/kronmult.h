/*
 * kronmult_b200 -- batched Kronecker matrix-vector products on NVIDIA B200
 * (sm_100a).  For every batch entry k:
 *
 *     Y(:,k) += kron(A_1(k), ..., A_d(k)) * X(:,k),      d = 1..6
 *
 * with A_d's index fastest in X and Y and every matrix column major.
 *
 * Two layers are exported from libkronmult_b200.so:
 *
 *  1. The reference KRONMULT host entry points with their exact C++
 *     signatures (C++ linkage, so existing C++ callers relink unchanged).
 *     They launch on the legacy default stream, return nothing, and record
 *     their status for kron_get_last_status() -- the reference has no error
 *     return at all.
 *
 *  2. An extern "C" twin for each, suffixed _async, that takes an explicit
 *     stream and returns a kron_status_t; plus extensions with no reference
 *     counterpart (FP32 / split precision, deterministic segmented
 *     accumulation, per-entry-shape vbatched, workspace queries).
 *
 * Every pointer argument (data, pointer arrays, ld arrays) is a DEVICE
 * pointer, as in the reference GPU build (test_kronmult6_xbatched.cpp:243-271),
 * unless a comment says "host".  All calls are asynchronous on their stream.
 *
 * Differences from the reference that callers may observe (all are
 * strict relaxations):
 *   - X is never modified (the reference batched/pbatched clobber X and W,
 *     kronmult6_batched.hpp:10);
 *   - W is accepted but only used for vectors too large for on-chip
 *     storage; its contents are never relied upon;
 *   - entries whose outputs alias are summed on the GPU in an unspecified
 *     order in the default (atomic) mode, like the reference's atomicAdd.
 */
#ifndef KRONMULT_B200_H
#define KRONMULT_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Same type as cudaStream_t; NULL is the legacy default stream. */
typedef struct CUstream_st *kron_stream_t;

typedef enum kron_status
{
  KRON_SUCCESS             = 0,
  KRON_ERROR_INVALID_VALUE = 1, /* bad size, null pointer, d out of 1..6 */
  KRON_ERROR_WORKSPACE     = 2, /* the W provided is too small for the path */
  KRON_ERROR_LAUNCH        = 3, /* a CUDA runtime / launch error */
  KRON_ERROR_NOT_SUPPORTED = 4, /* combination not implemented */
  KRON_ERROR_ALLOC         = 5, /* device or host allocation failed */
  KRON_ERROR_INTERNAL      = 6
} kron_status_t;

const char *kron_status_string(int status);

/* Status of the last reference-signature (void) call made on this host
 * thread; KRON_SUCCESS if none failed.  Reading it does not reset it. */
int kron_get_last_status(void);
void kron_clear_last_status(void);

/* Library version "major.minor.patch". */
const char *kron_version(void);

/* ------------------------------------------------------------------------
 * batched: A is (n,n,d,batchCount) contiguous; X, Y, W are (n^d, batchCount).
 * Replaces kronmult{d}_batched (kronmult6_batched.cpp:4-18).  Every entry
 * writes its own Y column.  W may be NULL when n^d doubles fit on chip
 * (kron_batched_workspace_bytes() returns 0 then), and for d = 6, n = 6,
 * where a null W keeps the intermediate in a two-block cluster's shared
 * memory (the query still returns the workspace form's need, the faster
 * form when W is given).  The same holds for the pointer layouts.
 * ---------------------------------------------------------------------- */
int kronmult1_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);
int kronmult2_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);
int kronmult3_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);
int kronmult4_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);
int kronmult5_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);
int kronmult6_batched_async(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                            double Warray_[], int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * pbatched: A as in batched; X, Y, W are arrays of batchCount device
 * pointers to n^d doubles.  Y pointers may alias (outputs are then summed).
 * Replaces kronmult{d}_pbatched (kronmult6_pbatched.cpp:4-19).
 * ---------------------------------------------------------------------- */
int kronmult1_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);
int kronmult2_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);
int kronmult3_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);
int kronmult4_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);
int kronmult5_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);
int kronmult6_pbatched_async(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                             double *Warray_[], int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * xbatched: Aarray_ holds d*batchCount device pointers, entry k's A_l at
 * Aarray_[(l-1) + (k-1)*d], each n x n with leading dimension lda >= n.
 * X, Y, W are pointer arrays; Y may alias.  subbatchCount <= 0 means the
 * reference default max(1, batchCount/2); it bounds how many W pointers
 * are used (2*subbatchCount, each n^d doubles) when W is needed at all.
 * Replaces kronmult{d}_xbatched (kronmult6_xbatched.cpp:4-28,
 * kronmult_xbatched.hpp:17-162).
 * ---------------------------------------------------------------------- */
int kronmult1_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);
int kronmult2_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);
int kronmult3_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);
int kronmult4_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);
int kronmult5_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);
int kronmult6_xbatched_async(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                             double *Yarray_[], double *Warray_[], int batchCount,
                             int subbatchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * vbatched: rectangular A_l (m_l x n_l, leading dimension m_l), the same
 * shapes for every entry; Aarray_ as in xbatched; X has prod(n_l), Y has
 * prod(m_l) entries per vector; W is one flat device buffer of
 * Wcapacity_bytes (may be 0 / NULL when everything fits on chip;
 * kron_vbatched_workspace_bytes() gives the exact need -- the reference's
 * own sizing is too small for Alg. 993 on rectangular shapes,
 * kronmult_vbatched.hpp:107-135).  The reference only has the kernel
 * templates kronmult{d}_vbatched<T> (kronmult6_vbatched.hpp:10-34); these
 * are the host entry points it lacks.
 * ---------------------------------------------------------------------- */
int kronmult1_vbatched_async(int m1, int n1, double const *const Aarray_[], double *pX_[],
                             double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream);
int kronmult2_vbatched_async(int m1, int n1, int m2, int n2, double const *const Aarray_[],
                             double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                             int batchCount, kron_stream_t stream);
int kronmult3_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3,
                             double const *const Aarray_[], double *pX_[], double *pY_[],
                             double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream);
int kronmult4_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             double const *const Aarray_[], double *pX_[], double *pY_[],
                             double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream);
int kronmult5_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             int m5, int n5, double const *const Aarray_[], double *pX_[],
                             double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount,
                             kron_stream_t stream);
int kronmult6_vbatched_async(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                             int m5, int n5, int m6, int n6, double const *const Aarray_[],
                             double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                             int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * kgemm_{nn,nt,tt}_batched: C_k = alpha op(A_k) op(B_k) + beta C_k with
 * op(A) = A (nn, nt) or A^T (tt), op(B) = B (nn) or B^T (nt, tt); mm x kk
 * times kk x nn; pointer arrays and per-entry leading dimensions.
 * beta == 1 accumulates atomically (C pointers may alias), beta == 0 never
 * reads C.  Replaces kgemm_{nn,nt,tt}_batched (kgemm_nn_batched.cpp:5-25).
 * ---------------------------------------------------------------------- */
int kgemm_nn_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream);
int kgemm_nt_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream);
int kgemm_tt_batched_async(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                           int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                           double beta, double *const Carray_[], int const ldCarray_[],
                           int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * Workspace queries (no reference counterpart): bytes of W the
 * corresponding call needs; 0 means W may be NULL.
 * ---------------------------------------------------------------------- */
size_t kron_batched_workspace_bytes(int d, int n, int batchCount);
size_t kron_vbatched_workspace_bytes(int d, int const m[], int const n[], int batchCount);

/* ------------------------------------------------------------------------
 * Precision extensions of the batched layout (no reference counterpart).
 *   kronmult_batched_f32_async   : FP32 storage, FP32 accumulation.
 *   kronmult_batched_split_async : FP64 storage; every product is formed
 *     from hi+lo FP32 parts of A and X (three cross products, error-free
 *     FP32 products and compensated FP32 sums), and the result is added to
 *     Y in FP64.
 * d is 1..6; W as in batched (may be NULL when n^d fits on chip).
 * ---------------------------------------------------------------------- */
int kronmult_batched_f32_async(int d, int n, float const A[], float X[], float Y[], float W[],
                               int batchCount, kron_stream_t stream);
int kronmult_batched_split_async(int d, int n, double const A[], double X[], double Y[],
                                 double W[], int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * No reference counterpart.  The batched FP64 product for callers that
 * cannot call cudaMalloc where they apply the operator (a stream capture in
 * global mode, a memory pool that owns all of HBM, a callback handed only
 * A, X and Y): it takes no W.  Vectors too large for shared memory use one
 * 16 MiB file-scope device array instead, which every GPU that loads the
 * library holds until exit.  n^d above 2,097,152 (16 MiB of doubles) is
 * rejected with KRON_ERROR_WORKSPACE.  Calls share that array: calls that
 * overlap on the GPU race; calls ordered on one stream are safe.  Every call
 * outside stream capture looks the array's address up on the current device
 * (any shape); a call under capture uses the address the last such lookup
 * found, so the first call on a device should precede any stream capture.
 * Allocates nothing.
 * ---------------------------------------------------------------------- */
int kronmult_batched_noalloc_async(int d, int n, double const A[], double const X[], double Y[],
                                   int batchCount, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * Deterministic (bitwise reproducible) accumulation for aliasing outputs
 * (no reference counterpart).  A segment plan groups the entries by output
 * pointer once (stable, keeps each group's entry order); an execution with
 * the plan sums every group in that fixed order on one thread block and
 * writes each output exactly once -- no atomics.
 * kron_segments_create reads the device pointer array Yarray_ (batchCount
 * entries) and synchronises `stream`.
 * ---------------------------------------------------------------------- */
typedef struct kron_segments_st *kron_segments_t;

int kron_segments_create(kron_segments_t *plan, double *const Yarray_[], int batchCount,
                         kron_stream_t stream);
int kron_segments_destroy(kron_segments_t plan);
int kron_segments_count(kron_segments_t plan);

int kronmult_xbatched_segmented_async(int d, int n, double const *const Aarray_[], int lda,
                                      double *Xarray_[], double *Yarray_[], double *Warray_[],
                                      int batchCount, kron_segments_t plan,
                                      kron_stream_t stream);
int kronmult_pbatched_segmented_async(int d, int n, double const Aarray_[], double *Xarray_[],
                                      double *Yarray_[], double *Warray_[], int batchCount,
                                      kron_segments_t plan, kron_stream_t stream);

/* ------------------------------------------------------------------------
 * Uneven batch (no reference counterpart): every entry has its own d and
 * rectangular shapes.  shapes (host) holds 13 ints per entry:
 * {d, m1, n1, m2, n2, ..., m6, n6}.  The plan orders the entries by cost
 * (largest first) for one persistent launch, picks Alg. 993 forward or
 * backward per entry by flop count (kronm.hpp:39-89), and sizes the
 * workspace for the chosen variant.  Execution reads entry k's A_l from
 * Aarray_[(l-1) + 6*(k-1)] (leading dimension m_l), X from pX_[k], adds
 * into pY_[k] (outputs may alias).
 * ---------------------------------------------------------------------- */
typedef struct kron_vplan_st *kron_vplan_t;

int kron_vplan_create(kron_vplan_t *plan, int batchCount, int const shapes[]);
int kron_vplan_destroy(kron_vplan_t plan);
size_t kron_vplan_workspace_bytes(kron_vplan_t plan);
double kron_vplan_flops(kron_vplan_t plan);
int kron_vplan_execute_async(kron_vplan_t plan, double const *const Aarray_[], double *pX_[],
                             double *pY_[], void *W, size_t Wcapacity_bytes,
                             kron_stream_t stream);

/* kron_flops (kroncommon.hpp:154-185) restated: flops of one entry of the
 * recursive algorithm. */
double kron_flops_c(int d, int const m[], int const n[]);

/* Diagnostics (no reference counterpart): measures the current device's
 * FP64 throughput in TFLOP/s -- tensor-core (mma.sync f64) and CUDA-core
 * fma -- for roofline reporting.  Synchronises the device; allocates 2 KB. */
int kron_measure_fp64_peak(double *tensor_tflops, double *cuda_core_tflops);

/* Device-side status word of the library's kernels: 0 when every bounded
 * wait completed, 1 after a kernel gave up waiting on an asynchronous copy
 * (the affected results are then invalid).  Synchronises with the device;
 * clear != 0 resets the word.  Returns -1 if it cannot be read. */
int kron_device_status(int clear);

/* Bound on the polls of every asynchronous-copy wait in the kernels launched
 * after this call (default 2^26; 0 restores the default).  A testing aid: a
 * small bound makes a wait give up early -- the kernel then records 1 in the
 * status word above, lets its copies land (always with the default bound),
 * leaves y untouched for the entries it gave up on and returns -- so a test
 * can drive the time-out path without a hung or faulted GPU.  Process-wide. */
int kron_set_wait_limit(long long polls);

/* Testing aid: the nth (0-based) device allocation the library makes after
 * this call fails as if cudaMalloc had (-1: none; the default).  The calls
 * that allocate -- kron_segments_create, kron_vplan_create, kron_autotune,
 * kron_measure_fp64_peak -- then return KRON_ERROR_ALLOC with nothing left
 * allocated.  Process-wide; the injection is used up by the failure. */
int kron_test_fail_alloc(int nth);
/* Testing aid: device allocations the library made and has not freed yet
 * (plans alive, nothing else: every call frees its temporaries). */
long long kron_test_live_allocs(void);

/* ------------------------------------------------------------------------
 * Pointer arrays built on the device from integer lists (no reference
 * counterpart; the reference's tests build them on the host and copy them,
 * test_kronmult6_xbatched.cpp:231-271).  All arrays are device arrays;
 * a NULL list means the identity (entry k, or block l + k*d):
 *   Xarray_out[k]         = X + xlist[k] * xstride
 *   Yarray_out[k]         = Y + ylist[k] * ystride
 *   Aarray_out[l + k * d] = A + alist[l + k * d] * astride
 * Any output may be NULL (not built).  Indices are not range-checked.
 * Asynchronous on `stream`.
 * ---------------------------------------------------------------------- */
int kron_build_pointers_async(int d, int batchCount, double const *A, long long astride,
                              int const alist[], double const *X, long long xstride,
                              int const xlist[], double *Y, long long ystride,
                              int const ylist[], double const *Aarray_out[],
                              double *Xarray_out[], double *Yarray_out[], kron_stream_t stream);

/* ------------------------------------------------------------------------
 * Owner-computes sharding over several GPUs (no reference counterpart: the
 * reference runs one device).  Host function, no GPU needed.  Outputs of an
 * xbatched / pbatched batch may alias (ylist[k] == ylist[k'] for entries
 * that add into one column); kron_owner_partition gives every output index
 * to exactly one of nranks ranks, with every entry that writes it, so each
 * rank finishes its outputs alone and no partial sums cross GPUs:
 *   rank r owns outputs [out_bounds[r], out_bounds[r+1]) and computes the
 *   entries entry_order[entry_bounds[r] .. entry_bounds[r+1]), listed by
 *   increasing output index, entries of one output in batch order.
 * The cuts balance entry counts as far as whole output groups allow.
 * ylist (batchCount non-negative ints), entry_order (batchCount),
 * entry_bounds and out_bounds (nranks + 1 each) are host arrays;
 * out_bounds[0] = 0, out_bounds[nranks] = 1 + max(ylist).
 * KRON_ERROR_INVALID_VALUE for a negative index or count, nranks < 1 or a
 * missing array; KRON_ERROR_ALLOC if host memory runs out.
 * ---------------------------------------------------------------------- */
int kron_owner_partition(int batchCount, int const ylist[], int nranks, int entry_order[],
                         int entry_bounds[], int out_bounds[]);

/* ------------------------------------------------------------------------
 * Repeated application with a fixed operand (no reference counterpart): an
 * iterative solver applies the same kron(A_1..A_d) to a new X every
 * iteration.  kron_l2_persist_async keeps [ptr, ptr + bytes) -- typically A
 * -- resident in L2 for the kernels launched on `stream` afterwards (a
 * persisting access-policy window on the stream, also captured into graphs
 * with the kernels; this context's persisting L2 carve-out is set to the
 * window, capped at the device maximum).  kron_l2_persist_reset clears the
 * window, returns the lines to normal and the carve-out to 0.  Both settings
 * end with the process.
 * ---------------------------------------------------------------------- */
int kron_l2_persist_async(const void *ptr, size_t bytes, kron_stream_t stream);
int kron_l2_persist_reset(kron_stream_t stream);

/* ------------------------------------------------------------------------
 * Autotuner (no reference counterpart).  For square shapes the library picks
 * among kernel variants, each with one tuning parameter:
 *   KRON_VARIANT_MMA8   FP64 tensor-core kernel for d = 3, n = 8
 *   KRON_VARIANT_PIPE   TMA-pipelined passes (n = 3..5, 4-64 KB vectors)
 *   KRON_VARIANT_SQ     on-chip square kernel; param = entries per thread
 *                       block (0: as many as fit)
 *   KRON_VARIANT_GEN    on-chip runtime-shape kernel
 *   KRON_VARIANT_BIG    cluster two-phase kernel; param = cluster size
 *                       (0: default), plus KRON_BIG_CUDA_CORES to keep
 *                       FP64 d = 6, n = 8 off the tensor cores (CUDA-core
 *                       FMAs; other shapes ignore the bit), plus
 *                       KRON_BIG_SMEM_W to keep the intermediate in the
 *                       cluster's shared memory instead of the workspace W
 *                       (FP64 d = 6, n = 6; that form also runs, without
 *                       the bit, when the caller passes no W), plus
 *                       KRON_BIG_NO_L2_HINTS to drop the L2 cache policies
 *                       that keep W resident (a comparison form)
 *   KRON_VARIANT_LARGE  two-phase launches through the workspace W
 *   KRON_VARIANT_SPLIT_TC  split precision (KRON_PREC_SPLIT) for d = 6,
 *                       n = 8 in the batched layout with W: the two phases'
 *                       8x8 mode products as exact BF16 slice products on the
 *                       tcgen05 tensor cores, FP32 accumulators, FP64
 *                       reconstruction (param unused)
 *   KRON_VARIANT_SLAB   slab-cluster kernel for d = 6, n = 6 (FP64 and
 *                       FP32): one cluster of 12 blocks per entry, each
 *                       block holding half of one n^5 slab, no workspace;
 *                       param bits (comparison forms): KRON_SLAB_WHOLE --
 *                       clusters of 6 blocks holding whole slabs;
 *                       KRON_SLAB_NO_ROTATE -- no lane rotation in its first
 *                       FP64 pass (which keeps that pass free of bank
 *                       conflicts); KRON_SLAB_PLAIN_Y -- distinct outputs
 *                       added by loads and stores instead of L2 atomics;
 *                       KRON_SLAB_NO_SIDE -- no side kernel: by default,
 *                       for FP64 batches of 512 entries or more with a
 *                       workspace W, a share of the entries runs
 *                       concurrently on the cluster two-phase kernel (a
 *                       library-owned second stream, joined by events) on
 *                       the SMs the 12-block clusters leave idle
 * kron_autotune times every variant that runs (d, n, precision) on a
 * synthetic batched problem of up to batchCount entries (capped at 1 GiB),
 * records the fastest for that key and returns it (outputs may be NULL).
 * It allocates and frees device memory and synchronises `stream`: call it
 * at set-up, outside stream capture.  Every later call with that square
 * shape and precision, in any layout, tries the recorded variant first and
 * falls back to the built-in choice when the variant cannot run it.
 * kron_tune_set records a choice by hand (variant 0 removes it),
 * kron_tune_get reads it (variant 0: none), kron_tune_save / _load keep the
 * table in a text file.  Precision codes: KRON_PREC_F64 (the drop-in and
 * segmented calls), KRON_PREC_F32 (kronmult_batched_f32_async),
 * KRON_PREC_SPLIT (kronmult_batched_split_async).
 * ---------------------------------------------------------------------- */
#define KRON_PREC_F64 0
#define KRON_PREC_F32 1
#define KRON_PREC_SPLIT 2
#define KRON_VARIANT_MMA8 1
#define KRON_VARIANT_PIPE 2
#define KRON_VARIANT_SQ 3
#define KRON_VARIANT_GEN 4
#define KRON_VARIANT_BIG 5
#define KRON_VARIANT_LARGE 6
#define KRON_VARIANT_SLAB 7
#define KRON_VARIANT_SPLIT_TC 8
#define KRON_BIG_CUDA_CORES 256
#define KRON_BIG_SMEM_W 512
#define KRON_BIG_NO_L2_HINTS 1024
#define KRON_SLAB_NO_ROTATE 1
#define KRON_SLAB_WHOLE 2
#define KRON_SLAB_PLAIN_Y 4
#define KRON_SLAB_NO_SIDE 8

int kron_autotune(int d, int n, int precision, int batchCount, int *variant, int *param,
                  double *best_us, kron_stream_t stream);
int kron_tune_set(int d, int n, int precision, int variant, int param);
int kron_tune_get(int d, int n, int precision, int *variant, int *param);
void kron_tune_clear(void);
int kron_tune_save(const char *path);
int kron_tune_load(const char *path);

#ifdef __cplusplus
} /* extern "C" */

/* ------------------------------------------------------------------------
 * The reference signatures, C++ linkage (mangled names identical to the
 * reference wrappers', e.g. _Z17kronmult6_batchediPKdPdS1_S1_i).  Each
 * forwards to its _async twin on stream 0 and records the status.
 * ---------------------------------------------------------------------- */
void kronmult1_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);
void kronmult2_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);
void kronmult3_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);
void kronmult4_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);
void kronmult5_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);
void kronmult6_batched(int n, double const Aarray_[], double Xarray_[], double Yarray_[],
                       double Warray_[], int batchCount);

void kronmult1_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);
void kronmult2_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);
void kronmult3_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);
void kronmult4_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);
void kronmult5_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);
void kronmult6_pbatched(int n, double const Aarray_[], double *Xarray_[], double *Yarray_[],
                        double *Warray_[], int batchCount);

void kronmult1_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);
void kronmult2_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);
void kronmult3_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);
void kronmult4_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);
void kronmult5_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);
void kronmult6_xbatched(int n, double const *const Aarray_[], int lda, double *Xarray_[],
                        double *Yarray_[], double *Warray_[], int batchCount,
                        int subbatchCount = 0);

void kronmult1_vbatched(int m1, int n1, double const *const Aarray_[], double *pX_[],
                        double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount);
void kronmult2_vbatched(int m1, int n1, int m2, int n2, double const *const Aarray_[],
                        double *pX_[], double *pY_[], double *W_, size_t Wcapacity_bytes,
                        int batchCount);
void kronmult3_vbatched(int m1, int n1, int m2, int n2, int m3, int n3,
                        double const *const Aarray_[], double *pX_[], double *pY_[], double *W_,
                        size_t Wcapacity_bytes, int batchCount);
void kronmult4_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4,
                        double const *const Aarray_[], double *pX_[], double *pY_[], double *W_,
                        size_t Wcapacity_bytes, int batchCount);
void kronmult5_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4, int m5,
                        int n5, double const *const Aarray_[], double *pX_[], double *pY_[],
                        double *W_, size_t Wcapacity_bytes, int batchCount);
void kronmult6_vbatched(int m1, int n1, int m2, int n2, int m3, int n3, int m4, int n4, int m5,
                        int n5, int m6, int n6, double const *const Aarray_[], double *pX_[],
                        double *pY_[], double *W_, size_t Wcapacity_bytes, int batchCount);

void kgemm_nn_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount);
void kgemm_nt_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount);
void kgemm_tt_batched(int mm, int nn, int kk, double alpha, double *const Aarray_[],
                      int const ldAarray_[], double *const Barray_[], int const ldBarray_[],
                      double beta, double *const Carray_[], int const ldCarray_[],
                      int batchCount);
#endif /* __cplusplus */

#endif /* KRONMULT_B200_H */

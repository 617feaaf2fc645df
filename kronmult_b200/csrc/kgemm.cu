// Batched small GEMM:  C_k = alpha op(A_k) op(B_k) + beta C_k
// Replaces kgemm_{nn,nt,tt}_batched (kgemm_nn_batched.hpp:7-58 and the
// device GEMMs kgemm_nn.hpp:12-203, kgemm_nt.hpp:10-202, kgemm_tt.hpp:10-200).
//
// Semantics kept from the reference: beta == 1 adds alpha*op(A)op(B) with
// atomics (C of different entries may alias, kgemm_nt.hpp:184-187),
// beta == 0 stores without reading C, any other beta is a read-modify-write.
//
// Design: entries up to 64 x 64 x 64 run on the FP64 tensor cores, one entry
// per block (kgemm_dmma_kernel, below).  Larger entries: one 64x64 output
// tile per block (16x16 threads, 4x4 outputs per thread), K staged through
// shared memory in steps of 16 with the operand transposes folded into the
// staging loads, FP64 FMA accumulation.
#include <algorithm>
#include <cstdlib>

#include "kron_launch.h"

namespace kron {

namespace {

constexpr int TM = 64, TN = 64, TK = 16;

template <int OP> // 0 = nn, 1 = nt, 2 = tt
__global__ void __launch_bounds__(256)
    kgemm_batched_kernel(int mm, int nn, int kk, double alpha, double *const *Aarr,
                         const int *ldAarr, double *const *Barr, const int *ldBarr, double beta,
                         double *const *Carr, const int *ldCarr, int batch, int tiles_m,
                         int tiles_n)
{
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  const long long ntiles = (long long)tiles_m * tiles_n;

  for (long long job = blockIdx.x; job < ntiles * batch; job += gridDim.x)
  {
    const int k    = (int)(job / ntiles);
    const int tile = (int)(job - (long long)k * ntiles);
    const int i0 = (tile % tiles_m) * TM, j0 = (tile / tiles_m) * TN;
    const double *A = Aarr[k];
    const double *B = Barr[k];
    double *C       = Carr[k];
    const long long ldA = ldAarr[k], ldB = ldBarr[k], ldC = ldCarr[k];

    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
        acc[a][b] = 0.0;

    for (int k0 = 0; k0 < kk; k0 += TK)
    {
      __syncthreads();
      // op(A) tile: rows i0..i0+63, cols k0..k0+15
      for (int q = threadIdx.x; q < TM * TK; q += 256)
      {
        int i, kq;
        if (OP == 2)
        { // A^T: element (i, kq) = A[kq + i*ldA]; consecutive threads walk kq
          kq = q % TK;
          i  = q / TK;
        }
        else
        { // element (i, kq) = A[i + kq*ldA]; consecutive threads walk i
          i  = q % TM;
          kq = q / TM;
        }
        const int gi = i0 + i, gk = k0 + kq;
        double v     = 0.0;
        if (gi < mm && gk < kk)
          v = (OP == 2) ? A[gk + gi * ldA] : A[gi + gk * ldA];
        As[kq][i] = v;
      }
      // op(B) tile: rows k0..k0+15, cols j0..j0+63
      for (int q = threadIdx.x; q < TK * TN; q += 256)
      {
        int j, kq;
        if (OP == 0)
        { // element (kq, j) = B[kq + j*ldB]
          kq = q % TK;
          j  = q / TK;
        }
        else
        { // B^T: element (kq, j) = B[j + kq*ldB]
          j  = q % TN;
          kq = q / TN;
        }
        const int gj = j0 + j, gk = k0 + kq;
        double v     = 0.0;
        if (gj < nn && gk < kk)
          v = (OP == 0) ? B[gk + gj * ldB] : B[gj + gk * ldB];
        Bs[kq][j] = v;
      }
      __syncthreads();
#pragma unroll
      for (int kq = 0; kq < TK; kq++)
      {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
        {
          a[u] = As[kq][tx + 16 * u];
          b[u] = Bs[kq][ty + 16 * u];
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
          for (int w = 0; w < 4; w++)
            acc[u][w] = fma(a[u], b[w], acc[u][w]);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
      for (int w = 0; w < 4; w++)
      {
        const int gi = i0 + tx + 16 * u, gj = j0 + ty + 16 * w;
        if (gi < mm && gj < nn)
        {
          double *c = C + gi + gj * ldC;
          if (beta == 1.0)
            atomicAdd(c, alpha * acc[u][w]);
          else if (beta == 0.0)
            *c = alpha * acc[u][w];
          else
            *c = beta * (*c) + alpha * acc[u][w];
        }
      }
  }
}

// ---------------------------------------------------------------------------
// Entries up to 64 x 64 x 64 on the FP64 tensor cores (mma.sync m8n8k4):
// one entry per block of four warps at a time, warp w computing the 32 x 32
// block of C at rows 32 (w / 2), columns 32 (w % 2) as 4 x 4 tiles of 8 x 8
// held in fragments (D[g][2t], D[g][2t+1] per lane 4g + t), K in steps of 4
// (A fragment op(A)[g][k], B fragment op(B)[k][g]).  op(A) and op(B) are
// staged in shared memory, zero padded to whole tiles, in the orientation
// that keeps both the global reads and the shared writes contiguous (stride
// 68 doubles, so the fragment reads of either orientation are conflict free:
// a half-warp's 16 lanes hit words 4g + t or 4t + g mod 16).
constexpr int DM_THREADS = 128;
constexpr int DM_S       = 68;
constexpr int DM_MAX     = 64;

__device__ __forceinline__ void dm_mma(double &d0, double &d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// dst = *src (8 bytes) by an asynchronous copy, or 0 when !valid (zero
// fill: nothing is read)
__device__ __forceinline__ void dm_cp8(double *dst, const double *src, bool valid)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(src),
               "r"(valid ? 8 : 0)
               : "memory");
}

template <int OP> // 0 = nn, 1 = nt, 2 = tt
__global__ void __launch_bounds__(DM_THREADS, 3)
    kgemm_dmma_kernel(int mm, int nn, int kk, double alpha, double *const *Aarr,
                      const int *ldAarr, double *const *Barr, const int *ldBarr, double beta,
                      double *const *Carr, const int *ldCarr, int batch)
{
  extern __shared__ double dm_smem[];
  double *As = dm_smem;                // op(A): [k][i] (nn, nt) or [i][k] (tt)
  double *Bs = dm_smem + DM_MAX * DM_S; // op(B): [j][k] (nn) or [k][j] (nt, tt)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int mt = (mm + 7) >> 3, nt = (nn + 7) >> 3, kt = (kk + 3) >> 2;
  const int rows = mt * 8, cols = nt * 8, kp = kt * 4;
  const int m0 = 4 * (warp >> 1), n0 = 4 * (warp & 1); // first tile of this warp
  constexpr bool A_KM = OP != 2; // A staged [k][i]
  constexpr bool B_NK = OP == 0; // B staged [j][k]

  for (int e = blockIdx.x; e < batch; e += gridDim.x)
  {
    const double *A     = Aarr[e];
    const double *B     = Barr[e];
    double *C           = Carr[e];
    const long long lda = ldAarr[e], ldb = ldBarr[e], ldc = ldCarr[e];
    __syncthreads(); // the previous entry's fragments are read
    // every copy of the entry in flight at once (zero fill outside mm, nn, kk)
    for (int q = tid; q < rows * kp; q += DM_THREADS)
    {
      if constexpr (A_KM)
      { // op(A)(i, k) = A[i + k lda]; consecutive threads walk i
        const int i = q % rows, k = q / rows;
        const bool ok = i < mm && k < kk;
        dm_cp8(As + k * DM_S + i, ok ? A + i + k * lda : A, ok);
      }
      else
      { // op(A)(i, k) = A[k + i lda]; consecutive threads walk k
        const int k = q % kp, i = q / kp;
        const bool ok = i < mm && k < kk;
        dm_cp8(As + i * DM_S + k, ok ? A + k + i * lda : A, ok);
      }
    }
    for (int q = tid; q < cols * kp; q += DM_THREADS)
    {
      if constexpr (B_NK)
      { // op(B)(k, j) = B[k + j ldb]; consecutive threads walk k
        const int k = q % kp, j = q / kp;
        const bool ok = j < nn && k < kk;
        dm_cp8(Bs + j * DM_S + k, ok ? B + k + j * ldb : B, ok);
      }
      else
      { // op(B)(k, j) = B[j + k ldb]; consecutive threads walk j
        const int j = q % cols, k = q / cols;
        const bool ok = j < nn && k < kk;
        dm_cp8(Bs + k * DM_S + j, ok ? B + j + k * ldb : B, ok);
      }
    }
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
    __syncthreads();

    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
        acc[a][b][0] = acc[a][b][1] = 0.0;
    for (int ks = 0; ks < kt; ks++)
    {
      const int k = ks * 4 + t;
      double af[4], bf[4];
#pragma unroll
      for (int u = 0; u < 4; u++)
      {
        const int r = (m0 + u) * 8 + g, c = (n0 + u) * 8 + g;
        af[u] = (m0 + u < mt) ? (A_KM ? As[k * DM_S + r] : As[r * DM_S + k]) : 0.0;
        bf[u] = (n0 + u < nt) ? (B_NK ? Bs[c * DM_S + k] : Bs[k * DM_S + c]) : 0.0;
      }
#pragma unroll
      for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
          if (m0 + a < mt && n0 + b < nt) // warp-uniform
            dm_mma(acc[a][b][0], acc[a][b][1], af[a], bf[b]);
    }
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
      for (int b = 0; b < 4; b++)
#pragma unroll
        for (int pp = 0; pp < 2; pp++)
        {
          const int i = (m0 + a) * 8 + g, j = (n0 + b) * 8 + 2 * t + pp;
          if (m0 + a < mt && n0 + b < nt && i < mm && j < nn)
          {
            double *c      = C + i + j * ldc;
            const double v = alpha * acc[a][b][pp];
            if (beta == 1.0)
              atomicAdd(c, v);
            else if (beta == 0.0)
              *c = v;
            else
              *c = beta * (*c) + v;
          }
        }
  }
}

template <int OP>
int launch_dmma(int mm, int nn, int kk, double alpha, double *const *A, const int *ldA,
                double *const *B, const int *ldB, double beta, double *const *C, const int *ldC,
                int batch, cudaStream_t stream)
{
  const void *fn    = reinterpret_cast<const void *>(&kgemm_dmma_kernel<OP>);
  const size_t smem = 2 * (size_t)DM_MAX * DM_S * sizeof(double);
  int per_sm        = 1;
  if (cached_occupancy(fn, DM_THREADS, smem, &per_sm) != KRON_SUCCESS)
    return KRON_ERROR_LAUNCH;
  const long long grid =
      std::max<long long>(1, std::min<long long>(batch, (long long)device_info().sms * per_sm));
  void *args[] = {&mm, &nn, &kk, &alpha, const_cast<double *const **>(&A),
                  const_cast<const int **>(&ldA), const_cast<double *const **>(&B),
                  const_cast<const int **>(&ldB), &beta, const_cast<double *const **>(&C),
                  const_cast<const int **>(&ldC), &batch};
  return cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(DM_THREADS), args, smem, stream) ==
                 cudaSuccess
             ? KRON_SUCCESS
             : KRON_ERROR_LAUNCH;
}

} // namespace

int launch_kgemm(int op, int mm, int nn, int kk, double alpha, double *const *A, const int *ldA,
                 double *const *B, const int *ldB, double beta, double *const *C,
                 const int *ldC, int batch, cudaStream_t stream)
{
  if (batch <= 0 || mm <= 0 || nn <= 0)
    return KRON_SUCCESS;
  // entries up to 64 x 64 x 64 (the reference tests' sizes) on the FP64
  // tensor cores, one entry per block
  if (mm <= DM_MAX && nn <= DM_MAX && kk <= DM_MAX && !std::getenv("KRON_KGEMM_CUDA_CORES"))
  {
    switch (op)
    {
    case 0: return launch_dmma<0>(mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, stream);
    case 1: return launch_dmma<1>(mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, stream);
    case 2: return launch_dmma<2>(mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, stream);
    default: return KRON_ERROR_INVALID_VALUE;
    }
  }
  const int tiles_m = (mm + TM - 1) / TM, tiles_n = (nn + TN - 1) / TN;
  const long long jobs = (long long)tiles_m * tiles_n * batch;
  const int sms        = device_info().sms;
  long long grid       = std::min<long long>(jobs, (long long)sms * 8);
  if (grid < 1)
    grid = 1;
  switch (op)
  {
  case 0:
    kgemm_batched_kernel<0><<<(unsigned)grid, 256, 0, stream>>>(
        mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, tiles_m, tiles_n);
    break;
  case 1:
    kgemm_batched_kernel<1><<<(unsigned)grid, 256, 0, stream>>>(
        mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, tiles_m, tiles_n);
    break;
  case 2:
    kgemm_batched_kernel<2><<<(unsigned)grid, 256, 0, stream>>>(
        mm, nn, kk, alpha, A, ldA, B, ldB, beta, C, ldC, batch, tiles_m, tiles_n);
    break;
  default: return KRON_ERROR_INVALID_VALUE;
  }
  return cudaGetLastError() == cudaSuccess ? KRON_SUCCESS : KRON_ERROR_LAUNCH;
}

} // namespace kron

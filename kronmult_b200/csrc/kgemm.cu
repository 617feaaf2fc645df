// Batched small GEMM:  C_k = alpha op(A_k) op(B_k) + beta C_k
// Replaces kgemm_{nn,nt,tt}_batched (kgemm_nn_batched.hpp:7-58 and the
// device GEMMs kgemm_nn.hpp:12-203, kgemm_nt.hpp:10-202, kgemm_tt.hpp:10-200).
//
// Semantics kept from the reference: beta == 1 adds alpha*op(A)op(B) with
// atomics (C of different entries may alias, kgemm_nt.hpp:184-187),
// beta == 0 stores without reading C, any other beta is a read-modify-write.
//
// Design: one 64x64 output tile per block (16x16 threads, 4x4 outputs per
// thread), K staged through shared memory in steps of 16 with the operand
// transposes folded into the staging loads, FP64 FMA accumulation.
#include "kron_internal.cuh"

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

} // namespace

int launch_kgemm(int op, int mm, int nn, int kk, double alpha, double *const *A, const int *ldA,
                 double *const *B, const int *ldB, double beta, double *const *C,
                 const int *ldC, int batch, cudaStream_t stream)
{
  if (batch <= 0 || mm <= 0 || nn <= 0)
    return KRON_SUCCESS;
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

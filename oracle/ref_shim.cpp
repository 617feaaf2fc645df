// Oracle support (test infrastructure only, never part of the product):
// a C-linkage shim over the reference KRONMULT CPU (OpenMP) implementation.
//
// The reference is a header-only template library.  Its per-entry host
// wrappers (kronmult6_batched.cpp etc.) cannot be linked together and
// include hip/hip_runtime.h unconditionally, so this translation unit
// includes the template headers directly -- exactly as the reference's own
// tests do -- and instantiates the CPU (non -DUSE_GPU) code path.
//
// Built by oracle/Makefile with -I<reference dir> into oracle/_ref/ (twice:
// the default recursive algorithm and -DUSE_ALG993), never copied here.
//
// Entry points mirror (reference file:line):
//   kronmult{d}_batched<T>   kronmult6_batched.hpp:12-75
//   kronmult{d}_pbatched<T>  kronmult6_pbatched.hpp:12-67
//   kronmult{d}_xbatched<T>  kronmult6_xbatched.hpp:10-31 -> kronmult_xbatched.hpp:17-162
//   kronmult{d}_vbatched<T>  kronmult6_vbatched.hpp:10-34 -> kronmult_vbatched.hpp:17-228
//   kgemm_{nn,nt,tt}_batched kgemm_nn_batched.hpp:7-58 (nt/tt analogous)
//   kron_flops               kroncommon.hpp:154-185

#include <cstdio>

#include "kroncommon.hpp"

#include "kronmult1_batched.hpp"
#include "kronmult2_batched.hpp"
#include "kronmult3_batched.hpp"
#include "kronmult4_batched.hpp"
#include "kronmult5_batched.hpp"
#include "kronmult6_batched.hpp"

#include "kronmult1_pbatched.hpp"
#include "kronmult2_pbatched.hpp"
#include "kronmult3_pbatched.hpp"
#include "kronmult4_pbatched.hpp"
#include "kronmult5_pbatched.hpp"
#include "kronmult6_pbatched.hpp"

#include "kronmult1_xbatched.hpp"
#include "kronmult2_xbatched.hpp"
#include "kronmult3_xbatched.hpp"
#include "kronmult4_xbatched.hpp"
#include "kronmult5_xbatched.hpp"
#include "kronmult6_xbatched.hpp"

#include "kronmult1_vbatched.hpp"
#include "kronmult2_vbatched.hpp"
#include "kronmult3_vbatched.hpp"
#include "kronmult4_vbatched.hpp"
#include "kronmult5_vbatched.hpp"
#include "kronmult6_vbatched.hpp"

#include "kgemm_nn_batched.hpp"
#include "kgemm_nt_batched.hpp"
#include "kgemm_tt_batched.hpp"

#include <omp.h>
#include <vector>

extern "C" {

int ref_uses_alg993(void)
{
#ifdef USE_ALG993
  return 1;
#else
  return 0;
#endif
}

int ref_max_threads(void) { return omp_get_max_threads(); }

void ref_set_threads(int nthreads)
{
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
}

double ref_kron_flops(int d, int const *m, int const *n)
{
  return kron_flops(d, m, n);
}

// Y(:,k) += kron(A1..Ad)(k) X(:,k); A is (n,n,d,batch); X and W are clobbered.
int ref_kronmult_batched(int d, int n, double const *A, double *X, double *Y,
                         double *W, int batch)
{
  switch (d)
  {
  case 1: kronmult1_batched<double>(n, A, X, Y, W, batch); break;
  case 2: kronmult2_batched<double>(n, A, X, Y, W, batch); break;
  case 3: kronmult3_batched<double>(n, A, X, Y, W, batch); break;
  case 4: kronmult4_batched<double>(n, A, X, Y, W, batch); break;
  case 5: kronmult5_batched<double>(n, A, X, Y, W, batch); break;
  case 6: kronmult6_batched<double>(n, A, X, Y, W, batch); break;
  default: return 1;
  }
  return 0;
}

int ref_kronmult_pbatched(int d, int n, double const *A, double **pX,
                          double **pY, double **pW, int batch)
{
  switch (d)
  {
  case 1: kronmult1_pbatched<double>(n, A, pX, pY, pW, batch); break;
  case 2: kronmult2_pbatched<double>(n, A, pX, pY, pW, batch); break;
  case 3: kronmult3_pbatched<double>(n, A, pX, pY, pW, batch); break;
  case 4: kronmult4_pbatched<double>(n, A, pX, pY, pW, batch); break;
  case 5: kronmult5_pbatched<double>(n, A, pX, pY, pW, batch); break;
  case 6: kronmult6_pbatched<double>(n, A, pX, pY, pW, batch); break;
  default: return 1;
  }
  return 0;
}

int ref_kronmult_xbatched(int d, int n, double const *const *pA, int lda,
                          double **pX, double **pY, double **pW, int batch,
                          int subbatch)
{
  switch (d)
  {
  case 1: kronmult1_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  case 2: kronmult2_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  case 3: kronmult3_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  case 4: kronmult4_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  case 5: kronmult5_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  case 6: kronmult6_xbatched<double>(n, pA, lda, pX, pY, pW, batch, subbatch); break;
  default: return 1;
  }
  return 0;
}

// Uniform rectangular shapes; m[], n[] have d entries.
int ref_kronmult_vbatched(int d, int const *m, int const *n,
                          double const *const *pA, double **pX, double **pY,
                          double *W, size_t Wcapacity_bytes, int batch)
{
  int mm[6] = {1, 1, 1, 1, 1, 1};
  int nn[6] = {1, 1, 1, 1, 1, 1};
  for (int i = 0; i < d && i < 6; i++)
  {
    mm[i] = m[i];
    nn[i] = n[i];
  }
  switch (d)
  {
  case 1:
    kronmult1_vbatched<double>(mm[0], nn[0], pA, pX, pY, W, Wcapacity_bytes, batch);
    break;
  case 2:
    kronmult2_vbatched<double>(mm[0], nn[0], mm[1], nn[1], pA, pX, pY, W,
                               Wcapacity_bytes, batch);
    break;
  case 3:
    kronmult3_vbatched<double>(mm[0], nn[0], mm[1], nn[1], mm[2], nn[2], pA,
                               pX, pY, W, Wcapacity_bytes, batch);
    break;
  case 4:
    kronmult4_vbatched<double>(mm[0], nn[0], mm[1], nn[1], mm[2], nn[2], mm[3],
                               nn[3], pA, pX, pY, W, Wcapacity_bytes, batch);
    break;
  case 5:
    kronmult5_vbatched<double>(mm[0], nn[0], mm[1], nn[1], mm[2], nn[2], mm[3],
                               nn[3], mm[4], nn[4], pA, pX, pY, W,
                               Wcapacity_bytes, batch);
    break;
  case 6:
    kronmult6_vbatched<double>(mm[0], nn[0], mm[1], nn[1], mm[2], nn[2], mm[3],
                               nn[3], mm[4], nn[4], mm[5], nn[5], pA, pX, pY, W,
                               Wcapacity_bytes, batch);
    break;
  default: return 1;
  }
  return 0;
}

// Uneven batch driven through the reference's kronmult{d}_vbatched one entry
// at a time (batchCount = 1; the reference has no per-entry-shape batch),
// entries spread over OpenMP threads, each with private workspace.
// shapes: 13 ints per entry {d, m1, n1, ..., m6, n6}; pA: 6 pointers per
// entry.  Outputs must not alias between entries.
int ref_kronmult_vbatched_entries(int nent, int const *shapes, double const *const *pA,
                                  double **pX, double **pY, size_t Wbytes_per_thread)
{
  int bad = 0;
#pragma omp parallel
  {
    std::vector<double> W(Wbytes_per_thread / sizeof(double) + 1);
#pragma omp for schedule(dynamic, 8)
    for (int k = 0; k < nent; k++)
    {
      int const *s = shapes + 13L * k;
      int m[6], n[6];
      for (int l = 0; l < 6; l++)
      {
        m[l] = s[1 + 2 * l];
        n[l] = s[2 + 2 * l];
      }
      int rc = ref_kronmult_vbatched(s[0], m, n, pA + 6L * k, pX + k, pY + k, W.data(),
                                     Wbytes_per_thread, 1);
      if (rc)
      {
#pragma omp atomic write
        bad = 1;
      }
    }
  }
  return bad;
}

// op: 0 = nn, 1 = nt, 2 = tt
int ref_kgemm_batched(int op, int mm, int nn, int kk, double alpha,
                      double *const *pA, int const *ldA, double *const *pB,
                      int const *ldB, double beta, double *const *pC,
                      int const *ldC, int batch)
{
  switch (op)
  {
  case 0:
    kgemm_nn_batched<double>(mm, nn, kk, alpha, pA, ldA, pB, ldB, beta, pC, ldC, batch);
    break;
  case 1:
    kgemm_nt_batched<double>(mm, nn, kk, alpha, pA, ldA, pB, ldB, beta, pC, ldC, batch);
    break;
  case 2:
    kgemm_tt_batched<double>(mm, nn, kk, alpha, pA, ldA, pB, ldB, beta, pC, ldC, batch);
    break;
  default: return 1;
  }
  return 0;
}

} // extern "C"

/*
 * ORACLE -- test infrastructure only.
 *
 * Plain-C restatement of the reference KRONMULT arithmetic, used by the test
 * suite, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg to
 * check the CUDA library.  Nothing in the product (kronmult_b200/, include/)
 * calls, links or loads this file.
 *
 * Parity is pinned two ways (tests/test_oracle.py):
 *   - against golden vectors produced by the reference's own CPU build
 *     (oracle/ref_shim.cpp compiled from the reference headers, see
 *     tests/golden/make_golden.py);
 *   - against the reference tests' known-answer construction (closed-form X
 *     and A, dense-Kronecker check), test_kronmult6_batched.cpp:117-154,
 *     345-406.
 *
 * Conventions (shared with the reference):
 *   - matrices are column major, A(i,j) at A[i + j*ld]   (kroncommon.hpp:72)
 *   - kron(A1,...,Ad) has A_d's index fastest in X and Y
 *     (test_kronmult6_batched.cpp:352-353,371-373)
 *   - Y is accumulated (+=), never overwritten
 */
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_MAXD 6

static long prod_int(int d, int const *v)
{
  long p = 1;
  for (int i = 0; i < d; i++)
    p *= v[i];
  return p;
}

/*
 * y += kron(A_1,...,A_d) x by successive mode products, A_1 (slowest index)
 * first.  Same contraction order as the reference's recursive algorithm
 * (kronmultv_recur.hpp:90-145: X * A1^T first, then recurse on A2..Ad).
 * A_l is m[l] x n[l] with leading dimension ld[l].
 * work must hold 2 * max intermediate size doubles (oracle_work_size()).
 */
long oracle_work_size(int d, int const *m, int const *n)
{
  long best = prod_int(d, n);
  for (int l = 0; l < d; l++)
  {
    /* size after applying modes 0..l: m_0..m_l, n_{l+1}..n_{d-1} */
    long s = 1;
    for (int k = 0; k < d; k++)
      s *= (k <= l) ? m[k] : n[k];
    if (s > best)
      best = s;
  }
  return 2 * best;
}

void oracle_kron_apply(int d, int const *m, int const *n,
                       double const *const *A, int const *ld,
                       double const *x, double *y, double *work)
{
  long cur_size = prod_int(d, n);
  long half     = oracle_work_size(d, m, n) / 2;
  double *bufs[2] = {work, work + half};
  int which       = 0;
  memcpy(bufs[0], x, sizeof(double) * (size_t)cur_size);

  for (int l = 0; l < d; l++)
  {
    long outer = 1, inner = 1;
    for (int k = 0; k < l; k++)
      outer *= m[k];
    for (int k = l + 1; k < d; k++)
      inner *= n[k];
    double const *in  = bufs[which];
    double *out       = bufs[1 - which];
    double const *Al  = A[l];
    int const ml = m[l], nl = n[l], ldl = ld[l];
    for (long o = 0; o < outer; o++)
      for (int i = 0; i < ml; i++)
        for (long r = 0; r < inner; r++)
        {
          double acc = 0.0;
          for (int j = 0; j < nl; j++)
            acc += Al[i + (long)j * ldl] * in[(o * nl + j) * inner + r];
          out[(o * ml + i) * inner + r] = acc;
        }
    which    = 1 - which;
    cur_size = outer * ml * inner;
  }
  for (long i = 0; i < cur_size; i++)
    y[i] += bufs[which][i];
}

/*
 * y += kron(A_1..A_d) x by the explicit dense Kronecker element
 * prod_l A_l(i_l, j_l) -- the reference tests' check
 * (test_kronmult6_batched.cpp:345-406), generalised to rectangular A_l.
 * O(M*N*d): small cases only.
 */
void oracle_kron_dense(int d, int const *m, int const *n,
                       double const *const *A, int const *ld,
                       double const *x, double *y)
{
  long M = prod_int(d, m), N = prod_int(d, n);
  int ii[ORACLE_MAXD], jj[ORACLE_MAXD];
  for (long io = 0; io < M; io++)
  {
    long t = io;
    for (int l = d - 1; l >= 0; l--)
    {
      ii[l] = (int)(t % m[l]);
      t /= m[l];
    }
    double acc = 0.0;
    for (long jo = 0; jo < N; jo++)
    {
      long u = jo;
      for (int l = d - 1; l >= 0; l--)
      {
        jj[l] = (int)(u % n[l]);
        u /= n[l];
      }
      double c = 1.0;
      for (int l = 0; l < d; l++)
        c *= A[l][ii[l] + (long)jj[l] * ld[l]];
      acc += c * x[jo];
    }
    y[io] += acc;
  }
}

/* ---- batch drivers (the reference's batch layouts) ---------------------- */

static int max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

int oracle_num_threads(void) { return max_threads(); }

void oracle_set_threads(int nthreads)
{
#ifdef _OPENMP
  if (nthreads > 0)
    omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
}

/* A is (n,n,d,batch) contiguous; X, Y are (n^d, batch)
 * (kronmult6_batched.hpp:16-19).  Distinct Y columns: no atomics needed. */
void oracle_kronmult_batched(int d, int n, double const *A, double const *X,
                             double *Y, int batch)
{
  int mv[ORACLE_MAXD], nv[ORACLE_MAXD], ldv[ORACLE_MAXD];
  for (int l = 0; l < d; l++)
  {
    mv[l] = n;
    nv[l] = n;
    ldv[l] = n;
  }
  long L  = prod_int(d, nv);
  long ws = oracle_work_size(d, mv, nv);
#pragma omp parallel
  {
    double *work = (double *)malloc(sizeof(double) * (size_t)ws);
#pragma omp for schedule(static)
    for (int k = 0; k < batch; k++)
    {
      double const *Ap[ORACLE_MAXD];
      for (int l = 0; l < d; l++)
        Ap[l] = A + ((long)k * d + l) * n * n;
      oracle_kron_apply(d, mv, nv, Ap, ldv, X + (long)k * L, Y + (long)k * L,
                        work);
    }
    free(work);
  }
}

/*
 * General pointer-array form used for pbatched/xbatched/vbatched: entry k
 * uses A pointers pA[l + k*d] with leading dimension ld[l], input pX[k],
 * output pY[k].  Outputs may alias between entries: each entry computes its
 * contribution into private storage and adds it under a critical section
 * (the reference's CPU atomicAdd shim, kroncommon.hpp:35-59).
 */
void oracle_kronmult_general(int d, int const *m, int const *n,
                             double const *const *pA, int const *ld,
                             double const *const *pX, double *const *pY,
                             int batch)
{
  long M  = prod_int(d, m);
  long ws = oracle_work_size(d, m, n);
#pragma omp parallel
  {
    double *work = (double *)malloc(sizeof(double) * (size_t)ws);
    double *ybuf = (double *)malloc(sizeof(double) * (size_t)M);
#pragma omp for schedule(dynamic, 16)
    for (int k = 0; k < batch; k++)
    {
      memset(ybuf, 0, sizeof(double) * (size_t)M);
      oracle_kron_apply(d, m, n, pA + (long)k * d, ld, pX[k], ybuf, work);
      double *yk = pY[k];
#pragma omp critical(oracle_y)
      for (long i = 0; i < M; i++)
        yk[i] += ybuf[i];
    }
    free(ybuf);
    free(work);
  }
}

/* ---- kgemm (kgemm_nn.hpp, kgemm_nt.hpp, kgemm_tt.hpp) --------------------
 * C = alpha op(A) op(B) + beta C, op = N or T; beta == 0 never reads C.
 * op: 0 = nn (C = A B), 1 = nt (C = A B^T), 2 = tt (C = A^T B^T).
 */
void oracle_kgemm(int op, int mm, int nn, int kk, double alpha, double const *A,
                  int ldA, double const *B, int ldB, double beta, double *C,
                  int ldC)
{
  for (int j = 0; j < nn; j++)
    for (int i = 0; i < mm; i++)
    {
      double acc = 0.0;
      for (int k = 0; k < kk; k++)
      {
        double a = (op == 2) ? A[k + (long)i * ldA] : A[i + (long)k * ldA];
        double b = (op == 0) ? B[k + (long)j * ldB] : B[j + (long)k * ldB];
        acc += a * b;
      }
      double *c = &C[i + (long)j * ldC];
      if (beta == 0.0)
        *c = alpha * acc;
      else
        *c = beta * (*c) + alpha * acc;
    }
}

void oracle_kgemm_batched(int op, int mm, int nn, int kk, double alpha,
                          double const *const *pA, int const *ldA,
                          double const *const *pB, int const *ldB, double beta,
                          double *const *pC, int const *ldC, int batch)
{
  /* entries may share C when beta == 1 (the atomic case): keep it serial */
  for (int k = 0; k < batch; k++)
    oracle_kgemm(op, mm, nn, kk, alpha, pA[k], ldA[k], pB[k], ldB[k], beta,
                 pC[k], ldC[k]);
}

/* ---- flop counts --------------------------------------------------------- */

/* kroncommon.hpp:154-185: recursive count, A_1 applied first as
 * X * A1^T then d-1 levels on m_1 vectors. */
double oracle_kron_flops(int d, int const *m, int const *n)
{
  if (d <= 0)
    return 0.0;
  if (d == 1)
    return 2.0 * m[0] * n[0];
  double rest_n = 1.0;
  for (int l = 1; l < d; l++)
    rest_n *= n[l];
  double first = 2.0 * rest_n * n[0] * m[0];
  return first + (double)m[0] * oracle_kron_flops(d - 1, m + 1, n + 1);
}

/* kronm.hpp:39-81: Alg. 993 forward (A_1 first) and backward (A_d first). */
double oracle_flops_forward(int d, int const *m, int const *n)
{
  double size = (double)prod_int(d, n), total = 0.0;
  for (int l = 0; l < d; l++)
  {
    double cols = size / n[l];
    total += 2.0 * m[l] * cols * n[l];
    size = m[l] * cols;
  }
  return total;
}

double oracle_flops_backward(int d, int const *m, int const *n)
{
  double size = (double)prod_int(d, n), total = 0.0;
  for (int l = d - 1; l >= 0; l--)
  {
    double rows = size / n[l];
    total += 2.0 * rows * m[l] * n[l];
    size = rows * m[l];
  }
  return total;
}

/* kronm.hpp:89: forward only when strictly cheaper (ties go backward). */
int oracle_use_forward(int d, int const *m, int const *n)
{
  return oracle_flops_forward(d, m, n) < oracle_flops_backward(d, m, n);
}

// FP64 tensor-core building block shared by the 8x8-factor kernels: one warp
// applies kron(A_1, A_2, A_3) (8x8 each) to a 512-element block held in
// mma.sync f64 fragments and adds the result into its accumulators.
//
//   input  v[q][p]   = X(j0 = q, j1 = g, j2 = 2t+p)     (G=j1, P=j2, Q=j0)
//   output acc[q][p] += Y(i0 = 2t+p, i1 = q, i2 = g)     (G=i2, P=i0, Q=i1)
//
// with lane = 4g + t.  Mode 3 runs as m8n8k4 with A_3 as the A operand,
// modes 2 and 1 as m16n8k8 with the data as the A operand; one quad-local
// transpose of 2x2 blocks goes through a 512-double shared buffer (XOR
// swizzled; both sides conflict free).  The K order implied by reusing an
// accumulator as the next operand (k = t holds column 2t, k = t+4 column
// 2t+1) is absorbed by permuting the rows of the constant A fragments.
#pragma once

#include "kron_internal.cuh"

namespace kron {

__device__ __forceinline__ void mma884(double &d0, double &d1, double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void mma1688(double &c0, double &c1, double &c2, double &c3, double a0,
                                        double a1, double a2, double a3, double b0, double b1)
{
  asm volatile("mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, "
               "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
               : "+d"(c0), "+d"(c1), "+d"(c2), "+d"(c3)
               : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}


struct AFrag8
{
  double a3[2]; // A_3(g, 2t+s), s = 0,1   (A operand of the m8n8k4 steps)
  double b2[2]; // A_2(g, 2t), A_2(g, 2t+1) (B operand, K rows permuted)
  double b1[2]; // A_1(g, 2t), A_1(g, 2t+1)
};

// A_1, A_2, A_3 column major with leading dimensions ld1..ld3.
__device__ __forceinline__ void load_afrag8(AFrag8 &f, const double *A1, int ld1,
                                            const double *A2, int ld2, const double *A3, int ld3,
                                            int g, int t)
{
  f.b1[0] = __ldg(A1 + g + (long long)(2 * t) * ld1);
  f.b1[1] = __ldg(A1 + g + (long long)(2 * t + 1) * ld1);
  f.b2[0] = __ldg(A2 + g + (long long)(2 * t) * ld2);
  f.b2[1] = __ldg(A2 + g + (long long)(2 * t + 1) * ld2);
  f.a3[0] = __ldg(A3 + g + (long long)(2 * t) * ld3);
  f.a3[1] = __ldg(A3 + g + (long long)(2 * t + 1) * ld3);
}

// v is consumed; sw (512 doubles, per warp) may be the buffer v was read from.
__device__ __forceinline__ void kron8x3_tile(double (&v)[8][2], double (&acc)[8][2],
                                             const AFrag8 &fc, double *xs, int g, int t)
{
    // ---- mode 3 (contract j2): D(i2, j1) = A_3 * X_q, m8n8k4, K = j2 as {2t, 2t+1}
    double r[8][2];
#pragma unroll
    for (int q = 0; q < 8; q++)
    {
      r[q][0] = r[q][1] = 0.0;
      mma884(r[q][0], r[q][1], fc.a3[0], v[q][0]);
      mma884(r[q][0], r[q][1], fc.a3[1], v[q][1]);
    }
    // r[q][p] = T(j0 = q, i2 = g, j1 = 2t+p)

    // ---- mode 2 (contract j1): rows (tile q, i2 = g), K = j1, B = A_2^T
#pragma unroll
    for (int rr = 0; rr < 4; rr++)
    {
      double c0 = 0.0, c1 = 0.0, c2 = 0.0, c3 = 0.0;
      mma1688(c0, c1, c2, c3, r[2 * rr][0], r[2 * rr + 1][0], r[2 * rr][1], r[2 * rr + 1][1],
              fc.b2[0], fc.b2[1]);
      v[2 * rr][0]     = c0;
      v[2 * rr][1]     = c1;
      v[2 * rr + 1][0] = c2;
      v[2 * rr + 1][1] = c3;
    }
    // v[q][p] = U(j0 = q, i2 = g, i1 = 2t+p)

    // ---- transpose P <-> Q inside each quad: 2x2 blocks (i1 pair a, j0 pair b)
    // block (a, b) of lane-group g at 32-byte slot g*16 + a*4 + (b ^ a); its two
    // 16-byte halves swap places for odd g so both sides are conflict free.
    {
      __syncwarp(); // every lane has read its X tile from xs
      const int gpar = g & 1;
#pragma unroll
      for (int b = 0; b < 4; b++)
      {
        double *blk = xs + 4 * (g * 16 + t * 4 + (b ^ t));
        // half 0: (i1 = 2t, j0 = 2b, 2b+1); half 1: (i1 = 2t+1, ...)
        *reinterpret_cast<double2 *>(blk + 2 * gpar) = make_double2(v[2 * b][0], v[2 * b + 1][0]);
        *reinterpret_cast<double2 *>(blk + 2 * (1 - gpar)) =
            make_double2(v[2 * b][1], v[2 * b + 1][1]);
      }
      __syncwarp();
#pragma unroll
      for (int a = 0; a < 4; a++)
      {
        const double *blk = xs + 4 * (g * 16 + a * 4 + (t ^ a));
        double2 h0 = *reinterpret_cast<const double2 *>(blk + 2 * gpar);       // i1 = 2a
        double2 h1 = *reinterpret_cast<const double2 *>(blk + 2 * (1 - gpar)); // i1 = 2a+1
        r[2 * a][0]     = h0.x; // (i1 = 2a,   j0 = 2t)
        r[2 * a][1]     = h0.y; // (i1 = 2a,   j0 = 2t+1)
        r[2 * a + 1][0] = h1.x;
        r[2 * a + 1][1] = h1.y;
      }
    }
    // r[q][p] = U(i1 = q, i2 = g, j0 = 2t+p)

    // ---- mode 1 (contract j0), accumulate into the output-group sum
#pragma unroll
    for (int rr = 0; rr < 4; rr++)
      mma1688(acc[2 * rr][0], acc[2 * rr][1], acc[2 * rr + 1][0], acc[2 * rr + 1][1],
              r[2 * rr][0], r[2 * rr + 1][0], r[2 * rr][1], r[2 * rr + 1][1], fc.b1[0],
              fc.b1[1]);
    // acc[q][p] = Y(i0 = 2t+p, i1 = q, i2 = g)

}

} // namespace kron

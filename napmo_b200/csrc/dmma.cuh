// FP64 tensor-core tile product (DMMA) shared by the density, quadrature and
// Poisson projection kernels.
#pragma once

namespace napmo {

// d += a (16x8, row) * b (8x8, col), FP64.  Fragments (g = lane / 4,
// q = lane % 4): a = {A[g][q], A[g+8][q], A[g][q+4], A[g+8][q+4]},
// b = {B[q][g], B[q+4][g]}, d = {C[g][2q], C[g][2q+1], C[g+8][2q], C[g+8][2q+1]}.
__device__ __forceinline__ void dmma(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

}  // namespace napmo

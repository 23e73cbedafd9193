// element.cuh -- P1 element geometry, element matrices' building blocks and
// the scatter into CSR values, shared by the assembly kernels (assembly.cu)
// and the batched solver (batch.cu).
#pragma once

#include "internal.cuh"

namespace ofg {
namespace elem {

constexpr double kThird = 0.33333333333333333333333333333;  // util/constants.h:70
constexpr double kSixth = 0.16666666666666666666666666667;  // util/constants.h:78

__device__ __forceinline__ double dot3(const double* a, const double* b)
{
   return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

// Triang3::set (src/shape_functions/Triang3.cpp:68-93)
__device__ __forceinline__ bool tri3(const double* xy, const int32_t* en, double g[3][3],
                                     double& area)
{
   double x0 = xy[2 * en[0]], y0 = xy[2 * en[0] + 1];
   double x1 = xy[2 * en[1]], y1 = xy[2 * en[1] + 1];
   double x2 = xy[2 * en[2]], y2 = xy[2 * en[2] + 1];
   double det = (x1 - x0) * (y2 - y0) - (y1 - y0) * (x2 - x0);
   area = 0.5 * det;
   if (!(det > 0.0)) return false;
   g[0][0] = (y1 - y2) / det; g[0][1] = (x2 - x1) / det; g[0][2] = 0.0;
   g[1][0] = (y2 - y0) / det; g[1][1] = (x0 - x2) / det; g[1][2] = 0.0;
   g[2][0] = (y0 - y1) / det; g[2][1] = (x1 - x0) / det; g[2][2] = 0.0;
   return true;
}

// Tetra4::CalculateShape (src/shape_functions/Tetra4.cpp:76-114): Jacobian,
// its cofactors, det, gradients J^{-T} grad(phi_ref); volume det/6.
__device__ __forceinline__ bool tet4(const double* xyz, const int32_t* en, double g[4][3],
                                     double& vol)
{
   double X[4][3];
#pragma unroll
   for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int d = 0; d < 3; ++d) X[k][d] = xyz[3 * en[k] + d];
   // J(r,c) = sum_k dphi_k/dxi_c * x_k[r]; reference gradients (-1,-1,-1), e1, e2, e3
   double J[3][3];
#pragma unroll
   for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) J[r][c] = X[c + 1][r] - X[0][r];
   double C[3][3];  // C[a][b] = cofactor matrix entry IJ(a+1,b+1) of the reference
#pragma unroll
   for (int i = 0; i < 3; ++i) {
      int j = (i + 1) % 3, k = (j + 1) % 3;
      C[i][i] = J[j][j] * J[k][k] - J[j][k] * J[k][j];
      C[j][i] = J[j][k] * J[k][i] - J[j][i] * J[k][k];
      C[i][j] = J[k][j] * J[i][k] - J[i][j] * J[k][k];
   }
   double det = J[0][0] * C[0][0] + J[1][0] * C[0][1] + J[2][0] * C[0][2];
   vol = kSixth * det;
   if (!(det > 0.0)) return false;
   double c = 1.0 / det;
   const double dl[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
#pragma unroll
   for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int d = 0; d < 3; ++d)
         g[i][d] = c * (C[0][d] * dl[i][0] + C[1][d] * dl[i][1] + C[2][d] * dl[i][2]);
   return true;
}

template <int NEN>
__device__ __forceinline__ void scatter(int64_t e, const int32_t* en, const int32_t* dof,
                                        const int32_t* __restrict__ emap, const double (&Ke)[NEN][NEN],
                                        const double (&Fe)[NEN], double* a, double* b)
{
   const int32_t* mp = emap + e * NEN * NEN;
#pragma unroll
   for (int i = 0; i < NEN; ++i) {
      int32_t r = dof[en[i]];
      if (!r) continue;
#pragma unroll
      for (int j = 0; j < NEN; ++j) {
         int32_t pos = mp[i * NEN + j];
         if (pos >= 0) a[pos] += Ke[i][j];
      }
      b[r - 1] += Fe[i];
   }
}

// Equation::updateBC (include/equations/Equation_impl.h:160-176)
template <int NEN>
__device__ __forceinline__ void lift_bc(const int32_t* en, const int32_t* code, const double* bc,
                                        const double (&Ke)[NEN][NEN], double (&Fe)[NEN])
{
#pragma unroll
   for (int j = 0; j < NEN; ++j) {
      if (code[en[j]] > 0) {
         double v = bc[en[j]];
#pragma unroll
         for (int i = 0; i < NEN; ++i) Fe[i] -= Ke[i][j] * v;
      }
   }
}

}  // namespace elem
}  // namespace ofg

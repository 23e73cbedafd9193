// element.cuh -- P1 element geometry, the element rows of the equations on
// the path and the row gather into CSR values, shared by the assembly kernel
// (assembly.cu) and the batched solver (batch.cu).
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

// Each element kind computes row li of its element matrix and RHS -- the row
// of the thread's own node i = en[li] -- with the arithmetic of the full
// element computation (the same products and sums in the same order), and
// lifts imposed values as Equation::updateBC does
// (include/equations/Equation_impl.h:160-176): a column j whose DOF is
// imposed (CSR position -1 in the element map) with code > 0 subtracts
// Ke(li, j) * bc(en[j]).  Only the node's own source value and the imposed
// columns' codes and values are loaded.

template <int NEN>
__device__ __forceinline__ void lift_row(const int32_t (&en)[NEN], const int32_t (&pos)[NEN],
                                         const int32_t* code, const double* bc,
                                         const double (&krow)[NEN], double& frow)
{
#pragma unroll
   for (int j = 0; j < NEN; ++j)
      if (pos[j] < 0 && code[en[j]] > 0) frow -= krow[j] * bc[en[j]];
}

// g[li] without dynamic register indexing
template <int NEN>
__device__ __forceinline__ void gradient_of(const double (&g)[NEN][3], int li, double (&gl)[3])
{
   gl[0] = g[0][0], gl[1] = g[0][1], gl[2] = g[0][2];
#pragma unroll
   for (int t = 1; t < NEN; ++t)
      if (t == li) gl[0] = g[t][0], gl[1] = g[t][1], gl[2] = g[t][2];
}

// Laplace2DT3::LHS (times k) + BodyRHS: Ke = area*(g_i.g_j)*k, Fe = f*area/3
// (src/equations/laplace/Laplace2DT3.cpp:131-143)
struct LaplaceT3 {
   static constexpr int NEN = 3;
   const double* xy;
   const int32_t* code;
   const double* kel;
   const double* f;
   const double* bc;
   __device__ __forceinline__ bool geometry_ok(const int32_t (&en)[3]) const
   {
      double g[3][3], area;
      return tri3(xy, en, g, area);
   }
   __device__ __forceinline__ bool row(int64_t e, const int32_t (&en)[3], int li, int64_t node,
                                       const int32_t (&pos)[3], double (&krow)[3],
                                       double& frow) const
   {
      double g[3][3], area, gl[3];
      if (!tri3(xy, en, g, area)) return false;
      gradient_of<3>(g, li, gl);
      const double k = kel ? kel[e] : 1.0;
#pragma unroll
      for (int j = 0; j < 3; ++j) krow[j] = area * dot3(gl, g[j]) * k;
      frow = f ? f[node] * area * kThird : 0.0;
      if (bc) lift_row<3>(en, pos, code, bc, krow, frow);
      return true;
   }
};

// DC3DT4::Diffusion(k) + BodyRHS: Ke = (k*vol)*(g_i.g_j), Fe = f*vol/4
// (src/equations/therm/DC3DT4.cpp:128-135, 207-211)
struct DiffusionT4 {
   static constexpr int NEN = 4;
   const double* xyz;
   const int32_t* code;
   const double* kel;
   const double* f;
   const double* bc;
   __device__ __forceinline__ bool geometry_ok(const int32_t (&en)[4]) const
   {
      double g[4][3], vol;
      return tet4(xyz, en, g, vol);
   }
   __device__ __forceinline__ bool row(int64_t e, const int32_t (&en)[4], int li, int64_t node,
                                       const int32_t (&pos)[4], double (&krow)[4],
                                       double& frow) const
   {
      double g[4][3], vol, gl[3];
      if (!tet4(xyz, en, g, vol)) return false;
      gradient_of<4>(g, li, gl);
      const double c = (kel ? kel[e] : 1.0) * vol;
#pragma unroll
      for (int j = 0; j < 4; ++j) krow[j] = c * dot3(gl, g[j]);
      frow = f ? f[node] * 0.25 * vol : 0.0;
      if (bc) lift_row<4>(en, pos, code, bc, krow, frow);
      return true;
   }
};

// DC2DT3 under OFELI's time schemes (Equa_Therm::build,
// include/equations/therm/Equa_Therm.h:162-218): eA1 = Capacity + LCapacity
// (src/equations/therm/DC2DT3.cpp:121-138), eA0 = Diffusion(eps) +
// Convection (:141-147, 185-207); with dti = 1/dt,
//   BACKWARD_EULER (2): eMat = dti eA1 + eA0,       eRHS += (dti eA1) u_old
//   FORWARD_EULER  (1): eMat = dti eA1,             eRHS += (dti eA1 - eA0) u_old
//   CRANK_NICOLSON (3): eMat = dti eA1 + 0.5 eA0,   eRHS += (dti eA1 - 0.5 eA0) u_old
// after updateBC has lifted the imposed values with eMat.
struct ConvDiffT3 {
   static constexpr int NEN = 3;
   const double* xy;
   const int32_t* code;
   double eps, dti;
   const double* v;
   const double* u_old;
   const double* bc;
   int scheme;
   __device__ __forceinline__ bool geometry_ok(const int32_t (&en)[3]) const
   {
      double g[3][3], area;
      return tri3(xy, en, g, area);
   }
   __device__ __forceinline__ bool row(int64_t, const int32_t (&en)[3], int li, int64_t,
                                       const int32_t (&pos)[3], double (&krow)[3],
                                       double& frow) const
   {
      double g[3][3], area, gl[3];
      if (!tri3(xy, en, g, area)) return false;
      gradient_of<3>(g, li, gl);
      const double cc = kSixth * area, dd = 0.5 * cc, cl = kThird * area;
      const double v3[3] = {v[2 * en[0]] + v[2 * en[1]] + v[2 * en[2]],
                            v[2 * en[0] + 1] + v[2 * en[1] + 1] + v[2 * en[2] + 1], 0.0};
      const double cv = kThird * kThird * area;
      double m1row[3], a0row[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
         const double m1 = (li == j) ? cc + cl : dd;
         m1row[j] = dti * m1;
         a0row[j] = eps * area * dot3(gl, g[j]) + cv * dot3(v3, g[j]);
         krow[j] = scheme == 1 ? m1row[j] : scheme == 3 ? m1row[j] + 0.5 * a0row[j]
                                                        : m1row[j] + a0row[j];
      }
      frow = 0.0;
      if (bc) lift_row<3>(en, pos, code, bc, krow, frow);
      double r[3];
#pragma unroll
      for (int j = 0; j < 3; ++j)
         r[j] = scheme == 1 ? m1row[j] - a0row[j] : scheme == 3 ? m1row[j] - 0.5 * a0row[j]
                                                                : m1row[j];
      frow += r[0] * u_old[en[0]] + r[1] * u_old[en[1]] + r[2] * u_old[en[2]];
      return true;
   }
};

// The rows of one node, gathered over its elements in ascending order:
// zeroes the node's CSR row (when it has an equation), adds its row of each
// element there and returns the RHS entry; the Jacobian of an element is
// checked by the thread of its first node and a bad element reported through
// report(e).  Used by the single-problem kernel (assembly.cu) and the
// batched solver (batch.cu).  The connectivity of the next element is loaded
// while the current one is computed.
// longest row summed in shared memory by gather_node_rows
constexpr int kRowAcc = 16;

template <class Elem, class Report>
__device__ __forceinline__ double gather_node_rows(int64_t i, int32_t r, int32_t q0, int32_t q1,
                                                   const int32_t* __restrict__ n2e,
                                                   const int32_t* __restrict__ elem,
                                                   const int32_t* __restrict__ emap,
                                                   const int32_t* __restrict__ row_ptr,
                                                   const Elem& el, double* __restrict__ a,
                                                   Report&& report, double* racc = nullptr,
                                                   int rstride = 0)
{
   constexpr int NEN = Elem::NEN;
   // the row is summed in racc (entry j at racc[j * rstride], shared
   // memory) when given and the row fits, then stored once; the additions
   // are the same, in the same order, as in place
   int32_t rs = 0, rl = 0;
   bool local = false;
   if (r) {
      rs = row_ptr[r - 1];
      rl = row_ptr[r] - rs;
      local = racc != nullptr && rl <= kRowAcc;
      if (local)
         for (int32_t j = 0; j < rl; ++j) racc[j * rstride] = 0.0;
      else
         for (int32_t k = rs; k < rs + rl; ++k) a[k] = 0.0;
   }
   double bi = 0.0;
   int64_t e_next = q0 < q1 ? n2e[q0] : 0;
   int32_t en_next[NEN];
#pragma unroll
   for (int j = 0; j < NEN; ++j) en_next[j] = q0 < q1 ? elem[NEN * e_next + j] : 0;
   for (int32_t q = q0; q < q1; ++q) {
      const int64_t e = e_next;
      int32_t en[NEN];
#pragma unroll
      for (int j = 0; j < NEN; ++j) en[j] = en_next[j];
      if (q + 1 < q1) {
         e_next = n2e[q + 1];
#pragma unroll
         for (int j = 0; j < NEN; ++j) en_next[j] = elem[NEN * e_next + j];
      }
      int li = 0;
#pragma unroll
      for (int j = NEN - 1; j > 0; --j)
         if (en[j] == (int32_t)i) li = j;
      if (!r) {   // no row here: only the Jacobian check of the elements it leads
         if (li == 0 && !el.geometry_ok(en)) report(e);
         continue;
      }
      int32_t pos[NEN];
      const int32_t* mp = emap + (e * NEN + li) * NEN;
#pragma unroll
      for (int j = 0; j < NEN; ++j) pos[j] = mp[j];
      double krow[NEN], frow;
      if (!el.row(e, en, li, i, pos, krow, frow)) {
         if (li == 0) report(e);
         continue;
      }
      if (local) {
#pragma unroll
         for (int j = 0; j < NEN; ++j)
            if (pos[j] >= 0) racc[(pos[j] - rs) * rstride] += krow[j];
      }
      else {
#pragma unroll
         for (int j = 0; j < NEN; ++j)
            if (pos[j] >= 0) a[pos[j]] += krow[j];
      }
      bi += frow;
   }
   if (local)
      for (int32_t j = 0; j < rl; ++j) a[rs + j] = racc[j * rstride];
   return bi;
}

}  // namespace elem
}  // namespace ofg

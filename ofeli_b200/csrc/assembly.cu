// assembly.cu -- Equation::build() for P1 elements on the device.
//
// One thread per mesh node gathers the CSR row of the node's equation and its
// RHS entry: it zeroes the row, then walks the node's elements in ascending
// element number (the node-to-element lists are sorted), computes each
// element's matrix and RHS in registers (FP64, the same formulas as
// Triang3/Tetra4 and the element classes, imposed values lifted as
// Equation::updateBC does) and adds the element row into its own CSR row and
// RHS entry.  Every matrix entry and RHS entry therefore receives its element
// contributions in OFELI's element-loop order, starting from zero, so the
// assembled values are the reference's bit for bit on any mesh; a thread
// writes only its own row, so there are no atomics and no element colouring.
// Each node computes only its own row of an element (geometry is recomputed
// by each of the element's 3 or 4 nodes; the FP64 arithmetic is cheap beside
// the gathers).  An element's Jacobian is checked by
// the thread of its first node, equation or not, and the lowest bad element
// is reported as OFELI's element loop would meet it first.
//
// Algorithmic bytes per launch: node-to-element lists 4*(nn+1) + 4*nen*ne,
// connectivity 4*nen*ne, coordinates 8*dim*nn, code and equation number
// 8*nn, the element-to-CSR map 4*nen^2*ne, the node fields read
// (f, or u_old and v) 8*nn each, k 8*ne when given, CSR row pointers
// 4*(n+1), A written 8*nnz,
// b written 8*n.
#include "element.cuh"

namespace ofg {
namespace {

using namespace elem;

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

// DC2DT3 under backward Euler (include/equations/therm/Equa_Therm.h:162-218):
// eA1 = Capacity + LCapacity (src/equations/therm/DC2DT3.cpp:121-138),
// eA0 = Diffusion(eps) + Convection (:141-147, 185-207),
// eMat = eA1/dt + eA0, eRHS = updateBC + (eA1/dt) u_old.
struct ConvDiffT3 {
   static constexpr int NEN = 3;
   const double* xy;
   const int32_t* code;
   double eps, dti;
   const double* v;
   const double* u_old;
   const double* bc;
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
      double m1row[3];
#pragma unroll
      for (int j = 0; j < 3; ++j) {
         const double m1 = (li == j) ? cc + cl : dd;
         m1row[j] = dti * m1;
         krow[j] = m1row[j] + (eps * area * dot3(gl, g[j]) + cv * dot3(v3, g[j]));
      }
      frow = 0.0;
      if (bc) lift_row<3>(en, pos, code, bc, krow, frow);
      frow += m1row[0] * u_old[en[0]] + m1row[1] * u_old[en[1]] + m1row[2] * u_old[en[2]];
      return true;
   }
};

// One thread per node: the node's CSR row and RHS entry, gathered over its
// elements in ascending order (see the file comment).
template <class Elem>
__global__ void __launch_bounds__(256) assemble_rows(int64_t nn, const int32_t* __restrict__ n2e_ptr,
                                                     const int32_t* __restrict__ n2e,
                                                     const int32_t* __restrict__ elem,
                                                     const int32_t* __restrict__ dof,
                                                     const int32_t* __restrict__ emap,
                                                     const int32_t* __restrict__ row_ptr, Elem el,
                                                     double* __restrict__ a, double* __restrict__ b,
                                                     int* bad)
{
   constexpr int NEN = Elem::NEN;
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride) {
      const int32_t r = dof[i];   // 1-based equation, 0 for an imposed node
      if (r)
         for (int32_t k = row_ptr[r - 1]; k < row_ptr[r]; ++k) a[k] = 0.0;
      double bi = 0.0;
      const int32_t q0 = n2e_ptr[i], q1 = n2e_ptr[i + 1];
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
            if (li == 0 && !el.geometry_ok(en)) atomicMin(bad, (int)e);
            continue;
         }
         int32_t pos[NEN];
         const int32_t* mp = emap + (e * NEN + li) * NEN;
#pragma unroll
         for (int j = 0; j < NEN; ++j) pos[j] = mp[j];
         double krow[NEN], frow;
         if (!el.row(e, en, li, i, pos, krow, frow)) {
            if (li == 0) atomicMin(bad, (int)e);
            continue;
         }
#pragma unroll
         for (int j = 0; j < NEN; ++j)
            if (pos[j] >= 0) a[pos[j]] += krow[j];
         bi += frow;
      }
      if (r) b[r - 1] = bi;
   }
}

void check_jacobian(const DBuf<int>& bad)
{
   int h = 0;
   bad.download(&h, 1);
   if (h != INT32_MAX)
      throw Error(OFG_ERR_JACOBIAN,
                  "non-positive Jacobian determinant in element " + std::to_string(h + 1));
}

// Launches the row-gather kernel for one element kind and checks Jacobians.
template <class Elem>
void assemble(ofg_mesh* m, ofg_matrix* A, const Elem& el, double* db, int node_fields,
              int elem_fields)
{
   OFG_REQUIRE(A->mesh == m, OFG_ERR_ARG, "matrix pattern was not built from this mesh");
   DBuf<int> bad(1);
   int big = INT32_MAX;
   bad.upload(&big, 1);
   if (m->nn) {
      const int nen = m->nen;
      double bytes = 4.0 * (m->nn + 1) + 8.0 * nen * m->ne + 8.0 * m->dim * m->nn + 8.0 * m->nn +
                     4.0 * nen * nen * m->ne + 8.0 * node_fields * m->nn +
                     8.0 * elem_fields * m->ne + 4.0 * (A->n + 1) +
                     8.0 * A->nnz + 8.0 * A->n;
      int* worked = prof_begin();
      if (worked) OFG_CUDA(cudaMemsetAsync(worked, 1, sizeof(int), stream()));
      assemble_rows<Elem><<<grid_for(m->nn, 256, 16), 256, 0, stream()>>>(
          m->nn, m->n2e_ptr.p, m->n2e.p, m->elem.p, m->dof.p, A->emap.p, A->row_ptr.p, el,
          A->val.p, db, bad.p);
      prof_end(PROF_ASSEMBLY, bytes);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
   matrix_touch(A);
   check_jacobian(bad);
}

__global__ void insert_bc_kernel(int64_t nn, const int32_t* code, const int32_t* dof,
                                 const double* x, const double* bc, double* u)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride)
      u[i] = code[i] == 0 ? x[dof[i] - 1] : (bc ? bc[i] : 0.0);
}

}  // namespace

}  // namespace ofg

using namespace ofg;

extern "C" {

int ofg_assemble_p1(ofg_mesh* m, ofg_matrix* A, const double* kel, const double* f,
                    const double* bc, double* b)
{
   return guarded("ofg_assemble_p1", [&] {
      OFG_REQUIRE(m && A && b, OFG_ERR_ARG, "null argument");
      In<double> dk(kel, m->ne), df(f, m->nn), dbc(bc, m->nn);
      InOut<double> db(b, A->n, false);
      if (m->dim == 2)
         assemble(m, A, LaplaceT3{m->coords.p, m->code.p, dk.d, df.d, dbc.d}, db.d, f ? 1 : 0,
                  kel ? 1 : 0);
      else
         assemble(m, A, DiffusionT4{m->coords.p, m->code.p, dk.d, df.d, dbc.d}, db.d, f ? 1 : 0,
                  kel ? 1 : 0);
      db.finish();
   });
}

int ofg_assemble_cd2d(ofg_mesh* m, ofg_matrix* A, double eps, const double* v, double dt,
                      const double* u_old, const double* bc, double* b)
{
   return guarded("ofg_assemble_cd2d", [&] {
      OFG_REQUIRE(m && A && b && v && u_old, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(m->dim == 2, OFG_ERR_ARG, "DC2DT3 needs a 2-D mesh");
      OFG_REQUIRE(dt > 0, OFG_ERR_ARG, "time step must be positive");
      In<double> dv(v, 2 * m->nn), du(u_old, m->nn), dbc(bc, m->nn);
      InOut<double> db(b, A->n, false);
      assemble(m, A, ConvDiffT3{m->coords.p, m->code.p, eps, 1. / dt, dv.d, du.d, dbc.d}, db.d, 3,
               0);
      db.finish();
   });
}

int ofg_insert_bc(const ofg_mesh* m, const double* x, const double* bc, double* u)
{
   return guarded("ofg_insert_bc", [&] {
      OFG_REQUIRE(m && x && u, OFG_ERR_ARG, "null argument");
      In<double> dx(x, m->neq), dbc(bc, m->nn);
      InOut<double> du(u, m->nn, false);
      insert_bc_kernel<<<grid_for(m->nn, 256), 256, 0, stream()>>>(m->nn, m->code.p, m->dof.p, dx.d,
                                                                    dbc.d, du.d);
      count_launch();
      OFG_LAUNCH_CHECK();
      du.finish();
   });
}

}  // extern "C"

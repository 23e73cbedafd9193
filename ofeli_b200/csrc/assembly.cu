// assembly.cu -- Equation::build() for P1 elements on the device.
//
// One launch per element colour.  A thread owns one element: it computes the
// element geometry and the local matrix / RHS in registers (FP64, the same
// formulas as Triang3/Tetra4 and the element classes), lifts imposed values
// (Equation::updateBC) and scatters through the precomputed element-to-CSR
// map.  Elements of one colour share no node, so no two threads of a launch
// touch the same CSR entry or RHS row: the scatter needs no atomics, and the
// launches of successive colours are ordered by the stream.
//
// Algorithmic bytes per element (2-D / 3-D): connectivity 4*nen, node
// coordinates 8*dim*nen (gathered; each node is shared by ~6 / ~24
// elements), k 8, f 8*nen (gathered), the map 4*nen^2, A updates
// 16*nen^2 (read-modify-write), b updates 16*nen.
#include "element.cuh"

namespace ofg {
namespace {

using namespace elem;

// Laplace2DT3::LHS (times k) + BodyRHS: Ke = area*(g_i.g_j)*k, Fe = f*area/3
// (src/equations/laplace/Laplace2DT3.cpp:131-143)
__global__ void __launch_bounds__(256) assemble_t3(int64_t cnt, const int32_t* __restrict__ list,
                                                   const int32_t* __restrict__ elem,
                                                   const double* __restrict__ xy,
                                                   const int32_t* __restrict__ code,
                                                   const int32_t* __restrict__ dof,
                                                   const int32_t* __restrict__ emap,
                                                   const double* __restrict__ kel,
                                                   const double* __restrict__ f,
                                                   const double* __restrict__ bc, double* a,
                                                   double* b, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += stride) {
      int64_t e = list[t];
      int32_t en[3] = {elem[3 * e], elem[3 * e + 1], elem[3 * e + 2]};
      double g[3][3], area;
      if (!tri3(xy, en, g, area)) {
         atomicMin(bad, (int)e);
         continue;
      }
      double k = kel ? kel[e] : 1.0;
      double Ke[3][3], Fe[3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
         for (int j = 0; j < 3; ++j) Ke[i][j] = area * dot3(g[i], g[j]) * k;
#pragma unroll
      for (int i = 0; i < 3; ++i) Fe[i] = f ? f[en[i]] * area * kThird : 0.0;
      if (bc) lift_bc<3>(en, code, bc, Ke, Fe);
      scatter<3>(e, en, dof, emap, Ke, Fe, a, b);
   }
}

// DC3DT4::Diffusion(k) + BodyRHS: Ke = (k*vol)*(g_i.g_j), Fe = f*vol/4
// (src/equations/therm/DC3DT4.cpp:128-135, 207-211)
__global__ void __launch_bounds__(256) assemble_t4(int64_t cnt, const int32_t* __restrict__ list,
                                                   const int32_t* __restrict__ elem,
                                                   const double* __restrict__ xyz,
                                                   const int32_t* __restrict__ code,
                                                   const int32_t* __restrict__ dof,
                                                   const int32_t* __restrict__ emap,
                                                   const double* __restrict__ kel,
                                                   const double* __restrict__ f,
                                                   const double* __restrict__ bc, double* a,
                                                   double* b, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += stride) {
      int64_t e = list[t];
      int32_t en[4] = {elem[4 * e], elem[4 * e + 1], elem[4 * e + 2], elem[4 * e + 3]};
      double g[4][3], vol;
      if (!tet4(xyz, en, g, vol)) {
         atomicMin(bad, (int)e);
         continue;
      }
      double c = (kel ? kel[e] : 1.0) * vol;
      double Ke[4][4], Fe[4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
         for (int j = 0; j < 4; ++j) Ke[i][j] = c * dot3(g[i], g[j]);
#pragma unroll
      for (int i = 0; i < 4; ++i) Fe[i] = f ? f[en[i]] * 0.25 * vol : 0.0;
      if (bc) lift_bc<4>(en, code, bc, Ke, Fe);
      scatter<4>(e, en, dof, emap, Ke, Fe, a, b);
   }
}

// DC2DT3 under backward Euler (include/equations/therm/Equa_Therm.h:162-218):
// eA1 = Capacity + LCapacity (src/equations/therm/DC2DT3.cpp:121-138),
// eA0 = Diffusion(eps) + Convection (:141-147, 185-207),
// eMat = eA1/dt + eA0, eRHS = updateBC + (eA1/dt) u_old.
__global__ void __launch_bounds__(256) assemble_cd2d(int64_t cnt, const int32_t* __restrict__ list,
                                                     const int32_t* __restrict__ elem,
                                                     const double* __restrict__ xy,
                                                     const int32_t* __restrict__ code,
                                                     const int32_t* __restrict__ dof,
                                                     const int32_t* __restrict__ emap, double eps,
                                                     const double* __restrict__ v, double dti,
                                                     const double* __restrict__ u_old,
                                                     const double* __restrict__ bc, double* a,
                                                     double* b, int* bad)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < cnt; t += stride) {
      int64_t e = list[t];
      int32_t en[3] = {elem[3 * e], elem[3 * e + 1], elem[3 * e + 2]};
      double g[3][3], area;
      if (!tri3(xy, en, g, area)) {
         atomicMin(bad, (int)e);
         continue;
      }
      double cc = kSixth * area, dd = 0.5 * cc, cl = kThird * area;
      double v3[3] = {v[2 * en[0]] + v[2 * en[1]] + v[2 * en[2]],
                      v[2 * en[0] + 1] + v[2 * en[1] + 1] + v[2 * en[2] + 1], 0.0};
      double cv = kThird * kThird * area;
      double Ke[3][3], M1[3][3], Fe[3];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
         for (int j = 0; j < 3; ++j) {
            double m1 = (i == j) ? cc + cl : dd;
            M1[i][j] = dti * m1;
            Ke[i][j] = M1[i][j] + (eps * area * dot3(g[i], g[j]) + cv * dot3(v3, g[j]));
         }
#pragma unroll
      for (int i = 0; i < 3; ++i) Fe[i] = 0.0;
      if (bc) lift_bc<3>(en, code, bc, Ke, Fe);
#pragma unroll
      for (int i = 0; i < 3; ++i)
         Fe[i] += M1[i][0] * u_old[en[0]] + M1[i][1] * u_old[en[1]] + M1[i][2] * u_old[en[2]];
      scatter<3>(e, en, dof, emap, Ke, Fe, a, b);
   }
}

__global__ void insert_bc_kernel(int64_t nn, const int32_t* code, const int32_t* dof,
                                 const double* x, const double* bc, double* u)
{
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride)
      u[i] = code[i] == 0 ? x[dof[i] - 1] : (bc ? bc[i] : 0.0);
}

void check_jacobian(const DBuf<int>& bad)
{
   int h = 0;
   bad.download(&h, 1);
   if (h != INT32_MAX)
      throw Error(OFG_ERR_JACOBIAN,
                  "non-positive Jacobian determinant in element " + std::to_string(h + 1));
}

void prepare(ofg_mesh* m, ofg_matrix* A, double* db)
{
   OFG_REQUIRE(A->mesh == m, OFG_ERR_ARG, "matrix pattern was not built from this mesh");
   A->val.zero();
   if (A->n) OFG_CUDA(cudaMemsetAsync(db, 0, A->n * sizeof(double), stream()));
}

}  // namespace

// Launches the element kernel once per colour.
template <class Launch>
static void for_each_color(ofg_mesh* m, Launch&& launch)
{
   for (size_t c = 0; c + 1 < m->color_ptr.size(); ++c) {
      int64_t beg = m->color_ptr[c], cnt = m->color_ptr[c + 1] - beg;
      if (!cnt) continue;
      int* worked = prof_begin();
      if (worked) OFG_CUDA(cudaMemsetAsync(worked, 1, sizeof(int), stream()));
      launch(m->color_elems.p + beg, cnt, grid_for(cnt, 256, 16));
      prof_end(PROF_ASSEMBLY, 0.0);
      count_launch();
      OFG_LAUNCH_CHECK();
   }
}

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
      prepare(m, A, db.d);
      DBuf<int> bad(1);
      int big = INT32_MAX;
      bad.upload(&big, 1);
      for_each_color(m, [&](const int32_t* list, int64_t cnt, unsigned grid) {
         if (m->dim == 2)
            assemble_t3<<<grid, 256, 0, stream()>>>(cnt, list, m->elem.p, m->coords.p, m->code.p,
                                                     m->dof.p, A->emap.p, dk.d, df.d, dbc.d,
                                                     A->val.p, db.d, bad.p);
         else
            assemble_t4<<<grid, 256, 0, stream()>>>(cnt, list, m->elem.p, m->coords.p, m->code.p,
                                                     m->dof.p, A->emap.p, dk.d, df.d, dbc.d,
                                                     A->val.p, db.d, bad.p);
      });
      matrix_touch(A);
      check_jacobian(bad);
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
      prepare(m, A, db.d);
      DBuf<int> bad(1);
      int big = INT32_MAX;
      bad.upload(&big, 1);
      double dti = 1. / dt;
      for_each_color(m, [&](const int32_t* list, int64_t cnt, unsigned grid) {
         assemble_cd2d<<<grid, 256, 0, stream()>>>(cnt, list, m->elem.p, m->coords.p, m->code.p,
                                                    m->dof.p, A->emap.p, eps, dv.d, dti, du.d,
                                                    dbc.d, A->val.p, db.d, bad.p);
      });
      matrix_touch(A);
      check_jacobian(bad);
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

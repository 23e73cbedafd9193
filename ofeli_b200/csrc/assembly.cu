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
   // each thread sums its row in shared memory (a column per thread)
   __shared__ double racc[kRowAcc * 256];
   int64_t stride = (int64_t)gridDim.x * blockDim.x;
   for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += stride) {
      const int32_t r = dof[i];   // 1-based equation, 0 for an imposed node
      const double bi =
         gather_node_rows(i, r, n2e_ptr[i], n2e_ptr[i + 1], n2e, elem, emap, row_ptr, el, a,
                          [&](int64_t e) { atomicMin(bad, (int)e); }, racc + threadIdx.x, 256);
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

int ofg_assemble_cd2d_scheme(ofg_mesh* m, ofg_matrix* A, double eps, const double* v, double dt,
                             int scheme, const double* u_old, const double* bc, double* b)
{
   return guarded("ofg_assemble_cd2d_scheme", [&] {
      OFG_REQUIRE(m && A && b && v && u_old, OFG_ERR_ARG, "null argument");
      OFG_REQUIRE(m->dim == 2, OFG_ERR_ARG, "DC2DT3 needs a 2-D mesh");
      OFG_REQUIRE(dt > 0, OFG_ERR_ARG, "time step must be positive");
      OFG_REQUIRE(scheme == 1 || scheme == 2 || scheme == 3, OFG_ERR_ARG,
                  "scheme must be FORWARD_EULER (1), BACKWARD_EULER (2) or CRANK_NICOLSON (3)");
      In<double> dv(v, 2 * m->nn), du(u_old, m->nn), dbc(bc, m->nn);
      InOut<double> db(b, A->n, false);
      assemble(m, A, ConvDiffT3{m->coords.p, m->code.p, eps, 1. / dt, dv.d, du.d, dbc.d, scheme},
               db.d, 3, 0);
      db.finish();
   });
}

int ofg_assemble_cd2d(ofg_mesh* m, ofg_matrix* A, double eps, const double* v, double dt,
                      const double* u_old, const double* bc, double* b)
{
   return ofg_assemble_cd2d_scheme(m, A, eps, v, dt, 2, u_old, bc, b);
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

/* ofeli_oracle.h -- CPU restatement of OFELI's P1 assembly + preconditioned
 * Krylov path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check
 * and the CPU-baseline leg of the benchmark call it as the checker.  The
 * product (libofeli_gpu.so) neither links nor calls it.
 *
 * Conventions follow OFELI's SpMatrix (include/linear_algebra/SpMatrix_impl.h
 * :108-119,392-413): row_ptr is 0-based (n+1 entries), col_ind is 1-based.
 * Node / element indices handed to these functions are 0-based.
 */
#ifndef OFELI_ORACLE_H
#define OFELI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { OR_IDENT = 0, OR_DIAG = 1, OR_DILU = 2, OR_ILU = 3, OR_SSOR = 4 };

/* a1: structured triangulation, Mesh.cpp:547-676 (x-major nodes) */
void or_mesh2d(int64_t nx, int64_t ny, double xmin, double xmax, double ymin, double ymax,
               int cx0, int cxN, int cy0, int cyN,
               double* xy, int32_t* elem, int32_t* code);
/* Kuhn cube subdivision, 6 positively oriented tetrahedra per cell */
void or_mesh3d_kuhn(int64_t M, double* xyz, int32_t* elem, int32_t* code);
/* a3: Mesh::NumberEquations with imposed DOF removed, Mesh.cpp:1483-1509 */
int64_t or_number_equations(int64_t nn, const int32_t* code, int64_t* dof);
/* a4: NodeGraph + FinalizeGraph + StoreGraph, GraphOfMatrix.cpp:347-375,52-67,619-634.
 * Returns nnz; col_ind must hold at least ne*nen*nen entries. */
int64_t or_node_graph(int64_t ne, int nen, const int32_t* elem, const int64_t* dof, int64_t n,
                      int64_t* row_ptr, int64_t* col_ind);
/* a6-a13: element loop of Equa_Laplace::build (2-D, Laplace2DT3) or
 * Equa_Therm::build (3-D, DC3DT4) with updateBC and the CSR scatter.
 * kel (per element, may be NULL = 1), f (per node, may be NULL), bc (per node,
 * may be NULL).  Returns 0, or -(element+1) on a non-positive Jacobian. */
int64_t or_assemble_p1(int dim, int64_t nn, int64_t ne, const double* coords, const int32_t* elem,
                       const int64_t* dof, const int32_t* code, const double* kel, const double* f,
                       const double* bc, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                       double* a, double* b);
/* a9: one backward-Euler build of DC2DT3 (capacity bit 0x20 = consistent +
 * lumped, diffusion eps, convection by the nodal velocity v[2*nn]); u_old is
 * the nodal field of the previous step. */
int64_t or_assemble_cd2d_scheme(int64_t nn, int64_t ne, const double* xy, const int32_t* elem,
                                const int64_t* dof, const int32_t* code, double eps,
                                const double* v, double dt, int scheme, const double* u_old,
                                const double* bc, int64_t n, const int64_t* row_ptr,
                                const int64_t* col_ind, double* a, double* b);
int64_t or_assemble_cd2d(int64_t nn, int64_t ne, const double* xy, const int32_t* elem,
                         const int64_t* dof, const int32_t* code, double eps, const double* v,
                         double dt, const double* u_old, const double* bc, int64_t n,
                         const int64_t* row_ptr, const int64_t* col_ind, double* a, double* b);
/* a14: y = A x (SpMatrix::Mult) */
void or_spmv(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a,
             const double* x, double* y);
void or_spmv_transpose_add(int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                           const double* a, const double* x, double* y);
int64_t or_matrix_edit(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, double* a,
                       int64_t count, const int64_t* ii, const int64_t* jj, const double* v,
                       int set);
/* a18: Prec setup.  id (n) receives the 1-based position after the diagonal
 * (OFELI's "id"), pivot (n) the inverse pivots / diagonal.  Returns 0 or
 * -(row+1) on a zero pivot. */
int64_t or_prec_setup(int type, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                      const double* a, int64_t* id, double* pivot);
void or_prec_apply(int type, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                   const double* a, const int64_t* id, const double* pivot, const double* b,
                   double* x);
/* a16: CG(A,P,b,x,max_it,tol), CG.h:99-157.  hist (max_it+1, may be NULL)
 * receives the relative residual after each iteration. */
int or_cg(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a, int prec,
          const double* b, double* x, int max_it, double tol, double* hist);
/* a17: GMRes(A,P,b,x,m,max_it,tol), GMRes.h:67-241 */
int or_bicgstab(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a,
                int prec, const double* b, double* x, int max_it, double tol);
int or_gmres(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a, int prec,
             const double* b, double* x, int m, int max_it, double tol);
/* a21: Vect::insertBC, Vect_impl.h:1098-1130 */
void or_insert_bc(int64_t nn, const int32_t* code, const double* x, const double* bc, double* u);

#ifdef __cplusplus
}
#endif
#endif

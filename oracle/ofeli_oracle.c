/* ofeli_oracle.c -- CPU restatement of OFELI's P1 assembly + preconditioned
 * Krylov path (OFELI 5.3.3).  TEST INFRASTRUCTURE ONLY: called by the parity
 * tests, by the smoke check and by the CPU-baseline leg of the benchmark, as
 * the checker.  The product library never links or calls it.
 *
 * Every function restates one reference routine (cited by path:line within
 * the OFELI project) with the same loop order and the same floating-point
 * operation order, so that it reproduces the reference bit for bit when both
 * are compiled without FMA contraction (-ffp-contract=off).  It is pinned
 * against the reference itself (oracle/_ref, built from the reference's own
 * sources) by tests/test_oracle_pins.py.
 */
#include "ofeli_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define THIRD 0.33333333333333333333333333333  /* util/constants.h:70 */
#define SIXTH 0.16666666666666666666666666667  /* util/constants.h:78 */

/* ---------------------------------------------------------------- meshes -- */

/* Mesh::Mesh(xmin,xmax,ymin,ymax,nx,ny,cx0,cxN,cy0,cyN,TRIANGLE),
 * src/mesh/Mesh.cpp:547-676.  Coordinates are accumulated by repeated
 * addition exactly as the reference does (x.y += hy per node, x.x += hx per
 * column). */
void or_mesh2d(int64_t nx, int64_t ny, double xmin, double xmax, double ymin, double ymax,
               int cx0, int cxN, int cy0, int cyN, double* xy, int32_t* elem, int32_t* code)
{
   double hx = (xmax - xmin) / (double)nx, hy = (ymax - ymin) / (double)ny;
   double x = xmin;
   int64_t n = 0, ne = 0;
   for (int64_t i = 0; i <= nx; ++i) {
      double y = ymin;
      for (int64_t j = 0; j <= ny; ++j) {
         n++;
         int c = 0;
         if (j == 0 && cy0 > 0) c = cy0;
         if (j == ny && cyN > 0) c = cyN;
         if (i == 0 && cx0 > 0) c = cx0;
         if (i == nx && cxN > 0) c = cxN;
         xy[2 * (n - 1)] = x;
         xy[2 * (n - 1) + 1] = y;
         code[n - 1] = c;
         y += hy;
         if (i > 0 && j > 0) {
            /* theNodes[n-ny-3], theNodes[n-2], theNodes[n-1] and
               theNodes[n-1], theNodes[n-ny-2], theNodes[n-ny-3] */
            int32_t* e = elem + 3 * ne;
            e[0] = (int32_t)(n - ny - 3); e[1] = (int32_t)(n - 2); e[2] = (int32_t)(n - 1);
            e[3] = (int32_t)(n - 1); e[4] = (int32_t)(n - ny - 2); e[5] = (int32_t)(n - ny - 3);
            ne += 2;
         }
      }
      x += hx;
   }
}

/* Kuhn subdivision (OFELI's own structured tetrahedral generator,
 * src/mesh/Mesh.cpp:678-836, never advances its node cursor for tetrahedra,
 * so this generator replaces it).  Nodes x fastest; 6 tetrahedra per cell
 * along the axis permutations, odd permutations reordered for det > 0. */
void or_mesh3d_kuhn(int64_t M, double* xyz, int32_t* elem, int32_t* code)
{
   static const int perm[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};
   static const int odd[6] = {0, 1, 1, 0, 0, 1};
   int64_t P = M + 1;
   double h = 1.0 / (double)M;
   int64_t nn = 0;
   for (int64_t kz = 0; kz < P; ++kz)
      for (int64_t jy = 0; jy < P; ++jy)
         for (int64_t ix = 0; ix < P; ++ix) {
            xyz[3 * nn] = (double)ix * h;
            xyz[3 * nn + 1] = (double)jy * h;
            xyz[3 * nn + 2] = (double)kz * h;
            code[nn] = (ix == 0 || jy == 0 || kz == 0 || ix == M || jy == M || kz == M) ? 1 : 0;
            nn++;
         }
   int64_t ne = 0;
   for (int64_t kz = 0; kz < M; ++kz)
      for (int64_t jy = 0; jy < M; ++jy)
         for (int64_t ix = 0; ix < M; ++ix)
            for (int t = 0; t < 6; ++t) {
               int64_t c[3] = {ix, jy, kz};
               int64_t v[4];
               v[0] = c[0] + P * (c[1] + P * c[2]);
               for (int s = 0; s < 3; ++s) {
                  c[perm[t][s]]++;
                  v[s + 1] = c[0] + P * (c[1] + P * c[2]);
               }
               if (odd[t]) { int64_t tmp = v[1]; v[1] = v[2]; v[2] = tmp; }
               for (int q = 0; q < 4; ++q) elem[4 * ne + q] = (int32_t)v[q];
               ne++;
            }
}

/* Mesh::NumberEquations, _no_imposed_dof branch, src/mesh/Mesh.cpp:1497-1509 */
int64_t or_number_equations(int64_t nn, const int32_t* code, int64_t* dof)
{
   int64_t neq = 0;
   for (int64_t i = 0; i < nn; ++i) dof[i] = code[i] == 0 ? ++neq : 0;
   return neq;
}

/* -------------------------------------------------------------- graph ---- */

static int cmp_i64(const void* a, const void* b)
{
   int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
   return (x > y) - (x < y);
}

/* NodeGraph pushes (nk-1,nl-1) and (nl-1,nk-1) for every pair of local nodes
 * with non-zero DOF, then sort + unique + StoreGraph
 * (src/linear_algebra/GraphOfMatrix.cpp:347-375, 52-67, 619-634).  The
 * resulting pattern is the set of pairs sorted by (row, col); it is built here
 * row by row, which yields the same arrays. */
int64_t or_node_graph(int64_t ne, int nen, const int32_t* elem, const int64_t* dof, int64_t n,
                      int64_t* row_ptr, int64_t* col_ind)
{
   int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
   for (int64_t e = 0; e < ne; ++e)
      for (int a = 0; a < nen; ++a) {
         int64_t r = dof[elem[e * nen + a]];
         if (!r) continue;
         for (int b = 0; b < nen; ++b)
            if (dof[elem[e * nen + b]]) cnt[r - 1]++;
      }
   int64_t* start = (int64_t*)malloc(((size_t)n + 1) * sizeof(int64_t));
   start[0] = 0;
   for (int64_t i = 0; i < n; ++i) start[i + 1] = start[i] + cnt[i];
   int64_t* buf = (int64_t*)malloc((size_t)(start[n] > 0 ? start[n] : 1) * sizeof(int64_t));
   memset(cnt, 0, ((size_t)n + 1) * sizeof(int64_t));
   for (int64_t e = 0; e < ne; ++e)
      for (int a = 0; a < nen; ++a) {
         int64_t r = dof[elem[e * nen + a]];
         if (!r) continue;
         for (int b = 0; b < nen; ++b) {
            int64_t c = dof[elem[e * nen + b]];
            if (c) buf[start[r - 1] + cnt[r - 1]++] = c;
         }
      }
   int64_t nnz = 0;
   row_ptr[0] = 0;
   for (int64_t i = 0; i < n; ++i) {
      int64_t* seg = buf + start[i];
      int64_t len = start[i + 1] - start[i];
      qsort(seg, (size_t)len, sizeof(int64_t), cmp_i64);
      for (int64_t k = 0; k < len; ++k)
         if (k == 0 || seg[k] != seg[k - 1]) col_ind[nnz++] = seg[k];
      row_ptr[i + 1] = nnz;
   }
   free(cnt);
   free(start);
   free(buf);
   return nnz;
}

/* ------------------------------------------------------- element kernels -- */

/* Triang3::set, src/shape_functions/Triang3.cpp:68-93 */
static int tri3(const double* xy, const int32_t* en, double g[3][3], double* area)
{
   double x0 = xy[2 * en[0]], y0 = xy[2 * en[0] + 1];
   double x1 = xy[2 * en[1]], y1 = xy[2 * en[1] + 1];
   double x2 = xy[2 * en[2]], y2 = xy[2 * en[2] + 1];
   double det = (x1 - x0) * (y2 - y0) - (y1 - y0) * (x2 - x0);
   *area = 0.5 * det;
   if (det <= 0.0) return -1;
   g[0][0] = (y1 - y2) / det; g[0][1] = (x2 - x1) / det;
   g[1][0] = (y2 - y0) / det; g[1][1] = (x0 - x2) / det;
   g[2][0] = (y0 - y1) / det; g[2][1] = (x1 - x0) / det;
   g[0][2] = g[1][2] = g[2][2] = 0.0;
   return 0;
}

/* Tetra4::CalculateShape, src/shape_functions/Tetra4.cpp:76-114, and
 * getVolume = OFELI_SIXTH*det (include/shape_functions/Tetra4.h:87) */
static int tet4(const double* xyz, const int32_t* en, double g[4][3], double* vol)
{
   static const double dl[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
   double J[4][4], IJ[4][4];
   for (int r = 1; r <= 3; ++r)
      for (int c = 1; c <= 3; ++c) J[r][c] = 0.0;
   for (int k = 0; k < 4; ++k) {
      const double* X = xyz + 3 * en[k];
      for (int r = 1; r <= 3; ++r)
         for (int c = 1; c <= 3; ++c) J[r][c] += dl[k][c - 1] * X[r - 1];
   }
   for (int i = 1; i <= 3; ++i) {
      int j = i % 3 + 1, k = j % 3 + 1;
      IJ[i][i] = J[j][j] * J[k][k] - J[j][k] * J[k][j];
      IJ[j][i] = J[j][k] * J[k][i] - J[j][i] * J[k][k];
      IJ[i][j] = J[k][j] * J[i][k] - J[i][j] * J[k][k];
   }
   double det = J[1][1] * IJ[1][1] + J[2][1] * IJ[1][2] + J[3][1] * IJ[1][3];
   *vol = SIXTH * det;
   if (det <= 0.0) return -1;
   double c = 1. / det;
   for (int i = 0; i < 4; ++i) {
      g[i][0] = c * (IJ[1][1] * dl[i][0] + IJ[2][1] * dl[i][1] + IJ[3][1] * dl[i][2]);
      g[i][1] = c * (IJ[1][2] * dl[i][0] + IJ[2][2] * dl[i][1] + IJ[3][2] * dl[i][2]);
      g[i][2] = c * (IJ[1][3] * dl[i][0] + IJ[2][3] * dl[i][1] + IJ[3][3] * dl[i][2]);
   }
   return 0;
}

/* Point::operator, (include/linear_algebra/Point.h:217) */
static double pdot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* SpMatrix::add(i,j,v) with the linear column search of _col_index
 * (include/linear_algebra/SpMatrix_impl.h:798-804, 1009-1015); i, j 1-based */
static void sp_add(const int64_t* row_ptr, const int64_t* col_ind, double* a, int64_t i, int64_t j,
                   double v)
{
   for (int64_t k = row_ptr[i - 1]; k < row_ptr[i]; ++k)
      if (col_ind[k] == j) { a[k] += v; return; }
}

/* Matrix::Assembly (include/linear_algebra/Matrix_impl.h:172-201) and
 * Vect::Assembly (include/linear_algebra/Vect_impl.h:1523-1535) */
static void scatter(int nen, const int32_t* en, const int64_t* dof, const double* Ke,
                    const double* Fe, const int64_t* row_ptr, const int64_t* col_ind, double* a,
                    double* b)
{
   for (int i = 0; i < nen; ++i) {
      int64_t r = dof[en[i]];
      if (!r) continue;
      for (int j = 0; j < nen; ++j) {
         int64_t c = dof[en[j]];
         if (c) sp_add(row_ptr, col_ind, a, r, c, Ke[i * nen + j]);
      }
   }
   for (int i = 0; i < nen; ++i) {
      int64_t r = dof[en[i]];
      if (r) b[r - 1] += Fe[i];
   }
}

/* Equation::updateBC(el, bc), include/equations/Equation_impl.h:160-176 */
static void update_bc(int nen, const int32_t* en, const int32_t* code, const double* Ke,
                      const double* bc, double* Fe)
{
   for (int i = 0; i < nen; ++i)
      for (int j = 0; j < nen; ++j)
         if (code[en[j]] > 0) Fe[i] -= Ke[i * nen + j] * bc[en[j]];
}

/* Equa_Laplace::build (include/equations/laplace/Equa_Laplace.h:112-133) with
 * Laplace2DT3::LHS/BodyRHS (src/equations/laplace/Laplace2DT3.cpp:131-143),
 * the per-element coefficient applied as eMat *= k after LHS; and
 * Equa_Therm::build (include/equations/therm/Equa_Therm.h:162-218) with
 * DC3DT4::Diffusion(k)/BodyRHS (src/equations/therm/DC3DT4.cpp:128-135,
 * 207-211) in 3-D. */
int64_t or_assemble_p1(int dim, int64_t nn, int64_t ne, const double* coords, const int32_t* elem,
                       const int64_t* dof, const int32_t* code, const double* kel, const double* f,
                       const double* bc, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                       double* a, double* b)
{
   (void)nn;
   memset(a, 0, sizeof(double) * (size_t)row_ptr[n]);
   memset(b, 0, sizeof(double) * (size_t)n);
   int nen = dim + 1;
   double Ke[16], Fe[4];
   for (int64_t e = 0; e < ne; ++e) {
      const int32_t* en = elem + nen * e;
      if (dim == 2) {
         double g[3][3], area;
         if (tri3(coords, en, g, &area)) return -(e + 1);
         for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
               Ke[3 * i + j] = 0.0 + area * pdot(g[i], g[j]);
               if (kel) Ke[3 * i + j] *= kel[e];
            }
         for (int i = 0; i < 3; ++i) Fe[i] = f ? 0.0 + f[en[i]] * area * THIRD : 0.0;
      }
      else {
         double g[4][3], vol;
         if (tet4(coords, en, g, &vol)) return -(e + 1);
         double c = (kel ? 1.0 * kel[e] : 1.0) * 1.0 * vol;
         for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) Ke[4 * i + j] = 0.0 + (0.0 + c * pdot(g[i], g[j]));
         for (int i = 0; i < 4; ++i) Fe[i] = f ? 0.0 + f[en[i]] * 0.25 * vol : 0.0;
      }
      if (bc) update_bc(nen, en, code, Ke, bc, Fe);
      scatter(nen, en, dof, Ke, Fe, row_ptr, col_ind, a, b);
   }
   return 0;
}

/* Equa_Therm::build for DC2DT3 under BACKWARD_EULER
 * (include/equations/therm/Equa_Therm.h:162-218): PDE_Terms::CAPACITY and
 * LUMPED_CAPACITY share the bit 0x20, so Capacity() and LCapacity() both run
 * (src/equations/therm/DC2DT3.cpp:121-138); Diffusion (eps, :141-147);
 * Convection by the element-summed nodal velocity (:185-207); eMat = dti*eA1
 * + eA0; eRHS = updateBC + (dti*eA1)*u_old. */
int64_t or_assemble_cd2d_scheme(int64_t nn, int64_t ne, const double* xy, const int32_t* elem,
                                const int64_t* dof, const int32_t* code, double eps,
                                const double* v, double dt, int scheme, const double* u_old,
                                const double* bc, int64_t n, const int64_t* row_ptr,
                                const int64_t* col_ind, double* a, double* b)
{
   (void)nn;
   memset(a, 0, sizeof(double) * (size_t)row_ptr[n]);
   memset(b, 0, sizeof(double) * (size_t)n);
   double dti = 1. / dt;
   for (int64_t e = 0; e < ne; ++e) {
      const int32_t* en = elem + 3 * e;
      double g[3][3], area, A0[9], A1[9], Ke[9], Fe[3];
      if (tri3(xy, en, g, &area)) return -(e + 1);
      for (int q = 0; q < 9; ++q) A0[q] = A1[q] = 0.0;
      /* Capacity (consistent) */
      double c = SIXTH * area * 1.0 * 1.0 * 1.0, d = 0.5 * c;
      for (int i = 0; i < 3; ++i)
         for (int j = 0; j < 3; ++j) A1[3 * i + j] += (i == j) ? c : d;
      /* LCapacity (lumped) */
      c = THIRD * area * 1.0 * 1.0 * 1.0;
      for (int i = 0; i < 3; ++i) A1[4 * i] += c;
      /* Diffusion(coef = eps): coef*_diff*area*(dSh_i,dSh_j) */
      for (int i = 0; i < 3; ++i)
         for (int j = 0; j < 3; ++j) A0[3 * i + j] += eps * 1.0 * area * pdot(g[i], g[j]);
      /* Convection(): v3 = sum of the nodal velocities */
      double v3[3];
      v3[0] = v[2 * en[0]] + v[2 * en[1]] + v[2 * en[2]];
      v3[1] = v[2 * en[0] + 1] + v[2 * en[1] + 1] + v[2 * en[2] + 1];
      v3[2] = 0.0;
      c = THIRD * THIRD * area * 1.0;
      for (int i = 0; i < 3; ++i)
         for (int j = 0; j < 3; ++j) A0[3 * i + j] += c * pdot(v3, g[j]);
      /* Equa_Therm::build (include/equations/therm/Equa_Therm.h:191-208):
         eMat and the matrix applied to u_old by scheme (1 forward Euler,
         2 backward Euler, 3 Crank-Nicolson) */
      double R[9];
      for (int q = 0; q < 9; ++q) {
         if (scheme == 1) {
            Ke[q] = dti * A1[q];
            R[q] = dti * A1[q] - A0[q];
         }
         else if (scheme == 3) {
            Ke[q] = dti * A1[q] + 0.5 * A0[q];
            R[q] = dti * A1[q] - 0.5 * A0[q];
         }
         else {
            Ke[q] = dti * A1[q] + A0[q];
            R[q] = dti * A1[q];
         }
      }
      for (int i = 0; i < 3; ++i) Fe[i] = 0.0;
      if (bc) update_bc(3, en, code, Ke, bc, Fe);
      for (int i = 0; i < 3; ++i) {
         double s = 0.0;
         for (int j = 0; j < 3; ++j) s += R[3 * i + j] * u_old[en[j]];
         Fe[i] += s;
      }
      scatter(3, en, dof, Ke, Fe, row_ptr, col_ind, a, b);
   }
   return 0;
}

int64_t or_assemble_cd2d(int64_t nn, int64_t ne, const double* xy, const int32_t* elem,
                         const int64_t* dof, const int32_t* code, double eps, const double* v,
                         double dt, const double* u_old, const double* bc, int64_t n,
                         const int64_t* row_ptr, const int64_t* col_ind, double* a, double* b)
{
   return or_assemble_cd2d_scheme(nn, ne, xy, elem, dof, code, eps, v, dt, 2, u_old, bc, n,
                                  row_ptr, col_ind, a, b);
}

/* ------------------------------------------------------------ algebra ---- */

/* SpMatrix::Mult / MultAdd, include/linear_algebra/SpMatrix_impl.h:729-745 */
void or_spmv(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a,
             const double* x, double* y)
{
   int64_t l = 0;
   for (int64_t i = 0; i < n; ++i) {
      y[i] = 0.0;
      for (int64_t j = 0; j < row_ptr[i + 1] - row_ptr[i]; ++j, ++l) y[i] += a[row_ptr[i] + j] * x[col_ind[l] - 1];
   }
}

/* SpMatrix::TMult, the product its loop intends (SpMatrix_impl.h:760-767):
 * y[col] += a * x[row] over the rows in ascending order, into y as given.
 * (The loop itself reads col_ind one entry early.) */
void or_spmv_transpose_add(int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                           const double* a, const double* x, double* y)
{
   for (int64_t i = 0; i < n; ++i)
      for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) y[col_ind[k] - 1] += a[k] * x[i];
}

/* SpMatrix::set / add (SpMatrix_impl.h:785-802) for count 1-based pairs in
 * order, with _col_index's linear row search (:1009-1015); returns the index
 * of the first pair outside the pattern, or -1. */
int64_t or_matrix_edit(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, double* a,
                       int64_t count, const int64_t* ii, const int64_t* jj, const double* v,
                       int set)
{
   for (int64_t e = 0; e < count; ++e) {
      int64_t i = ii[e], j = jj[e], found = -1;
      if (i < 1 || i > n || j < 1 || j > n) return e;
      for (int64_t k = row_ptr[i - 1]; k < row_ptr[i]; ++k)
         if (col_ind[k] == j) {
            found = k;
            break;
         }
      if (found < 0) return e;
      if (set) a[found] = v[e];
      else a[found] += v[e];
   }
   return -1;
}

static double norm2(int64_t n, const double* x)
{
   double s = 0;
   for (int64_t i = 0; i < n; ++i) s += x[i] * x[i];
   return sqrt(s);
}

static double dot(int64_t n, const double* x, const double* y)
{
   double p = 0;
   for (int64_t i = 0; i < n; ++i) p += x[i] * y[i];
   return p;
}

/* Prec::setMatrix (include/solvers/Prec_impl.h:164-195): inv_diag (:306-316)
 * for DIAG; SpMatrix::DILUFactorize (SpMatrix_impl.h:837-870) for DILU and
 * ILU (ILUFactorize is DILUFactorize, :874-878); SSOR needs the diagonal
 * position only (SSORSolve, :914-929). */
int64_t or_prec_setup(int type, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                      const double* a, int64_t* id, double* pivot)
{
   if (type == OR_IDENT) return 0;
   for (int64_t i = 0; i < n; ++i) {
      id[i] = 0;
      for (int64_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k)
         if (col_ind[k] == i + 1) {
            id[i] = k + 1;
            if (a[k] == 0.0) return -(i + 1);
            pivot[i] = a[k];
         }
      if (!id[i]) return -(i + 1);
   }
   if (type == OR_DIAG) {
      for (int64_t i = 0; i < n; ++i) pivot[i] = 1.0 / pivot[i];
      return 0;
   }
   if (type == OR_SSOR) return 0;
   for (int64_t i = 0; i < n; ++i) {
      pivot[i] = 1.0 / pivot[i];
      for (int64_t j = id[i]; j < row_ptr[i + 1]; ++j) {
         int found = 0;
         double c = 0.0;
         int64_t l = col_ind[j] - 1;
         for (int64_t k = row_ptr[l]; k < id[l] - 1; ++k)
            if (col_ind[k] == i + 1) { found = 1; c = a[k]; }
         if (found) pivot[l] -= c * pivot[i] * a[j];
      }
   }
   return 0;
}

/* Prec::solve(b,x) (Prec_impl.h:227-255): DILUSolve (SpMatrix_impl.h:882-900)
 * and SSORSolve (:914-942).  b and x must not alias. */
void or_prec_apply(int type, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                   const double* a, const int64_t* id, const double* pivot, const double* b,
                   double* x)
{
   if (type == OR_IDENT) {
      memcpy(x, b, sizeof(double) * (size_t)n);
      return;
   }
   if (type == OR_DIAG) {
      for (int64_t i = 0; i < n; ++i) x[i] = b[i] * pivot[i];
      return;
   }
   double* z = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
   if (type == OR_SSOR) {
      for (int64_t i = 0; i < n; ++i) {
         double s = 0;
         for (int64_t j = row_ptr[i]; j < id[i] - 1; ++j) s += a[j] * z[col_ind[j] - 1];
         z[i] = (b[i] - s) / a[id[i] - 1];
      }
      for (int64_t i = n - 1; i >= 0; --i) {
         double s = 0;
         for (int64_t j = id[i]; j < row_ptr[i + 1]; ++j) s += a[j] * x[col_ind[j] - 1];
         x[i] = z[i] - s / a[id[i] - 1];
      }
   }
   else {
      for (int64_t i = 0; i < n; ++i) {
         double s = 0;
         for (int64_t j = row_ptr[i]; j < id[i] - 1; ++j) s += a[j] * z[col_ind[j] - 1];
         z[i] = pivot[i] * (b[i] - s);
      }
      for (int64_t i = n - 1; i >= 0; --i) {
         double s = 0;
         for (int64_t j = id[i]; j < row_ptr[i + 1]; ++j) s += a[j] * x[col_ind[j] - 1];
         x[i] = z[i] - pivot[i] * s;
      }
   }
   free(z);
}

/* DILUSolve's forward loop runs to j < id[i], which also visits the diagonal
 * entry times the not yet computed z[i] = 0; that adds an exact zero, so the
 * loops above stop before the diagonal. */

/* CG(const SpMatrix&, const Prec&, b, x, max_it, toler), include/solvers/CG.h:99-157 */
int or_cg(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a, int prec,
          const double* b, double* x, int max_it, double tol, double* hist)
{
   size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
   int64_t* id = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
   double *pivot = (double*)malloc(sz), *r = (double*)malloc(sz), *p = (double*)malloc(sz),
          *q = (double*)malloc(sz), *z = (double*)malloc(sz);
   int ret;
   if (or_prec_setup(prec, n, row_ptr, col_ind, a, id, pivot) < 0) { ret = -(1 << 30); goto done; }
   double nrm = norm2(n, b), res, rho = 0, rho_1 = 1, beta = 0;
   if (nrm == 0) nrm = 1;
   or_spmv(n, row_ptr, col_ind, a, x, q);
   for (int64_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
   if ((res = norm2(n, r) / nrm) <= tol) { ret = 0; goto done; }
   int it;
   for (it = 1; it <= max_it; it++) {
      or_prec_apply(prec, n, row_ptr, col_ind, a, id, pivot, r, z);
      rho = dot(n, r, z);
      if (it == 1)
         memcpy(p, z, sz);
      else {
         beta = rho / rho_1;
         for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
      }
      or_spmv(n, row_ptr, col_ind, a, p, q);
      double alpha = rho / dot(n, p, q);
      for (int64_t i = 0; i < n; ++i) x[i] += alpha * p[i];
      for (int64_t i = 0; i < n; ++i) r[i] -= alpha * q[i];
      res = norm2(n, r) / nrm;
      if (hist) hist[it] = res;
      if (res <= tol) { ret = it; goto done; }
      rho_1 = rho;
   }
   ret = -it;
done:
   free(id); free(pivot); free(r); free(p); free(q); free(z);
   return ret;
}

/* BiCGStab(A, P, b, x, max_it, toler), include/solvers/BiCGStab.h:87-161:
 * the same vector operations in the same order (p = r + beta*(p - omega*v),
 * x += (alpha*pp + omega*ss)), serial dot products; returns the iteration
 * count, 2 when (rr, r) vanishes, 3 when omega vanishes, -(max_it+1) when
 * the loop runs out. */
int or_bicgstab(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a,
                int prec, const double* b, double* x, int max_it, double tol)
{
   size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
   int64_t* id = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
   double *pivot = (double*)malloc(sz), *p = (double*)malloc(sz), *pp = (double*)malloc(sz),
          *s = (double*)malloc(sz), *ss = (double*)malloc(sz), *t = (double*)malloc(sz),
          *v = (double*)malloc(sz), *r = (double*)malloc(sz), *rr = (double*)malloc(sz);
   int ret;
   if (or_prec_setup(prec, n, row_ptr, col_ind, a, id, pivot) < 0) { ret = -(1 << 30); goto done; }
   double rho_1 = 0, rho_2 = 0, alpha = 0, beta = 0, omega = 0, res, nrm = norm2(n, b);
   or_spmv(n, row_ptr, col_ind, a, x, v);
   for (int64_t i = 0; i < n; ++i) r[i] = b[i] - v[i];
   memcpy(rr, r, sz);
   if (nrm == 0.0) nrm = 1;
   if ((res = norm2(n, r) / nrm) <= tol) { ret = 0; goto done; }
   int it;
   for (it = 1; it <= max_it; it++) {
      rho_1 = dot(n, rr, r);
      if (rho_1 == 0.0) { ret = 2; goto done; }
      if (it == 1)
         memcpy(p, r, sz);
      else {
         beta = (rho_1 / rho_2) * (alpha / omega);
         for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
      }
      or_prec_apply(prec, n, row_ptr, col_ind, a, id, pivot, p, pp);
      or_spmv(n, row_ptr, col_ind, a, pp, v);
      alpha = rho_1 / dot(n, rr, v);
      for (int64_t i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
      if ((res = norm2(n, s) / nrm) < tol) {
         for (int64_t i = 0; i < n; ++i) x[i] += alpha * pp[i];
         ret = it;
         goto done;
      }
      or_prec_apply(prec, n, row_ptr, col_ind, a, id, pivot, s, ss);
      or_spmv(n, row_ptr, col_ind, a, ss, t);
      omega = dot(n, t, s) / dot(n, t, t);
      for (int64_t i = 0; i < n; ++i) x[i] += alpha * pp[i] + omega * ss[i];
      for (int64_t i = 0; i < n; ++i) r[i] = s[i] - omega * t[i];
      rho_2 = rho_1;
      if ((res = norm2(n, r) / nrm) < tol) { ret = it; goto done; }
      if (omega == 0.0) { ret = 3; goto done; }
   }
   ret = -it;
done:
   free(id); free(pivot); free(p); free(pp); free(s); free(ss); free(t); free(v); free(r); free(rr);
   return ret;
}

/* GMRes helpers rotate / set_rotation / update, include/solvers/GMRes.h:67-115 */
static void rotate(double* dx, double* dy, double cs, double sn)
{
   double temp = cs * *dx + sn * *dy;
   *dy = cs * *dy - sn * *dx;
   *dx = temp;
}

static void set_rotation(double dx, double dy, double* cs, double* sn)
{
   if (dy == 0.0) { *cs = 1.0; *sn = 0.0; }
   else if (fabs(dy) > fabs(dx)) {
      double temp = dx / dy;
      *sn = 1.0 / sqrt(1.0 + temp * temp);
      *cs = temp * *sn;
   }
   else {
      double temp = dy / dx;
      *cs = 1.0 / sqrt(1.0 + temp * temp);
      *sn = temp * *cs;
   }
}

#define HH(i, j) H[((i) - 1) * (size_t)(m + 1) + ((j) - 1)]

static void gm_update(int64_t n, double* x, int k, const double* H, int m, const double* s,
                      double** v)
{
   double* y = (double*)malloc(sizeof(double) * (size_t)(m + 1));
   memcpy(y, s, sizeof(double) * (size_t)(m + 1));
   for (int i = k; i >= 0; i--) {
      y[i] /= HH(i + 1, i + 1);
      for (int j = i - 1; j >= 0; j--) y[j] -= HH(j + 1, i + 1) * y[i];
   }
   for (int j = 0; j <= k; j++)
      for (int64_t l = 0; l < n; l++) x[l] += v[j][l] * y[j];
   free(y);
}

/* In-place preconditioner application, Prec::solve(x) (Prec_impl.h:198-224) */
static void prec_inplace(int type, int64_t n, const int64_t* row_ptr, const int64_t* col_ind,
                         const double* a, const int64_t* id, const double* pivot, double* x,
                         double* tmp)
{
   if (type == OR_IDENT) return;
   memcpy(tmp, x, sizeof(double) * (size_t)n);
   or_prec_apply(type, n, row_ptr, col_ind, a, id, pivot, tmp, x);
}

/* GMRes(const SpMatrix&, const Prec&, b, x, m, max_it, toler), GMRes.h:148-241 */
int or_gmres(int64_t n, const int64_t* row_ptr, const int64_t* col_ind, const double* a, int prec,
             const double* b, double* x, int m, int max_it, double tol)
{
   size_t sz = sizeof(double) * (size_t)(n > 0 ? n : 1);
   int64_t* id = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
   double *pivot = (double*)malloc(sz), *r = (double*)malloc(sz), *w = (double*)malloc(sz),
          *tmp = (double*)malloc(sz);
   double *s = (double*)calloc((size_t)m + 1, sizeof(double)),
          *cs = (double*)calloc((size_t)m + 1, sizeof(double)),
          *sn = (double*)calloc((size_t)m + 1, sizeof(double)),
          *H = (double*)calloc((size_t)(m + 1) * (size_t)(m + 1), sizeof(double));
   double** v = NULL;
   int ret, it = 1;
   double res = 0;
   if (or_prec_setup(prec, n, row_ptr, col_ind, a, id, pivot) < 0) { ret = -(1 << 30); goto done; }
   double normb = norm2(n, b);
   or_spmv(n, row_ptr, col_ind, a, x, tmp);
   for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
   prec_inplace(prec, n, row_ptr, col_ind, a, id, pivot, r, tmp);
   double beta = norm2(n, r);
   if (normb == 0.0) normb = 1;
   if ((res = norm2(n, r) / normb) <= tol) { ret = it; goto done; }
   v = (double**)malloc(sizeof(double*) * (size_t)(m + 1));
   for (int i = 0; i <= m; ++i) v[i] = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
   while (it <= max_it) {
      double sc = 1.0 / beta;
      for (int64_t l = 0; l < n; ++l) v[0][l] = sc * r[l];
      for (int q = 0; q <= m; ++q) s[q] = 0.0;
      s[0] = beta;
      for (int i = 0; i < m && it <= max_it; i++, it++) {
         or_spmv(n, row_ptr, col_ind, a, v[i], w);
         prec_inplace(prec, n, row_ptr, col_ind, a, id, pivot, w, tmp);
         for (int k = 0; k <= i; k++) {
            HH(k + 1, i + 1) = dot(n, w, v[k]);
            for (int64_t j = 0; j < n; j++) w[j] -= HH(k + 1, i + 1) * v[k][j];
         }
         HH(i + 2, i + 1) = norm2(n, w);
         double sc2 = 1.0 / HH(i + 2, i + 1);
         for (int64_t l = 0; l < n; ++l) v[i + 1][l] = sc2 * w[l];
         for (int k = 0; k < i; k++) rotate(&HH(k + 1, i + 1), &HH(k + 2, i + 1), cs[k], sn[k]);
         set_rotation(HH(i + 1, i + 1), HH(i + 2, i + 1), &cs[i], &sn[i]);
         rotate(&HH(i + 1, i + 1), &HH(i + 2, i + 1), cs[i], sn[i]);
         rotate(&s[i], &s[i + 1], cs[i], sn[i]);
         if ((res = fabs(s[i + 1]) / normb) < tol) {
            gm_update(n, x, i, H, m, s, v);
            ret = it;
            goto done;
         }
      }
      gm_update(n, x, m - 1, H, m, s, v);
      or_spmv(n, row_ptr, col_ind, a, x, tmp);
      for (int64_t i = 0; i < n; ++i) r[i] = b[i] - tmp[i];
      prec_inplace(prec, n, row_ptr, col_ind, a, id, pivot, r, tmp);
      beta = norm2(n, r);
      if ((res = beta / normb) < tol) { ret = it; goto done; }
   }
   ret = -it;
done:
   if (v) {
      for (int i = 0; i <= m; ++i) free(v[i]);
      free(v);
   }
   free(id); free(pivot); free(r); free(w); free(tmp); free(s); free(cs); free(sn); free(H);
   return ret;
}

/* Vect::insertBC(mesh, v, bc), include/linear_algebra/Vect_impl.h:1098-1113 */
void or_insert_bc(int64_t nn, const int32_t* code, const double* x, const double* bc, double* u)
{
   int64_t j = 0;
   for (int64_t i = 0; i < nn; ++i) u[i] = code[i] == 0 ? x[j++] : (bc ? bc[i] : 0.0);
}

// OFELI.h -- OFELI's C++ API for the P1 assembly + Krylov path, backed by
// libofeli_gpu.so (include/ofeli_gpu.h).  Header-only; link with
// -lofeli_gpu.
//
// Names, argument meanings, 1-based indexing and return values follow
// OFELI 5.3.3 (paths within that project):
//   Mesh(xmin,xmax,ymin,ymax,nx,ny,cx0,cxN,cy0,cyN,TRIANGLE)
//                                        src/mesh/Mesh.cpp:547-676
//   SpMatrix<real_t>                     include/linear_algebra/SpMatrix.h:78-611
//   Vect<real_t> (std::vector subclass)  include/linear_algebra/Vect.h:138
//   Prec<real_t>                         include/solvers/Prec.h:73-176
//   CG, GMRes, BiCGStab                  include/solvers/CG.h:99-213, GMRes.h:148-298,
//                                        BiCGStab.h:87-161
//   LinearSolver                         include/solvers/LinearSolver.h:68-273
//   Laplace2DT3, Laplace3DT4/DC3DT4,     src/equations/laplace/Laplace2DT3.cpp,
//   DC2DT3: build(), run()               src/equations/therm/DC3DT4.cpp, DC2DT3.cpp
// Only real_t = double is provided (SpMatrix<real_t> is the path's type).
// Errors raise OFELIException, as OFELI does.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../ofeli_gpu.h"

namespace OFELI {

typedef double real_t;

class OFELIException : public std::runtime_error {
 public:
   explicit OFELIException(const std::string& s) : std::runtime_error(s) { }
};

inline void ofg_check(int status, const char* what)
{
   if (status != OFG_OK)
      throw OFELIException(std::string(what) + ": " + ofg_last_error());
}

// OFELI's time schemes on the path (include/equations/Equa.h:124-137)
enum TimeScheme { NONE = 0, FORWARD_EULER = 1, BACKWARD_EULER = 2, CRANK_NICOLSON = 3 };

enum Iteration {
   DIRECT_SOLVER = 1, CG_SOLVER = 2, CGS_SOLVER = 3, BICG_SOLVER = 4, BICG_STAB_SOLVER = 5,
   GMRES_SOLVER = 6
};
enum Preconditioner { IDENT_PREC = 0, DIAG_PREC = 1, DILU_PREC = 2, ILU_PREC = 3, SSOR_PREC = 4 };
enum { TRIANGLE = 3, TETRAHEDRON = 4 };

// ---------------------------------------------------------------- Vect ----
template <class T_>
class Vect : public std::vector<T_> {
 public:
   Vect() { }
   explicit Vect(size_t n, T_ v = T_(0)) : std::vector<T_>(n, v) { }
   T_& operator()(size_t i) { return (*this)[i - 1]; }
   T_ operator()(size_t i) const { return (*this)[i - 1]; }
   void clear() { std::fill(this->begin(), this->end(), T_(0)); }
   void setSize(size_t n) { this->assign(n, T_(0)); }
   Vect& operator=(T_ v)
   {
      std::fill(this->begin(), this->end(), v);
      return *this;
   }
   T_ getNorm2() const
   {
      T_ s = 0;
      for (size_t i = 0; i < this->size(); ++i) s += (*this)[i] * (*this)[i];
      return std::sqrt(s);
   }
   T_ operator,(const Vect& v) const
   {
      T_ p = 0;
      for (size_t i = 0; i < this->size(); ++i) p += (*this)[i] * v[i];
      return p;
   }
};

// ---------------------------------------------------------------- Mesh ----
class Mesh {
 public:
   // Mesh(xmin,xmax,ymin,ymax,nx,ny,cx0,cxN,cy0,cyN,TRIANGLE)
   Mesh(real_t xmin, real_t xmax, real_t ymin, real_t ymax, size_t nx, size_t ny, int cx0,
        int cxN, int cy0, int cyN, int opt = TRIANGLE, size_t nb_dof = 1)
   {
      if (opt != TRIANGLE || nb_dof != 1)
         throw OFELIException("Mesh: the GPU path provides P1 triangles with 1 DOF per node");
      ofg_check(ofg_mesh_create_rect(xmin, xmax, ymin, ymax, (int64_t)nx, (int64_t)ny, cx0, cxN,
                                     cy0, cyN, &_h),
                "Mesh");
      info();
   }
   // unit cube, M^3 cells of 6 positively oriented tetrahedra, code 1 on faces
   static Mesh Kuhn(size_t M)
   {
      ofg_mesh* h = nullptr;
      ofg_check(ofg_mesh_create_kuhn((int64_t)M, &h), "Mesh::Kuhn");
      return Mesh(h);
   }
   // general P1 mesh: coords (nn*dim), 0-based connectivity, node codes
   Mesh(int dim, const std::vector<real_t>& coords, const std::vector<int32_t>& elem,
        const std::vector<int32_t>& code)
   {
      ofg_check(ofg_mesh_create(dim, (int64_t)code.size(), coords.data(),
                                (int64_t)(elem.size() / (dim + 1)), elem.data(), code.data(), &_h),
                "Mesh");
      info();
   }
   // Mesh(file, bc): a P1 mesh from OFELI's XML format (Mesh::get).  The
   // equations are numbered over the code-0 nodes whatever bc is, as the P1
   // equations' removeImposedDOF leaves them.
   explicit Mesh(const std::string& file, bool bc = false)
   {
      (void)bc;
      get(file);
   }
   // Mesh::get(file) -- src/mesh/Mesh.cpp:2639-2668, tokenised and converted
   // on the device
   void get(const std::string& file)
   {
      ofg_mesh* h = nullptr;
      ofg_check(ofg_mesh_read(file.c_str(), &h), "Mesh::get");
      if (_h) ofg_mesh_destroy(_h);
      _h = h;
      _path = file;
      info();
   }
   // Mesh::put(file) -- src/mesh/Mesh.cpp:2731-2806; a mesh read from a file
   // writes that file's content (read again on the host)
   void put(const std::string& file) const
   {
      ofg_mesh_file* f = nullptr;
      if (!_path.empty())
         ofg_check(ofg_mesh_file_read(_path.c_str(), &f), "Mesh::put");
      else
         ofg_check(ofg_mesh_file_from_mesh(_h, &f), "Mesh::put");
      int rc = ofg_mesh_file_write(f, file.c_str());
      std::string msg = rc != OFG_OK ? std::string("Mesh::put: ") + ofg_last_error() : "";
      ofg_mesh_file_destroy(f);
      if (rc != OFG_OK) throw OFELIException(msg);
   }
   // Mesh::save for the ".m" format
   void save(const std::string& file) const
   {
      if (file.size() < 2 || file.compare(file.size() - 2, 2, ".m") != 0)
         throw OFELIException("Mesh::save: only OFELI's .m format is written");
      put(file);
   }
   Mesh(const Mesh&) = delete;
   Mesh& operator=(const Mesh&) = delete;
   Mesh(Mesh&& o) noexcept { *this = std::move(o); }
   Mesh& operator=(Mesh&& o) noexcept
   {
      std::swap(_h, o._h);
      std::swap(_path, o._path);
      _dim = o._dim; _nn = o._nn; _ne = o._ne; _neq = o._neq;
      return *this;
   }
   ~Mesh()
   {
      if (_h) ofg_mesh_destroy(_h);
   }
   size_t getDim() const { return (size_t)_dim; }
   size_t getNbNodes() const { return (size_t)_nn; }
   size_t getNbElements() const { return (size_t)_ne; }
   size_t getNbEq() const { return (size_t)_neq; }
   ofg_mesh* handle() const { return _h; }

 private:
   explicit Mesh(ofg_mesh* h) : _h(h) { info(); }
   void info() { ofg_check(ofg_mesh_info(_h, &_dim, &_nn, &_ne, &_neq), "Mesh"); }
   ofg_mesh* _h = nullptr;
   std::string _path;   // the file a mesh was read from (put writes its content)
   int _dim = 0;
   int64_t _nn = 0, _ne = 0, _neq = 0;
};

template <class T_> class Prec;

// ------------------------------------------------------------ SpMatrix ----
template <class T_>
class SpMatrix;

template <>
class SpMatrix<real_t> {
 public:
   // SpMatrix(mesh): NodeGraph pattern of the mesh (bit-identical to OFELI's)
   explicit SpMatrix(Mesh& mesh, size_t dof = 0, int is_diag = 0)
   {
      if (dof != 0 || is_diag != 0) throw OFELIException("SpMatrix(Mesh&): only dof = 0 is provided");
      ofg_check(ofg_matrix_create_from_mesh(mesh.handle(), &_h), "SpMatrix(Mesh&)");
      info();
   }
   // SpMatrix(row_ptr, col_ind[, a]): OFELI's layout, 0-based row pointer,
   // 1-based column indices
   SpMatrix(const std::vector<size_t>& row_ptr, const std::vector<size_t>& col_ind)
   {
      std::vector<int64_t> rp(row_ptr.begin(), row_ptr.end()), ci(col_ind.begin(), col_ind.end());
      ofg_check(ofg_matrix_create((int64_t)rp.size() - 1, (int64_t)ci.size(), rp.data(), ci.data(),
                                  &_h),
                "SpMatrix(row_ptr,col_ind)");
      info();
   }
   SpMatrix(const std::vector<size_t>& row_ptr, const std::vector<size_t>& col_ind,
            const std::vector<real_t>& a)
      : SpMatrix(row_ptr, col_ind)
   {
      setValues(a);
   }
   SpMatrix(const SpMatrix&) = delete;
   SpMatrix& operator=(const SpMatrix&) = delete;
   ~SpMatrix()
   {
      if (_h) ofg_matrix_destroy(_h);
   }
   size_t size() const { return (size_t)_n; }
   size_t getNbRows() const { return (size_t)_n; }
   size_t getNbColumns() const { return (size_t)_n; }
   size_t getLength() const { return (size_t)_nnz; }
   // getRowPtr(i) / getColInd(i): 1-based argument, as SpMatrix_impl.h:816-826
   size_t getRowPtr(size_t i) const { pattern(); return (size_t)_rp[i - 1]; }
   size_t getColInd(size_t i) const { pattern(); return (size_t)_ci[i - 1]; }
   // (i,j), 1-based; 0 outside the pattern
   real_t operator()(size_t i, size_t j) const
   {
      pattern();
      std::vector<real_t> a = values();
      for (int64_t k = _rp[i - 1]; k < _rp[i]; ++k)
         if ((size_t)_ci[k] == j) return a[k];
      return 0.0;
   }
   std::vector<real_t> values() const
   {
      std::vector<real_t> a(_nnz);
      ofg_check(ofg_matrix_get_values(_h, a.data()), "SpMatrix::get");
      return a;
   }
   void setValues(const std::vector<real_t>& a)
   {
      if ((int64_t)a.size() != _nnz) throw OFELIException("SpMatrix: value array size");
      ofg_check(ofg_matrix_set_values(_h, a.data()), "SpMatrix::set");
   }
   void clear() { ofg_check(ofg_matrix_clear(_h), "SpMatrix::clear"); }
   void Mult(const Vect<real_t>& x, Vect<real_t>& y) const
   {
      y.resize(_n);
      ofg_check(ofg_spmv(_h, x.data(), y.data()), "SpMatrix::Mult");
   }
   void MultAdd(const Vect<real_t>& x, Vect<real_t>& y) const
   {
      ofg_check(ofg_spmv_add(_h, x.data(), y.data()), "SpMatrix::MultAdd");
   }
   Vect<real_t> operator*(const Vect<real_t>& x) const
   {
      Vect<real_t> y(_n);
      Mult(x, y);
      return y;
   }
   // SpMatrix::TMult: y += A^T x (SpMatrix_impl.h:760-767, the intended
   // product; OFELI's loop indexes the column one entry early)
   void TMult(const Vect<real_t>& x, Vect<real_t>& y) const
   {
      y.resize(_n);
      ofg_check(ofg_spmv_transpose_add(_h, x.data(), y.data()), "SpMatrix::TMult");
   }
   // SpMatrix::set(i,j,v) / add(i,j,v), 1-based (SpMatrix_impl.h:785-802); a
   // pair outside the pattern throws (OFELI's add would write into the
   // previous row instead).  For many entries, edit() applies them in one call.
   void set(size_t i, size_t j, real_t v) { edit({i}, {j}, {v}, true); }
   void add(size_t i, size_t j, real_t v) { edit({i}, {j}, {v}, false); }
   void edit(const std::vector<size_t>& i, const std::vector<size_t>& j,
             const std::vector<real_t>& v, bool set_values)
   {
      if (i.size() != j.size() || i.size() != v.size())
         throw OFELIException("SpMatrix::edit: index and value arrays differ in size");
      std::vector<int64_t> ii(i.begin(), i.end()), jj(j.begin(), j.end());
      ofg_check(ofg_matrix_edit(_h, (int64_t)ii.size(), ii.data(), jj.data(), v.data(),
                                set_values ? 1 : 0),
                set_values ? "SpMatrix::set" : "SpMatrix::add");
   }
   // SpMatrix::DILUFactorize / ILUFactorize (SpMatrix_impl.h:837-878): id =
   // 1-based diagonal positions, pivot = the inverted D-ILU pivots; returns
   // 0, or the 1-based row of a zero pivot.  DILUSolve / ILUSolve / SSORSolve
   // apply the factorisation of the matrix's current values.
   int DILUFactorize(std::vector<size_t>& id, std::vector<real_t>& pivot) const;
   int ILUFactorize(std::vector<size_t>& id, std::vector<real_t>& pivot) const
   {
      return DILUFactorize(id, pivot);
   }
   void DILUSolve(const std::vector<size_t>& id, const std::vector<real_t>& pivot,
                  const Vect<real_t>& b, Vect<real_t>& x) const;
   void ILUSolve(const std::vector<size_t>& id, const std::vector<real_t>& pivot,
                 const Vect<real_t>& b, Vect<real_t>& x) const
   {
      DILUSolve(id, pivot, b, x);
   }
   void SSORSolve(const Vect<real_t>& b, Vect<real_t>& x) const;
   // SpMatrix::setSolver / solve (SpMatrix_impl.h:957-971)
   void setSolver(Iteration s = CG_SOLVER, Preconditioner p = DIAG_PREC, int max_it = 1000,
                  real_t toler = 1.e-8)
   {
      _s = s, _p = p, _max_it = max_it, _toler = toler;
   }
   int solve(const Vect<real_t>& b, Vect<real_t>& x);
   ofg_matrix* handle() const { return _h; }

 private:
   void info() { ofg_check(ofg_matrix_info(_h, &_n, &_nnz), "SpMatrix"); }
   void pattern() const
   {
      if (!_rp.empty()) return;
      _rp.resize(_n + 1);
      _ci.resize(_nnz);
      ofg_check(ofg_matrix_get_pattern(_h, _rp.data(), _ci.data()), "SpMatrix pattern");
   }
   ofg_matrix* _h = nullptr;
   int64_t _n = 0, _nnz = 0;
   mutable std::vector<int64_t> _rp, _ci;
   Iteration _s = CG_SOLVER;
   Preconditioner _p = DIAG_PREC;
   int _max_it = 1000;
   real_t _toler = 1.e-8;
};

// ---------------------------------------------------------------- Prec ----
template <class T_>
class Prec;

template <>
class Prec<real_t> {
 public:
   Prec(const SpMatrix<real_t>& A, int type) : _type(type)
   {
      ofg_check(ofg_prec_create(A.handle(), type, &_h), "Prec");
   }
   Prec(const Prec&) = delete;
   Prec& operator=(const Prec&) = delete;
   ~Prec()
   {
      if (_h) ofg_prec_destroy(_h);
   }
   int getType() const { return _type; }
   // recompute after the matrix values changed
   void setMatrix() { ofg_check(ofg_prec_update(_h), "Prec::setMatrix"); }
   void solve(const Vect<real_t>& b, Vect<real_t>& x) const
   {
      x.resize(b.size());
      ofg_check(ofg_prec_apply(_h, b.data(), x.data()), "Prec::solve");
   }
   void solve(Vect<real_t>& x) const
   {
      Vect<real_t> b(x);
      solve(b, x);
   }
   std::vector<real_t> getPivots(size_t n) const
   {
      std::vector<real_t> p(n);
      ofg_check(ofg_prec_get_pivot(_h, p.data()), "Prec::getPivot");
      return p;
   }
   ofg_prec* handle() const { return _h; }

 private:
   ofg_prec* _h = nullptr;
   int _type;
};

inline int SpMatrix<real_t>::DILUFactorize(std::vector<size_t>& id,
                                           std::vector<real_t>& pivot) const
{
   ofg_prec* P = nullptr;
   int rc = ofg_prec_create(_h, DILU_PREC, &P);
   if (rc == OFG_ERR_PIVOT) {
      // OFELI returns the row of the zero pivot; the message names it
      std::string m = ofg_last_error();
      size_t at = m.rfind(' ');
      return at == std::string::npos ? 1 : std::max(1, std::atoi(m.c_str() + at + 1));
   }
   ofg_check(rc, "SpMatrix::DILUFactorize");
   pivot.assign(_n, 0.0);
   rc = ofg_prec_get_pivot(P, pivot.data());
   ofg_prec_destroy(P);
   ofg_check(rc, "SpMatrix::DILUFactorize");
   pattern();
   id.assign(_n, 0);
   for (int64_t i = 0; i < _n; ++i)
      for (int64_t k = _rp[i]; k < _rp[i + 1]; ++k)
         if (_ci[k] == i + 1) id[i] = (size_t)k + 1;
   return 0;
}

inline void SpMatrix<real_t>::DILUSolve(const std::vector<size_t>&, const std::vector<real_t>&,
                                        const Vect<real_t>& b, Vect<real_t>& x) const
{
   Prec<real_t> P(*this, DILU_PREC);
   P.solve(b, x);
}

inline void SpMatrix<real_t>::SSORSolve(const Vect<real_t>& b, Vect<real_t>& x) const
{
   Prec<real_t> P(*this, SSOR_PREC);
   P.solve(b, x);
}

// ------------------------------------------------------------ CG, GMRes ----
// Return: iterations when converged, -iterations otherwise (CG.h:99-157).
inline int CG(const SpMatrix<real_t>& A, const Prec<real_t>& P, const Vect<real_t>& b,
              Vect<real_t>& x, int max_it, real_t toler)
{
   (void)A;
   x.resize(b.size());
   int it = 0;
   ofg_check(ofg_cg(P.handle(), b.data(), x.data(), max_it, toler, &it, nullptr), "CG");
   return it;
}

inline int CG(const SpMatrix<real_t>& A, int prec, const Vect<real_t>& b, Vect<real_t>& x,
              int max_it, real_t toler)
{
   Prec<real_t> P(A, prec);
   return CG(A, P, b, x, max_it, toler);
}

inline int GMRes(const SpMatrix<real_t>& A, const Prec<real_t>& P, const Vect<real_t>& b,
                 Vect<real_t>& x, size_t m, int max_it, real_t toler)
{
   (void)A;
   x.resize(b.size());
   int it = 0;
   ofg_check(ofg_gmres(P.handle(), b.data(), x.data(), (int)m, max_it, toler, &it, nullptr),
             "GMRes");
   return it;
}

inline int GMRes(const SpMatrix<real_t>& A, int prec, const Vect<real_t>& b, Vect<real_t>& x,
                 size_t m, int max_it, real_t toler)
{
   Prec<real_t> P(A, prec);
   return GMRes(A, P, b, x, m, max_it, toler);
}

// BiCGStab (include/solvers/BiCGStab.h:87-161): iterations; 2 or 3 on a
// breakdown; -(max_it+1) when the loop runs out.
inline int BiCGStab(const SpMatrix<real_t>& A, const Prec<real_t>& P, const Vect<real_t>& b,
                    Vect<real_t>& x, int max_it, real_t toler)
{
   (void)A;
   x.resize(b.size());
   int it = 0;
   ofg_check(ofg_bicgstab(P.handle(), b.data(), x.data(), max_it, toler, &it, nullptr),
             "BiCGStab");
   return it;
}

inline int BiCGStab(const SpMatrix<real_t>& A, int prec, const Vect<real_t>& b, Vect<real_t>& x,
                    int max_it, real_t toler)
{
   Prec<real_t> P(A, prec);
   return BiCGStab(A, P, b, x, max_it, toler);
}

// -------------------------------------------------------- LinearSolver ----
class LinearSolver {
 public:
   LinearSolver() { }
   LinearSolver(SpMatrix<real_t>& A, const Vect<real_t>& b, Vect<real_t>& x)
      : _A(&A), _b(&b), _x(&x), _s(CG_SOLVER) { }
   void setMaxIter(int m) { _max_it = m; }
   void setTolerance(real_t t) { _toler = t; }
   void setMatrix(SpMatrix<real_t>& A) { _A = &A; }
   void setRHS(const Vect<real_t>& b) { _b = &b; }
   void setSolution(Vect<real_t>& x) { _x = &x; }
   void setSolver(Iteration s, Preconditioner p = DIAG_PREC) { _s = s, _p = p; }
   int getNbIter() const { return _nb_it; }
   int solve(Iteration s, Preconditioner p)
   {
      setSolver(s, p);
      return solve();
   }
   // LinearSolver::solve (src/solvers/LinearSolver.cpp:194-244): 0 on
   // success, the iteration count on failure; GMRES restarts every n/5
   int solve()
   {
      if (!_A) throw OFELIException("In LinearSolver::solve(): No matrix has been defined.");
      if (_s == CG_SOLVER) _nb_it = CG(*_A, _p, *_b, *_x, _max_it, _toler);
      else if (_s == GMRES_SOLVER) {
         size_t m = _b->size() / 5;
         _nb_it = GMRes(*_A, _p, *_b, *_x, m ? m : 1, _max_it, _toler);
      }
      else if (_s == BICG_STAB_SOLVER)
         _nb_it = BiCGStab(*_A, _p, *_b, *_x, _max_it, _toler);
      else
         throw OFELIException("LinearSolver: solver outside the GPU path");
      return _nb_it < 0 ? -_nb_it : 0;
   }

 private:
   SpMatrix<real_t>* _A = nullptr;
   const Vect<real_t>* _b = nullptr;
   Vect<real_t>* _x = nullptr;
   Iteration _s = DIRECT_SOLVER;
   Preconditioner _p = DIAG_PREC;
   int _max_it = 1000;
   real_t _toler = std::sqrt(2.220446049250313e-16);
   int _nb_it = 0;
};

inline int SpMatrix<real_t>::solve(const Vect<real_t>& b, Vect<real_t>& x)
{
   if (_s == DIRECT_SOLVER) throw OFELIException("In SpMatrix::solve(...): No solver provided.");
   LinearSolver ls(*this, b, x);
   ls.setMaxIter(_max_it);
   ls.setTolerance(_toler);
   return ls.solve(_s, _p);
}

// ----------------------------------------------------------- equations ----
// Equation<...>::build() and Equa::run() for the stationary P1 problems.
class P1Equation {
 public:
   P1Equation(Mesh& ms, Vect<real_t>& u) : _mesh(&ms), _u(&u)
   {
      _ls.setSolver(CG_SOLVER, DILU_PREC);
   }
   virtual ~P1Equation() { delete _A; }
   void setSolver(Iteration s, Preconditioner p = DIAG_PREC)
   {
      _ls.setSolver(s, p);
      if (!_A) _A = new SpMatrix<real_t>(*_mesh);
   }
   LinearSolver& getLinearSolver() { return _ls; }
   void setSource(const Vect<real_t>& f) { _bf = &f; }
   void setBodyForce(const Vect<real_t>& f) { _bf = &f; }
   void setDirichlet(const Vect<real_t>& bc) { _bc = &bc; }
   // per-element stiffness scale (variable conductivity), one value per element
   void setElementCoefficient(const Vect<real_t>& k) { _k = &k; }
   SpMatrix<real_t>* getMatrix() { return _A; }
   Vect<real_t>& getRHS() { return _b; }
   Vect<real_t>& getSolution() { return _x; }
   void build()
   {
      if (!_A) _A = new SpMatrix<real_t>(*_mesh);
      _b.setSize(_A->size());
      ofg_check(ofg_assemble_p1(_mesh->handle(), _A->handle(), _k ? _k->data() : nullptr,
                                _bf ? _bf->data() : nullptr, _bc ? _bc->data() : nullptr,
                                _b.data()),
                "Equation::build");
   }
   int run()
   {
      build();
      _x.setSize(_A->size());
      _ls.setMatrix(*_A);
      _ls.setRHS(_b);
      _ls.setSolution(_x);
      int ret = _ls.solve();
      _u->resize(_mesh->getNbNodes());
      ofg_check(ofg_insert_bc(_mesh->handle(), _x.data(), _bc ? _bc->data() : nullptr, _u->data()),
                "Vect::insertBC");
      return ret;
   }

 protected:
   Mesh* _mesh;
   Vect<real_t>* _u;
   SpMatrix<real_t>* _A = nullptr;
   const Vect<real_t>* _bf = nullptr;
   const Vect<real_t>* _bc = nullptr;
   const Vect<real_t>* _k = nullptr;
   Vect<real_t> _b, _x;
   LinearSolver _ls;
};

// area (grad phi_i . grad phi_j), lumped source f area / 3
class Laplace2DT3 : public P1Equation {
 public:
   Laplace2DT3(Mesh& ms, Vect<real_t>& u) : P1Equation(ms, u) { }
};

// k vol (grad phi_i . grad phi_j), lumped source f vol / 4
class DC3DT4 : public P1Equation {
 public:
   DC3DT4(Mesh& ms, Vect<real_t>& u) : P1Equation(ms, u) { }
};
typedef DC3DT4 Laplace3DT4;

// Backward-Euler steps of DC2DT3: consistent + lumped capacity, diffusion
// eps, convection by the nodal velocity v (2 values per node); one build()
// and one GMRES(m) solve per step, warm-started.
class DC2DT3 {
 public:
   DC2DT3(Mesh& ms, Vect<real_t>& u, const Vect<real_t>& v, real_t eps, real_t dt)
      : _mesh(&ms), _u(&u), _v(&v), _eps(eps), _dt(dt), _A(ms)
   {
      _x.setSize(_A.size());
   }
   void setDirichlet(const Vect<real_t>& bc) { _bc = &bc; }
   // Equa::setTransient: FORWARD_EULER, BACKWARD_EULER (default) or CRANK_NICOLSON
   void setTransient(TimeScheme s)
   {
      if (s != FORWARD_EULER && s != BACKWARD_EULER && s != CRANK_NICOLSON)
         throw OFELIException("DC2DT3::setTransient: unsupported time scheme");
      _scheme = s;
   }
   void build()
   {
      _b.setSize(_A.size());
      ofg_check(ofg_assemble_cd2d_scheme(_mesh->handle(), _A.handle(), _eps, _v->data(), _dt,
                                         (int)_scheme, _u->data(), _bc ? _bc->data() : nullptr,
                                         _b.data()),
                "DC2DT3::build");
   }
   int step(Preconditioner p = ILU_PREC, size_t m = 30, int max_it = 1000, real_t toler = 1e-10)
   {
      build();
      Prec<real_t> P(_A, p);
      int it = GMRes(_A, P, _b, _x, m, max_it, toler);
      ofg_check(ofg_insert_bc(_mesh->handle(), _x.data(), _bc ? _bc->data() : nullptr, _u->data()),
                "Vect::insertBC");
      return it;
   }
   SpMatrix<real_t>& getMatrix() { return _A; }
   Vect<real_t>& getRHS() { return _b; }
   // Equa::getLinearSolver(): the solver of TimeStepping's implicit steps
   LinearSolver& getLinearSolver() { return _ls; }

 private:
   friend class TimeStepping;
   Mesh* _mesh;
   Vect<real_t>* _u;
   const Vect<real_t>* _v;
   real_t _eps, _dt;
   TimeScheme _scheme = BACKWARD_EULER;
   SpMatrix<real_t> _A;
   const Vect<real_t>* _bc = nullptr;
   Vect<real_t> _b, _x;
   LinearSolver _ls;
};

// TimeStepping (src/solvers/TimeStepping.cpp) for a DC2DT3 equation under
// its first-order schemes.  Backward Euler and Crank-Nicolson: build() of
// the scheme's system and the equation's LinearSolver (the solver and
// preconditioner of setLinearSolver, GMRES restarting every n/5 steps,
// warm-started from the previous step); forward Euler: x = b / D with D the
// assembled diagonal (ofg_matrix_diag_solve).  As OFELI's set() tests the
// scheme against HEUN and NEWMARK with bitwise ANDs, forward Euler (1) and
// Crank-Nicolson (3) make two sub-steps per runOneTimeStep (NEWMARK = 5).
class TimeStepping {
 public:
   TimeStepping(TimeScheme s, real_t time_step, real_t final_time = 1.0)
      : _s(s), _dt(time_step), _final(final_time)
   {
      if (s != FORWARD_EULER && s != BACKWARD_EULER && s != CRANK_NICOLSON)
         throw OFELIException("In TimeStepping::set(...): scheme outside the GPU path");
      _nb_ssteps = ((int)s & 4) || ((int)s & 5) ? 2 : 1;  // HEUN = 4, NEWMARK = 5
   }
   void setPDE(DC2DT3& eq)
   {
      _eq = &eq;
      eq._dt = _dt;
      eq.setTransient(_s);
   }
   void setInitial(Vect<real_t>& u) { *_eq->_u = u; }
   void setBC(const Vect<real_t>& bc) { _eq->setDirichlet(bc); }
   void setLinearSolver(Iteration s = GMRES_SOLVER, Preconditioner p = DIAG_PREC)
   {
      _it = s, _p = p;
   }
   real_t runOneTimeStep()
   {
      if (!_eq) throw OFELIException("TimeStepping: no equation (setPDE)");
      DC2DT3& eq = *_eq;
      for (int k = 0; k < _nb_ssteps; ++k) {
         eq.build();
         if (_s == FORWARD_EULER)
            ofg_check(ofg_matrix_diag_solve(eq._A.handle(), eq._b.data(), eq._x.data()),
                      "TimeStepping::solveForwardEuler");
         else {
            eq._ls.setMatrix(eq._A);
            eq._ls.setRHS(eq._b);
            eq._ls.setSolution(eq._x);
            eq._ls.solve(_it, _p);
         }
         ofg_check(ofg_insert_bc(eq._mesh->handle(), eq._x.data(),
                                 eq._bc ? eq._bc->data() : nullptr, eq._u->data()),
                   "TimeStepping::insertBC");
      }
      return _dt;
   }
   void run()
   {
      for (real_t t = 0; t < _final - 0.5 * _dt; t += _dt) runOneTimeStep();
   }

 private:
   TimeScheme _s;
   real_t _dt, _final;
   int _nb_ssteps = 1;
   DC2DT3* _eq = nullptr;
   Iteration _it = GMRES_SOLVER;
   Preconditioner _p = DIAG_PREC;
};

}  // namespace OFELI

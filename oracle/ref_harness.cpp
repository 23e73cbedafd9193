// ref_harness.cpp -- drives the reference OFELI library, compiled from its own
// sources into oracle/_ref by oracle/Makefile, on the P1 assembly + Krylov
// workloads.  TEST INFRASTRUCTURE ONLY: it produces golden vectors for the
// parity tests and times the reference CPU path for the baseline.  Nothing in
// the product links or calls it.
//
// Usage (all inputs are little-endian binaries written by the caller):
//   ofeli_ref p2d  NX NY   SOLVER PREC TOL MAXIT INDIR OUTDIR
//   ofeli_ref p3d  M       SOLVER PREC TOL MAXIT INDIR OUTDIR
//   ofeli_ref cd2d NX NY   NSTEPS DT EPS SOLVER PREC TOL MAXIT INDIR OUTDIR [BE|FE|CN]
//   ofeli_ref ts2d NX NY   NSTEPS DT EPS BE|FE|CN SOLVER PREC TOL MAXIT INDIR OUTDIR
//   ofeli_ref mget FILE INDIR OUTDIR            (Mesh::get, dump, Mesh::put)
//   ofeli_ref mrect NX NY CX0 CXN CY0 CYN INDIR OUTDIR  (Mesh(rect), dump, put)
//   ofeli_ref mlap FILE SOLVER PREC TOL MAXIT INDIR OUTDIR
//   SOLVER = CG | GMRES<m> | BICGSTAB ; PREC = IDENT | DIAG | DILU | ILU | SSOR
// INDIR holds f.f64 (one value per node), optionally k.f64 (one value per
// element: scales the element stiffness), xy.f64 (2-D node coordinates that
// replace the structured ones), u0.f64 / v.f64 (cd2d initial field and the
// nodal velocity, interleaved vx,vy).
// OUTDIR receives info.txt (key=value), row_ptr.i64 (0-based), col_ind.i64
// (1-based, OFELI's own convention), a.f64, b.f64, x.f64 (equation space),
// u.f64 (nodal, boundary values inserted).  mget writes the mesh as Mesh::get
// keeps it (coords.f64, node_code.i32, elem.i32 with 1-based node labels,
// elem_code.i32, side.i32, side_code.i32, shapes and sizes in info.txt) and
// OUTDIR/put.m from Mesh::put; mlap solves the P1 problem of p2d (2-D) or
// p3d (3-D) on the mesh read from FILE by Mesh(FILE, true).
//
// Reference entry points used (paths within the OFELI project):
//   Mesh(xmin,xmax,ymin,ymax,nx,ny,c..,TRIANGLE)   src/mesh/Mesh.cpp:547-676
//   Mesh::Add / Node / Element                      include/mesh/Mesh.h:321-325
//   Laplace2DT3::LHS / BodyRHS                      src/equations/laplace/Laplace2DT3.cpp:131-143
//   DC3DT4::Diffusion / BodyRHS                     src/equations/therm/DC3DT4.cpp:128-135,207-211
//   DC2DT3 Capacity/LCapacity/Diffusion/Convection  src/equations/therm/DC2DT3.cpp:121-207
//   Equa_Laplace::build, Equa_Therm::build          include/equations/laplace/Equa_Laplace.h:112-133,
//                                                   include/equations/therm/Equa_Therm.h:162-218
//   Mesh::get / Mesh::put                           src/mesh/Mesh.cpp:2639-2668, 2731-2806
//   TimeStepping (setPDE, setInitial, setBC, setLinearSolver, runOneTimeStep)
//                                                   src/solvers/TimeStepping.cpp:141-250,341-460
//   Prec<real_t>(A,type), CG(A,P,b,x,..), GMRes(A,P,b,x,m,..)
//                                                   include/solvers/{Prec.h,CG.h:99-157,GMRes.h:148-241}
#include "OFELI.h"
#include "Laplace.h"
#include "Therm.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <string>
#include <vector>

using namespace OFELI;

namespace {

double now_s()
{
   using namespace std::chrono;
   return duration<double>(steady_clock::now().time_since_epoch()).count();
}

bool file_exists(const std::string& p)
{
   std::ifstream f(p, std::ios::binary);
   return bool(f);
}

std::vector<double> read_f64(const std::string& p, size_t n)
{
   std::ifstream f(p, std::ios::binary);
   if (!f) {
      fprintf(stderr, "missing input %s\n", p.c_str());
      exit(2);
   }
   std::vector<double> v(n);
   f.read(reinterpret_cast<char*>(v.data()), n * sizeof(double));
   if (size_t(f.gcount()) != n * sizeof(double)) {
      fprintf(stderr, "short input %s (want %zu values)\n", p.c_str(), n);
      exit(2);
   }
   return v;
}

template <class T>
void write_bin(const std::string& p, const T* d, size_t n)
{
   std::ofstream f(p, std::ios::binary);
   f.write(reinterpret_cast<const char*>(d), n * sizeof(T));
}

Preconditioner parse_prec(const std::string& s)
{
   if (s == "IDENT") return IDENT_PREC;
   if (s == "DIAG") return DIAG_PREC;
   if (s == "DILU") return DILU_PREC;
   if (s == "ILU") return ILU_PREC;
   if (s == "SSOR") return SSOR_PREC;
   fprintf(stderr, "unknown preconditioner %s\n", s.c_str());
   exit(2);
}

struct Info {
   std::map<std::string, std::string> kv;
   void set(const std::string& k, double v) { char b[64]; snprintf(b, 64, "%.17g", v); kv[k] = b; }
   void seti(const std::string& k, long long v) { kv[k] = std::to_string(v); }
   void sets(const std::string& k, const std::string& v) { kv[k] = v; }
   void write(const std::string& dir)
   {
      std::ofstream f(dir + "/info.txt");
      for (auto& e : kv) f << e.first << "=" << e.second << "\n";
   }
};

void dump_matrix(const SpMatrix<real_t>& A, const std::string& out, Info& info)
{
   size_t n = A.getNbRows(), nnz = A.getLength();
   std::vector<long long> rp(n + 1), ci(nnz);
   for (size_t i = 1; i <= n + 1; ++i) rp[i - 1] = (long long)A.getRowPtr(i);
   for (size_t k = 1; k <= nnz; ++k) ci[k - 1] = (long long)A.getColInd(k);
   write_bin(out + "/row_ptr.i64", rp.data(), n + 1);
   write_bin(out + "/col_ind.i64", ci.data(), nnz);
   std::vector<double> a(nnz);
   for (size_t k = 0; k < nnz; ++k) a[k] = A[k];
   write_bin(out + "/a.f64", a.data(), nnz);
   info.seti("n", (long long)n);
   info.seti("nnz", (long long)nnz);
}

// The stationary steps of Equa::run (src/equations/Equa.cpp:381-399) are
// replayed with each phase timed; the solve goes through the free Krylov
// functions so that the GMRES restart length can be chosen (LinearSolver
// forces m = n/5, src/solvers/LinearSolver.cpp:238).
template <class E>
int solve_system(E& eq, SpMatrix<real_t>& A, Vect<real_t>& b, Vect<real_t>& x,
                 const std::string& solver, Preconditioner p, int maxit, double tol,
                 double& t_prec, double& t_solve)
{
   double t0 = now_s();
   Prec<real_t> P(A, p);
   double t1 = now_s();
   int it;
   if (solver == "CG")
      it = CG(A, P, b, x, maxit, tol);
   else if (solver.rfind("GMRES", 0) == 0) {
      size_t m = std::stoul(solver.substr(5));
      it = GMRes(A, P, b, x, m, maxit, tol);
   }
   else if (solver == "BICGSTAB")
      it = BiCGStab(A, P, b, x, maxit, tol);
   else {
      fprintf(stderr, "unknown solver %s\n", solver.c_str());
      exit(2);
   }
   double t2 = now_s();
   t_prec = t1 - t0;
   t_solve = t2 - t1;
   return it;
}

// --- 2-D P1 Poisson with an optional per-element coefficient ---------------
class KLaplace2DT3 : public Laplace2DT3 {
 public:
   KLaplace2DT3(Mesh& ms, Vect<real_t>& u) : Equation<3,3,2,2>(ms, u), Laplace2DT3() { }
   const double* k = nullptr;
   void LHS() override
   {
      Laplace2DT3::LHS();
      if (k) eMat *= k[_theElement->n() - 1];
   }
   Matrix<real_t>* mat() { return _A; }
   Vect<real_t>* rhs() { return _b; }
   Vect<real_t>& sol() { return _uu; }
   size_t neq() const { return _nb_eq; }
};

// The same element with the setup of Equation(mesh,u) (Equation_impl.h
// :75-85,111-122) done by hand, so that the matrix graph is built once (by
// setSolver) instead of three times: Equa::setMesh (Equa.cpp:334-348) would
// build SpMatrix(mesh) twice before the caller's setSolver builds it again.
class BenchLaplace2DT3 : public Laplace2DT3 {
 public:
   BenchLaplace2DT3(Mesh& ms, Vect<real_t>& u) : Equation<3,3,2,2>(), Laplace2DT3()
   {
      _theMesh = &ms;
      _theMesh->removeImposedDOF();
      _nb_nodes = ms.getNbNodes();
      _nb_sides = ms.getNbSides();
      _nb_boundary_sides = ms.getNbBoundarySides();
      _nb_el = ms.getNbElements();
      _nb_dof_total = ms.getNbDOF();
      _nb_eq = ms.getNbEq();
      _nb_dof = 1;
      _b = new Vect<real_t>(_nb_eq);
      _uu.setSize(_nb_eq);
      _u = &u;
   }
   Matrix<real_t>* mat() { return _A; }
   Vect<real_t>* rhs() { return _b; }
   Vect<real_t>& sol() { return _uu; }
   size_t neq() const { return _nb_eq; }
};

// --- 3-D P1 diffusion (DC3DT4) with a per-element conductivity -------------
class KDC3DT4 : public DC3DT4 {
 public:
   KDC3DT4(Mesh& ms, Vect<real_t>& u) : Equation<4,4,3,3>(ms, u), DC3DT4() { }
   const double* k = nullptr;
   void Diffusion(real_t coef = 1) override
   {
      DC3DT4::Diffusion(k ? coef * k[_theElement->n() - 1] : coef);
   }
   Matrix<real_t>* mat() { return _A; }
   Vect<real_t>* rhs() { return _b; }
   Vect<real_t>& sol() { return _uu; }
   size_t neq() const { return _nb_eq; }
};

// --- 2-D transient convection-diffusion (DC2DT3) ---------------------------
class KDC2DT3 : public DC2DT3 {
 public:
   KDC2DT3(Mesh& ms, Vect<real_t>& u) : Equation<3,3,2,2>(ms, u), DC2DT3() { }
   double eps = 1.0;
   void Diffusion(real_t coef = 1) override { DC2DT3::Diffusion(coef * eps); }
   Matrix<real_t>* mat() { return _A; }
   Vect<real_t>* rhs() { return _b; }
   Vect<real_t>& sol() { return _uu; }
   size_t neq() const { return _nb_eq; }
   void set_dt(double dt) { _TimeInt.delta = dt; }
};

// Kuhn subdivision of the unit cube into M^3 cells, 6 tetrahedra per cell
// around the (0,0,0)-(1,1,1) diagonal.  Nodes are numbered x fastest; a node
// on any face gets code 1.  Odd permutations swap their last two interior
// vertices so every tetrahedron has a positive Jacobian.
void build_kuhn(Mesh& ms, size_t M)
{
   theMaterial.set(1, "Generic");
   ms.setDim(3);
   size_t P = M + 1;
   double h = 1.0 / double(M);
   std::vector<Node*> nodes;
   nodes.reserve(P * P * P);
   size_t lab = 0;
   for (size_t kz = 0; kz < P; ++kz)
      for (size_t jy = 0; jy < P; ++jy)
         for (size_t ix = 0; ix < P; ++ix) {
            Node* nd = new Node(++lab, Point<real_t>(ix * h, jy * h, kz * h));
            nd->setNbDOF(1);
            int code = (ix == 0 || jy == 0 || kz == 0 || ix == M || jy == M || kz == M) ? 1 : 0;
            nd->setCode(1, code);
            ms.Add(nd);
            nodes.push_back(nd);
         }
   // permutations of the axes (x=0,y=1,z=2) and their parity
   static const int perm[6][3] = {{0,1,2},{0,2,1},{1,0,2},{1,2,0},{2,0,1},{2,1,0}};
   static const int odd[6] = {0, 1, 1, 0, 0, 1};
   size_t el = 0;
   for (size_t kz = 0; kz < M; ++kz)
      for (size_t jy = 0; jy < M; ++jy)
         for (size_t ix = 0; ix < M; ++ix) {
            for (int t = 0; t < 6; ++t) {
               size_t c[3] = {ix, jy, kz};
               size_t v[4];
               v[0] = c[0] + P * (c[1] + P * c[2]);
               for (int s = 0; s < 3; ++s) {
                  c[perm[t][s]]++;
                  v[s + 1] = c[0] + P * (c[1] + P * c[2]);
               }
               if (odd[t]) std::swap(v[1], v[2]);
               Element* e = new Element(++el, TETRAHEDRON, 1);
               for (int q = 0; q < 4; ++q) e->Add(nodes[v[q]]);
               ms.Add(e);
            }
         }
   ms.setNodesForDOF();
   ms.NumberEquations();
}

int run_p2d(int argc, char** argv)
{
   if (argc < 10) return 2;
   size_t nx = std::stoul(argv[2]), ny = std::stoul(argv[3]);
   std::string solver = argv[4];
   Preconditioner prec = parse_prec(argv[5]);
   double tol = std::stod(argv[6]);
   int maxit = std::stoi(argv[7]);
   std::string in = argv[8], out = argv[9];
   Info info;

   // optional boundary line codes cx0 cxN cy0 cyN after OUTDIR
   int cx0 = 1, cxN = 1, cy0 = 1, cyN = 1;
   if (argc >= 14) {
      cx0 = std::stoi(argv[10]); cxN = std::stoi(argv[11]);
      cy0 = std::stoi(argv[12]); cyN = std::stoi(argv[13]);
   }
   double t0 = now_s();
   Mesh ms(0., 1., 0., 1., nx, ny, cx0, cxN, cy0, cyN, TRIANGLE);
   size_t nn = ms.getNbNodes(), ne = ms.getNbElements();
   if (file_exists(in + "/xy.f64")) {
      std::vector<double> xy = read_f64(in + "/xy.f64", 2 * nn);
      for (size_t i = 1; i <= nn; ++i) {
         ms.getPtrNode(i)->setCoord(1, xy[2 * (i - 1)]);
         ms.getPtrNode(i)->setCoord(2, xy[2 * (i - 1) + 1]);
      }
   }
   double t_mesh = now_s() - t0;
   std::vector<double> fv = read_f64(in + "/f.f64", nn);
   std::vector<double> kv;
   if (file_exists(in + "/k.f64")) kv = read_f64(in + "/k.f64", ne);

   Vect<real_t> u(ms), f(ms), bc(ms);
   for (size_t i = 0; i < nn; ++i) f[i] = fv[i];
   bc = 0;
   if (file_exists(in + "/bc.f64")) {
      std::vector<double> bv = read_f64(in + "/bc.f64", nn);
      for (size_t i = 0; i < nn; ++i) bc[i] = bv[i];
   }
   KLaplace2DT3 eq(ms, u);
   if (!kv.empty()) eq.k = kv.data();
   double t1 = now_s();
   eq.setSolver(CG_SOLVER, prec);          // SpMatrix(mesh): graph construction
   double t_graph = now_s() - t1;
   eq.setSource(f);
   eq.setDirichlet(bc);

   Vect<real_t>& b = *eq.rhs();
   b.clear();
   eq.sol().setSize(eq.neq());
   double t2 = now_s();
   eq.build();
   double t_asm = now_s() - t2;
   SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
   double t_prec = 0, t_solve = 0;
   int it = solve_system(eq, A, b, eq.sol(), solver, prec, maxit, tol, t_prec, t_solve);
   u.insertBC(ms, eq.sol(), bc);

   dump_matrix(A, out, info);
   write_bin(out + "/b.f64", &b[0], b.size());
   write_bin(out + "/x.f64", &eq.sol()[0], eq.sol().size());
   write_bin(out + "/u.f64", &u[0], u.size());
   info.seti("nodes", (long long)nn);
   info.seti("elements", (long long)ne);
   info.seti("iters", it);
   info.set("t_mesh", t_mesh);
   info.set("t_graph", t_graph);
   info.set("t_assembly", t_asm);
   info.set("t_prec", t_prec);
   info.set("t_solve", t_solve);
   info.set("norm_u", u.getNorm2());
   info.sets("solver", solver);
   info.sets("prec", argv[5]);
   info.write(out);
   return 0;
}

// Timed CPU baseline: graph once, then NSTEPS steps of {build, Prec, ITERS CG
// iterations}; the caller extrapolates the per-iteration time to a full solve.
int run_bench2d(int argc, char** argv)
{
   if (argc < 8) return 2;
   size_t nx = std::stoul(argv[2]);
   Preconditioner prec = parse_prec(argv[3]);
   int iters = std::stoi(argv[4]);
   int nsteps = std::stoi(argv[5]);
   std::string in = argv[6], out = argv[7];
   Info info;
   double t0 = now_s();
   Mesh ms(0., 1., 0., 1., nx, nx, 1, 1, 1, 1, TRIANGLE);
   size_t nn = ms.getNbNodes();
   double t_mesh = now_s() - t0;
   std::vector<double> fv = read_f64(in + "/f.f64", nn);
   Vect<real_t> u(ms), f(ms), bc(ms);
   for (size_t i = 0; i < nn; ++i) f[i] = fv[i];
   bc = 0;
   BenchLaplace2DT3 eq(ms, u);
   double t1 = now_s();
   eq.setSolver(CG_SOLVER, prec);
   double t_graph = now_s() - t1;
   eq.setSource(f);
   eq.setDirichlet(bc);
   std::string sa, sp, si;
   int it = 0;
   for (int s = 0; s < nsteps; ++s) {
      Vect<real_t>& b = *eq.rhs();
      b.clear();
      eq.sol().setSize(eq.neq());
      eq.sol() = 0;
      double ta = now_s();
      eq.build();
      double t_asm = now_s() - ta;
      SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
      double tp = now_s();
      Prec<real_t> P(A, prec);
      double t_prec = now_s() - tp;
      double tc = now_s();
      it = CG(A, P, b, eq.sol(), iters, 1e-300);
      double t_it = now_s() - tc;
      char buf[96];
      snprintf(buf, sizeof buf, "%s%.6f", s ? "," : "", t_asm); sa += buf;
      snprintf(buf, sizeof buf, "%s%.6f", s ? "," : "", t_prec); sp += buf;
      snprintf(buf, sizeof buf, "%s%.6f", s ? "," : "", t_it); si += buf;
   }
   info.seti("nodes", (long long)nn);
   info.seti("n", (long long)eq.neq());
   info.seti("iters", it);
   info.set("t_mesh", t_mesh);
   info.set("t_graph", t_graph);
   info.sets("t_assembly_steps", sa);
   info.sets("t_prec_steps", sp);
   info.sets("t_iters_steps", si);
   info.seti("iters_per_step", iters);
   info.write(out);
   return 0;
}

int run_p3d(int argc, char** argv)
{
   if (argc < 9) return 2;
   size_t M = std::stoul(argv[2]);
   std::string solver = argv[3];
   Preconditioner prec = parse_prec(argv[4]);
   double tol = std::stod(argv[5]);
   int maxit = std::stoi(argv[6]);
   std::string in = argv[7], out = argv[8];
   Info info;

   double t0 = now_s();
   Mesh ms;
   build_kuhn(ms, M);
   double t_mesh = now_s() - t0;
   size_t nn = ms.getNbNodes(), ne = ms.getNbElements();
   std::vector<double> fv = read_f64(in + "/f.f64", nn);
   std::vector<double> kv;
   if (file_exists(in + "/k.f64")) kv = read_f64(in + "/k.f64", ne);

   Vect<real_t> u(ms), f(ms), bc(ms);
   for (size_t i = 0; i < nn; ++i) f[i] = fv[i];
   bc = 0;
   KDC3DT4 eq(ms, u);
   if (!kv.empty()) eq.k = kv.data();
   double t1 = now_s();
   eq.setSolver(CG_SOLVER, prec);
   double t_graph = now_s() - t1;
   eq.setSource(f);
   eq.setDirichlet(bc);

   Vect<real_t>& b = *eq.rhs();
   b.clear();
   eq.sol().setSize(eq.neq());
   double t2 = now_s();
   eq.build();
   double t_asm = now_s() - t2;
   SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
   double t_prec = 0, t_solve = 0;
   int it = solve_system(eq, A, b, eq.sol(), solver, prec, maxit, tol, t_prec, t_solve);
   u.insertBC(ms, eq.sol(), bc);

   dump_matrix(A, out, info);
   write_bin(out + "/b.f64", &b[0], b.size());
   write_bin(out + "/x.f64", &eq.sol()[0], eq.sol().size());
   write_bin(out + "/u.f64", &u[0], u.size());
   info.seti("nodes", (long long)nn);
   info.seti("elements", (long long)ne);
   info.seti("iters", it);
   info.set("t_mesh", t_mesh);
   info.set("t_graph", t_graph);
   info.set("t_assembly", t_asm);
   info.set("t_prec", t_prec);
   info.set("t_solve", t_solve);
   info.set("norm_u", u.getNorm2());
   info.sets("solver", solver);
   info.sets("prec", argv[4]);
   info.write(out);
   return 0;
}

// Backward-Euler steps of Equa_Therm::build with capacity, diffusion (eps)
// and convection terms; b is cleared before every step and the previous
// equation-space solution is the GMRES initial guess.
int run_cd2d(int argc, char** argv)
{
   if (argc < 13) return 2;
   size_t nx = std::stoul(argv[2]), ny = std::stoul(argv[3]);
   int nsteps = std::stoi(argv[4]);
   double dt = std::stod(argv[5]), eps = std::stod(argv[6]);
   std::string solver = argv[7];
   Preconditioner prec = parse_prec(argv[8]);
   double tol = std::stod(argv[9]);
   int maxit = std::stoi(argv[10]);
   std::string in = argv[11], out = argv[12];
   Info info;

   Mesh ms(0., 1., 0., 1., nx, ny, 1, 1, 1, 1, TRIANGLE);
   size_t nn = ms.getNbNodes(), ne = ms.getNbElements();
   std::vector<double> u0 = read_f64(in + "/u0.f64", nn);
   std::vector<double> vv = read_f64(in + "/v.f64", 2 * nn);
   Vect<real_t> u(ms), v(2 * nn), bc(ms);
   for (size_t i = 0; i < nn; ++i) u[i] = u0[i];
   for (size_t i = 0; i < 2 * nn; ++i) v[i] = vv[i];
   bc = 0;
   KDC2DT3 eq(ms, u);
   eq.eps = eps;
   double t1 = now_s();
   eq.setSolver(GMRES_SOLVER, prec);
   double t_graph = now_s() - t1;
   eq.setTerms(PDE_Terms::CAPACITY);
   eq.setTerms(PDE_Terms::CONVECTION);
   eq.setInput(EType::VELOCITY, v);
   eq.setDirichlet(bc);
   // optional time scheme after OUTDIR: BE (default), FE, CN
   TimeScheme scheme = BACKWARD_EULER;
   if (argc >= 14) {
      std::string sc = argv[13];
      scheme = sc == "FE" ? FORWARD_EULER : sc == "CN" ? CRANK_NICOLSON : BACKWARD_EULER;
   }
   eq.setTransient(scheme);
   eq.set_dt(dt);

   Vect<real_t>& b = *eq.rhs();
   eq.sol().setSize(eq.neq());
   double t_asm = 0, t_prec = 0, t_solve = 0;
   long long it_total = 0;
   int it_last = 0, worst = 1 << 30;
   std::vector<int> its;
   for (int s = 0; s < nsteps; ++s) {
      b.clear();
      double ta = now_s();
      eq.build();
      t_asm += now_s() - ta;
      SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
      double tp = 0, ts = 0;
      it_last = solve_system(eq, A, b, eq.sol(), solver, prec, maxit, tol, tp, ts);
      t_prec += tp;
      t_solve += ts;
      its.push_back(it_last);
      it_total += it_last > 0 ? it_last : -it_last;
      if (it_last < worst) worst = it_last;
      u.insertBC(ms, eq.sol(), bc);
      if (s == 0) {
         dump_matrix(A, out, info);
         write_bin(out + "/b0.f64", &b[0], b.size());
         write_bin(out + "/x0.f64", &eq.sol()[0], eq.sol().size());
      }
   }
   SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
   std::vector<double> a_last(A.getLength());
   for (size_t k = 0; k < a_last.size(); ++k) a_last[k] = A[k];
   write_bin(out + "/a_last.f64", a_last.data(), a_last.size());
   write_bin(out + "/b.f64", &b[0], b.size());
   write_bin(out + "/x.f64", &eq.sol()[0], eq.sol().size());
   write_bin(out + "/u.f64", &u[0], u.size());
   write_bin(out + "/iters.i32", its.data(), its.size());
   info.seti("nodes", (long long)nn);
   info.seti("elements", (long long)ne);
   info.seti("iters", it_last);
   info.seti("iters_total", it_total);
   info.seti("iters_min", worst);
   info.seti("steps", nsteps);
   info.set("t_graph", t_graph);
   info.set("t_assembly", t_asm);
   info.set("t_prec", t_prec);
   info.set("t_solve", t_solve);
   info.set("norm_u", u.getNorm2());
   info.sets("solver", solver);
   info.sets("prec", argv[8]);
   info.write(out);
   return 0;
}

// DC2DT3 steps driven by OFELI's TimeStepping class (src/solvers/
// TimeStepping.cpp): setPDE, setInitial, setBC (a zero vector: without one,
// TimeStepping::insertBC assigns the equation-space solution to the nodal
// field), setLinearSolver, runOneTimeStep per step.  The linear solves are
// the equation's LinearSolver (GMRES restarts every n/5 steps) with the
// given tolerance; forward Euler is explicit (lumped diagonal).  Writes the
// nodal field after every step (u_steps.f64) and the solver's iteration
// count per step.
int run_ts2d(int argc, char** argv)
{
   if (argc < 14) return 2;
   size_t nx = std::stoul(argv[2]), ny = std::stoul(argv[3]);
   int nsteps = std::stoi(argv[4]);
   double dt = std::stod(argv[5]), eps = std::stod(argv[6]);
   std::string sc = argv[7], solver = argv[8];
   Preconditioner prec = parse_prec(argv[9]);
   double tol = std::stod(argv[10]);
   int maxit = std::stoi(argv[11]);
   std::string in = argv[12], out = argv[13];
   Info info;
   TimeScheme scheme = sc == "FE" ? FORWARD_EULER : sc == "CN" ? CRANK_NICOLSON : BACKWARD_EULER;
   Iteration it_kind = solver == "CG" ? CG_SOLVER
                       : solver == "BICGSTAB" ? BICG_STAB_SOLVER : GMRES_SOLVER;

   Mesh ms(0., 1., 0., 1., nx, ny, 1, 1, 1, 1, TRIANGLE);
   size_t nn = ms.getNbNodes();
   std::vector<double> u0 = read_f64(in + "/u0.f64", nn);
   std::vector<double> vv = read_f64(in + "/v.f64", 2 * nn);
   Vect<real_t> u(ms), v(2 * nn), bc(ms);
   for (size_t i = 0; i < nn; ++i) u[i] = u0[i];
   for (size_t i = 0; i < 2 * nn; ++i) v[i] = vv[i];
   bc = 0;
   KDC2DT3 eq(ms, u);
   eq.eps = eps;
   eq.setSolver(it_kind, prec);
   eq.getLinearSolver().setTolerance(tol);
   eq.getLinearSolver().setMaxIter(maxit);
   eq.setTerms(PDE_Terms::CAPACITY);
   eq.setTerms(PDE_Terms::CONVECTION);
   eq.setInput(EType::VELOCITY, v);
   TimeStepping ts(scheme, dt, nsteps * dt);
   ts.setPDE(eq);
   ts.setInitial(u);
   ts.setBC(bc);
   ts.setLinearSolver(it_kind, prec);
   std::vector<double> steps;
   std::vector<int> its;
   double t0 = now_s();
   for (int s = 0; s < nsteps; ++s) {
      ts.runOneTimeStep();
      its.push_back(scheme == FORWARD_EULER ? 0 : eq.getLinearSolver().getNbIter());
      for (size_t i = 0; i < nn; ++i) steps.push_back(u[i]);
   }
   double t_steps = now_s() - t0;
   write_bin(out + "/u_steps.f64", steps.data(), steps.size());
   write_bin(out + "/iters.i32", its.data(), its.size());
   info.seti("nodes", (long long)nn);
   info.seti("steps", nsteps);
   info.set("t_steps", t_steps);
   info.set("norm_u", u.getNorm2());
   info.sets("scheme", sc);
   info.write(out);
   return 0;
}

// The data a Mesh keeps (coords, codes, 1-based element / side node labels)
// and Mesh::put of it.
void dump_mesh(Mesh& ms, const std::string& out, Info& info)
{
   size_t nn = ms.getNbNodes(), ne = ms.getNbElements(), ns = ms.getNbSides();
   size_t dim = ms.getDim();
   size_t nd = nn ? ms.getPtrNode(1)->getNbDOF() : 0;
   std::vector<double> xy;
   std::vector<int> nc;
   for (size_t i = 1; i <= nn; ++i) {
      Node* p = ms.getPtrNode(i);
      for (size_t k = 1; k <= dim; ++k) xy.push_back(p->getCoord(k));
      for (size_t k = 1; k <= nd; ++k) nc.push_back(p->getCode(k));
   }
   std::vector<int> el, ec, sd, sc;
   size_t enn = ne ? ms.getPtrElement(1)->getNbNodes() : 0;
   for (size_t i = 1; i <= ne; ++i) {
      Element* e = ms.getPtrElement(i);
      for (size_t k = 1; k <= e->getNbNodes(); ++k) el.push_back((int)(*e)(k)->n());
      ec.push_back(e->getCode());
   }
   size_t snn = ns ? ms.getPtrSide(1)->getNbNodes() : 0;
   for (size_t i = 1; i <= ns; ++i) {
      Side* s = ms.getPtrSide(i);
      for (size_t k = 1; k <= s->getNbNodes(); ++k) sd.push_back((int)(*s)(k)->n());
      for (size_t k = 1; k <= nd; ++k) sc.push_back(s->getCode(k));
   }
   write_bin(out + "/coords.f64", xy.data(), xy.size());
   write_bin(out + "/node_code.i32", nc.data(), nc.size());
   write_bin(out + "/elem.i32", el.data(), el.size());
   write_bin(out + "/elem_code.i32", ec.data(), ec.size());
   write_bin(out + "/side.i32", sd.data(), sd.size());
   write_bin(out + "/side_code.i32", sc.data(), sc.size());
   double t1 = now_s();
   ms.put(out + "/put.m");
   info.set("t_put", now_s() - t1);
   info.seti("dim", (long long)dim);
   info.seti("nb_dof", (long long)nd);
   info.seti("nodes", (long long)nn);
   info.seti("elements", (long long)ne);
   info.seti("sides", (long long)ns);
   info.seti("el_shape", ne ? (long long)ms.getPtrElement(1)->getShape() : 0);
   info.seti("el_nodes", (long long)enn);
   info.seti("sd_shape", ns ? (long long)ms.getPtrSide(1)->getShape() : 0);
   info.seti("sd_nodes", (long long)snn);
}

// Mesh::get of an OFELI .m file (INDIR unused).
int run_mget(int argc, char** argv)
{
   if (argc < 5) return 2;
   std::string file = argv[2], out = argv[4];
   Info info;
   double t0 = now_s();
   Mesh ms;
   ms.get(file);
   info.set("t_get", now_s() - t0);
   dump_mesh(ms, out, info);
   info.write(out);
   return 0;
}

// The structured rectangle mesh of Mesh(0,1,0,1,nx,ny,cx0,cxN,cy0,cyN,
// TRIANGLE), whose negative line codes give negative node codes and sides.
int run_mrect(int argc, char** argv)
{
   if (argc < 10) return 2;
   size_t nx = std::stoul(argv[2]), ny = std::stoul(argv[3]);
   int c[4];
   for (int i = 0; i < 4; ++i) c[i] = std::stoi(argv[4 + i]);
   std::string out = argv[9];
   Info info;
   Mesh ms(0., 1., 0., 1., nx, ny, c[0], c[1], c[2], c[3], TRIANGLE);
   dump_mesh(ms, out, info);
   info.write(out);
   return 0;
}

// The p2d / p3d problem on a mesh read from a file: Mesh(FILE, true), then
// the 2-D Laplace (KLaplace2DT3) or 3-D diffusion (KDC3DT4) equation.
template <class EQ>
int solve_on_file_mesh(Mesh& ms, const std::string& solver, Preconditioner prec, const char* pname,
                       double tol, int maxit, const std::string& in, const std::string& out,
                       Info& info)
{
   size_t nn = ms.getNbNodes(), ne = ms.getNbElements();
   std::vector<double> fv = read_f64(in + "/f.f64", nn);
   std::vector<double> kv;
   if (file_exists(in + "/k.f64")) kv = read_f64(in + "/k.f64", ne);
   Vect<real_t> u(ms), f(ms), bc(ms);
   for (size_t i = 0; i < nn; ++i) f[i] = fv[i];
   bc = 0;
   if (file_exists(in + "/bc.f64")) {
      std::vector<double> bv = read_f64(in + "/bc.f64", nn);
      for (size_t i = 0; i < nn; ++i) bc[i] = bv[i];
   }
   EQ eq(ms, u);
   if (!kv.empty()) eq.k = kv.data();
   double t1 = now_s();
   eq.setSolver(CG_SOLVER, prec);
   double t_graph = now_s() - t1;
   eq.setSource(f);
   eq.setDirichlet(bc);
   Vect<real_t>& b = *eq.rhs();
   b.clear();
   eq.sol().setSize(eq.neq());
   double t2 = now_s();
   eq.build();
   double t_asm = now_s() - t2;
   SpMatrix<real_t>& A = *dynamic_cast<SpMatrix<real_t>*>(eq.mat());
   double t_prec = 0, t_solve = 0;
   int it = solve_system(eq, A, b, eq.sol(), solver, prec, maxit, tol, t_prec, t_solve);
   u.insertBC(ms, eq.sol(), bc);
   dump_matrix(A, out, info);
   write_bin(out + "/b.f64", &b[0], b.size());
   write_bin(out + "/x.f64", &eq.sol()[0], eq.sol().size());
   write_bin(out + "/u.f64", &u[0], u.size());
   info.seti("nodes", (long long)nn);
   info.seti("elements", (long long)ne);
   info.seti("iters", it);
   info.set("t_graph", t_graph);
   info.set("t_assembly", t_asm);
   info.set("t_prec", t_prec);
   info.set("t_solve", t_solve);
   info.set("norm_u", u.getNorm2());
   info.sets("solver", solver);
   info.sets("prec", pname);
   return 0;
}

int run_mlap(int argc, char** argv)
{
   if (argc < 9) return 2;
   std::string file = argv[2], solver = argv[3];
   Preconditioner prec = parse_prec(argv[4]);
   double tol = std::stod(argv[5]);
   int maxit = std::stoi(argv[6]);
   std::string in = argv[7], out = argv[8];
   Info info;
   double t0 = now_s();
   Mesh ms(file, true);
   info.set("t_mesh", now_s() - t0);
   int rc;
   if (ms.getDim() == 3)
      rc = solve_on_file_mesh<KDC3DT4>(ms, solver, prec, argv[4], tol, maxit, in, out, info);
   else
      rc = solve_on_file_mesh<KLaplace2DT3>(ms, solver, prec, argv[4], tol, maxit, in, out, info);
   info.write(out);
   return rc;
}

}  // namespace

int main(int argc, char** argv)
{
   Verbosity = 0;
   if (argc < 2) {
      fprintf(stderr, "usage: ofeli_ref p2d|p3d|cd2d ...\n");
      return 2;
   }
   std::string mode = argv[1];
   try {
      if (mode == "p2d") return run_p2d(argc, argv);
      if (mode == "p3d") return run_p3d(argc, argv);
      if (mode == "cd2d") return run_cd2d(argc, argv);
      if (mode == "ts2d") return run_ts2d(argc, argv);
      if (mode == "bench2d") return run_bench2d(argc, argv);
      if (mode == "mget") return run_mget(argc, argv);
      if (mode == "mrect") return run_mrect(argc, argv);
      if (mode == "mlap") return run_mlap(argc, argv);
   }
   catch (std::exception& e) {
      fprintf(stderr, "OFELI exception: %s\n", e.what());
      return 3;
   }
   fprintf(stderr, "bad arguments\n");
   return 2;
}

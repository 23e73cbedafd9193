// laplace_demo.cpp -- OFELI-style program on the GPU path: -Delta u = f on
// the unit square, P1 triangles, u = 0 on the boundary, solved with CG and
// the preconditioner named on the command line.
//   laplace_demo NX PREC f.f64 u.f64
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>

#include "ofeli_b200/OFELI.h"

using namespace OFELI;

int main(int argc, char** argv)
{
   if (argc < 5) {
      fprintf(stderr, "usage: laplace_demo NX DIAG|DILU|ILU|SSOR f.f64 u.f64\n");
      return 2;
   }
   size_t nx = std::strtoul(argv[1], nullptr, 10);
   Preconditioner p = DIAG_PREC;
   if (!std::strcmp(argv[2], "DILU")) p = DILU_PREC;
   if (!std::strcmp(argv[2], "ILU")) p = ILU_PREC;
   if (!std::strcmp(argv[2], "SSOR")) p = SSOR_PREC;
   try {
      Mesh ms(0., 1., 0., 1., nx, nx, 1, 1, 1, 1, TRIANGLE);
      Vect<real_t> u(ms.getNbNodes()), f(ms.getNbNodes()), bc(ms.getNbNodes());
      std::ifstream in(argv[3], std::ios::binary);
      in.read(reinterpret_cast<char*>(f.data()), f.size() * sizeof(real_t));
      if (!in) throw OFELIException("cannot read f");
      Laplace2DT3 eq(ms, u);
      eq.setSolver(CG_SOLVER, p);
      eq.getLinearSolver().setTolerance(1.e-10);
      eq.getLinearSolver().setMaxIter(20000);
      eq.setSource(f);
      eq.setDirichlet(bc);
      int ret = eq.run();
      std::ofstream out(argv[4], std::ios::binary);
      out.write(reinterpret_cast<const char*>(u.data()), u.size() * sizeof(real_t));
      printf("equations %zu nonzeros %zu iterations %d ret %d norm %.17g\n", ms.getNbEq(),
             eq.getMatrix()->getLength(), eq.getLinearSolver().getNbIter(), ret, u.getNorm2());
      // SpMatrix / Prec / CG used directly, as OFELI's linear-algebra demos do
      SpMatrix<real_t>& A = *eq.getMatrix();
      Vect<real_t> x(A.size()), b(eq.getRHS());
      int it = CG(A, Prec<real_t>(A, p), b, x, 20000, 1.e-10);
      Vect<real_t> r = A * x;
      for (size_t i = 0; i < r.size(); ++i) r[i] = b[i] - r[i];
      printf("direct CG iterations %d residual %.3e\n", it, r.getNorm2() / b.getNorm2());
   }
   catch (OFELIException& e) {
      fprintf(stderr, "OFELI exception: %s\n", e.what());
      return 1;
   }
   return 0;
}

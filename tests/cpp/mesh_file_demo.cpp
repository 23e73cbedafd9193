// mesh_file_demo.cpp -- OFELI-style program reading its mesh from an OFELI
// .m file: -div(grad u) = f with u = 0 on the coded nodes, P1 elements (2-D
// Laplace2DT3 or 3-D DC3DT4 by the file's dimension), CG + D-ILU; the mesh
// is written back with Mesh::put.
//   mesh_file_demo MESH.m f.f64 u.f64 PUT.m
#include <cstdio>
#include <fstream>

#include "ofeli_b200/OFELI.h"

using namespace OFELI;

template <class EQ>
int solve(Mesh& ms, Vect<real_t>& u, Vect<real_t>& f, Vect<real_t>& bc)
{
   EQ eq(ms, u);
   eq.setSolver(CG_SOLVER, DILU_PREC);
   eq.getLinearSolver().setTolerance(1.e-10);
   eq.getLinearSolver().setMaxIter(20000);
   eq.setSource(f);
   eq.setDirichlet(bc);
   eq.run();
   return eq.getLinearSolver().getNbIter();
}

int main(int argc, char** argv)
{
   if (argc < 5) {
      fprintf(stderr, "usage: mesh_file_demo MESH.m f.f64 u.f64 PUT.m\n");
      return 2;
   }
   try {
      Mesh ms(argv[1], true);
      size_t nn = ms.getNbNodes();
      Vect<real_t> u(nn), f(nn), bc(nn);
      std::ifstream in(argv[2], std::ios::binary);
      in.read(reinterpret_cast<char*>(f.data()), f.size() * sizeof(real_t));
      if (!in) throw OFELIException("cannot read f");
      int it = ms.getDim() == 3 ? solve<DC3DT4>(ms, u, f, bc) : solve<Laplace2DT3>(ms, u, f, bc);
      std::ofstream out(argv[3], std::ios::binary);
      out.write(reinterpret_cast<const char*>(u.data()), u.size() * sizeof(real_t));
      ms.put(argv[4]);
      printf("dim %zu nodes %zu elements %zu equations %zu iterations %d\n", ms.getDim(), nn,
             ms.getNbElements(), ms.getNbEq(), it);
   }
   catch (OFELIException& e) {
      fprintf(stderr, "OFELI exception: %s\n", e.what());
      return 1;
   }
   return 0;
}

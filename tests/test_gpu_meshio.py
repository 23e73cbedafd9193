"""Meshes read from OFELI .m files feeding the CUDA path: Mesh(file, true)
with the 2-D Laplace and 3-D diffusion problems, against the reference
OFELI run on the same files (golden outputs in tests/golden/meshio.npz),
and Mesh::put of device meshes.

Bars as in the other parity tests: CSR pattern bit-exact; values, RHS and
solutions within 1e-12 relative (BiCGStab solutions 1e-8); iteration counts
within +-2; put output byte-identical."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_err
from ofeli_b200 import fields
from ofeli_b200 import ofeli as F

pytestmark = pytest.mark.gpu

VAL_TOL = 1e-12
SOL_TOL = 1e-12
BICG_SOL_TOL = 1e-8
IT_TOL = 2
PRECS = {"DIAG": F.DIAG_PREC, "DILU": F.DILU_PREC, "ILU": F.ILU_PREC}
SOLVERS = {"CG": F.CG_SOLVER, "BICGSTAB": F.BICG_STAB_SOLVER}


@pytest.fixture(scope="module")
def golden():
    return load_golden("meshio")


def file_problem(cuda, key, golden):
    g, info = golden
    mesh = F.Mesh.from_file(os.path.join(GOLDEN, "meshio_%s.m" % key))
    mf = F.MeshFile(os.path.join(GOLDEN, "meshio_%s.m" % key))
    a = mf.arrays()
    if key == "ring":
        eq = F.Laplace2DT3(mesh)
        code = a["node_code"][:, 0]
        eq.setSource(fields.uniform_pm1(info["ring"]["seed_f"], mesh.nn))
        eq.setDirichlet(np.where(code == 2, info["ring"]["bc_outer"], 0.0))
        eq.setElementCoefficient(np.where(a["elem_code"] == 2, 3.0, 1.0))
    else:
        eq = F.DC3DT4(mesh)
        eq.setSource(fields.uniform_pm1(info["tet"]["seed_f"], mesh.nn))
        eq.setDirichlet(np.zeros(mesh.nn))
    return g, info, mesh, eq


@pytest.mark.parametrize("key", ["ring", "tet"])
def test_file_mesh_assembly(cuda, golden, key):
    g, _, mesh, eq = file_problem(cuda, key, golden)
    c, e, code, _ = mesh.arrays()
    assert np.array_equal(c, g[key + "_coords"]) and np.array_equal(e, g[key + "_elem"])
    assert np.array_equal(code, g[key + "_node_code"])
    eq.build()
    A = eq.getMatrix()
    rp, ci = A.pattern()
    assert np.array_equal(rp, g[key + "_row_ptr"]) and np.array_equal(ci, g[key + "_col_ind"])
    assert rel_err(A.values(), g[key + "_a"]) <= VAL_TOL
    assert rel_err(eq.getRHS(), g[key + "_b"]) <= VAL_TOL


@pytest.mark.parametrize("run", ["ring_CG_DILU", "ring_CG_DIAG", "ring_BICGSTAB_ILU",
                                 "tet_CG_DILU"])
def test_file_mesh_solve(cuda, golden, run):
    key, solver, prec = run.split("_")
    g, info, mesh, eq = file_problem(cuda, key, golden)
    eq.setSolver(SOLVERS[solver], PRECS[prec])
    eq.getLinearSolver().setTolerance(1e-10)
    eq.getLinearSolver().setMaxIter(20000)
    eq.run()
    tol = BICG_SOL_TOL if solver == "BICGSTAB" else SOL_TOL
    assert abs(eq.getLinearSolver().getNbIter() - info["runs"][run]["iters"]) <= IT_TOL
    assert rel_err(eq.x, g["%s_x_%s_%s" % (key, solver, prec)]) <= tol
    assert rel_err(eq.u, g["%s_u_%s_%s" % (key, solver, prec)]) <= tol


def test_put_of_file_mesh(cuda, golden, tmp_path):
    g, _ = golden
    mesh = F.Mesh.from_file(os.path.join(GOLDEN, "meshio_ring.m"))
    mesh.put(tmp_path / "ring.m")
    assert (tmp_path / "ring.m").read_bytes() == g["ring_put"].tobytes()
    m2 = F.Mesh(0.0, 1.0, 0.0, 1.0, 2, 2)
    m2.get(os.path.join(GOLDEN, "meshio_tet.m"))
    assert (m2.dim, m2.nn, m2.ne) == (3, 64, 162)
    m2.save(tmp_path / "tet.m")
    assert (tmp_path / "tet.m").read_bytes() == g["tet_put"].tobytes()


def test_put_of_rectangle_with_sides(cuda, golden, tmp_path):
    """Mesh(0,1,0,1,4,3,-1,2,-3,0): OFELI adds LINE sides (code 1 on x = 0,
    3 on y = 0) for the negative line codes."""
    g, _ = golden
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, 4, 3, -1, 2, -3, 0)
    mesh.put(tmp_path / "rect.m")
    assert (tmp_path / "rect.m").read_bytes() == g["rect_put"].tobytes()


def test_non_p1_file_refused(cuda, tmp_path):
    p = tmp_path / "quad.m"
    p.write_text('<OFELI_File><Mesh dim="2" nb_dof="1"><Nodes>0 0 1 1 0 1 1 1 1 0 1 1</Nodes>'
                 '<Elements shape="quadrilateral" nodes="4">1 2 3 4 1</Elements></Mesh>'
                 '</OFELI_File>')
    with pytest.raises(F.OFELIException):
        F.Mesh.from_file(p)

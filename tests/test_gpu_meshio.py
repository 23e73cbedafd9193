"""Meshes read from OFELI .m files feeding the CUDA path: Mesh(file, true)
with the 2-D Laplace and 3-D diffusion problems, against the reference
OFELI run on the same files (golden outputs in tests/golden/meshio.npz),
and Mesh::put of device meshes.

Bars as in the other parity tests: CSR pattern, assembled values and RHS
bit-exact; solutions within 1e-12 relative (BiCGStab solutions 1e-8);
iteration counts within +-2; put output byte-identical; the device reader's
mesh bit-identical to the host reader's."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden, rel_err
from ofeli_b200 import fields
from ofeli_b200 import ofeli as F

pytestmark = pytest.mark.gpu

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
    assert np.array_equal(A.values(), g[key + "_a"])
    assert np.array_equal(eq.getRHS(), g[key + "_b"])


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


def both_readers(path):
    """(device reader's mesh arrays, host reader's mesh arrays)."""
    dev = F.Mesh.from_file(path).arrays()
    host = F.MeshFile(path).to_mesh().arrays()
    return dev, host


def assert_same_mesh(dev, host):
    assert np.array_equal(dev[0].view(np.int64), host[0].view(np.int64))  # bitwise coordinates
    for a, b in zip(dev[1:], host[1:]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("key", ["ring", "tet"])
def test_device_reader_matches_host_reader(cuda, golden, key):
    g, _ = golden
    dev, host = both_readers(os.path.join(GOLDEN, "meshio_%s.m" % key))
    assert_same_mesh(dev, host)
    assert np.array_equal(dev[0], g[key + "_coords"])


FORMS = {"put": lambda v: "%.8e" % v, "shortest": repr, "fixed3": lambda v: "%.3f" % v,
         "hex": float.hex}


def ring_text(nr, nt, seed, form="put"):
    from ofeli_b200 import problems
    xy, elem, code, _, _ = problems.ring_mesh(nr, nt, seed=seed)
    fmt = FORMS[form]
    lines = ['<?xml version="1.0"?>', "<OFELI_File>", '<Mesh dim="2" nb_dof="1">', "<Nodes>"]
    lines += ["%s %s %d" % (fmt(float(x)), fmt(float(y)), c) for (x, y), c in zip(xy, code)]
    lines += ["</Nodes>", '<Elements shape="triangle" nodes="3">']
    lines += ["%d %d %d 1" % tuple(e + 1) for e in elem]
    lines += ["</Elements>", "</Mesh>", "</OFELI_File>"]
    return "\n".join(lines) + "\n", xy.shape[0]


@pytest.mark.parametrize("form", sorted(FORMS))
def test_device_reader_number_forms(cuda, tmp_path, form):
    """Nine-digit exponent form (Mesh::put), shortest round-trip decimals,
    few digits, and C99 hexadecimal floats (host-converted) on a 30k-node
    file: device and host readers agree bit for bit."""
    text, _ = ring_text(60, 500, 3, form)
    p = tmp_path / "forms.m"
    p.write_text(text)
    assert_same_mesh(*both_readers(p))


def test_device_reader_hard_tokens(cuda, tmp_path):
    """Tokens off the device's fast path (sign '+', hexadecimal, long
    mantissas, wide exponents, exact float midpoints after double rounding,
    infinities) land on the host conversion and agree with it."""
    toks = ["1.0000000596046448", "-1.0000000596046448", "+0.5", "0x1.8p1", "1e-30", "3e25",
            "123456789012345678901234567890", "0.000000000000000000000000012345", "inf",
            "1.00000001e-01", "16777217", "0.30000001192092896", "1e", "-0", "5.", ".25",
            "1.17549435e-38", "3.40282346e38", "2.0000001192092896", "7.0000004"]
    text, nn = ring_text(4, 8, 5)
    lines = text.split("\n")
    i0 = lines.index("<Nodes>") + 1
    for j, t in enumerate(toks):
        parts = lines[i0 + j].split()
        lines[i0 + j] = "%s %s %s" % (t, parts[1], parts[2])
    p = tmp_path / "hard.m"
    p.write_text("\n".join(lines))
    dev, host = both_readers(p)
    assert_same_mesh(dev, host)
    assert dev[0][0] == np.float32(1.0000001192092896)


@pytest.mark.parametrize("bad", ["label", "int", "char", "cut", "code", "range"])
def test_device_reader_rejects_like_host(cuda, tmp_path, bad):
    text, nn = ring_text(4, 8, 5)
    if bad == "label":
        text = text.replace('nodes="3">\n', 'nodes="3">\n%d 1 2 1\n' % (nn + 1), 1)
    elif bad == "int":
        text = text.replace('nodes="3">\n', 'nodes="3">\n1 2 x 1\n', 1)
    elif bad == "char":
        text = text.replace("<Nodes>\n", "<Nodes>\n0 0 1 &amp;\n", 1)
    elif bad == "cut":
        text = text.replace("</Nodes>", "0.5\n</Nodes>", 1)
    elif bad == "code":
        text = text.replace("<Nodes>\n", "<Nodes>\n0 0 -2147483648\n", 1)
    else:
        text = text.replace('nodes="3">\n', 'nodes="3">\n1 2 99999999999 1\n', 1)
    p = tmp_path / ("bad_%s.m" % bad)
    p.write_text(text)
    with pytest.raises(F.OFELIException):
        F.MeshFile(p).to_mesh()
    with pytest.raises(F.OFELIException):
        F.Mesh.from_file(p)


def test_device_reader_large_file(cuda, tmp_path):
    """A 4.6M-triangle annulus written by put(): many tiles, tokens across
    every tile boundary."""
    from ofeli_b200 import problems
    xy, elem, code, sides, smark = problems.ring_mesh(600, 3840, seed=9)
    mf = F.MeshFile.create(2, xy, code, elem, np.ones(elem.shape[0], np.int32), F.TRIANGLE,
                           sides=sides, side_code=smark)
    p = tmp_path / "large.m"
    mf.put(p)
    assert_same_mesh(*both_readers(p))

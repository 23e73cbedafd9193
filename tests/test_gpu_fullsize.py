"""Full-size checks at the benchmark configuration (2049x2049 nodes, 4.19M
unknowns, 29.3M nonzeros) and the 3-D one (129^3 Kuhn cube): the pattern
bit-exact against the oracle's NodeGraph, values / SpMV / preconditioner
applications against the oracle, linearity, and the FP64 accuracy of the
solves."""
import numpy as np
import pytest

from conftest import rel_err
from ofeli_b200 import fields
from ofeli_b200 import ofeli as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NX = 2048


@pytest.fixture(scope="module")
def big(cuda):
    xy, elem, code = O.mesh2d(NX, NX)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    f = fields.uniform_pm1(1234, code.size)
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, NX, NX)
    eq = F.Laplace2DT3(mesh)
    eq.setSolver(F.CG_SOLVER, F.DIAG_PREC)
    eq.setSource(f)
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.build()
    return dict(rp=rp, ci=ci, a=a, b=b, eq=eq, A=eq.getMatrix(), n=n)


def test_bench_config_sizes(big):
    assert big["n"] == 4190209 and big["A"].nnz == 29315089


def test_pattern_and_values_full_size(big):
    rp, ci = big["A"].pattern()
    assert np.array_equal(rp, big["rp"]) and np.array_equal(ci, big["ci"])
    # the row gather adds each entry's element contributions in OFELI's
    # element order with separate roundings: bit for bit at full size too
    assert np.array_equal(big["A"].values(), big["a"])
    assert np.array_equal(big["eq"].getRHS(), big["b"])


def test_spmv_and_linearity_full_size(big):
    A = big["A"]
    x = fields.uniform_pm1(1, A.n)
    y = fields.uniform_pm1(2, A.n)
    Ax = A.Mult(x)
    assert rel_err(Ax, O.spmv(big["rp"], big["ci"], big["a"], x)) <= 1e-14
    lhs = A.Mult(2.5 * x + y)
    assert rel_err(lhs, 2.5 * Ax + A.Mult(y)) <= 1e-13


def test_dilu_full_size(big):
    A = big["A"]
    idv, piv = O.prec_setup(O.ILU, big["rp"], big["ci"], big["a"])
    P = F.Prec(A, F.ILU_PREC)
    assert np.array_equal(P.getPivot(), piv)
    r = fields.uniform_pm1(4, A.n)
    assert rel_err(P.solve(r), O.prec_apply(O.ILU, big["rp"], big["ci"], big["a"], idv, piv, r)) <= 1e-12


def test_mixed_solve_full_size(big):
    A = big["A"]
    x = np.zeros(A.n)
    outer, inner, res = F.solve_mixed(A, big["b"], x, prec=F.DIAG_PREC, inner_bits=32, toler=1e-10)
    assert res <= 1e-10 and F.residual(A, big["b"], x) <= 1e-10
    x64 = np.zeros(A.n)
    it = F.CG(A, F.Prec(A, F.DIAG_PREC), big["b"], x64, 100000, 1e-10)
    assert it > 0 and F.residual(A, big["b"], x64) <= 1.01e-10
    # both solutions meet the same residual bound; they agree to the
    # conditioning-limited accuracy of that bound
    assert rel_err(x, x64) <= 1e-5
    # every value of this matrix is exact in BF16, so the automatic value
    # format streams BF16 values and the solve is bit for bit the FP32 one
    xa = np.zeros(A.n)
    assert F.solve_mixed(A, big["b"], xa, prec=F.DIAG_PREC, inner_bits=0,
                         toler=1e-10) == (outer, inner, res)
    assert np.array_equal(xa, x)


def test_kuhn_129_pattern_and_values(cuda):
    M = 128
    xyz, elem, code = O.mesh3d(M)
    dof, n = O.number_equations(code)
    assert n == 2048383
    rp, ci = O.node_graph(elem, 4, dof, n)
    assert rp[-1] == 30340171
    cent = xyz.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
    k = fields.lognormal_k(3, cent, 1.5, 0.1, grid=64)
    f = fields.uniform_pm1(3, code.size)
    a, b = O.assemble(3, xyz, elem, dof, code, n, rp, ci, k=k, f=f, bc=np.zeros(code.size))
    mesh = F.Mesh.kuhn(M)
    eq = F.DC3DT4(mesh)
    eq.setSolver(F.CG_SOLVER, F.ILU_PREC)
    eq.setSource(f)
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.setElementCoefficient(k)
    eq.build()
    A = eq.getMatrix()
    rp2, ci2 = A.pattern()
    assert np.array_equal(rp2, rp) and np.array_equal(ci2, ci)
    assert np.array_equal(A.values(), a) and np.array_equal(eq.getRHS(), b)


def test_plain_cg_ilu_matches_reference_at_full_size(big):
    """OFELI's own CG + ILU run to convergence on this problem (pins in
    tests/golden/p2d_2049_pins.npz): same iteration count, same solution."""
    from conftest import load_golden
    pins, info = load_golden("p2d_2049_pins")
    A = big["A"]
    x = np.zeros(A.n)
    it = F.CG(A, F.Prec(A, F.ILU_PREC), big["b"], x, 100000, info["tol"])
    assert abs(it - info["iters"]) <= 2
    assert abs(np.linalg.norm(x) / info["x_norm2"] - 1) <= 1e-12
    sample = x[::info["x_sample_stride"]]
    assert rel_err(sample, pins["x_sample"]) <= 1e-11


def kuhn_129_system(seed=1234):
    """The 3-D benchmark problem: Kuhn cube 129^3 nodes, k = exp(g) with g the
    seeded Gaussian field (sigma 1.5, correlation length 0.1, 256^3 lattice),
    f ~ U[-1, 1], u = 0 on the faces."""
    mesh = F.Mesh.kuhn(128)
    coords, elem, _, _ = mesh.arrays()
    cent = coords.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
    k = fields.lognormal_k(seed, cent, 1.5, 0.1, grid=256)
    del coords, elem, cent
    eq = F.DC3DT4(mesh)
    eq.setSource(fields.uniform_pm1(seed, mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.setElementCoefficient(k)
    eq.build()
    return mesh, eq


@pytest.mark.parametrize("prec", ["ILU", "DIAG"])
def test_plain_cg_matches_reference_kuhn_129(cuda, prec):
    """OFELI's own CG (DILU and DIAG) run to convergence on the 3-D
    benchmark problem (pins in tests/golden/p3d_129_pins.npz): iterations
    +-2 and the same solution."""
    from conftest import load_golden
    pins, info = load_golden("p3d_129_pins")
    run = info["runs"][prec]
    mesh, eq = kuhn_129_system(info["seed_f"])
    A = eq.getMatrix()
    assert A.n == info["n"] and A.nnz == info["nnz"]
    x = np.zeros(A.n)
    it = F.CG(A, F.Prec(A, F.ILU_PREC if prec == "ILU" else F.DIAG_PREC), eq.getRHS(), x, 100000,
              info["tol"])
    assert abs(it - run["iters"]) <= 2
    assert abs(np.linalg.norm(x) / run["x_norm2"] - 1) <= 1e-12
    assert rel_err(x[::run["x_sample_stride"]], pins["x_sample_" + prec]) <= 1e-11


def test_transient_steps_match_reference_1025():
    """OFELI's own first three backward-Euler DC2DT3 steps at 1025^2 with
    GMRES(30) + ILU, warm-started (pins in tests/golden/cd2d_1025_pins.npz):
    iterations +-2 per step and the same field."""
    from conftest import load_golden
    pins, info = load_golden("cd2d_1025_pins")
    nx = info["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    eq = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"])
    eq.setDirichlet(np.zeros(mesh.nn))
    its = [eq.step(prec=F.ILU_PREC, m=info["m"], max_it=2000, toler=info["tol"])
           for _ in range(info["steps"])]
    assert all(abs(a - b) <= 2 for a, b in zip(its, info["iters"])), (its, info["iters"])
    assert abs(np.linalg.norm(eq.x) / info["x_norm2"] - 1) <= 1e-12
    assert rel_err(eq.x[::info["x_sample_stride"]], pins["x_sample"]) <= 1e-12

"""The CPU oracle (oracle/ofeli_oracle.c) against the golden vectors that the
reference OFELI produced (tests/golden/make_golden.py): the restatement must
reproduce the reference bit for bit -- pattern, assembled values, RHS,
solutions and iteration counts."""
import numpy as np
import pytest

from conftest import load_golden
from ofeli_b200 import fields
from oracle import oracle as O

PREC = {"IDENT": O.IDENT, "DIAG": O.DIAG, "DILU": O.DILU, "ILU": O.ILU, "SSOR": O.SSOR}


def centroids(coords, elem, dim):
    return coords.reshape(-1, dim)[elem.reshape(-1, dim + 1)].mean(axis=1)


def test_p2d_65_assembly_bit_exact():
    g, info = load_golden("p2d_65")
    xy, elem, code = O.mesh2d(64, 64)
    dof, n = O.number_equations(code)
    assert n == info["n"] == 3969
    rp, ci = O.node_graph(elem, 3, dof, n)
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert rp[-1] == info["nnz"] == 27281
    f = fields.uniform_pm1(1234, code.size)
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    assert np.array_equal(a, g["a"]) and np.array_equal(b, g["b"])


@pytest.mark.parametrize("key", ["CG_IDENT", "CG_DIAG", "CG_DILU", "CG_SSOR", "GMRES30_ILU",
                                 "GMRES30_DIAG", "GMRES10_SSOR"])
def test_p2d_65_solvers_bit_exact(key):
    g, info = load_golden("p2d_65")
    rp, ci, a, b = (g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64), g["a"], g["b"])
    solver, prec = key.split("_")
    if solver == "CG":
        x, it = O.cg(rp, ci, a, b, PREC[prec], 20000, 1e-10)
    else:
        x, it = O.gmres(rp, ci, a, b, PREC[prec], int(solver[5:]), 20000, 1e-10)
    assert it == info["runs"][key]["iters"]
    assert np.array_equal(x, g["x_" + key])


def test_cfg1_iteration_pins():
    # CG + DIAG on the 65x65 Poisson problem and the D-ILU / SSOR variants
    _, info = load_golden("p2d_65")
    runs = info["runs"]
    assert runs["CG_DIAG"]["iters"] == runs["CG_IDENT"]["iters"]  # constant diagonal
    assert runs["CG_DILU"]["iters"] < runs["CG_SSOR"]["iters"] < runs["CG_DIAG"]["iters"]


def test_p2d_jitter_bit_exact():
    g, info = load_golden("p2d_jitter_25")
    nx = info["nx"]
    xy, elem, code = O.mesh2d(nx, nx)
    xyj = fields.jitter_2d(5, xy, code, nx, nx)
    k = fields.lognormal_k(5, centroids(xyj, elem, 2), 1.0, 0.1, grid=128)
    f = fields.uniform_pm1(5, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    a, b = O.assemble(2, xyj, elem, dof, code, n, rp, ci, k=k, f=f, bc=np.zeros(code.size))
    assert np.array_equal(a, g["a"]) and np.array_equal(b, g["b"])
    x, it = O.cg(rp, ci, a, b, O.ILU, 20000, 1e-10)
    assert it == info["iters"] and np.array_equal(x, g["x"])
    assert np.array_equal(O.insert_bc(code, x), g["u"])


def test_p2d_ragged_dirichlet_lift_bit_exact():
    g, info = load_golden("p2d_ragged")
    xy, elem, code = O.mesh2d(info["nx"], info["ny"], codes=tuple(info["codes"]))
    P = xy.reshape(-1, 2)
    bc = 1.0 + P[:, 0] + 2.0 * P[:, 1]
    f = fields.uniform_pm1(9, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=bc)
    assert np.array_equal(a, g["a"]) and np.array_equal(b, g["b"])
    x, it = O.cg(rp, ci, a, b, O.DIAG, 20000, 1e-10)
    assert it == info["iters"] and np.array_equal(x, g["x"])
    assert np.array_equal(O.insert_bc(code, x, bc), g["u"])


def test_p3d_kuhn_bit_exact():
    g, info = load_golden("p3d_kuhn_9")
    xyz, elem, code = O.mesh3d(info["M"])
    k = fields.lognormal_k(7, centroids(xyz, elem, 3), 1.5, 0.1, grid=32)
    f = fields.uniform_pm1(99, code.size)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 4, dof, n)
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    a, b = O.assemble(3, xyz, elem, dof, code, n, rp, ci, k=k, f=f, bc=np.zeros(code.size))
    assert np.array_equal(a, g["a"]) and np.array_equal(b, g["b"])
    for prec in ("ILU", "DIAG"):
        x, it = O.cg(rp, ci, a, b, PREC[prec], 20000, 1e-10)
        assert it == info["runs"][prec]["iters"] and np.array_equal(x, g["x_" + prec])


def test_cd2d_bit_exact():
    g, info = load_golden("cd2d_17")
    nx, dt, eps = info["nx"], info["dt"], info["eps"]
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    x = np.zeros(n)
    its = []
    for s in range(info["steps"]):
        a, b = O.assemble_cd2d(xy, elem, dof, code, n, rp, ci, eps, v, dt, u, bc=np.zeros(code.size))
        if s == 0:
            assert np.array_equal(a, g["a0"]) and np.array_equal(b, g["b0"])
        x, it = O.gmres(rp, ci, a, b, O.ILU, info["m"], 2000, info["tol"], x0=x)
        its.append(it)
        u = O.insert_bc(code, x)
    assert its == list(g["iters"])
    assert np.array_equal(u, g["u"])


def test_dilu_is_not_ilu0():
    # OFELI's ILU is diagonal ILU: only the pivots change, the off-diagonal
    # factors are A's own entries, so M = (D+L) D^{-1} (D+U) with modified D
    g, _ = load_golden("p2d_65")
    rp, ci, a = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64), g["a"]
    idv, piv = O.prec_setup(O.ILU, rp, ci, a)
    n = rp.size - 1
    dense = np.zeros((n, n))
    for i in range(n):
        dense[i, ci[rp[i]:rp[i + 1]] - 1] = a[rp[i]:rp[i + 1]]
    D = np.diag(1.0 / piv)
    L = np.tril(dense, -1)
    U = np.triu(dense, 1)
    M = (D + L) @ np.diag(piv) @ (D + U)
    r = fields.uniform_pm1(3, n)
    z = O.prec_apply(O.ILU, rp, ci, a, idv, piv, r)
    assert np.abs(M @ z - r).max() <= 1e-12 * np.abs(r).max()


@pytest.mark.parametrize("prec", ["DIAG", "ILU"])
def test_bicgstab_p2d_bit_exact(prec):
    """OFELI's BiCGStab (include/solvers/BiCGStab.h) on the 65x65 system."""
    g, _ = load_golden("p2d_65")
    z, info = load_golden("bicgstab")
    rp, ci, a, b = (g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64), g["a"], g["b"])
    x, it = O.bicgstab(rp, ci, a, b, PREC[prec], 20000, 1e-10)
    assert it == info["runs"]["p2d_" + prec]["iters"]
    assert np.array_equal(x, z["x_p2d_" + prec])


def test_bicgstab_cd2d_bit_exact():
    """Five backward-Euler DC2DT3 steps solved by BiCGStab + ILU with the
    previous step as the initial guess, as OFELI runs them."""
    z, info = load_golden("bicgstab")
    c = info["cd2d"]
    nx, dt, eps = c["nx"], c["dt"], c["eps"]
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    x = np.zeros(n)
    its = []
    for s in range(c["steps"]):
        a, b = O.assemble_cd2d(xy, elem, dof, code, n, rp, ci, eps, v, dt, u, bc=np.zeros(code.size))
        x, it = O.bicgstab(rp, ci, a, b, O.ILU, 2000, 1e-10, x0=x)
        its.append(it)
        u = O.insert_bc(code, x)
    assert its == list(z["cd2d_iters"])
    assert np.array_equal(u, z["cd2d_u"])


@pytest.mark.parametrize("name", ["FE", "CN"])
def test_cd2d_schemes_bit_exact(name):
    """OFELI's forward Euler and Crank-Nicolson steps of DC2DT3
    (Equa_Therm::build) restated: first-step matrix and RHS, iteration
    counts and the final field equal the reference's."""
    g, info = load_golden("cd2d_schemes")
    nx, dt, eps = info["nx"], info["dt"], info["eps"]
    scheme = info["schemes"][name]
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    x = np.zeros(n)
    its = []
    for s in range(info["steps"]):
        a, b = O.assemble_cd2d(xy, elem, dof, code, n, rp, ci, eps, v, dt, u,
                               bc=np.zeros(code.size), scheme=scheme)
        if s == 0:
            assert np.array_equal(a, g[name + "_a0"]) and np.array_equal(b, g[name + "_b0"])
        x, it = O.gmres(rp, ci, a, b, O.ILU, info["m"], 2000, info["tol"], x0=x)
        its.append(it)
        u = O.insert_bc(code, x)
    assert its == list(g[name + "_iters"])
    assert np.array_equal(u, g[name + "_u"])


@pytest.mark.parametrize("name", ["FE", "BE", "CN"])
def test_timestepping_bit_exact(name):
    """OFELI's TimeStepping class driving DC2DT3 (src/solvers/TimeStepping.cpp)
    restated from the Equa_Therm systems: forward Euler is x = b / diag(A),
    the implicit schemes the equation's LinearSolver (GMRES restarting every
    n/5 steps, warm start); forward Euler and Crank-Nicolson make two
    sub-steps per call (the scheme tests of TimeStepping::set).  Every
    step's field equals the reference's bit for bit."""
    g, info = load_golden("ts2d_17")
    nx, dt, eps = info["nx"], info["dt"], info["eps"]
    scheme = {"FE": 1, "BE": 2, "CN": 3}[name]
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    dpos = np.array([rp[r] + np.nonzero(ci[rp[r]:rp[r + 1]] - 1 == r)[0][0] for r in range(n)])
    x = np.zeros(n)
    substeps = 1 if name == "BE" else 2
    for s in range(info["steps"]):
        for _ in range(substeps):
            a, b = O.assemble_cd2d(xy, elem, dof, code, n, rp, ci, eps, v, dt, u,
                                   bc=np.zeros(code.size), scheme=scheme)
            if name == "FE":
                x = b / a[dpos]
            else:
                x, it = O.gmres(rp.astype(np.int64), ci.astype(np.int64), a, b, O.ILU, n // 5,
                                2000, info["tol"], x0=x)
                assert it > 0
            u = O.insert_bc(code, x)
        assert np.array_equal(u, g[name + "_u_steps"][s])

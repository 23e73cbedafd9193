"""Parity of the CUDA path (through the C ABI) with the reference OFELI's
golden vectors (tests/golden, produced by OFELI itself) and with the oracle.

Bars: CSR pattern bit-exact; assembled values and RHS bit-exact (each entry
receives its element contributions in the reference's element order, with
the same element arithmetic and no fused multiply-adds); solutions within
1e-12 relative (max-norm, relative to the reference's max entry); iteration
counts within +-2 of the reference's (they come out equal); D-ILU pivots
bit-exact (the factorisation keeps the reference's operation order)."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from ofeli_b200 import fields
from ofeli_b200 import ofeli as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SOL_TOL = 1e-12
IT_TOL = 2
PRECS = {"IDENT": F.IDENT_PREC, "DIAG": F.DIAG_PREC, "DILU": F.DILU_PREC, "ILU": F.ILU_PREC,
         "SSOR": F.SSOR_PREC}


def centroids(coords, elem, dim):
    return coords.reshape(-1, dim)[elem.reshape(-1, dim + 1)].mean(axis=1)


@pytest.fixture(scope="module")
def p2d65(cuda):
    g, info = load_golden("p2d_65")
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, 64, 64, 1, 1, 1, 1)
    eq = F.Laplace2DT3(mesh)
    eq.setSolver(F.CG_SOLVER, F.DIAG_PREC)
    eq.setSource(fields.uniform_pm1(1234, mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.build()
    return g, info, mesh, eq


def test_mesh_matches_reference_generator(p2d65):
    _, _, mesh, _ = p2d65
    xy, elem, code = O.mesh2d(64, 64)
    c2, e2, code2, dof2 = mesh.arrays()
    assert np.array_equal(c2, xy)  # coordinates accumulated as the reference does
    assert np.array_equal(e2, elem) and np.array_equal(code2, code)
    dof, n = O.number_equations(code)
    assert np.array_equal(dof2, dof) and mesh.neq == n == 3969


def test_pattern_bit_exact(p2d65):
    g, info, _, eq = p2d65
    rp, ci = eq.getMatrix().pattern()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert eq.getMatrix().nnz == info["nnz"] == 27281


def test_assembly_matches_reference(p2d65):
    g, _, _, eq = p2d65
    assert np.array_equal(eq.getMatrix().values(), g["a"])
    assert np.array_equal(eq.getRHS(), g["b"])


@pytest.mark.parametrize("key", ["CG_IDENT", "CG_DIAG", "CG_DILU", "CG_SSOR"])
def test_cg_matches_reference(p2d65, key):
    g, info, _, eq = p2d65
    prec = key.split("_")[1]
    A = eq.getMatrix()
    x = np.zeros(A.n)
    it = F.CG(A, F.Prec(A, PRECS[prec]), g["b"], x, 20000, 1e-10)
    assert abs(it - info["runs"][key]["iters"]) <= IT_TOL
    assert rel_err(x, g["x_" + key]) <= SOL_TOL


def test_ilu_equals_dilu(p2d65):
    g, info, _, eq = p2d65
    A = eq.getMatrix()
    x1, x2 = np.zeros(A.n), np.zeros(A.n)
    i1 = F.CG(A, F.Prec(A, F.ILU_PREC), g["b"], x1, 20000, 1e-10)
    i2 = F.CG(A, F.Prec(A, F.DILU_PREC), g["b"], x2, 20000, 1e-10)
    assert i1 == i2 == info["runs"]["CG_DILU"]["iters"]
    assert np.array_equal(x1, x2)


@pytest.mark.parametrize("key", ["GMRES30_ILU", "GMRES30_DIAG", "GMRES10_SSOR"])
def test_gmres_matches_reference(p2d65, key):
    g, info, _, eq = p2d65
    solver, prec = key.split("_")
    A = eq.getMatrix()
    x = np.zeros(A.n)
    it = F.GMRes(A, F.Prec(A, PRECS[prec]), g["b"], x, int(solver[5:]), 20000, 1e-10)
    assert abs(it - info["runs"][key]["iters"]) <= IT_TOL
    assert rel_err(x, g["x_" + key]) <= SOL_TOL


def test_cg_residual_history_matches_oracle(p2d65):
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    _, it0, h0 = O.cg(rp, ci, g["a"], g["b"], O.ILU, 200, 1e-10, history=True)
    x = np.zeros(A.n)
    it, h = F.CG(A, F.Prec(A, F.ILU_PREC), g["b"], x, 200, 1e-10, history=True)
    assert it == it0
    assert np.abs(h[1:it + 1] / h0[1:it0 + 1] - 1).max() < 1e-9


def test_pivots_bit_exact(p2d65):
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    for pt in (O.DIAG, O.DILU, O.SSOR):
        _, piv = O.prec_setup(pt, rp, ci, g["a"])
        assert np.array_equal(F.Prec(A, pt).getPivot(), piv)


def test_prec_apply_matches_oracle(p2d65):
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    r = fields.uniform_pm1(77, A.n)
    for pt in (O.DIAG, O.DILU, O.SSOR):
        idv, piv = O.prec_setup(pt, rp, ci, g["a"])
        z0 = O.prec_apply(pt, rp, ci, g["a"], idv, piv, r)
        P = F.Prec(A, pt)
        z1 = P.solve(r)
        z2 = P.solve(r)  # buffers are reusable
        assert rel_err(z1, z0) <= 1e-13 and np.array_equal(z1, z2)


def test_spmv_matches_oracle(p2d65):
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    x = fields.uniform_pm1(5, A.n)
    y0 = O.spmv(rp, ci, g["a"], x)
    assert rel_err(A.Mult(x), y0) <= 1e-14
    y = np.ones(A.n)
    assert rel_err(A.MultAdd(x, y), y0 + 1.0) <= 1e-14


def test_jittered_variable_k():
    g, info = load_golden("p2d_jitter_25")
    nx = info["nx"]
    xy, elem, code = O.mesh2d(nx, nx)
    xyj = fields.jitter_2d(5, xy, code, nx, nx)
    k = fields.lognormal_k(5, centroids(xyj, elem, 2), 1.0, 0.1, grid=128)
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    mesh.setCoords(xyj)
    eq = F.Laplace2DT3(mesh)
    eq.setSolver(F.CG_SOLVER, F.ILU_PREC)
    eq.setSource(fields.uniform_pm1(5, mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.setElementCoefficient(k)
    eq.getLinearSolver().setTolerance(1e-10)
    eq.getLinearSolver().setMaxIter(20000)
    ret = eq.run()
    A = eq.getMatrix()
    rp, ci = A.pattern()
    assert ret == 0
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert np.array_equal(A.values(), g["a"]) and np.array_equal(eq.getRHS(), g["b"])
    assert rel_err(eq.x, g["x"]) <= SOL_TOL and rel_err(eq.u, g["u"]) <= SOL_TOL
    assert abs(eq.getLinearSolver().getNbIter() - info["iters"]) <= IT_TOL


def test_ragged_mesh_with_imposed_values():
    g, info = load_golden("p2d_ragged")
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, info["nx"], info["ny"], *info["codes"])
    xy = mesh.arrays()[0].reshape(-1, 2)
    bc = 1.0 + xy[:, 0] + 2.0 * xy[:, 1]
    eq = F.Laplace2DT3(mesh)
    eq.setSolver(F.CG_SOLVER, F.DIAG_PREC)
    eq.getLinearSolver().setTolerance(1e-10)
    eq.getLinearSolver().setMaxIter(20000)
    eq.setSource(fields.uniform_pm1(9, mesh.nn))
    eq.setDirichlet(bc)
    eq.run()
    A = eq.getMatrix()
    rp, ci = A.pattern()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert np.array_equal(A.values(), g["a"]) and np.array_equal(eq.getRHS(), g["b"])
    assert rel_err(eq.u, g["u"]) <= SOL_TOL
    assert abs(eq.getLinearSolver().getNbIter() - info["iters"]) <= IT_TOL


def test_kuhn_3d_variable_k():
    g, info = load_golden("p3d_kuhn_9")
    M = info["M"]
    xyz, elem, code = O.mesh3d(M)
    k = fields.lognormal_k(7, centroids(xyz, elem, 3), 1.5, 0.1, grid=32)
    mesh = F.Mesh.kuhn(M)
    c2, e2, code2, _ = mesh.arrays()
    assert np.array_equal(c2, xyz) and np.array_equal(e2, elem) and np.array_equal(code2, code)
    eq = F.DC3DT4(mesh)
    eq.setSolver(F.CG_SOLVER, F.ILU_PREC)
    eq.setSource(fields.uniform_pm1(99, mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.setElementCoefficient(k)
    eq.build()
    A = eq.getMatrix()
    rp, ci = A.pattern()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert np.array_equal(A.values(), g["a"]) and np.array_equal(eq.getRHS(), g["b"])
    for prec in ("ILU", "DIAG"):
        x = np.zeros(A.n)
        it = F.CG(A, F.Prec(A, PRECS[prec]), eq.getRHS(), x, 20000, 1e-10)
        assert abs(it - info["runs"][prec]["iters"]) <= IT_TOL
        assert rel_err(x, g["x_" + prec]) <= SOL_TOL


def test_transient_convection_diffusion():
    g, info = load_golden("cd2d_17")
    nx = info["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    eq = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"])
    eq.setDirichlet(np.zeros(mesh.nn))
    A, b = eq.build()
    rp, ci = A.pattern()
    assert np.array_equal(rp, g["row_ptr"]) and np.array_equal(ci, g["col_ind"])
    assert np.array_equal(A.values(), g["a0"]) and np.array_equal(b, g["b0"])
    eq2 = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"])
    eq2.setDirichlet(np.zeros(mesh.nn))
    its = [eq2.step(prec=F.ILU_PREC, m=info["m"], max_it=2000, toler=info["tol"])
           for _ in range(info["steps"])]
    assert all(abs(a - b) <= IT_TOL for a, b in zip(its, g["iters"]))
    assert rel_err(eq2.u, g["u"]) <= SOL_TOL


def test_linear_solver_gmres_uses_ofeli_restart(p2d65):
    # LinearSolver::solve with GMRES_SOLVER restarts every n/5 iterations
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    x0, it0 = O.gmres(rp, ci, g["a"], g["b"], O.ILU, A.n // 5, 1000, 1e-8)
    x = np.zeros(A.n)
    ls = F.LinearSolver(A, g["b"], x)
    ls.setTolerance(1e-8)
    ret = ls.solve(F.GMRES_SOLVER, F.ILU_PREC)
    assert ret == 0 and abs(ls.getNbIter() - it0) <= IT_TOL
    assert rel_err(x, x0) <= 1e-11


@pytest.mark.parametrize("bits,mode", [(32, 0), (16, 0), (32, 1)])
def test_mixed_precision_reaches_fp64_accuracy(p2d65, bits, mode):
    """FP64 true residual <= 1e-10; the error against the FP64 solution of
    the same system (oracle, residual 1e-13) is reported in the assert."""
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    xref, _ = O.cg(rp, ci, g["a"], g["b"], O.DIAG, 20000, 1e-13)
    x = np.zeros(A.n)
    outer, inner, res = F.solve_mixed(A, g["b"], x, prec=F.DIAG_PREC, inner_bits=bits,
                                      toler=1e-10, mode=mode)
    assert res <= 1e-10 and F.residual(A, g["b"], x) <= 1e-10
    err = rel_err(x, xref)
    assert err <= 1e-7, "error vs FP64 solution %.2e" % err


@pytest.mark.parametrize("permute", [False, True])
def test_mixed_precision_column_offset_formats(cuda, permute):
    """The FP32 SpMV streams 16-bit column offsets when every |column - row|
    fits in 16 bits and absolute int32 columns otherwise.  A 201x201 Poisson
    matrix (n = 39 601) in natural order takes the first form; the same
    matrix under a random symmetric permutation (offsets up to n) the second.
    Both reach the FP64 target and the oracle's FP64 solution."""
    xy, elem, code = O.mesh2d(200, 200)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    f = fields.uniform_pm1(41, code.size)
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    if permute:
        perm = np.random.default_rng(0).permutation(n)  # new index of old row i
        inv = np.argsort(perm)
        rows = np.repeat(np.arange(n), np.diff(rp))
        nr, nc = perm[rows], perm[ci - 1]
        order = np.lexsort((nc, nr))
        a, nr, nc = a[order], nr[order], nc[order]
        rp = np.concatenate([[0], np.cumsum(np.bincount(nr, minlength=n))]).astype(np.int64)
        ci = (nc + 1).astype(np.int64)
        b = b[inv]
    xref, _ = O.cg(rp, ci, a, b, O.DIAG, 40000, 1e-13)
    A = F.SpMatrix(rp, ci, a)
    x = np.zeros(n)
    outer, inner, res = F.solve_mixed(A, b, x, prec=F.DIAG_PREC, toler=1e-10)
    assert res <= 1e-10 and F.residual(A, b, x) <= 1e-10
    assert rel_err(x, xref) <= 1e-6


def solve_counting_formats(A, b, bits):
    """solve_mixed with the given inner_bits; returns (x, outer, inner,
    residual, SpMV launches with FP32 values, with BF16 values)."""
    from ofeli_b200 import capi
    x = np.zeros(A.n)
    capi.profile_enable(1)
    try:
        outer, inner, res = F.solve_mixed(A, b, x, prec=F.DIAG_PREC, inner_bits=bits,
                                          toler=1e-10)
        n32, n16 = capi.profile_read("spmv32")[0], capi.profile_read("spmv16")[0]
    finally:
        capi.profile_enable(0)
    return x, outer, inner, res, n32, n16


@pytest.mark.parametrize("exact", [True, False])
def test_mixed_precision_automatic_value_format(cuda, exact, p2d65):
    """inner_bits 0 streams BF16 matrix values only when every value of A
    comes back unchanged from BF16.  The 65x65 Laplacian (values -1, 0, 4)
    takes that path, and the solve is bit for bit the one with FP32 values;
    the same matrix scaled symmetrically, D A D with D = diag(1 .. 1.3), has
    values that BF16 does not hold and takes the FP32 path, bit for bit the
    inner_bits 32 solve."""
    import torch
    g, _, _, _ = p2d65
    a = g["a"]
    if not exact:
        rp = g["row_ptr"].astype(np.int64)
        rows = np.repeat(np.arange(rp.size - 1), np.diff(rp))
        d = 1.0 + 0.3 * np.random.default_rng(5).random(rp.size - 1)
        a = a * d[rows] * d[g["col_ind"].astype(np.int64) - 1]
    lossless = np.array_equal(torch.from_numpy(a).to(torch.bfloat16).to(torch.float64).numpy(), a)
    assert lossless == exact
    A = F.SpMatrix(g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64), a)
    auto = solve_counting_formats(A, g["b"], 0)
    fp32 = solve_counting_formats(A, g["b"], 32)
    assert auto[3] <= 1e-10 and F.residual(A, g["b"], auto[0]) <= 1e-10
    assert (auto[4] == 0 and auto[5] > 0) if exact else (auto[4] > 0 and auto[5] == 0)
    assert np.array_equal(auto[0], fp32[0]) and auto[1:4] == fp32[1:4]
    if exact:
        bf16 = solve_counting_formats(A, g["b"], 16)
        assert np.array_equal(auto[0], bf16[0]) and auto[1:4] == bf16[1:4]


def test_mixed_precision_uniform_slices_bit_identical(cuda):
    """Slices whose 32 rows share their column offsets (about 94 % of the
    entries of the 1025x1025 Laplacian in natural order) are streamed with
    one offset per slice position and vector gathers.  The same matrix with
    an explicit zero added to every 16th row (column row + 2) has no uniform
    slice and takes the per-entry path; adding exact zeros changes no sum,
    so both solves are bit for bit the same.  The profile's bytes per SpMV
    show which format each one streamed."""
    from ofeli_b200 import capi
    xy, elem, code = O.mesh2d(1024, 1024)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    f = fields.uniform_pm1(17, code.size)
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    rows = np.arange(0, n - 2, 16)
    cols = rows + 3  # 1-based column row + 2, absent from the 7-point pattern
    pos = np.array([rp[r] + np.count_nonzero(ci[rp[r]:rp[r + 1]] < c) for r, c in zip(rows, cols)])
    cnt = np.zeros(n, np.int64)
    cnt[rows] = 1
    rp2 = rp + np.concatenate([[0], np.cumsum(cnt)])
    ci2, a2 = np.insert(ci, pos, cols), np.insert(a, pos, 0.0)
    out = []
    for r_, c_, v_ in ((rp, ci, a), (rp2, ci2, a2)):
        A = F.SpMatrix(r_.astype(np.int64), c_.astype(np.int64), v_)
        x = np.zeros(n)
        capi.profile_enable(1)
        try:
            res = F.solve_mixed(A, b, x, prec=F.DIAG_PREC, inner_bits=0, toler=1e-10)
            launches, _, nbytes = capi.profile_read("spmv16")
        finally:
            capi.profile_enable(0)
        out.append((res, x, nbytes / launches, A.nnz))
    (res1, x1, b1, nnz1), (res2, x2, b2, nnz2) = out
    assert res1[2] <= 1e-10 and res1 == res2 and np.array_equal(x1, x2)
    assert nnz2 == nnz1 + rows.size
    assert b2 == 4.0 * nnz2 + 12.0 * n + 4.0  # BF16 value + 16-bit offset per entry
    # BF16 values, and index bytes of at most 0.2 per entry: at least 90 % of
    # the entries take their offset from the slice table
    assert b1 <= 2.2 * nnz1 + 12.0 * n + 4.0


@pytest.mark.parametrize("prec", ["DIAG", "ILU"])
def test_bicgstab_matches_reference(cuda, prec):
    """BiCGStab on the 65x65 system against OFELI's own run (golden
    bicgstab.npz): iteration count within the band, same solution."""
    g, _ = load_golden("p2d_65")
    z, info = load_golden("bicgstab")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    x = np.zeros(A.n)
    it = F.BiCGStab(A, F.Prec(A, PRECS[prec]), g["b"], x, 20000, 1e-10)
    assert it > 0 and abs(it - info["runs"]["p2d_" + prec]["iters"]) <= IT_TOL
    # BiCGStab amplifies the different summation order of the parallel dot
    # products more than CG does: both solutions have residual <= 1e-10 and
    # agree to 1e-8 (the conditioning bound here is ~2e-7)
    assert rel_err(x, z["x_p2d_" + prec]) <= 1e-8
    ls = F.LinearSolver(A, g["b"], np.zeros(A.n))
    ls.setTolerance(1e-10)
    ls.setMaxIter(20000)
    assert ls.solve(F.BICG_STAB_SOLVER, PRECS[prec]) == 0
    assert abs(ls.getNbIter() - it) <= IT_TOL


def test_bicgstab_transient_steps_match_reference(cuda):
    """Five DC2DT3 backward-Euler steps with BiCGStab + ILU and warm starts,
    as OFELI runs them (golden bicgstab.npz)."""
    z, info = load_golden("bicgstab")
    c = info["cd2d"]
    nx = c["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    eq = F.DC2DT3(mesh, u0, v, c["eps"], c["dt"])
    eq.setDirichlet(np.zeros(mesh.nn))
    its = [eq.step(prec=F.ILU_PREC, max_it=2000, toler=1e-10, solver=F.BICG_STAB_SOLVER)
           for _ in range(c["steps"])]
    assert all(abs(a - b) <= IT_TOL for a, b in zip(its, z["cd2d_iters"]))
    assert rel_err(eq.u, z["cd2d_u"]) <= 1e-8


def test_bicgstab_edges(cuda):
    g, _ = load_golden("p2d_65")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    x = np.zeros(A.n)
    assert F.BiCGStab(A, F.Prec(A, F.DIAG_PREC), np.zeros(A.n), x, 100, 1e-10) == 0
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    for pt in (O.IDENT, O.DIAG, O.SSOR):
        x = np.zeros(A.n)
        it = F.BiCGStab(A, F.Prec(A, pt), g["b"], x, 5, 1e-10)
        xo, ito = O.bicgstab(rp, ci, g["a"], g["b"], pt, 5, 1e-10)
        assert it == ito == -6
        assert rel_err(x, xo) <= 1e-10


def test_tmult_matches_oracle(p2d65):
    """SpMatrix::TMult (y += A^T x) against the oracle's row-ordered loop, bit
    for bit, on the assembled 65^2 matrix and on a non-symmetric pattern
    whose rows list their columns out of order."""
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = A.pattern()
    rng = np.random.default_rng(8)
    x, y0 = rng.standard_normal(A.n), rng.standard_normal(A.n)
    y = A.TMult(x, y0.copy())
    assert np.array_equal(y, O.spmv_transpose_add(rp, ci, A.values(), x, y0))
    n = 300
    rows = [rng.choice(n, size=rng.integers(1, 9), replace=False) + 1 for _ in range(n)]
    rp2 = np.concatenate([[0], np.cumsum([r.size for r in rows])]).astype(np.int64)
    ci2 = np.concatenate(rows).astype(np.int64)
    a2 = rng.standard_normal(ci2.size)
    B = F.SpMatrix(rp2, ci2, a2)
    x2, y2 = rng.standard_normal(n), rng.standard_normal(n)
    assert np.array_equal(B.TMult(x2, y2.copy()), O.spmv_transpose_add(rp2, ci2, a2, x2, y2))


def test_matrix_set_add_in_order(p2d65):
    """SpMatrix::set / add batches (repeated pairs included) applied in
    order, as the oracle's loop does; a pair outside the pattern raises
    after the pairs before it."""
    g, _, _, eq = p2d65
    A = eq.getMatrix()
    rp, ci = A.pattern()
    rng = np.random.default_rng(9)
    rows = rng.integers(1, A.n + 1, 500)
    ks = rp[rows - 1] + rng.integers(0, 10 ** 6, 500) % (rp[rows] - rp[rows - 1])
    cols = ci[ks]
    rows, cols = np.concatenate([rows, rows[:50]]), np.concatenate([cols, cols[:50]])
    vals = rng.standard_normal(rows.size)
    a0 = A.values()
    for set_values in (False, True):
        A.set_values(a0)
        A.edit(rows, cols, vals, set_values)
        want, bad = O.matrix_edit(rp, ci, a0, rows, cols, vals, set_values)
        assert bad == -1 and np.array_equal(A.values(), want)
    A.set_values(a0)
    A.add(1, 1, 0.5)
    assert A.values()[rp[0]] == a0[rp[0]] + 0.5
    bad_rows = np.array([1, 1, 2])
    bad_cols = np.array([1, A.n, 2])   # (1, n) is outside the pattern
    A.set_values(a0)
    with pytest.raises(F.OFELIException):
        A.edit(bad_rows, bad_cols, np.ones(3), False)
    want, bad = O.matrix_edit(rp, ci, a0, bad_rows, bad_cols, np.ones(3), False)
    assert bad == 1 and np.array_equal(A.values(), want)
    A.set_values(a0)


@pytest.mark.parametrize("name", ["FE", "CN"])
def test_transient_time_schemes(name):
    """Forward Euler and Crank-Nicolson DC2DT3 steps (Equa_Therm::build):
    first-step matrix and RHS bit-exact, iterations +-2, field 1e-12."""
    g, info = load_golden("cd2d_schemes")
    nx = info["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    scheme = {"FE": F.FORWARD_EULER, "CN": F.CRANK_NICOLSON}[name]
    eq = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"], scheme)
    eq.setDirichlet(np.zeros(mesh.nn))
    A, b = eq.build()
    assert np.array_equal(A.values(), g[name + "_a0"]) and np.array_equal(b, g[name + "_b0"])
    its = [eq.step(prec=F.ILU_PREC, m=info["m"], max_it=2000, toler=info["tol"])
           for _ in range(info["steps"])]
    assert all(abs(a - b) <= IT_TOL for a, b in zip(its, g[name + "_iters"]))
    assert rel_err(eq.u, g[name + "_u"]) <= SOL_TOL

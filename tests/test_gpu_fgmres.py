"""The mixed-precision flexible GMRES (ofg_fgmres_mixed, the chosen form of
the transient convection-diffusion steps) against OFELI's own FP64 GMRES(30)
+ ILU steps (tests/golden/cd2d_17.npz, produced by the reference) and the
oracle's FP64 solves: every result is converged on the FP64 true residual
(<= 1e-10) and its error against the FP64 solution is bounded."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from ofeli_b200 import fields
from ofeli_b200 import learned as LN
from ofeli_b200 import ofeli as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def cd2d_start(info):
    nx = info["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    eq = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"])
    eq.setDirichlet(np.zeros(mesh.nn))
    return eq


@pytest.mark.parametrize("m", [30, 4, 1])
def test_fgmres_mixed_steps_match_reference(cuda, m):
    """Five backward-Euler steps of OFELI's transient problem (17^2): each
    step's FP64 true residual <= 1e-10, and the field agrees with OFELI's
    own GMRES(30) + ILU steps to 1e-8 (both solves stop at 1e-10, by
    different residual measures)."""
    g, info = load_golden("cd2d_17")
    eq = cd2d_start(info)
    for _ in range(info["steps"]):
        cycles, steps, res, fell_back = eq.step_mixed(F.DIAG_PREC, m=m, toler=TOL)
        assert res <= TOL and not fell_back and steps >= 1
        A, b = eq._A, eq._b
        assert F.residual(A, b, eq.x) <= 1.01 * TOL
    assert rel_err(eq.u, g["u"]) <= 1e-8


def test_fgmres_mixed_against_fp64_gmres_oracle(cuda):
    """One step from the golden first-step system: against the oracle's FP64
    GMRES(30) + DIAG solved to 1e-13."""
    g, info = load_golden("cd2d_17")
    rp, ci = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64)
    x64, it = O.gmres(rp, ci, g["a0"], g["b0"], O.DIAG, 30, 2000, 1e-13)
    assert it > 0
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a0"])
    for prec in (F.DIAG_PREC, F.IDENT_PREC):
        x = np.zeros(A.n)
        cycles, steps, res, _ = F.fgmres_mixed(F.Prec(A, prec), g["b0"], x, m=30, toler=TOL)
        assert res <= TOL and F.residual(A, g["b0"], x) <= 1.01 * TOL
        assert rel_err(x, x64) <= 1e-8


def test_fgmres_mixed_spd_and_value_formats(cuda):
    """On the 65^2 Poisson system (SPD, every value exact in BF16): the FP64
    target is met, the solution agrees with OFELI's CG + ILU solution to
    the conditioning-limited bound, and the automatic value format (BF16,
    lossless here) reproduces the FP32 run bit for bit."""
    g, info = load_golden("p2d_65")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    P = F.Prec(A, F.DIAG_PREC)
    x32 = np.zeros(A.n)
    r32 = F.fgmres_mixed(P, g["b"], x32, m=30, inner_bits=32, toler=TOL)
    assert r32[2] <= TOL
    assert rel_err(x32, g["x_CG_DILU"]) <= 1e-7
    x0 = np.zeros(A.n)
    assert F.fgmres_mixed(P, g["b"], x0, m=30, inner_bits=0, toler=TOL) == r32
    assert np.array_equal(x0, x32)


def test_fgmres_mixed_edges(cuda):
    g, info = load_golden("cd2d_17")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a0"])
    P = F.Prec(A, F.DIAG_PREC)
    # zero right-hand side from a zero guess: converged at once, x stays 0
    x = np.zeros(A.n)
    assert F.fgmres_mixed(P, np.zeros(A.n), x, toler=TOL)[:2] == (0, 0)
    assert not x.any()
    # warm start at the solution: no cycle
    x = np.zeros(A.n)
    F.fgmres_mixed(P, g["b0"], x, toler=TOL)
    assert F.fgmres_mixed(P, g["b0"], x, toler=1e-6)[:2] == (0, 0)
    # restart length limits
    for m in (0, 65):
        with pytest.raises(F.OFELIException):
            F.fgmres_mixed(P, g["b0"], np.zeros(A.n), m=m)
    with pytest.raises(F.OFELIException):
        F.fgmres_mixed(F.Prec(A, F.ILU_PREC), g["b0"], np.zeros(A.n))
    # the cycle cap: not converged, residual reported
    x = np.zeros(A.n)
    cycles, steps, res, _ = F.fgmres_mixed(P, g["b0"], x, m=2, max_outer=1, toler=TOL)
    assert cycles == 1 and steps == 2 and res > TOL
    # a NaN in the right-hand side: never converged, never a fault
    b = g["b0"].copy()
    b[5] = np.nan
    cycles, steps, res, _ = F.fgmres_mixed(P, b, np.zeros(A.n), m=4, max_outer=3, toler=TOL)
    assert not res <= TOL


@pytest.mark.parametrize("inner_bits", [32, 16, 0])
def test_fgmres_mixed_zero_diagonal_raises(cuda, inner_bits):
    """A zero diagonal entry that appears after the preconditioner was made
    is an error for every value format (with FP32 values the flag travels in
    the solver state and is read with the first state read), and the matrix
    solves again once the entry is restored."""
    g, info = load_golden("cd2d_17")
    rp, ci = g["row_ptr"], g["col_ind"]
    A = F.SpMatrix(rp, ci, g["a0"])
    P = F.Prec(A, F.DIAG_PREC)
    a = np.array(g["a0"], dtype=np.float64)
    row = 40
    # (OFELI's 1-based column indices)
    d = next(k for k in range(rp[row], rp[row + 1]) if ci[k] == row + 1)
    a[d] = 0.0
    A.set_values(a)
    with pytest.raises(F.OFELIException, match="zero diagonal"):
        F.fgmres_mixed(P, g["b0"], np.zeros(A.n), inner_bits=inner_bits, toler=TOL)
    A.set_values(g["a0"])
    x = np.zeros(A.n)
    res = F.fgmres_mixed(P, g["b0"], x, inner_bits=inner_bits, toler=TOL)[2]
    assert res <= TOL


@pytest.fixture(scope="module")
def transient_net(cuda):
    net, info = LN.train_transient(nproblems=4, sizes=(64, 128), rounds=6)
    assert np.isfinite(info["loss_last"]) and info["loss_last"] < info["loss_first"]
    return net


def test_learned_fgmres_converges_and_gains(transient_net):
    """The learned preconditioner inside the mixed FGMRES, on a fresh
    velocity field at a size the network was not trained on: FP64 target
    met, and fewer Arnoldi steps than the diagonal preconditioner."""
    A, _ = LN.cd2d_problem(192, 999)
    b = A.Mult(fields.uniform_pm1(5, A.n))
    Pl = F.Prec(A, F.LEARNED_PREC, net=transient_net)
    Pd = F.Prec(A, F.DIAG_PREC)
    xl, xd = np.zeros(A.n), np.zeros(A.n)
    cl, sl, rl, fb = F.fgmres_mixed(Pl, b, xl, m=30, toler=TOL)
    cd, sd, rd, _ = F.fgmres_mixed(Pd, b, xd, m=30, toler=TOL)
    assert rl <= TOL and rd <= TOL and not fb
    assert F.residual(A, b, xl) <= 1.01 * TOL
    assert rel_err(xl, xd) <= 1e-8
    assert sl < sd, (sl, sd)


def test_learned_fgmres_frozen_across_steps(transient_net):
    """The transient driver computes the learned factor on the first step
    and keeps it (the matrix is the same at every step): the steps reach
    the FP64 target and follow OFELI's field."""
    g, info = load_golden("cd2d_17")
    eq = cd2d_start(info)
    for _ in range(info["steps"]):
        cycles, steps, res, fell_back = eq.step_mixed(F.LEARNED_PREC, net=transient_net, toler=TOL)
        assert res <= TOL and not fell_back
    assert rel_err(eq.u, g["u"]) <= 1e-8


def test_learned_fgmres_falls_back(cuda):
    """A network whose factor is not finite (NaN off-diagonal head weights,
    injected on the host): the solve notices the residual is not finite,
    finishes with the diagonal preconditioner and reports it.  (A NaN in the
    diagonal's offset c only drives the diagonal to its floor: a tiny
    multiple of a valid preconditioner, to which the right-preconditioned
    FGMRES is indifferent.)"""
    from oracle import learned_oracle as LO
    g, info = load_golden("cd2d_17")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a0"])
    net = F.LearnedNet(3)
    p, m1, m2, st = net.get_params()
    p[LO.P_U:LO.P_V] = np.nan
    net.set_params(p, m1, m2, st)
    x = np.zeros(A.n)
    cycles, steps, res, fell_back = F.fgmres_mixed(F.Prec(A, F.LEARNED_PREC, net=net), g["b0"], x,
                                                   toler=TOL)
    assert fell_back and res <= TOL and F.residual(A, g["b0"], x) <= 1.01 * TOL

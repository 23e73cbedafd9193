"""The CPU oracle of the learned preconditioner (oracle/learned_oracle.py)
pinned on its own: the hand-written reverse pass against central finite
differences of the FP64 loss (both objectives), the initial parameters
giving Jacobi, and the BF16 rounding helper."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import learned_oracle as LO
from oracle import oracle as O


def small_problem(M=4, seed=0):
    xyz, elem, code = O.mesh3d(M)
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 4, dof, n)
    k = np.exp(np.random.default_rng(seed).normal(size=elem.size // 4))
    a, b = O.assemble(3, xyz, elem, dof, code, n, rp, ci, k=k, f=np.ones(code.size))
    return rp, ci - 1, a, n


def params(seed):
    rng = np.random.default_rng(seed)
    P = LO.init_params(seed).astype(np.float64)
    P[LO.P_U:LO.P_C] = rng.normal(size=2 * LO.HID) * 0.3
    P[LO.P_B:LO.P_U] = rng.normal(size=LO.NLAYER * LO.HID) * 0.1
    P[LO.P_BIN:LO.P_W] = rng.normal(size=LO.HID) * 0.1
    return P


@pytest.mark.parametrize("kind", [0, 1])
def test_gradient_matches_finite_differences(kind):
    rp, col, a, n = small_problem()
    g = LO.Graph(rp, col, a)
    P = params(3)
    rng = np.random.default_rng(1)
    E = rng.normal(size=(3, n))
    R = (sp.csr_matrix((a, col, rp), shape=(n, n)) @ E.T).T
    loss, grad = LO.loss_and_grad(g, P, R, E, bf16=False, kind=kind)
    eps = 1e-6
    # directional derivative along a random direction (every parameter)
    d = rng.normal(size=LO.NPARAM)
    lp, _ = LO.loss_and_grad(g, P + eps * d, R, E, bf16=False, kind=kind)
    lm, _ = LO.loss_and_grad(g, P - eps * d, R, E, bf16=False, kind=kind)
    fd = (lp - lm) / (2 * eps)
    assert abs(fd - grad @ d) <= 1e-6 * max(1.0, abs(fd))
    # and single coordinates with a non-zero gradient in every group
    for lo_, hi in ((LO.P_WIN, LO.P_BIN), (LO.P_W, LO.P_B), (LO.P_B, LO.P_U), (LO.P_U, LO.NPARAM)):
        i = lo_ + int(np.argmax(np.abs(grad[lo_:hi])))
        e = np.zeros(LO.NPARAM)
        e[i] = eps
        lp, _ = LO.loss_and_grad(g, P + e, R, E, bf16=False, kind=kind)
        lm, _ = LO.loss_and_grad(g, P - e, R, E, bf16=False, kind=kind)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-5 * abs(fd) + 1e-10


def test_initial_parameters_give_jacobi():
    rp, col, a, n = small_problem()
    g = LO.Graph(rp, col, a)
    f = LO.forward(g, LO.init_params(5), bf16=True)
    assert np.allclose(f["g"][g.diag], 1.0 / g.dsq, rtol=1e-7)
    assert not f["g"][~g.diag].any()


def test_round_bf16():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0, 3.0e38])
    r = LO.round_bf16(x)
    # ties to even: 1 + 2^-8 -> 1, 1 + 3*2^-8 -> 1 + 2^-6
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6
    assert r[3] == -2.5 and r[4] == 0.0
    assert abs(r[5] - 3.0e38) <= 3.0e38 * 2 ** -8

"""The learned preconditioner on the GPU (ofeli_b200/csrc/learned.cu) against
its CPU oracle (oracle/learned_oracle.py): initial parameters, the
tensor-core layer product, loss and gradient of both objectives, training,
the gain over the method without it (Jacobi), the mixed-precision CG with
the learned preconditioner and its fallback on stagnation."""
import ctypes

import numpy as np
import pytest
import scipy.sparse as sp

from conftest import load_golden, rel_err
from ofeli_b200 import capi, fields
from ofeli_b200 import ofeli as F
from ofeli_b200.learned import kuhn_problem
from oracle import learned_oracle as LO

pytestmark = pytest.mark.gpu


def host_csr(A):
    rp, ci = A.pattern()
    return rp, ci - 1, A.values()


def perturbed_params(seed):
    rng = np.random.default_rng(seed)
    P = LO.init_params(seed).astype(np.float32)
    P[LO.P_U:LO.P_C] = (rng.normal(size=2 * LO.HID) * 0.3).astype(np.float32)
    P[LO.P_B:LO.P_U] = (rng.normal(size=LO.NLAYER * LO.HID) * 0.1).astype(np.float32)
    P[LO.P_BIN:LO.P_W] = (rng.normal(size=LO.HID) * 0.1).astype(np.float32)
    return P


def test_initial_parameters_match_oracle(cuda):
    for seed in (1, 12345):
        net = F.LearnedNet(seed)
        p, m, v, step = net.get_params()
        assert np.array_equal(p, LO.init_params(seed))
        assert not m.any() and not v.any() and step == 0


def test_tensor_core_layer_product(cuda):
    """tcgen05 layer product (BF16 operands, FP32 accumulation in tensor
    memory) against the CUDA-core product and FP64 numpy, on a row count that
    is not a multiple of the 128-row tile."""
    net = F.LearnedNet(3)
    params = perturbed_params(3)
    net.set_params(params)
    rows = 1000
    X = LO.round_bf16(np.random.default_rng(0).normal(size=(rows, 2 * LO.HID)))
    bits = (X.astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)
    for layer in (0, 3):
        tc = np.zeros((rows, LO.HID), np.float32)
        cc = np.zeros((rows, LO.HID), np.float32)
        capi.call("ofg_learned_gemm_check", net._h, layer, rows, F._ptr(bits), F._ptr(tc),
                  F._ptr(cc))
        W = LO.round_bf16(LO.split_params(params)["W"][layer])
        ref = X @ W
        assert rel_err(cc, ref) <= 1e-6
        assert rel_err(tc, ref) <= 1e-6
        assert np.abs(tc - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("kind", [0, 1])
def test_gradient_matches_oracle(cuda, kind):
    """Loss and the full gradient (both layer products on the tensor cores)
    against the oracle restated with the GPU's BF16 rounding points."""
    A, b, _ = kuhn_problem(6, 21)
    rp, col, a = host_csr(A)
    g = LO.Graph(rp, col, a)
    params = perturbed_params(5)
    rng = np.random.default_rng(2)
    E = rng.normal(size=(6, A.n)).astype(np.float32)
    Ah = sp.csr_matrix((a, col, rp), shape=(A.n, A.n))
    R = (Ah @ E.T.astype(np.float64)).T.astype(np.float32)
    net = F.LearnedNet(5, loss=kind)
    net.set_params(params)
    loss, grad, fac = net.grad(A, R, E)
    loss_o, grad_o = LO.loss_and_grad(g, params, R, E, bf16=True, kind=kind)
    f_o = LO.forward(g, params, bf16=True)["g"]
    keep = g.diag | g.lower
    assert rel_err(fac[keep], f_o[keep]) <= 1e-3
    assert abs(loss - loss_o) <= 1e-4 * max(1.0, abs(loss_o))
    groups = {"W_in": (LO.P_WIN, LO.P_BIN), "b_in": (LO.P_BIN, LO.P_W),
              "W": (LO.P_W, LO.P_B), "b": (LO.P_B, LO.P_U), "head": (LO.P_U, LO.NPARAM)}
    for name, (lo_, hi) in groups.items():
        assert np.abs(grad_o[lo_:hi]).max() > 0, name
        assert rel_err(grad[lo_:hi], grad_o[lo_:hi]) <= 2e-2, name
    # the CUDA-core path of the same products gives the same gradient
    net.set_tensor_cores(False)
    loss_c, grad_c, _ = net.grad(A, R, E)
    assert abs(loss_c - loss) <= 1e-5 * max(1.0, abs(loss))
    assert rel_err(grad_c, grad) <= 1e-3


def test_initial_network_is_jacobi(cuda):
    g, info = load_golden("p3d_kuhn_9")
    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    net = F.LearnedNet(1)
    _, _, fac = net.grad(A, np.ones((1, A.n), np.float32), np.ones((1, A.n), np.float32))
    rp, col, a = g["row_ptr"], g["col_ind"] - 1, g["a"]
    rows = np.repeat(np.arange(A.n), np.diff(rp))
    d = col == rows
    dsq = np.sqrt(np.abs(a[d])).astype(np.float32)
    assert rel_err(fac[d], 1.0 / dsq) <= 1e-6
    assert not fac[~d].any()
    x1, x2 = np.zeros(A.n), np.zeros(A.n)
    it_l = F.CG(A, F.Prec(A, F.LEARNED_PREC, net=net), g["b"], x1, 5000, 1e-10)
    it_d = F.CG(A, F.Prec(A, F.DIAG_PREC), g["b"], x2, 5000, 1e-10)
    assert it_l > 0 and abs(it_l - it_d) <= 2
    assert rel_err(x1, x2) <= 1e-8


@pytest.fixture(scope="module")
def trained(cuda):
    """A network trained by the library's own kernels on three 16^3 Kuhn
    problems with log-normal conductivities (sigma 1.5)."""
    net = F.LearnedNet(7)
    data = []
    for s in (11, 12, 13):
        A, b, mesh = kuhn_problem(16, s)
        R, E = F.LearnedNet.make_pairs(A, b, 64, seed=s)
        data.append((A, R, E, mesh))
    def loss():
        return np.mean([net.grad(A, R, E)[0] for A, R, E, _ in data])

    before = loss()
    for rnd in range(10):
        for A, R, E, _ in data:
            net.train(A, R, E, steps=10, batch=16, lr=1e-3)
    return net, before, loss()


def test_training_reduces_loss(trained):
    """The Kaporin objective (log of the condition-number measure) falls."""
    net, before, after = trained
    assert after < before - 0.02, (before, after)
    p, m, v, step = net.get_params()
    assert step == 300 and np.isfinite(p).all()


def test_trained_network_gains_over_jacobi(trained):
    """On a fresh conductivity field and a larger mesh than it was trained
    on, CG with the learned preconditioner needs markedly fewer iterations
    than CG with the method without it (Jacobi), to the same FP64 tolerance
    and the same solution."""
    net = trained[0]
    A, b, _ = kuhn_problem(24, 99)
    xl, xd = np.zeros(A.n), np.zeros(A.n)
    it_l = F.CG(A, F.Prec(A, F.LEARNED_PREC, net=net), b, xl, 20000, 1e-10)
    it_d = F.CG(A, F.Prec(A, F.DIAG_PREC), b, xd, 20000, 1e-10)
    assert it_l > 0 and it_d > 0
    assert it_l <= 0.75 * it_d, (it_l, it_d)
    assert rel_err(xl, xd) <= 1e-8


def test_learned_cg_mixed_precision(trained):
    net = trained[0]
    A, b, _ = kuhn_problem(24, 98)
    P = F.Prec(A, F.LEARNED_PREC, net=net)
    x = np.zeros(A.n)
    outer, inner, res, fell_back = F.fcg_learned(P, b, x, toler=1e-10)
    assert not fell_back and res <= 1e-10
    assert F.residual(A, b, x) <= 1e-10
    x64 = np.zeros(A.n)
    it = F.CG(A, F.Prec(A, F.DIAG_PREC), b, x64, 20000, 1e-12)
    assert it > 0 and rel_err(x, x64) <= 1e-8
    # fewer inner iterations than the Jacobi mixed solve
    xj = np.zeros(A.n)
    _, inner_j, res_j = F.solve_mixed(A, b, xj, prec=F.DIAG_PREC, toler=1e-10)
    assert res_j <= 1e-10 and inner <= 0.75 * inner_j, (inner, inner_j)


def test_fallback_on_stagnation(cuda):
    """Host-side fault injection: a network whose output is not finite makes
    the learned iteration stagnate; the solve falls back to the plain
    iteration and still converges on the FP64 true residual."""
    A, b, _ = kuhn_problem(8, 31)
    net = F.LearnedNet(2)
    p, _, _, _ = net.get_params()
    p[LO.P_C] = np.nan
    net.set_params(p)
    P = F.Prec(A, F.LEARNED_PREC, net=net)
    x = np.zeros(A.n)
    outer, inner, res, fell_back = F.fcg_learned(P, b, x, toler=1e-10)
    assert fell_back and res <= 1e-10
    assert F.residual(A, b, x) <= 1e-10


def test_checkpoint_round_trip(trained):
    net = trained[0]
    A, b, _ = kuhn_problem(6, 40)
    ones = np.ones((1, A.n), np.float32)
    state = net.get_params()
    l1, g1, f1 = net.grad(A, ones, ones)
    other = F.LearnedNet(99)
    other.set_params(*state)
    l2, g2, f2 = other.grad(A, ones, ones)
    assert l1 == l2 and np.array_equal(g1, g2) and np.array_equal(f1, f2)
    assert other.get_params()[3] == state[3]

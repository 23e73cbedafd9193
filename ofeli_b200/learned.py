"""Host-side driver of the learned preconditioner: the training problems and
the training schedule.  The network, its loss, gradients and Adam steps run
in the library's own kernels (LearnedNet -> ofg_learned_*)."""
import time

import numpy as np

from . import fields
from . import ofeli as F


def kuhn_problem(M, seed, sigma=1.5, corr_len=0.1, grid=64):
    """3-D P1 diffusion -div(k grad u) = 1 on the Kuhn cube with M^3 cells,
    u = 0 on the boundary, k = exp(g) per element with g a Gaussian field
    (standard deviation sigma, correlation length corr_len).  Returns the
    assembled matrix, the right-hand side and the mesh."""
    mesh = F.Mesh.kuhn(M)
    coords, elem, _, _ = mesh.arrays()
    cent = coords.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
    k = fields.lognormal_k(seed, cent, sigma, corr_len, grid=grid)
    eq = F.DC3DT4(mesh)
    eq.setSource(np.ones(mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    eq.setElementCoefficient(k)
    eq.build()
    return eq.getMatrix(), np.array(eq.getRHS()), mesh


def square_problem(nx, seed, sigma=None, corr_len=0.1, grid=128):
    """2-D P1 problem -div(k grad u) = f on the unit square with nx x nx cells
    (Laplace2DT3), f ~ U[-1, 1] per node, u = 0 on the boundary, k = 1 or
    log-normal with standard deviation sigma.  Returns (A, b, mesh)."""
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
    eq = F.Laplace2DT3(mesh)
    eq.setSource(fields.uniform_pm1(seed, mesh.nn))
    eq.setDirichlet(np.zeros(mesh.nn))
    if sigma:
        xy, elem, _, _ = mesh.arrays()
        cent = xy.reshape(-1, 2)[elem.reshape(-1, 3)].mean(axis=1)
        eq.setElementCoefficient(fields.lognormal_k(seed, cent, sigma, corr_len, grid=grid))
    eq.build()
    return eq.getMatrix(), np.array(eq.getRHS()), mesh


def train(net, problems, rounds=8, steps=10, batch=16, lr=1e-3, npairs=64):
    """Trains on residual / error pairs of every problem in turn (`steps`
    Adam steps per visit, `rounds` visits each).  problems: (A, b) pairs.
    Returns the per-visit mean batch losses."""
    data = []
    for q, (A, b) in enumerate(problems):
        R, E = F.LearnedNet.make_pairs(A, b, npairs, seed=1000 + q)
        data.append((A, R, E))
    hist = []
    for _ in range(rounds):
        for A, R, E in data:
            hist.append(float(net.train(A, R, E, steps=steps, batch=batch, lr=lr).mean()))
    return hist


def train_default(seed=7, M=20, nproblems=None, rounds=None, dim=3):
    """The networks used by the benchmark: trained on `nproblems` problems
    (seeds 100, 101, ...) with 64 residual / error pairs each -- 3-D: 32
    Kuhn cubes of M^3 cells, each with its own seeded log-normal
    conductivity field (sigma 1.5, correlation length 0.1), 2048 pairs in
    all, each problem visited twice; 2-D: 4 squares of (6M + 8)^2 cells,
    alternately k = 1 and log-normal k (sigma 1), visited 8 times.  Returns
    (net, info)."""
    if nproblems is None:
        nproblems = 32 if dim == 3 else 4
    if rounds is None:
        rounds = 2 if dim == 3 else 8
    t0 = time.perf_counter()
    net = F.LearnedNet(seed)
    problems = []
    keep = []
    for s in range(nproblems):
        if dim == 3:
            A, b, mesh = kuhn_problem(M, 100 + s)
        else:
            A, b, mesh = square_problem(6 * M + 8, 100 + s, None if s % 2 == 0 else 1.0)
        problems.append((A, b))
        keep.append(mesh)
    hist = train(net, problems, rounds=rounds)
    what = ("%d Kuhn cubes %d^3 nodes, lognormal k (sigma 1.5)" % (nproblems, M + 1) if dim == 3
            else "%d squares %d^2 nodes, k = 1 and lognormal k (sigma 1)" % (nproblems, 6 * M + 9))
    info = {"train_s": time.perf_counter() - t0, "adam_steps": rounds * nproblems * 10,
            "problems": what, "pairs_per_problem": 64, "pairs": 64 * nproblems,
            "loss_first": hist[0],
            "loss_last": hist[-1], "objective": "Kaporin number of M A on the pairs"}
    return net, info


def cd2d_problem(nx, seed, eps=1e-3, dt=1e-3, nx_target=1024):
    """A DC2DT3 backward-Euler matrix on nx x nx cells whose mass, diffusion
    and convection terms stand in the proportions they have on nx_target
    cells with (eps, dt): all three scale with h when eps and dt do, so
    eps and dt are multiplied by nx_target / nx.  The velocity field is a
    rotation about a seeded centre near (0.5, 0.5) with a seeded speed in
    [0.5, 1.5].  Returns (A, mesh)."""
    rng = np.random.default_rng(seed)
    c = 0.5 + 0.1 * rng.uniform(-1, 1, 2)
    w = rng.uniform(0.5, 1.5)
    s = nx_target / float(nx)
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    v = np.stack([-w * (P[:, 1] - c[1]), w * (P[:, 0] - c[0])], axis=1).reshape(-1)
    eq = F.DC2DT3(mesh, np.zeros(mesh.nn), v, eps * s, dt * s)
    eq.setDirichlet(np.zeros(mesh.nn))
    A, _ = eq.build()
    return A, mesh


def train_transient(seed=7, sizes=(128, 256), nproblems=4, rounds=8, npairs=64, steps=10):
    """The network of the transient benchmark's chosen form: trained on
    `nproblems` convection-diffusion matrices (cd2d_problem, seeds 200, 201,
    ..., sizes taken in turn) with the Kaporin objective on operator pairs
    (make_pairs_operator).  Returns (net, info)."""
    t0 = time.perf_counter()
    net = F.LearnedNet(seed)
    data, keep = [], []
    for q in range(nproblems):
        A, mesh = cd2d_problem(sizes[q % len(sizes)], 200 + q)
        R, E = F.LearnedNet.make_pairs_operator(A, npairs, seed=2000 + q)
        data.append((A, R, E))
        keep.append(mesh)
    hist = []
    for _ in range(rounds):
        for A, R, E in data:
            hist.append(float(net.train(A, R, E, steps=steps, batch=16).mean()))
    info = {"train_s": time.perf_counter() - t0, "adam_steps": rounds * nproblems * steps,
            "problems": "%d DC2DT3 backward-Euler matrices, %s cells, eps and dt scaled to the "
                        "1024^2-cell proportions, seeded rotations" % (nproblems, list(sizes)),
            "pairs_per_problem": npairs, "loss_first": hist[0], "loss_last": hist[-1],
            "objective": "Kaporin number of M A_sym on operator pairs r = A e"}
    return net, info

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


def train_default(seed=7, M=20, nproblems=4, rounds=8):
    """The network used by the benchmark: trained on `nproblems` Kuhn cubes
    of M^3 cells with log-normal conductivities (sigma 1.5, correlation
    length 0.1; seeds 100, 101, ...).  Returns (net, info)."""
    t0 = time.perf_counter()
    net = F.LearnedNet(seed)
    problems = []
    keep = []
    for s in range(nproblems):
        A, b, mesh = kuhn_problem(M, 100 + s)
        problems.append((A, b))
        keep.append(mesh)
    hist = train(net, problems, rounds=rounds)
    info = {"train_s": time.perf_counter() - t0, "adam_steps": rounds * nproblems * 10,
            "problems": "%d Kuhn cubes %d^3 nodes, lognormal k (sigma 1.5)" % (nproblems, M + 1),
            "pairs_per_problem": 64, "loss_first": hist[0], "loss_last": hist[-1],
            "objective": "Kaporin number of M A on the pairs"}
    return net, info

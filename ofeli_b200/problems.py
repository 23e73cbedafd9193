"""Seeded synthetic problem sets.

uneven_batch: the batched-solve workload -- `count` independent 2-D P1
diffusion problems on the unit square, node counts log-uniform in
[nmin, nmax] (square grids of side ~sqrt(N)), interior nodes jittered by a
radius <= 0.3 h (which keeps every triangle positively oriented), each with
its own log-normal conductivity (sigma 1, correlation length 0.1) and its
own source f ~ U[-1, 1] per node, u = 0 on the boundary."""
import math

import numpy as np

from . import fields
from . import ofeli as F


def uneven_sizes(seed, count=1024, nmin=1000, nmax=64000):
    """Grid cells per side of every problem (nodes = (nx + 1)^2)."""
    u = fields.uniform01(seed, count, 21)
    nodes = np.exp(math.log(nmin) + u * (math.log(nmax) - math.log(nmin)))
    return np.maximum(2, np.rint(np.sqrt(nodes)).astype(np.int64) - 1)


def uneven_batch(seed=1234, count=1024, nmin=1000, nmax=64000, k_grid=128):
    """(meshes, k, f): meshes on the device, k per element and f per node
    concatenated in problem order."""
    meshes, ks, fs = [], [], []
    for p, nx in enumerate(uneven_sizes(seed, count, nmin, nmax)):
        s = seed * 7919 + p
        m = F.Mesh(0.0, 1.0, 0.0, 1.0, int(nx), int(nx), 1, 1, 1, 1)
        xy, elem, code, _ = m.arrays()
        xy = fields.jitter_2d(s, xy, code, int(nx), int(nx), radius=0.3)
        m.setCoords(xy)
        cent = xy.reshape(-1, 2)[elem.reshape(-1, 3)].mean(axis=1)
        ks.append(fields.lognormal_k(s, cent, 1.0, 0.1, grid=k_grid))
        fs.append(fields.uniform_pm1(s, code.size))
        meshes.append(m)
    return meshes, np.concatenate(ks), np.concatenate(fs)

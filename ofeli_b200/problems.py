"""Seeded synthetic problem sets.

uneven_batch: the batched-solve workload -- `count` independent 2-D P1
diffusion problems on the unit square, node counts log-uniform in
[nmin, nmax] (square grids of side ~sqrt(N)), interior nodes jittered by a
radius <= 0.3 h (which keeps every triangle positively oriented), each with
its own log-normal conductivity (sigma 1, correlation length 0.1) and its
own source f ~ U[-1, 1] per node, u = 0 on the boundary.

ring_mesh: an annulus triangulated with a random diagonal per cell and a
random node numbering -- the shape of an unstructured user mesh read from a
file (code 1 on the inner circle, 2 on the outer one)."""
import math

import numpy as np

from . import fields
from . import ofeli as F


def uneven_sizes(seed, count=1024, nmin=1000, nmax=64000):
    """Grid cells per side of every problem (nodes = (nx + 1)^2)."""
    u = fields.uniform01(seed, count, 21)
    nodes = np.exp(math.log(nmin) + u * (math.log(nmax) - math.log(nmin)))
    return np.maximum(2, np.rint(np.sqrt(nodes)).astype(np.int64) - 1)


def partition_by_cost(costs, parts):
    """Independent problems split over `parts` ranks by estimated cost
    (longest first, each to the least loaded rank; ties to the lower rank):
    a list of `parts` ascending index arrays."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(costs.size), key=lambda i: (-costs[i], i))
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in order:
        r = min(range(parts), key=lambda j: (load[j], j))
        out[r].append(i)
        load[r] += costs[i]
    return [np.array(sorted(o), dtype=np.int64) for o in out]


def batch_costs(seed=1234, count=1024, nmin=1000, nmax=64000):
    """Estimated cost of every problem of the batch: its node count."""
    return (uneven_sizes(seed, count, nmin, nmax) + 1).astype(np.float64) ** 2


def uneven_batch(seed=1234, count=1024, nmin=1000, nmax=64000, k_grid=128, indices=None):
    """(meshes, k, f): meshes on the device, k per element and f per node
    concatenated in problem order; `indices` selects a subset of the batch
    (each problem keeps its own seeds)."""
    meshes, ks, fs = [], [], []
    sizes = uneven_sizes(seed, count, nmin, nmax)
    for p in (range(count) if indices is None else indices):
        nx = sizes[p]
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


def ring_mesh(nr, nt, seed=0, r0=0.5, r1=1.0, jitter=0.2):
    """(coords (nn, 2), elem (ne, 3) 0-based and positively oriented, node
    code (nn,), sides (ns, 2) 0-based boundary segments, side mark (ns,)).
    nr + 1 circles of nt nodes; interior nodes moved by up to `jitter` of the
    radial and angular spacing; nodes numbered by a random permutation."""
    rng = np.random.default_rng(seed)
    i, j = np.meshgrid(np.arange(nr + 1), np.arange(nt), indexing="ij")
    r = r0 + (r1 - r0) * i / nr
    t = 2 * np.pi * j / nt
    inner = (i > 0) & (i < nr)
    r = r + inner * rng.uniform(-jitter, jitter, r.shape) * (r1 - r0) / nr
    t = t + inner * rng.uniform(-jitter, jitter, t.shape) * 2 * np.pi / nt
    xy = np.stack([r * np.cos(t), r * np.sin(t)], axis=-1).reshape(-1, 2)
    code = np.where(i == 0, 1, np.where(i == nr, 2, 0)).reshape(-1).astype(np.int32)
    gid = lambda a, b: a * nt + b % nt  # noqa: E731
    ii, jj = np.meshgrid(np.arange(nr), np.arange(nt), indexing="ij")
    ii, jj = ii.ravel(), jj.ravel()
    p00, p10, p11, p01 = gid(ii, jj), gid(ii + 1, jj), gid(ii + 1, jj + 1), gid(ii, jj + 1)
    flip = rng.random(ii.size) < 0.5
    t1 = np.where(flip[:, None], np.stack([p00, p10, p01], 1), np.stack([p00, p10, p11], 1))
    t2 = np.where(flip[:, None], np.stack([p10, p11, p01], 1), np.stack([p00, p11, p01], 1))
    elem = np.stack([t1, t2], 1).reshape(-1, 3)
    k = np.arange(nt)
    sides = np.concatenate([np.stack([gid(0, k + 1), gid(0, k)], 1),
                            np.stack([gid(nr, k), gid(nr, k + 1)], 1)])
    smark = np.concatenate([np.full(nt, 1), np.full(nt, 2)]).astype(np.int32)
    perm = rng.permutation(xy.shape[0])          # new number of old node
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    xy_new = np.empty_like(xy)
    xy_new[perm] = xy
    code_new = np.empty_like(code)
    code_new[perm] = code
    return (xy_new, perm[elem].astype(np.int32), code_new, perm[sides].astype(np.int32), smark)

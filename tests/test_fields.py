"""Deterministic synthetic inputs."""
import numpy as np

from ofeli_b200 import fields
from oracle import oracle as O


def test_uniform_is_deterministic_and_in_range():
    a = fields.uniform_pm1(1234, 100000)
    b = fields.uniform_pm1(1234, 100000)
    assert np.array_equal(a, b)
    assert a.min() >= -1.0 and a.max() < 1.0
    assert abs(a.mean()) < 0.01 and abs(a.std() - 1 / np.sqrt(3)) < 0.01
    assert not np.array_equal(a, fields.uniform_pm1(1235, 100000))
    # prefix property: the first values do not depend on the count
    assert np.array_equal(fields.uniform_pm1(7, 10), fields.uniform_pm1(7, 1000)[:10])


def test_gaussian_field_statistics():
    g = fields.gaussian_field(3, 2, 128, 1.5, 0.1)
    assert abs(g.mean()) < 1e-12 and abs(g.std() - 1.5) < 1e-12
    # correlated: neighbouring lattice values are close
    c = np.corrcoef(g[:, :-1].ravel(), g[:, 1:].ravel())[0, 1]
    assert c > 0.9


def test_lognormal_contrast():
    xyz, elem, code = O.mesh3d(6)
    cent = xyz.reshape(-1, 3)[elem.reshape(-1, 4)].mean(axis=1)
    k = fields.lognormal_k(7, cent, 1.5, 0.1, grid=32)
    assert (k > 0).all() and k.max() / k.min() > 100


def test_jitter_stays_within_radius_and_keeps_boundary():
    nx = 20
    xy, elem, code = O.mesh2d(nx, nx)
    j = fields.jitter_2d(5, xy, code, nx, nx, radius=0.3)
    d = np.hypot(*(j - xy).reshape(-1, 2).T)
    assert d.max() <= 0.3 / nx + 1e-15
    assert np.array_equal(j.reshape(-1, 2)[code > 0], xy.reshape(-1, 2)[code > 0])
    # every triangle keeps a positive Jacobian
    P = j.reshape(-1, 2)[elem.reshape(-1, 3)]
    det = (P[:, 1, 0] - P[:, 0, 0]) * (P[:, 2, 1] - P[:, 0, 1]) - \
          (P[:, 1, 1] - P[:, 0, 1]) * (P[:, 2, 0] - P[:, 0, 0])
    assert (det > 0).all()


def test_uneven_batch_sizes():
    """The batched workload: 1024 problems, node counts log-uniform in
    [1000, 64000], about 15.4 million nodes in all."""
    from ofeli_b200 import problems
    s = problems.uneven_sizes(1234)
    nodes = (s + 1) ** 2
    assert len(s) == 1024 and nodes.min() >= 900 and nodes.max() <= 66000
    assert 15.0e6 < nodes.sum() < 16.0e6

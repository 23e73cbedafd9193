"""Deterministic synthetic inputs for the P1 Poisson / diffusion workloads.

Every generator is a pure function of (seed, size) so the oracle, the
reference harness and the GPU path all read the same numbers:

* ``uniform_pm1`` -- values in [-1, 1) from a counter-based splitmix64 hash
  (one 64-bit draw per index, top 53 bits used).  This is the source term
  ``f`` "uniform in [-1,1] per node from the seed".
* ``gaussian_field`` -- a stationary Gaussian field with squared-exponential
  covariance ``sigma^2 exp(-r^2 / (2 l^2))`` on the periodic unit square/cube,
  synthesised spectrally on a ``G^d`` grid from Box-Muller normals, then
  standardised to zero mean and standard deviation ``sigma`` and sampled
  (multi)linearly.  ``k = exp(g)`` gives the lognormal conductivities.
* ``jitter_2d`` -- moves every interior node of a structured grid by a random
  vector of length <= ``r*h`` (uniform angle, uniform radius fraction).
"""
import numpy as np

_M1 = np.uint64(0x9E3779B97F4A7C15)
_M2 = np.uint64(0xBF58476D1CE4E5B9)
_M3 = np.uint64(0x94D049BB133111EB)
_MS = np.uint64(0xD1B54A32D192ED03)
_MT = np.uint64(0x8CB92BA72F3D8DD7)


def _splitmix(seed, stream, n):
    i = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) * _MS + np.uint64(stream) * _MT + i * _M1
        z = (z ^ (z >> np.uint64(30))) * _M2
        z = (z ^ (z >> np.uint64(27))) * _M3
        z = z ^ (z >> np.uint64(31))
    return z


def uniform01(seed, n, stream=0):
    """n doubles in [0, 1)."""
    return (_splitmix(seed, stream, n) >> np.uint64(11)).astype(np.float64) * (2.0 ** -53)


def uniform_pm1(seed, n, stream=0):
    """n doubles in [-1, 1)."""
    return uniform01(seed, n, stream) * 2.0 - 1.0


def normal(seed, n, stream=0):
    """n standard normals by Box-Muller on two uniform streams."""
    u1 = uniform01(seed, n, 2 * stream + 101)
    u2 = uniform01(seed, n, 2 * stream + 102)
    return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)


def gaussian_field(seed, dim, grid, sigma, corr_len, stream=0):
    """Periodic stationary Gaussian field on a grid**dim lattice (values at
    the lattice points i/grid)."""
    shape = (grid,) * dim
    w = normal(seed, grid ** dim, stream).reshape(shape)
    k1 = np.fft.fftfreq(grid, d=1.0 / grid)
    kk = np.zeros(shape)
    for ax in range(dim):
        sh = [1] * dim
        sh[ax] = grid
        kk = kk + (k1.reshape(sh)) ** 2
    # spectral density of exp(-r^2/(2 l^2)) up to a constant factor
    spec = np.exp(-2.0 * np.pi ** 2 * corr_len ** 2 * kk)
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.sqrt(spec)))
    g = g - g.mean()
    sd = g.std()
    if sd > 0:
        g = g * (sigma / sd)
    return g


def sample_periodic(g, pts):
    """(Multi)linear interpolation of a periodic lattice field at points in
    the unit box; pts has shape (m, dim)."""
    dim = g.ndim
    G = g.shape[0]
    s = np.asarray(pts, dtype=np.float64) * G
    i0 = np.floor(s).astype(np.int64)
    t = s - i0
    out = np.zeros(s.shape[0])
    for corner in range(1 << dim):
        wgt = np.ones(s.shape[0])
        idx = []
        for ax in range(dim):
            b = (corner >> ax) & 1
            wgt = wgt * (t[:, ax] if b else (1.0 - t[:, ax]))
            idx.append((i0[:, ax] + b) % G)
        out += wgt * g[tuple(idx)]
    return out


def lognormal_k(seed, centroids, sigma, corr_len, grid=None, stream=0):
    """Per-element conductivity exp(g(centroid))."""
    dim = centroids.shape[1]
    if grid is None:
        grid = 256 if dim == 3 else 512
    g = gaussian_field(seed, dim, grid, sigma, corr_len, stream)
    return np.exp(sample_periodic(g, centroids))


def jitter_2d(seed, xy, code, nx, ny, radius=0.3):
    """Interior nodes (code 0) moved by at most radius*min(hx,hy)."""
    h = min(1.0 / nx, 1.0 / ny)
    nn = xy.shape[0] // 2
    a = uniform01(seed, nn, 11) * 2.0 * np.pi
    r = uniform01(seed, nn, 12) * radius * h
    out = xy.copy().reshape(nn, 2)
    m = code == 0
    out[m, 0] += r[m] * np.cos(a[m])
    out[m, 1] += r[m] * np.sin(a[m])
    return out.reshape(-1)

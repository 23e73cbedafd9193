"""The batched solver (ofeli_b200/csrc/batch.cu): many uneven 2-D problems
assembled and solved in one persistent launch, checked problem by problem
against the oracle (OFELI's assembly and CG + DIAG restated): assembled
values and RHS bit-exact, solutions 1e-9; for every launch shape of the
autotuner, and for run-to-run determinism."""
import numpy as np
import pytest

from conftest import rel_err
from ofeli_b200 import fields
from ofeli_b200 import ofeli as F
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-10


def small_batch(sizes, seed=5, bc=False):
    meshes, ks, fs, bcs, ref = [], [], [], [], []
    for p, nx in enumerate(sizes):
        s = seed * 31 + p
        xy, elem, code = O.mesh2d(nx, nx)
        xy = fields.jitter_2d(s, xy, code, nx, nx, radius=0.3)
        cent = xy.reshape(-1, 2)[elem.reshape(-1, 3)].mean(axis=1)
        k = fields.lognormal_k(s, cent, 1.0, 0.1, grid=64)
        f = fields.uniform_pm1(s, code.size)
        g = fields.uniform_pm1(s, code.size, 3) if bc else np.zeros(code.size)
        m = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
        m.setCoords(xy)
        meshes.append(m)
        ks.append(k)
        fs.append(f)
        bcs.append(g)
        dof, n = O.number_equations(code)
        rp, ci = O.node_graph(elem, 3, dof, n)
        a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, k=k, f=f, bc=g)
        x, it = O.cg(rp, ci, a, b, O.DIAG, 100000, TOL)
        ref.append({"a": a, "b": b, "x": x, "it": it, "u": O.insert_bc(code, x, g),
                    "nnz": int(rp[-1]), "n": n})
    B = F.Batch(meshes)
    B.set_inputs(np.concatenate(ks), np.concatenate(fs), np.concatenate(bcs) if bc else None)
    return B, ref, meshes


def check_against_oracle(B, ref, matrices=True):
    u, it, res = B.results()
    off = 0
    for p, r in enumerate(ref):
        up = u[off:off + r["u"].size]
        off += r["u"].size
        assert res[p] <= TOL
        assert abs(int(it[p]) - r["it"]) <= 2, (p, it[p], r["it"])
        assert rel_err(up, r["u"]) <= 1e-9, p
        if matrices:
            a, b = B.matrix(p, r["nnz"], r["n"])
            assert np.array_equal(a, r["a"]) and np.array_equal(b, r["b"]), p


def test_batch_matches_oracle_problem_by_problem(cuda):
    B, ref, _ = small_batch([4, 30, 9, 17, 2, 41, 12])
    B.solve(100000, TOL)
    check_against_oracle(B, ref)


def test_batch_with_dirichlet_data(cuda):
    B, ref, _ = small_batch([6, 19, 11], seed=9, bc=True)
    B.solve(100000, TOL)
    check_against_oracle(B, ref)


def test_every_launch_shape_and_the_tuner(cuda):
    B, ref, _ = small_batch([25, 7, 14, 33, 3, 20], seed=11)
    for c in range(F.Batch.NCONFIGS):
        B.set_config(c)
        B.solve(100000, TOL)
        check_against_oracle(B, ref, matrices=False)
    chosen, times = B.tune(100000, TOL)
    assert 0 <= chosen < F.Batch.NCONFIGS and (times > 0).all()
    assert times[chosen] == times.min()
    B.solve(100000, TOL)
    check_against_oracle(B, ref, matrices=False)


def test_graph_replay_is_deterministic(cuda):
    B, ref, _ = small_batch([15, 26, 8, 31], seed=13)
    B.solve(100000, TOL)
    u1, it1, r1 = B.results()
    B.solve(100000, TOL)
    u2, it2, r2 = B.results()
    assert np.array_equal(u1, u2) and np.array_equal(it1, it2) and np.array_equal(r1, r2)


def test_iteration_cap_reports_failure(cuda):
    B, ref, _ = small_batch([20, 10], seed=17)
    B.solve(5, TOL)
    _, it, res = B.results()
    assert (it == -5).all() and (res > TOL).all()


def test_inverted_element_is_reported(cuda):
    """A mesh with an inverted triangle (made on the host) is refused with
    OFELI's "negative determinant" error, as the single-problem assembly
    does."""
    meshes = []
    for nx in (5, 6):
        m = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx, 1, 1, 1, 1)
        meshes.append(m)
    xy, elem, code, _ = meshes[1].arrays()
    xy = xy.copy().reshape(-1, 2)
    i = int(np.nonzero(code == 0)[0][0])
    xy[i] += 1.5 / 6  # moves an interior node across its neighbours
    meshes[1].setCoords(xy.ravel())
    B = F.Batch(meshes)
    B.set_inputs()
    with pytest.raises(F.OFELIException, match="Jacobian"):
        B.solve(1000, TOL)



def test_clusters_mix_shared_and_per_block_problems(cuda):
    """With thread-block clusters, the large problems are solved by a whole
    cluster and the small ones one per block: both paths against the
    oracle, for every clustered launch shape (concurrency limited so that
    the small problems fall below one block's share of the work)."""
    rng = np.random.default_rng(3)
    sizes = [44, 37] + list(rng.integers(2, 7, size=300))
    B, ref, _ = small_batch(sizes, seed=23)
    for c in range(6, F.Batch.NCONFIGS):
        B.set_config(c, blocks_per_sm=1)
        B.solve(100000, TOL)
        check_against_oracle(B, ref, matrices=False)
    a, b = B.matrix(0, ref[0]["nnz"], ref[0]["n"])
    assert np.array_equal(a, ref[0]["a"]) and np.array_equal(b, ref[0]["b"])


def check_mixed(B, ref):
    """FP32 inner CG inside FP64 refinement: the same FP64 target, the
    oracle's FP64 solution up to the conditioning of each problem."""
    u, it, res = B.results()
    off = 0
    for p, r in enumerate(ref):
        up = u[off:off + r["u"].size]
        off += r["u"].size
        assert res[p] <= TOL and it[p] > 0, (p, res[p], it[p])
        assert it[p] <= 2 * r["it"] + 20, (p, it[p], r["it"])
        assert rel_err(up, r["u"]) <= 1e-7, p


def test_mixed_precision_batch(cuda):
    B, ref, _ = small_batch([4, 30, 9, 17, 2, 41, 12], seed=29)
    B.set_precision(32)
    B.solve(100000, TOL)
    check_mixed(B, ref)
    a, b = B.matrix(5, ref[5]["nnz"], ref[5]["n"])
    assert np.array_equal(a, ref[5]["a"]) and np.array_equal(b, ref[5]["b"])
    B.set_precision(64)
    B.solve(100000, TOL)
    check_against_oracle(B, ref, matrices=False)


def test_mixed_precision_batch_with_clusters(cuda):
    rng = np.random.default_rng(7)
    sizes = [44, 37] + list(rng.integers(2, 7, size=200))
    B, ref, _ = small_batch(sizes, seed=31, bc=True)
    B.set_precision(32)
    for c in (0, 4, 6, 12, 16):
        B.set_config(c, blocks_per_sm=1)
        B.solve(100000, TOL)
        check_mixed(B, ref)

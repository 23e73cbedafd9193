"""The reference OFELI (oracle/_ref, compiled from its own sources) against
the oracle on fresh seeds -- skipped where the reference was not built."""
import numpy as np
import pytest

from ofeli_b200 import fields
from oracle import oracle as O

pytestmark = pytest.mark.skipif(not O.have_reference("o2"),
                                reason="oracle/_ref not built (needs the reference sources)")


@pytest.mark.parametrize("seed,prec", [(11, "DILU"), (12, "SSOR"), (13, "DIAG")])
def test_reference_matches_oracle_2d(seed, prec):
    nx, ny = 20, 17
    xy, elem, code = O.mesh2d(nx, ny)
    f = fields.uniform_pm1(seed, code.size)
    info, out = O.run_reference(["p2d", nx, ny, "CG", prec, 1e-10, 5000], {"f": f})
    dof, n = O.number_equations(code)
    rp, ci = O.node_graph(elem, 3, dof, n)
    a, b = O.assemble(2, xy, elem, dof, code, n, rp, ci, f=f, bc=np.zeros(code.size))
    assert np.array_equal(out["row_ptr"], rp) and np.array_equal(out["col_ind"], ci)
    assert np.array_equal(out["a"], a) and np.array_equal(out["b"], b)
    x, it = O.cg(rp, ci, a, b, O.PREC_NAMES[prec], 5000, 1e-10)
    assert it == info["iters"] and np.array_equal(x, out["x"])


def test_reference_bench_mode_runs():
    f = fields.uniform_pm1(1234, 33 * 33)
    info, _ = O.run_reference(["bench2d", 32, "ILU", 5, 2], {"f": f})
    assert info["iters"] == -6 and len(str(info["t_iters_steps"]).split(",")) == 2

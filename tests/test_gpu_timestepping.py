"""OFELI's TimeStepping driver (src/solvers/TimeStepping.cpp) on the device:
the first-order schemes of a DC2DT3 equation against the reference's own
TimeStepping runs (tests/golden/ts2d_17.npz): forward Euler bit for bit
(assembly and the explicit division are exact), the implicit schemes with
iterations +-2 and the field to 1e-12."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from ofeli_b200 import ofeli as F

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["FE", "BE", "CN"])
def test_timestepping_first_order_schemes(cuda, name):
    g, info = load_golden("ts2d_17")
    nx = info["nx"]
    mesh = F.Mesh(0.0, 1.0, 0.0, 1.0, nx, nx)
    xy, _, code, _ = mesh.arrays()
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    scheme = {"FE": F.FORWARD_EULER, "BE": F.BACKWARD_EULER, "CN": F.CRANK_NICOLSON}[name]
    eq = F.DC2DT3(mesh, u0, v, info["eps"], info["dt"])
    eq.getLinearSolver().setTolerance(info["tol"])
    eq.getLinearSolver().setMaxIter(2000)
    ts = F.TimeStepping(scheme, info["dt"], info["steps"] * info["dt"])
    ts.setPDE(eq)
    ts.setInitial(u0)
    ts.setBC(np.zeros(mesh.nn))
    ts.setLinearSolver(F.GMRES_SOLVER, F.ILU_PREC)
    for s in range(info["steps"]):
        ts.runOneTimeStep()
        ref = g[name + "_u_steps"][s]
        if name == "FE":
            assert np.array_equal(ts.getSolution(), ref)
        else:
            assert abs(eq.getLinearSolver().getNbIter() - g[name + "_iters"][s]) <= 2
            assert rel_err(ts.getSolution(), ref) <= 1e-12


def test_timestepping_rejects_other_schemes(cuda):
    with pytest.raises(F.OFELIException):
        F.TimeStepping(F.NEWMARK, 1e-3)

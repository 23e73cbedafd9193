"""Generates the golden fixtures of tests/golden/ by running the reference
OFELI itself (oracle/_ref/o2/ofeli_ref, compiled by oracle/Makefile from the
reference's own sources at -O2) on seeded synthetic inputs.

    make -C oracle ref && python tests/golden/make_golden.py

Each case is one .npz (CSR pattern in OFELI's layout, assembled values,
RHS, solutions) plus the harness' info (iteration counts, norms) under the
key "info" as JSON.  Inputs come from ofeli_b200.fields with the seeds
recorded in the file, so the tests regenerate them instead of storing them.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from ofeli_b200 import fields  # noqa: E402
from oracle import oracle as O  # noqa: E402


def centroids(coords, elem, dim):
    return coords.reshape(-1, dim)[elem.reshape(-1, dim + 1)].mean(axis=1)


def save(name, arrays, meta):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, info=np.array(json.dumps(meta)), **arrays)
    print("wrote", path, os.path.getsize(path), "bytes")


def case_p2d_65():
    """65x65-node Poisson (8192 triangles), f ~ U[-1,1] seed 1234, u = 0 on
    the boundary: every preconditioner with CG, GMRES(30) and GMRES(10)."""
    nx = 64
    f = fields.uniform_pm1(1234, (nx + 1) ** 2)
    arrays, meta = {}, {"nx": nx, "ny": nx, "seed_f": 1234, "tol": 1e-10, "runs": {}}
    for solver, prec in [("CG", "IDENT"), ("CG", "DIAG"), ("CG", "DILU"), ("CG", "SSOR"),
                         ("GMRES30", "ILU"), ("GMRES30", "DIAG"), ("GMRES10", "SSOR")]:
        info, out = O.run_reference(["p2d", nx, nx, solver, prec, 1e-10, 20000], {"f": f})
        if not arrays:
            arrays["row_ptr"] = out["row_ptr"].astype(np.int32)
            arrays["col_ind"] = out["col_ind"].astype(np.int32)
            arrays["a"] = out["a"]
            arrays["b"] = out["b"]
            meta["n"], meta["nnz"] = info["n"], info["nnz"]
        key = "%s_%s" % (solver, prec)
        arrays["x_" + key] = out["x"]
        meta["runs"][key] = {"iters": info["iters"], "norm_u": info["norm_u"]}
    save("p2d_65", arrays, meta)


def case_p2d_jitter():
    """25x25 nodes, interior nodes jittered by <= 0.3h (seed 5), per-element
    lognormal k (sigma 1, l 0.1, seed 5), f seed 5; CG + ILU."""
    nx = 24
    xy, elem, code = O.mesh2d(nx, nx)
    xyj = fields.jitter_2d(5, xy, code, nx, nx)
    k = fields.lognormal_k(5, centroids(xyj, elem, 2), 1.0, 0.1, grid=128)
    f = fields.uniform_pm1(5, code.size)
    info, out = O.run_reference(["p2d", nx, nx, "CG", "ILU", 1e-10, 20000],
                                {"f": f, "k": k, "xy": xyj})
    save("p2d_jitter_25", {"row_ptr": out["row_ptr"].astype(np.int32),
                           "col_ind": out["col_ind"].astype(np.int32), "a": out["a"],
                           "b": out["b"], "x": out["x"], "u": out["u"]},
         {"nx": nx, "seed": 5, "sigma": 1.0, "corr": 0.1, "grid": 128, "tol": 1e-10,
          "iters": info["iters"], "n": info["n"], "nnz": info["nnz"]})


def case_p2d_ragged():
    """13x6 nodes (ragged), Dirichlet only on the x = 0 and x = 1 lines
    (codes 1, 2; natural conditions on the y lines), non-zero imposed values
    bc = 1 + x + 2y, f seed 9; CG + DIAG."""
    nx, ny = 12, 5
    xy, elem, code = O.mesh2d(nx, ny, codes=(1, 2, 0, 0))
    P = xy.reshape(-1, 2)
    bc = 1.0 + P[:, 0] + 2.0 * P[:, 1]
    f = fields.uniform_pm1(9, code.size)
    info, out = O.run_reference(["p2d", nx, ny, "CG", "DIAG", 1e-10, 20000], {"f": f, "bc": bc},
                                extra=(1, 2, 0, 0))
    save("p2d_ragged", {"row_ptr": out["row_ptr"].astype(np.int32),
                        "col_ind": out["col_ind"].astype(np.int32), "a": out["a"], "b": out["b"],
                        "x": out["x"], "u": out["u"]},
         {"nx": nx, "ny": ny, "codes": [1, 2, 0, 0], "seed_f": 9, "tol": 1e-10,
          "iters": info["iters"], "n": info["n"], "nnz": info["nnz"]})


def case_p3d():
    """Kuhn cube 9^3 nodes (8^3 cells, 3072 tetrahedra), lognormal k
    (sigma 1.5, l 0.1, grid 32, seed 7), f seed 99; CG + ILU and CG + DIAG."""
    M = 8
    xyz, elem, code = O.mesh3d(M)
    k = fields.lognormal_k(7, centroids(xyz, elem, 3), 1.5, 0.1, grid=32)
    f = fields.uniform_pm1(99, code.size)
    arrays, meta = {}, {"M": M, "seed_k": 7, "seed_f": 99, "sigma": 1.5, "corr": 0.1, "grid": 32,
                        "tol": 1e-10, "runs": {}}
    for prec in ("ILU", "DIAG"):
        info, out = O.run_reference(["p3d", M, "CG", prec, 1e-10, 20000], {"f": f, "k": k})
        if not arrays:
            arrays.update(row_ptr=out["row_ptr"].astype(np.int32),
                          col_ind=out["col_ind"].astype(np.int32), a=out["a"], b=out["b"])
            meta["n"], meta["nnz"] = info["n"], info["nnz"]
        arrays["x_" + prec] = out["x"]
        meta["runs"][prec] = {"iters": info["iters"], "norm_u": info["norm_u"]}
    save("p3d_kuhn_9", arrays, meta)


def case_cd2d():
    """17x17-node convection-diffusion, eps 1e-3, v = (-(y-0.5), x-0.5),
    Gaussian bump (width 0.05 at (0.3, 0.5)), backward Euler dt 1e-3, 5
    steps, GMRES(30) + ILU with the previous step as initial guess."""
    nx, steps, dt, eps = 16, 5, 1e-3, 1e-3
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    info, out = O.run_reference(["cd2d", nx, nx, steps, dt, eps, "GMRES30", "ILU", 1e-10, 2000],
                                {"u0": u0, "v": v})
    save("cd2d_17", {"row_ptr": out["row_ptr"].astype(np.int32),
                     "col_ind": out["col_ind"].astype(np.int32), "a0": out["a"], "b0": out["b0"],
                     "u": out["u"], "iters": out["iters"]},
         {"nx": nx, "steps": steps, "dt": dt, "eps": eps, "tol": 1e-10, "m": 30,
          "n": info["n"], "nnz": info["nnz"]})


def case_bicgstab():
    """OFELI's BiCGStab: the 65x65 Poisson system of case_p2d_65 with DIAG and
    ILU, and the 17x17 convection-diffusion steps of case_cd2d with ILU."""
    nx = 64
    f = fields.uniform_pm1(1234, (nx + 1) ** 2)
    arrays, meta = {}, {"nx": nx, "tol": 1e-10, "runs": {}}
    for prec in ("DIAG", "ILU"):
        info, out = O.run_reference(["p2d", nx, nx, "BICGSTAB", prec, 1e-10, 20000], {"f": f})
        arrays["x_p2d_" + prec] = out["x"]
        meta["runs"]["p2d_" + prec] = {"iters": info["iters"]}
    nx2, steps, dt, eps = 16, 5, 1e-3, 1e-3
    xy, elem, code = O.mesh2d(nx2, nx2)
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    info, out = O.run_reference(["cd2d", nx2, nx2, steps, dt, eps, "BICGSTAB", "ILU", 1e-10, 2000],
                                {"u0": u0, "v": v})
    arrays.update(cd2d_u=out["u"], cd2d_iters=out["iters"])
    meta["cd2d"] = {"nx": nx2, "steps": steps, "dt": dt, "eps": eps}
    save("bicgstab", arrays, meta)


if __name__ == "__main__":
    if not O.have_reference("o2"):
        raise SystemExit("build the reference first: make -C oracle ref")
    case_p2d_65()
    case_p2d_jitter()
    case_p2d_ragged()
    case_p3d()
    case_cd2d()
    case_bicgstab()

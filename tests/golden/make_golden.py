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
import tempfile

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


def case_cd2d_schemes():
    """The 17x17 convection-diffusion steps of case_cd2d under OFELI's other
    time schemes: forward Euler and Crank-Nicolson, GMRES(30) + ILU, 5 steps."""
    nx, steps, dt, eps = 16, 5, 1e-3, 1e-3
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    arrays, meta = {}, {"nx": nx, "steps": steps, "dt": dt, "eps": eps, "tol": 1e-10, "m": 30,
                        "schemes": {"FE": 1, "CN": 3}}
    for name in ("FE", "CN"):
        info, out = O.run_reference(["cd2d", nx, nx, steps, dt, eps, "GMRES30", "ILU", 1e-10, 2000],
                                    {"u0": u0, "v": v}, extra=[name])
        arrays.update({name + "_a0": out["a"], name + "_b0": out["b0"], name + "_u": out["u"],
                       name + "_iters": out["iters"]})
    save("cd2d_schemes", arrays, meta)


# nb_dof 2 with negative and multi-digit marks, the "tria" alias, attributes
# in either order (one pair written without a blank between them), tabs and a
# CR, comments outside the blocks, a node no element uses, element code 3
# only (no material "Generic" under code 1, so Mesh::put writes an empty
# Material block).
MESHIO_CODES = (
    '<?xml version="1.0"?>\n'
    "<!-- nb_dof 2, negative and multi-digit marks, sides with negative marks -->\n"
    "<OFELI_File>\n<info><title>codes</title></info>\n"
    "<Mesh nb_dof=\"2\"   dim=\"2\" >\n"
    "   <Nodes>\n\t0.0 0.0 11\n   1.0  0.0   -12\r\n   1.0 1.0 3\n 0.0 1.0 -1\n"
    " 0.5 0.5 0\n 1e-1 2.5E-1 120\n 0.3333333333333333 -7.25e-3 -99\n   </Nodes>\n"
    "   <!-- four triangles around the centre -->\n"
    '   <Elements shape="tria" nodes="3">\n 1 2 5 3\n 2 3 5 3\n 3 4 5 3\n 4 1 5 3\n'
    "   </Elements>\n"
    "   <Sides nodes=\"2\"shape=\"line\">\n 1 2 -21\n 2 3 10\n 3 4 0\n 4 1 -3\n   </Sides>\n"
    "</Mesh>\n</OFELI_File>\n")


def kuhn_permuted(M, seed):
    xyz, elem, code = O.mesh3d(M)
    rng = np.random.default_rng(seed)
    perm = rng.permutation(code.size)
    xyz2 = np.empty_like(xyz.reshape(-1, 3))
    xyz2[perm] = xyz.reshape(-1, 3)
    code2 = np.empty_like(code)
    code2[perm] = code
    return xyz2, perm[elem.reshape(-1, 4)].astype(np.int32), code2


def case_meshio():
    """OFELI's .m mesh files: Mesh::get of three files written here (an
    annulus with a random numbering, sides and a Material block; a small
    hand-written nb_dof 2 file; a Kuhn cube with a random numbering), their
    Mesh::put bytes, Mesh(rect).put with negative line codes, and the P1
    problems solved on the two P1 meshes by Mesh(file, true)."""
    from ofeli_b200 import problems
    from oracle import mesh_oracle as MO
    xy, elem, code, sides, smark = problems.ring_mesh(6, 24, seed=1)
    ecode = np.where(np.arange(elem.shape[0]) % 4 == 0, 2, 1).astype(np.int32)
    ring = dict(dim=2, nb_dof=1, el_shape=3, el_nodes=3, sd_shape=2, sd_nodes=2, coords=xy,
                node_code=code[:, None], elem=elem, elem_code=ecode, sides=sides,
                side_code=smark[:, None])
    text = MO.put(ring).decode().replace(
        "</Mesh>", "   <Material>\n     1   Generic\n     2   Copper\n   </Material>\n</Mesh>")
    xyz, tet, tcode = kuhn_permuted(3, seed=2)
    tetm = dict(dim=3, nb_dof=1, el_shape=5, el_nodes=4, sd_shape=0, sd_nodes=0, coords=xyz,
                node_code=tcode[:, None], elem=tet, elem_code=np.ones(tet.shape[0], np.int32),
                sides=np.zeros((0, 1), np.int32), side_code=np.zeros((0, 1), np.int32))
    files = {"meshio_ring": text, "meshio_codes": MESHIO_CODES,
             "meshio_tet": MO.put(tetm).decode()}
    arrays, meta = {}, {"files": {}, "runs": {}}
    for name, body in files.items():
        path = os.path.join(HERE, name + ".m")
        with open(path, "w", newline="") as fh:
            fh.write(body)
        info, out = O.run_reference(["mget", path], {})
        tmp = tempfile.mkdtemp(prefix="mget_")
        O.run_reference(["mget", path], {}, keep=tmp)
        put = open(os.path.join(tmp, "out", "put.m"), "rb").read()
        key = name.split("_", 1)[1]
        arrays.update({key + "_coords": out["coords"], key + "_node_code": out["node_code"],
                       key + "_elem": out["elem"] - 1, key + "_elem_code": out["elem_code"],
                       key + "_side": out["side"] - 1, key + "_side_code": out["side_code"],
                       key + "_put": np.frombuffer(put, np.uint8)})
        meta["files"][key] = {k: info[k] for k in ("dim", "nb_dof", "nodes", "elements", "sides",
                                                   "el_shape", "el_nodes", "sd_shape", "sd_nodes")}
    # Mesh(0,1,0,1,4,3,-1,2,-3,0): sides on x = 0 and y = 0, code 2 on x = 1
    tmp = tempfile.mkdtemp(prefix="mrect_")
    O.run_reference(["mrect", 4, 3, -1, 2, -3, 0], {}, keep=tmp)
    arrays["rect_put"] = np.fromfile(os.path.join(tmp, "out", "put.m"), np.uint8)
    # P1 problems on the meshes read back: the annulus with k = 1 (element
    # code 1) or 3 (code 2), f seed 11, u = 1 on the outer circle; the cube
    # with f seed 12, u = 0 on the boundary
    nn = xy.shape[0]
    ring_bc = np.where(code == 2, 1.0, 0.0)
    ring_k = np.where(ecode == 2, 3.0, 1.0)
    ring_f = fields.uniform_pm1(11, nn)
    tet_f = fields.uniform_pm1(12, xyz.shape[0])
    for key, path, inputs, runs in [
            ("ring", "meshio_ring.m", {"f": ring_f, "bc": ring_bc, "k": ring_k},
             [("CG", "DILU"), ("CG", "DIAG"), ("BICGSTAB", "ILU")]),
            ("tet", "meshio_tet.m", {"f": tet_f}, [("CG", "DILU")])]:
        for solver, prec in runs:
            info, out = O.run_reference(["mlap", os.path.join(HERE, path), solver, prec, 1e-10,
                                         20000], inputs)
            if key + "_row_ptr" not in arrays:
                arrays.update({key + "_row_ptr": out["row_ptr"].astype(np.int32),
                               key + "_col_ind": out["col_ind"].astype(np.int32),
                               key + "_a": out["a"], key + "_b": out["b"]})
            arrays["%s_x_%s_%s" % (key, solver, prec)] = out["x"]
            arrays["%s_u_%s_%s" % (key, solver, prec)] = out["u"]
            meta["runs"]["%s_%s_%s" % (key, solver, prec)] = {"iters": info["iters"]}
    meta["ring"] = {"seed_f": 11, "k": [1.0, 3.0], "bc_outer": 1.0}
    meta["tet"] = {"seed_f": 12}
    save("meshio", arrays, meta)


def case_ts2d():
    """OFELI's TimeStepping class driving DC2DT3 on the 17x17-node transient
    problem of case_cd2d (eps 1e-3, v = (-(y-0.5), x-0.5), Gaussian bump,
    u = 0 on the boundary): 5 runOneTimeStep calls of dt 1e-3 under forward
    Euler, backward Euler and Crank-Nicolson, GMRES + ILU to 1e-10 for the
    implicit schemes; the nodal field after every call."""
    nx, steps, dt, eps = 16, 5, 1e-3, 1e-3
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    arrays, meta = {}, {"nx": nx, "steps": steps, "dt": dt, "eps": eps, "tol": 1e-10,
                        "solver": "GMRES", "prec": "ILU"}
    for sc in ("FE", "BE", "CN"):
        info, out = O.run_reference(["ts2d", nx, nx, steps, dt, eps, sc, "GMRES", "ILU", 1e-10,
                                     2000], {"u0": u0, "v": v})
        arrays[sc + "_u_steps"] = out["u_steps"].reshape(steps, -1)
        arrays[sc + "_iters"] = out["iters"]
    save("ts2d_17", arrays, meta)


def _sample_pins(x, stride):
    return {"x_norm2": float(np.linalg.norm(x)), "x_sum": float(x.sum()),
            "x_sample_stride": stride}, {"x_sample": x[::stride].copy()}


def pins_p2d_2049():
    """The benchmark's 2-D problem at full size (2049x2049 nodes, f seed
    1234, u = 0 on the boundary): OFELI's CG + ILU to 1e-10, run to
    convergence (about 11 minutes of one core at -O2)."""
    nx = 2048
    f = fields.uniform_pm1(1234, (nx + 1) ** 2)
    info, out = O.run_reference(["p2d", nx, nx, "CG", "ILU", 1e-10, 100000], {"f": f})
    meta, arrays = _sample_pins(out["x"], 4096)
    meta.update(nx=nx, seed_f=1234, solver="CG", prec="ILU", tol=1e-10, iters=info["iters"],
                n=info["n"], nnz=info["nnz"], norm_u=info["norm_u"],
                t_solve_cpu_o2_s=info["t_solve"], t_assembly_cpu_o2_s=info["t_assembly"],
                t_graph_cpu_o2_s=info["t_graph"])
    save("p2d_2049_pins", arrays, meta)


def pins_p3d_129():
    """The benchmark's 3-D problem at full size (Kuhn cube 129^3 nodes,
    12.6M tetrahedra; k = exp(g), g the seeded Gaussian field of sigma 1.5
    and correlation length 0.1 synthesised on a 256^3 lattice, seed 1234;
    f seed 1234; u = 0 on the faces): OFELI's CG + ILU and CG + DIAG to
    1e-10, run to convergence."""
    M = 128
    xyz, elem, code = O.mesh3d(M)
    k = fields.lognormal_k(1234, centroids(xyz, elem, 3), 1.5, 0.1, grid=256)
    f = fields.uniform_pm1(1234, code.size)
    del xyz, elem
    meta = {"M": M, "seed_k": 1234, "seed_f": 1234, "sigma": 1.5, "corr": 0.1, "grid": 256,
            "tol": 1e-10, "runs": {}}
    arrays = {}
    for prec in ("ILU", "DIAG"):
        info, out = O.run_reference(["p3d", M, "CG", prec, 1e-10, 100000], {"f": f, "k": k})
        m, a = _sample_pins(out["x"], 2048)
        m.update(iters=info["iters"], norm_u=info["norm_u"], t_solve_cpu_o2_s=info["t_solve"],
                 t_assembly_cpu_o2_s=info["t_assembly"], t_graph_cpu_o2_s=info["t_graph"])
        meta["runs"][prec] = m
        arrays["x_sample_" + prec] = a["x_sample"]
        meta["n"], meta["nnz"] = info["n"], info["nnz"]
        del out
    save("p3d_129_pins", arrays, meta)


def pins_cd2d_1025():
    """The benchmark's transient problem at full size (DC2DT3 on 1025x1025
    nodes, eps 1e-3, v = (-(y-0.5), x-0.5), Gaussian bump at (0.3, 0.5) of
    width 0.05, u = 0 on the boundary, backward Euler dt 1e-3): the first
    three steps with OFELI's GMRES(30) + ILU, warm-started, to 1e-10."""
    nx, steps, dt, eps = 1024, 3, 1e-3, 1e-3
    xy, elem, code = O.mesh2d(nx, nx)
    P = xy.reshape(-1, 2)
    u0 = np.exp(-((P[:, 0] - 0.3) ** 2 + (P[:, 1] - 0.5) ** 2) / (2 * 0.05 ** 2))
    u0[code > 0] = 0.0
    v = np.stack([-(P[:, 1] - 0.5), P[:, 0] - 0.5], axis=1).reshape(-1)
    info, out = O.run_reference(["cd2d", nx, nx, steps, dt, eps, "GMRES30", "ILU", 1e-10, 2000],
                                {"u0": u0, "v": v})
    meta, arrays = _sample_pins(out["x"], 1024)
    meta.update(nx=nx, steps=steps, dt=dt, eps=eps, tol=1e-10, m=30, n=info["n"],
                nnz=info["nnz"], iters=[int(i) for i in out["iters"]],
                u_norm2=float(np.linalg.norm(out["u"])), t_graph_cpu_o2_s=info["t_graph"],
                t_assembly_cpu_o2_s=info["t_assembly"], t_prec_cpu_o2_s=info["t_prec"],
                t_solve_cpu_o2_s=info["t_solve"])
    save("cd2d_1025_pins", arrays, meta)


FULLSIZE = {"p2d_2049": pins_p2d_2049, "p3d_129": pins_p3d_129, "cd2d_1025": pins_cd2d_1025}


if __name__ == "__main__":
    if not O.have_reference("o2"):
        raise SystemExit("build the reference first: make -C oracle ref")
    if len(sys.argv) > 1:
        # full-size pins, each minutes to tens of minutes of one core:
        #   python tests/golden/make_golden.py p3d_129 cd2d_1025 [p2d_2049]
        for name in sys.argv[1:]:
            FULLSIZE[name]()
        raise SystemExit(0)
    case_p2d_65()
    case_p2d_jitter()
    case_p2d_ragged()
    case_p3d()
    case_cd2d()
    case_bicgstab()
    case_meshio()
    case_cd2d_schemes()
    case_ts2d()

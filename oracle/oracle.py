"""Python access to the CPU oracle (liboracle.so, the C restatement in
ofeli_oracle.c) and to the reference OFELI harness (oracle/_ref/*/ofeli_ref).

TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py use it as the checker; the product
(ofeli_b200 + libofeli_gpu.so) never imports it.
"""
import ctypes
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

IDENT, DIAG, DILU, ILU, SSOR = 0, 1, 2, 3, 4
PREC_NAMES = {"IDENT": IDENT, "DIAG": DIAG, "DILU": DILU, "ILU": ILU, "SSOR": SSOR}

_lib = None

_p = ctypes.c_void_p
_i64 = ctypes.c_int64


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


def build_port():
    subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build_port()
        L = ctypes.CDLL(path)
        L.or_mesh2d.argtypes = [_i64, _i64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, _p, _p, _p]
        L.or_mesh3d_kuhn.argtypes = [_i64, _p, _p, _p]
        L.or_number_equations.argtypes = [_i64, _p, _p]
        L.or_number_equations.restype = _i64
        L.or_node_graph.argtypes = [_i64, ctypes.c_int, _p, _p, _i64, _p, _p]
        L.or_node_graph.restype = _i64
        L.or_assemble_p1.argtypes = [ctypes.c_int, _i64, _i64, _p, _p, _p, _p, _p, _p, _p, _i64,
                                     _p, _p, _p, _p]
        L.or_assemble_p1.restype = _i64
        L.or_assemble_cd2d.argtypes = [_i64, _i64, _p, _p, _p, _p, ctypes.c_double, _p,
                                       ctypes.c_double, _p, _p, _i64, _p, _p, _p, _p]
        L.or_assemble_cd2d.restype = _i64
        L.or_assemble_cd2d_scheme.argtypes = [_i64, _i64, _p, _p, _p, _p, ctypes.c_double, _p,
                                              ctypes.c_double, ctypes.c_int, _p, _p, _i64, _p,
                                              _p, _p, _p]
        L.or_assemble_cd2d_scheme.restype = _i64
        L.or_spmv.argtypes = [_i64, _p, _p, _p, _p, _p]
        L.or_prec_setup.argtypes = [ctypes.c_int, _i64, _p, _p, _p, _p, _p]
        L.or_prec_setup.restype = _i64
        L.or_prec_apply.argtypes = [ctypes.c_int, _i64, _p, _p, _p, _p, _p, _p, _p]
        L.or_cg.argtypes = [_i64, _p, _p, _p, ctypes.c_int, _p, _p, ctypes.c_int,
                            ctypes.c_double, _p]
        L.or_cg.restype = ctypes.c_int
        L.or_gmres.argtypes = [_i64, _p, _p, _p, ctypes.c_int, _p, _p, ctypes.c_int,
                               ctypes.c_int, ctypes.c_double]
        L.or_gmres.restype = ctypes.c_int
        L.or_bicgstab.argtypes = [_i64, _p, _p, _p, ctypes.c_int, _p, _p, ctypes.c_int,
                                  ctypes.c_double]
        L.or_bicgstab.restype = ctypes.c_int
        L.or_insert_bc.argtypes = [_i64, _p, _p, _p, _p]
        L.or_spmv_transpose_add.argtypes = [_i64, _p, _p, _p, _p, _p]
        L.or_matrix_edit.argtypes = [_i64, _p, _p, _p, _i64, _p, _p, _p, ctypes.c_int]
        L.or_matrix_edit.restype = _i64
        _lib = L
    return _lib


# ----------------------------------------------------------------- meshes --

def mesh2d(nx, ny, codes=(1, 1, 1, 1)):
    nn = (nx + 1) * (ny + 1)
    xy = np.zeros(2 * nn)
    elem = np.zeros(6 * nx * ny, dtype=np.int32)
    code = np.zeros(nn, dtype=np.int32)
    lib().or_mesh2d(nx, ny, 0.0, 1.0, 0.0, 1.0, codes[0], codes[1], codes[2], codes[3],
                    _ptr(xy), _ptr(elem), _ptr(code))
    return xy, elem, code


def mesh3d(M):
    nn = (M + 1) ** 3
    xyz = np.zeros(3 * nn)
    elem = np.zeros(24 * M ** 3, dtype=np.int32)
    code = np.zeros(nn, dtype=np.int32)
    lib().or_mesh3d_kuhn(M, _ptr(xyz), _ptr(elem), _ptr(code))
    return xyz, elem, code


def number_equations(code):
    dof = np.zeros(code.size, dtype=np.int64)
    n = lib().or_number_equations(code.size, _ptr(code), _ptr(dof))
    return dof, int(n)


def node_graph(elem, nen, dof, n):
    ne = elem.size // nen
    rp = np.zeros(n + 1, dtype=np.int64)
    ci = np.zeros(max(1, ne * nen * nen), dtype=np.int64)
    nnz = lib().or_node_graph(ne, nen, _ptr(elem), _ptr(dof), n, _ptr(rp), _ptr(ci))
    return rp, ci[:nnz].copy()


def assemble(dim, coords, elem, dof, code, n, rp, ci, k=None, f=None, bc=None):
    nen = dim + 1
    ne = elem.size // nen
    a = np.zeros(int(rp[-1]))
    b = np.zeros(n)
    ret = lib().or_assemble_p1(dim, code.size, ne, _ptr(coords), _ptr(elem), _ptr(dof),
                               _ptr(code), _ptr(k), _ptr(f), _ptr(bc), n, _ptr(rp), _ptr(ci),
                               _ptr(a), _ptr(b))
    if ret < 0:
        raise ValueError("non-positive Jacobian in element %d" % (-ret))
    return a, b


def assemble_cd2d(xy, elem, dof, code, n, rp, ci, eps, v, dt, u_old, bc=None, scheme=2):
    """scheme: OFELI's TimeScheme (1 forward Euler, 2 backward Euler, 3
    Crank-Nicolson)."""
    ne = elem.size // 3
    a = np.zeros(int(rp[-1]))
    b = np.zeros(n)
    ret = lib().or_assemble_cd2d_scheme(code.size, ne, _ptr(xy), _ptr(elem), _ptr(dof),
                                        _ptr(code), eps, _ptr(v), dt, scheme, _ptr(u_old),
                                        _ptr(bc), n, _ptr(rp), _ptr(ci), _ptr(a), _ptr(b))
    if ret < 0:
        raise ValueError("non-positive Jacobian in element %d" % (-ret))
    return a, b


def spmv(rp, ci, a, x):
    y = np.zeros(rp.size - 1)
    lib().or_spmv(rp.size - 1, _ptr(rp), _ptr(ci), _ptr(a), _ptr(x), _ptr(y))
    return y


def spmv_transpose_add(rp, ci, a, x, y):
    y = np.array(y, dtype=np.float64)
    lib().or_spmv_transpose_add(rp.size - 1, _ptr(rp), _ptr(ci), _ptr(a), _ptr(x), _ptr(y))
    return y


def matrix_edit(rp, ci, a, i, j, v, set_values):
    """(new values, index of the first pair outside the pattern or -1)."""
    a = np.array(a, dtype=np.float64)
    i = np.ascontiguousarray(i, dtype=np.int64)
    j = np.ascontiguousarray(j, dtype=np.int64)
    v = np.ascontiguousarray(v, dtype=np.float64)
    bad = lib().or_matrix_edit(rp.size - 1, _ptr(rp), _ptr(ci), _ptr(a), i.size, _ptr(i), _ptr(j),
                               _ptr(v), 1 if set_values else 0)
    return a, int(bad)


def prec_setup(ptype, rp, ci, a):
    n = rp.size - 1
    idv = np.zeros(n, dtype=np.int64)
    piv = np.zeros(n)
    r = lib().or_prec_setup(ptype, n, _ptr(rp), _ptr(ci), _ptr(a), _ptr(idv), _ptr(piv))
    if r < 0:
        raise ZeroDivisionError("zero pivot in row %d" % (-r))
    return idv, piv


def prec_apply(ptype, rp, ci, a, idv, piv, b):
    x = np.zeros(rp.size - 1)
    lib().or_prec_apply(ptype, rp.size - 1, _ptr(rp), _ptr(ci), _ptr(a), _ptr(idv), _ptr(piv),
                        _ptr(b), _ptr(x))
    return x


def cg(rp, ci, a, b, ptype, max_it, tol, x0=None, history=False):
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    hist = np.zeros(max_it + 1) if history else None
    it = lib().or_cg(n, _ptr(rp), _ptr(ci), _ptr(a), ptype, _ptr(b), _ptr(x), max_it, tol,
                     _ptr(hist))
    return (x, it, hist) if history else (x, it)


def bicgstab(rp, ci, a, b, ptype, max_it, tol, x0=None):
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    it = lib().or_bicgstab(n, _ptr(rp), _ptr(ci), _ptr(a), ptype, _ptr(b), _ptr(x), max_it, tol)
    return x, it


def gmres(rp, ci, a, b, ptype, m, max_it, tol, x0=None):
    n = rp.size - 1
    x = np.zeros(n) if x0 is None else np.array(x0, dtype=np.float64)
    it = lib().or_gmres(n, _ptr(rp), _ptr(ci), _ptr(a), ptype, _ptr(b), _ptr(x), m, max_it, tol)
    return x, it


def insert_bc(code, x, bc=None):
    u = np.zeros(code.size)
    lib().or_insert_bc(code.size, _ptr(code), _ptr(x), _ptr(bc), _ptr(u))
    return u


# --------------------------------------------------- the reference itself --

def ref_binary(flavour="o2"):
    return os.path.join(REF_DIR, flavour, "ofeli_ref")


def have_reference(flavour="o2"):
    return os.path.exists(ref_binary(flavour))


def read_info(outdir):
    info = {}
    with open(os.path.join(outdir, "info.txt")) as fh:
        for line in fh:
            k, _, v = line.strip().partition("=")
            try:
                info[k] = int(v)
            except ValueError:
                try:
                    info[k] = float(v)
                except ValueError:
                    info[k] = v
    return info


def run_reference(args, inputs, flavour="o2", keep=None, timeout=None, extra=()):
    """Runs ofeli_ref with the given argument list (INDIR / OUTDIR appended,
    then `extra`) and returns (info, outputs) with outputs loaded as numpy
    arrays."""
    tmp = keep or tempfile.mkdtemp(prefix="ofeli_ref_")
    indir, outdir = os.path.join(tmp, "in"), os.path.join(tmp, "out")
    os.makedirs(indir, exist_ok=True)
    os.makedirs(outdir, exist_ok=True)
    for name, arr in inputs.items():
        np.ascontiguousarray(arr, dtype=np.float64).tofile(os.path.join(indir, name + ".f64"))
    env = dict(os.environ)
    env["OFELI_PATH_MATERIAL"] = os.path.join(REF_DIR, "material")
    cmd = [ref_binary(flavour)] + [str(a) for a in args] + [indir, outdir] + [str(e) for e in extra]
    subprocess.run(cmd, check=True, env=env, timeout=timeout)
    info = read_info(outdir)
    out = {}
    for fn in os.listdir(outdir):
        stem, ext = os.path.splitext(fn)
        if ext == ".f64":
            out[stem] = np.fromfile(os.path.join(outdir, fn), dtype=np.float64)
        elif ext == ".i64":
            out[stem] = np.fromfile(os.path.join(outdir, fn), dtype=np.int64)
        elif ext == ".i32":
            out[stem] = np.fromfile(os.path.join(outdir, fn), dtype=np.int32)
    return info, out

"""OFELI's API for the P1 assembly + Krylov path, backed by libofeli_gpu.so.

Names, argument meanings, 1-based/0-based conventions and return values
follow OFELI 5.3.3 (paths within that project):

* ``Mesh(xmin, xmax, ymin, ymax, nx, ny, cx0, cxN, cy0, cyN)``: the structured
  triangulation of src/mesh/Mesh.cpp:547-676; ``Mesh.kuhn(M)`` the unit cube;
  ``Mesh.from_arrays`` a general P1 mesh (Mesh::Add); ``Mesh.from_file`` /
  ``get`` / ``put`` OFELI's XML mesh files (``MeshFile`` holds a file's
  content on the host).
* ``SpMatrix(mesh)`` / ``SpMatrix(row_ptr, col_ind[, a])``: CSR with OFELI's
  layout (0-based row_ptr, 1-based col_ind), include/linear_algebra/SpMatrix.h.
* ``Prec(A, type)``, ``CG(A, P, b, x, max_it, toler)``,
  ``GMRes(A, P, b, x, m, max_it, toler)``, ``LinearSolver``: include/solvers.
* ``Laplace2DT3``, ``Laplace3DT4`` / ``DC3DT4``, ``DC2DT3``: ``build()``,
  ``updateBC`` (folded into build), ``run()``.

Vectors are numpy float64 arrays (host) or CUDA tensors (device pointers).
Errors raise ``OFELIException`` as OFELI throws on zero pivots, negative
Jacobians, missing matrices.
"""
import ctypes
import math

import numpy as np

from . import capi, fields

IDENT_PREC, DIAG_PREC, DILU_PREC, ILU_PREC, SSOR_PREC = 0, 1, 2, 3, 4
# no OFELI counterpart: M = G^T G predicted by a trained network (LearnedNet)
LEARNED_PREC = 5
DIRECT_SOLVER, CG_SOLVER, CGS_SOLVER, BICG_SOLVER, BICG_STAB_SOLVER, GMRES_SOLVER = 1, 2, 3, 4, 5, 6
# OFELI's TimeScheme values (include/equations/Equa.h:124-137) on the path
FORWARD_EULER, BACKWARD_EULER, CRANK_NICOLSON = 1, 2, 3
OFELI_EPSMCH = 2.220446049250313e-16


class OFELIException(RuntimeError):
    pass


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return ctypes.c_void_p(a.ctypes.data)
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    raise TypeError("expected a numpy array or a CUDA tensor")


def _call(name, *args):
    try:
        capi.call(name, *args)
    except capi.OFGError as e:
        raise OFELIException(str(e)) from e


def _f64(a, n=None):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return a
    out = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None and out.size != n:
        raise OFELIException("vector size %d, expected %d" % (out.size, n))
    return out


class Mesh:
    """Mesh(xmin, xmax, ymin, ymax, nx, ny, cx0, cxN, cy0, cyN) -- structured
    triangulation, 2 triangles per cell, equations on code-0 nodes."""

    def __init__(self, xmin=0.0, xmax=1.0, ymin=0.0, ymax=1.0, nx=None, ny=None, cx0=1, cxN=1,
                 cy0=1, cyN=1, _handle=None):
        if _handle is not None:
            self._h = _handle
        else:
            h = ctypes.c_void_p()
            _call("ofg_mesh_create_rect", xmin, xmax, ymin, ymax, nx, ny, cx0, cxN, cy0, cyN,
                  ctypes.byref(h))
            self._h = h
        self._info()

    @classmethod
    def kuhn(cls, M):
        h = ctypes.c_void_p()
        _call("ofg_mesh_create_kuhn", M, ctypes.byref(h))
        return cls(_handle=h)

    @classmethod
    def from_arrays(cls, dim, coords, elem, code):
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        code = np.ascontiguousarray(code, dtype=np.int32)
        h = ctypes.c_void_p()
        _call("ofg_mesh_create", dim, code.size, _ptr(coords), elem.size // (dim + 1), _ptr(elem),
              _ptr(code), ctypes.byref(h))
        return cls(_handle=h)

    def _info(self):
        d = ctypes.c_int()
        nn, ne, neq = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _call("ofg_mesh_info", self._h, ctypes.byref(d), ctypes.byref(nn), ctypes.byref(ne),
              ctypes.byref(neq))
        self.dim, self.nn, self.ne, self.neq = d.value, nn.value, ne.value, neq.value

    def getNbNodes(self):
        return self.nn

    def getNbElements(self):
        return self.ne

    def getNbEq(self):
        return self.neq

    def arrays(self):
        coords = np.zeros(self.nn * self.dim)
        elem = np.zeros(self.ne * (self.dim + 1), dtype=np.int32)
        code = np.zeros(self.nn, dtype=np.int32)
        dof = np.zeros(self.nn, dtype=np.int64)
        _call("ofg_mesh_get", self._h, _ptr(coords), _ptr(elem), _ptr(code), _ptr(dof))
        return coords, elem, code, dof

    def setCoords(self, coords):
        coords = _f64(coords, self.nn * self.dim)
        _call("ofg_mesh_set_coords", self._h, _ptr(coords))
        self._coords_changed = True

    @classmethod
    def from_file(cls, path):
        """Mesh(file, true): a P1 mesh read from OFELI's XML format, equations
        on the code-0 nodes, tokenised and converted on the device
        (ofg_mesh_read).  put() writes the file's own content (sides,
        element codes), read again from `path` on the host when asked."""
        h = ctypes.c_void_p()
        _call("ofg_mesh_read", str(path).encode(), ctypes.byref(h))
        m = cls(_handle=h)
        m._path = str(path)
        return m

    def get(self, path):
        """Mesh::get(file) (src/mesh/Mesh.cpp:2639-2668): replaces this mesh."""
        m = Mesh.from_file(path)
        old = getattr(self, "_h", None)
        self._h, m._h = m._h, old
        self._path, self._file = m._path, None
        self._coords_changed = False
        self._info()

    def put(self, path):
        """Mesh::put(file) (src/mesh/Mesh.cpp:2731-2806)."""
        mf = getattr(self, "_file", None)
        if mf is None and getattr(self, "_path", None) and not getattr(self, "_coords_changed",
                                                                      False):
            mf = self._file = MeshFile(self._path)
        if mf is None or getattr(self, "_coords_changed", False):
            mf = MeshFile.from_mesh(self)
        mf.put(path)

    def save(self, path):
        """Mesh::save for the ".m" format."""
        if not str(path).endswith(".m"):
            raise OFELIException("only OFELI's .m format is written")
        self.put(path)

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_mesh_destroy(self._h)
            self._h = None


# OFELI's element shape codes (include/OFELI_Config.h:274-282)
POINT, LINE, TRIANGLE, QUADRILATERAL, TETRAHEDRON, HEXAHEDRON, PENTAHEDRON = 1, 2, 3, 4, 5, 6, 7


class MeshFile:
    """The host-side content of an OFELI ``.m`` mesh file, as Mesh::get keeps
    it: ``coords`` (nn x dim, float-rounded as OFELI's stof does),
    ``node_code`` (nn x nb_dof), ``elem`` (ne x el_nodes, 0-based),
    ``elem_code``, ``sides`` (ns x sd_nodes, 0-based), ``side_code``
    (ns x nb_dof).  Reading and writing need no GPU."""

    def __init__(self, path=None, _handle=None):
        if _handle is None:
            h = ctypes.c_void_p()
            _call("ofg_mesh_file_read", str(path).encode(), ctypes.byref(h))
            _handle = h
        self._h = _handle
        i = [ctypes.c_int() for _ in range(6)]
        n = [ctypes.c_int64() for _ in range(3)]
        _call("ofg_mesh_file_info", self._h, ctypes.byref(i[0]), ctypes.byref(i[1]),
              ctypes.byref(n[0]), ctypes.byref(i[2]), ctypes.byref(i[3]), ctypes.byref(n[1]),
              ctypes.byref(i[4]), ctypes.byref(i[5]), ctypes.byref(n[2]))
        self.dim, self.nb_dof = i[0].value, i[1].value
        self.el_shape, self.el_nodes, self.sd_shape, self.sd_nodes = (i[2].value, i[3].value,
                                                                      i[4].value, i[5].value)
        self.nn, self.ne, self.ns = n[0].value, n[1].value, n[2].value

    @classmethod
    def create(cls, dim, coords, node_code, elem, elem_code, el_shape, nb_dof=1, sides=None,
               side_code=None, sd_shape=LINE):
        coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1)
        node_code = np.ascontiguousarray(node_code, dtype=np.int32).reshape(-1)
        elem = np.ascontiguousarray(elem, dtype=np.int32)
        elem_code = np.ascontiguousarray(elem_code, dtype=np.int32).reshape(-1)
        nn, ne = coords.size // dim, elem_code.size
        el_nodes = elem.size // max(ne, 1)
        if sides is None:
            sides = np.zeros(0, np.int32)
            side_code = np.zeros(0, np.int32)
        sides = np.ascontiguousarray(sides, dtype=np.int32)
        side_code = np.ascontiguousarray(side_code, dtype=np.int32).reshape(-1)
        ns = side_code.size // nb_dof
        sd_nodes = sides.size // ns if ns else 0
        h = ctypes.c_void_p()
        _call("ofg_mesh_file_create", dim, nb_dof, nn, _ptr(coords), _ptr(node_code), el_shape,
              el_nodes, ne, _ptr(elem), _ptr(elem_code), sd_shape, sd_nodes, ns, _ptr(sides),
              _ptr(side_code), ctypes.byref(h))
        return cls(_handle=h)

    @classmethod
    def from_mesh(cls, mesh):
        h = ctypes.c_void_p()
        _call("ofg_mesh_file_from_mesh", mesh._h, ctypes.byref(h))
        return cls(_handle=h)

    def arrays(self):
        coords = np.zeros((self.nn, self.dim))
        node_code = np.zeros((self.nn, self.nb_dof), np.int32)
        elem = np.zeros((self.ne, self.el_nodes), np.int32)
        elem_code = np.zeros(self.ne, np.int32)
        sides = np.zeros((self.ns, self.sd_nodes), np.int32)
        side_code = np.zeros((self.ns, self.nb_dof), np.int32)
        _call("ofg_mesh_file_get", self._h, _ptr(coords), _ptr(node_code), _ptr(elem),
              _ptr(elem_code), _ptr(sides), _ptr(side_code))
        return dict(coords=coords, node_code=node_code, elem=elem, elem_code=elem_code,
                    sides=sides, side_code=side_code)

    def put(self, path):
        _call("ofg_mesh_file_write", self._h, str(path).encode())

    def to_mesh(self):
        h = ctypes.c_void_p()
        _call("ofg_mesh_create_from_file", self._h, ctypes.byref(h))
        return Mesh(_handle=h)

    @staticmethod
    def set_threads(n):
        _call("ofg_mesh_file_set_threads", n)

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_mesh_file_destroy(self._h)
            self._h = None


class SpMatrix:
    """SpMatrix<real_t>: SpMatrix(mesh) builds the node graph on the device;
    SpMatrix(row_ptr, col_ind[, a]) takes OFELI's CSR layout."""

    def __init__(self, *args):
        h = ctypes.c_void_p()
        self.mesh = None
        if len(args) == 1 and isinstance(args[0], Mesh):
            self.mesh = args[0]
            _call("ofg_matrix_create_from_mesh", self.mesh._h, ctypes.byref(h))
        else:
            rp = np.ascontiguousarray(args[0], dtype=np.int64)
            ci = np.ascontiguousarray(args[1], dtype=np.int64)
            _call("ofg_matrix_create", rp.size - 1, ci.size, _ptr(rp), _ptr(ci), ctypes.byref(h))
        self._h = h
        n, nnz = ctypes.c_int64(), ctypes.c_int64()
        _call("ofg_matrix_info", self._h, ctypes.byref(n), ctypes.byref(nnz))
        self.n, self.nnz = n.value, nnz.value
        if len(args) >= 3 and args[2] is not None:
            self.set_values(args[2])

    def size(self):
        return self.n

    def getNbRows(self):
        return self.n

    def getLength(self):
        return self.nnz

    def pattern(self):
        rp = np.zeros(self.n + 1, dtype=np.int64)
        ci = np.zeros(self.nnz, dtype=np.int64)
        _call("ofg_matrix_get_pattern", self._h, _ptr(rp), _ptr(ci))
        return rp, ci

    def set_values(self, a):
        a = _f64(a, self.nnz)
        _call("ofg_matrix_set_values", self._h, _ptr(a))

    def values(self):
        a = np.zeros(self.nnz)
        _call("ofg_matrix_get_values", self._h, _ptr(a))
        return a

    def clear(self):
        _call("ofg_matrix_clear", self._h)

    def Mult(self, x, y=None):
        x = _f64(x, self.n)
        if y is None:
            y = np.zeros(self.n)
        _call("ofg_spmv", self._h, _ptr(x), _ptr(y))
        return y

    def MultAdd(self, x, y):
        x = _f64(x, self.n)
        _call("ofg_spmv_add", self._h, _ptr(x), _ptr(y))
        return y

    def __mul__(self, x):
        return self.Mult(x)

    def TMult(self, x, y):
        """SpMatrix::TMult: y += A^T x (the intended product of
        SpMatrix_impl.h:760-767)."""
        x = _f64(x, self.n)
        _call("ofg_spmv_transpose_add", self._h, _ptr(x), _ptr(y))
        return y

    def edit(self, i, j, v, set_values):
        """SpMatrix::set / add for many 1-based (i, j, v), applied in order."""
        i = np.ascontiguousarray(i, dtype=np.int64).reshape(-1)
        j = np.ascontiguousarray(j, dtype=np.int64).reshape(-1)
        v = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        if not (i.size == j.size == v.size):
            raise OFELIException("index and value arrays differ in size")
        _call("ofg_matrix_edit", self._h, i.size, _ptr(i), _ptr(j), _ptr(v), 1 if set_values else 0)

    def set(self, i, j, v):
        """SpMatrix::set(i, j, v), 1-based (SpMatrix_impl.h:785-795)."""
        self.edit([i], [j], [v], True)

    def add(self, i, j, v):
        """SpMatrix::add(i, j, v), 1-based (SpMatrix_impl.h:797-802)."""
        self.edit([i], [j], [v], False)

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_matrix_destroy(self._h)
            self._h = None


class Prec:
    """Prec<real_t>(A, type): DIAG, DILU/ILU (diagonal ILU), SSOR (SGS); and
    Prec(A, LEARNED_PREC, net=LearnedNet) for the learned M = G^T G."""

    def __init__(self, A, type=DIAG_PREC, net=None):
        self.A = A
        self.type = type
        self.net = net
        h = ctypes.c_void_p()
        if type == LEARNED_PREC:
            if net is None:
                raise OFELIException("LEARNED_PREC needs a LearnedNet")
            _call("ofg_prec_create_learned", net._h, A._h, ctypes.byref(h))
        else:
            _call("ofg_prec_create", A._h, type, ctypes.byref(h))
        self._h = h

    def setMatrix(self, A=None):
        if A is not None and A is not self.A:
            self.__init__(A, self.type, self.net)
        else:
            _call("ofg_prec_update", self._h)

    def freeze(self, on=True):
        """Keep this preconditioner as it is while the matrix values change
        (the solvers then skip their refresh; setMatrix() still refreshes).
        The learned factor of a time-stepping scheme whose matrix stays the
        same from step to step is computed once this way."""
        _call("ofg_prec_freeze", self._h, 1 if on else 0)

    def solve(self, b, x=None):
        b = _f64(b, self.A.n)
        if x is None:
            x = np.zeros(self.A.n)
        _call("ofg_prec_apply", self._h, _ptr(b), _ptr(x))
        return x

    def getPivot(self):
        p = np.zeros(self.A.n)
        _call("ofg_prec_get_pivot", self._h, _ptr(p))
        return p

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_prec_destroy(self._h)
            self._h = None


def _as_prec(A, P):
    return P if isinstance(P, Prec) else Prec(A, int(P))


def CG(A, P, b, x, max_it, toler, history=False):
    """CG(A, P|prec, b, x, max_it, toler) -> iterations (negative when max_it
    was reached); x holds the initial guess and receives the solution."""
    P = _as_prec(A, P)
    b = _f64(b, A.n)
    res = ctypes.c_int()
    rr = ctypes.c_double()
    if history:
        hist = np.zeros(max_it + 1)
        _call("ofg_cg_history", P._h, _ptr(b), _ptr(x), max_it, toler, ctypes.byref(res),
              ctypes.byref(rr), _ptr(hist))
        return res.value, hist
    _call("ofg_cg", P._h, _ptr(b), _ptr(x), max_it, toler, ctypes.byref(res), ctypes.byref(rr))
    return res.value


def GMRes(A, P, b, x, m, max_it, toler):
    """GMRes(A, P|prec, b, x, m, max_it, toler) -> iterations or -iterations."""
    P = _as_prec(A, P)
    b = _f64(b, A.n)
    res = ctypes.c_int()
    rr = ctypes.c_double()
    _call("ofg_gmres", P._h, _ptr(b), _ptr(x), m, max_it, toler, ctypes.byref(res),
          ctypes.byref(rr))
    return res.value


def BiCGStab(A, P, b, x, max_it, toler):
    """BiCGStab(A, P|prec, b, x, max_it, toler) -> iterations; 2 or 3 on a
    breakdown ((rr, r) or omega vanishing); -(max_it+1) when max_it ran out."""
    P = _as_prec(A, P)
    b = _f64(b, A.n)
    res = ctypes.c_int()
    rr = ctypes.c_double()
    _call("ofg_bicgstab", P._h, _ptr(b), _ptr(x), max_it, toler, ctypes.byref(res),
          ctypes.byref(rr))
    return res.value


def solve_mixed(A, b, x, prec=DIAG_PREC, inner_bits=32, toler=1e-10, max_outer=200,
                max_inner=1000000, inner_tol=0.05, mode=0):
    """FP64 iterative refinement around an FP32 (or BF16-matrix) PCG; mode 0
    keeps the CG direction across refinements, mode 1 restarts the inner CG.
    inner_bits 0 takes BF16 matrix values when every value of A is exact in
    BF16 and FP32 values otherwise.  Returns (refinement steps, inner iterations, FP64 true relative residual)."""
    b = _f64(b, A.n)
    o, i, r = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    _call("ofg_solve_mixed", A._h, prec, inner_bits, mode, _ptr(b), _ptr(x), max_outer,
          max_inner, inner_tol, toler, ctypes.byref(o), ctypes.byref(i), ctypes.byref(r))
    return o.value, i.value, r.value


class LearnedNet:
    """The network of the learned preconditioner (4 message-passing layers of
    width 64, BF16 tensor-core layer products, FP32 master weights, Adam).
    loss 1 (default): Kaporin number of M A estimated on the pairs; loss 0:
    mean ||M r - e||^2 / ||e||^2."""

    def __init__(self, seed=1, loss=1):
        h = ctypes.c_void_p()
        _call("ofg_learned_create", ctypes.c_uint64(seed), ctypes.byref(h))
        self._h = h
        self.set_loss(loss)

    @staticmethod
    def num_params():
        return int(capi.lib().ofg_learned_num_params())

    def set_loss(self, kind):
        _call("ofg_learned_set_loss", self._h, int(kind))

    def set_tensor_cores(self, on):
        _call("ofg_learned_set_tensor_cores", self._h, 1 if on else 0)

    def get_params(self):
        """(params, adam_m, adam_v, step): a checkpoint."""
        k = self.num_params()
        p, m, v = np.zeros(k, np.float32), np.zeros(k, np.float32), np.zeros(k, np.float32)
        st = ctypes.c_int64()
        _call("ofg_learned_get_params", self._h, _ptr(p), _ptr(m), _ptr(v), ctypes.byref(st))
        return p, m, v, st.value

    def set_params(self, params, adam_m=None, adam_v=None, step=0):
        k = self.num_params()
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float32)
        params, adam_m, adam_v = f(params), f(adam_m), f(adam_v)
        if params.size != k:
            raise OFELIException("expected %d parameters" % k)
        _call("ofg_learned_set_params", self._h, _ptr(params), _ptr(adam_m), _ptr(adam_v),
              int(step))

    @staticmethod
    def _pairs(A, R, E):
        R = np.ascontiguousarray(R, dtype=np.float32) if not hasattr(R, "data_ptr") else R
        E = np.ascontiguousarray(E, dtype=np.float32) if not hasattr(E, "data_ptr") else E
        npairs = R.shape[0]
        if tuple(R.shape) != (npairs, A.n) or tuple(E.shape) != (npairs, A.n):
            raise OFELIException("pairs must be (npairs, n)")
        return R, E, npairs

    @staticmethod
    def make_pairs(A, b, npairs, seed=0, toler=1e-12):
        """Residual / error pairs from the plain solve of A x = b: the plain
        Jacobi-CG gives x*; for random starting guesses x0 (white noise ten
        times the size of x*) the pair is (r, e) = (b - A x0, x* - x0).
        Returns R, E as (npairs, n) float32 arrays."""
        n = A.n
        b = _f64(b, n)
        xs = np.zeros(n)
        it = CG(A, DIAG_PREC, b, xs, 100000, toler)
        if it < 0:
            raise OFELIException("plain solve did not converge")
        s = 10.0 * max(np.sqrt(np.mean(xs * xs)), 1e-30)
        R = np.zeros((npairs, n), np.float32)
        E = np.zeros((npairs, n), np.float32)
        for p in range(npairs):
            x0 = s * fields.normal(seed * 1000003 + p, n)
            R[p] = b - A.Mult(x0)
            E[p] = xs - x0
        return R, E

    @staticmethod
    def make_pairs_operator(A, npairs, seed=0):
        """Residual / error pairs without a solve: e_p white noise and
        r_p = A e_p, the spectrally flat errors the Kaporin objective wants
        (what make_pairs' random starting guesses give, up to the solve's
        tolerance).  Works for nonsymmetric A, where the objective fits
        G^T G to the symmetric part.  Returns R, E as (npairs, n) float32."""
        n = A.n
        R = np.zeros((npairs, n), np.float32)
        E = np.zeros((npairs, n), np.float32)
        for p in range(npairs):
            e = fields.normal(seed * 1000003 + p, n)
            R[p] = A.Mult(e)
            E[p] = e
        return R, E

    def train(self, A, R, E, steps, batch=16, lr=1e-3):
        """Adam steps on residual / error pairs (rows of R and E); returns the
        per-step batch losses."""
        R, E, npairs = self._pairs(A, R, E)
        hist = np.zeros(steps, np.float32)
        _call("ofg_learned_train", self._h, A._h, _ptr(R), _ptr(E), npairs, steps,
              min(batch, npairs), ctypes.c_float(lr), _ptr(hist))
        return hist

    def grad(self, A, R, E):
        """(loss, gradient, factor values at A's CSR positions)."""
        R, E, npairs = self._pairs(A, R, E)
        loss = ctypes.c_double()
        g = np.zeros(self.num_params(), np.float32)
        fac = np.zeros(A.nnz, np.float32)
        _call("ofg_learned_grad", self._h, A._h, _ptr(R), _ptr(E), npairs, ctypes.byref(loss),
              _ptr(g), _ptr(fac))
        return loss.value, g, fac

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_learned_destroy(self._h)
            self._h = None


def fcg_learned(P, b, x, inner_bits=32, toler=1e-10, max_outer=200, max_inner=1000000,
                inner_tol=0.05):
    """CG with the learned preconditioner (M = G^T G, one fixed linear
    operator within a solve) in FP32 inside FP64 refinement, falling back to the plain Jacobi iteration on stagnation
    (inner_bits as in solve_mixed).  Returns (refinement steps, inner iterations, FP64 true relative residual,
    fell_back)."""
    b = _f64(b, P.A.n)
    o, i, r, fb = ctypes.c_int(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
    _call("ofg_fcg_learned", P._h, inner_bits, _ptr(b), _ptr(x), max_outer, max_inner, inner_tol,
          toler, ctypes.byref(o), ctypes.byref(i), ctypes.byref(r), ctypes.byref(fb))
    return o.value, i.value, r.value, bool(fb.value)


def fgmres_mixed(P, b, x, m=30, inner_bits=0, toler=1e-10, inner_tol=1e-5, max_outer=50,
                 max_inner=100000):
    """Flexible GMRES(m), right preconditioned by P (DIAG, IDENT or the learned
    M = G^T G), with an FP32 matrix-vector product and preconditioner inside
    FP64 iterative refinement, FP64 classical Gram-Schmidt applied twice; x
    is the initial guess (warm start) and receives the solution.  Converged
    on the FP64 true residual ||b - A x|| / ||b|| <= toler.  inner_bits: 32
    (FP32 values), 16 (BF16 values) or 0 (BF16 only when every value is
    exact).  Returns (cycles, Arnoldi steps, true relative residual,
    fell_back): fell_back is True when the learned preconditioner stopped
    reducing the residual and the last cycles used the diagonal one."""
    b = _f64(b, P.A.n)
    o, i, r, fb = ctypes.c_int(), ctypes.c_int(), ctypes.c_double(), ctypes.c_int()
    _call("ofg_fgmres_mixed", P._h, inner_bits, _ptr(b), _ptr(x), m, max_outer, max_inner,
          inner_tol, toler, ctypes.byref(o), ctypes.byref(i), ctypes.byref(r), ctypes.byref(fb))
    return o.value, i.value, r.value, bool(fb.value)


class Batch:
    """Many independent P1 problems assembled and solved in one persistent
    launch (ofg_batch_*): per problem build() + CG with the diagonal
    preconditioner in FP64 + insertBC.  Inputs are concatenated in problem
    order (k per element, f and bc per node)."""

    NCONFIGS = 18

    def __init__(self, meshes):
        arr = (ctypes.c_void_p * len(meshes))(*[m._h.value for m in meshes])
        h = ctypes.c_void_p()
        _call("ofg_batch_create", len(meshes), ctypes.cast(arr, ctypes.c_void_p), ctypes.byref(h))
        self._h = h
        npb, nn, ne, nr, nnz = (ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64(),
                                ctypes.c_int64(), ctypes.c_int64())
        _call("ofg_batch_info", h, ctypes.byref(npb), ctypes.byref(nn), ctypes.byref(ne),
              ctypes.byref(nr), ctypes.byref(nnz))
        self.nprob, self.nodes, self.elements = npb.value, nn.value, ne.value
        self.rows, self.nnz = nr.value, nnz.value

    def problem_info(self):
        """Per problem (nodes, elements, rows, nonzeros) as an (nprob, 4) array."""
        out = np.zeros((self.nprob, 4), np.int64)
        v = [ctypes.c_int64() for _ in range(4)]
        for p in range(self.nprob):
            _call("ofg_batch_problem_info", self._h, p, *[ctypes.byref(x) for x in v])
            out[p] = [x.value for x in v]
        return out

    def set_inputs(self, k=None, f=None, bc=None):
        k, f, bc = _f64(k, self.elements), _f64(f, self.nodes), _f64(bc, self.nodes)
        _call("ofg_batch_set_inputs", self._h, _ptr(k), _ptr(f), _ptr(bc))

    def solve(self, max_it=100000, toler=1e-10):
        _call("ofg_batch_solve", self._h, max_it, toler)

    def results(self):
        """(nodal solutions, iterations, FP64 true relative residuals)."""
        u = np.zeros(self.nodes)
        it = np.zeros(self.nprob, np.int32)
        res = np.zeros(self.nprob)
        _call("ofg_batch_get_results", self._h, _ptr(u), _ptr(it), _ptr(res))
        return u, it, res

    def matrix(self, p, nnz, n):
        a, b = np.zeros(nnz), np.zeros(n)
        _call("ofg_batch_get_matrix", self._h, p, _ptr(a), _ptr(b))
        return a, b

    def tune(self, max_it=100000, toler=1e-10):
        """Autotuner: (chosen launch shape index, time of every shape in ms)."""
        c = ctypes.c_int()
        t = np.zeros(self.NCONFIGS, np.float32)
        _call("ofg_batch_tune", self._h, max_it, toler, ctypes.byref(c), _ptr(t))
        return c.value, t

    def set_precision(self, bits):
        """64: FP64 CG; 32: FP32 CG inside FP64 refinement (same FP64 target)."""
        _call("ofg_batch_set_precision", self._h, int(bits))

    def set_config(self, config, blocks_per_sm=0):
        _call("ofg_batch_set_config", self._h, config, blocks_per_sm)

    @staticmethod
    def config_shape(config):
        """(threads per block, lanes per CSR row, blocks per cluster)."""
        t, l, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _call("ofg_batch_config_shape", config, ctypes.byref(t), ctypes.byref(l), ctypes.byref(c))
        return t.value, l.value, c.value

    def __del__(self):
        if getattr(self, "_h", None) and capi is not None and capi._lib is not None:
            capi.lib().ofg_batch_destroy(self._h)
            self._h = None


def residual(A, b, x):
    r = ctypes.c_double()
    _call("ofg_residual", A._h, _ptr(_f64(b, A.n)), _ptr(_f64(x, A.n)), ctypes.byref(r))
    return r.value


class LinearSolver:
    """LinearSolver (src/solvers/LinearSolver.cpp): defaults max_it 1000,
    toler sqrt(eps); GMRES uses OFELI's restart length n/5."""

    def __init__(self, A=None, b=None, x=None):
        self._A, self._b, self._x = A, b, x
        self._max_it = 1000
        self._toler = math.sqrt(OFELI_EPSMCH)
        self._s, self._p = CG_SOLVER, DIAG_PREC
        self._nb_it = 0

    def setMaxIter(self, m):
        self._max_it = m

    def setTolerance(self, t):
        self._toler = t

    def setMatrix(self, A):
        self._A = A

    def setRHS(self, b):
        self._b = b

    def setSolution(self, x):
        self._x = x

    def setSolver(self, s, p):
        self._s, self._p = s, p

    def getNbIter(self):
        return self._nb_it

    def solve(self, s=None, p=None):
        if s is not None:
            self.setSolver(s, p)
        if self._A is None:
            raise OFELIException("In LinearSolver::solve(): No matrix has been defined.")
        if self._s == CG_SOLVER:
            self._nb_it = CG(self._A, self._p, self._b, self._x, self._max_it, self._toler)
        elif self._s == GMRES_SOLVER:
            self._nb_it = GMRes(self._A, self._p, self._b, self._x, max(1, self._A.n // 5),
                                self._max_it, self._toler)
        elif self._s == BICG_STAB_SOLVER:
            self._nb_it = BiCGStab(self._A, self._p, self._b, self._x, self._max_it,
                                   self._toler)
        else:
            raise OFELIException("solver %d is outside the GPU path" % self._s)
        return -self._nb_it if self._nb_it < 0 else 0


class _P1Equation:
    """Equation<...>::build() / run() for one P1 element family."""

    def __init__(self, mesh, u=None):
        self.mesh = mesh
        self.u = u
        self._A = None
        self._b = None
        self._bf = None
        self._bc = None
        self._k = None
        self._ls = LinearSolver()
        self._ls.setSolver(CG_SOLVER, DILU_PREC)

    def setSolver(self, s, p=DIAG_PREC):
        self._ls.setSolver(s, p)
        if self._A is None:
            self._A = SpMatrix(self.mesh)

    def getLinearSolver(self):
        return self._ls

    def setSource(self, f):
        self._bf = _f64(f, self.mesh.nn)

    setBodyForce = setSource

    def setDirichlet(self, bc):
        self._bc = _f64(bc, self.mesh.nn)

    setBoundaryCondition = setDirichlet

    def setElementCoefficient(self, k):
        """Per-element scale of the stiffness (conductivity), ne values."""
        self._k = _f64(k, self.mesh.ne)

    def getMatrix(self):
        return self._A

    def getRHS(self):
        return self._b

    def build(self):
        if self._A is None:
            self._A = SpMatrix(self.mesh)
        self._b = np.zeros(self._A.n)
        _call("ofg_assemble_p1", self.mesh._h, self._A._h, _ptr(self._k), _ptr(self._bf),
              _ptr(self._bc), _ptr(self._b))

    def run(self):
        self.build()
        x = np.zeros(self._A.n)
        self._ls.setMatrix(self._A)
        self._ls.setRHS(self._b)
        self._ls.setSolution(x)
        ret = self._ls.solve()
        u = np.zeros(self.mesh.nn) if self.u is None else self.u
        _call("ofg_insert_bc", self.mesh._h, _ptr(x), _ptr(self._bc), _ptr(u))
        self.u = u
        self.x = x
        return ret


class Laplace2DT3(_P1Equation):
    """Laplace2DT3: area*(grad phi_i . grad phi_j) (times the element
    coefficient), lumped source f*area/3 (src/equations/laplace/Laplace2DT3.cpp)."""


class DC3DT4(_P1Equation):
    """DC3DT4 stationary diffusion: k*vol*(grad phi_i . grad phi_j), lumped
    source f*vol/4 (src/equations/therm/DC3DT4.cpp)."""


Laplace3DT4 = DC3DT4


class DC2DT3:
    """DC2DT3 transient steps: capacity (consistent + lumped, as OFELI's
    shared CAPACITY bit gives), diffusion eps, convection by the nodal
    velocity, under backward Euler (default), forward Euler or
    Crank-Nicolson (setTransient); one build() per time step
    (include/equations/therm/Equa_Therm.h:162-218)."""

    def __init__(self, mesh, u0, v, eps, dt, scheme=BACKWARD_EULER):
        self.mesh = mesh
        self.u = _f64(u0, mesh.nn).copy()
        self.v = _f64(v, 2 * mesh.nn)
        self.eps, self.dt = eps, dt
        self.setTransient(scheme)
        self._A = SpMatrix(mesh)
        self._bc = None
        self.x = np.zeros(self._A.n)

    def setDirichlet(self, bc):
        self._bc = _f64(bc, self.mesh.nn)

    def getLinearSolver(self):
        """Equa::getLinearSolver(): the solver the time steps of a
        TimeStepping driver use (its tolerance and iteration cap)."""
        if getattr(self, "_ls", None) is None:
            self._ls = LinearSolver()
        return self._ls

    def setTransient(self, scheme):
        """Equa::setTransient: FORWARD_EULER, BACKWARD_EULER or CRANK_NICOLSON."""
        if scheme not in (FORWARD_EULER, BACKWARD_EULER, CRANK_NICOLSON):
            raise OFELIException("unsupported time scheme %r" % (scheme,))
        self.scheme = scheme

    def build(self):
        self._b = np.zeros(self._A.n)
        _call("ofg_assemble_cd2d_scheme", self.mesh._h, self._A._h, self.eps, _ptr(self.v),
              self.dt, self.scheme, _ptr(self.u), _ptr(self._bc), _ptr(self._b))
        return self._A, self._b

    def step(self, prec=ILU_PREC, m=30, max_it=1000, toler=1e-10, solver=GMRES_SOLVER):
        """One time step; the solver is GMRes(m) (default) or BiCGStab
        (BICG_STAB_SOLVER, OFELI's default for convection)."""
        self.build()
        if solver == BICG_STAB_SOLVER:
            it = BiCGStab(self._A, Prec(self._A, prec), self._b, self.x, max_it, toler)
        else:
            it = GMRes(self._A, Prec(self._A, prec), self._b, self.x, m, max_it, toler)
        _call("ofg_insert_bc", self.mesh._h, _ptr(self.x), _ptr(self._bc), _ptr(self.u))
        return it

    def step_mixed(self, prec=DIAG_PREC, net=None, m=30, toler=1e-10, inner_tol=1e-5,
                   inner_bits=0):
        """One time step with the chosen form: flexible GMRES(m) in mixed
        precision (fgmres_mixed), warm-started from the previous step,
        converged on the FP64 true residual.  prec: DIAG_PREC, or
        LEARNED_PREC with `net`, whose factor is computed on the first
        step's matrix and kept (frozen) for the later steps: with a fixed
        time step the matrix is the same at every step.  Returns (cycles,
        Arnoldi steps, FP64 true relative residual, fell_back)."""
        self.build()
        P = getattr(self, "_mixed_prec", None)
        if P is None or P.type != prec:
            P = self._mixed_prec = Prec(self._A, prec, net=net)
            if prec == LEARNED_PREC:
                P.freeze()
        out = fgmres_mixed(P, self._b, self.x, m=m, inner_bits=inner_bits, toler=toler,
                           inner_tol=inner_tol)
        _call("ofg_insert_bc", self.mesh._h, _ptr(self.x), _ptr(self._bc), _ptr(self.u))
        return out


# OFELI's HEUN and NEWMARK values (include/equations/Equa.h:124-137)
HEUN, NEWMARK = 4, 5


class TimeStepping:
    """OFELI's TimeStepping driver (src/solvers/TimeStepping.cpp) for a DC2DT3
    equation under its first-order schemes, each step on the device:

    * BACKWARD_EULER: build() of the backward-Euler system, then the
      equation's LinearSolver (getLinearSolver(): tolerance, iteration cap;
      the solver and preconditioner of setLinearSolver, GMRES restarting
      every n/5 steps) from the previous step's solution, insertBC;
    * CRANK_NICOLSON: the same with the Crank-Nicolson system;
    * FORWARD_EULER: the explicit step x = b / D, D the assembled diagonal
      (ofg_matrix_diag_solve), insertBC.

    Each element matrix and right-hand side is the one OFELI's
    AssembleBackwardEuler / AssembleCrankNicolson / AssembleForwardEuler
    builds (:635-734), which for a zero source and zero Dirichlet data are
    the Equa_Therm::build systems of setTransient, bit for bit.  As in
    OFELI, set() tests the scheme with bitwise ANDs against HEUN and
    NEWMARK (:141-170): FORWARD_EULER (1) and CRANK_NICOLSON (3) share a bit
    with NEWMARK (5), so runOneTimeStep makes two sub-steps of time_step for
    them and one for BACKWARD_EULER."""

    def __init__(self, scheme, time_step, final_time=1.0):
        if scheme not in (FORWARD_EULER, BACKWARD_EULER, CRANK_NICOLSON):
            raise OFELIException("In TimeStepping::set(...): only the first-order schemes "
                                 "(forward and backward Euler, Crank-Nicolson) are on this path")
        self.scheme, self.time_step, self.final_time = scheme, time_step, final_time
        self._nb_ssteps = 2 if (scheme & HEUN or scheme & NEWMARK) else 1
        self._eq = None
        self._s, self._p = None, None
        self._step = 0

    def setPDE(self, eq):
        if not isinstance(eq, DC2DT3):
            raise OFELIException("TimeStepping drives a DC2DT3 equation on this path")
        self._eq = eq
        eq.dt = self.time_step
        eq.setTransient(self.scheme)

    def setInitial(self, u):
        self._eq.u = _f64(u, self._eq.mesh.nn).copy()

    def setBC(self, bc):
        self._eq.setDirichlet(bc)

    def setLinearSolver(self, s=GMRES_SOLVER, p=DIAG_PREC):
        self._s, self._p = s, p

    def runOneTimeStep(self):
        """One time step (the scheme's sub-steps); returns the time step."""
        eq = self._eq
        if eq is None:
            raise OFELIException("TimeStepping: no equation (setPDE)")
        if eq._bc is None:
            eq.setDirichlet(np.zeros(eq.mesh.nn))
        self._step += 1
        ls = eq.getLinearSolver()
        for _ in range(self._nb_ssteps):
            A, b = eq.build()
            if self.scheme == FORWARD_EULER:
                _call("ofg_matrix_diag_solve", A._h, _ptr(b), _ptr(eq.x))
            else:
                ls.setMatrix(A)
                ls.setRHS(b)
                ls.setSolution(eq.x)
                ls.solve(self._s if self._s is not None else GMRES_SOLVER,
                         self._p if self._p is not None else DIAG_PREC)
            _call("ofg_insert_bc", eq.mesh._h, _ptr(eq.x), _ptr(eq._bc), _ptr(eq.u))
        return self.time_step

    def run(self):
        """Steps until final_time (TimeStepping::run)."""
        t = 0.0
        while t < self.final_time - 0.5 * self.time_step:
            self.runOneTimeStep()
            t += self.time_step

    def getSolution(self):
        return self._eq.u

"""ofg_cg_diag_noalloc: the Jacobi-preconditioned CG for callers that cannot
allocate device memory while running (pre-reserved memory budgets, host
frameworks that own the allocator).  Its scratch is a fixed array inside the
library; the test checks it against the allocating entry point (ofg_cg with
a DIAG preconditioner) on two calls in a row, with the solution tolerance
and iteration band the other parity tests use, and checks that those calls
change neither the device's free memory nor its default memory pool."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden, rel_err
from ofeli_b200 import capi
from ofeli_b200 import ofeli as F

pytestmark = pytest.mark.gpu

_POOL_RESERVED, _POOL_USED = 5, 7  # CU_MEMPOOL_ATTR_{RESERVED,USED}_MEM_CURRENT


def _memory_state():
    """(free device bytes, default pool reserved bytes, default pool used
    bytes) of device 0, read through the driver API."""
    import torch
    cu = ctypes.CDLL("libcuda.so.1")
    dev = ctypes.c_int()
    assert cu.cuDeviceGet(ctypes.byref(dev), 0) == 0
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), dev) == 0
    state = [torch.cuda.mem_get_info(0)[0]]
    for attr in (_POOL_RESERVED, _POOL_USED):
        v = ctypes.c_uint64()
        assert cu.cuMemPoolGetAttribute(pool, attr, ctypes.byref(v)) == 0
        state.append(v.value)
    return tuple(state)


def _device_system(cuda, g):
    import torch
    rp = torch.from_numpy(g["row_ptr"].astype(np.int32)).to(cuda)
    col = torch.from_numpy(g["col_ind"].astype(np.int32) - 1).to(cuda)
    val = torch.from_numpy(g["a"]).to(cuda)
    b = torch.from_numpy(g["b"]).to(cuda)
    return rp, col, val, b


def test_noalloc_cg_matches_allocating_cg(cuda):
    import torch
    g, info = load_golden("p2d_65")
    n = int(info["n"])
    rp, col, val, b = _device_system(cuda, g)

    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    x_ref = np.zeros(n)
    it_ref = F.CG(A, F.Prec(A, F.DIAG_PREC), g["b"], x_ref, 20000, 1e-10)

    # everything the calls read or write exists before the no-allocation phase
    capi.call("ofg_init", 0)
    xs = [torch.zeros(n, dtype=torch.float64, device=cuda) for _ in range(2)]
    its = [ctypes.c_int() for _ in range(2)]
    ress = [ctypes.c_double() for _ in range(2)]
    torch.cuda.synchronize()
    before = _memory_state()
    for x, it, res in zip(xs, its, ress):  # the shared scratch keeps the last call's contents
        capi.call("ofg_cg_diag_noalloc", n, F._ptr(rp), F._ptr(col), F._ptr(val), F._ptr(b),
                  F._ptr(x), 20000, 1e-10, ctypes.byref(it), ctypes.byref(res))
    torch.cuda.synchronize()
    assert _memory_state() == before, "a no-allocation solve changed the device's memory"
    for x, it, res in zip(xs, its, ress):
        assert abs(it.value - it_ref) <= 2
        assert abs(it.value - info["runs"]["CG_DIAG"]["iters"]) <= 2
        assert res.value <= 1e-10
        assert rel_err(x.cpu().numpy(), x_ref) <= 1e-12


def test_noalloc_missing_diagonal_is_a_pivot_error(cuda):
    import torch
    g, info = load_golden("p2d_65")
    n = int(info["n"])
    rp_h, ci_h, a_h = g["row_ptr"].astype(np.int64), g["col_ind"].astype(np.int64), g["a"].copy()
    # row 17 loses its diagonal entry: the pattern keeps every other entry
    r = 17
    k = rp_h[r] + int(np.nonzero(ci_h[rp_h[r]:rp_h[r + 1]] - 1 == r)[0][0])
    ci2 = np.delete(ci_h, k)
    a2 = np.delete(a_h, k)
    rp2 = rp_h.copy()
    rp2[r + 1:] -= 1
    rp, col, val, b = _device_system(cuda, {"row_ptr": rp2, "col_ind": ci2, "a": a2, "b": g["b"]})
    for bad_val in (None, np.nan):  # missing, then present but NaN (row 23)
        if bad_val is not None:
            a3 = a_h.copy()
            a3[rp_h[23] + int(np.nonzero(ci_h[rp_h[23]:rp_h[23 + 1]] - 1 == 23)[0][0])] = bad_val
            rp, col, val, b = _device_system(cuda, {"row_ptr": rp_h, "col_ind": ci_h, "a": a3,
                                                    "b": g["b"]})
        x = torch.full((n,), 0.25, dtype=torch.float64, device=cuda)
        it, res = ctypes.c_int(), ctypes.c_double()
        status = capi.lib().ofg_cg_diag_noalloc(n, F._ptr(rp), F._ptr(col), F._ptr(val),
                                                 F._ptr(b), F._ptr(x), 100, 1e-10,
                                                 ctypes.byref(it), ctypes.byref(res))
        assert status == -3  # OFG_ERR_PIVOT
        assert b"diagonal" in capi.lib().ofg_last_error()
        assert bool((x == 0.25).all()), "x changed on the error path"


def test_noalloc_rejects_oversized_systems(cuda):
    import torch
    n = (1 << 17) + 1
    rp = torch.zeros(n + 1, dtype=torch.int32, device=cuda)
    buf = torch.zeros(4, dtype=torch.float64, device=cuda)
    it, res = ctypes.c_int(), ctypes.c_double()
    status = capi.lib().ofg_cg_diag_noalloc(n, F._ptr(rp), F._ptr(rp), F._ptr(buf), F._ptr(buf),
                                             F._ptr(buf), 10, 1e-10, ctypes.byref(it),
                                             ctypes.byref(res))
    assert status == -8  # OFG_ERR_SIZE, nothing launched
    assert b"131072" in capi.lib().ofg_last_error()

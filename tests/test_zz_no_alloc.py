"""ofg_cg_diag_noalloc: the Jacobi-preconditioned CG for callers that cannot
allocate device memory while running (pre-reserved memory budgets, host
frameworks that own the allocator).  Its scratch is a fixed array inside the
library; the test checks it against the allocating entry point (ofg_cg with
a DIAG preconditioner) on two calls in a row, with the solution tolerance
and iteration band the other parity tests use."""
import ctypes

import numpy as np
import pytest

from conftest import load_golden, rel_err
from ofeli_b200 import capi
from ofeli_b200 import ofeli as F

pytestmark = pytest.mark.gpu


def test_noalloc_cg_matches_allocating_cg(cuda):
    import torch
    g, info = load_golden("p2d_65")
    n = int(info["n"])
    rp = torch.from_numpy(g["row_ptr"].astype(np.int32)).to(cuda)
    col = torch.from_numpy(g["col_ind"].astype(np.int32) - 1).to(cuda)
    val = torch.from_numpy(g["a"]).to(cuda)
    b = torch.from_numpy(g["b"]).to(cuda)

    A = F.SpMatrix(g["row_ptr"], g["col_ind"], g["a"])
    x_ref = np.zeros(n)
    it_ref = F.CG(A, F.Prec(A, F.DIAG_PREC), g["b"], x_ref, 20000, 1e-10)

    for _ in range(2):  # the shared scratch keeps the previous call's contents
        x = torch.zeros(n, dtype=torch.float64, device=cuda)
        it, res = ctypes.c_int(), ctypes.c_double()
        torch.cuda.synchronize()
        capi.call("ofg_cg_diag_noalloc", n, F._ptr(rp), F._ptr(col), F._ptr(val), F._ptr(b),
                  F._ptr(x), 20000, 1e-10, ctypes.byref(it), ctypes.byref(res))
        assert abs(it.value - it_ref) <= 2
        assert abs(it.value - info["runs"]["CG_DIAG"]["iters"]) <= 2
        assert res.value <= 1e-10
        assert rel_err(x.cpu().numpy(), x_ref) <= 1e-12


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

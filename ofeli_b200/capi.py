"""ctypes binding of libofeli_gpu.so (the C ABI declared in include/ofeli_gpu.h).

Loading fails loudly when the library is missing or was built for another
architecture: there is no CPU fallback.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libofeli_gpu.so")

OFG_OK = 0
IDENT, DIAG, DILU, ILU, SSOR = 0, 1, 2, 3, 4
PREC = {"IDENT": IDENT, "DIAG": DIAG, "DILU": DILU, "ILU": ILU, "SSOR": SSOR}

ERRORS = {-1: "OFG_ERR_ARG", -2: "OFG_ERR_CUDA", -3: "OFG_ERR_PIVOT", -4: "OFG_ERR_JACOBIAN",
          -5: "OFG_ERR_PATTERN", -6: "OFG_ERR_TIMEOUT", -7: "OFG_ERR_NOMEM", -8: "OFG_ERR_SIZE"}

_p = ctypes.c_void_p
_pp = ctypes.POINTER(ctypes.c_void_p)
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_d = ctypes.c_double
_pi64 = ctypes.POINTER(ctypes.c_int64)
_pi32 = ctypes.POINTER(ctypes.c_int)
_pd = ctypes.POINTER(ctypes.c_double)

# name -> (restype, argtypes); every function returns an int status unless noted
SIGNATURES = {
    "ofg_last_error": (ctypes.c_char_p, []),
    "ofg_version": (ctypes.c_char_p, []),
    "ofg_set_stream": (_i32, [_p]),
    "ofg_get_stream": (_p, []),
    "ofg_launch_count": (_i64, []),
    "ofg_init": (_i32, [_i32]),
    "ofg_shutdown": (_i32, []),
    "ofg_selftest_wait": (_i32, []),
    "ofg_profile_enable": (_i32, [_i32]),
    "ofg_profile_read": (_i32, [ctypes.c_char_p, _pi64, _pd, _pd]),
    "ofg_matrix_create": (_i32, [_i64, _i64, _p, _p, _pp]),
    "ofg_matrix_destroy": (_i32, [_p]),
    "ofg_spmv_transpose_add": (_i32, [_p, _p, _p]),
    "ofg_matrix_diag_solve": (_i32, [_p, _p, _p]),
    "ofg_matrix_edit": (_i32, [_p, _i64, _p, _p, _p, _i32]),
    "ofg_matrix_info": (_i32, [_p, _pi64, _pi64]),
    "ofg_matrix_get_pattern": (_i32, [_p, _p, _p]),
    "ofg_matrix_set_values": (_i32, [_p, _p]),
    "ofg_matrix_get_values": (_i32, [_p, _p]),
    "ofg_matrix_device_arrays": (_i32, [_p, _pp, _pp, _pp]),
    "ofg_matrix_clear": (_i32, [_p]),
    "ofg_spmv": (_i32, [_p, _p, _p]),
    "ofg_spmv_add": (_i32, [_p, _p, _p]),
    "ofg_spmv_device": (_i32, [_p, _i32, _p, _p]),
    "ofg_spmv32_device": (_i32, [_p, _i32, _i32, _p, _p]),
    "ofg_mesh_create_rect": (_i32, [_d, _d, _d, _d, _i64, _i64, _i32, _i32, _i32, _i32, _pp]),
    "ofg_mesh_create_kuhn": (_i32, [_i64, _pp]),
    "ofg_mesh_create": (_i32, [_i32, _i64, _p, _i64, _p, _p, _pp]),
    "ofg_mesh_destroy": (_i32, [_p]),
    "ofg_mesh_info": (_i32, [_p, _pi32, _pi64, _pi64, _pi64]),
    "ofg_mesh_get": (_i32, [_p, _p, _p, _p, _p]),
    "ofg_mesh_set_coords": (_i32, [_p, _p]),
    "ofg_matrix_create_from_mesh": (_i32, [_p, _pp]),
    "ofg_assemble_p1": (_i32, [_p, _p, _p, _p, _p, _p]),
    "ofg_assemble_cd2d": (_i32, [_p, _p, _d, _p, _d, _p, _p, _p]),
    "ofg_assemble_cd2d_scheme": (_i32, [_p, _p, _d, _p, _d, _i32, _p, _p, _p]),
    "ofg_insert_bc": (_i32, [_p, _p, _p, _p]),
    "ofg_mesh_file_read": (_i32, [ctypes.c_char_p, _pp]),
    "ofg_mesh_file_write": (_i32, [_p, ctypes.c_char_p]),
    "ofg_mesh_file_create": (_i32, [_i32, _i32, _i64, _p, _p, _i32, _i32, _i64, _p, _p, _i32, _i32,
                                    _i64, _p, _p, _pp]),
    "ofg_mesh_file_from_mesh": (_i32, [_p, _pp]),
    "ofg_mesh_file_info": (_i32, [_p, _pi32, _pi32, _pi64, _pi32, _pi32, _pi64, _pi32, _pi32, _pi64]),
    "ofg_mesh_file_get": (_i32, [_p, _p, _p, _p, _p, _p, _p]),
    "ofg_mesh_file_destroy": (_i32, [_p]),
    "ofg_mesh_file_set_threads": (_i32, [_i32]),
    "ofg_mesh_create_from_file": (_i32, [_p, _pp]),
    "ofg_mesh_read": (_i32, [ctypes.c_char_p, _pp]),
    "ofg_prec_create": (_i32, [_p, _i32, _pp]),
    "ofg_prec_destroy": (_i32, [_p]),
    "ofg_prec_update": (_i32, [_p]),
    "ofg_prec_apply": (_i32, [_p, _p, _p]),
    "ofg_prec_get_pivot": (_i32, [_p, _p]),
    "ofg_cg": (_i32, [_p, _p, _p, _i32, _d, _pi32, _pd]),
    "ofg_cg_history": (_i32, [_p, _p, _p, _i32, _d, _pi32, _pd, _p]),
    "ofg_gmres": (_i32, [_p, _p, _p, _i32, _i32, _d, _pi32, _pd]),
    "ofg_bicgstab": (_i32, [_p, _p, _p, _i32, _d, _pi32, _pd]),
    "ofg_solve_mixed": (_i32, [_p, _i32, _i32, _i32, _p, _p, _i32, _i32, _d, _d, _pi32, _pi32,
                               _pd]),
    "ofg_residual": (_i32, [_p, _p, _p, _pd]),
    "ofg_cg_diag_noalloc": (_i32, [_i64, _p, _p, _p, _p, _p, _i32, _d, _pi32, _pd]),
    "ofg_learned_create": (_i32, [ctypes.c_uint64, _pp]),
    "ofg_learned_destroy": (_i32, [_p]),
    "ofg_learned_num_params": (_i32, []),
    "ofg_learned_get_params": (_i32, [_p, _p, _p, _p, _pi64]),
    "ofg_learned_set_params": (_i32, [_p, _p, _p, _p, _i64]),
    "ofg_learned_set_tensor_cores": (_i32, [_p, _i32]),
    "ofg_learned_set_loss": (_i32, [_p, _i32]),
    "ofg_learned_train": (_i32, [_p, _p, _p, _p, _i32, _i32, _i32, ctypes.c_float, _p]),
    "ofg_learned_grad": (_i32, [_p, _p, _p, _p, _i32, _pd, _p, _p]),
    "ofg_learned_gemm_check": (_i32, [_p, _i32, _i64, _p, _p, _p]),
    "ofg_prec_create_learned": (_i32, [_p, _p, _pp]),
    "ofg_fcg_learned": (_i32, [_p, _i32, _p, _p, _i32, _i32, _d, _d, _pi32, _pi32, _pd, _pi32]),
    "ofg_fgmres_mixed": (_i32, [_p, _i32, _p, _p, _i32, _i32, _i32, _d, _d, _pi32, _pi32, _pd,
                                _pi32]),
    "ofg_prec_freeze": (_i32, [_p, _i32]),
    "ofg_batch_create": (_i32, [_i32, _p, _pp]),
    "ofg_batch_destroy": (_i32, [_p]),
    "ofg_batch_info": (_i32, [_p, _pi32, _pi64, _pi64, _pi64, _pi64]),
    "ofg_batch_problem_info": (_i32, [_p, _i32, _pi64, _pi64, _pi64, _pi64]),
    "ofg_batch_set_inputs": (_i32, [_p, _p, _p, _p]),
    "ofg_batch_solve": (_i32, [_p, _i32, _d]),
    "ofg_batch_get_results": (_i32, [_p, _p, _p, _p]),
    "ofg_batch_get_matrix": (_i32, [_p, _i32, _p, _p]),
    "ofg_batch_tune": (_i32, [_p, _i32, _d, _pi32, _p]),
    "ofg_batch_set_config": (_i32, [_p, _i32, _i32]),
    "ofg_batch_set_precision": (_i32, [_p, _i32]),
    "ofg_batch_config_shape": (_i32, [_i32, _pi32, _pi32, _pi32]),
}

_lib = None


class OFGError(RuntimeError):
    """A non-zero status from libofeli_gpu (OFELIException in OFELI)."""

    def __init__(self, fn, code, msg):
        super().__init__("%s failed (%s): %s" % (fn, ERRORS.get(code, code), msg))
        self.code = code


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libofeli_gpu.so is not built (run __graft_entry__.build() or "
                               "python -m ofeli_b200.build): no CPU fallback exists")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(SIGNATURES)


def check(fn, status):
    if status != OFG_OK:
        msg = lib().ofg_last_error()
        raise OFGError(fn, status, msg.decode() if msg else "")


def call(name, *args):
    check(name, getattr(lib(), name)(*args))


def launch_count():
    return int(lib().ofg_launch_count())


def profile_enable(on=True):
    call("ofg_profile_enable", 1 if on else 0)


def profile_read(family):
    """(launches, total ms, algorithmic bytes) of a kernel family."""
    n, ms, b = ctypes.c_int64(), ctypes.c_double(), ctypes.c_double()
    call("ofg_profile_read", family.encode(), ctypes.byref(n), ctypes.byref(ms), ctypes.byref(b))
    return n.value, ms.value, b.value

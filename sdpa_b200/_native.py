"""ctypes binding of the C ABI in include/sdpa_b200.h (libsdpa_b200.so).

The library is loaded from sdpa_b200/_lib/ only; there is no fallback: if the
shared object is missing every solver entry point raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_longlong, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libsdpa_b200.so")

# status codes
OK, EINVAL, ECUDA, ESIZE, ENODEV, ESTATE, EIO = 0, -1, -2, -3, -4, -5, -6
PREC_FP64, PREC_MIXED, PREC_MIXED_SIMT = 0, 1, 2
PHASES = ["noINFO", "pFEAS", "dFEAS", "pdFEAS", "pdINF", "pFEAS_dINF", "pINF_dFEAS", "pdOPT",
          "pUNBD", "dUNBD"]


class Params(ctypes.Structure):
    _fields_ = [("maxIteration", c_int), ("epsilonStar", c_double), ("lambdaStar", c_double),
                ("omegaStar", c_double), ("lowerBound", c_double), ("upperBound", c_double),
                ("betaStar", c_double), ("betaBar", c_double), ("gammaStar", c_double),
                ("epsilonDash", c_double)]


class Batch(ctypes.Structure):
    _fields_ = [("count", c_int), ("nmax", c_int), ("mmax", c_int), ("n", c_void_p), ("m", c_void_p),
                ("vec_off", c_void_p), ("b", c_void_p), ("mat_off", c_void_p), ("mat_ptr", c_void_p),
                ("row", c_void_p), ("col", c_void_p), ("val", c_void_p), ("dense_off", c_void_p),
                ("nblock", c_void_p), ("blk_off", c_void_p), ("blk_size", c_void_p)]


BATCH_MAX_BLOCKS = 64


class BatchInit(ctypes.Structure):
    _fields_ = [("flag", c_void_p), ("xvec", c_void_p), ("X", c_void_p), ("Y", c_void_p),
                ("init_margin", c_double), ("V", c_void_p), ("rank", c_int), ("init_mu", c_double)]


class GraphBatch(ctypes.Structure):
    _fields_ = [("num_nodes", c_int), ("num_edges", c_longlong), ("rowptr", c_void_p), ("col", c_void_p),
                ("aval", c_void_p), ("aval_t", c_void_p), ("feat", c_void_p), ("mask_count", c_int)]


class BatchResult(ctypes.Structure):
    _fields_ = [("xvec", c_void_p), ("X", c_void_p), ("Y", c_void_p), ("primal_obj", c_void_p),
                ("dual_obj", c_void_p), ("mu", c_void_p), ("primal_error", c_void_p),
                ("dual_error", c_void_p), ("iterations", c_void_p), ("phase", c_void_p),
                ("status", c_void_p)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("precision", c_int), ("ctas_per_sm", c_int), ("mixed_switch_gap", c_double),
                ("staging_doubles", c_int), ("mixed_products", c_int), ("block_threads", c_int),
                ("refine_tol", c_double), ("factor_smem", c_int)]


class SdpaInfo(ctypes.Structure):
    _fields_ = [("primal_obj", c_double), ("dual_obj", c_double), ("primal_error", c_double),
                ("dual_error", c_double), ("mu", c_double), ("duality_gap", c_double),
                ("solve_seconds", c_double), ("iterations", c_int), ("phase", c_int), ("m", c_int),
                ("nblock", c_int)]


# (name, restype, argtypes) of every exported function of include/sdpa_b200.h
SIGNATURES = [
    ("sdpab_default_params", c_int, [c_int, POINTER(Params)]),
    ("sdpab_read_params", c_int, [c_char_p, POINTER(Params)]),
    ("sdpab_last_error", c_char_p, []),
    ("sdpab_version", c_char_p, []),
    ("sdpab_batch_solve", c_int, [POINTER(Batch), POINTER(BatchInit), POINTER(Params),
                                  POINTER(BatchConfig), POINTER(BatchResult), c_void_p, c_void_p]),
    ("sdpab_batch_solve_host", c_int, [POINTER(Batch), POINTER(BatchInit), POINTER(Params),
                                       POINTER(BatchConfig), POINTER(BatchResult)]),
    ("sdpab_batch_solve_noalloc", c_int, [POINTER(Batch), POINTER(BatchInit), POINTER(Params),
                                          POINTER(BatchResult), c_void_p, c_void_p]),
    ("sdpab_workspace_bytes", c_longlong, []),
    ("sdpab_lowrank_factor", c_int, [POINTER(Batch), c_longlong, c_int, c_int, c_double, c_longlong,
                                     ctypes.c_ulonglong, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sdpab_lowrank_default_rank", c_int, [c_int]),
    ("sdpab_mpnn_num_params", c_longlong, []),
    ("sdpab_mpnn_act_floats", c_longlong, [c_int]),
    ("sdpab_mpnn_scratch_floats", c_longlong, [c_int]),
    ("sdpab_mpnn_forward", c_int, [POINTER(GraphBatch), c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sdpab_mpnn_loss_grad", c_int, [POINTER(GraphBatch), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_void_p]),
    ("sdpab_mpnn_adam", c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, ctypes.c_float,
                                ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, c_void_p]),
    ("sdpab_mpnn_to_bf16", c_int, [c_void_p, c_void_p, c_void_p]),
    ("sdpab_mpnn_propose_x", c_int, [c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sdpab_sdpa_new", c_void_p, []),
    ("sdpab_sdpa_free", None, [c_void_p]),
    ("sdpab_sdpa_set_params", c_int, [c_void_p, POINTER(Params)]),
    ("sdpab_sdpa_read_input", c_int, [c_void_p, c_char_p, c_int]),
    ("sdpab_sdpa_read_init", c_int, [c_void_p, c_char_p, c_int]),
    ("sdpab_sdpa_read_param", c_int, [c_void_p, c_char_p]),
    ("sdpab_sdpa_input_problem", c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p, c_longlong, c_void_p,
                                         c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sdpab_sdpa_set_init", c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    ("sdpab_sdpa_set_precision", c_int, [c_void_p, c_int, c_double]),
    ("sdpab_sdpa_set_tc_wait", c_int, [c_void_p, c_longlong]),
    ("sdpab_sdpa_tc_timeouts", c_int, [c_void_p, POINTER(c_int)]),
    ("sdpab_sdpa_solve", c_int, [c_void_p]),
    ("sdpab_sdpa_info", c_int, [c_void_p, POINTER(SdpaInfo)]),
    ("sdpab_sdpa_phase_times", c_int, [c_void_p, c_void_p]),
    ("sdpab_sdpa_schur_pattern", c_int, [c_void_p, POINTER(c_int), c_void_p]),
    ("sdpab_constraint_order", c_int, [c_int, c_int, c_void_p, c_longlong, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    ("sdpab_sdpa_get_xvec", c_int, [c_void_p, c_void_p]),
    ("sdpab_sdpa_get_block", c_int, [c_void_p, c_int, c_int, c_void_p]),
    ("sdpab_sdpa_block_size", c_int, [c_void_p, c_int, POINTER(c_int), POINTER(c_int)]),
    ("sdpab_sdpa_dimacs", c_int, [c_void_p, c_void_p]),
    ("sdpab_min_eigenvalue", c_int, [c_int, c_void_p, POINTER(c_double), c_void_p]),
    ("sdpab_sdpa_write_init", c_int, [c_void_p, c_char_p]),
    ("sdpab_sdpa_copy_current_to_init", c_int, [c_void_p]),
    ("sdpab_release_workspace", c_int, []),
    ("sdpab_tc_syrk_work_bytes", c_longlong, [c_int, c_int]),
    ("sdpab_tc_syrk", c_int, [c_int, c_int, c_void_p, c_int, c_void_p, c_int, c_void_p, c_longlong, c_void_p]),
    ("sdpab_tc_gemm_work_bytes", c_longlong, [c_int, c_int, c_int, c_int]),
    ("sdpab_tc_gemm", c_int, [c_int, c_int, c_int, c_int, c_void_p, c_int, c_longlong, c_void_p, c_int, c_void_p,
                              c_int, c_longlong, c_void_p, c_longlong, c_void_p]),
]

_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"sdpa_b200 native library missing: {LIB_PATH} "
                               "(build it with `python -m sdpa_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class SolverError(RuntimeError):
    pass


def check(rc: int, what: str):
    if rc != OK:
        msg = lib().sdpab_last_error().decode(errors="replace")
        raise SolverError(f"{what} failed ({rc}): {msg}")


def default_params(kind: int = 0) -> Params:
    p = Params()
    check(lib().sdpab_default_params(kind, ctypes.byref(p)), "sdpab_default_params")
    return p


def read_params(path: str) -> Params:
    p = Params()
    check(lib().sdpab_read_params(path.encode(), ctypes.byref(p)), "sdpab_read_params")
    return p

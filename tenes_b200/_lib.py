"""ctypes binding of libtenes_gpu.so (include/tenes_gpu.h).

The shared library is built in-tree (``python -m tenes_b200.build``).  There
is no fallback: if the library is missing or fails to load, every entry point
raises.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtenes_gpu.so")

TG_OK, TG_E_INPUT, TG_E_LOAD, TG_E_RUNTIME, TG_E_NOCONV, TG_E_CUDA, TG_E_STATE = range(7)
STATUS_NAMES = {0: "TG_OK", 1: "TG_E_INPUT", 2: "TG_E_LOAD", 3: "TG_E_RUNTIME", 4: "TG_E_NOCONV",
                5: "TG_E_CUDA", 6: "TG_E_STATE"}

# every symbol declared in include/tenes_gpu.h
EXPORTED = [
    "tg_params_default", "tg_last_error", "tg_version", "tg_ctx_create", "tg_ctx_destroy",
    "tg_set_site_tensor", "tg_get_site_tensor", "tg_set_lambda", "tg_get_lambda", "tg_set_env",
    "tg_get_env", "tg_ctm_init", "tg_ctm_move", "tg_ctm_sweep", "tg_ctm_check_convergence",
    "tg_ctm_run", "tg_corner_spectrum", "tg_measure_onesite", "tg_measure_bond_op12",
    "tg_su_onesite", "tg_su_bond", "tg_init_tensors", "tg_sync", "tg_measure_window",
    "tg_tm_eigenvalues", "tg_kernel_launch_count", "tg_ctx_stream",
    "tg_profile_enable", "tg_profile_reset", "tg_profile_query", "tg_corner_spectra_noalloc",
    "tg_bench_gemm", "tg_gemm_host", "tg_cholqr_host", "tg_energy_grad", "tg_measure_bond_rdm", "tg_fu_params_default", "tg_fu_bond", "tg_su_fix_gauge", "tg_measure_correlation",
    "tg_projector_svd_stats", "tenes_gpu_main", "tg_su_bonds", "tg_gemm_group_host", "tg_gemm_group_stats",
]


class TGError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class LatticeDesc(C.Structure):
    _fields_ = [("LX", C.c_int), ("LY", C.c_int), ("skew", C.c_int),
                ("physical_dims", C.POINTER(C.c_int)), ("virtual_dims", C.POINTER(C.c_int))]


class WindowTerm(C.Structure):
    """tg_window_term: one product term of an energy on a window."""
    _fields_ = [("source", C.c_int), ("nrow", C.c_int), ("ncol", C.c_int), ("source_row", C.c_int),
                ("source_col", C.c_int), ("nops", C.c_int), ("op_row", C.POINTER(C.c_int)),
                ("op_col", C.POINTER(C.c_int)), ("ops", C.POINTER(C.c_double)), ("coeff", C.c_double)]


class FuParams(C.Structure):
    """tg_fu_params: full-update knobs."""
    _fields_ = [("inverse_env_cut", C.c_double), ("inverse_precision", C.c_double),
                ("convergence_epsilon", C.c_double), ("max_iteration", C.c_int), ("gauge_fix", C.c_int)]


class Params(C.Structure):
    _fields_ = [("chi", C.c_int), ("inverse_projector_cut", C.c_double),
                ("ctm_convergence_epsilon", C.c_double), ("max_ctm_iteration", C.c_int),
                ("projector_corner", C.c_int), ("use_rsvd", C.c_int),
                ("rsvd_oversampling_factor", C.c_double), ("rsvd_oversample_abs", C.c_int),
                ("rsvd_power_iters", C.c_int), ("rsvd_seed", C.c_uint64),
                ("inverse_lambda_cut", C.c_double), ("mixed", C.c_int), ("cuda_graph", C.c_int),
                ("svd_solver", C.c_int), ("density", C.c_int)]


_lib = None


def load() -> C.CDLL:
    """Load libtenes_gpu.so (raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} not built; run `python -m tenes_b200.build`")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    dp = P(C.c_double)
    vp = C.c_void_p
    sig = {
        "tg_params_default": (None, [P(Params)]),
        "tg_last_error": (C.c_char_p, []),
        "tg_version": (C.c_char_p, []),
        "tg_ctx_create": (C.c_int, [P(LatticeDesc), P(Params), C.c_int, C.c_int, P(vp)]),
        "tg_ctx_destroy": (C.c_int, [vp]),
        "tg_set_site_tensor": (C.c_int, [vp, C.c_int, dp]),
        "tg_get_site_tensor": (C.c_int, [vp, C.c_int, dp]),
        "tg_set_lambda": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_get_lambda": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_set_env": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_get_env": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_ctm_init": (C.c_int, [vp]),
        "tg_ctm_move": (C.c_int, [vp, C.c_int, C.c_int]),
        "tg_ctm_sweep": (C.c_int, [vp]),
        "tg_ctm_check_convergence": (C.c_int, [vp, P(C.c_int), dp]),
        "tg_projector_svd_stats": (C.c_int, [vp, P(C.c_int64)]),
        "tenes_gpu_main": (C.c_int, [C.c_char_p, C.c_int]),
        "tg_su_bonds": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_int), P(C.c_void_p)]),
        "tg_ctm_run": (C.c_int, [vp, C.c_int, P(C.c_int), P(C.c_int), dp]),
        "tg_corner_spectrum": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_measure_onesite": (C.c_int, [vp, C.c_int, dp, dp]),
        "tg_measure_bond_op12": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, dp, dp]),
        "tg_measure_bond_rdm": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, dp]),
        "tg_measure_correlation": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, dp, C.c_int, dp, dp]),
        "tg_su_onesite": (C.c_int, [vp, C.c_int, dp]),
        "tg_measure_window": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int),
                                        P(C.c_int), dp, dp]),
        "tg_tm_eigenvalues": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                        C.c_double, dp, P(C.c_int)]),
        "tg_su_bond": (C.c_int, [vp, C.c_int, C.c_int, dp]),
        "tg_fu_params_default": (None, [P(FuParams)]),
        "tg_fu_bond": (C.c_int, [vp, C.c_int, C.c_int, dp, P(FuParams), P(C.c_int), P(C.c_int)]),
        "tg_su_fix_gauge": (C.c_int, [vp, C.c_int, C.c_double, P(C.c_int), P(C.c_double)]),
        "tg_init_tensors": (C.c_int, [vp, C.c_int, dp, P(C.c_int), dp]),
        "tg_sync": (C.c_int, [vp]),
        "tg_kernel_launch_count": (C.c_uint64, []),
        "tg_ctx_stream": (C.c_int, [vp, P(vp)]),
        "tg_profile_enable": (C.c_int, [C.c_int]),
        "tg_profile_reset": (C.c_int, []),
        "tg_profile_query": (C.c_int, [C.c_int, P(C.c_uint64), dp, dp, dp]),
        "tg_corner_spectra_noalloc": (C.c_int, [P(vp), C.c_int, C.c_int, C.c_int, dp, vp]),
        "tg_bench_gemm": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int, C.c_int, dp]),
        "tg_gemm_host": (C.c_int, [C.c_int64, C.c_int64, C.c_int64, dp, C.c_int64, C.c_int64, dp, C.c_int64,
                                   C.c_int64, dp, C.c_int64, C.c_int64, C.c_int]),
        "tg_cholqr_host": (C.c_int, [C.c_int64, C.c_int64, dp, C.c_int, P(C.c_int)]),
        "tg_gemm_group_host": (C.c_int, [C.c_int, P(C.c_int64), P(C.c_int), C.c_int, dp, dp, dp]),
        "tg_gemm_group_stats": (C.c_int, [P(C.c_int64), P(C.c_int64), C.c_int]),
        "tg_energy_grad": (C.c_int, [vp, C.c_int, P(WindowTerm), C.c_int, C.c_int, C.c_double, dp, dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(code: int) -> None:
    if code != TG_OK:
        raise TGError(code, load().tg_last_error().decode())


def dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def as_host(a: np.ndarray, is_complex: bool) -> np.ndarray:
    """Contiguous float64 / complex128 host copy in the ABI's layout."""
    if is_complex:
        return np.ascontiguousarray(a, dtype=np.complex128)
    if np.iscomplexobj(a):
        if np.any(a.imag != 0):
            raise ValueError("complex data passed to a real context")
        a = a.real
    return np.ascontiguousarray(a, dtype=np.float64)

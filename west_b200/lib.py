"""ctypes binding of ``libwestb200.so`` (declarations in include/west_b200.h).

The library is loaded from the package directory only; there is no fallback:
if it is missing, ``load()`` raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwestb200.so")

WB_OK = 0
WB_ERR_ARG = -1
WB_ERR_CUDA = -2
WB_ERR_UNSUPPORTED = -3
WB_ERR_NOMEM = -4
WB_PRECISION_FP64 = 0
WB_PRECISION_MIXED = 1
WB_NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024

# Every symbol include/west_b200.h declares.
EXPORTS = (
    "wb_ctx_create", "wb_ctx_destroy", "wb_apply_operator", "wb_apply_operator_device",
    "wb_apply_operator_device_noalloc",
    "wb_apply_operator_multi", "wb_set_precision", "wb_set_batch", "wb_get_stats", "wb_set_profiling",
    "wb_set_graphs", "wb_get_tuning", "wb_set_autotune", "wb_davidson", "wb_davidson_set_apply", "wb_diagox",
    "wb_pdep_db_write",
    "wb_pdep_db_read", "wb_last_error", "wb_version",
)
NSTAGES = 10
STAGES = ("vloc_zinv", "vloc_plane", "vloc_zfwd", "gemm_tn", "gemm_reduce", "gemm_nn", "cg", "rhs", "drho",
          "other")

_p = ctypes.c_void_p
_i = ctypes.c_int
_d = ctypes.c_double


class WbSystem(ctypes.Structure):
    _fields_ = [
        ("npw", _i), ("npwx", _i), ("nr1", _i), ("nr2", _i), ("nr3", _i),
        ("nbnd_occ", _i), ("nkb", _i), ("n_dfpt_maxiter", _i), ("l_kinetic_only", _i), ("gstart", _i),
        ("nl", _p), ("nlm", _p), ("g2kin", _p), ("vrs", _p), ("evc", _p), ("et", _p),
        ("occupation", _p), ("vkb", _p), ("deeq", _p), ("sqvc", _p),
        ("alpha_pv", _d), ("omega", _d), ("wk", _d),
    ]


class WbStats(ctypes.Structure):
    _fields_ = [("m", _i), ("cg_iterations", _i), ("cg_active_sum", ctypes.c_longlong),
                ("fft_boxes", ctypes.c_longlong), ("launches", ctypes.c_longlong), ("ms_total", _d),
                ("stage_ms", _d * 10), ("stage_launches", ctypes.c_longlong * 10),
                ("stage_items", ctypes.c_longlong * 10), ("refinements", _i)]


class WbDavidsonParams(ctypes.Structure):
    _fields_ = [("n_pdep_eigen", _i), ("n_pdep_basis", _i), ("n_pdep_maxiter", _i),
                ("tr2_dfpt", _d), ("trev_pdep", _d), ("trev_pdep_rel", _d),
                ("n_steps_write_restart", _i), ("restart", _i), ("restart_dir", ctypes.c_char_p)]


# int (*wb_apply_fn)(void* user, int col0, int m, const double* dvg, double* dng, int ld, double tr2)
WB_APPLY_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.c_int, ctypes.c_double)


class WbDavidsonInfo(ctypes.Structure):
    _fields_ = [("dav_iter", _i), ("notcnv", _i), ("converged", _i), ("apply_calls", _i),
                ("perturbations", ctypes.c_longlong), ("seconds", _d), ("seconds_apply", _d)]


class WbTuning(ctypes.Structure):
    _fields_ = [("autotune", _i), ("tuned_fp64", _i), ("tuned_mixed", _i), ("dmma_ctas_per_sm", _i),
                ("tc_braket_ctas_per_sm", _i), ("tc_update_systems", _i), ("plane_fused_fp64", _i),
                ("plane_fused_mixed", _i), ("dmma_prefetch", _i), ("tuning_ms", ctypes.c_float)]


class WestB200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"west_b200 error {code}: {msg}")
        self.code = code


_lib = None


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the library (once) and declare argument types."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: run `python -m west_b200.build` (nvcc, sm_100a)")
    lib = ctypes.CDLL(path)
    lib.wb_ctx_create.argtypes = [ctypes.POINTER(_p), ctypes.POINTER(WbSystem), _i]
    lib.wb_ctx_destroy.argtypes = [_p]
    for name in ("wb_apply_operator", "wb_apply_operator_device", "wb_apply_operator_device_noalloc"):
        getattr(lib, name).argtypes = [_p, _i, _p, _i, _p, _i, _d, _i, _p]
    lib.wb_set_precision.argtypes = [_p, _i]
    lib.wb_set_batch.argtypes = [_p, _i]
    lib.wb_set_profiling.argtypes = [_p, _i]
    lib.wb_set_graphs.argtypes = [_p, _i]
    lib.wb_get_tuning.argtypes = [_p, ctypes.POINTER(WbTuning)]
    lib.wb_set_autotune.argtypes = [_p, _i]
    lib.wb_apply_operator_multi.argtypes = [_i, _p, _p, _p, _p, _p, _p, _d, _i, _p, _i]
    lib.wb_get_stats.argtypes = [_p, ctypes.POINTER(WbStats)]
    lib.wb_davidson_set_apply.argtypes = [_p, WB_APPLY_FN, _p]
    lib.wb_davidson.argtypes = [_p, ctypes.POINTER(WbDavidsonParams), _p, _i, _p, _p, _p, _i,
                                ctypes.POINTER(WbDavidsonInfo)]
    lib.wb_diagox.argtypes = [_p, _i, _i, _p, _i, _p, _p, _i]
    lib.wb_pdep_db_write.argtypes = [ctypes.c_char_p, _i, _p, _p, _i, _p, _p, _i, _i]
    lib.wb_pdep_db_read.argtypes = [ctypes.c_char_p, _i, _i, _p, _p, _i, _i]
    lib.wb_last_error.restype = ctypes.c_char_p
    lib.wb_last_error.argtypes = []
    lib.wb_version.argtypes = []
    for name in EXPORTS:
        if name not in ("wb_last_error",):
            getattr(lib, name).restype = _i
    _lib = lib
    return lib


def check(rc: int) -> int:
    if rc < 0:
        msg = _lib.wb_last_error().decode() if _lib is not None else ""
        raise WestB200Error(rc, msg)
    return rc

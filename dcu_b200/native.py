"""ctypes binding of libdcu_spai.so (the C ABI in include/dcu_spai.h).

Loading fails loudly when the library has not been built: there is no
Python or CPU fallback for anything this module exposes.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libdcu_spai.so")
CLI_PATH = os.path.join(_HERE, "lib", "spai_multi_dcu")
CLI_SINGLE_PATH = os.path.join(_HERE, "lib", "spai_single_dcu")

# dcu_status
OK, ERR_ARG, ERR_CUDA, ERR_ALLOC, ERR_NO_DEVICE, ERR_LIMIT = range(6)
# dcu_schedule
SCHED_BALANCED_COLUMNS, SCHED_BALANCED_NNZ = 0, 1
# dcu_precision
PREC_FP64, PREC_MIXED_FP32, PREC_MIXED_BF16, PREC_M_FP32, PREC_M_BF16 = 0, 1, 2, 3, 4
# dcu_ls_method
LS_AUTO, LS_HOUSEHOLDER, LS_NORMAL_EQ = 0, 1, 2
# dcu_tol_mode
TOL_ABS, TOL_REL = 0, 1
# dcu_solve_status
SOLVE_CONVERGED, SOLVE_MAXITER, SOLVE_BREAKDOWN = 0, 1, 2


class Options(C.Structure):
    _fields_ = [("schedule", C.c_int), ("precision", C.c_int), ("tol_mode", C.c_int), ("maxiter", C.c_int),
                ("tol", C.c_double), ("verify", C.c_int), ("col_start", C.c_int), ("col_end", C.c_int),
                ("ls_method", C.c_int)]


class BuildInfo(C.Structure):
    _fields_ = [("cols_total", C.c_int), ("cols_small", C.c_int), ("cols_large", C.c_int),
                ("cols_singular", C.c_int), ("max_nj", C.c_int), ("max_ni", C.c_int), ("ms", C.c_float),
                ("cols_staged", C.c_int), ("cols_hub", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iters", C.c_int), ("status", C.c_int), ("replacements", C.c_int), ("res", C.c_double),
                ("true_res", C.c_double), ("bnorm", C.c_double), ("ms", C.c_float), ("a_fp32", C.c_int)]


class Tuning(C.Structure):
    """dcu_tuning: launch configuration of one precision form and the autotuner's report."""
    _fields_ = [("k1_split", C.c_int), ("grid_p", C.c_int), ("grid_y", C.c_int), ("grid_py", C.c_int),
                ("grid_sz", C.c_int), ("group_max_ni", C.c_int), ("cta_max_area", C.c_int),
                ("iter_us_default", C.c_float),
                ("iter_us_tuned", C.c_float), ("build_ms_default", C.c_float), ("build_ms_tuned", C.c_float),
                ("candidates", C.c_int)]

    CONFIG = ("k1_split", "grid_p", "grid_y", "grid_py", "grid_sz", "group_max_ni", "cta_max_area")

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


_LIB = None
_vp = C.c_void_p
_i = C.c_int
_OPT = C.POINTER(Options)

# name -> (restype, argtypes): every function of include/dcu_spai.h
SIGNATURES = {
    "dcu_options_default": (None, [_OPT]),
    "dcu_spai_create": (_i, [C.POINTER(_vp), _i, _i]),
    "dcu_spai_destroy": (None, [_vp]),
    "dcu_spai_last_error": (C.c_char_p, [_vp]),
    "dcu_spai_set_stream": (_i, [_vp, _vp]),
    "dcu_spai_units": (_i, [_vp]),
    "dcu_spai_launch_count": (C.c_longlong, [_vp]),
    "dcu_spai_distribute_columns": (_i, [_vp, _i, _i, _i, _i, _vp, _vp]),
    "dcu_spai_pattern_d": (_i, [_vp, _i, _vp, _vp, _i, _i, _vp, _vp, _vp, C.c_longlong, C.POINTER(C.c_longlong)]),
    "dcu_spai_build_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _OPT, _vp, _vp, C.POINTER(BuildInfo)]),
    "dcu_spai_build_h": (_i, [_vp, _i, _i, _vp, _vp, _vp, _OPT, _vp, _vp, C.POINTER(BuildInfo)]),
    "dcu_csc_to_csr_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dcu_csc_to_csr_noalloc_d": (_i, [_i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "dcu_bicgstab_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _OPT, C.POINTER(SolveInfo)]),
    "dcu_bicgstab_h": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _OPT, C.POINTER(SolveInfo)]),
    "dcu_bicgstab_transpose_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _vp, _OPT, C.POINTER(SolveInfo)]),
    "dcu_sampled_outer_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, C.c_double, _vp]),
    "dcu_spai_solve_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _OPT, _vp, C.POINTER(BuildInfo),
                              C.POINTER(SolveInfo)]),
    "dcu_spai_solve_h": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _vp, _OPT, _vp, C.POINTER(BuildInfo),
                              C.POINTER(SolveInfo)]),
    "dcu_batch_solve_d": (_i, [_vp, _i, _vp, _i, _i, _vp, _vp, _vp, _i, _vp, _vp, _OPT, _vp, _vp, _vp,
                               C.POINTER(BuildInfo), C.POINTER(SolveInfo)]),
    "dcu_profile_iteration_kernels": (_i, [_vp, _i, C.POINTER(C.c_float), _i, C.POINTER(_i)]),
    "dcu_sell_plan_stats": (_i, [_vp, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "dcu_set_wide_prepass": (_i, [_vp, _i]),
    "dcu_set_exact_a32": (_i, [_vp, _i]),
    "dcu_tuning_default": (None, [C.POINTER(Tuning)]),
    "dcu_set_tuning": (_i, [_vp, _i, C.POINTER(Tuning)]),
    "dcu_get_tuning": (_i, [_vp, _i, C.POINTER(Tuning)]),
    "dcu_autotune_d": (_i, [_vp, _i, _i, _vp, _vp, _vp, _vp, _OPT, _i, C.POINTER(Tuning)]),
    "dcu_mtx_read": (_i, [C.c_char_p, C.POINTER(_i), C.POINTER(_i), C.POINTER(C.POINTER(_i)),
                          C.POINTER(C.POINTER(_i)), C.POINTER(C.POINTER(C.c_double))]),
    "dcu_mtx_free": (None, [_vp]),
}


def lib():
    """The loaded library; raises if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run dcu_b200.build.build() (nvcc, sm_100a) first")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def default_options(**kw) -> Options:
    o = Options()
    lib().dcu_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o

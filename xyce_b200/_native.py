"""Loader for the package's native library (libxyce_b200.so) and its C ABI (include/xyce_devload.h,
include/xyce_tia.h, include/xyce_surrogate.h, include/xyce_rf.h).

The library is built in-tree by ``xyce_b200.build.build()``. There is no fallback: if the
library is missing or was built for another architecture, loading fails with an error.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libxyce_b200.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_cpp = ctypes.POINTER(ctypes.c_char_p)


class XdFlags(ctypes.Structure):
    """Mirror of ``xd_flags`` (SolverState / DeviceOptions fields the loads read)."""

    _fields_ = [
        ("dcop", ctypes.c_int), ("init_tran", ctypes.c_int), ("newton_iter", ctypes.c_int),
        ("init_jct", ctypes.c_int), ("init_fix", ctypes.c_int), ("transient", ctypes.c_int),
        ("tranop", ctypes.c_int), ("acop", ctypes.c_int), ("voltlim", ctypes.c_int),
        ("input_op", ctypes.c_int), ("gmin", ctypes.c_double), ("pdt", ctypes.c_double),
    ]


class XdMosfetFamily(ctypes.Structure):
    _fields_ = [
        ("level", ctypes.c_int), ("n_models", ctypes.c_int), ("model_is_pmos", _ip), ("model_nparams", _ip),
        ("model_param_names", _cpp), ("model_param_values", _dp), ("n_inst", ctypes.c_int),
        ("inst_model", _ip), ("inst_nodes", _ip), ("n_inst_params", ctypes.c_int),
        ("inst_param_names", _cpp), ("inst_param_values", _dp), ("temp_c", ctypes.c_double),
        ("tnom_c", ctypes.c_double), ("inst_internal", _ip), ("inst_internal_gen", _ip),
    ]


class XdCsr(ctypes.Structure):
    _fields_ = [("n_rows", ctypes.c_int), ("rowptr", _ip), ("colind", _ip)]


class XdTiaCoef(ctypes.Structure):
    """Mirror of ``xd_tia_coef``."""

    _fields_ = [("mode", ctypes.c_int), ("qscale", ctypes.c_double), ("fscale", ctypes.c_double),
                ("inv_h", ctypes.c_double), ("hist_scale", ctypes.c_double), ("gshunt", ctypes.c_double)]


class XdGemmArgs(ctypes.Structure):
    """Mirror of ``xd_gemm_args`` (include/xyce_surrogate.h)."""

    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("M", ctypes.c_int), ("N", ctypes.c_int),
                ("K", ctypes.c_int), ("lda", ctypes.c_int), ("ldb", ctypes.c_int), ("ldc", ctypes.c_int),
                ("ldt", ctypes.c_int), ("tile_n", ctypes.c_int), ("epilogue", ctypes.c_int),
                ("C32", ctypes.c_void_p), ("bias", ctypes.c_void_p), ("Z", ctypes.c_void_p), ("H", ctypes.c_void_p),
                ("HT", ctypes.c_void_p), ("Zin", ctypes.c_void_p), ("err", ctypes.c_void_p)]


class XdMlpNet(ctypes.Structure):
    """Mirror of ``xd_mlp_net``."""

    _fields_ = [("n_in", ctypes.c_int), ("w1", ctypes.c_void_p), ("ldw1", ctypes.c_int), ("w", ctypes.c_void_p * 3),
                ("w5", ctypes.c_void_p), ("b", ctypes.c_void_p * 5)]


class XdAdamArgs(ctypes.Structure):
    _fields_ = [("lr", ctypes.c_float), ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float),
                ("bias_corr1", ctypes.c_float), ("bias_corr2", ctypes.c_float)]


# Every symbol the headers declare, with its ctypes signature.
XD_DENSE_MAX_N = 160  # include/xyce_tia.h

SIGNATURES = {
    "xd_create": (ctypes.c_int, [ctypes.POINTER(XdMosfetFamily), ctypes.POINTER(XdCsr), ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_void_p)]),
    "xd_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_last_error": (ctypes.c_char_p, []),
    "xd_num_instances": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_num_state_slots": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_num_store_slots": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_update_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdFlags), ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_load_vectors": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 4 + [ctypes.c_void_p]),
    "xd_load_matrices": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_load": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdFlags)] + [ctypes.c_void_p] * 12),
    "xd_load_abs": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 7),
    "xd_copy_stamps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_num_stage_slots": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_launches_per_load": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_eval_launch_shape": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip]),
    "xd_num_eval_variants": (ctypes.c_int, []),
    "xd_internal_nodes": (ctypes.c_int, [ctypes.POINTER(XdMosfetFamily), _ip]),
    "xd_internal_nodes_gen": (ctypes.c_int, [ctypes.POINTER(XdMosfetFamily), _ip]),
    "xd_general_stamp": (ctypes.c_int, [_ip, _ip]),
    "xd_eval_variant_info": (ctypes.c_int, [ctypes.c_int, _ip, _ip]),
    "xd_eval_variant_persistent": (ctypes.c_int, [ctypes.c_int]),
    "xd_eval_variant_split": (ctypes.c_int, [ctypes.c_int]),
    "xd_eval_variant_general": (ctypes.c_int, [ctypes.c_int]),
    "xd_get_eval_variant": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_set_eval_variant": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "xd_load_static_scratch": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdFlags)] + [ctypes.c_void_p] * 12),
    "xd_probe_fp64_fma": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "xd_load_assign": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdFlags)] + [ctypes.c_void_p] * 12),
    "xd_tia_create": (ctypes.c_int, [ctypes.POINTER(XdCsr), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "xd_tia_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_tia_combine": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdTiaCoef)] + [ctypes.c_void_p] * 17),
    "xd_pwl_create": (ctypes.c_int, [ctypes.c_int, _ip, _ip, _dp, _dp, _dp, _dp, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "xd_pwl_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_pwl_eval": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_tia_fused_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "xd_tia_fused_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_tia_load_combine": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(XdFlags), ctypes.POINTER(XdTiaCoef)] +
                            [ctypes.c_void_p] * 13 + [ctypes.c_int] + [ctypes.c_void_p] * 8),
    "xd_tia_dense_solve": (ctypes.c_int, [ctypes.c_void_p] * 8),
    "xd_tia_dense_resolve": (ctypes.c_int, [ctypes.c_void_p] * 6),
    "xd_tia_dense_solve_fallback": (ctypes.c_int, [ctypes.c_void_p] * 8),
    "xd_tia_newton_update": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                                    ctypes.c_void_p, ctypes.c_void_p]),
    "xd_tia_residual_norm": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "xd_slu_create": (ctypes.c_int, [ctypes.c_int, _ip, _ip, _dp, ctypes.c_double, ctypes.c_int,
                                     ctypes.POINTER(ctypes.c_void_p)]),
    "xd_slu_solve": (ctypes.c_int, [ctypes.c_void_p] * 7),
    "xd_slu_resolve": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "xd_slu_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_gemm_bf16": (ctypes.c_int, [ctypes.POINTER(XdGemmArgs), ctypes.c_int, ctypes.c_void_p]),
    "xd_mlp_input_layer": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "xd_mlp_input_grad": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                         ctypes.c_void_p]),
    "xd_surrogate_features": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_void_p]),
    "xd_surrogate_stage": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_load_vectors_staged": (ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_void_p] * 5 + [ctypes.c_int,
                                                                                        ctypes.c_void_p]),
    "xd_mlp_forward": (ctypes.c_int, [ctypes.POINTER(XdMlpNet), ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                      ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    "xd_rf_create": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _ip, _ip, _dp, ctypes.c_int, _ip, _ip, _dp,
                                    ctypes.c_int, _ip, _ip, _dp, _ip, _ip, ctypes.c_int,
                                    ctypes.POINTER(ctypes.c_void_p)]),
    "xd_rf_refactor": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "xd_rf_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "xd_rf_solve_library": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "xd_rf_refactor_library": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "xd_rf_stats": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, ctypes.POINTER(ctypes.c_longlong)]),
    "xd_rf_copy_factors": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "xd_rf_levels": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip]),
    "xd_rf_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "xd_mse_grad": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                   ctypes.c_void_p]),
    "xd_bias_grad": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                    ctypes.c_void_p]),
    "xd_splitk_sum": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "xd_column_sum": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_void_p]),
    "xd_adam": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_void_p, ctypes.POINTER(XdAdamArgs), ctypes.c_void_p, ctypes.c_void_p,
                               ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
}

_LIB = None


class NativeError(RuntimeError):
    pass


def library_path() -> str:
    return LIB_PATH


def load():
    """Loads libxyce_b200.so and binds every C-ABI entry point (raises if it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise NativeError(f"native library not built: {LIB_PATH} (run python -c 'import xyce_b200.build as b; b.build()')")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = _LIB.xd_last_error().decode() if _LIB is not None else ""
        raise NativeError(f"{what} failed ({rc}): {msg}")

"""ctypes binding of libtdda.so (the C ABI declared in include/tdda.h).

The library is built in tree next to this file (``python build_lib.py`` in the
package root).  There is no fallback: importing the package without the
library, or calling it on a machine without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtdda.so")

TDDA_OK = 0
STATUS_NAMES = {
    0: "ok", 1: "bad argument", 2: "out of device memory", 3: "not converged", 4: "breakdown",
    5: "CUDA error", 6: "timeout", 7: "unsupported", 8: "invalid state",
}
SOLVE_STATUS = {0: "running", 1: "converged", 2: "max_iter", 3: "breakdown", 4: "nonfinite",
                5: "zero_rhs", 6: "stagnated", 7: "timeout"}

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


class Params(ctypes.Structure):
    _fields_ = [
        ("beta_min", ctypes.c_double), ("beta_max", ctypes.c_double), ("ita", ctypes.c_double),
        ("beta_type", ctypes.c_char_p),
        ("use_filter", ctypes.c_int),
        ("symmetry_type", ctypes.c_char_p),
        ("symmetry_axis", ctypes.c_double * 2),
        ("is_periodic", ctypes.c_int),
        ("objective_name", ctypes.c_char_p),
        ("obj_para", _dp),
        ("n_obj_para", ctypes.c_int),
        ("num_x", ctypes.c_int), ("num_y", ctypes.c_int), ("num_z", ctypes.c_int),
        ("num_total", ctypes.c_int),
        ("n_K", ctypes.c_double * 3),
        ("E0", ctypes.c_double),
        ("n_E0", ctypes.c_double * 3),
        ("lam", ctypes.c_double),
        ("material", ctypes.c_double * 4),
        ("nback", ctypes.c_double),
        ("MAXm", ctypes.c_int), ("MAXn", ctypes.c_int),
        ("Lm", ctypes.c_double), ("Ln", ctypes.c_double),
        ("matrix_method", ctypes.c_char_p),
        ("d", ctypes.c_double),
        ("integral_delta", ctypes.c_double),
        ("verbose", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("filter_iterations", _ip),
        ("filter_radii", _dp),
        ("n_filters", ctypes.c_int),
    ]


class AscentStep(ctypes.Structure):
    """tdda_ascent_step (include/tdda.h)."""
    _fields_ = [("penalty", ctypes.c_int), ("sigma", ctypes.c_double), ("mu", ctypes.c_double),
                ("slope", ctypes.c_double), ("coeff", ctypes.c_double), ("one_minus_coeff", ctypes.c_double),
                ("step", ctypes.c_double), ("beta1", ctypes.c_double), ("beta2", ctypes.c_double),
                ("one_minus_beta1", ctypes.c_double), ("one_minus_beta2", ctypes.c_double),
                ("bias1", ctypes.c_double), ("bias2", ctypes.c_double)]


class SolveInfo(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int),
        ("error", ctypes.c_double),
        ("status", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("inner_iterations", ctypes.c_int),
        ("true_error", ctypes.c_double),
    ]

    def as_dict(self):
        return {
            "iterations": self.iterations, "error": self.error,
            "status": SOLVE_STATUS.get(self.status, str(self.status)),
            "refinements": self.refinements, "inner_iterations": self.inner_iterations,
            "true_error": self.true_error,
        }


class ModelInfo(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("NFpara", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("Lx", ctypes.c_int), ("Ly", ctypes.c_int), ("Lz", ctypes.c_int),
        ("K", ctypes.c_double),
        ("material", ctypes.c_double * 4),
        ("device_bytes", ctypes.c_longlong),
        ("lattice_ms", ctypes.c_double), ("tensor_fft_ms", ctypes.c_double),
    ]


MAX_POL = 4  # TDDA_SERVER_MAX_POL


class ServerConfig(ctypes.Structure):
    _fields_ = [
        ("hbm_budget_bytes", ctypes.c_int64), ("workers", ctypes.c_int32), ("max_rhs", ctypes.c_int32),
        ("use_graphs", ctypes.c_int32), ("graph_steps", ctypes.c_int32),
    ]


class Request(ctypes.Structure):
    _fields_ = [
        ("num_x", ctypes.c_int32), ("num_y", ctypes.c_int32), ("num_z", ctypes.c_int32),
        ("d", ctypes.c_double), ("lam", ctypes.c_double), ("nback", ctypes.c_double), ("E0", ctypes.c_double),
        ("material", ctypes.c_double * 4),
        ("MAXm", ctypes.c_int32), ("MAXn", ctypes.c_int32),
        ("Lm", ctypes.c_double), ("Ln", ctypes.c_double),
        ("method", ctypes.c_int32),
        ("n_K", ctypes.c_double * 3),
        ("npol", ctypes.c_int32),
        ("n_E0", (ctypes.c_double * 3) * MAX_POL),
        ("rho", _dp),
        ("precision", ctypes.c_int32),
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("P_out", _dp), ("E_out", _dp),
    ]


class RequestResult(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int32),
        ("info", SolveInfo * MAX_POL),
        ("batch_rhs", ctypes.c_int32), ("batch_requests", ctypes.c_int32), ("cache_hit", ctypes.c_int32),
        ("worker", ctypes.c_int32),
        ("queue_ms", ctypes.c_double), ("build_ms", ctypes.c_double), ("solve_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
    ]


class ServerStats(ctypes.Structure):
    _fields_ = [
        ("submitted", ctypes.c_int64), ("completed", ctypes.c_int64), ("failed", ctypes.c_int64),
        ("cache_hits", ctypes.c_int64), ("cache_misses", ctypes.c_int64), ("evictions", ctypes.c_int64),
        ("batches", ctypes.c_int64), ("merged_requests", ctypes.c_int64),
        ("bytes_in_use", ctypes.c_int64), ("peak_bytes", ctypes.c_int64), ("cached_tensors", ctypes.c_int64),
        ("max_concurrent", ctypes.c_int32), ("admission_waits", ctypes.c_int32),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


# every symbol include/tdda.h declares, with its ctypes signature
SIGNATURES = {
    "tdda_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "tdda_last_error": (ctypes.c_char_p, []),
    "tdda_abi_version": (ctypes.c_int, []),
    "tdda_model_create": (ctypes.c_int, [ctypes.POINTER(Params), _ip, _dp, _dp, _dp, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "tdda_model_destroy": (None, [ctypes.c_void_p]),
    "tdda_model_get_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ModelInfo)]),
    "tdda_solve_electric_field": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, ctypes.c_double,
                                                 ctypes.POINTER(SolveInfo)]),
    "tdda_calculate_objective": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "tdda_calculate_gradients": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int64]),
    "tdda_set_parameters": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_get_parameters": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_get_parameter_map": (ctypes.c_int, [ctypes.c_void_p, _ip, ctypes.c_int64]),
    "tdda_get_dielectrics": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_get_electric_field": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_get_polarization": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_matvec": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    "tdda_matvec_c64": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    "tdda_solve_batch_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                               ctypes.c_void_p, ctypes.POINTER(SolveInfo)]),
    "tdda_matvec_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_void_p]),
    "tdda_set_densities": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_gradient_densities": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp,
                                               ctypes.c_int64, ctypes.POINTER(SolveInfo)]),
    "tdda_profile_matvec": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           _dp, _dp]),
    "tdda_kernel_launches": (ctypes.c_longlong, []),
    "tdda_lattice_offsets_device": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, ctypes.c_void_p, ctypes.c_void_p]),
    "tdda_set_precision": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tdda_set_preconditioner": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "tdda_set_time_limit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "tdda_profile_gram_schmidt": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(ctypes.c_double)]),
    "tdda_set_solver": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    "tdda_filter_update": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64, ctypes.c_int, ctypes.c_int]),
    "tdda_filter_gradients": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64, ctypes.c_int, ctypes.c_int, _dp]),
    "tdda_filter_state": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int64, _dp]),
    "tdda_set_densities_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "tdda_gradient_densities_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(SolveInfo)]),
    "tdda_patch_gradient_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(SolveInfo)]),
    "tdda_design_forward_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                                  ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "tdda_design_backward_device": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                                   ctypes.c_double, ctypes.c_double, ctypes.c_void_p,
                                                   ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                   ctypes.c_void_p]),
    "tdda_params_to_densities_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "tdda_densities_to_params_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.c_void_p]),
    "tdda_solve_electric_field_warm": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                      ctypes.POINTER(SolveInfo)]),
    "tdda_ascent_step_device": (ctypes.c_int, [ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.POINTER(AscentStep), ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "tdda_set_observation_points": (ctypes.c_int, [ctypes.c_void_p, _ip, ctypes.c_int64]),
    "tdda_observation_field": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int64]),
    "tdda_patch_objective": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "tdda_patch_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _dp, ctypes.c_int64,
                                           ctypes.POINTER(SolveInfo)]),
    "tdda_matvec_device_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_int, ctypes.c_void_p]),
    "tdda_server_create": (ctypes.c_int, [ctypes.POINTER(ServerConfig), _dp, _dp, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "tdda_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_int64)]),
    "tdda_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                        ctypes.POINTER(RequestResult)]),
    "tdda_server_reserve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_int32]),
    "tdda_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats)]),
    "tdda_server_destroy": (None, [ctypes.c_void_p]),
}

_lib = None


def load():
    """Load libtdda.so once; raise if it is missing (no CPU fallback exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libtdda.so not found at {LIB_PATH}: build the CUDA library first "
                "(python topo-dda_b200/build_lib.py)")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


class TddaError(RuntimeError):
    """A libtdda call failed; `.status` holds the tdda_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def check(status: int):
    if status != TDDA_OK:
        msg = load().tdda_last_error()
        raise TddaError(status, msg.decode() if msg else "")

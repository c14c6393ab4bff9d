"""ctypes binding of the C ABI declared in include/e3d.h (libe3d.so, built in-tree).

The library is the product: this module only marshals arguments.  A missing
library is an error; there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libe3d.so")

E3D_OK = 0
ERRORS = {
    -1: "E3D_ERR_ARG", -2: "E3D_ERR_IO", -3: "E3D_ERR_FORMAT", -4: "E3D_ERR_MESH", -5: "E3D_ERR_CUDA",
    -6: "E3D_ERR_NONFINITE", -7: "E3D_ERR_STATE", -9: "E3D_ERR_LIMIT",
}
ERRORS_BY_NAME = {v: k for k, v in ERRORS.items()}
GRAD = {"greengauss": 0, "leastsquares": 1}
LIM = {"barthjespersen": 0, "venkatakrishnan": 1}
FLUX = {"roe": 0, "ausm": 1}
FP64, FP32, FP64_FMA, FP32_DELTA = 0, 1, 2, 3
# e3d_options.renumber: a base order, optionally "+boundary_last" (cells with a ghost neighbour last)
RENUMBER = {f"{k}{suffix}": v + flag for k, v in {"none": 0, "rcm": 1, "morton": 2, "shuffle": 3}.items()
            for suffix, flag in (("", 0), ("+boundary_last", 16))}
SURROGATE_PARAMS, SURROGATE_NORM = 36232, 24


class E3DError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class DeckInfo(C.Structure):
    _fields_ = [("cfl", C.c_double), ("gamma", C.c_double), ("aoa_deg", C.c_double), ("mach", C.c_double),
                ("cmac", C.c_double), ("criterion", C.c_double), ("omega", C.c_double), ("k", C.c_double),
                ("stages", C.c_int), ("max_iter", C.c_int), ("smoothing", C.c_int), ("order", C.c_int),
                ("flux", C.c_int), ("gradient", C.c_int), ("limiter", C.c_int)]


class BlockInfo(C.Structure):
    _fields_ = [("n_real", C.c_int), ("n_all", C.c_int), ("n_faces", C.c_int), ("n_nodes", C.c_int),
                ("n_markers", C.c_int), ("n_real_boundaries", C.c_int), ("n_wall_faces", C.c_int)]


class Options(C.Structure):
    _fields_ = [("precision", C.c_int), ("carry_w0", C.c_int), ("use_graph", C.c_int), ("device", C.c_int),
                ("stream", C.c_void_p), ("hist_capacity", C.c_int), ("renumber", C.c_int)]


class IterRecord(C.Structure):
    _fields_ = [("iter", C.c_int), ("rms", C.c_double * 5), ("conv", C.c_double * 5), ("cl", C.c_double),
                ("cd", C.c_double), ("cmx", C.c_double), ("cmy", C.c_double), ("cmz", C.c_double)]


_lib = None

# (name, argtypes) of every exported entry point; tests check the header declares
# exactly these and that the library exports them.
SIGNATURES = {
    "e3d_last_error": ([], C.c_char_p),
    "e3d_version": ([], C.c_char_p),
    "e3d_default_options": ([C.POINTER(Options)], None),
    "e3d_case_load": ([C.c_char_p, C.c_char_p, C.POINTER(C.c_void_p)], C.c_int),
    "e3d_case_free": ([C.c_void_p], C.c_int),
    "e3d_case_deck": ([C.c_void_p, C.POINTER(DeckInfo)], C.c_int),
    "e3d_case_n_blocks": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "e3d_case_block_info": ([C.c_void_p, C.c_int, C.POINTER(BlockInfo)], C.c_int),
    "e3d_case_get_f64": ([C.c_void_p, C.c_int, C.c_char_p, C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "e3d_case_get_i32": ([C.c_void_p, C.c_int, C.c_char_p, C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "e3d_case_cell_order": ([C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int64], C.c_int),
    "e3d_solver_create": ([C.c_void_p, C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int),
    "e3d_solver_free": ([C.c_void_p], C.c_int),
    "e3d_solver_sync": ([C.c_void_p], C.c_int),
    "e3d_solver_device_bytes": ([C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "e3d_save_w0": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_spectral_radius": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_timestep": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_gradients": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "e3d_limiters": ([C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_double], C.c_int),
    "e3d_flux_conv": ([C.c_void_p, C.c_int, C.c_int], C.c_int),
    "e3d_flux_diss": ([C.c_void_p, C.c_int, C.c_int, C.c_double], C.c_int),
    "e3d_update_internal": ([C.c_void_p, C.c_int, C.c_double], C.c_int),
    "e3d_update_boundary": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_smooth_residual": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_halo": ([C.c_void_p], C.c_int),
    "e3d_flow_data": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_iterate": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_solve": ([C.c_void_p, C.c_int, C.c_double, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "e3d_iterate_timed": ([C.c_void_p, C.c_int, C.POINTER(C.c_double)], C.c_int),
    "e3d_state_bytes": ([C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "e3d_state_export": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_state_import": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_history_length": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "e3d_history": ([C.c_void_p, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "e3d_state_get": ([C.c_void_p, C.c_int, C.c_char_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_state_set": ([C.c_void_p, C.c_int, C.c_char_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_time_kernels": ([C.c_void_p, C.c_int, C.c_char_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                          C.POINTER(C.c_int)], C.c_int),
    "e3d_launches_per_iteration": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "e3d_batch_create": ([C.c_void_p, C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)], C.c_int),
    "e3d_batch_solve": ([C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int, C.c_void_p, C.POINTER(C.c_double)],
                        C.c_int),
    "e3d_case_count": ([C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "e3d_case_history_length": ([C.c_void_p, C.c_int, C.POINTER(C.c_int)], C.c_int),
    "e3d_case_history": ([C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p], C.c_int),
    "e3d_batch_tuning": ([C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double),
                          C.POINTER(C.c_int)], C.c_int),
    "e3d_solver_set_precision": ([C.c_void_p, C.c_int], C.c_int),
    "e3d_cell_features": ([C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_surrogate_create": ([C.c_int, C.c_uint64, C.c_double, C.POINTER(C.c_void_p)], C.c_int),
    "e3d_surrogate_free": ([C.c_void_p], C.c_int),
    "e3d_surrogate_add_solution": ([C.c_void_p, C.c_void_p], C.c_int),
    "e3d_surrogate_add_samples": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64], C.c_int),
    "e3d_surrogate_sample_count": ([C.c_void_p, C.POINTER(C.c_int64)], C.c_int),
    "e3d_surrogate_clear": ([C.c_void_p], C.c_int),
    "e3d_surrogate_train": ([C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p, C.POINTER(C.c_double)], C.c_int),
    "e3d_surrogate_gradient": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_double)],
                               C.c_int),
    "e3d_surrogate_predict": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p], C.c_int),
    "e3d_surrogate_get_params": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "e3d_surrogate_set_params": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "e3d_warm_start": ([C.c_void_p, C.c_void_p, C.POINTER(C.c_int)], C.c_int),
    "e3d_shard_first_blocks": ([C.c_int, C.c_int, C.c_void_p], C.c_int),
    "e3d_case_shard_plan": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                             C.c_void_p], C.c_int),
    "e3d_shard_create": ([C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(Options), C.POINTER(C.c_void_p)],
                         C.c_int),
    "e3d_shard_halo_counts": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "e3d_shard_pack": ([C.c_void_p, C.c_void_p], C.c_int),
    "e3d_shard_unpack": ([C.c_void_p, C.c_void_p], C.c_int),
    "e3d_shard_flow_data": ([C.c_void_p, C.c_void_p, C.c_int64, C.POINTER(C.c_int)], C.c_int),
    "e3d_shard_push_flow_data": ([C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "e3d_residual_norms_noalloc": ([C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                    C.c_void_p], C.c_int),
}


def lib():
    """Load libe3d.so once (raises when the native library has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `make -C euler3d_b200/csrc` "
                              "or __graft_entry__.build()")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != E3D_OK:
        raise E3DError(rc, lib().e3d_last_error().decode(errors="replace"))


def ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)

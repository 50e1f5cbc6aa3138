"""Loader of the in-tree CUDA library (libxmcml_b200.so) with ctypes signatures of its C-ABI.

There is no CPU fallback: if the library is missing or a CUDA call fails, the functions here
raise. The library is built by xmcml_b200.build (or __graft_entry__.build()).
"""
from __future__ import annotations

import ctypes as C
import os

from . import structs as S

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libxmcml_b200.so")

_lib = None


class XmcError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"xmcml_b200 error {status}: {msg}")
        self.status = status


def load(path: str | None = None) -> C.CDLL:
    """Load libxmcml_b200.so once (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python -m xmcml_b200.build`")
    lib = C.CDLL(p)
    P = C.POINTER
    sig = {
        "xmc_version": (C.c_int, []),
        "xmc_last_error": (C.c_char_p, []),
        "xmc_default_options": (None, [P(S.XmcOptions)]),
        "xmc_create": (C.c_int, [P(S.InputInfo), P(S.XmcOptions), P(C.c_void_p)]),
        "xmc_run": (C.c_int, [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, P(S.OutputInfo), P(S.XmcLedger)]),
        "xmc_read_tallies": (C.c_int, [C.c_void_p] + [P(C.c_uint64)] * 9),
        "xmc_cancel": (C.c_int, [C.c_void_p]),
        "xmc_read_maps": (C.c_int, [C.c_void_p, P(C.c_uint64), P(C.c_uint64)]),
        "xmc_destroy": (C.c_int, [C.c_void_p]),
        "xmc_launch": (C.c_int, [P(S.InputInfo), P(S.OutputInfo), C.c_uint64, C.c_uint64, P(S.XmcOptions),
                                 P(S.XmcLedger)]),
        "xmc_launch_omp": (C.c_int, [P(S.InputInfo), P(S.OutputInfo), P(S.MCG59), C.c_int]),
        "xmc_launch_set_options": (C.c_int, [P(S.XmcOptions)]),
        "xmc_init_output": (None, [P(S.InputInfo), P(S.OutputInfo)]),
        "xmc_free_output": (None, [P(S.OutputInfo)]),
        "xmc_parse_input_file": (C.c_bool, [C.c_char_p, P(S.InputInfo)]),
        "xmc_parse_surface_file": (C.c_bool, [C.c_char_p, P(S.InputInfo)]),
        "xmc_free_input": (None, [P(S.InputInfo)]),
        "xmc_write_output_file": (C.c_bool, [P(S.InputInfo), P(S.OutputInfo), C.c_char_p]),
        "xmc_specular_reflectance": (C.c_double, [P(S.LayerInfo)]),
        "xmc_philox4x32_10": (None, [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]),
        "xmc_layout_offsets": (C.c_int, [P(C.c_int64), C.c_int]),
        "xmc_device_philox": (C.c_int, [C.c_uint64, C.c_uint64, C.c_uint32, P(C.c_uint32)]),
        "xmc_atomic_throughput": (C.c_int, [C.c_int, C.c_uint, C.c_uint, P(C.c_double), P(C.c_double)]),
        "xmc_autotune": (C.c_int, [P(S.InputInfo), P(S.XmcOptions), C.c_uint64, P(S.XmcOptions), P(C.c_double)]),
        "xmc_generate_bvh_tree": (P(S.BVHTree), [P(S.Surface), C.c_int]),
        "xmc_free_bvh_tree": (None, [P(S.BVHTree)]),
        "xmc_debug_nearest": (C.c_int, [P(S.InputInfo), C.c_int, P(C.c_float), C.c_float, C.c_float,
                                        P(C.c_float), P(C.c_int), P(C.c_float), C.c_int]),
        "xmc_run_noalloc": (C.c_int, [P(S.InputInfo), P(S.XmcOptions), C.c_uint64, C.c_uint64, C.c_uint64,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
        "xmc_batch_validate": (C.c_int, [P(S.BatchSpec), P(S.BatchInstance), C.c_int]),
        "xmc_batch_create": (C.c_int, [P(S.BatchSpec), P(C.c_void_p)]),
        "xmc_batch_run": (C.c_int, [C.c_void_p, P(S.BatchInstance), C.c_int, P(C.c_double), P(C.c_double),
                                    P(S.BatchResult), P(C.c_double)]),
        "xmc_batch_read_tallies": (C.c_int, [C.c_void_p, C.c_int, P(C.c_uint64), P(C.c_uint64), P(C.c_uint64)]),
        "xmc_batch_set_tuning": (C.c_int, [C.c_void_p, P(S.BatchTuning)]),
        "xmc_batch_get_tuning": (C.c_int, [C.c_void_p, P(S.BatchTuning)]),
        "xmc_batch_autotune": (C.c_int, [C.c_void_p, P(S.BatchInstance), C.c_int, C.c_uint64, P(S.BatchTuning)]),
        "xmc_batch_destroy": (C.c_int, [C.c_void_p]),
        "xmc_mlp_create": (C.c_int, [P(S.MlpSpec), P(C.c_void_p)]),
        "xmc_mlp_param_count": (C.c_int64, [C.c_void_p]),
        "xmc_mlp_set_params": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "xmc_mlp_get_params": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "xmc_mlp_forward": (C.c_int, [C.c_void_p, P(C.c_float), C.c_int, P(C.c_float), P(C.c_double)]),
        "xmc_mlp_forward_timed": (C.c_int, [C.c_void_p, C.c_int, C.c_int, P(C.c_double)]),
        "xmc_mlp_gradients": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_int, P(C.c_float), P(C.c_float)]),
        "xmc_mlp_set_dataset": (C.c_int, [C.c_void_p, P(C.c_float), P(C.c_float), C.c_int]),
        "xmc_mlp_train": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                    C.c_uint64, P(C.c_float), P(C.c_double)]),
        "xmc_mlp_destroy": (C.c_int, [C.c_void_p]),
        "xmc_mlp_set_output_weights": (C.c_int, [C.c_void_p, P(C.c_float)]),
        "xmc_weight_integral_table": (C.c_int, [P(S.InputInfo), C.c_int]),
        "xmc_launch_release": (C.c_int, []),
        "xmc_gemm_bf16": (C.c_int, [P(C.c_uint16), P(C.c_uint16), C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                    P(C.c_float)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def last_error() -> str:
    return load().xmc_last_error().decode(errors="replace")


def check(status: int) -> int:
    if status != S.XMC_OK:
        raise XmcError(status, last_error())
    return status


# Exported C-ABI symbols, as declared in include/xmcml_b200.h.
EXPORTS = [
    "xmc_version", "xmc_last_error", "xmc_default_options", "xmc_create", "xmc_run", "xmc_read_tallies",
    "xmc_cancel", "xmc_read_maps", "xmc_destroy", "xmc_launch", "xmc_launch_omp", "xmc_init_output", "xmc_free_output",
    "xmc_parse_input_file", "xmc_parse_surface_file", "xmc_free_input", "xmc_write_output_file",
    "xmc_specular_reflectance", "xmc_philox4x32_10", "xmc_layout_offsets", "xmc_device_philox",
    "xmc_generate_bvh_tree", "xmc_free_bvh_tree", "xmc_debug_nearest", "xmc_run_noalloc",
    "xmc_batch_validate", "xmc_batch_create", "xmc_batch_run", "xmc_batch_read_tallies", "xmc_batch_set_tuning",
    "xmc_batch_get_tuning", "xmc_batch_autotune", "xmc_batch_destroy",
    "xmc_mlp_create", "xmc_mlp_param_count", "xmc_mlp_set_params", "xmc_mlp_get_params", "xmc_mlp_forward",
    "xmc_mlp_forward_timed", "xmc_mlp_gradients", "xmc_mlp_set_dataset", "xmc_mlp_train", "xmc_mlp_destroy",
    "xmc_mlp_set_output_weights", "xmc_weight_integral_table", "xmc_launch_release",
    "xmc_gemm_bf16", "xmc_atomic_throughput", "xmc_autotune", "xmc_launch_set_options",
]

"""Loader and prototypes of libgpuga_b200.so (the C ABI of include/gpuga.h).

The library is built in-tree (``gpuga_b200/_build``) by ``gpuga_b200.build``;
there is no fallback implementation: if it is missing, importing the bindings
raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgpuga_b200.so")
CLI_PATH = os.path.join(HERE, "_build", "gpuga")

OK = 0
ERR_IO, ERR_PARSE, ERR_UNSUPPORTED, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_NAN, ERR_ARG = -1, -2, -3, -4, -5, -6, -7, -8
ERR_BUDGET, ERR_CANCELLED, ERR_NOT_READY = -9, -10, -11
PATH_BATCHED, PATH_PLAIN64, PATH_PLAIN32 = 0, 1, 2

STATUS_NAMES = {OK: "OK", ERR_IO: "IO", ERR_PARSE: "PARSE", ERR_UNSUPPORTED: "UNSUPPORTED", ERR_OOM: "OOM",
                ERR_CUDA: "CUDA", ERR_TIMEOUT: "TIMEOUT", ERR_NAN: "NAN", ERR_ARG: "ARG", ERR_BUDGET: "BUDGET",
                ERR_CANCELLED: "CANCELLED", ERR_NOT_READY: "NOT_READY"}


class GpugaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"[{STATUS_NAMES.get(status, status)}] {message}")
        self.status = status


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("path", C.c_int), ("use_graph", C.c_int), ("nn2b_consistent", C.c_int),
                ("nn2b_r1", C.c_float), ("nn2b_r2", C.c_float), ("verbose", C.c_int), ("neighbor_cells", C.c_int),
                ("ri_self_energy", C.c_int), ("tiles", C.c_int), ("fitness_fold", C.c_int)]


FITNESS_CB = C.CFUNCTYPE(None, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_void_p)

vp = C.c_void_p
i32 = C.c_int
PROTOTYPES = {
    "gpuga_default_options": (None, [vp]),
    "gpuga_last_error": (C.c_char_p, []),
    "gpuga_version": (C.c_char_p, []),
    "gpuga_engine_create": (i32, [C.c_char_p, vp, vp]),
    "gpuga_engine_create_from_arrays": (i32, [i32, i32, C.c_float] + [vp] * 3 + [i32, i32] + [vp] * 7 + [vp, vp]),
    "gpuga_engine_destroy": (i32, [vp]),
    "gpuga_parse_inputs": (i32, [C.c_char_p, vp]),
    "gpuga_engine_info": (i32, [vp, vp]),
    "gpuga_engine_bounds": (i32, [vp, vp, vp]),
    "gpuga_engine_norms": (i32, [vp, vp]),
    "gpuga_engine_neighbors": (i32, [vp, vp, vp]),
    "gpuga_engine_neighbors_csr": (i32, [vp, vp, vp]),
    "gpuga_fitness": (i32, [vp, i32, vp, vp]),
    "gpuga_fitness_ex": (i32, [vp, i32, i32, vp, vp, vp]),
    "gpuga_fitness_device": (i32, [vp, i32, vp, vp, vp]),
    "gpuga_last_config_results": (i32, [vp, i32, vp, vp, vp]),
    "gpuga_batched_forces": (i32, [vp, i32, vp, vp]),
    "gpuga_plan_info": (i32, [vp, i32, vp, vp, i32]),
    "gpuga_plan_kernels": (i32, [vp, i32, vp]),
    "gpuga_kernel_timing": (i32, [vp, i32, i32]),
    "gpuga_calibrate_fp32": (i32, [i32, vp]),
    "gpuga_find_force64": (i32, [vp, vp, vp, vp, vp]),
    "gpuga_find_force32": (i32, [vp, vp, vp, vp, vp]),
    "gpuga_predict": (i32, [vp, C.c_char_p, vp]),
    "gpuga_decode": (i32, [vp, vp, vp]),
    "gpuga_ga_create": (i32, [vp, C.c_char_p, C.c_uint, vp]),
    "gpuga_ga_create_params": (i32, [vp, i32, i32, C.c_float, i32, C.c_uint, vp]),
    "gpuga_ga_create_host": (i32, [i32, vp, vp, i32, i32, C.c_float, i32, C.c_uint, FITNESS_CB, vp, vp]),
    "gpuga_ga_step": (i32, [vp, C.c_char_p, i32]),
    "gpuga_ga_run": (i32, [vp, C.c_char_p]),
    "gpuga_ga_advance": (i32, [vp, i32, C.c_char_p, C.c_longlong]),
    "gpuga_ga_set_device_loop": (i32, [vp, i32, i32]),
    "gpuga_ga_rank_device": (i32, [i32, i32, vp, vp, vp]),
    "gpuga_ga_state": (i32, [vp, vp, vp, vp]),
    "gpuga_ga_destroy": (i32, [vp]),
    "gpuga_potential_create": (i32, [i32, i32, vp]),
    "gpuga_potential_initialize": (i32, [vp, i32, i32]),
    "gpuga_potential_update": (i32, [vp, vp, i32]),
    "gpuga_potential_find_force": (i32, [vp, i32, i32, vp, vp, i32] + [vp] * 9),
    "gpuga_potential_destroy": (i32, [vp]),
    "gpuga_potential_find_force_noalloc": (i32, [i32, i32, vp, i32, i32, i32, vp, vp, i32] + [vp] * 9),
    "gpuga_neighbor_compute": (i32, [i32, i32, i32, vp, vp, vp, vp, C.c_float, vp, vp, vp]),
    "gpuga_server_create": (i32, [i32, C.c_double, i32, vp]),
    "gpuga_server_submit": (i32, [vp, C.c_char_p, C.c_uint, i32, vp]),
    "gpuga_server_submit_engine": (i32, [vp, vp, i32, i32, C.c_float, i32, C.c_uint, vp]),
    "gpuga_server_poll": (i32, [vp, i32, vp]),
    "gpuga_server_result": (i32, [vp, i32, vp, vp]),
    "gpuga_server_cancel": (i32, [vp, i32]),
    "gpuga_server_drain": (i32, [vp, C.c_double]),
    "gpuga_server_stats": (i32, [vp, vp, i32]),
    "gpuga_server_hold": (i32, [vp, i32]),
    "gpuga_plan_tiles": (i32, [vp, i32, vp, i32, vp]),
    "gpuga_server_destroy": (i32, [vp]),
}

_lib = None


def load():
    """Load the in-tree library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m gpuga_b200.build` (or __graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != OK:
        raise GpugaError(status, load().gpuga_last_error().decode(errors="replace"))


def exported_symbols() -> list[str]:
    return list(PROTOTYPES)

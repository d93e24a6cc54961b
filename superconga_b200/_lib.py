"""ctypes binding of libscb200.so (declared in include/scb200.h).

The library is built in-tree by superconga_b200/build.py.  Loading fails loudly
when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libscb200.so")

_c_int_p = ctypes.POINTER(ctypes.c_int)
_c_double_p = ctypes.c_void_p

# name -> (restype, argtypes); mirrors include/scb200.h.
SIGNATURES = {
    "sc_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sc_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sc_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sc_get_dims": (ctypes.c_int, [ctypes.c_void_p] + [_c_int_p] * 5),
    "sc_site_updates": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "sc_set_state": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_get_state": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_compute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _c_int_p]),
    "sc_burn_in": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _c_int_p]),
    "sc_get_results": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p, _c_double_p]),
    "sc_get_scalars": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "sc_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sc_set_state_device": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_get_state_device": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_get_frame_labels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, _c_int_p]),
    "sc_get_domain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sc_boundary_sizes": (ctypes.c_int, [ctypes.c_void_p, _c_int_p]),
    "sc_sweep_plan": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p]),
    "sc_get_boundary": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "sc_set_boundary": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "sc_boundary_initial": (ctypes.c_int, [ctypes.c_void_p]),
    "sc_angle_greens": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_double_p, _c_double_p, _c_double_p]),
    "sc_poisson": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "sc_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sc_profile_read": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                       ctypes.POINTER(ctypes.c_longlong)]),
    "sc_poisson_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, _c_int_p,
                                          ctypes.c_double, ctypes.c_int, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "sc_ldos_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]),
    "sc_ldos_dims": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p, _c_int_p]),
    "sc_ldos_energies": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, ctypes.POINTER(ctypes.c_double)]),
    "sc_ldos_begin_block": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sc_ldos_iterate": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double), _c_int_p]),
    "sc_ldos_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_int_p, _c_int_p]),
    "sc_ldos_get": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "sc_ldos_get_device": (ctypes.c_int, [ctypes.c_void_p, _c_double_p]),
    "sc_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(ctypes.c_void_p)]),
    "sc_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sc_batch_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "sc_batch_size": (ctypes.c_int, [ctypes.c_void_p, _c_int_p]),
    "sc_batch_grain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]),
    "sc_batch_compute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _c_int_p]),
    "sc_batch_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "sc_batch_set_graph": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "sc_batch_grain_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sc_batch_config": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "sc_batch_get_config": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p, _c_int_p]),
    "sc_batch_autotune": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_int_p, ctypes.POINTER(ctypes.c_double)]),
    "sc_batch_time_sweeps": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "sc_batch_launch_count": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "sc_set_external_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "sc_get_external_field": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "sc_evaluate": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "sc_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _c_double_p, _c_double_p, _c_double_p,
                                  ctypes.POINTER(ctypes.c_double)]),
    "sc_bulk_order_parameter_s_wave": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                                      ctypes.c_double, _c_double_p]),
    "sc_bulk_free_energy_s_wave": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                  _c_double_p]),
    "sc_bulk_yoshida_s_wave": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                              _c_double_p]),
    "sc_grid_extend": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_int, _c_double_p]),
    "sc_grid_resample": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _c_double_p, _c_double_p]),
    "sc_measure_fma_peak": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "sc_setup_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "sc_setup_last_error": (ctypes.c_char_p, []),
    "sc_setup_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "sc_setup_dims": (ctypes.c_int, [ctypes.c_void_p] + [_c_int_p] * 5),
    "sc_setup_energies": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_setup_frame": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, _c_int_p]),
    "sc_setup_fermi_surface": (ctypes.c_int, [ctypes.c_void_p, _c_double_p, _c_double_p]),
    "sc_setup_domain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "sc_setup_boundary_sizes": (ctypes.c_int, [ctypes.c_void_p, _c_int_p]),
    "sc_setup_filters": (ctypes.c_int, [ctypes.c_void_p, _c_int_p, _c_double_p, _c_int_p,
                                        ctypes.POINTER(ctypes.c_double)]),
    "sc_setup_site_updates": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
}

_lib = None


class EngineError(RuntimeError):
    """Error status returned by the C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load(path: str | None = None) -> ctypes.CDLL:
    """Loads libscb200.so and declares every exported function."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(
            f"{p} is missing: build it with `python superconga_b200/build.py` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, handle=None):
    if status != 0:
        msg = load().sc_last_error(handle)
        raise EngineError(status, msg.decode() if msg else "unknown error")

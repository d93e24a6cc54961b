"""superconga_b200 -- Blackwell-native SuperConga self-consistency hot path.

The engine (libscb200.so, C ABI in include/scb200.h) runs the Riccati sweep,
Green accumulation, specular boundary condition, vector-potential Poisson
solve and accelerators as CUDA kernels for sm_100a.  ``Context`` is the Python
face of one engine handle; ``LdosContext`` runs the LDOS postprocess and
``Batch`` advances many grains together.
"""
from .engine import (Batch, Context, Dims, LdosContext, Setup,  # noqa: F401
                     bulk_free_energy_s_wave, bulk_order_parameter_s_wave,
                     bulk_yoshida_s_wave)
from ._lib import EngineError, LIB_PATH, load  # noqa: F401

__all__ = ["Batch", "Context", "Dims", "LdosContext", "Setup", "bulk_order_parameter_s_wave",
           "bulk_free_energy_s_wave", "bulk_yoshida_s_wave", "EngineError", "LIB_PATH", "load"]

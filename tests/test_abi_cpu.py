"""The C ABI library loads without a GPU and exports every function that
include/scb200.h declares."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "scb200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_api():
    names = declared_functions()
    for must in ("sc_create", "sc_destroy", "sc_compute", "sc_set_state", "sc_get_results",
                 "sc_burn_in", "sc_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(engine_lib):
    lib = ctypes.CDLL(os.path.join(ROOT, "superconga_b200", "libscb200.so"))
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header(engine_lib):
    from superconga_b200 import _lib
    assert set(declared_functions()) <= set(_lib.SIGNATURES)


def test_create_without_gpu_fails_cleanly(engine_lib):
    """Without a usable GPU sc_create returns an error status and a message."""
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is present")
    from tests import configs
    import json
    h = ctypes.c_void_p()
    st = engine_lib.sc_create(json.dumps(configs.small_disc()).encode(), 0, ctypes.byref(h))
    assert st != 0
    assert engine_lib.sc_last_error(None)

"""The C ABI library loads without a GPU, exports exactly the functions that
include/scb200.h declares, and a C++ caller builds against the header alone."""
import ctypes
import os
import re
import subprocess

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


def exported_functions():
    """sc_* symbols the built library defines in its dynamic symbol table."""
    out = subprocess.run(["nm", "-D", "--defined-only",
                          os.path.join(ROOT, "superconga_b200", "libscb200.so")],
                         check=True, capture_output=True, text=True).stdout
    return sorted({ln.split()[-1] for ln in out.splitlines() if re.search(r" T sc_[a-z0-9_]+$", ln)})


def test_header_declares_every_exported_symbol(engine_lib):
    undeclared = sorted(set(exported_functions()) - set(declared_functions()))
    assert not undeclared, undeclared


# The flows of INTEGRATION.md sections 1 and 7 (iterate, then the gradient of
# the frozen-boundary free energy), written against the header only.
CALLER = r"""
#include "scb200.h"
#include <cstdio>
#include <vector>
int run(const char *json) {
  sc_ctx *ctx = nullptr;
  if (sc_create(json, SC_MODE_FP64, &ctx) != SC_OK) { std::puts(sc_last_error(nullptr)); return 1; }
  int n0, n1, na, ne, nc;
  sc_get_dims(ctx, &n0, &n1, &na, &ne, &nc);
  const size_t nn = (size_t)n0 * n0;
  std::vector<double> d(2 * nc * nn, 0.1), a(2 * nn, 0.0), beta(2 * nn, 0.0);
  std::vector<double> gd(d.size()), ga(a.size());
  double res = 0, omega = 0, gb = 0, s[11];
  int conv = 0;
  sc_set_state(ctx, d.data(), a.data());
  sc_burn_in(ctx, 2, &res, &conv);
  sc_compute(ctx, 1, &res, &conv);
  sc_get_scalars(ctx, s);
  sc_set_external_field(ctx, 0.05);
  sc_evaluate(ctx, &omega);
  sc_adjoint(ctx, 1.0, beta.data(), gd.data(), ga.data(), &gb);
  return sc_destroy(ctx);
}
int main(int argc, char **argv) { return argc > 1 ? run(argv[1]) : 0; }
"""


def test_cpp_caller_builds_against_the_header(engine_lib, tmp_path):
    src = tmp_path / "caller.cpp"
    src.write_text(CALLER)
    exe = tmp_path / "caller"
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), str(src),
                    "-o", str(exe), "-L", os.path.join(ROOT, "superconga_b200"), "-lscb200"],
                   check=True)
    assert exe.exists()


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

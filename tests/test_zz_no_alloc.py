"""The allocation-free Poisson entry point (sc_poisson_noalloc) against the
allocating one (sc_poisson), through the C ABI on the GPU.

sc_poisson_noalloc is for callers that cannot allocate device memory (a
plugin inside a framework that owns the device memory pool, a service with a
footprint fixed at start-up): every buffer is the caller's and the
intermediates live in a fixed device array of the library.  Two calls in a row
with different currents must both match sc_poisson; a lattice beyond the
array's limit must be rejected.  This file is collected last.
"""
import ctypes

import numpy as np
import pytest

from tests import configs

pytestmark = pytest.mark.gpu


def _noalloc_inputs(cfg):
    import torch
    import superconga_b200 as sb
    setup = sb.Setup(cfg)
    f, pos, scale = setup.filters()
    n0 = setup.dims.n0
    h = 1.0 / cfg["numerics"]["points_per_coherence_length"]
    n_grain = int(np.count_nonzero(setup.domain()))
    d_f = torch.tensor(f, dtype=torch.float64, device="cuda").contiguous()
    return setup, n0, d_f, np.ascontiguousarray(pos, np.int32), -(h * h) * scale, n_grain


@pytest.mark.parametrize("cfg", [configs.small_square_d(), configs.small_disc()],
                         ids=["small_square_d", "small_disc"])
def test_noalloc_matches_poisson_twice(engine_lib, cfg):
    import torch
    import superconga_b200 as sb
    torch.cuda.set_device(0)
    setup, n0, d_f, pos, factor, n_grain = _noalloc_inputs(cfg)
    ctx = sb.Context(cfg)
    dom = setup.domain() > 0
    rng = np.random.default_rng(13)
    stream = torch.cuda.current_stream()
    for call in range(2):
        j = rng.standard_normal((2, n0, n0)) * dom * (1.0 + call)
        want = ctx.poisson(j)
        d_j = torch.tensor(j, dtype=torch.float64, device="cuda").contiguous()
        d_a = torch.full((2, n0, n0), float("nan"), dtype=torch.float64, device="cuda")
        st = engine_lib.sc_poisson_noalloc(
            n0, int(d_f.shape[0]), ctypes.c_void_p(d_f.data_ptr()),
            pos.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), factor, n_grain,
            ctypes.c_void_p(d_j.data_ptr()), ctypes.c_void_p(d_a.data_ptr()),
            ctypes.c_void_p(stream.cuda_stream))
        assert st == 0
        torch.cuda.synchronize()
        got = d_a.cpu().numpy()
        assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want)), call
    ctx.close()


def test_noalloc_rejects_oversized_lattice(engine_lib):
    import torch
    torch.cuda.set_device(0)
    cfg = configs.small_square_d()
    _, n0, d_f, pos, factor, n_grain = _noalloc_inputs(cfg)
    d_j = torch.zeros((2, n0, n0), dtype=torch.float64, device="cuda")
    d_a = torch.zeros((2, n0, n0), dtype=torch.float64, device="cuda")
    st = engine_lib.sc_poisson_noalloc(
        800, int(d_f.shape[0]), ctypes.c_void_p(d_f.data_ptr()),
        pos.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), factor, n_grain,
        ctypes.c_void_p(d_j.data_ptr()), ctypes.c_void_p(d_a.data_ptr()), None)
    assert st == -4  # SC_ERR_SIZE: rejected before any work
    torch.cuda.synchronize()

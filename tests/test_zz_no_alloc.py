"""The allocation-free Poisson entry point (sc_poisson_noalloc) against the
allocating one (sc_poisson), through the C ABI on the GPU.

sc_poisson_noalloc is for callers that cannot allocate device memory (a
plugin inside a framework that owns the device memory pool, a service with a
footprint fixed at start-up): every buffer is the caller's and the
intermediates live in a fixed device array of the library.  Two calls in a row
with different currents must both match sc_poisson; a lattice beyond the
array's limit (n0 = 724) must be rejected, the limit itself accepted.  This
file is collected last.
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


def _disc_with_n0(n0: int) -> dict:
    """A disc whose lattice is exactly n0 (2R * 8 points/xi0 = n0 - 6, exact in
    binary), four angles; only its Poisson filters and solve are used."""
    cfg = configs.disc_n256()
    cfg["geometry"][0]["disc"]["radius"] = (n0 - 6) / 16.0
    cfg["numerics"]["points_per_coherence_length"] = 8.0
    return cfg


def _call(lib, n0, d_f, pos, factor, n_grain, d_j, d_a, stream=None):
    return lib.sc_poisson_noalloc(
        n0, int(d_f.shape[0]), ctypes.c_void_p(d_f.data_ptr()),
        pos.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), factor, n_grain,
        ctypes.c_void_p(d_j.data_ptr()), ctypes.c_void_p(d_a.data_ptr()),
        None if stream is None else ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_largest_lattice_matches_poisson(engine_lib):
    """n0 = 724 is the largest lattice the fixed array holds (128 + 6 n0^2
    doubles of 24 MiB): accepted, and equal to sc_poisson at that size."""
    import torch
    import superconga_b200 as sb
    torch.cuda.set_device(0)
    cfg = _disc_with_n0(724)
    setup, n0, d_f, pos, factor, n_grain = _noalloc_inputs(cfg)
    assert n0 == 724
    ctx = sb.Context(cfg)
    dom = setup.domain() > 0
    j = np.random.default_rng(29).standard_normal((2, n0, n0)) * dom
    want = ctx.poisson(j)
    d_j = torch.tensor(j, dtype=torch.float64, device="cuda").contiguous()
    d_a = torch.full((2, n0, n0), float("nan"), dtype=torch.float64, device="cuda")
    assert _call(engine_lib, n0, d_f, pos, factor, n_grain, d_j, d_a, torch.cuda.current_stream()) == 0
    torch.cuda.synchronize()
    got = d_a.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-10 * np.max(np.abs(want))
    ctx.close()


@pytest.mark.parametrize("n0", [725, 800])
def test_noalloc_rejects_oversized_lattice(engine_lib, n0):
    """One site past the limit (n0 = 725) and far past it: SC_ERR_SIZE before
    any work, with the caller's buffers untouched."""
    import torch
    torch.cuda.set_device(0)
    cfg = configs.small_square_d()
    _, small, d_f, pos, factor, n_grain = _noalloc_inputs(cfg)
    d_j = torch.zeros((2, small, small), dtype=torch.float64, device="cuda")
    d_a = torch.full((2, small, small), 7.0, dtype=torch.float64, device="cuda")
    assert _call(engine_lib, n0, d_f, pos, factor, n_grain, d_j, d_a) == -4  # SC_ERR_SIZE
    torch.cuda.synchronize()
    assert bool(torch.all(d_a == 7.0))

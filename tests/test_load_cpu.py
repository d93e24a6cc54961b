"""Load-path helpers for runs saved on another lattice (CPU only): the
library's extension and resampling against the oracle's restatement of
extendValuesAtBoundary (domain_ops.h:11-69) and resample_kernel
(GridFunctions_GPU.h:547-600)."""
import ctypes

import numpy as np
import pytest


@pytest.fixture(scope="module")
def libs():
    from superconga_b200 import build, _lib
    from oracle import oracle
    build.build()
    oracle.build()
    return _lib.load(), oracle


def _disc(n, r):
    yy, xx = np.mgrid[0:n, 0:n]
    c = 0.5 * (n - 1)
    return (np.hypot(xx - c, yy - c) < r).astype(np.int8)


def test_extend_matches_oracle(libs):
    lib, O = libs
    rng = np.random.default_rng(0)
    for n, r in ((40, 15.3), (57, 20.0)):
        dom = _disc(n, r)
        v = rng.standard_normal((2, n, n)) * dom
        want = np.stack([O.extend_grid(dom, v[k]) for k in range(2)])
        got = np.ascontiguousarray(v.copy())
        assert lib.sc_grid_extend(n, dom.ctypes.data_as(ctypes.c_void_p), 2,
                                  got.ctypes.data_as(ctypes.c_void_p)) == 0
        assert np.array_equal(got, want)
        # sites next to the grain took values, sites far outside kept theirs
        ring = (dom == 0) & (want != 0)
        assert ring.any()


@pytest.mark.parametrize("n_old,n_new", [(40, 57), (57, 40), (46, 46), (30, 91)])
def test_resample_matches_oracle(libs, n_old, n_new):
    lib, O = libs
    rng = np.random.default_rng(1)
    src = np.ascontiguousarray(rng.standard_normal((3, n_old, n_old)))
    got = np.zeros((3, n_new, n_new))
    assert lib.sc_grid_resample(n_old, n_new, 3, src.ctypes.data_as(ctypes.c_void_p),
                                got.ctypes.data_as(ctypes.c_void_p)) == 0
    want = O.resample_grid(src, n_new)
    assert np.max(np.abs(got - want)) <= 1e-14
    if n_old == n_new:
        assert np.array_equal(got, src)


def test_resample_preserves_linear_fields(libs):
    """Bilinear resampling reproduces a linear field exactly inside the margin."""
    lib, O = libs
    n_old, n_new = 50, 83
    yy, xx = np.mgrid[0:n_old, 0:n_old].astype(np.float64)
    src = np.ascontiguousarray((0.3 * xx - 0.7 * yy + 2.0)[None])
    got = np.zeros((1, n_new, n_new))
    lib.sc_grid_resample(n_old, n_new, 1, src.ctypes.data_as(ctypes.c_void_p), got.ctypes.data_as(ctypes.c_void_p))
    s = (n_old - 7) / (n_new - 7)
    y2, x2 = np.mgrid[0:n_new, 0:n_new].astype(np.float64)
    want = 0.3 * (s * (x2 - 3) + 3) - 0.7 * (s * (y2 - 3) + 3) + 2.0
    inner = (slice(3, n_new - 4), slice(3, n_new - 4))
    assert np.max(np.abs(got[0][inner] - want[inner])) < 1e-12

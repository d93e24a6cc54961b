"""The oracle held against the reference's own code, where the reference
compiles without third-party libraries: oracle/_ref/libscb_ref.so, built by
oracle.build_ref() from the reference's headers (riccati/RiccatiSolutions.h,
green/LocalGreens.h, order_parameter/OrderParameterBulk.h,
fermi_surface/FermiSurfaceCircle.h, Parameters.h).

On seeded samples covering the ranges the hot path meets (order parameters
up to twice the bulk gap, Matsubara energies with Doppler shifts, real LDOS
energies with a broadening, full and partial steps, coherence functions inside
the unit disc): the oracle's Riccati step, homogeneous solutions and Green
functions agree with the reference's to a few ulp (1e-13 relative), and the
bulk thermodynamics, Fermi-surface tables, lattice sizes and Ozaki pole counts
of the oracle and of the engine's host set-up equal the reference's.
No GPU is needed; the tests skip where the library was not built (no
reference tree).
"""
import ctypes
import math

import numpy as np
import pytest

from tests import configs


def _ref():
    from oracle import oracle as O
    path = O.build_ref()
    if path is None:
        pytest.skip("the reference's source tree is not present and oracle/_ref was not built")
    lib = ctypes.CDLL(path)
    lib.ref_bulk_gap.restype = ctypes.c_double
    lib.ref_bulk_gap.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]
    for f in ("ref_bulk_free_energy", "ref_bulk_yoshida"):
        getattr(lib, f).restype = ctypes.c_double
        getattr(lib, f).argtypes = [ctypes.c_double] * 3
    lib.ref_num_ozaki.restype = ctypes.c_int
    lib.ref_num_ozaki.argtypes = [ctypes.c_double, ctypes.c_double]
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _samples(n, seed):
    """Seeded per-site inputs: Delta (|Delta| <= 2 Delta_bulk(0)), energies
    (Matsubara i w plus a Doppler shift, or real E + i delta), g0 inside the
    unit disc, steps h and partial steps."""
    rng = np.random.default_rng(seed)
    d0 = 2.0 * 0.5 * math.exp(-0.5772156649015329)
    delta = d0 * np.sqrt(rng.uniform(0, 1, n)) * np.exp(2j * np.pi * rng.uniform(0, 1, n))
    mats = rng.uniform(0, 1, n) < 0.7
    w = np.exp(rng.uniform(math.log(1e-3), math.log(20.0), n))
    doppler = rng.normal(0, 0.05, n)
    e_real = rng.uniform(-2 * d0, 2 * d0, n)
    energy = np.where(mats, doppler + 1j * w, e_real + 1j * rng.uniform(1e-3, 0.05, n))
    g0 = np.sqrt(rng.uniform(0, 1, n)) * np.exp(2j * np.pi * rng.uniform(0, 1, n))
    h = rng.choice([0.05, 0.1, 1.0 / 15, 1.0 / 16], n) * np.where(rng.uniform(0, 1, n) < 0.2,
                                                                  rng.uniform(0, 1, n), 1.0)
    return delta, energy, g0, h


def _pairs(z):
    return np.ascontiguousarray(np.stack([z.real, z.imag], -1).ravel())


def _rel(a, b):
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def test_riccati_step_against_reference():
    from oracle import oracle as O
    lib = _ref()
    n = 20000
    delta, energy, g0, h = _samples(n, 71)
    out = np.zeros(2 * n)
    lib.ref_riccati_step(n, _p(_pairs(delta)), _p(_pairs(energy)), _p(_pairs(g0)),
                         _p(np.ascontiguousarray(h)), _p(out))
    ref = out[0::2] + 1j * out[1::2]
    ora = np.array([O.riccati_step(complex(d), complex(e), complex(g), float(s))
                    for d, e, g, s in zip(delta, energy, g0, h)])
    assert np.all(np.isfinite(ref))
    assert _rel(ora, ref) < 1e-13


def test_homogeneous_and_greens_against_reference():
    from oracle import oracle as O
    lib = _ref()
    n = 20000
    delta, energy, g0, _ = _samples(n, 72)
    out = np.zeros(4 * n)
    lib.ref_homogeneous(n, _p(_pairs(delta)), _p(_pairs(energy)), _p(out))
    g_ref, gt_ref = out[0::4] + 1j * out[1::4], out[2::4] + 1j * out[3::4]
    hom = [O.homogeneous(complex(d), complex(e)) for d, e in zip(delta, energy)]
    assert _rel(np.array([x[0] for x in hom]), g_ref) < 1e-13
    assert _rel(np.array([x[1] for x in hom]), gt_ref) < 1e-13
    # Green functions of a coherence pair inside the unit disc.
    gt = np.sqrt(np.random.default_rng(73).uniform(0, 0.95, n)) * np.exp(
        2j * np.pi * np.random.default_rng(74).uniform(0, 1, n))
    out = np.zeros(4 * n)
    lib.ref_greens(n, _p(_pairs(g0 * 0.97)), _p(_pairs(gt)), _p(out))
    gg_ref, fd_ref = out[0::4] + 1j * out[1::4], out[2::4] + 1j * out[3::4]
    grn = [O.greens(complex(a), complex(b)) for a, b in zip(g0 * 0.97, gt)]
    assert _rel(np.array([x[0] for x in grn]), gg_ref) < 1e-13
    assert _rel(np.array([x[1] for x in grn]), fd_ref) < 1e-13


@pytest.mark.parametrize("temperature", [0.001, 0.05, 0.1, 0.3, 0.5, 0.9, 0.999])
def test_bulk_thermodynamics_against_reference(temperature):
    """computeOrderParameterBulkSWave, computeFreeEnergyBulkSWave and
    computeYoshidaBulkSWave: the oracle's restatement and the engine's
    exported host functions against the reference's, at its defaults."""
    from oracle import oracle as O
    import superconga_b200 as sb
    lib = _ref()
    eps10 = 10.0 * np.finfo(np.float64).eps
    gap = lib.ref_bulk_gap(temperature, eps10, 10, 100.0)
    assert O.bulk_s_wave(temperature) == pytest.approx(gap, rel=1e-14, abs=1e-300)
    assert sb.bulk_order_parameter_s_wave(temperature) == pytest.approx(gap, rel=1e-14)
    fe = lib.ref_bulk_free_energy(temperature, gap, 100.0)
    assert O.bulk_free_energy_s_wave(temperature, gap) == pytest.approx(fe, rel=1e-12)
    y = lib.ref_bulk_yoshida(temperature, gap, 100.0)
    assert O.bulk_yoshida_s_wave(temperature, gap, 100.0) == pytest.approx(y, rel=1e-12)


@pytest.mark.parametrize("n_angles", [16, 24, 27, 32, 64, 98, 128, 256, 720])
def test_fermi_circle_against_reference(n_angles):
    """FermiSurfaceCircle: the engine's host tables (polar and system angles,
    Fermi velocity, integrand factor) against the reference's."""
    import superconga_b200 as sb
    lib = _ref()
    arrs = [np.zeros(n_angles) for _ in range(5)]
    lib.ref_fermi_circle(n_angles, *[_p(a) for a in arrs])
    phi, sys_angle, vx, vy, factor = arrs
    cfg = configs.small_disc()
    cfg["numerics"]["num_fermi_momenta"] = n_angles
    t = sb.Setup(cfg).fermi_surface()
    np.testing.assert_allclose(t["phi"], phi, rtol=0, atol=1e-15)
    np.testing.assert_allclose(t["theta"], sys_angle, rtol=0, atol=1e-15)
    np.testing.assert_allclose(t["vx"], vx, rtol=0, atol=1e-15)
    np.testing.assert_allclose(t["vy"], vy, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(t["weight"], factor)


@pytest.mark.parametrize("width,ppxi", [(10.0, 3.0), (20.0, 10.0), (30.0, 20.0), (30.0, 15.0),
                                        (100.0, 16.0), (8.0, 5.0), (40.0, 10.0), (1.0, 1000.0)])
def test_lattice_sizes_against_reference(width, ppxi):
    from oracle import oracle as O
    lib = _ref()
    n0, n1, gf = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
    lib.ref_lattice(ctypes.c_double(width), ctypes.c_double(ppxi), ctypes.byref(n0), ctypes.byref(n1),
                    ctypes.byref(gf))
    assert O.lattice(width, ppxi) == (n0.value, n1.value, gf.value)


def test_ozaki_pole_counts_against_reference():
    """Pole counts over the table and past it (the polynomial fallback)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    lib = _ref()
    for t in (0.001, 0.005, 0.01, 0.05, 0.1, 0.2, 0.3, 0.5, 0.7, 0.9, 1.0):
        for cutoff in (1.0, 8.0, 10.0 / (2 * math.pi), 16.0, 32.0, 100.0):
            want = lib.ref_num_ozaki(t, cutoff)
            assert O.num_ozaki_poles(t, cutoff) == want, (t, cutoff)
    cfg = configs.small_disc()
    for t in (0.001, 0.1, 0.5, 0.9):
        cfg["physics"]["temperature"] = t
        assert sb.Setup(cfg).dims.n_energies == lib.ref_num_ozaki(t, 8.0)

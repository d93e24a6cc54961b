"""Bulk s-wave thermodynamics (CPU only): the oracle's restatement and the
library's exported solver (sc_bulk_order_parameter_s_wave,
sc_bulk_free_energy_s_wave) against the known answers of
tests/order_parameter_bulk_test.cu in the reference project."""
import math

import numpy as np
import pytest

EPS = np.finfo(np.float64).eps
APERY = 1.2020569031595942853997381615114  # zeta(3)


def approx(value, expected, epsilon):
    """doctest::Approx(expected).epsilon(epsilon) with its default scale 1."""
    return abs(value - expected) < epsilon * (1.0 + max(abs(value), abs(expected)))


@pytest.fixture(scope="module", params=["oracle", "library"])
def bulk(request):
    if request.param == "oracle":
        from oracle import oracle as O
        return (lambda t, crit=10 * EPS: O.bulk_s_wave(t, crit)), O.bulk_free_energy_s_wave
    import superconga_b200 as sb
    return (lambda t, crit=10 * EPS: sb.bulk_order_parameter_s_wave(t, crit)), sb.bulk_free_energy_s_wave


def test_zero_temperature(bulk):
    # order_parameter_bulk_test.cu:17-31,151-161: T = 0.001 gives S_WAVE_BULK (1e-6).
    from oracle.oracle import S_WAVE_BULK
    op, _ = bulk
    assert approx(op(0.001), S_WAVE_BULK, 1e-6)


def test_critical_temperature(bulk):
    # order_parameter_bulk_test.cu:35-49,173-183: T = 1 gives 0.
    op, _ = bulk
    assert approx(op(1.0), 0.0, 1e-6)


def test_near_critical_temperature(bulk):
    # order_parameter_bulk_test.cu:53-87,197-207: Delta = sqrt(2/(7 zeta(3))
    # (1 - T)) for T in linspace(0.99, 0.999999, 10), relative 1e-3.
    op, _ = bulk
    pre = math.sqrt(2.0 / (7.0 * APERY))
    for t in np.linspace(0.99, 0.999999, 10):
        assert approx(op(float(t)), pre * math.sqrt(1.0 - t), 1e-3), t


def test_free_energy_zero_and_critical_temperature(bulk):
    # order_parameter_bulk_test.cu:91-103,220-248: F(T = 0.001) = -S_WAVE_BULK^2 / 2
    # and F(T = 1) = 0 (1e-6).
    from oracle.oracle import S_WAVE_BULK
    op, fe = bulk
    assert approx(fe(0.001, op(0.001)), -0.5 * S_WAVE_BULK * S_WAVE_BULK, 1e-6)
    assert approx(fe(1.0, op(1.0)), 0.0, 1e-6)


def test_free_energy_minimum(bulk):
    # order_parameter_bulk_test.cu:109-137,252-256: the free energy is smallest
    # at the solved gap, against Delta +- 1e-3, for T in linspace(0.1, 0.9, 10).
    op, fe = bulk
    for t in np.linspace(0.1, 0.9, 10):
        d = op(float(t))
        f = fe(float(t), d)
        assert f < fe(float(t), d + 1e-3) and f < fe(float(t), d - 1e-3), t


def test_library_matches_oracle():
    from oracle import oracle as O
    import superconga_b200 as sb
    for t in (0.001, 0.05, 0.2, 0.5, 0.9, 0.999):
        d = sb.bulk_order_parameter_s_wave(t)
        assert abs(d - O.bulk_s_wave(t)) <= 4 * EPS * d, t
        assert abs(sb.bulk_free_energy_s_wave(t, d) - O.bulk_free_energy_s_wave(t, d)) <= 1e-13 * abs(O.bulk_free_energy_s_wave(t, d)), t


def test_yoshida_library_matches_oracle():
    # computeYoshidaBulkSWave: 1 at zero temperature, the oracle's sum elsewhere.
    from oracle import oracle as O
    import superconga_b200 as sb
    assert sb.bulk_yoshida_s_wave(0.0, 0.3, 16.0) == 1.0
    for t in (0.05, 0.1, 0.5, 0.9):
        d = O.bulk_s_wave(t)
        y = O.bulk_yoshida_s_wave(t, d, 16.0)
        assert 0.0 < y < 1.0
        assert abs(sb.bulk_yoshida_s_wave(t, d, 16.0) - y) <= 1e-13 * y, t


def test_invalid_arguments_rejected():
    import superconga_b200 as sb
    from superconga_b200 import _lib
    with pytest.raises(_lib.EngineError):
        sb.bulk_order_parameter_s_wave(-0.5)
    with pytest.raises(_lib.EngineError):
        sb.bulk_free_energy_s_wave(0.0, 0.1)

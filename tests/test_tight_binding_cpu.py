"""Tight-binding Fermi surfaces (CPU only).

The oracle's restatement of FermiSurfaceTightBinding is pinned to the
reference's own known answers (tests/fermi_surface_tight_binding_test.cu and
tests/basis_function_normalization_test.cu in the reference project), and the
engine's host set-up is checked against the oracle table by table.
"""
import copy
import math

import numpy as np
import pytest

from tests import configs

# tests/fermi_surface_tight_binding_test.cu:15-28 (the BdG paper's surfaces).
FS1 = dict(t1=-0.25, t2=0.0, mu=0.0, avg_p=2.61870038, avg_v=2.53562285)
FS2 = dict(t1=-0.495, t2=0.156, mu=-1.267, avg_p=2.08128010, avg_v=2.39512296)
EPS = np.finfo(np.float64).eps


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build()
    return oracle


def tb_config(fs: dict, n_angles: int = 24, symmetry: str = "dx2-y2") -> dict:
    cfg = configs.small_square_d() if symmetry != "s" else configs.small_disc()
    cfg = copy.deepcopy(cfg)
    if symmetry not in cfg["physics"]["order_parameter"]:
        cfg["physics"]["order_parameter"] = {symmetry: {"critical_temperature": 1.0}}
    cfg["numerics"]["num_fermi_momenta"] = n_angles
    cfg["physics"]["fermi_surface"] = {"type": "tight_binding", "hopping_nnn": fs["t1"],
                                       "hopping_nnnn": fs["t2"], "chemical_potential": fs["mu"]}
    return cfg


@pytest.mark.parametrize("fs", [FS1, FS2], ids=["FS1", "FS2"])
def test_averages_match_reference(O, fs):
    # tests/fermi_surface_tight_binding_test.cu:238-258,364-398: 100 angles,
    # relative tolerance 1e-8 in double precision.
    t = O.tight_binding(fs["t1"], fs["t2"], fs["mu"], 100)
    assert t["avg_fermi_speed"] == pytest.approx(fs["avg_v"], rel=1e-8)
    assert t["avg_fermi_momentum"] == pytest.approx(fs["avg_p"], rel=1e-8)


@pytest.mark.parametrize("mu,origin", [(-1.0, 0.0), (1.0, math.pi)])
def test_momentum_origin(O, mu, origin):
    # tests/fermi_surface_tight_binding_test.cu:120-145 (19 angles).
    t = O.tight_binding(0.0, 0.0, mu, 19)
    assert t["origin"][0] == pytest.approx(origin, abs=10 * EPS)
    assert t["origin"][1] == pytest.approx(origin, abs=10 * EPS)


def test_square_surface(O):
    # tests/fermi_surface_tight_binding_test.cu:165-213: t' = t'' = mu = 0 gives
    # the square |kx| + |ky| = pi around the origin; 12 angles, 100 eps.
    n = 12
    t = O.tight_binding(0.0, 0.0, 0.0, n)
    ox, oy = t["origin"]
    for k in range(n):
        ang = 2.0 * math.pi / n * k + 0.5 * math.pi
        ux, uy = math.cos(ang), math.sin(ang)
        mag = math.pi / (abs(ux) + abs(uy))
        ex, ey = mag * ux + ox, mag * uy + oy
        assert math.cos(t["px"][k]) == pytest.approx(math.cos(ex), rel=100 * EPS, abs=100 * EPS)
        assert math.cos(t["py"][k]) == pytest.approx(math.cos(ey), rel=100 * EPS, abs=100 * EPS)


def test_integrand_factor_sums_to_one(O):
    # tests/fermi_surface_tight_binding_test.cu:215-236 (default surface, 9 angles).
    t = O.tight_binding(0.0, 0.0, 1.0, 9)
    assert np.all(t["weight"] > 0.0)
    assert t["weight"].sum() == pytest.approx(1.0, rel=10 * EPS)


@pytest.mark.parametrize("fs", [FS1, FS2], ids=["FS1", "FS2"])
def test_integrand_factor_is_the_jacobian(O, fs):
    # tests/fermi_surface_tight_binding_test.cu:30-103: the factor equals
    # |dk/dphi| / |v_F| (1e-3); checked here on a fine prime-sized grid
    # (trapezoid weights) by central differences between neighbouring angles.
    n = 4099
    t = O.tight_binding(fs["t1"], fs["t2"], fs["mu"], n)
    ox, oy = t["origin"]
    kx = np.mod(t["px"] - ox + math.pi, 2 * math.pi) - math.pi
    ky = np.mod(t["py"] - oy + math.pi, 2 * math.pi) - math.pi
    dphi = 2.0 * math.pi / n
    dkx = (np.roll(kx, -1) - np.roll(kx, 1)) / (2 * dphi)
    dky = (np.roll(ky, -1) - np.roll(ky, 1)) / (2 * dphi)
    speed = np.hypot(t["vx"], t["vy"])  # normalised speeds: a common factor
    jac = np.hypot(dkx, dky) / speed
    ratio = jac / t["weight"]
    assert np.max(np.abs(ratio / np.median(ratio) - 1.0)) < 1e-3


@pytest.mark.parametrize("fs", [FS1, FS2], ids=["FS1", "FS2"])
def test_basis_normalisation(O, fs):
    # tests/basis_function_normalization_test.cu:33-100: with the lattice
    # harmonics of a non-circular surface, <|eta|^2> = 1 after normalising.
    t = O.tight_binding(fs["t1"], fs["t2"], fs["mu"], 100)
    for eta in (np.cos(t["px"]) + np.cos(t["py"]), np.cos(t["px"]) - np.cos(t["py"])):
        norm = 1.0 / math.sqrt(np.sum(eta * eta * t["weight"]))
        assert np.sum((eta * norm) ** 2 * t["weight"]) == pytest.approx(1.0, rel=50 * EPS)


@pytest.mark.parametrize("fs", [FS1, FS2], ids=["FS1", "FS2"])
def test_engine_tables_match_oracle(O, fs):
    from superconga_b200.engine import Setup
    n = 100
    s = Setup(tb_config(fs, n_angles=n)).fermi_surface()
    t = O.tight_binding(fs["t1"], fs["t2"], fs["mu"], n)
    for k in ("phi", "theta", "px", "py", "vx", "vy", "weight"):
        assert np.max(np.abs(s[k] - t[k])) < 1e-13, k
    h = 1.0 / tb_config(fs)["numerics"]["points_per_coherence_length"]
    assert np.max(np.abs(s["step"] - h / t["speed"])) < 1e-13
    assert s["avg_fermi_speed"] == pytest.approx(fs["avg_v"], rel=1e-8)
    assert s["avg_fermi_momentum"] == pytest.approx(fs["avg_p"], rel=1e-8)
    assert s["origin"] == pytest.approx(t["origin"])


def test_engine_circle_tables():
    # The default circle: momentum = velocity on the unit circle, step h.
    from superconga_b200.engine import Setup
    cfg = configs.small_disc()
    s = Setup(cfg).fermi_surface()
    assert np.allclose(s["px"], np.cos(s["phi"])) and np.allclose(s["vx"], s["px"])
    assert np.all(s["step"] == 1.0 / cfg["numerics"]["points_per_coherence_length"])
    assert s["origin"] == (0.0, 0.0)


@pytest.mark.parametrize("n", [7, 9, 11, 12])
def test_engine_circle_matches_reference_tests(n):
    # tests/fermi_surface_circle_test.cu:70-192 on the engine's tables: system
    # angle phi - pi/2 on the uniform grid offset by pi/2, unit momentum and
    # velocity along phi, positive integrand factors summing to 1 (10 eps).
    from superconga_b200.engine import Setup
    cfg = configs.small_disc()
    cfg["numerics"]["num_fermi_momenta"] = n
    s = Setup(cfg).fermi_surface()
    for k in range(n):
        ang = 2.0 * math.pi / n * k + 0.5 * math.pi
        sys_expected = math.fmod(ang - 0.5 * math.pi + 4 * math.pi, 2 * math.pi)
        assert math.fmod(s["theta"][k] + 4 * math.pi, 2 * math.pi) == pytest.approx(sys_expected, rel=10 * EPS, abs=10 * EPS)
        assert s["px"][k] == pytest.approx(math.cos(ang), abs=10 * EPS)
        assert s["py"][k] == pytest.approx(math.sin(ang), abs=10 * EPS)
        assert math.hypot(s["vx"][k], s["vy"][k]) == pytest.approx(1.0, rel=10 * EPS)
    assert np.all(s["weight"] > 0.0)
    assert s["weight"].sum() == pytest.approx(1.0, rel=10 * EPS)


def test_unknown_fermi_surface_rejected():
    from superconga_b200 import _lib
    from superconga_b200.engine import Setup
    cfg = configs.small_disc()
    cfg["physics"]["fermi_surface"] = {"type": "hexagonal"}
    with pytest.raises(_lib.EngineError):
        Setup(cfg)


def test_oracle_iteration_on_tight_binding(O):
    # The oracle runs a tight-binding grain: one iteration stays finite and the
    # order parameter keeps its scale.
    cfg = tb_config(FS2, n_angles=16)
    o = O.Oracle(cfg)
    st = o.setup
    delta, a0 = configs.seeded_state(st.n_comp, st.n0, 0.2, seed=7)
    o.set_state(delta, a0)
    o.compute()
    d, j, a = o.results()
    assert np.all(np.isfinite(d)) and np.all(np.isfinite(j))
    assert 0.01 < np.max(np.abs(d)) < 2.0

"""The LDOS postprocess of the CPU oracle (CPU only).

Known answers: a uniform s-wave order parameter in a grain with specular
walls and no field is the bulk state everywhere, so the LDOS is the broadened
BCS density of states at every site; and particle-hole symmetry makes the
angle-integrated LDOS even in energy.
"""
import numpy as np
import pytest

from tests import configs


@pytest.fixture(scope="module")
def O():
    from oracle import oracle
    oracle.build()
    return oracle


def _uniform_s_disc():
    cfg = configs.small_disc()
    cfg["physics"]["external_flux_quanta"] = 0.0
    cfg["physics"]["penetration_depth"] = -1.0
    cfg["numerics"]["points_per_coherence_length"] = 3.0
    return cfg


def test_bcs_bulk_dos(O):
    sim = _uniform_s_disc()
    s = O.make_setup(sim)
    db = O.delta_bulk(s.temperature, "s")
    pp = configs.ldos_postprocess(db, n_energies=8, per_block=8, n_angles=16, broadening=0.04)
    L = O.LdosOracle(sim, pp)
    d = np.zeros((1, 2, L.n0, L.n0))
    d[0, 0] = db
    L.set_state(d, np.zeros((2, L.n0, L.n0)))
    L.begin_block(0)
    L.burn_in()
    L.iterate()
    dom = L.oracle.domain() > 0
    want = configs.bcs_dos(L.energies, 0.04, db)
    for k in range(len(L.energies)):
        got = L.ldos[k][dom]
        assert np.max(np.abs(got - want[k])) < 1e-9 * max(1.0, want[k]), (k, got[:3], want[k])
        assert np.all(L.ldos[k][~dom] == 0.0)


def test_particle_hole_symmetry(O):
    sim = configs.small_disc()
    s = O.make_setup(sim)
    db = O.delta_bulk(s.temperature, "s")
    pp = configs.ldos_postprocess(db, n_energies=6, per_block=6, n_angles=16)
    L = O.LdosOracle(sim, pp)
    d, a = configs.seeded_state(1, L.n0, db, 2, 0.01, False, 0.05)
    L.set_state(d, a)
    L.begin_block(0)
    for _ in range(3):
        L.burn_in()
    for _ in range(40):
        r, _, _ = L.iterate()
        if r < 1e-9:
            break
    n = len(L.energies)
    scale = np.max(np.abs(L.ldos))
    for k in range(n // 2):
        assert np.max(np.abs(L.ldos[k] - L.ldos[n - 1 - k])) < 1e-6 * scale, k


@pytest.mark.parametrize("swave", [True, False], ids=["s-wave disc", "d-wave square"])
def test_reference_dos(O, swave):
    """tests/physics/dos_test.cu:218-240 (double): the grain-averaged LDOS of a
    bulk s-wave disc and of a d_{x2-y2} square without pair breaking converges
    within 42 iterations and matches the angle-averaged bulk DOS to 1e-8."""
    sim, pp = configs.dos_test_case(swave)
    L = O.LdosOracle(sim, pp)
    s = L.oracle.setup
    db = O.delta_bulk(0.5, s.symmetries[0])
    d = np.zeros((1, 2, L.n0, L.n0))
    d[0, 0] = db
    L.set_state(d, np.zeros((2, L.n0, L.n0)))
    L.begin_block(0)
    res = 1.0
    for _ in range(42):
        res = L.iterate()[0]
        if res < 1e-8:
            break
    assert res < 1e-8
    dom = L.oracle.domain() > 0
    got = np.array([L.ldos[k][dom].mean() for k in range(len(L.energies))])
    want = configs.bulk_dos(np.asarray(L.energies), 0.008, db, swave, 160)
    assert np.max(np.abs(got - want) / (1.0 + np.abs(want))) < 1e-8

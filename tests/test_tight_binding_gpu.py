"""GPU parity on tight-binding Fermi surfaces (FermiSurfaceTightBinding.h):
the CUDA engine (through the C ABI) against the CPU oracle.  A non-circular
surface changes the Riccati step per angle (h/|v_F|), the system angles, the
integrand factors, the velocity in the current and the Doppler shift, the
lattice-harmonic basis functions and the momentum origin of the boundary
condition; every one of them reaches these results."""
import numpy as np
import pytest

from tests import configs
from tests.test_tight_binding_cpu import FS1, FS2, tb_config

pytestmark = pytest.mark.gpu

TOL = 1e-10

CASES = {
    # FS2 (less circular, origin (pi,pi)): d-wave square with a field and a
    # self-consistent vector potential.
    "fs2_square_d": (tb_config(FS2, n_angles=24), dict(complex_noise=True, noise=0.1, a_scale=0.05)),
    # FS1 (nearly circular): s-wave disc in a field.
    "fs1_disc_s": (tb_config(FS1, n_angles=32, symmetry="s"), dict(a_scale=0.05)),
}


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / scale)


def _pair(cfg, seed=1, noise=0.01, complex_noise=False, a_scale=0.0, mode="fp64"):
    from oracle import oracle as O
    import superconga_b200 as sb
    o = O.Oracle(cfg)
    e = sb.Context(cfg, mode=mode)
    s = o.setup
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, seed, noise, complex_noise, a_scale)
    o.set_state(d, a)
    e.set_state(d, a)
    return o, e, db


@pytest.mark.parametrize("case", list(CASES))
def test_geometry_and_boundary_initial(engine_lib, case):
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    for a in range(o.setup.n_angles):
        assert np.array_equal(e.frame_labels(a)[0], o.geometry(a)[0]), a
    assert e.boundary_sizes() == o.boundary_sizes()
    o.set_boundary_initial()
    e.boundary_initial()
    for which in range(4):
        assert _rel(e.boundary(which), o.boundary(which)) < TOL, which


@pytest.mark.parametrize("case", list(CASES))
def test_angle_sweep(engine_lib, case):
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    o.set_boundary_initial()
    e.boundary_initial()
    na = o.setup.n_angles
    for a in sorted({0, 1, na // 3, na // 2, na - 1}):
        f_o, g_o, i_o, _ = o.angle_greens(a)
        f_e, g_e, i_e = e.angle_greens(a)
        assert _rel(f_e, f_o) < TOL, (a, "F")
        assert _rel(g_e, g_o) < TOL, (a, "G")
        assert _rel(i_e, i_o) < TOL, (a, "I")


@pytest.mark.parametrize("case", list(CASES))
def test_iterations(engine_lib, case):
    """Three Context::compute iterations: g(x), x, Omega and the boundary."""
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    for it in range(3):
        o.compute()
        e.compute(1)
        d_o, j_o, a_o = o.results()
        d_e, j_e, a_e = e.results()
        assert _rel(d_e, d_o) < TOL, (it, "delta")
        assert _rel(j_e, j_o) < TOL, (it, "current")
        assert _rel(a_e, a_o) < TOL, (it, "vector potential")
        assert _rel(e.state()[0], o.state()[0]) < TOL, (it, "x")
        so, se = o.scalars(), e.scalars()
        for k in ("free_energy", "magnetic_free_energy"):
            assert abs(se[k] - so[k]) <= TOL * max(abs(so[k]), 1e-12), (it, k)
        assert abs(se["residual"] - so["residual"]) <= 1e-8 * so["residual"], it
        for which in range(4):
            assert _rel(e.boundary(which), o.boundary(which)) < TOL, (it, which)


def test_mixed_precision(engine_lib):
    """FP32 stepping (no mirror pairing on a tight-binding surface) against FP64."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfg, kw = CASES["fs2_square_d"]
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 3, 0.1, True, 0.05)
    out = []
    for mode in ("fp64", "mixed"):
        e = sb.Context(cfg, mode=mode)
        e.set_state(d, a)
        e.compute(4)
        out.append(e.results())
        e.close()
    (d64, j64, _), (d32, j32, _) = out
    assert np.max(np.abs(d32 - d64)) / db <= 1e-5
    assert _rel(j32, j64) <= 1e-4


def test_ldos(engine_lib):
    """LDOS postprocess on the tight-binding d-wave square, one block."""
    from oracle import oracle as O
    import superconga_b200 as sb
    sim, _ = CASES["fs2_square_d"]
    s = O.make_setup(sim)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    pp = configs.ldos_postprocess(db, n_energies=8, per_block=8, n_angles=24, broadening=0.03)
    L = O.LdosOracle(sim, pp)
    e = sb.LdosContext(sim, pp, mode="fp64")
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 2, 0.05, True, 0.05)
    L.set_state(d, a)
    e.set_state(d, a)
    L.begin_block(0)
    e.begin_block(0)
    L.burn_in()
    e.burn_in(1)
    for _ in range(2):
        L.iterate()
        e.iterate(1)
    assert _rel(e.ldos(), L.ldos) < TOL


def test_batch_matches_single(engine_lib):
    """A tight-binding grain and a circular one advanced in one batch give the
    results of the same grains run on their own."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfgs = [CASES["fs2_square_d"][0], configs.small_disc()]
    states = []
    for c in cfgs:
        s = O.make_setup(c)
        db = O.delta_bulk(s.temperature, s.symmetries[0])
        states.append(configs.seeded_state(s.n_comp, s.n0, db, 9, 0.05, True, 0.05))
    b = sb.Batch(cfgs, mode="fp64")
    for g, (d, a) in zip(b.grains, states):
        g.set_state(d, a)
    b.compute(2)
    for g, c, (d, a) in zip(b.grains, cfgs, states):
        e = sb.Context(c, mode="fp64")
        e.set_state(d, a)
        e.compute(2)
        assert _rel(g.results()[0], e.results()[0]) < 1e-11
        assert _rel(g.results()[1], e.results()[1]) < 1e-11
        e.close()
    b.close()


def test_adjoint_vs_fd(engine_lib):
    """dOmega/d(Delta, A, B_ext) of the frozen-boundary pass on the
    tight-binding square against central differences (step 1e-4, 1e-6)."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfg, _ = CASES["fs2_square_d"]
    e = sb.Context(cfg, mode="fp64")
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 5, 0.1, True, 0.05)
    e.set_state(d, a)
    for _ in range(3):
        e.burn_in(1)
    dom = e.domain() > 0
    d = d * dom
    b0 = e.external_field()
    e.set_state(d, a)
    e.evaluate()
    gd, ga, gb = e.adjoint(1.0)
    rng = np.random.default_rng(13)
    eps = 1e-4
    for _ in range(3):
        vd = rng.standard_normal(d.shape) * db * dom
        va = rng.standard_normal(a.shape) * 0.05
        vb = float(rng.standard_normal()) * 0.01
        vals = []
        for sgn in (1.0, -1.0):
            e.set_state(d + sgn * eps * vd, a + sgn * eps * va)
            e.set_external_field(b0 + sgn * eps * vb)
            vals.append(e.evaluate())
        fd = (vals[0] - vals[1]) / (2 * eps)
        ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
        assert abs(fd - ad) <= 1e-6 * max(abs(ad), abs(fd)), (fd, ad)
    e.close()

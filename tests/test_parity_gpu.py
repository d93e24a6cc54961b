"""GPU parity: the CUDA engine (through the C ABI) against the CPU oracle.

FP64 results must agree with the oracle to 1e-10 relative (relative to the
largest magnitude of the compared field); the mixed-precision form must stay
within 1e-5 of the FP64 form relative to the bulk gap.
"""
import numpy as np
import pytest

from tests import configs

pytestmark = pytest.mark.gpu

TOL = 1e-10


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


CASES = {
    "golden_disc": (configs.golden_disc(), dict(a_scale=0.0)),
    "small_disc": (configs.small_disc(), dict(a_scale=0.05)),
    "small_square_d": (configs.small_square_d(), dict(complex_noise=True, noise=0.1, a_scale=0.05)),
    "chiral_annulus": (configs.chiral_annulus(), dict(complex_noise=True, noise=0.1, a_scale=0.02)),
}


@pytest.mark.parametrize("case", list(CASES))
def test_dims_and_geometry(engine_lib, case):
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    assert (e.dims.n0, e.dims.n1, e.dims.n_energies) == (o.n0, o.n1, o.setup.n_energies)
    assert np.array_equal(e.domain(), o.domain())
    assert e.boundary_sizes() == o.boundary_sizes()
    x0, x1, y0, y1 = o.ranges()
    for a in range(o.setup.n_angles):
        lab, box = e.frame_labels(a)
        assert np.array_equal(lab, o.geometry(a)[0])
        assert box == (x0[a], x1[a], y0[a], y1[a])


@pytest.mark.parametrize("case", list(CASES))
def test_boundary_initial(engine_lib, case):
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    o.set_boundary_initial()
    e.boundary_initial()
    for which in range(4):
        assert _rel(e.boundary(which), o.boundary(which)) < TOL, which


@pytest.mark.parametrize("case", list(CASES))
def test_angle_sweep(engine_lib, case):
    """Frame Green sums and out-going boundary values of single angles."""
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
    for which in (1, 3):
        assert _rel(e.boundary(which), o.boundary(which)) < TOL, which


@pytest.mark.parametrize("case", list(CASES))
def test_iterations(engine_lib, case):
    """Three full Context::compute iterations (the second and third include the
    accelerator step): g(x), x, free energy and residuals."""
    cfg, kw = CASES[case]
    o, e, _ = _pair(cfg, **kw)
    for it in range(3):
        o.compute()
        e.compute(1)
        d_o, j_o, a_o = o.results()
        d_e, j_e, a_e = e.results()
        assert _rel(d_e, d_o) < TOL, (it, "delta")
        assert _rel(j_e, j_o) < TOL, (it, "current")
        if o.setup.params.penetration_depth > 0:
            assert _rel(a_e, a_o) < TOL, (it, "vector potential")
        x_o, ax_o = o.state()
        x_e, ax_e = e.state()
        assert _rel(x_e, x_o) < TOL, (it, "x")
        so, se = o.scalars(), e.scalars()
        for k in ("free_energy", "free_energy_per_area", "magnetic_free_energy"):
            assert abs(se[k] - so[k]) <= TOL * max(abs(so[k]), 1e-12), (it, k)
        for k in ("res_order_parameter", "res_current", "res_free_energy", "res_boundary",
                  "res_vector_potential", "residual"):
            assert abs(se[k] - so[k]) <= 1e-8 * max(abs(so[k]), 1e-12), (it, k, se[k], so[k])
        for which in range(4):
            assert _rel(e.boundary(which), o.boundary(which)) < TOL, (it, which)


def test_state_into_caller_buffers(engine_lib):
    """Context.state writes into the caller's (pinned) arrays and rejects
    arrays of the wrong type or size."""
    import torch
    cfg, kw = CASES["small_disc"]
    o, e, _ = _pair(cfg, **kw)
    e.compute(1)
    d_ref, a_ref = e.state()
    d = torch.empty(d_ref.shape, dtype=torch.float64, pin_memory=True).numpy()
    a = torch.empty(a_ref.shape, dtype=torch.float64, pin_memory=True).numpy()
    e.state(d, a)
    assert np.array_equal(d, d_ref) and np.array_equal(a, a_ref)
    with pytest.raises(ValueError):
        e.state(np.zeros(d_ref.shape, np.float32), a)


def test_burn_in(engine_lib):
    cfg, kw = CASES["small_disc"]
    o, e, _ = _pair(cfg, **kw)
    for _ in range(2):
        o.burn_in()
        r_e, _ = e.burn_in(1)
    assert abs(r_e - o.scalars()["res_boundary"]) <= 1e-8 * o.scalars()["res_boundary"]
    for which in range(4):
        assert _rel(e.boundary(which), o.boundary(which)) < TOL


def test_poisson(engine_lib):
    cfg, _ = CASES["small_square_d"]
    from oracle import oracle as O
    import superconga_b200 as sb
    o = O.Oracle(cfg)
    e = sb.Context(cfg)
    rng = np.random.default_rng(7)
    j = rng.standard_normal((2, o.n0, o.n0)) * (o.domain() > 0)
    assert _rel(e.poisson(j), o.poisson(j)) < 1e-10


@pytest.mark.parametrize("which", ["disc_n71", "c1_n206"])
def test_poisson_mixed_radix(engine_lib, which):
    """The FFT Poisson solve on transform sides with radix-5 and radix-3 stages
    (N0 = 71: P = 160 = 4*4*2*5; C1, N0 = 206: P = 480 = 4*4*2*3*5) against
    the oracle's direct sums of the separable filters."""
    import copy
    from oracle import oracle as O
    import superconga_b200 as sb
    from superconga_b200 import workloads
    if which == "disc_n71":
        cfg = copy.deepcopy(configs.small_disc())
        cfg["geometry"][0]["disc"]["radius"] = 6.5
    else:
        cfg = workloads.c1()
    o = O.Oracle(cfg)
    e = sb.Context(cfg)
    rng = np.random.default_rng(11)
    j = rng.standard_normal((2, o.n0, o.n0)) * (o.domain() > 0)
    assert _rel(e.poisson(j), o.poisson(j)) < 1e-10


@pytest.mark.parametrize("case", ["small_disc", "small_square_d"])
def test_anderson_iterations(engine_lib, case):
    """The Anderson accelerator (Anderson.h:201-355) on the GPU against the
    oracle over six iterations, so that its history fills (rank 4) and the
    oldest slot is reused: x, g(x) and the free energy within 1e-10."""
    cfg, kw = CASES[case]
    o, e, _ = _pair(configs.with_accelerator(cfg, "anderson"), **kw)
    for it in range(6):
        o.compute()
        e.compute(1)
        assert _rel(e.state()[0], o.state()[0]) < TOL, (it, "x")
        assert _rel(e.results()[0], o.results()[0]) < TOL, (it, "delta")
        fo, fe = o.scalars()["free_energy"], e.scalars()["free_energy"]
        assert abs(fe - fo) <= TOL * abs(fo), it


def test_poisson_magnetostatics_disc(engine_lib):
    """tests/physics/vector_potential_test.cu:238-245 on the engine's FFT solve
    (256 x 256, spacing 0.1): within 2e-4 of the magnetostatic solution of a
    rotating disc current, rotation symmetries to 1e-8, and the oracle's
    filter sums to 1e-10."""
    import math
    from oracle import oracle as O
    import superconga_b200 as sb
    cfg = configs.disc_n256()
    e = sb.Context(cfg)
    assert e.dims.n0 == 256
    j, expected = configs.rotating_disc_current(256, 0.1)
    a = e.poisson(j)
    assert math.sqrt(np.sum((a - expected) ** 2) / np.sum(expected ** 2)) < 2e-4
    assert configs.vector_potential_symmetry_error(a) < 1e-8
    assert _rel(a, O.Oracle(cfg).poisson(j)) < 1e-10
    e.close()


@pytest.mark.parametrize("acc", ["congacc", "picard", "polyak", "barzilai-borwein", "anderson"])
def test_golden_free_energy(engine_lib, acc):
    """tests/accelerators_test.cu:45-149 on the engine: converged within 100
    iterations to Omega/area = -0.0185386592 within 1e-3 relative."""
    from oracle import oracle as O
    import superconga_b200 as sb
    cfg = configs.golden_disc(acc)
    e = sb.Context(cfg)
    n0, nc = e.dims.n0, e.dims.n_comp
    d = np.zeros((nc, 2, n0, n0))
    d[0, 0] = O.delta_bulk(0.5, "s")
    e.set_state(d, np.zeros((2, n0, n0)))
    it, conv = e.run(0, 100)
    fe = e.scalars()["free_energy_per_area"]
    assert conv
    assert abs(fe - configs.GOLDEN_FREE_ENERGY_PER_AREA) <= 1e-3 * abs(configs.GOLDEN_FREE_ENERGY_PER_AREA)


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_swave_disc_analytic_free_energy(engine_lib, mode):
    """tests/physics/swave_disc_test.cu:66-174 on the engine: converged within
    100 iterations, free energy per area within 1e-3 of the London value."""
    from oracle import oracle as O
    import superconga_b200 as sb
    cfg = configs.swave_disc_field()
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    db = O.delta_bulk(0.2, "s")
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = db
    e.set_state(d, np.zeros((2, n0, n0)))
    it, conv = e.run(0, 100)
    expected = configs.swave_disc_free_energy(0.2, 16.0, 5.0, 5.0, 20.0, db)
    fe = e.scalars()["free_energy_per_area"]
    assert conv
    assert abs(fe - expected) <= 1e-3 * abs(expected), (fe, expected)
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("case", ["s_disc", "s_square", "d_square"])
def test_low_temperature_bulk_values(engine_lib, case, mode):
    """tests/physics/low_temp_free_energy_test.cu:62-281 on the engine (281
    Ozaki poles, 32 or 360 angles): converged within 50 iterations, grain-
    averaged gap within 1e-5 of the zero-temperature bulk value, no current
    (machine epsilon of the stepping type, as the reference's float and double
    cases), free energy per area within 1e-4 of -Delta^2/2.  FP64 also matches
    the oracle's converged fields (1e-10)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    from tests.test_oracle_golden import LOW_TEMPERATURE_CASES, low_temperature_observables
    swave, disc = LOW_TEMPERATURE_CASES[case]
    cfg = configs.low_temperature_bulk(swave, disc)
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = O.delta_bulk(0.001, "s" if swave else "dx2-y2")
    e.set_state(d, np.zeros((2, n0, n0)))
    it, conv = e.run(1, 50)
    delta, current, _ = e.results()
    sc = e.scalars()
    avg_d, avg_j, fe = low_temperature_observables(delta, current, e.domain(), sc["free_energy_per_area"])
    expected = O.S_WAVE_BULK if swave else O.D_WAVE_BULK
    eps = np.finfo(np.float64 if mode == "fp64" else np.float32).eps
    assert conv
    assert avg_d == pytest.approx(expected, rel=1e-5)
    assert abs(avg_j) <= eps * (1.0 + abs(avg_j))
    assert fe == pytest.approx(-0.5 * expected * expected, rel=1e-4)
    if mode == "fp64":
        o = O.Oracle(cfg)
        o.set_state(d, np.zeros((2, n0, n0)))
        for _ in range(it):
            o.compute()
        assert _rel(delta, o.results()[0]) < TOL
        so = o.scalars()["free_energy_per_area"]
        assert abs(sc["free_energy_per_area"] - so) <= TOL * abs(so)
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_current_follows_phase_gradient(engine_lib, mode):
    """tests/physics/current_phase_gradient_test.cu:22-122 on the engine: one
    iteration from a phase winding of +1 (charge sign -1); the current runs
    against the phase gradient at every site, and FP64 matches the oracle."""
    from oracle import oracle as O
    import superconga_b200 as sb
    from tests.test_oracle_golden import phase_gradient_signs_ok
    cfg = configs.phase_gradient_disc()
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    d = configs.phase_winding_state(n0, O.delta_bulk(0.9, "s"), 1.0)
    e.set_state(d, np.zeros((2, n0, n0)))
    e.compute(1)
    _, current, _ = e.results()
    x = e.state()[0]
    assert np.max(np.abs(current)) > 0.0
    assert phase_gradient_signs_ok(x, current, -1)
    if mode == "fp64":
        o = O.Oracle(cfg)
        o.set_state(d, np.zeros((2, n0, n0)))
        o.compute()
        assert _rel(current, o.results()[1]) < TOL
        assert _rel(x, o.state()[0]) < TOL
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_penetration_depth(engine_lib, mode):
    """tests/physics/penetration_depth_test.cu:89-179 on the engine: converged
    within 100 iterations and the London-fitted penetration depth within 0.1
    of lambda = 1.  FP64 follows the oracle's first five CongAcc iterations
    (1e-10); after that the adaptive step sizes let rounding differences grow
    (3e-5 relative in A at convergence, below the 1e-3 criterion), so the
    converged fits are compared to 1e-3."""
    from oracle import oracle as O
    import superconga_b200 as sb
    cfg = configs.penetration_depth_disc()
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = O.delta_bulk(0.1, "s")
    e.set_state(d, np.zeros((2, n0, n0)))
    it, conv = e.run(0, 100)
    a = e.state()[1]
    lam = configs.penetration_depth_from_state(a, e.domain(), 0.2, 0.5, 20.0, 1.0)
    assert conv
    assert abs(lam - 1.0) < 0.1 * max(abs(lam), 1.0), lam
    if mode == "fp64":
        o = O.Oracle(cfg)
        o.set_state(d, np.zeros((2, n0, n0)))
        for _ in range(5):
            o.compute()
        e2 = sb.Context(cfg, mode=mode)
        e2.set_state(d, np.zeros((2, n0, n0)))
        e2.compute(5)
        assert _rel(e2.state()[1], o.state()[1]) < TOL
        assert _rel(e2.state()[0], o.state()[0]) < TOL
        e2.close()
        while not o.is_converged():
            o.compute()
        lam_o = configs.penetration_depth_from_state(o.state()[1], o.domain(), 0.2, 0.5, 20.0, 1.0)
        assert abs(lam - lam_o) < 1e-3 * lam_o, (lam, lam_o)
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
@pytest.mark.parametrize("temperature", [0.1, 0.9])
def test_current_linear_response(engine_lib, temperature, mode):
    """tests/physics/current_linear_response_test.cu on the engine: one
    iteration in a uniform vector potential (0.01, 0.01); the middle current
    is -Y(T) A within 1 %, and FP64 matches the oracle's current."""
    from oracle import oracle as O
    import superconga_b200 as sb
    from tests.test_oracle_golden import LINEAR_RESPONSE_A, linear_response_check
    cfg = configs.linear_response_square(temperature)
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = O.delta_bulk(temperature, "s")
    a = np.full((2, n0, n0), LINEAR_RESPONSE_A)
    e.set_state(d, a)
    e.compute(1)
    current = e.results()[1]
    linear_response_check(current, temperature, sb.bulk_yoshida_s_wave)
    if mode == "fp64":
        o = O.Oracle(cfg)
        o.set_state(d, a)
        o.compute()
        assert _rel(current, o.results()[1]) < TOL
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_solenoid_annulus_free_energy(engine_lib, mode):
    """tests/physics/swave_annulus_solenoid_gauge_test.cu on the engine: the
    free energy per area of the once-winding annulus is the parabola in the
    flux about Phi = q w (1e-3), and FP64 ends on the oracle's free energy
    (1e-9)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    from tests.test_oracle_golden import solenoid_annulus_check
    fes, conv = [], []
    for flux in configs.SOLENOID_FLUXES:
        cfg = configs.solenoid_annulus(flux)
        e = sb.Context(cfg, mode=mode)
        n0 = e.dims.n0
        d = configs.phase_winding_state(n0, O.bulk_s_wave(0.2), 1.0)
        e.set_state(d, np.zeros((2, n0, n0)))
        it, ok = e.run(0, 100)
        fes.append(e.scalars()["free_energy_per_area"])
        conv.append(ok)
        e.close()
        if mode == "fp64":
            o = O.Oracle(cfg)
            o.set_state(d, np.zeros((2, n0, n0)))
            for _ in range(it):
                o.compute()
            so = o.scalars()["free_energy_per_area"]
            # Same iteration count; Barzilai-Borwein steps let rounding
            # differences grow over the ~20 iterations, which the converged
            # free energy feels only at second order.
            assert abs(fes[-1] - so) <= 1e-9 * abs(so), (flux, fes[-1], so)
    solenoid_annulus_check(fes, conv, (sb.bulk_order_parameter_s_wave, sb.bulk_free_energy_s_wave,
                                       sb.bulk_yoshida_s_wave))


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_radial_annulus(engine_lib, mode):
    """tests/physics/swave_annulus_radial_gauge_test.cu on the engine: free
    energy, magnetic free energy and magnetic moment of the converged annulus
    against the London solution (1e-3, 2e-2, 1e-3); FP64 follows the oracle's
    first three iterations (1e-10)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    from tests.test_oracle_golden import radial_annulus_check
    cfg = configs.radial_annulus()
    e = sb.Context(cfg, mode=mode)
    n0 = e.dims.n0
    d = configs.phase_winding_state(n0, O.bulk_s_wave(0.2), -2.0)
    e.set_state(d, np.zeros((2, n0, n0)))
    if mode == "fp64":
        o = O.Oracle(cfg)
        o.set_state(d, np.zeros((2, n0, n0)))
        for it in range(3):
            o.compute()
            e.compute(1)
            assert _rel(e.state()[0], o.state()[0]) < TOL, it
            assert _rel(e.state()[1], o.state()[1]) < TOL, it
            assert _rel(e.results()[1], o.results()[1]) < TOL, it
    _, conv = e.run(0, 100)
    sc = e.scalars()
    moment = configs.magnetic_moment(e.results()[1], 1.0 / 6.2, int(sc["n_grain"]))
    radial_annulus_check(sc["free_energy_per_area"], sc["magnetic_free_energy_per_area"], moment, conv,
                         (sb.bulk_order_parameter_s_wave, sb.bulk_free_energy_s_wave, sb.bulk_yoshida_s_wave))
    e.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_iteration_graph_equals_eager(engine_lib, mode):
    """sc_compute replays steady iterations from a captured CUDA graph; with
    kernel profiling on it runs them eagerly.  Both give bit-identical states,
    results and scalars over eight CongAcc iterations of the disc in a field
    (vector potential solved); a change of the external field between calls
    and a new state written under a kept graph reach the replayed
    iterations."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfg = configs.small_disc()
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 8, 0.05, True, 0.05)
    out = []
    for eager in (False, True):
        e = sb.Context(cfg, mode=mode)
        if eager:
            e.profile(True)
        e.set_state(d, a)
        e.compute(3)
        b0 = e.external_field()
        e.set_external_field(1.5 * b0)
        e.compute(3)
        x_d, x_a = e.state()
        e.set_state(0.9 * x_d, x_a)  # new values under a kept graph
        e.compute(2)
        out.append((e.state(), e.results(), e.scalars(), e.launch_count()))
        e.close()
    (sg, rg, cg, lg), (se, re_, ce, le) = out
    for x, y in zip(sg + rg, se + re_):
        assert np.array_equal(x, y)
    assert cg == ce
    assert lg == le


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_compute_under_caller_capture(engine_lib, mode):
    """sc_compute on a stream that the caller is capturing into a CUDA graph.
    On a fresh context (no steady iteration yet) it returns SC_ERR_STATE and
    records nothing.  After one iteration it records steady iterations into
    the caller's graph and reads nothing back (residual and convergence flag
    untouched); three replays of a graph holding one iteration give the state,
    results and scalars of four eager iterations bit for bit."""
    import ctypes
    import torch
    import superconga_b200 as sb
    from oracle import oracle as O
    torch.cuda.set_device(0)
    cfg = configs.small_disc()
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 8, 0.05, True, 0.05)
    ref = sb.Context(cfg, mode=mode)
    ref.set_state(d, a)
    ref.compute(4)
    want = ref.state() + ref.results()
    want_scalars = ref.scalars()
    ref.close()

    e = sb.Context(cfg, mode=mode)
    stream = torch.cuda.Stream()
    e.set_stream(stream.cuda_stream)
    e.set_state(d, a)
    marker = torch.zeros(1, device="cuda")
    g0 = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g0, stream=stream):
        marker += 1.0
        st0 = engine_lib.sc_compute(e._h, 1, None, None)
    assert st0 == -3  # SC_ERR_STATE: nothing steady to record yet
    e.compute(1)
    g = torch.cuda.CUDAGraph()
    r, c = ctypes.c_double(-7.0), ctypes.c_int(-7)
    with torch.cuda.graph(g, stream=stream):
        st = engine_lib.sc_compute(e._h, 1, ctypes.byref(r), ctypes.byref(c))
    assert st == 0
    assert r.value == -7.0 and c.value == -7  # nothing read back under capture
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    got = e.state() + e.results()
    for x, y in zip(got, want):
        assert np.array_equal(x, y)
    assert e.scalars() == want_scalars
    del g, g0
    e.close()


def _many_energies_disc():
    """The small disc in a field with a self-consistent vector potential at
    T = 0.005 and cutoff 16: 89 Ozaki energies, more than one sweep pass
    takes, so the sweep runs three energy passes (32, 32, 25)."""
    cfg = configs.small_disc()
    cfg["physics"]["temperature"] = 0.005
    cfg["numerics"]["energy_cutoff"] = 16.0
    return cfg


def test_energy_passes_match_oracle(engine_lib):
    """Three iterations over three energy passes against the oracle: fields,
    free energy and every boundary value (1e-10)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    cfg = _many_energies_disc()
    o = O.Oracle(cfg)
    e = sb.Context(cfg, mode="fp64")
    assert e.dims.n_energies == 89
    s = o.setup
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 4, 0.05, True, 0.05)
    o.set_state(d, a)
    e.set_state(d, a)
    for it in range(3):
        o.compute()
        e.compute(1)
        d_o, j_o, a_o = o.results()
        d_e, j_e, a_e = e.results()
        assert _rel(d_e, d_o) < TOL, (it, "delta")
        assert _rel(j_e, j_o) < TOL, (it, "current")
        assert _rel(a_e, a_o) < TOL, (it, "vector potential")
        so, se = o.scalars(), e.scalars()
        assert abs(se["free_energy"] - so["free_energy"]) <= TOL * abs(so["free_energy"]), it
        for which in range(4):
            assert _rel(e.boundary(which), o.boundary(which)) < TOL, (it, which)
    e.close()


def test_energy_passes_mixed(engine_lib):
    """Mixed precision (mirror-paired angles) over three energy passes against
    FP64 after four iterations."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfg = _many_energies_disc()
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 6, 0.05, True, 0.05)
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


def test_mixed_precision(engine_lib):
    """FP32 stepping with FP64 accumulation against the FP64 form after five
    iterations: |Delta - Delta_FP64| / Delta_bulk <= 1e-5."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfg = configs.small_square_d()
    e64 = sb.Context(cfg, mode="fp64")
    e32 = sb.Context(cfg, mode="mixed")
    s = O.make_setup(cfg)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, 3, 0.1, True, 0.05)
    for e in (e64, e32):
        e.set_state(d, a)
        e.compute(5)
    d64, j64, a64 = e64.results()
    d32, j32, a32 = e32.results()
    assert np.max(np.abs(d32 - d64)) / db <= 1e-5
    assert _rel(j32, j64) <= 1e-4


def test_mixed_mirror_pairing(engine_lib, monkeypatch):
    """Mixed mode sweeps only half of the angles and obtains the other half from
    the particle-hole mirror (gammaTilde(theta) = conj(gamma(theta + pi))); the
    result agrees with sweeping every angle within the mixed-precision bound."""
    import superconga_b200 as sb
    from oracle import oracle as O
    for cfg in (configs.small_square_d(), configs.small_disc()):
        s = O.make_setup(cfg)
        db = O.delta_bulk(s.temperature, s.symmetries[0])
        d, a = configs.seeded_state(s.n_comp, s.n0, db, 4, 0.1, True, 0.05)
        out = []
        for pairing in (True, False):
            if pairing:
                monkeypatch.delenv("SCB_NO_PAIRING", raising=False)
            else:
                monkeypatch.setenv("SCB_NO_PAIRING", "1")
            e = sb.Context(cfg, mode="mixed")
            e.set_state(d, a)
            e.compute(3)
            out.append(e.results())
            e.close()
        (d1, j1, a1), (d2, j2, a2) = out
        assert np.max(np.abs(d1 - d2)) / db <= 1e-5
        assert _rel(j1, j2) <= 1e-4


@pytest.mark.parametrize("groups", [1, 2, 4, 8])
def test_group_sizes_match_oracle(engine_lib, monkeypatch, groups):
    """Every threads-per-column mapping (SCB_ENERGY_GROUPS: one thread holds
    all energies and stores the whole frame record; two share the record by
    halves; four and eight store one value each) against the oracle over two
    iterations in FP64 (1e-10), and in mixed precision against FP64 (1e-5 of
    the bulk gap)."""
    import superconga_b200 as sb
    cfg, kw = CASES["small_square_d"]
    monkeypatch.setenv("SCB_ENERGY_GROUPS", str(groups))
    o, e, db = _pair(cfg, **kw)
    m = sb.Context(cfg, mode="mixed")
    m.set_state(*e.state())
    for it in range(2):
        o.compute()
        e.compute(1)
        m.compute(1)
        d_o, j_o, _ = o.results()
        d_e, j_e, _ = e.results()
        assert _rel(d_e, d_o) < TOL, (groups, it, "delta")
        assert _rel(j_e, j_o) < TOL, (groups, it, "current")
        so, se = o.scalars(), e.scalars()
        assert abs(se["free_energy"] - so["free_energy"]) <= TOL * abs(so["free_energy"]), (groups, it)
        d_m = m.results()[0]
        assert np.max(np.abs(d_m - d_e)) / db <= 1e-5, (groups, it)
    e.close()
    m.close()

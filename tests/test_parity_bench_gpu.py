"""GPU parity at the benchmark sizes: the engine (through the C ABI) against
the CPU oracle on the seeded workloads the bench measures, so that the code
paths only large grains take are checked too:

* C1 (s-wave disc, N0 = 206, 64 angles, 7 energies, self-consistent A): three
  full iterations with accelerator steps, in one angle chunk and in several
  (a small scratch budget forces the chunked sweep), every field, scalar and
  boundary value;
* C2 (d-wave square, N0 = 606, N1 = 858, 256 angles, 14 energies): the frame
  Green sums of ten seeded angles, then one full iteration of all 256 angles,
  unchunked and in five chunks; mixed precision (mirror-paired sweep) against
  FP64 after the same iteration;
* C4 (chiral d + i d_xy disc, N0 = 456, two components, 128 angles, field):
  one frozen-boundary evaluation (the pass the adjoint differentiates).

FP64 agrees with the oracle to 1e-10 relative to the largest magnitude of each
compared field; mixed precision stays within 1e-5 of FP64 (relative to the
bulk gap for the order parameter, to the largest magnitude otherwise; the free
energy within 1e-6 of its largest term, see test_c2_mixed_against_fp64).
Reference: RiccatiSolverConfined.h:513-671, IntegrationIteratorOzaki.h:302-404,
Context.h:391-447.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-10
MIXED_TOL = 1e-5


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / scale)


def _workload(name):
    from superconga_b200 import workloads as W
    from oracle import oracle as O
    cfg = W.WORKLOADS[name]()
    o = O.Oracle(cfg)
    d, a = W.initial_state(name, cfg, o.n0)
    o.set_state(d, a)
    return cfg, o, d, a


def _engine(cfg, d, a, monkeypatch, scratch_mb=None, mode="fp64"):
    import superconga_b200 as sb
    if scratch_mb is None:
        monkeypatch.delenv("SCB_SCRATCH_MB", raising=False)
    else:
        monkeypatch.setenv("SCB_SCRATCH_MB", str(scratch_mb))
    e = sb.Context(cfg, mode=mode)
    e.set_state(d, a)
    return e


def _condensation_scale(cfg, x_delta):
    """|sum_c sum_r |Delta_c|^2 (ln(T/Tc_c) + T sum_n r_n / e_n)|, the largest
    term of the free energy (ComputeFreeEnergy.h:281-414).  On a rough start
    the free energy is a difference of terms about a hundred times larger than
    itself, so the mixed form's free energy is compared relative to this scale
    (the fields relative to their own magnitude)."""
    import math
    import superconga_b200 as sb
    e_im, res = sb.Setup(cfg).energies()
    t = cfg["physics"]["temperature"]
    si = float(np.sum(res / e_im))
    scale = 0.0
    for c, (_, comp) in enumerate(sorted(cfg["physics"]["order_parameter"].items(),
                                         key=lambda kv: ("dx2-y2", "dxy", "g", "s").index(kv[0]))):
        tc = comp.get("critical_temperature", 1.0)
        scale += float(np.sum(x_delta[c, 0] ** 2 + x_delta[c, 1] ** 2)) * (math.log(t / tc) + t * si)
    return abs(scale)


def _snapshot(ctx):
    """Everything an iteration produces: g(x), x, scalars, boundary values."""
    res = ctx.results()
    x = ctx.state()
    return {"results": res, "state": x, "scalars": ctx.scalars(),
            "boundary": [ctx.boundary(w) for w in range(4)]}


def _compare(got, want, tag, has_vp=True):
    (d_e, j_e, a_e), (d_o, j_o, a_o) = got["results"], want["results"]
    assert _rel(d_e, d_o) < TOL, (tag, "delta")
    assert _rel(j_e, j_o) < TOL, (tag, "current")
    if has_vp:
        assert _rel(a_e, a_o) < TOL, (tag, "vector potential")
    assert _rel(got["state"][0], want["state"][0]) < TOL, (tag, "x delta")
    if has_vp:
        assert _rel(got["state"][1], want["state"][1]) < TOL, (tag, "x A")
    se, so = got["scalars"], want["scalars"]
    for k in ("free_energy", "free_energy_per_area", "magnetic_free_energy"):
        assert abs(se[k] - so[k]) <= TOL * max(abs(so[k]), 1e-12), (tag, k, se[k], so[k])
    for k in ("res_order_parameter", "res_current", "res_free_energy", "res_boundary",
              "res_vector_potential", "residual"):
        assert abs(se[k] - so[k]) <= 1e-8 * max(abs(so[k]), 1e-12), (tag, k, se[k], so[k])
    for w in range(4):
        assert _rel(got["boundary"][w], want["boundary"][w]) < TOL, (tag, "boundary", w)


@pytest.fixture(scope="module")
def c1_reference():
    """The oracle's C1 run: the state after each of three iterations."""
    cfg, o, d, a = _workload("c1")
    snaps = []
    for _ in range(3):
        o.compute()
        snaps.append(_snapshot(o))
    return cfg, d, a, snaps


@pytest.mark.parametrize("scratch_mb", [None, 64], ids=["one_chunk", "chunked"])
def test_c1_iterations(engine_lib, c1_reference, monkeypatch, scratch_mb):
    cfg, d, a, snaps = c1_reference
    e = _engine(cfg, d, a, monkeypatch, scratch_mb)
    n_chunks, _ = e.sweep_plan()
    assert (n_chunks == 1) if scratch_mb is None else (n_chunks >= 4), n_chunks
    for it, want in enumerate(snaps):
        e.compute(1)
        _compare(_snapshot(e), want, ("c1", scratch_mb, it))
    e.close()


def test_c1_mixed_against_fp64(engine_lib, c1_reference, monkeypatch):
    """C1 in mixed precision (mirror-paired FP32 sweep) after the same three
    iterations: within 1e-5 of the oracle's FP64 run."""
    from superconga_b200 import workloads as W
    cfg, d, a, snaps = c1_reference
    e = _engine(cfg, d, a, monkeypatch, None, mode="mixed")
    assert e.sweep_plan() == (1, True)
    e.compute(3)
    (d_m, j_m, a_m), (d_o, j_o, a_o) = e.results(), snaps[-1]["results"]
    db = W.delta_bulk(cfg["physics"]["temperature"], "s")
    assert float(np.max(np.abs(d_m - d_o))) / db < MIXED_TOL
    assert _rel(j_m, j_o) < MIXED_TOL
    assert _rel(a_m, a_o) < MIXED_TOL
    fe_m, fe_o = e.scalars()["free_energy"], snaps[-1]["scalars"]["free_energy"]
    assert abs(fe_m - fe_o) <= MIXED_TOL * abs(fe_o)
    assert abs(fe_m - fe_o) <= 1e-6 * _condensation_scale(cfg, snaps[-1]["state"][0])
    e.close()


@pytest.fixture(scope="module")
def c2_reference():
    """The oracle's C2 frame Green sums of ten seeded angles (from the initial
    boundary values) and its first full iteration."""
    cfg, o, d, a = _workload("c2")
    na = o.setup.n_angles
    rng = np.random.default_rng(2)
    angles = sorted({0, na - 1, *rng.choice(na, size=8, replace=False).tolist()})
    o.set_boundary_initial()
    greens = {}
    for ang in angles:
        f, g, i, _ = o.angle_greens(ang)
        greens[ang] = (f, g, i)
    out_bnd = [o.boundary(1), o.boundary(3)]
    # The full iteration starts again from the initial boundary values.
    o.set_boundary_initial()
    o.compute()
    return cfg, d, a, greens, out_bnd, _snapshot(o)


def test_c2_angle_greens(engine_lib, c2_reference, monkeypatch):
    cfg, d, a, greens, out_bnd, _ = c2_reference
    e = _engine(cfg, d, a, monkeypatch)
    e.boundary_initial()
    for ang, (f_o, g_o, i_o) in greens.items():
        f_e, g_e, i_e = e.angle_greens(ang)
        assert _rel(f_e, f_o) < TOL, (ang, "F")
        assert _rel(g_e, g_o) < TOL, (ang, "G")
        assert _rel(i_e, i_o) < TOL, (ang, "I")
    # Out-going boundary values: the sampled angles swept, the others still at
    # their initial values, in both.
    assert _rel(e.boundary(1), out_bnd[0]) < TOL
    assert _rel(e.boundary(3), out_bnd[1]) < TOL
    e.close()


@pytest.mark.parametrize("scratch_mb", [None, 12000], ids=["one_chunk", "chunked"])
def test_c2_iteration(engine_lib, c2_reference, monkeypatch, scratch_mb):
    cfg, d, a, _, _, want = c2_reference
    e = _engine(cfg, d, a, monkeypatch, scratch_mb)
    n_chunks, _ = e.sweep_plan()
    assert (n_chunks == 1) if scratch_mb is None else (n_chunks >= 4), n_chunks
    e.compute(1)
    _compare(_snapshot(e), want, ("c2", scratch_mb))
    e.close()


def test_c2_mixed_against_fp64(engine_lib, c2_reference, monkeypatch):
    """One C2 iteration in mixed precision against the oracle's FP64 one.  On
    this start (10% complex noise on the bulk gap, T = 0.1) the free energy is
    a ~130x cancellation of its condensation and quasiparticle terms: its
    mixed-precision error is held to 1e-6 of the condensation term (measured
    on B200: 1.45e-5 of the free energy itself, 1e-7 of that term)."""
    from superconga_b200 import workloads as W
    cfg, d, a, _, _, want = c2_reference
    e = _engine(cfg, d, a, monkeypatch, None, mode="mixed")
    assert e.sweep_plan() == (1, True)
    e.compute(1)
    (d_m, j_m, a_m), (d_o, j_o, a_o) = e.results(), want["results"]
    db = W.delta_bulk(cfg["physics"]["temperature"], "dx2-y2")
    assert float(np.max(np.abs(d_m - d_o))) / db < MIXED_TOL
    assert _rel(j_m, j_o) < MIXED_TOL
    assert _rel(a_m, a_o) < MIXED_TOL
    fe_m, fe_o = e.scalars()["free_energy"], want["scalars"]["free_energy"]
    assert abs(fe_m - fe_o) <= 1e-6 * _condensation_scale(cfg, want["state"][0])
    e.close()


def test_c4_frozen_boundary_evaluation(engine_lib, monkeypatch):
    """C4: one frozen-boundary pass from the initial boundary values (the
    functional the adjoint differentiates): free energy, g(x) and j."""
    cfg, o, d, a = _workload("c4")
    o.set_boundary_initial()
    fe_o = o.evaluate()
    want = o.results()
    e = _engine(cfg, d, a, monkeypatch)
    e.boundary_initial()
    fe_e = e.evaluate()
    got = e.results()
    assert abs(fe_e - fe_o) <= TOL * abs(fe_o), (fe_e, fe_o)
    for x, y, tag in zip(got, want, ("delta", "current", "vector potential")):
        assert _rel(x, y) < TOL, tag
    e.close()

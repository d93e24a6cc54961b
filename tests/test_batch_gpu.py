"""Batched grains: the persistent multi-grain sweep, the CUDA-graph replay and
the autotuner give the results of the grains run one by one, and every grain
converges on its own."""
import numpy as np
import pytest

from tests import configs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / scale)


def _grains():
    cfgs = [configs.small_disc(), configs.small_square_d(), configs.chiral_annulus(),
            configs.golden_disc("picard")]
    states = []
    from oracle import oracle as O
    for i, c in enumerate(cfgs):
        s = O.make_setup(c)
        db = O.delta_bulk(s.temperature, s.symmetries[0])
        states.append(configs.seeded_state(s.n_comp, s.n0, db, 10 + i, 0.05, True, 0.02))
    return cfgs, states


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_matches_single(engine_lib, mode):
    import superconga_b200 as sb
    cfgs, states = _grains()
    b = sb.Batch(cfgs, mode=mode)
    singles = []
    for c, (d, a), g in zip(cfgs, states, b.grains):
        g.set_state(d, a)
        e = sb.Context(c, mode=mode)
        e.set_state(d, a)
        e.compute(4)
        singles.append(e)
    b.compute(4)  # iteration 1 eager, 2-4 graph replays
    tol = 1e-11 if mode == "fp64" else 1e-4
    for g, e in zip(b.grains, singles):
        d_b, j_b, a_b = g.results()
        d_s, j_s, a_s = e.results()
        assert _rel(d_b, d_s) < tol
        assert _rel(j_b, j_s) < 100 * tol
        assert abs(g.scalars()["free_energy"] - e.scalars()["free_energy"]) <= tol * abs(e.scalars()["free_energy"])
    act, it, _ = b.status()
    assert np.all(it == 4)
    b.close()


def test_batch_graph_equals_eager(engine_lib):
    import superconga_b200 as sb
    cfgs, states = _grains()
    out = []
    for graph in (True, False):
        b = sb.Batch(cfgs, mode="fp64")
        b.set_graph(graph)
        for g, (d, a) in zip(b.grains, states):
            g.set_state(d, a)
        b.compute(3)
        out.append([g.results()[0] for g in b.grains])
        b.close()
    for x, y in zip(*out):
        assert np.array_equal(x, y)


def test_batch_autotune(engine_lib):
    import superconga_b200 as sb
    cfgs, states = _grains()
    b = sb.Batch(cfgs, mode="fp64")
    for g, (d, a) in zip(b.grains, states):
        g.set_state(d, a)
    b.compute(1)
    ept, mb, ms = b.autotune()
    assert ept in (1, 2, 4, 8) and mb in (1, 4, 6) and ms > 0
    assert b.get_config()[:2] == (ept, mb)
    b.compute(2)
    ref = []
    for c, (d, a) in zip(cfgs, states):
        e = sb.Context(c, mode="fp64")
        e.set_state(d, a)
        e.compute(3)
        ref.append(e.results()[0])
    for g, r in zip(b.grains, ref):
        assert _rel(g.results()[0], r) < 1e-11
    b.close()


def test_batch_converges_independently(engine_lib):
    """Grains leave the batch when they converge; the golden disc reaches the
    reference's known free energy with two accelerators."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfgs = [configs.golden_disc("congacc"), configs.golden_disc("barzilai-borwein")]
    capped = configs.small_disc()
    capped["numerics"]["num_iterations_max"] = 5
    cfgs.append(capped)
    for c in cfgs[:2]:
        c["numerics"]["num_iterations_max"] = 100
    b = sb.Batch(cfgs, mode="fp64")
    for g in b.grains[:2]:
        n0 = g.dims.n0
        d = np.zeros((1, 2, n0, n0))
        d[0, 0] = O.delta_bulk(0.5, "s")
        g.set_state(d, np.zeros((2, n0, n0)))
    s = O.make_setup(capped)
    d, a = configs.seeded_state(1, s.n0, O.delta_bulk(0.5, "s"), 1, 0.01, False, 0.0)
    b.grains[2].set_state(d, a)
    left = b.compute(200)
    assert left == 0
    act, it, res = b.status()
    assert not act.any()
    assert it[2] == 5
    for k in range(2):
        assert res[k] < 1e-5 and it[k] < 100
        fe = b.grains[k].scalars()["free_energy_per_area"]
        assert abs(fe - configs.GOLDEN_FREE_ENERGY_PER_AREA) <= 1e-3 * abs(configs.GOLDEN_FREE_ENERGY_PER_AREA)
    b.close()


def test_batch_vs_oracle(engine_lib):
    """Seeded grains of the batched workload (coarsened to 3 points/xi0 so the
    CPU oracle runs them in seconds), advanced together in one FP64 batch,
    against the oracle run grain by grain: two iterations within 1e-10."""
    import superconga_b200 as sb
    from oracle import oracle as O
    from superconga_b200 import workloads
    cfgs, states = workloads.c3_grains(128, ppxi=3.0)
    pick = [0, 1, 64, 65]  # two discs, two squares
    cfgs = [cfgs[i] for i in pick]
    states = [states[i] for i in pick]
    b = sb.Batch(cfgs, mode="fp64")
    oracles = []
    for g, c, st in zip(b.grains, cfgs, states):
        d, a = workloads.c3_initial_state(c, st, g.dims.n0)
        g.set_state(d, a)
        o = O.Oracle(c)
        o.set_state(d, a)
        oracles.append(o)
    for it in range(2):
        b.compute(1)
        for o in oracles:
            o.compute()
        for g, o in zip(b.grains, oracles):
            d_b, j_b, _ = g.results()
            d_o, j_o, _ = o.results()
            assert _rel(d_b, d_o) < 1e-10, it
            assert _rel(j_b, j_o) < 1e-10, it
            assert abs(g.scalars()["free_energy"] - o.scalars()["free_energy"]) <= 1e-10 * abs(o.scalars()["free_energy"])
    b.close()


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_batch_low_temperature_grains(engine_lib, mode):
    """A temperature sweep in one batch: the small disc at T = 0.5 (7 Ozaki
    energies), T = 0.01 at cutoff 8 (45: one pass, eight energies per thread
    for some threads) and T = 0.005 at cutoff 16 (89: three energy passes of
    32, 32 and 25) give the results of the same grains run on their own."""
    import superconga_b200 as sb
    from oracle import oracle as O
    cfgs = []
    for t, cut in ((0.5, 8.0), (0.01, 8.0), (0.005, 16.0)):
        c = configs.small_disc()
        c["physics"]["temperature"] = t
        c["numerics"]["energy_cutoff"] = cut
        cfgs.append(c)
    states = []
    for i, c in enumerate(cfgs):
        s = O.make_setup(c)
        db = O.delta_bulk(s.temperature, s.symmetries[0])
        states.append(configs.seeded_state(s.n_comp, s.n0, db, 20 + i, 0.05, True, 0.02))
    b = sb.Batch(cfgs, mode=mode)
    assert [g.dims.n_energies for g in b.grains] == [7, 45, 89]
    for g, (d, a) in zip(b.grains, states):
        g.set_state(d, a)
    b.compute(3)  # iteration 1 eager, 2-3 graph replays
    tol = 1e-11 if mode == "fp64" else 1e-4
    for g, c, (d, a) in zip(b.grains, cfgs, states):
        e = sb.Context(c, mode=mode)
        e.set_state(d, a)
        e.compute(3)
        assert _rel(g.results()[0], e.results()[0]) < tol
        assert _rel(g.results()[1], e.results()[1]) < 100 * tol
        assert abs(g.scalars()["free_energy"] - e.scalars()["free_energy"]) <= tol * abs(e.scalars()["free_energy"])
        e.close()
    b.close()


def test_diverged_grain_is_frozen_and_reported(engine_lib):
    """A grain whose order parameter holds a NaN (written on the host through
    its context's set_state; no fault of any kind on the GPU) is reported as
    diverged after its first iteration and frozen there, while the other
    grains continue and give the results of a batch without it."""
    import superconga_b200 as sb
    cfgs, states = _grains()
    bad = 1
    d_bad = states[bad][0].copy()
    n0 = d_bad.shape[-1]
    d_bad[0, 0, n0 // 2, n0 // 2] = np.nan  # a site inside the grain
    b = sb.Batch(cfgs, mode="fp64")
    for i, (g, (d, a)) in enumerate(zip(b.grains, states)):
        g.set_state(d_bad if i == bad else d, a)
    b.compute(3)
    st = b.grain_states()
    act, it, res = b.status()
    assert st[bad] == "diverged"
    assert it[bad] == 1 and not act[bad] and not np.isfinite(res[bad])
    assert all(s == "running" for i, s in enumerate(st) if i != bad)
    assert all(it[i] == 3 for i in range(len(cfgs)) if i != bad)
    keep = [i for i in range(len(cfgs)) if i != bad]
    b2 = sb.Batch([cfgs[i] for i in keep], mode="fp64")
    for g, i in zip(b2.grains, keep):
        g.set_state(*states[i])
    b2.compute(3)
    for g2, i in zip(b2.grains, keep):
        for x, y in zip(b.grains[i].results(), g2.results()):
            assert _rel(x, y) < 1e-12
    b.close()
    b2.close()


def test_nan_state_never_reads_as_converged(engine_lib):
    """One context with a NaN in its order parameter: the residual of the
    iteration is not finite and the iteration does not report convergence
    (the residual maxima keep NaNs; an fmax would drop them)."""
    import superconga_b200 as sb
    cfgs, states = _grains()
    for norm in ("l2", "linf"):
        cfg = dict(cfgs[0])
        cfg["numerics"] = dict(cfg["numerics"], norm=norm)
        d, a = (x.copy() for x in states[0])
        n0 = d.shape[-1]
        d[0, 1, n0 // 2, n0 // 2] = np.nan
        e = sb.Context(cfg, mode="fp64")
        e.set_state(d, a)
        res, conv = e.compute(2)
        assert not np.isfinite(res) and not conv, norm
        e.close()

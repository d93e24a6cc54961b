"""The hand-written adjoint of the frozen-boundary free energy (and of a
linear functional of the current) against central finite differences of the
engine and of the CPU oracle, and through torch.autograd."""
import numpy as np
import pytest

from tests import configs

pytestmark = pytest.mark.gpu

# Central differences along random directions whose entries are of order
# Delta_bulk (order-parameter part), 0.05 (vector potential) and 0.01 (field).
# The step 1e-4 perturbs each site by ~3e-5 Delta_bulk: small enough that the
# truncation error stays below 1e-7 relative, large enough that the rounding
# error of the free energy (a sum over the whole grain) does not swamp small
# directional derivatives, as it does for steps of 1e-6 and below.
EPS = 1e-4
TOL = 1e-6  # relative agreement of directional derivatives


CASES = {
    "small_disc": configs.small_disc(),
    "chiral_annulus": configs.chiral_annulus(),
    "small_square_d": configs.small_square_d(),
}


def _setup(cfg, seed=5):
    import superconga_b200 as sb
    from oracle import oracle as O
    e = sb.Context(cfg, mode="fp64")
    o = O.Oracle(cfg)
    s = o.setup
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    d, a = configs.seeded_state(s.n_comp, s.n0, db, seed, 0.1, True, 0.05)
    e.set_state(d, a)
    o.set_state(d, a)
    for _ in range(3):
        e.burn_in(1)
        o.burn_in()
    dom = e.domain() > 0
    return e, o, d * dom, a, db, dom


def _directions(rng, d, a, dom, db, k):
    for _ in range(k):
        vd = rng.standard_normal(d.shape) * db * dom
        va = rng.standard_normal(a.shape) * 0.05
        vb = float(rng.standard_normal()) * 0.01
        yield vd, va, vb


def _engine_f(e, d, a, b, beta=None):
    e.set_state(d, a)
    e.set_external_field(b)
    fe = e.evaluate()
    if beta is None:
        return fe
    return float(np.sum(beta * e.results()[1]))


@pytest.mark.parametrize("case", list(CASES))
def test_adjoint_free_energy_vs_fd(engine_lib, case):
    e, o, d, a, db, dom = _setup(CASES[case])
    b0 = e.external_field()
    e.evaluate()
    gd, ga, gb = e.adjoint(1.0)
    assert np.all(gd[:, :, ~dom] == 0.0)
    rng = np.random.default_rng(11)
    for vd, va, vb in _directions(rng, d, a, dom, db, 4):
        fp = _engine_f(e, d + EPS * vd, a + EPS * va, b0 + EPS * vb)
        fm = _engine_f(e, d - EPS * vd, a - EPS * va, b0 - EPS * vb)
        fd = (fp - fm) / (2 * EPS)
        ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
        assert abs(fd - ad) <= TOL * max(abs(ad), abs(fd)), (case, fd, ad)


def test_adjoint_edge_current_vs_fd(engine_lib):
    from superconga_b200.autograd import edge_current_weights
    cfg = CASES["small_disc"]
    e, o, d, a, db, dom = _setup(cfg)
    h = 1.0 / cfg["numerics"]["points_per_coherence_length"]
    beta = edge_current_weights(e.domain(), h, 2.0)
    b0 = e.external_field()
    e.evaluate()
    gd, ga, gb = e.adjoint(0.0, beta)
    rng = np.random.default_rng(12)
    for vd, va, vb in _directions(rng, d, a, dom, db, 3):
        fp = _engine_f(e, d + EPS * vd, a + EPS * va, b0 + EPS * vb, beta)
        fm = _engine_f(e, d - EPS * vd, a - EPS * va, b0 - EPS * vb, beta)
        fd = (fp - fm) / (2 * EPS)
        ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
        assert abs(fd - ad) <= TOL * max(abs(ad), abs(fd)), (fd, ad)


@pytest.mark.parametrize("case", ["small_disc", "chiral_annulus"])
def test_adjoint_vs_oracle_fd(engine_lib, case):
    """The engine's adjoint against finite differences of the CPU oracle."""
    cfg = CASES[case]
    e, o, d, a, db, dom = _setup(cfg)
    import math
    area = o.setup.h ** 2 * float(np.count_nonzero(o.domain()))
    b0 = e.external_field()
    e.evaluate()
    gd, ga, gb = e.adjoint(1.0)
    rng = np.random.default_rng(13)
    for vd, va, vb in _directions(rng, d, a, dom, db, 2):
        vals = []
        for s in (1.0, -1.0):
            o.set_state(d + s * EPS * vd, a + s * EPS * va)
            o.set_flux((b0 + s * EPS * vb) * area / math.pi)
            vals.append(o.evaluate())
        fd = (vals[0] - vals[1]) / (2 * EPS)
        ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
        assert abs(fd - ad) <= TOL * max(abs(ad), abs(fd)), (case, fd, ad)


def test_autograd_function(engine_lib):
    import torch
    from superconga_b200.autograd import FreeEnergy
    cfg = CASES["chiral_annulus"]
    e, o, d, a, db, dom = _setup(cfg)
    delta = torch.tensor(d[:, 0] + 1j * d[:, 1], dtype=torch.complex128, requires_grad=True)
    av = torch.tensor(a, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(e.external_field(), dtype=torch.float64, requires_grad=True)
    loss = FreeEnergy.apply(delta, av, b, e, 1.0, None)
    loss.backward()
    gd, ga, gb = e.adjoint(1.0)
    assert np.allclose(delta.grad.numpy(), gd[:, 0] + 1j * gd[:, 1], rtol=0, atol=1e-14)
    assert np.allclose(av.grad.numpy(), ga, rtol=0, atol=1e-14)
    assert abs(float(b.grad) - gb) <= 1e-14 * max(1.0, abs(gb))
    # a step along -grad lowers the loss (first order)
    with torch.no_grad():
        step = 1e-4 / max(float(delta.grad.abs().max()), 1e-30)
        loss2 = FreeEnergy.apply(delta - step * delta.grad, av, b, e, 1.0, None)
    assert float(loss2.detach()) < float(loss.detach())


@pytest.mark.parametrize("temperature,cutoff,n_energies", [(0.01, 8.0, 45), (0.005, 16.0, 89)])
def test_adjoint_energy_passes_vs_fd(engine_lib, temperature, cutoff, n_energies):
    """The adjoint over energy passes of four energies per thread (45
    energies: two passes; 89: three, beside the forward sweep's own passes)
    against central differences of the engine."""
    cfg = configs.small_disc()
    cfg["physics"]["temperature"] = temperature
    cfg["numerics"]["energy_cutoff"] = cutoff
    e, o, d, a, db, dom = _setup(cfg)
    assert e.dims.n_energies == n_energies
    b0 = e.external_field()
    e.evaluate()
    gd, ga, gb = e.adjoint(1.0)
    rng = np.random.default_rng(17)
    for vd, va, vb in _directions(rng, d, a, dom, db, 3):
        fp = _engine_f(e, d + EPS * vd, a + EPS * va, b0 + EPS * vb)
        fm = _engine_f(e, d - EPS * vd, a - EPS * va, b0 - EPS * vb)
        fd = (fp - fm) / (2 * EPS)
        ad = float(np.sum(gd * vd) + np.sum(ga * va) + gb * vb)
        assert abs(fd - ad) <= TOL * max(abs(ad), abs(fd)), (fd, ad)

"""Host-side setup of the engine (no GPU): the static tables built by
libscb200's set-up code against the CPU oracle's restatement."""
import numpy as np
import pytest

from tests import configs

CASES = {
    "golden_disc": configs.golden_disc(),
    "small_disc": configs.small_disc(),
    "small_square_d": configs.small_square_d(),
    "chiral_annulus": configs.chiral_annulus(),
}


@pytest.fixture(scope="module")
def both():
    from superconga_b200 import build
    build.build()
    from oracle import oracle as O
    import superconga_b200 as sb
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = (O.Oracle(CASES[name]), sb.Setup(CASES[name]))
        return cache[name]
    return get


@pytest.mark.parametrize("case", list(CASES))
def test_lattice_and_energies(both, case):
    o, s = both(case)
    assert (s.dims.n0, s.dims.n1, s.dims.n_angles) == (o.n0, o.n1, o.setup.n_angles)
    assert s.dims.n_energies == o.setup.n_energies
    e, r = s.energies()
    # Own tridiagonal QL solver against LAPACK dsygv.
    assert np.max(np.abs(e - o.setup.energies_im) / o.setup.energies_im) < 1e-12
    assert np.max(np.abs(r - o.setup.residues) / o.setup.residues) < 1e-12


@pytest.mark.parametrize("case", list(CASES))
def test_geometry_tables(both, case):
    o, s = both(case)
    assert np.array_equal(s.domain(), o.domain())
    assert s.boundary_sizes() == o.boundary_sizes()
    x0, x1, y0, y1 = o.ranges()
    for a in range(s.dims.n_angles):
        lab, box = s.frame(a)
        assert np.array_equal(lab, o.geometry(a)[0]), a
        assert box == (x0[a], x1[a], y0[a], y1[a]), a


@pytest.mark.parametrize("case", ["golden_disc", "small_square_d"])
def test_poisson_filters(both, case):
    o, s = both(case)
    f, pos, scale = s.filters()
    assert f.shape == o.setup.filters.shape
    assert np.array_equal(pos, o.setup.filter_pos)
    assert abs(scale - o.setup.vp_scale) <= 1e-12 * o.setup.vp_scale
    for k in range(len(f)):
        # eigenvectors are defined up to sign; small eigenvalues have less
        # accurate eigenvectors
        err = min(np.max(np.abs(f[k] - o.setup.filters[k])), np.max(np.abs(f[k] + o.setup.filters[k])))
        assert err < 1e-8 * np.max(np.abs(o.setup.filters[k]))
    # The separable kernel they assemble, sum_k (+/-) f_k(dx) f_k(dy), is
    # independent of signs and of rotations inside degenerate eigenspaces.
    sign = np.where(pos > 0, 1.0, -1.0)
    k_e = np.einsum("k,ki,kj->ij", sign, f, f)
    k_o = np.einsum("k,ki,kj->ij", sign, o.setup.filters, o.setup.filters)
    assert np.max(np.abs(k_e - k_o)) <= 1e-11 * np.max(np.abs(k_o))


def test_site_update_count(both):
    o, s = both("small_disc")
    inside = sum(int(np.count_nonzero(o.geometry(a)[0] > 0)) for a in range(o.setup.n_angles))
    assert s.site_updates() == 2 * o.setup.n_energies * inside


def test_config_errors():
    """Bad configurations are reported through the status code, never by
    exiting (the reference exits in geometry_utils.h:105,160)."""
    import superconga_b200 as sb
    bad = configs.small_disc()
    bad["numerics"]["norm"] = "l3"
    with pytest.raises(sb.EngineError, match="norm"):
        sb.Setup(bad)
    bad = configs.small_disc()
    bad["geometry"] = [{"ellipse": {"add": True}}]
    with pytest.raises(sb.EngineError, match="unknown geometry"):
        sb.Setup(bad)
    with pytest.raises(sb.EngineError):
        sb.Setup("{not json")
    bad = configs.small_disc()
    bad["physics"]["order_parameter"] = {}
    with pytest.raises(sb.EngineError, match="order-parameter"):
        sb.Setup(bad)

"""GPU parity of the LDOS postprocess: the CUDA engine (through the C ABI)
against the CPU oracle on the same seeded state, FP64 to 1e-10 relative."""
import numpy as np
import pytest

from tests import configs

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _rel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / scale)


def _pair(sim, pp, mode="fp64", seed=1, a_scale=0.05):
    from oracle import oracle as O
    import superconga_b200 as sb
    s = O.make_setup(sim)
    db = O.delta_bulk(s.temperature, s.symmetries[0])
    L = O.LdosOracle(sim, pp)
    e = sb.LdosContext(sim, pp, mode=mode)
    d, a = configs.seeded_state(s.n_comp, s.n0, db, seed, 0.05, True, a_scale)
    L.set_state(d, a)
    e.set_state(d, a)
    return L, e, db


def test_ldos_blocks(engine_lib):
    """Both blocks (the second one short): burn-in, then LDOS iterations."""
    sim = configs.small_disc()
    from oracle import oracle as O
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=12, per_block=8, n_angles=32)
    L, e, _ = _pair(sim, pp)
    en, delta = e.energies()
    assert np.allclose(en, L.energies, rtol=0, atol=1e-15) and delta == pp["spectroscopy"]["energy_broadening"]
    for b in range(2):
        L.begin_block(b)
        e.begin_block(b)
        for _ in range(2):
            rb_o = L.burn_in()
            rb_e, _ = e.burn_in(1)
            assert abs(rb_e - rb_o) <= 1e-8 * rb_o
        for it in range(3):
            r_o, rl_o, _ = L.iterate()
            r_e, _ = e.iterate(1)
            assert abs(r_e - r_o) <= 1e-8 * r_o, (b, it, r_e, r_o)
            assert abs(e.scalars()["res_vector_potential"] - rl_o) <= 1e-8 * rl_o
        for which in range(4):
            assert _rel(e.boundary(which), L.oracle.boundary(which)) < TOL
    assert _rel(e.ldos(), L.ldos) < TOL


def test_ldos_block_passes(engine_lib):
    """A block of 80 real energies, more than one sweep pass takes (64), is
    swept in passes of 32, 32 and 16 into one LDOS frame; the block and the
    short one after it (20 energies) match the oracle (1e-10)."""
    sim = configs.small_disc()
    from oracle import oracle as O
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=100, per_block=80, n_angles=32)
    L, e, _ = _pair(sim, pp)
    for b in range(2):
        L.begin_block(b)
        e.begin_block(b)
        L.burn_in()
        e.burn_in(1)
        for it in range(2):
            r_o, _, _ = L.iterate()
            r_e, _ = e.iterate(1)
            assert abs(r_e - r_o) <= 1e-8 * r_o, (b, it, r_e, r_o)
        for which in range(4):
            assert _rel(e.boundary(which), L.oracle.boundary(which)) < TOL
    assert _rel(e.ldos(), L.ldos) < TOL


@pytest.mark.parametrize("scratch_mb", [None, 1], ids=["one_chunk", "chunked"])
def test_ldos_d_wave_square(engine_lib, monkeypatch, scratch_mb):
    """d-wave square with pair-breaking edges, vector potential, two blocks;
    once with all angles in one chunk and once in many (a 1 MB budget): the
    LDOS frame buffer is reused across chunks and iterations without being
    cleared, and the LDOS inside the grain must not depend on it."""
    sim = configs.small_square_d()
    from oracle import oracle as O
    if scratch_mb is None:
        monkeypatch.delenv("SCB_SCRATCH_MB", raising=False)
    else:
        monkeypatch.setenv("SCB_SCRATCH_MB", str(scratch_mb))
    db = O.delta_bulk(0.1, "dx2-y2")
    pp = configs.ldos_postprocess(db, n_energies=16, per_block=8, n_angles=24, broadening=0.03)
    L, e, _ = _pair(sim, pp, seed=3)
    n_chunks, _ = e.sweep_plan()
    assert (n_chunks == 1) if scratch_mb is None else (n_chunks >= 4), n_chunks
    for b in range(2):
        L.begin_block(b)
        e.begin_block(b)
        L.burn_in()
        e.burn_in(1)
        for _ in range(2):
            L.iterate()
            e.iterate(1)
    assert _rel(e.ldos(), L.ldos) < TOL


def test_ldos_run_converges(engine_lib):
    """runPostprocess on the engine against the oracle's block loop."""
    sim = configs.small_disc()
    from oracle import oracle as O
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=6, per_block=4, n_angles=16, crit=1e-6)
    L, e, _ = _pair(sim, pp)
    n_it = 0
    for b in range(L.n_blocks):
        L.begin_block(b)
        for _ in range(2):
            L.burn_in()
            n_it += 1
        for i in range(1, 61):
            r, _, _ = L.iterate()
            n_it += 1
            if r < 1e-6:
                break
    conv, it = e.run(2, 0, 60)
    assert conv and it == n_it
    assert _rel(e.ldos(), L.ldos) < TOL


def test_ldos_bcs_bulk(engine_lib):
    """Uniform s-wave, no field: the engine's LDOS is the broadened BCS density
    of states at every grain site."""
    import superconga_b200 as sb
    from oracle import oracle as O
    sim = configs.small_disc()
    sim["physics"]["external_flux_quanta"] = 0.0
    sim["physics"]["penetration_depth"] = -1.0
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=8, per_block=8, n_angles=16, broadening=0.04)
    for mode, tol in (("fp64", 1e-9), ("mixed", 1e-4)):
        e = sb.LdosContext(sim, pp, mode=mode)
        n0 = e.dims.n0
        d = np.zeros((1, 2, n0, n0))
        d[0, 0] = db
        e.set_state(d, np.zeros((2, n0, n0)))
        e.begin_block(0)
        e.burn_in(1)
        e.iterate(1)
        ld = e.ldos()
        dom = e.domain() > 0
        en, _ = e.energies()
        want = configs.bcs_dos(en, 0.04, db)
        for k in range(len(en)):
            assert np.max(np.abs(ld[k][dom] - want[k])) < tol * max(1.0, want[k]), (mode, k)
        e.close()


def test_ldos_mixed(engine_lib):
    """FP32 stepping against FP64 on the seeded state."""
    sim = configs.small_disc()
    from oracle import oracle as O
    import superconga_b200 as sb
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=8, per_block=8, n_angles=32)
    out = []
    for mode in ("fp64", "mixed"):
        e = sb.LdosContext(sim, pp, mode=mode)
        d, a = configs.seeded_state(1, e.dims.n0, db, 1, 0.05, True, 0.05)
        e.set_state(d, a)
        e.begin_block(0)
        e.burn_in(2)
        e.iterate(3)
        out.append(e.ldos())
        e.close()
    assert _rel(out[1], out[0]) < 1e-4


@pytest.mark.parametrize("swave", [True, False], ids=["s-wave disc", "d-wave square"])
@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_reference_dos(engine_lib, swave, mode):
    """tests/physics/dos_test.cu:211-240 on the engine: the grain-averaged LDOS
    converges within 42 iterations and matches the bulk DOS to 1e-8 (FP64,
    criterion 1e-8); mixed precision takes the reference's single-precision
    case (criterion 1e-4, bound 1e-5)."""
    from oracle import oracle as O
    import superconga_b200 as sb
    sim, pp = configs.dos_test_case(swave)
    if mode == "mixed":
        sim["numerics"]["convergence_criterion"] = 1e-4
        pp["numerics"]["convergence_criterion"] = 1e-4
    e = sb.LdosContext(sim, pp, mode=mode)
    n0 = e.dims.n0
    db = O.delta_bulk(0.5, "s" if swave else "dx2-y2")
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = db
    e.set_state(d, np.zeros((2, n0, n0)))
    conv, it = e.run(0, 0, 42)
    assert conv
    en, _ = e.energies()
    ldos = e.ldos()
    dom = e.domain() > 0
    got = np.array([ldos[k][dom].mean() for k in range(len(en))])
    want = configs.bulk_dos(np.asarray(en), 0.008, db, swave, 160)
    tol = 1e-8 if mode == "fp64" else 1e-5
    assert np.max(np.abs(got - want) / (1.0 + np.abs(want))) < tol

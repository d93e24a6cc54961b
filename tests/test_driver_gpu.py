"""The drop-in simulation executable (superconga_b200/bin/simulation_b200):
the reference's JSON configuration in, the reference's output files out
(src/simulation.cu, SimulationWriter.h:57-246)."""
import csv
import json
import os
import subprocess

import pytest

from tests import configs

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "superconga_b200", "bin", "simulation_b200")


def _run(cfg, tmp_path):
    path = tmp_path / "simulation_config.json"
    path.write_text(json.dumps(cfg))
    return subprocess.run([EXE, str(path)], capture_output=True, text=True, timeout=600)


def test_driver_golden_disc(engine_lib, tmp_path):
    cfg = configs.golden_disc("congacc")
    cfg["physics"]["order_parameter"]["s"].update({"initial_noise_stddev": 0.0,
                                                  "initial_phase_shift": 0.0, "vortices": []})
    cfg["numerics"].update({"num_iterations_burnin": 0, "num_iterations_min": 0,
                            "num_iterations_max": 100})
    out = tmp_path / "out"
    cfg["misc"] = {"save_path": str(out), "save_frequency": -1, "load_path": "",
                   "verbose": False, "data_format": "csv"}
    r = _run(cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    for name in ("domain.csv", "order_parameter.csv", "current_density.csv",
                 "vector_potential.csv", "magnetic_flux_density.csv", "simulation_config.json",
                 "simulation_results.json", "internal_parameters.json",
                 "simulation_convergence.csv"):
        assert (out / name).exists(), name
    res = json.loads((out / "simulation_results.json").read_text())
    fe = res["free_energy_per_unit_area"]
    assert abs(fe - configs.GOLDEN_FREE_ENERGY_PER_AREA) <= 1e-3 * abs(configs.GOLDEN_FREE_ENERGY_PER_AREA)
    with open(out / "order_parameter.csv") as f:
        rows = list(csv.reader(f))
    assert rows[0] == ["x_idx", "y_idx", "s_re", "s_im"]
    n0 = int(round(len(rows[1:]) ** 0.5))
    assert n0 * n0 == len(rows) - 1
    conv = list(csv.reader(open(out / "simulation_convergence.csv")))
    assert conv[0][0] == "iteration" and len(conv) > 2
    # Continue from the written state: load_path reads the files back
    # (src/simulation.cu:300-377) and the first iteration stays converged.
    cfg2 = json.loads(json.dumps(cfg))
    cfg2["misc"]["load_path"] = str(out)
    cfg2["misc"]["save_path"] = str(tmp_path / "out2")
    cfg2["numerics"]["num_iterations_max"] = 3
    r2 = _run(cfg2, tmp_path)
    assert r2.returncode == 0, r2.stderr
    res2 = json.loads((tmp_path / "out2" / "simulation_results.json").read_text())
    assert abs(res2["free_energy_per_unit_area"] - fe) <= 1e-4 * abs(fe)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_driver_low_temperature(engine_lib, tmp_path, precision):
    """The d_{x2-y2} square of tests/physics/low_temp_free_energy_test.cu (T =
    0.001, cutoff 32: 281 Ozaki energies, swept in energy passes) run by the
    drop-in executable from the reference's JSON: converged within 50
    iterations, free energy per area within 1e-4 of the bulk value
    -D_WAVE_BULK^2 / 2 and mean gap within 1e-5 of D_WAVE_BULK."""
    from oracle.oracle import D_WAVE_BULK
    cfg = configs.low_temperature_bulk(swave=False, disc=False)
    cfg["physics"]["order_parameter"]["dx2-y2"].update({"initial_noise_stddev": 0.0,
                                                        "initial_phase_shift": 0.0, "vortices": []})
    cfg["numerics"].update({"num_iterations_burnin": 0, "num_iterations_min": 1,
                            "num_iterations_max": 50})
    out = tmp_path / "out"
    cfg["misc"] = {"save_path": str(out), "save_frequency": -1, "load_path": "",
                   "verbose": False, "data_format": "csv"}
    if precision == "mixed":
        cfg["b200"] = {"precision": "mixed"}
    r = _run(cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    conv = list(csv.reader(open(out / "simulation_convergence.csv")))
    last = [float(v) for v in conv[-1][1:6]]
    assert len(conv) - 1 <= 50 and max(last) < 1e-3, conv[-1]
    res = json.loads((out / "simulation_results.json").read_text())
    expected = -0.5 * D_WAVE_BULK * D_WAVE_BULK
    assert abs(res["free_energy_per_unit_area"] - expected) <= 1e-4 * abs(expected), res
    assert abs(res["order_parameter_average_magnitude"] - D_WAVE_BULK) <= 1e-5 * D_WAVE_BULK, res


def test_driver_load_other_lattice(engine_lib, tmp_path):
    """A run saved at 3 points/xi0 continued at 4 points/xi0: the order
    parameter is extended past the grain and resampled onto the finer lattice
    (csv.h:297-395); the continued run reaches the free energy of a run started
    afresh on the fine lattice, in fewer iterations."""
    cfg = configs.golden_disc("congacc")
    cfg["physics"]["order_parameter"]["s"].update({"initial_noise_stddev": 0.0,
                                                  "initial_phase_shift": 0.0, "vortices": []})
    cfg["numerics"].update({"num_iterations_burnin": 0, "num_iterations_min": 0,
                            "num_iterations_max": 100})
    coarse = tmp_path / "coarse"
    cfg["misc"] = {"save_path": str(coarse), "save_frequency": -1, "load_path": "",
                   "verbose": False, "data_format": "csv"}
    assert _run(cfg, tmp_path).returncode == 0
    fine_cfg = json.loads(json.dumps(cfg))
    fine_cfg["numerics"]["points_per_coherence_length"] = 4.0
    fine_cfg["misc"]["load_path"] = str(coarse)
    fine_cfg["misc"]["save_path"] = str(tmp_path / "fine")
    r = _run(fine_cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    # the same fine configuration from the default start
    fresh_cfg = json.loads(json.dumps(fine_cfg))
    fresh_cfg["misc"]["load_path"] = ""
    fresh_cfg["misc"]["save_path"] = str(tmp_path / "fresh")
    assert _run(fresh_cfg, tmp_path).returncode == 0
    fe = [json.loads((tmp_path / d / "simulation_results.json").read_text())["free_energy_per_unit_area"]
          for d in ("fine", "fresh")]
    assert abs(fe[0] - fe[1]) <= 1e-4 * abs(fe[1])
    its = [len(list(csv.reader(open(tmp_path / d / "simulation_convergence.csv")))) - 1 for d in ("fine", "fresh")]
    assert its[0] < its[1]  # the resampled state starts closer to the solution


def test_driver_bad_config(engine_lib, tmp_path):
    cfg = configs.golden_disc()
    cfg["numerics"]["norm"] = "l7"
    r = _run(cfg, tmp_path)
    assert r.returncode != 0
    assert "norm" in r.stderr


PP_EXE = os.path.join(ROOT, "superconga_b200", "bin", "postprocess_b200")


def test_postprocess_driver(engine_lib, tmp_path):
    """simulation_b200 writes a run, postprocess_b200 reads it back
    (src/postprocess.cu:86-360) and writes ldos.csv; the LDOS agrees with the
    oracle's postprocess of the same files."""
    import numpy as np
    from oracle import oracle as O
    cfg = configs.small_disc()
    cfg["physics"]["order_parameter"]["s"].update({"initial_noise_stddev": 0.0,
                                                  "initial_phase_shift": 0.0, "vortices": []})
    cfg["numerics"].update({"num_iterations_burnin": 0, "num_iterations_min": 0,
                            "num_iterations_max": 4})
    sim_out = tmp_path / "sim"
    cfg["misc"] = {"save_path": str(sim_out), "save_frequency": -1, "load_path": "",
                   "verbose": False, "data_format": "csv"}
    r = _run(cfg, tmp_path)
    assert r.returncode == 0, r.stderr
    db = O.delta_bulk(0.5, "s")
    pp = configs.ldos_postprocess(db, n_energies=6, per_block=4, n_angles=16, crit=1e-6)
    pp["misc"] = {"data_format": "csv", "load_path": str(sim_out), "save_path": str(tmp_path / "pp"),
                  "verbose": False}
    ppath = tmp_path / "postprocess_config.json"
    ppath.write_text(json.dumps(pp))
    r = subprocess.run([PP_EXE, str(ppath)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    for name in ("ldos.csv", "postprocess_config.json", "postprocess_convergence.csv"):
        assert (tmp_path / "pp" / name).exists(), name
    rows = list(csv.reader(open(tmp_path / "pp" / "ldos.csv")))
    assert rows[0] == ["x_idx", "y_idx", "e_idx", "ldos"]
    vals = np.array([float(r[3]) for r in rows[1:]])
    # The oracle on the state read from the written files.
    sim_cfg = json.loads((sim_out / "simulation_config.json").read_text())
    L = O.LdosOracle(sim_cfg, pp)
    n0 = L.n0
    assert len(vals) == 6 * n0 * n0
    op = list(csv.reader(open(sim_out / "order_parameter.csv")))[1:]
    vp = list(csv.reader(open(sim_out / "vector_potential.csv")))[1:]
    d = np.zeros((1, 2, n0, n0))
    d[0, 0] = np.array([float(r[2]) for r in op]).reshape(n0, n0)
    d[0, 1] = np.array([float(r[3]) for r in op]).reshape(n0, n0)
    lam2 = cfg["physics"]["penetration_depth"] ** 2
    a = np.zeros((2, n0, n0))
    a[0] = np.array([float(r[2]) for r in vp]).reshape(n0, n0) * lam2
    a[1] = np.array([float(r[3]) for r in vp]).reshape(n0, n0) * lam2
    L.set_state(d, a)
    for b in range(L.n_blocks):
        L.begin_block(b)
        for _ in range(2):
            L.burn_in()
        for _ in range(60):
            if L.iterate()[0] < 1e-6:
                break
    want = L.ldos.reshape(-1)
    assert np.max(np.abs(vals - want)) <= 1e-7 * np.max(np.abs(want))

"""Seeded configurations and inputs shared by the tests.

The configurations use the reference's JSON schema
(examples/swave_disc_vortex/simulation_config.json in the reference project).
Sizes are kept small enough for the CPU oracle to finish in seconds.
"""
from __future__ import annotations

import copy
import math

import numpy as np


def golden_disc(accelerator: str = "congacc") -> dict:
    """The accelerator known-answer case of tests/accelerators_test.cu:45-149:
    disc of width 10 xi0 at 3 points/xi0, 16 angles, T = 0.5, cutoff 16,
    one flux quantum, lambda = 10, symmetric gauge, L-infinity residuals,
    convergence 1e-5, bulk s-wave start."""
    return {
        "physics": {"temperature": 0.5, "external_flux_quanta": 1.0, "penetration_depth": 10.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 5.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 3.0, "num_fermi_momenta": 16,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-5, "norm": "linf",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": accelerator},
    }


GOLDEN_FREE_ENERGY_PER_AREA = -0.0185386592  # tests/accelerators_test.cu:136


def small_disc() -> dict:
    """C1 in miniature: s-wave disc R = 5 xi0 at 5 points/xi0, 32 angles,
    T = 0.5, cutoff 8 (7 Ozaki poles), b = 0.02 B0, kappa = 2, CongAcc."""
    r = 5.0
    return {
        "physics": {"temperature": 0.5, "external_flux_quanta": 0.02 * math.pi * r * r / math.pi,
                    "penetration_depth": 2.0, "charge_sign": -1, "gauge": "symmetric",
                    "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": r, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 5.0, "num_fermi_momenta": 32,
                     "energy_cutoff": 8.0, "convergence_criterion": 1e-6, "norm": "l2",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "congacc"},
    }


def small_square_d() -> dict:
    """C2 in miniature: d_{x2-y2} square of side 8 xi0 with axes at 45 degrees,
    5 points/xi0, 24 angles, T = 0.1 (14 Ozaki poles), no external field,
    kappa = 2."""
    return {
        "physics": {"temperature": 0.1, "external_flux_quanta": 0.0, "penetration_depth": 2.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.125,
                    "order_parameter": {"dx2-y2": {"critical_temperature": 1.0}}},
        "geometry": [{"regular_polygon": {"add": True, "num_edges": 4, "side_length": 8.0,
                                          "rotation": 0.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 5.0, "num_fermi_momenta": 24,
                     "energy_cutoff": 8.0, "convergence_criterion": 1e-6, "norm": "l2",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "congacc"},
    }


def chiral_annulus() -> dict:
    """d + i d_xy with a hole: a disc with a smaller disc removed (the remove
    operator of GeometryGroup.h:216-334), Landau gauge, L1 residuals."""
    return {
        "physics": {"temperature": 0.3, "external_flux_quanta": 0.5, "penetration_depth": 3.0,
                    "charge_sign": -1, "gauge": "landau", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"dx2-y2": {"critical_temperature": 1.0},
                                        "dxy": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 5.0, "center_x": 0.0, "center_y": 0.0}},
                     {"disc": {"add": False, "radius": 1.5, "center_x": 1.0, "center_y": 0.5}}],
        "numerics": {"points_per_coherence_length": 4.0, "num_fermi_momenta": 20,
                     "energy_cutoff": 6.0, "convergence_criterion": 1e-6, "norm": "l1",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "congacc"},
    }


def swave_disc_field() -> dict:
    """tests/physics/swave_disc_test.cu:66-150: s-wave disc R = 20 xi0 at 2.7
    points/xi0, 16 angles, T = 0.2, cutoff 16, five flux quanta, lambda = 5,
    symmetric gauge, L-infinity residuals, criterion 1e-3, Barzilai-Borwein,
    bulk start."""
    r = 20.0
    return {
        "physics": {"temperature": 0.2, "external_flux_quanta": 5.0, "penetration_depth": 5.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": r, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 2.7, "num_fermi_momenta": 16,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-3, "norm": "linf",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "barzilai-borwein"},
    }


def swave_disc_free_energy(temperature: float, cutoff: float, lam: float, flux_quanta: float,
                           radius: float, delta: float) -> float:
    """Analytic free energy per area of a field-penetrated s-wave disc without
    phase winding (tests/physics/swave_disc_test.cu:18-57): the bulk free
    energy (OrderParameterBulk.h:225-246) plus the London magnetic and kinetic
    terms with the Yoshida-renormalised penetration depth (:256-277) and the
    modified Bessel functions I0, I1."""
    from scipy.special import iv
    n = int(cutoff / temperature - 0.5) + 1
    esum, ysum = 0.0, 0.0
    for k in range(n - 1, -1, -1):
        e = temperature * (k + 0.5)
        om = math.hypot(delta, e)
        esum += 1.0 / e - 2.0 / (e + om)
        ysum += 1.0 / om ** 3
    f_bulk = delta * delta * (math.log(temperature) + temperature * esum)
    yoshida = temperature * delta * delta * ysum
    kk = lam / math.sqrt(yoshida)
    area = math.pi * radius * radius
    b = math.pi * flux_quanta / area
    factor = 2.0 * math.pi * yoshida * (kk * b) ** 2 / (2.0 * area)
    i0, i1 = iv(0, radius / kk), iv(1, radius / kk)
    tmp = radius * i1 / i0
    f_mag = factor * (radius * radius - 2.0 * kk * tmp - 0.5 * tmp * tmp)
    f_kin = factor * 0.5 * radius * (-radius * i0 * i0 + 2 * kk * i0 * i1 + radius * i1 * i1) / (i0 * i0)
    return f_bulk + f_kin + f_mag


def disc_n256() -> dict:
    """A disc whose lattice is N0 = 256 at 10 points/xi0 (spacing 0.1), the
    size of tests/physics/vector_potential_test.cu; four angles (only the
    Poisson solve is used)."""
    r = 12.475
    return {
        "physics": {"temperature": 0.5, "external_flux_quanta": 0.0, "penetration_depth": 2.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": r, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 10.0, "num_fermi_momenta": 4,
                     "energy_cutoff": 8.0, "convergence_criterion": 1e-6, "norm": "l2",
                     "vector_potential_error": 1e-6},
    }


def rotating_disc_current(n: int, h: float):
    """tests/physics/vector_potential_test.cu:130-176: j = (-y, x) inside the
    disc of radius R = 0.4 h (n - 1) about the lattice centre, and the
    magnetostatic vector potential it induces, A = f(r) (-y, x) with
    f = (2 R^2 - r^2) / 8 inside and R^4 / (8 r^2) outside."""
    c = 0.5 * (n - 1)
    R = h * (n - 1) * 0.4
    y, x = np.meshgrid(h * (np.arange(n) - c), h * (np.arange(n) - c), indexing="ij")
    r2 = x * x + y * y
    inside = np.sqrt(r2) <= R
    j = np.stack([np.where(inside, -y, 0.0), np.where(inside, x, 0.0)])
    with np.errstate(divide="ignore", invalid="ignore"):
        f = np.where(inside, 0.125 * (2.0 * R * R - r2), 0.125 * R ** 4 / r2)
    return j, np.stack([-f * y, f * x])


def vector_potential_symmetry_error(a: np.ndarray) -> float:
    """Largest violation of the 90/180/270-degree rotation and transposition
    symmetries that tests/physics/vector_potential_test.cu:56-89 requires of
    the disc's vector potential, in doctest's Approx measure
    |u - v| / (1 + max(|u|, |v|))."""
    X, Y = a
    n = X.shape[0]
    J, I = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    def d(u, v):
        return np.max(np.abs(u - v) / (1.0 + np.maximum(np.abs(u), np.abs(v))))
    errs = [d(-Y, X[I, n - 1 - J]), d(X, Y[I, n - 1 - J]),
            d(-X, X[n - 1 - J, n - 1 - I]), d(-Y, Y[n - 1 - J, n - 1 - I]),
            d(Y, X[n - 1 - I, J]), d(-X, Y[n - 1 - I, J]),
            d(np.hypot(X, Y), np.hypot(X[I, J], Y[I, J]))]
    return float(max(errs))


def with_accelerator(cfg: dict, name: str) -> dict:
    c = copy.deepcopy(cfg)
    c["accelerator"] = {"name": name}
    return c


def seeded_state(n_comp: int, n0: int, delta_bulk: float, seed: int, noise: float = 0.01,
                 complex_noise: bool = False, a_scale: float = 0.0):
    """Delta = delta_bulk * (1 + noise N(0,1)) per component (the complex
    variant adds i * noise N(0,1)), A = a_scale * N(0,1); planar layouts."""
    rng = np.random.default_rng(seed)
    d = np.zeros((n_comp, 2, n0, n0))
    for c in range(n_comp):
        d[c, 0] = delta_bulk * (1.0 + noise * rng.standard_normal((n0, n0)))
        if complex_noise:
            d[c, 1] = delta_bulk * noise * rng.standard_normal((n0, n0))
    a = a_scale * rng.standard_normal((2, n0, n0))
    return d, a


def ldos_postprocess(delta0: float, n_energies: int = 12, per_block: int = 8, n_angles: int = 32,
                     broadening: float = 0.05, crit: float = 1e-5) -> dict:
    """Postprocess configuration (examples/*/postprocess_config.json schema):
    energies uniform in [-2 delta0, 2 delta0]; a block size that leaves a short
    last block when n_energies is not a multiple of it."""
    return {
        "spectroscopy": {"energy_min": -2.0 * delta0, "energy_max": 2.0 * delta0,
                         "num_energies": n_energies, "energy_broadening": broadening},
        "numerics": {"convergence_criterion": crit, "norm": "l2", "num_energies_per_block": per_block,
                     "num_fermi_momenta": n_angles, "num_iterations_burnin": 2,
                     "num_iterations_min": 0, "num_iterations_max": 60},
        "misc": {"data_format": "csv", "load_path": "", "save_path": "", "verbose": False},
    }


def dos_test_case(swave: bool):
    """tests/physics/dos_test.cu:10-21,23-69: an s-wave disc or a d_{x2-y2}
    square with axes along its edges (no pair breaking), width 5 xi0 at 2
    points/xi0, 160 angles, T = 0.5; the LDOS of 32 energies in [0, 0.5] with
    broadening 0.008 in one block, criterion 1e-8 (L-infinity), at most 42
    iterations.  Returns (simulation, postprocess) configurations."""
    geom = ({"disc": {"add": True, "radius": 2.5, "center_x": 0.0, "center_y": 0.0}} if swave else
            {"regular_polygon": {"add": True, "num_edges": 4, "side_length": 5.0, "rotation": 0.0,
                                 "center_x": 0.0, "center_y": 0.0}})
    sim = {
        "physics": {"temperature": 0.5, "external_flux_quanta": 0.0, "penetration_depth": -1.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {("s" if swave else "dx2-y2"): {"critical_temperature": 1.0}}},
        "geometry": [geom],
        "numerics": {"points_per_coherence_length": 2.0, "num_fermi_momenta": 160,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-8, "norm": "linf"},
    }
    pp = {
        "spectroscopy": {"energy_min": 0.0, "energy_max": 0.5, "num_energies": 32,
                         "energy_broadening": 0.008},
        "numerics": {"convergence_criterion": 1e-8, "norm": "linf", "num_energies_per_block": 32,
                     "num_fermi_momenta": 160, "num_iterations_burnin": 0,
                     "num_iterations_min": 0, "num_iterations_max": 42},
        "misc": {"data_format": "csv", "load_path": "", "save_path": "", "verbose": False},
    }
    return sim, pp


def low_temperature_bulk(swave: bool, disc: bool) -> dict:
    """tests/physics/low_temp_free_energy_test.cu:30-60,62-160: an s-wave disc,
    an s-wave square or a d_{x2-y2} square (axes along the edges) of width 10
    xi0 at 1 point/xi0, T = 0.001, cutoff 32 (281 Ozaki poles), 32 (s-wave) or
    360 (d-wave) angles, no field and no vector potential, L-infinity
    residuals, criterion 1e-3, Barzilai-Borwein, bulk start."""
    geom = ({"disc": {"add": True, "radius": 5.0, "center_x": 0.0, "center_y": 0.0}} if disc else
            {"regular_polygon": {"add": True, "num_edges": 4, "side_length": 10.0, "rotation": 0.0,
                                 "center_x": 0.0, "center_y": 0.0}})
    return {
        "physics": {"temperature": 0.001, "external_flux_quanta": 0.0, "penetration_depth": -1.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {("s" if swave else "dx2-y2"): {"critical_temperature": 1.0}}},
        "geometry": [geom],
        "numerics": {"points_per_coherence_length": 1.0, "num_fermi_momenta": 32 if swave else 360,
                     "energy_cutoff": 32.0, "convergence_criterion": 1e-3, "norm": "linf"},
        "accelerator": {"name": "barzilai-borwein"},
    }


def phase_gradient_disc() -> dict:
    """tests/physics/current_phase_gradient_test.cu:22-78: s-wave disc of width
    10 xi0 at 2 points/xi0, 16 angles, T = 0.9, cutoff 16, criterion 1e-5
    (L-infinity), no field, charge sign -1, no vector potential,
    Barzilai-Borwein."""
    return {
        "physics": {"temperature": 0.9, "external_flux_quanta": 0.0, "penetration_depth": -1.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 5.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 2.0, "num_fermi_momenta": 16,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-5, "norm": "linf"},
        "accelerator": {"name": "barzilai-borwein"},
    }


def phase_winding_state(n0: int, delta_bulk: float, winding: float, phase_shift: float = 0.0,
                        center=(0.0, 0.0)) -> np.ndarray:
    """Initial<T>::phaseWinding without noise (OrderParameterInitial.h:187-235,
    375-381): Delta_bulk exp(i (shift + w atan2(y, x))) on the lattice
    normalised to [-1, 1], the winding centre taking phase 0.  Returns
    [1][2][n0][n0]."""
    c = np.arange(n0, dtype=np.float64)
    u = 2.0 * c / (n0 - 1) - 1.0
    x = u[None, :] - center[0]
    y = u[:, None] - center[1]
    ang = np.where(np.hypot(x, y) > 0.0, np.arctan2(y, x), 0.0)
    phase = phase_shift + winding * ang
    out = np.zeros((1, 2, n0, n0))
    out[0, 0] = delta_bulk * np.cos(phase)
    out[0, 1] = delta_bulk * np.sin(phase)
    return out


def complex_phase_gradient(re: np.ndarray, im: np.ndarray, h: float = 1.0) -> np.ndarray:
    """GridFunctions::complexPhaseGradient (GridFunctions_GPU.h:209-267):
    central differences of the phase, (f' g - f g') / (2 h |z|^2) with f = Im
    z, g = Re z, zero on the lattice border and where 2 h |z|^2 <= 1e-5.
    Returns [2][n][n] (x, y)."""
    n = re.shape[0]
    out = np.zeros((2, n, n))
    g1, f1 = re[1:-1, 1:-1], im[1:-1, 1:-1]
    denom = 2.0 * h * (f1 * f1 + g1 * g1)
    ok = denom > 1e-5
    inv = np.where(ok, 1.0 / np.where(ok, denom, 1.0), 0.0)
    dx = ((im[1:-1, 2:] - im[1:-1, :-2]) * g1 - f1 * (re[1:-1, 2:] - re[1:-1, :-2])) * inv
    dy = ((im[2:, 1:-1] - im[:-2, 1:-1]) * g1 - f1 * (re[2:, 1:-1] - re[:-2, 1:-1])) * inv
    out[0, 1:-1, 1:-1] = np.where(ok, dx, 0.0)
    out[1, 1:-1, 1:-1] = np.where(ok, dy, 0.0)
    return out


def penetration_depth_disc() -> dict:
    """tests/physics/penetration_depth_test.cu:89-131: s-wave disc of width 20
    xi0 at 5 points/xi0, 16 angles, T = 0.1, cutoff 16, half a flux quantum,
    lambda = 1, symmetric gauge, L-infinity residuals, criterion 1e-3, CongAcc
    with initial step 0.001, bulk start."""
    return {
        "physics": {"temperature": 0.1, "external_flux_quanta": 0.5, "penetration_depth": 1.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 10.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 5.0, "num_fermi_momenta": 16,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-3, "norm": "linf",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "congacc", "step_size": 0.001},
    }


def curl(ax: np.ndarray, ay: np.ndarray, h: float) -> np.ndarray:
    """GridFunctions::curl (GridFunctions_GPU.h:327-353): dAy/dx - dAx/dy by
    central differences, one-sided on the lattice border, divided by h."""
    n = ax.shape[0]
    i = np.arange(n)
    nxt, prv = np.minimum(i + 1, n - 1), np.maximum(i - 1, 0)
    span = (nxt - prv).astype(np.float64)
    day_dx = (ay[:, nxt] - ay[:, prv]) / span[None, :]
    dax_dy = (ax[nxt, :] - ax[prv, :]) / span[:, None]
    return (day_dx - dax_dy) / h


def fit_penetration_depth(guess: float, b_ext: float, width: float, flux: float) -> float:
    """Newton fit of the London flux through a disc, 2 pi b k ((R - k) + k
    exp(-R/k)) with R = width / 2, to the measured flux
    (tests/physics/penetration_depth_test.cu:15-81)."""
    r = 0.5 * width
    factor = 2.0 * math.pi * b_ext
    k = guess
    for _ in range(200):
        res = factor * k * ((r - k) + k * math.exp(-r / k)) - flux
        drdk = factor * ((r + 2.0 * k) * math.exp(-r / k) + r - 2.0 * k)
        dk = res * math.copysign(1.0, drdk) / max(abs(drdk), np.finfo(np.float64).eps)
        done = abs(dk / k) < 1e-6
        k -= dk
        if done:
            return k
    raise RuntimeError("penetration-depth fit did not converge")


def penetration_depth_from_state(a: np.ndarray, domain: np.ndarray, h: float, flux_quanta: float,
                                 width: float, guess: float) -> float:
    """The fitted penetration depth of tests/physics/penetration_depth_test.cu:
    133-150: flux = area (b_ext + <curl A>_grain) with area = sites h^2 and
    b_ext = pi flux_quanta / area."""
    grain = domain > 0
    n = grain.sum()
    area = n * h * h
    b_ext = math.pi * flux_quanta / area
    b = curl(a[0], a[1], h)
    flux = area * (b_ext + (b * grain).sum() / n)
    return fit_penetration_depth(guess, b_ext, width, flux)


def linear_response_square(temperature: float) -> dict:
    """tests/physics/current_linear_response_test.cu:15-120: s-wave square of
    side 20 xi0 at 1 point/xi0, 32 angles, cutoff 16, lambda = 1, no external
    field, bulk start; the induced vector potential is held at (0.01, 0.01)
    for the one iteration the test runs."""
    return {
        "physics": {"temperature": temperature, "external_flux_quanta": 0.0, "penetration_depth": 1.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"regular_polygon": {"add": True, "num_edges": 4, "side_length": 20.0,
                                          "rotation": 0.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 1.0, "num_fermi_momenta": 32,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-4, "norm": "l2",
                     "vector_potential_error": 1e-6},
        "accelerator": {"name": "congacc"},
    }


def solenoid_annulus(flux_quanta: float) -> dict:
    """tests/physics/swave_annulus_solenoid_gauge_test.cu:37-134: s-wave
    annulus with outer radius 20 xi0 and inner radius 10 xi0 at 3.5
    points/xi0, 16 angles, T = 0.2, cutoff 16, the solenoid gauge, charge sign
    -1, no vector potential, L-infinity residuals, criterion 1e-4,
    Barzilai-Borwein; the initial order parameter winds once."""
    return {
        "physics": {"temperature": 0.2, "external_flux_quanta": flux_quanta, "penetration_depth": -1.0,
                    "charge_sign": -1, "gauge": "solenoid", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 20.0, "center_x": 0.0, "center_y": 0.0}},
                     {"disc": {"add": False, "radius": 10.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 3.5, "num_fermi_momenta": 16,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-4, "norm": "linf"},
        "accelerator": {"name": "barzilai-borwein"},
    }


def solenoid_annulus_free_energy(flux_quanta: float, bulk_gap: float, bulk_free_energy: float,
                                 yoshida: float, charge_winding: float = -1.0) -> float:
    """The expected free energy per area of the solenoid-gauge annulus
    (tests/physics/swave_annulus_solenoid_gauge_test.cu:138-160): the bulk
    value plus the kinetic term Y ln(R/r) / (4 (R^2 - r^2)) (Phi - q w)^2 with
    R = 20 and r = 10."""
    outer, inner = 20.0, 10.0
    factor = 0.25 * yoshida * math.log(outer / inner) / (outer * outer - inner * inner)
    return bulk_free_energy + factor * (flux_quanta - charge_winding) ** 2


SOLENOID_FLUXES = (-1.5, -1.0, -0.5)


def radial_annulus() -> dict:
    """tests/physics/swave_annulus_radial_gauge_test.cu:345-425: s-wave annulus
    with outer radius 20 xi0 and inner radius 10 xi0 at 6.2 points/xi0, 32
    angles, T = 0.2, cutoff 16, one flux quantum, lambda = 30 with a
    self-consistent vector potential (error 1e-3), symmetric gauge, charge
    sign -1, L-infinity residuals, criterion 1e-4, Barzilai-Borwein; the
    initial order parameter winds -2 times (q w = 2)."""
    return {
        "physics": {"temperature": 0.2, "external_flux_quanta": 1.0, "penetration_depth": 30.0,
                    "charge_sign": -1, "gauge": "symmetric", "crystal_axes_rotation": 0.0,
                    "order_parameter": {"s": {"critical_temperature": 1.0}}},
        "geometry": [{"disc": {"add": True, "radius": 20.0, "center_x": 0.0, "center_y": 0.0}},
                     {"disc": {"add": False, "radius": 10.0, "center_x": 0.0, "center_y": 0.0}}],
        "numerics": {"points_per_coherence_length": 6.2, "num_fermi_momenta": 32,
                     "energy_cutoff": 16.0, "convergence_criterion": 1e-4, "norm": "linf",
                     "vector_potential_error": 1e-3},
        "accelerator": {"name": "barzilai-borwein"},
    }


def _annulus_factors(outer, inner, lam_t, flux, winding, charge):
    """The London solution of a thick annulus in the radial gauge
    (tests/physics/swave_annulus_radial_gauge_test.cu:96-150): the
    coefficients a, b of B = a I0(r/k) - b K0(r/k) in the grain and the
    fluxoid coefficient c, with k = lam_t the temperature-dependent
    penetration depth and the pi of the flux unit A0 = Phi0 / (pi xi0)."""
    from scipy.special import iv, kv
    hole = math.pi * inner * inner
    grain = math.pi * outer * outer - hole
    big, small = outer / lam_t, inner / lam_t
    qw = charge * winding
    inv_m = math.pi / (iv(0, big) * kv(2, small) - iv(2, small) * kv(0, big))
    a = inv_m * (flux * kv(2, small) / grain - qw * kv(0, big) / hole)
    b = inv_m * (flux * iv(2, small) / grain - qw * iv(0, big) / hole)
    c = inv_m * (2.0 * math.pi * lam_t * lam_t * flux / grain
                 + qw * (iv(0, big) * kv(0, small) - iv(0, small) * kv(0, big)))
    return a, b, c, grain, hole


def annulus_analytic(outer, inner, lam, flux, winding, charge, temperature, cutoff, bulk):
    """Expected free energy per area, magnetic free energy per area and
    magnetic moment per area of the annulus
    (tests/physics/swave_annulus_radial_gauge_test.cu:152-337): bulk energy
    plus the kinetic and magnetic London terms, integrated over the grain by
    32-point Gauss-Legendre quadrature, plus the field energy in the hole; the
    moment in closed form.  ``bulk`` = (gap(T), free energy(T, gap),
    Yoshida(T, gap, cutoff))."""
    from scipy.special import iv, kv
    op_fn, fe_fn, y_fn = bulk
    d = op_fn(temperature)
    f_bulk = fe_fn(temperature, d)
    k = lam / math.sqrt(y_fn(temperature, d, cutoff))
    a, b, c, grain, hole = _annulus_factors(outer, inner, k, flux, winding, charge)
    scale = 2.0 * math.pi * lam * lam / (2.0 * grain)
    b_ext = math.pi * flux / grain
    x, w = np.polynomial.legendre.leggauss(32)
    r = 0.5 * (outer - inner) * x + 0.5 * (outer + inner)
    w = 0.5 * (outer - inner) * w
    mag = scale * np.sum(w * r * (a * iv(0, r / k) - b * kv(0, r / k) - b_ext) ** 2)
    mag += scale * 0.5 * ((c / hole - b_ext) * inner) ** 2
    kin = scale * np.sum(w * r * (a * iv(1, r / k) + b * kv(1, r / k)) ** 2)
    moment = annulus_moment(outer, inner, lam, flux, winding, charge, temperature, cutoff, (op_fn, y_fn))
    return f_bulk + kin + mag, mag, moment


def annulus_moment(outer, inner, lam, flux, winding, charge, temperature, cutoff, bulk):
    """The closed-form magnetic moment per area of the annulus
    (tests/physics/swave_annulus_radial_gauge_test.cu:152-205); ``bulk`` =
    (gap(T), Yoshida(T, gap, cutoff))."""
    from scipy.special import iv, kv
    op_fn, y_fn = bulk
    d = op_fn(temperature)
    k = lam / math.sqrt(y_fn(temperature, d, cutoff))
    a, b, _, grain, _ = _annulus_factors(outer, inner, k, flux, winding, charge)
    scale = 2.0 * math.pi * lam * lam / (2.0 * grain)
    return -scale * (outer * outer * (a * iv(2, outer / k) - b * kv(2, outer / k))
                     - inner * inner * (a * iv(2, inner / k) - b * kv(2, inner / k)))


def magnetic_moment(current: np.ndarray, h: float, n_grain: int) -> float:
    """GridFunctions::moment (GridFunctions_GPU.h:602-616,726-754) per grain
    area: 0.5 h^3 sum (x j_y - y j_x) over the lattice, x and y in sites from
    its centre, divided by n_grain h^2."""
    n = current.shape[-1]
    c = np.arange(n, dtype=np.float64) - 0.5 * (n - 1)
    return 0.5 * h ** 3 * float(np.sum(c[None, :] * current[1] - c[:, None] * current[0])) / (n_grain * h * h)


def bulk_dos(energy: np.ndarray, broadening: float, delta: float, swave: bool, n_angles: int) -> np.ndarray:
    """The expected DOS of tests/physics/dos_test.cu:168-198: sum over the
    circle's angles of w_k Im[e / sqrt(|eta_k delta|^2 - e^2)], e = E + i delta_b,
    with the normalised basis function eta at the Fermi momentum (1 for s,
    cos 2 phi normalised for d_{x2-y2}) and the Boole / Simpson weights."""
    k = np.arange(n_angles)
    phi = np.mod(2 * np.pi * k / n_angles + 0.5 * np.pi, 2 * np.pi)
    w = np.where(k % 4 == 0, 28.0, np.where(k % 2 == 0, 24.0, 64.0)) / 45.0 if n_angles % 4 == 0 else np.ones(n_angles)
    w = w / n_angles
    raw = np.ones(n_angles) if swave else np.cos(phi) ** 2 - np.sin(phi) ** 2
    eta = raw / np.sqrt(np.sum(raw * raw * w))
    out = np.zeros(len(energy))
    for i, e0 in enumerate(energy):
        e = e0 + 1j * broadening
        om = np.sqrt(np.abs(eta * delta) ** 2 - e * e + 0j)
        out[i] = np.sum(w * (e / om).imag)
    return out


def bcs_dos(energy: np.ndarray, broadening: float, delta: float) -> np.ndarray:
    """Bulk s-wave density of states Re[e / sqrt(e^2 - delta^2)], e = E + i delta_b
    (retarded branch: the root with positive imaginary part times sign)."""
    e = energy + 1j * broadening
    root = np.sqrt(e * e - delta * delta + 0j)
    root = np.where(np.imag(root) * np.sign(np.real(e) + 1e-300) < 0, -root, root)
    root = np.where(np.real(e / root) < 0, -root, root)
    return np.real(e / root)

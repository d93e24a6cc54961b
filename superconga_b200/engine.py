"""Python face of the B200 engine, shaped like the reference's C++ Context.

``Context`` owns one libscb200 handle.  Its methods follow the reference's
orchestration API (include/conga/Context.h): ``compute`` runs
``Context::compute`` iterations, ``burn_in`` runs ``Context::burnIn``,
``residual`` / ``is_converged`` mirror ``getResidual`` /
``isPartiallyConverged``, and the grids come back in the reference's planar
layout (GridData.h:276-291) as numpy arrays.
"""
from __future__ import annotations

import ctypes
import json
from dataclasses import dataclass

import numpy as np

from . import _lib

MODES = {"fp64": 0, "mixed": 1}


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


@dataclass
class Dims:
    n0: int
    n1: int
    n_angles: int
    n_energies: int
    n_comp: int


class Context:
    """One self-consistency context on the current CUDA device."""

    def __init__(self, config: dict | str, mode: str = "fp64"):
        cfg = config if isinstance(config, str) else json.dumps(config)
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sc_create(cfg.encode(), MODES[mode], ctypes.byref(h)))
        self._h = h
        self.mode = mode
        ints = [ctypes.c_int() for _ in range(5)]
        _lib.check(lib.sc_get_dims(h, *[ctypes.byref(i) for i in ints]), h)
        self.dims = Dims(*[i.value for i in ints])

    # ----------------------------------------------------------- lifetime --
    def close(self):
        if getattr(self, "_h", None):
            _lib.load().sc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, status: int):
        _lib.check(status, self._h)

    # ------------------------------------------------------------ state ----
    def _shape_delta(self):
        d = self.dims
        return (d.n_comp, 2, d.n0, d.n0)

    def _shape_vec(self):
        return (2, self.dims.n0, self.dims.n0)

    def set_state(self, delta: np.ndarray, a_internal: np.ndarray | None = None):
        """x = (order parameter [Nc][2][N0][N0], vector potential [2][N0][N0])."""
        d = np.ascontiguousarray(delta, np.float64).reshape(self._shape_delta())
        a = None if a_internal is None else np.ascontiguousarray(a_internal, np.float64).reshape(self._shape_vec())
        self._check(_lib.load().sc_set_state(self._h, _p(d), _p(a) if a is not None else None))

    def state(self, delta_out: np.ndarray | None = None, a_out: np.ndarray | None = None):
        """x as (order parameter, vector potential); into the caller's arrays
        (C-contiguous float64 of the right shapes, e.g. pinned host memory)
        when given, without an intermediate copy."""
        d = np.zeros(self._shape_delta()) if delta_out is None else delta_out
        a = np.zeros(self._shape_vec()) if a_out is None else a_out
        for arr, shape in ((d, self._shape_delta()), (a, self._shape_vec())):
            if arr.dtype != np.float64 or not arr.flags["C_CONTIGUOUS"] or arr.size != int(np.prod(shape)):
                raise ValueError("state(): output arrays must be C-contiguous float64 of the state's shape")
        self._check(_lib.load().sc_get_state(self._h, _p(d), _p(a)))
        return d, a

    def set_state_device(self, delta_ptr: int, a_ptr: int | None = None):
        self._check(_lib.load().sc_set_state_device(self._h, ctypes.c_void_p(delta_ptr),
                                                    ctypes.c_void_p(a_ptr) if a_ptr else None))

    def get_state_device(self, delta_ptr: int, a_ptr: int | None = None):
        self._check(_lib.load().sc_get_state_device(self._h, ctypes.c_void_p(delta_ptr),
                                                    ctypes.c_void_p(a_ptr) if a_ptr else None))

    def set_stream(self, stream_ptr: int):
        self._check(_lib.load().sc_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # ------------------------------------------------------- iteration ----
    def compute(self, n: int = 1):
        """n x Context::compute; returns (residual, converged) of the last one."""
        r = ctypes.c_double()
        c = ctypes.c_int()
        self._check(_lib.load().sc_compute(self._h, int(n), ctypes.byref(r), ctypes.byref(c)))
        return r.value, bool(c.value)

    def burn_in(self, n: int = 1):
        r = ctypes.c_double()
        c = ctypes.c_int()
        self._check(_lib.load().sc_burn_in(self._h, int(n), ctypes.byref(r), ctypes.byref(c)))
        return r.value, bool(c.value)

    def run(self, it_min: int, it_max: int, burn_in: int = 0):
        """runSimulation without I/O (run_simulation.h:124-187): burn-in, then
        iterate until converged and it_min reached, or it_max reached."""
        if burn_in:
            self.burn_in(burn_in)
        i, conv = 0, False
        while True:
            i += 1
            _, conv = self.compute(1)
            if (conv and i >= it_min) or (it_max >= 0 and i >= it_max):
                return i, conv

    def set_external_field(self, b: float):
        """External field B_ext = pi Phi / area in units of B0 (RiccatiSolver.h:137-139)."""
        self._check(_lib.load().sc_set_external_field(self._h, float(b)))

    def external_field(self) -> float:
        v = ctypes.c_double()
        self._check(_lib.load().sc_get_external_field(self._h, ctypes.byref(v)))
        return v.value

    def evaluate(self) -> float:
        """Frozen-boundary evaluation of the current state (no accelerator
        step, no boundary update); returns the free energy.  g(x) and j are
        then available from ``results``."""
        v = ctypes.c_double()
        self._check(_lib.load().sc_evaluate(self._h, ctypes.byref(v)))
        return v.value

    def adjoint(self, w_omega: float = 1.0, beta_j: np.ndarray | None = None):
        """Gradients of L = w_omega * Omega + sum(beta_j * j) at frozen boundary
        values: dL/dDelta [Nc][2][N0][N0] (d/dRe, d/dIm), dL/dA [2][N0][N0]
        (internal units), dL/dB_ext."""
        gd = np.zeros(self._shape_delta())
        ga = np.zeros(self._shape_vec())
        gb = ctypes.c_double()
        bj = None if beta_j is None else np.ascontiguousarray(beta_j, np.float64).reshape(self._shape_vec())
        self._check(_lib.load().sc_adjoint(self._h, float(w_omega), _p(bj) if bj is not None else None,
                                           _p(gd), _p(ga), ctypes.byref(gb)))
        return gd, ga, gb.value

    def results(self):
        """g(x): new order parameter, current density, new vector potential."""
        d = np.zeros(self._shape_delta())
        j = np.zeros(self._shape_vec())
        a = np.zeros(self._shape_vec())
        self._check(_lib.load().sc_get_results(self._h, _p(d), _p(j), _p(a)))
        return d, j, a

    def scalars(self) -> dict:
        out = np.zeros(11)
        self._check(_lib.load().sc_get_scalars(self._h, _p(out)))
        keys = ["free_energy", "free_energy_per_area", "magnetic_free_energy",
                "magnetic_free_energy_per_area", "res_order_parameter", "res_current",
                "res_free_energy", "res_vector_potential", "res_boundary", "residual",
                "n_grain"]
        return dict(zip(keys, out.tolist()))

    def site_updates(self) -> int:
        v = ctypes.c_longlong()
        self._check(_lib.load().sc_site_updates(self._h, ctypes.byref(v)))
        return v.value

    def launch_count(self) -> int:
        v = ctypes.c_longlong()
        self._check(_lib.load().sc_launch_count(self._h, ctypes.byref(v)))
        return v.value

    def profile(self, enable: bool = True):
        """Enables CUDA-event timing of the sweep (0), rotate-back (1), Poisson
        (2), boundary (3) and frame-field (4) kernels."""
        self._check(_lib.load().sc_profile(self._h, 1 if enable else 0))

    def profile_read(self, kernel: int):
        """(summed device ms, launches) of one kernel since the last read."""
        ms = ctypes.c_double()
        n = ctypes.c_longlong()
        self._check(_lib.load().sc_profile_read(self._h, kernel, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    # ---------------------------------------------------------- probes -----
    def frame_labels(self, angle: int):
        n1 = self.dims.n1
        lab = np.zeros((n1, n1), np.int8)
        box = (ctypes.c_int * 4)()
        self._check(_lib.load().sc_get_frame_labels(self._h, angle, _p(lab), box))
        return lab, tuple(box)

    def domain(self):
        d = np.zeros((self.dims.n0, self.dims.n0), np.int8)
        self._check(_lib.load().sc_get_domain(self._h, _p(d)))
        return d

    def boundary_sizes(self):
        s = (ctypes.c_int * 4)()
        self._check(_lib.load().sc_boundary_sizes(self._h, s))
        return list(s)

    def sweep_plan(self):
        """(number of angle chunks, mirror pairing on) of the sweep."""
        n, p = ctypes.c_int(), ctypes.c_int()
        self._check(_lib.load().sc_sweep_plan(self._h, ctypes.byref(n), ctypes.byref(p)))
        return n.value, bool(p.value)

    def boundary(self, which: int) -> np.ndarray:
        n = self.boundary_sizes()[which] * self.dims.n_energies
        v = np.zeros(2 * n)
        self._check(_lib.load().sc_get_boundary(self._h, which, _p(v)))
        return v[0::2] + 1j * v[1::2]

    def set_boundary(self, which: int, values: np.ndarray):
        v = np.ascontiguousarray(np.stack([values.real, values.imag], -1).ravel(), np.float64)
        self._check(_lib.load().sc_set_boundary(self._h, which, _p(v)))

    def boundary_initial(self):
        self._check(_lib.load().sc_boundary_initial(self._h))

    def angle_greens(self, angle: int):
        n1 = self.dims.n1
        f = np.zeros((2, n1, n1))
        g = np.zeros((n1, n1))
        i = np.zeros((n1, n1))
        self._check(_lib.load().sc_angle_greens(self._h, angle, _p(f), _p(g), _p(i)))
        return f[0] + 1j * f[1], g, i

    def poisson(self, j: np.ndarray) -> np.ndarray:
        jj = np.ascontiguousarray(j, np.float64).reshape(self._shape_vec())
        out = np.zeros(self._shape_vec())
        self._check(_lib.load().sc_poisson(self._h, _p(jj), _p(out)))
        return out


def fma_peak(precision: int = 64) -> float:
    """Measured FMA throughput of the current device in FLOP/s."""
    v = ctypes.c_double()
    _lib.check(_lib.load().sc_measure_fma_peak(int(precision), ctypes.byref(v)))
    return v.value


def bulk_order_parameter_s_wave(temperature: float, convergence_criterion: float = 10.0 * np.finfo(np.float64).eps,
                                max_iterations: int = 10, energy_cutoff: float = 100.0) -> float:
    """computeOrderParameterBulkSWave (OrderParameterBulk.h:88-221): the bulk
    s-wave gap at T/Tc, in units of 2 pi k_B Tc (host only)."""
    v = ctypes.c_double()
    _lib.check(_lib.load().sc_bulk_order_parameter_s_wave(float(temperature), float(convergence_criterion),
                                                         int(max_iterations), float(energy_cutoff),
                                                         ctypes.byref(v)))
    return v.value


def bulk_free_energy_s_wave(temperature: float, order_parameter: float, energy_cutoff: float = 100.0) -> float:
    """computeFreeEnergyBulkSWave (OrderParameterBulk.h:224-246): the bulk
    free energy density at the given gap (host only)."""
    v = ctypes.c_double()
    _lib.check(_lib.load().sc_bulk_free_energy_s_wave(float(temperature), float(order_parameter),
                                                     float(energy_cutoff), ctypes.byref(v)))
    return v.value


def bulk_yoshida_s_wave(temperature: float, order_parameter: float, energy_cutoff: float) -> float:
    """computeYoshidaBulkSWave (OrderParameterBulk.h:256-277): the bulk London
    response j = -Y A at the given gap (host only)."""
    v = ctypes.c_double()
    _lib.check(_lib.load().sc_bulk_yoshida_s_wave(float(temperature), float(order_parameter),
                                                 float(energy_cutoff), ctypes.byref(v)))
    return v.value


class Setup:
    """Host-only view of a configuration's static tables (no GPU needed)."""

    def __init__(self, config: dict | str):
        cfg = config if isinstance(config, str) else json.dumps(config)
        lib = _lib.load()
        h = ctypes.c_void_p()
        st = lib.sc_setup_create(cfg.encode(), ctypes.byref(h))
        if st != 0:
            raise _lib.EngineError(st, lib.sc_setup_last_error().decode())
        self._h = h
        ints = [ctypes.c_int() for _ in range(5)]
        lib.sc_setup_dims(h, *[ctypes.byref(i) for i in ints])
        self.dims = Dims(*[i.value for i in ints])

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                _lib.load().sc_setup_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def energies(self):
        ne = self.dims.n_energies
        e = np.zeros(ne)
        r = np.zeros(ne)
        _lib.load().sc_setup_energies(self._h, _p(e), _p(r))
        return e, r

    def frame(self, angle: int):
        n1 = self.dims.n1
        lab = np.zeros((n1, n1), np.int8)
        box = (ctypes.c_int * 4)()
        _lib.check(_lib.load().sc_setup_frame(self._h, angle, _p(lab), box))
        return lab, tuple(box)

    def domain(self):
        d = np.zeros((self.dims.n0, self.dims.n0), np.int8)
        _lib.load().sc_setup_domain(self._h, _p(d))
        return d

    def boundary_sizes(self):
        s = (ctypes.c_int * 4)()
        _lib.load().sc_setup_boundary_sizes(self._h, s)
        return list(s)

    def filters(self):
        lib = _lib.load()
        n = ctypes.c_int()
        lib.sc_setup_filters(self._h, ctypes.byref(n), None, None, None)
        f = np.zeros((n.value, 2 * self.dims.n0 - 1))
        pos = np.zeros(n.value, np.int32)
        sc = ctypes.c_double()
        lib.sc_setup_filters(self._h, ctypes.byref(n), _p(f), pos.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                             ctypes.byref(sc))
        return f, pos, sc.value

    def site_updates(self) -> int:
        v = ctypes.c_longlong()
        _lib.load().sc_setup_site_updates(self._h, ctypes.byref(v))
        return v.value

    def fermi_surface(self) -> dict:
        """Per-angle Fermi-surface tables (polar angle, system angle, momentum,
        normalised velocity, integrand factor, Riccati step) and the
        tight-binding averages and momentum origin."""
        na = self.dims.n_angles
        t = np.zeros((8, na))
        info = np.zeros(4)
        _lib.check(_lib.load().sc_setup_fermi_surface(self._h, _p(t), _p(info)))
        keys = ["phi", "theta", "px", "py", "vx", "vy", "weight", "step"]
        out = {k: t[i].copy() for i, k in enumerate(keys)}
        out.update(avg_fermi_momentum=float(info[0]), avg_fermi_speed=float(info[1]),
                   origin=(float(info[2]), float(info[3])))
        return out


class LdosContext(Context):
    """LDOS postprocess on the current CUDA device, shaped like the Context that
    src/postprocess.cu builds (IntegrationIteratorKeldysh + ComputeLDOS).

    ``simulation`` is the simulation configuration of the loaded run and
    ``postprocess`` the postprocess configuration.  Load the converged state
    with ``set_state`` (A in internal units), then ``run`` (runPostprocess) or
    ``begin_block`` / ``burn_in`` / ``iterate`` step by step; ``ldos`` returns
    [n_energies][N0][N0].
    """

    def __init__(self, simulation: dict | str, postprocess: dict | str, mode: str = "fp64"):
        sim = simulation if isinstance(simulation, str) else json.dumps(simulation)
        pp = postprocess if isinstance(postprocess, str) else json.dumps(postprocess)
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sc_ldos_create(sim.encode(), pp.encode(), MODES[mode], ctypes.byref(h)))
        self._h = h
        self.mode = mode
        ints = [ctypes.c_int() for _ in range(5)]
        _lib.check(lib.sc_get_dims(h, *[ctypes.byref(i) for i in ints]), h)
        self.dims = Dims(*[i.value for i in ints])
        ld = [ctypes.c_int() for _ in range(3)]
        _lib.check(lib.sc_ldos_dims(h, *[ctypes.byref(i) for i in ld]), h)
        self.n_ldos_energies, self.per_block, self.n_blocks = (i.value for i in ld)

    def energies(self):
        e = np.zeros(self.n_ldos_energies)
        d = ctypes.c_double()
        self._check(_lib.load().sc_ldos_energies(self._h, _p(e), ctypes.byref(d)))
        return e, d.value

    def begin_block(self, block: int):
        self._check(_lib.load().sc_ldos_begin_block(self._h, int(block)))

    def iterate(self, n: int = 1):
        """n LDOS iterations of the current block; returns (residual, converged)."""
        r = ctypes.c_double()
        c = ctypes.c_int()
        self._check(_lib.load().sc_ldos_iterate(self._h, int(n), ctypes.byref(r), ctypes.byref(c)))
        return r.value, bool(c.value)

    def run(self, burn_in: int, it_min: int, it_max: int):
        """runPostprocess: returns (converged, total iterations)."""
        c = ctypes.c_int()
        it = ctypes.c_int()
        self._check(_lib.load().sc_ldos_run(self._h, int(burn_in), int(it_min), int(it_max),
                                            ctypes.byref(c), ctypes.byref(it)))
        return bool(c.value), it.value

    def ldos(self):
        out = np.zeros((self.n_ldos_energies, self.dims.n0, self.dims.n0))
        self._check(_lib.load().sc_ldos_get(self._h, _p(out)))
        return out


class _Grain(Context):
    """Context view of one grain of a Batch (the batch owns the handle)."""

    def __init__(self, handle: ctypes.c_void_p, batch: "Batch"):
        self._h = handle
        self._batch = batch
        self.mode = batch.mode
        ints = [ctypes.c_int() for _ in range(5)]
        _lib.check(_lib.load().sc_get_dims(handle, *[ctypes.byref(i) for i in ints]), handle)
        self.dims = Dims(*[i.value for i in ints])

    def close(self):
        self._h = None


class Batch:
    """Many independent grains advanced together on the current CUDA device.

    ``grains[i]`` is a Context view of grain i (set its state, read its
    results).  ``compute(n)`` runs up to n iterations of every grain that has
    not finished (each converges, or stops, by its own configuration); the
    sweep of all grains of a wave is one persistent launch and, from the second
    iteration on, each iteration replays a CUDA graph.  ``autotune`` picks the
    column-to-thread mapping and register variant of the persistent sweep.
    """

    def __init__(self, configs: list, mode: str = "mixed"):
        texts = [c if isinstance(c, str) else json.dumps(c) for c in configs]
        arr = (ctypes.c_char_p * len(texts))(*[t.encode() for t in texts])
        lib = _lib.load()
        h = ctypes.c_void_p()
        st = lib.sc_batch_create(arr, len(texts), MODES[mode], ctypes.byref(h))
        if st != 0:
            raise _lib.EngineError(st, (lib.sc_batch_last_error(None) or b"").decode())
        self._h = h
        self.mode = mode
        self.n = len(texts)
        self.grains = []
        for i in range(self.n):
            g = ctypes.c_void_p()
            self._check(lib.sc_batch_grain(h, i, ctypes.byref(g)))
            self.grains.append(_Grain(g, self))

    def _check(self, st: int):
        if st != 0:
            msg = _lib.load().sc_batch_last_error(self._h)
            raise _lib.EngineError(st, (msg or b"").decode())

    def close(self):
        if getattr(self, "_h", None):
            for g in self.grains:
                g.close()
            _lib.load().sc_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def compute(self, n: int = 1) -> int:
        """Up to n iterations of the active grains; returns the number still active."""
        k = ctypes.c_int()
        self._check(_lib.load().sc_batch_compute(self._h, int(n), ctypes.byref(k)))
        return k.value

    def status(self):
        act = np.zeros(self.n, np.int32)
        it = np.zeros(self.n, np.int32)
        res = np.zeros(self.n)
        self._check(_lib.load().sc_batch_status(self._h, _p(act), _p(it), _p(res)))
        return act.astype(bool), it, res

    GRAIN_STATES = ("running", "converged", "at_cap", "diverged")

    def grain_states(self) -> list:
        """Per grain: 'running', 'converged', 'at_cap' (stopped at its
        num_iterations_max) or 'diverged' (frozen after a non-finite residual
        or free energy)."""
        st = np.zeros(self.n, np.int32)
        self._check(_lib.load().sc_batch_grain_state(self._h, _p(st)))
        return [self.GRAIN_STATES[int(v)] for v in st]

    def set_graph(self, enable: bool):
        self._check(_lib.load().sc_batch_set_graph(self._h, int(bool(enable))))

    def config(self, energies_per_thread: int, minb: int):
        """Each grain takes the fewest threads per column that keep at most
        ``energies_per_thread`` energies on a thread; ``minb`` the register variant."""
        self._check(_lib.load().sc_batch_config(self._h, int(energies_per_thread), int(minb)))

    def get_config(self):
        v = [ctypes.c_int() for _ in range(3)]
        self._check(_lib.load().sc_batch_get_config(self._h, *[ctypes.byref(x) for x in v]))
        return tuple(x.value for x in v)

    def autotune(self):
        """Returns the chosen (energies per thread, minb) and the sweep time in ms."""
        lg, mb, ms = ctypes.c_int(), ctypes.c_int(), ctypes.c_double()
        self._check(_lib.load().sc_batch_autotune(self._h, ctypes.byref(lg), ctypes.byref(mb), ctypes.byref(ms)))
        return lg.value, mb.value, ms.value

    def time_sweeps(self, repeats: int = 3) -> float:
        ms = ctypes.c_double()
        self._check(_lib.load().sc_batch_time_sweeps(self._h, int(repeats), ctypes.byref(ms)))
        return ms.value

    def launch_count(self) -> int:
        k = ctypes.c_longlong()
        self._check(_lib.load().sc_batch_launch_count(self._h, ctypes.byref(k)))
        return k.value

    def site_updates(self) -> np.ndarray:
        return np.array([g.site_updates() for g in self.grains], np.int64)

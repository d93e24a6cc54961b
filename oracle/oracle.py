"""TEST INFRASTRUCTURE ONLY -- the CPU oracle for superconga_b200.

A restatement of SuperConga's self-consistency hot path on the CPU, used as
the checker for the CUDA product path.  Only tests/, ``__graft_entry__.smoke()``
and bench.py's CPU-baseline leg may import this module; the product never
does.

The heavy per-angle work lives in ``conga_oracle.cpp`` (built into
``oracle/_build/libconga_oracle.so``).  This module does the host-side setup
the reference does in C++ with LAPACK/Armadillo, here with numpy/scipy's
LAPACK (the same routines: ``dsygv`` for the Ozaki poles, ``dsyevd`` for the
Poisson filters), and parses the reference's JSON configuration.

Reference citations are paths inside the reference project.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD, "libconga_oracle.so")

GRAIN_SIZE_MARGIN = 3  # include/conga/defines.h:25
MAXIMUM_COORDINATE = 0.5  # include/conga/defines.h:31
EULER_MASCHERONI = 0.57721566490153286060651209008240243
S_WAVE_BULK = 0.5 * math.exp(-EULER_MASCHERONI)  # defines.h:41
D_WAVE_BULK = math.exp(-EULER_MASCHERONI - 0.5) / math.sqrt(2.0)  # defines.h:46

# Parameters::m_maxOzakiPole, include/conga/Parameters.h:191-258 (first 60
# entries; larger counts use the polynomial fit of Parameters.h:402-418).
MAX_OZAKI_POLE = [
    3.464101615138, 13.043193723013, 27.182805923222, 46.319508681820,
    70.526709814647, 99.819209820145, 134.201334576035, 173.674723843717,
    218.240115243641, 267.897882477874, 322.648232120917, 382.491286239281,
    447.427120870950, 517.455785454923, 592.577313298030, 672.791727521291,
    758.099044591524, 848.499276499387, 943.992432147387, 1044.578518259219,
    1150.257539991102, 1261.029501351330, 1376.894405494319, 1497.852254930454,
    1623.903051677801, 1755.046797373544, 1891.283493357799, 2032.613140735255,
    2179.035740424027, 2330.551293191541, 2487.159799683865, 2648.861260447426,
    2815.655675948037, 2987.543046583090, 3164.523372695167, 3346.596654578822,
    3533.762892490810, 3726.022086653727, 3923.374237262044, 4125.819344486381,
    4333.357408476837, 4545.988429367131, 4763.712407272654, 4986.529342298375,
    5214.439234539534, 5447.442084074518, 5685.537890980710, 5928.726655323640,
    6177.008377162879, 6430.383056551208, 6688.850693540401, 6952.411288172675,
    7221.064840486898, 7494.811350521523, 7773.650818306208, 8057.583243876886,
    8346.608627256021, 8640.726968470750, 8939.938267543248, 9244.242524494641,
]

SYMMETRIES = ["dx2-y2", "dxy", "g", "s"]  # src/simulation.cu:213
SYMMETRY_ID = {"s": 0, "dx2-y2": 1, "dxy": 2, "g": 3}
ACCELERATOR_ID = {"congacc": 0, "picard": 1, "polyak": 2,
                  "barzilai-borwein": 3, "bb": 3, "anderson": 4}
GAUGE_ID = {"landau": 0, "symmetric": 1, "solenoid": 2}
NORM_ID = {"l1": 0, "l2": 1, "linf": 2}


def build(force: bool = False) -> str:
    """Compile conga_oracle.cpp into oracle/_build (g++ -O2 -fopenmp)."""
    src = os.path.join(HERE, "conga_oracle.cpp")
    if (not force and os.path.exists(LIB_PATH)
            and os.path.getmtime(LIB_PATH) >= os.path.getmtime(src)):
        return LIB_PATH
    os.makedirs(BUILD, exist_ok=True)
    tmp = LIB_PATH + ".tmp"
    subprocess.check_call(["g++", "-std=c++17", "-O2", "-fopenmp", "-fPIC",
                           "-shared", "-o", tmp, src])
    os.replace(tmp, LIB_PATH)
    return LIB_PATH


REF_INCLUDE = os.environ.get("SCB_REFERENCE_INCLUDE", "/root/reference/include")
REF_DIR = os.path.join(HERE, "_ref")
REF_LIB = os.path.join(REF_DIR, "libscb_ref.so")


def build_ref(force: bool = False):
    """Compile ref_harness.cpp against the reference's own header files, read
    where they lie (REF_INCLUDE), into oracle/_ref/libscb_ref.so: g++ on the
    reference's CPU backend (Thrust on OpenMP; the flags of the reference's
    CMakeLists.txt:192-214), Thrust from the CUDA toolkit's headers.  Returns
    the library path, or None when the reference tree is not present (then a
    library built earlier is used if there is one)."""
    src = os.path.join(HERE, "ref_harness.cpp")
    if not os.path.isdir(os.path.join(REF_INCLUDE, "conga")):
        return REF_LIB if os.path.exists(REF_LIB) else None
    if not force and os.path.exists(REF_LIB) and os.path.getmtime(REF_LIB) >= os.path.getmtime(src):
        return REF_LIB
    os.makedirs(REF_DIR, exist_ok=True)
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    tmp = REF_LIB + ".tmp"
    subprocess.check_call([
        "g++", "-std=c++17", "-O2", "-DNDEBUG", "-fopenmp", "-fPIC", "-shared", "-x", "c++",
        "-DCONGA_BACKEND_CPU=1", "-DTHRUST_DEVICE_SYSTEM=THRUST_DEVICE_SYSTEM_OMP",
        "-DTHRUST_HOST_SYSTEM=THRUST_HOST_SYSTEM_CPP", "-D_LIBCUDACXX_STRING_H_HAS_CONST_OVERLOADS=1",
        "-I", REF_INCLUDE, "-I", cuda_inc, src, "-o", tmp])
    os.replace(tmp, REF_LIB)
    return REF_LIB


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("n0", ctypes.c_int), ("n1", ctypes.c_int), ("n_angles", ctypes.c_int),
        ("n_energies", ctypes.c_int), ("n_comp", ctypes.c_int),
        ("h", ctypes.c_double), ("grain_fraction", ctypes.c_double),
        ("temperature", ctypes.c_double), ("flux_quanta", ctypes.c_double),
        ("penetration_depth", ctypes.c_double),
        ("convergence_criterion", ctypes.c_double),
        ("charge_sign", ctypes.c_int), ("norm_type", ctypes.c_int),
        ("gauge", ctypes.c_int), ("crystal_axes_rotation", ctypes.c_double),
        ("accelerator", ctypes.c_int), ("acc_step_size", ctypes.c_double),
        ("acc_step_size_factor", ctypes.c_double),
        ("acc_cos_similarity_min", ctypes.c_double),
        ("acc_step_size_max", ctypes.c_double),
        ("acc_step_size_min", ctypes.c_double), ("acc_drag", ctypes.c_double),
        ("acc_rank", ctypes.c_int), ("n_filters", ctypes.c_int),
        ("vp_scale", ctypes.c_double),
        ("fs_type", ctypes.c_int), ("tb_nnn", ctypes.c_double),
        ("tb_nnnn", ctypes.c_double), ("tb_mu", ctypes.c_double),
    ]


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(build())
        _lib.orc_create.restype = ctypes.c_void_p
        _lib.orc_compute_bc.restype = ctypes.c_double
        for name in ["orc_destroy", "orc_set_state", "orc_compute", "orc_burn_in",
                     "orc_get_state", "orc_get_results", "orc_get_scalars",
                     "orc_is_converged", "orc_get_geometry", "orc_get_domain",
                     "orc_boundary_sizes", "orc_get_boundary", "orc_set_boundary",
                     "orc_get_ranges", "orc_angle_greens", "orc_energy_shift",
                     "orc_set_boundary_initial", "orc_compute_bc", "orc_poisson",
                     "orc_num_iterations"]:
            getattr(_lib, name).argtypes = None
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------- setup ---
def num_ozaki_poles(temperature: float, cutoff: float) -> int:
    """Parameters::computeNumOzakiEnergies, include/conga/Parameters.h:380-420."""
    val = 2.0 * math.pi * (cutoff / temperature)
    for i, p in enumerate(MAX_OZAKI_POLE):
        if p > val:
            return i + 1
    c2, c1, c0 = 2.5465, 1.2744, 0.4651
    i = len(MAX_OZAKI_POLE) - 1
    while True:
        i += 1
        x = float(i)
        if x * (c2 * x + c1) + c0 >= val:
            return i


def ozaki_poles(n: int):
    """IntegrationIteratorOzaki::computeOzakiPoles, IntegrationIteratorOzaki.h:108-163.

    Generalized eigenproblem A z = w B z (LAPACK dsygv, ITYPE 1, upper), with
    B_ii = 2i+1 and A_{i,i+1} = A_{i+1,i} = -1/2 of size 2n.
    """
    import scipy.linalg
    N = 2 * n
    A = np.zeros((N, N))
    B = np.zeros((N, N))
    for i in range(N):
        B[i, i] = i * 2.0 + 1.0
        if i < N - 1:
            A[i, i + 1] = -0.5
            A[i + 1, i] = -0.5
    w, z = scipy.linalg.eigh(A, B, lower=False, type=1, driver="gv")
    poles = np.empty(n)
    residues = np.empty(n)
    for i in range(n):
        pole = -1.0 / w[i]
        rs = 0.5 * z[0, i] * pole
        poles[i] = pole
        residues[i] = rs * rs
    return poles, residues


def lattice(grain_width: float, ppxi: float):
    """Parameters::setLatticeResolution / computeGridResolutionRotated, Parameters.h:422-458."""
    frac = grain_width * ppxi
    n0 = int(math.ceil(frac)) + 2 * GRAIN_SIZE_MARGIN
    grain_fraction = frac / float(n0)
    margin = int(math.ceil(0.5 * (math.sqrt(2.0) - 1.0) * float(n0)))
    return n0, n0 + 2 * margin, grain_fraction


def geometry_scaling(cfg: dict):
    """geometry_utils::computeGeometryScaling, include/conga/geometry/geometry_utils.h:41-172."""
    tiny = np.finfo(np.float64).tiny
    big = np.finfo(np.float64).max
    x_max, x_min, y_max, y_min = tiny, big, tiny, big
    for comp in cfg["geometry"]:
        name = list(comp.keys())[0]
        d = comp[name]
        if not d.get("add", False):
            continue
        if name == "disc":
            r, cx, cy = float(d["radius"]), float(d.get("center_x", 0.0)), float(d.get("center_y", 0.0))
            x_max, x_min = max(x_max, cx + r), min(x_min, cx - r)
            y_max, y_min = max(y_max, cy + r), min(y_min, cy - r)
        elif name == "polygon":
            for x, y in zip(d["vertices_x"], d["vertices_y"]):
                x_max, x_min = max(x_max, float(x)), min(x_min, float(x))
                y_max, y_min = max(y_max, float(y)), min(y_min, float(y))
        elif name == "regular_polygon":
            side = float(d["side_length"])
            cx, cy = float(d.get("center_x", 0.0)), float(d.get("center_y", 0.0))
            rot = 2.0 * math.pi * float(d.get("rotation", 0.0))
            ne = float(int(d["num_edges"]))
            step = 2.0 * math.pi / ne
            radius = side / math.hypot(math.cos(step) - 1.0, math.sin(step))
            off = 0.5 * step + rot
            for k in range(int(ne)):
                ang = off + step * float(k)
                x, y = cx + radius * math.cos(ang), cy + radius * math.sin(ang)
                x_max, x_min = max(x_max, x), min(x_min, x)
                y_max, y_min = max(y_max, y), min(y_min, y)
        else:
            raise ValueError(f"unknown geometry type {name!r}")
    xe, ye = x_max - x_min, y_max - y_min
    return max(xe, ye), x_min + 0.5 * xe, y_min + 0.5 * ye


def geometry_components(cfg: dict, scaling: float, xo: float, yo: float, gf: float):
    """geometry_utils::addGeometryComponents + component constructors.

    geometry_utils.h:189-325, DiscGeometry.h:243-254, PolygonGeometry.h:255-325,
    Polygon.h:131-153.  Returns (type, add, nvert, data) lists.
    """
    types, adds, nverts, data = [], [], [], []
    for comp in cfg["geometry"]:
        name = list(comp.keys())[0]
        d = comp[name]
        add = 1 if d.get("add", False) else 0
        if name == "disc":
            cx = (float(d.get("center_x", 0.0)) - xo) / scaling
            cy = (float(d.get("center_y", 0.0)) - yo) / scaling
            r = float(d["radius"]) / scaling
            types.append(0); adds.append(add); nverts.append(0)
            data += [r * gf, cx * gf, cy * gf]
        elif name == "polygon":
            vx = [(float(v) - xo) / scaling * gf for v in d["vertices_x"]]
            vy = [(float(v) - yo) / scaling * gf for v in d["vertices_y"]]
            types.append(1); adds.append(add); nverts.append(len(vx))
            data += vx + vy
        elif name == "regular_polygon":
            cx = (float(d.get("center_x", 0.0)) - xo) / scaling
            cy = (float(d.get("center_y", 0.0)) - yo) / scaling
            side = float(d["side_length"]) / scaling
            n = int(d["num_edges"])
            rot = 2.0 * math.pi * float(d.get("rotation", 0.0))
            step = 2.0 * math.pi / float(n)
            rfs = side / math.hypot(math.cos(step) - 1.0, math.sin(step))
            radius = MAXIMUM_COORDINATE if side < 0.0 else rfs
            rp, cpx, cpy = radius * gf, cx * gf, cy * gf
            off = step * 0.5 + rot
            vx, vy = [], []
            for k in range(n):
                ang = step * float(k) + off
                vx.append(rp * math.cos(ang) + cpx)
                vy.append(rp * math.sin(ang) + cpy)
            types.append(1); adds.append(add); nverts.append(n)
            data += vx + vy
        else:
            raise ValueError(f"unknown geometry type {name!r}")
    return types, adds, nverts, data


def poisson_filters(n0: int, h: float, max_error: float, analytical: bool = True):
    """ComputeVectorPotential::makeFilter2D / initializeFilters / addFilter1D.

    include/conga/compute/ComputeVectorPotential.h:212-416, by default with the
    analytical matrix elements (the driver's default,
    ComputeVectorPotential.h:153-156); analytical=False takes the point values
    2 log|r| and the origin value pi/2 - log 2 - 3 (:269-282) as the reference's
    legacy comparison does.  Returns (filters [K, 2*n0-1], positive flags [K],
    scale).
    """
    i = np.arange(n0, dtype=np.float64)
    I, J = np.meshgrid(i, i, indexing="ij")

    def alpha(a, b):
        dist = np.hypot(a, b)
        return (a * b) * (2.0 * np.log(dist) - math.log(2.0))

    def beta(a, b):
        fac = 0.5 * ((2.0 - a + b) * (a + b) - 2.0)
        return fac * np.arctan(a / b)

    if analytical:
        Q = np.zeros((n0, n0))
        for jsgn in (-1.0, 1.0):
            b = 1.0 + 2.0 * (jsgn * J)
            for isgn in (-1.0, 1.0):
                a = 1.0 + 2.0 * (isgn * I)
                Q += alpha(a, b) + beta(a, b) + beta(b, a)
        Q *= 0.25
    else:
        with np.errstate(divide="ignore"):
            Q = 2.0 * np.log(np.hypot(I, J))
        Q[0, 0] = 0.5 * math.pi - math.log(2.0) - 3.0
    Q = 0.5 * (Q + Q.T)
    scale = 1.0 / (4.0 * math.pi)
    Q *= scale
    const = ((2.0 * math.log(h) - math.log(2.0) - 3.0) if analytical else 2.0 * math.log(h)) * scale
    meanQ = Q.mean()
    Q -= meanQ
    const += meanQ
    w, v = np.linalg.eigh(Q)
    m_scale = 0.5 * (np.abs(w).max() + abs(const))
    filters, pos = [], []

    def add_filter(vec, val):
        sq = math.sqrt(abs(val) / m_scale)
        idx = np.abs(np.arange(-n0 + 1, n0))
        filters.append(vec[idx] * sq)
        pos.append(1 if val > 0.0 else 0)

    if abs(const) > 0.0:
        add_filter(np.ones(n0), const)
    order = np.argsort(-np.abs(w), kind="stable")
    norm2 = float(np.linalg.norm(w)) ** 2
    partial = 0.0
    for k in order:
        val = float(w[k])
        add_filter(v[:, k], val)
        partial += val * val
        err = math.sqrt(max(1.0 - partial / norm2, 0.0))
        if err < max_error:
            break
    return np.array(filters), np.array(pos, dtype=np.int32), m_scale


def bulk_s_wave(temperature: float, crit: float = 10.0 * np.finfo(np.float64).eps,
                max_it: int = 10, cutoff: float = 100.0) -> float:
    """computeOrderParameterBulkSWave, include/conga/order_parameter/OrderParameterBulk.h:88-221."""
    if temperature >= 1.0:
        return 0.0
    if temperature < np.finfo(np.float64).eps:
        return S_WAVE_BULK
    ne = int(cutoff / temperature - 0.5) + 1
    esum = 0.0
    for n in range(ne - 1, -1, -1):
        esum += 1.0 / (temperature * (n + 0.5))
    coupling = 1.0 / (math.log(temperature) / temperature + esum)

    def resid(op):
        integrand = 0.0
        for n in range(ne - 1, -1, -1):
            integrand += 1.0 / math.hypot(op, temperature * (n + 0.5))
        return op * (integrand * coupling - 1.0)

    op = S_WAVE_BULK * math.sqrt(1.0 - temperature ** 3)
    ops = [op, math.sqrt(op)]
    res = [resid(ops[0]), resid(ops[1])]
    for _ in range(max_it):
        w = 1.0 / (1.0 - (ops[0] / ops[1]) / (res[0] / res[1]))
        op = (1.0 - w) * ops[0] + w * ops[1]
        r = resid(op)
        small = op < 10.0 * np.finfo(np.float64).eps
        rel = r if small else abs(r / op)
        if rel < crit:
            break
        k = 0 if abs(res[0]) > abs(res[1]) else 1
        ops[k], res[k] = op, r
    return op


def bulk_free_energy_s_wave(temperature: float, op: float, cutoff: float = 100.0) -> float:
    """computeFreeEnergyBulkSWave, include/conga/order_parameter/OrderParameterBulk.h:224-246."""
    ne = int(cutoff / temperature - 0.5) + 1
    esum = 0.0
    for n in range(ne - 1, -1, -1):
        e = temperature * (n + 0.5)
        esum += 1.0 / e - 2.0 / (e + math.hypot(op, e))
    return op * op * (math.log(temperature) + temperature * esum)


def bulk_yoshida_s_wave(temperature: float, op: float, cutoff: float) -> float:
    """computeYoshidaBulkSWave, include/conga/order_parameter/OrderParameterBulk.h:256-277."""
    if temperature < np.finfo(np.float64).eps:
        return 1.0
    ne = int(cutoff / temperature - 0.5) + 1
    esum = 0.0
    for n in range(ne - 1, -1, -1):
        esum += 1.0 / math.hypot(op, temperature * (n + 0.5)) ** 3
    return temperature * op * op * esum


def delta_bulk(temperature: float, symmetry: str) -> float:
    """OrderParameterComponent::deltaBulk, OrderParameterComponent.h:210-235."""
    s = bulk_s_wave(temperature)
    if symmetry in ("g", "dxy", "dx2-y2"):
        return s * (D_WAVE_BULK / S_WAVE_BULK)
    return s


@dataclass
class Setup:
    """Host-side setup values for one configuration (the Parameters module and
    friends)."""
    cfg: dict
    n0: int
    n1: int
    h: float
    grain_fraction: float
    grain_width: float
    temperature: float
    n_angles: int
    poles: np.ndarray
    residues: np.ndarray
    energies_im: np.ndarray
    symmetries: list
    tcs: list
    geom: tuple
    filters: np.ndarray
    filter_pos: np.ndarray
    vp_scale: float
    params: OrcParams = field(repr=False, default=None)

    @property
    def n_comp(self) -> int:
        return len(self.symmetries)

    @property
    def n_energies(self) -> int:
        return int(self.params.n_energies) if self.params is not None else len(self.poles)


def make_setup(cfg: dict, component_order: list | None = None) -> Setup:
    """Mirror of src/simulation.cu:90-463 (everything up to context.initialize).
    component_order: the order-parameter components in another order than the
    driver's (dx2-y2, dxy, g, s), as a C++ caller of OrderParameter::add may
    add them."""
    phys, num = cfg["physics"], cfg["numerics"]
    temperature = float(phys["temperature"])
    ppxi = float(num["points_per_coherence_length"])
    cutoff = float(num["energy_cutoff"])
    scaling, xo, yo = geometry_scaling(cfg)
    n0, n1, gf = lattice(scaling, ppxi)
    h = 1.0 / ppxi
    ne = num_ozaki_poles(temperature, cutoff)
    poles, residues = ozaki_poles(ne)
    energies_im = poles * temperature / (2.0 * math.pi)
    geom = geometry_components(cfg, scaling, xo, yo, gf)
    ops = phys["order_parameter"]
    syms = [s for s in SYMMETRIES if s in ops]
    if component_order is not None:
        if sorted(component_order) != sorted(syms):
            raise ValueError("component_order must list the configured components")
        syms = list(component_order)
    if not syms:
        raise ValueError("no order-parameter component")
    tcs = [float(ops[s].get("critical_temperature", 1.0)) for s in syms]
    lam = float(phys.get("penetration_depth", -1.0))
    if lam > 0.0:
        filters, fpos, vscale = poisson_filters(n0, h, float(num.get("vector_potential_error", 1e-6)))
    else:
        filters, fpos, vscale = np.zeros((0, 2 * n0 - 1)), np.zeros(0, np.int32), 1.0
    acc = cfg.get("accelerator", {"name": "congacc"})
    aname = acc.get("name", "congacc")
    defaults = {  # Accelerator default constants, include/conga/accelerators/*.h
        0: dict(step_size=0.5), 1: dict(step_size=1.0), 2: dict(step_size=2.0),
        3: dict(step_size=1.0), 4: dict(step_size=1.0)}
    aid = ACCELERATOR_ID[aname]
    p = OrcParams()
    p.n0, p.n1, p.n_angles = n0, n1, int(num["num_fermi_momenta"])
    p.n_energies, p.n_comp = ne, len(syms)
    p.h, p.grain_fraction, p.temperature = h, gf, temperature
    p.flux_quanta = float(phys.get("external_flux_quanta", 0.0))
    p.penetration_depth = lam
    p.convergence_criterion = float(num.get("convergence_criterion", 1e-6))
    cs = int(phys.get("charge_sign", -1))
    p.charge_sign = (cs > 0) - (cs < 0)
    p.norm_type = NORM_ID[num.get("norm", "l2")]
    p.gauge = GAUGE_ID[phys.get("gauge", "symmetric")]
    p.crystal_axes_rotation = 2.0 * math.pi * float(phys.get("crystal_axes_rotation", 0.0))
    p.accelerator = aid
    p.acc_step_size = float(acc.get("step_size", defaults[aid]["step_size"]))
    p.acc_step_size_factor = float(acc.get("step_size_factor", 1.234))
    p.acc_cos_similarity_min = float(acc.get("cos_similarity_min", 0.7))
    p.acc_step_size_max = float(acc.get("step_size_max", 100.0))
    p.acc_step_size_min = float(acc.get("step_size_min", 0.001))
    p.acc_drag = float(acc.get("drag", 0.5))
    p.acc_rank = int(acc.get("rank", 4))
    p.n_filters = len(filters)
    p.vp_scale = vscale
    # Fermi surface: the circle, or the tight-binding surface that the
    # reference sets in code (Context::set, Context.h:49-51); JSON spelling
    # physics.fermi_surface = {"type": "tight_binding", ...}.
    fs = phys.get("fermi_surface", {"type": "circle"})
    if fs.get("type", "circle") == "tight_binding":
        p.fs_type = 1
        p.tb_nnn = float(fs.get("hopping_nnn", 0.0))
        p.tb_nnnn = float(fs.get("hopping_nnnn", 0.0))
        p.tb_mu = float(fs.get("chemical_potential", 1.0))
    elif fs.get("type", "circle") != "circle":
        raise ValueError(f"fermi_surface type {fs.get('type')!r} not understood")
    return Setup(cfg=cfg, n0=n0, n1=n1, h=h, grain_fraction=gf, grain_width=scaling,
                 temperature=temperature, n_angles=p.n_angles, poles=poles,
                 residues=residues, energies_im=energies_im, symmetries=syms,
                 tcs=tcs, geom=geom, filters=np.ascontiguousarray(filters, np.float64),
                 filter_pos=np.ascontiguousarray(fpos, np.int32), vp_scale=vscale,
                 params=p)


class Oracle:
    """One self-consistency context on the CPU (mirror of conga::Context)."""

    def __init__(self, cfg: dict | str, energies: tuple | None = None,
                 component_order: list | None = None):
        """energies: optional (imaginary parts, residues) replacing the Ozaki
        set (the LDOS path sweeps real energies with a common broadening);
        component_order: see make_setup."""
        if isinstance(cfg, str):
            cfg = json.loads(cfg)
        self.setup = s = make_setup(cfg, component_order)
        e_im, e_res = s.energies_im, s.residues
        if energies is not None:
            e_im, e_res = (np.ascontiguousarray(v, np.float64) for v in energies)
            s.params.n_energies = len(e_im)
        L = lib()
        types, adds, nverts, data = s.geom
        self._keep = [
            np.ascontiguousarray(e_im, np.float64),
            np.ascontiguousarray(e_res, np.float64),
            np.array([SYMMETRY_ID[x] for x in s.symmetries], np.int32),
            np.array(s.tcs, np.float64),
            np.array(types, np.int32), np.array(adds, np.int32),
            np.array(nverts, np.int32), np.array(data, np.float64),
            s.filters if len(s.filters) else np.zeros(1), s.filter_pos if len(s.filter_pos) else np.zeros(1, np.int32),
        ]
        k = self._keep
        self.h = ctypes.c_void_p(L.orc_create(ctypes.byref(s.params), _ptr(k[0]), _ptr(k[1]),
                                              _ptr(k[2]), _ptr(k[3]), ctypes.c_int(len(types)),
                                              _ptr(k[4]), _ptr(k[5]), _ptr(k[6]), _ptr(k[7]),
                                              _ptr(k[8]), _ptr(k[9])))
        self.n0, self.n1 = s.n0, s.n1

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_destroy(self.h)
        except Exception:
            pass

    def set_state(self, delta: np.ndarray, a_internal: np.ndarray | None = None):
        d = np.ascontiguousarray(delta, np.float64)
        assert d.size == self.setup.n_comp * 2 * self.n0 * self.n0
        a = None if a_internal is None else np.ascontiguousarray(a_internal, np.float64)
        lib().orc_set_state(self.h, _ptr(d), _ptr(a) if a is not None else None)

    def compute(self):
        lib().orc_compute(self.h)

    def burn_in(self):
        lib().orc_burn_in(self.h)

    def evaluate(self) -> float:
        """Frozen-boundary evaluation; returns the free energy."""
        lib().orc_evaluate(self.h)
        return self.scalars()["free_energy"]

    def set_flux(self, flux_quanta: float):
        lib().orc_set_flux(self.h, ctypes.c_double(flux_quanta))

    def state(self):
        n = self.n0
        d = np.zeros((self.setup.n_comp, 2, n, n))
        a = np.zeros((2, n, n))
        lib().orc_get_state(self.h, _ptr(d), _ptr(a))
        return d, a

    def results(self):
        n = self.n0
        d = np.zeros((self.setup.n_comp, 2, n, n))
        j = np.zeros((2, n, n))
        a = np.zeros((2, n, n))
        lib().orc_get_results(self.h, _ptr(d), _ptr(j), _ptr(a))
        return d, j, a

    def scalars(self) -> dict:
        out = np.zeros(11)
        lib().orc_get_scalars(self.h, _ptr(out))
        keys = ["free_energy", "free_energy_per_area", "magnetic_free_energy",
                "magnetic_free_energy_per_area", "res_order_parameter", "res_current",
                "res_free_energy", "res_vector_potential", "res_boundary", "residual",
                "n_grain"]
        return dict(zip(keys, out.tolist()))

    def is_converged(self) -> bool:
        return bool(lib().orc_is_converged(self.h))

    def geometry(self, a: int):
        n = self.n1
        lab = np.zeros((n, n), np.int8)
        dist = np.zeros((n, n)); nx = np.zeros((n, n)); ny = np.zeros((n, n))
        lib().orc_get_geometry(self.h, ctypes.c_int(a), _ptr(lab), _ptr(dist), _ptr(nx), _ptr(ny))
        return lab, dist, nx, ny

    def domain(self):
        d = np.zeros((self.n0, self.n0), np.int8)
        lib().orc_get_domain(self.h, _ptr(d))
        return d

    def boundary_sizes(self):
        out = np.zeros(4, np.int32)
        lib().orc_boundary_sizes(self.h, _ptr(out))
        return out.tolist()

    def boundary(self, which: int) -> np.ndarray:
        n = self.boundary_sizes()[which] * self.setup.n_energies
        out = np.zeros(2 * n)
        lib().orc_get_boundary(self.h, ctypes.c_int(which), _ptr(out))
        return out[0::2] + 1j * out[1::2]

    def set_boundary(self, which: int, values: np.ndarray):
        v = np.ascontiguousarray(np.stack([values.real, values.imag], -1).ravel(), np.float64)
        lib().orc_set_boundary(self.h, ctypes.c_int(which), _ptr(v))

    def ranges(self):
        na = self.setup.n_angles
        x0, x1, y0, y1 = (np.zeros(na, np.int32) for _ in range(4))
        lib().orc_get_ranges(self.h, _ptr(x0), _ptr(x1), _ptr(y0), _ptr(y1))
        return x0, x1, y0, y1

    def angle_greens(self, a: int):
        n = self.n1
        arrs = [np.zeros((n, n)) for _ in range(6)]
        lib().orc_angle_greens(self.h, ctypes.c_int(a), *[_ptr(x) for x in arrs])
        fre, fim, gre, ire, dre, dim = arrs
        return fre + 1j * fim, gre, ire, dre + 1j * dim

    def energy_shift(self, a: int):
        es = np.zeros((self.n1, self.n1))
        lib().orc_energy_shift(self.h, ctypes.c_int(a), _ptr(es))
        return es

    def set_boundary_initial(self):
        lib().orc_set_boundary_initial(self.h)

    def compute_bc(self) -> float:
        return float(lib().orc_compute_bc(self.h))

    def poisson(self, j: np.ndarray) -> np.ndarray:
        jj = np.ascontiguousarray(j, np.float64)
        out = np.zeros((2, self.n0, self.n0))
        lib().orc_poisson(self.h, _ptr(jj), _ptr(out))
        return out


class LdosOracle:
    """The LDOS postprocess on the CPU (src/postprocess.cu:60-425 with
    runPostprocess, run_simulation.h:44-104): the simulation configuration with
    angles, criterion and norm from the postprocess configuration; real
    energies E_k + i delta (IntegrationIteratorKeldysh.h:91-160) swept one
    block at a time."""

    def __init__(self, simulation: dict, postprocess: dict):
        cfg = json.loads(json.dumps(simulation))
        num, ppn, sp = cfg["numerics"], postprocess["numerics"], postprocess["spectroscopy"]
        num["num_fermi_momenta"] = int(ppn["num_fermi_momenta"])
        num["convergence_criterion"] = float(ppn["convergence_criterion"])
        num["norm"] = ppn.get("norm", "l2")
        ne = int(sp["num_energies"])
        emin, emax = float(sp["energy_min"]), float(sp["energy_max"])
        step = (emax - emin) / (ne - 1) if ne > 1 else 0.0
        self.energies = np.array([emin + step * i for i in range(ne)])
        self.broadening = float(sp["energy_broadening"])
        per = int(ppn.get("num_energies_per_block", 0))
        self.block = ne if per < 1 else min(per, ne)
        self.n_blocks = (ne + self.block - 1) // self.block
        self.oracle = Oracle(cfg, (np.full(self.block, self.broadening), np.zeros(self.block)))
        self.n0 = self.oracle.n0
        self.ldos = np.zeros((ne, self.n0, self.n0))
        self.current = -1

    def set_state(self, delta, a_internal=None):
        self.oracle.set_state(delta, a_internal)

    def begin_block(self, b: int):
        ne = len(self.energies)
        e = np.array([self.energies[min(b * self.block + i, ne - 1)] for i in range(self.block)])
        self._e = np.ascontiguousarray(e)
        lib().orc_set_energies_re(self.oracle.h, _ptr(self._e))
        self.current = b

    def count(self, b: int) -> int:
        return min(self.block, len(self.energies) - b * self.block)

    def burn_in(self) -> float:
        self.oracle.burn_in()
        return self.oracle.scalars()["res_boundary"]

    def iterate(self):
        """One LDOS iteration; returns (residual, LDOS residual, boundary residual)."""
        nf = self.count(self.current)
        out = np.zeros((nf, self.n0, self.n0))
        rl, rb = ctypes.c_double(), ctypes.c_double()
        lib().orc_ldos_iterate(self.oracle.h, nf, _ptr(out), ctypes.byref(rl), ctypes.byref(rb))
        b0 = self.current * self.block
        self.ldos[b0:b0 + nf] = out
        return max(rl.value, rb.value), rl.value, rb.value


def extend_grid(labels: np.ndarray, values: np.ndarray) -> np.ndarray:
    """extendValuesAtBoundary of one plane (domain_ops.h:11-69)."""
    n = labels.shape[0]
    lab = np.ascontiguousarray(labels, np.int8)
    out = np.ascontiguousarray(values, np.float64).copy()
    lib().orc_extend_grid(ctypes.c_int(n), _ptr(lab), _ptr(out))
    return out


def resample_grid(src: np.ndarray, n_new: int, margin: int = 3) -> np.ndarray:
    """GridFunctions::resample, resample_kernel (GridFunctions_GPU.h:547-600):
    bilinear onto an n_new lattice with the safety margin mapped onto itself.
    Reads past the old lattice (only in the margin when shrinking) are
    clamped to the edge."""
    n_old = src.shape[-1]
    scale = (n_old - 1 - 2 * margin) / (n_new - 1 - 2 * margin)
    idx = np.arange(n_new)
    o = scale * (idx - margin).astype(np.float64) + margin
    f = np.trunc(o).astype(np.int64)
    fr = o - f
    nx = (idx < n_new - 1).astype(np.int64)
    c = lambda i: np.clip(i, 0, n_old - 1)
    y0, y1 = c(f)[:, None], c(f + nx)[:, None]
    x0, x1 = c(f)[None, :], c(f + nx)[None, :]
    fx, fy = fr[None, :], fr[:, None]
    p = np.asarray(src, np.float64)
    a = (1.0 - fx) * p[..., y0, x0] + fx * p[..., y0, x1]
    b = (1.0 - fx) * p[..., y1, x0] + fx * p[..., y1, x1]
    return (1.0 - fy) * a + fy * b


def riccati_step(delta: complex, energy: complex, g0: complex, h: float) -> complex:
    L = lib()
    d = np.array([delta.real, delta.imag]); e = np.array([energy.real, energy.imag])
    g = np.array([g0.real, g0.imag]); out = np.zeros(2)
    L.orc_riccati_step(_ptr(d), _ptr(e), _ptr(g), ctypes.c_double(h), _ptr(out))
    return complex(out[0], out[1])


def homogeneous(delta: complex, energy: complex):
    L = lib()
    d = np.array([delta.real, delta.imag]); e = np.array([energy.real, energy.imag])
    out = np.zeros(4)
    L.orc_homogeneous(_ptr(d), _ptr(e), _ptr(out))
    return complex(out[0], out[1]), complex(out[2], out[3])


def greens(g: complex, gt: complex):
    L = lib()
    a = np.array([g.real, g.imag]); b = np.array([gt.real, gt.imag]); out = np.zeros(4)
    L.orc_greens(_ptr(a), _ptr(b), _ptr(out))
    return complex(out[0], out[1]), complex(out[2], out[3])


def tight_binding(hopping_nnn: float, hopping_nnnn: float, chemical_potential: float,
                  n_angles: int) -> dict:
    """FermiSurfaceTightBinding<double>::initialize (FermiSurfaceTightBinding.h:
    384-470) on its own: per-angle polar angle, system angle, Fermi momentum,
    normalised Fermi velocity, integrand factor and speed, plus the mean |p_F|
    and |v_F| before normalisation and the momentum origin."""
    L = lib()
    t = np.zeros((8, n_angles))
    info = np.zeros(4)
    L.orc_tight_binding(ctypes.c_double(hopping_nnn), ctypes.c_double(hopping_nnnn),
                        ctypes.c_double(chemical_potential), ctypes.c_int(n_angles), _ptr(t), _ptr(info))
    keys = ["phi", "theta", "px", "py", "vx", "vy", "weight", "speed"]
    out = {k: t[i].copy() for i, k in enumerate(keys)}
    out.update(avg_fermi_momentum=float(info[0]), avg_fermi_speed=float(info[1]),
               origin=(float(info[2]), float(info[3])))
    return out

// conga_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of SuperConga's self-consistency iteration (the Riccati
// sweep, Green-function accumulation, specular boundary condition, vector
// potential Poisson solve and accelerators), written to be checked against
// and to check the CUDA path in superconga_b200.  Only tests/, the smoke()
// entry and bench.py's CPU-baseline leg may load this library; it is never
// part of the product.
//
// It follows the reference's structure on purpose: one Fermi angle at a time,
// full rotated-frame grids, the same interpolation and extension rules.  Every
// function cites the reference file:line it restates (paths relative to the
// reference project root).
//
// Eigen-decompositions (Ozaki poles, Poisson filters) are done by the Python
// driver (oracle/oracle.py) with LAPACK through scipy/numpy and passed in.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------- complex --
struct cx {
  double re, im;
};
inline cx mk(double r, double i) { return cx{r, i}; }
inline cx add(cx a, cx b) { return cx{a.re + b.re, a.im + b.im}; }
inline cx sub(cx a, cx b) { return cx{a.re - b.re, a.im - b.im}; }
inline cx mul(cx a, cx b) {
  return cx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
inline cx scl(cx a, double s) { return cx{a.re * s, a.im * s}; }
inline cx conj_(cx a) { return cx{a.re, -a.im}; }
inline cx neg(cx a) { return cx{-a.re, -a.im}; }
inline cx cdiv(cx a, cx b) {
  const double d = b.re * b.re + b.im * b.im;
  return cx{(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
}
// Principal square root (branch cut on the negative real axis).
inline cx csqrt_(cx z) {
  const double m = std::sqrt(z.re * z.re + z.im * z.im);
  if (z.re >= 0.0) {
    const double t = std::sqrt(0.5 * (m + z.re));
    if (t == 0.0) return cx{0.0, z.im};
    return cx{t, z.im / (2.0 * t)};
  }
  const double t = std::sqrt(0.5 * (m - z.re));
  return cx{std::fabs(z.im) / (2.0 * t), std::copysign(t, z.im)};
}

// ----------------------------------------------------- Riccati algebra ------
// riccati::computeHomogeneous, include/conga/riccati/RiccatiSolutions.h:36-54
inline void homogeneous(cx delta, cx energy, cx &g, cx &gt) {
  const double nd = delta.re * delta.re + delta.im * delta.im;
  const cx e2 = mul(energy, energy);
  const cx omega = csqrt_(cx{nd - e2.re, -e2.im});
  const cx iomega = cx{-omega.im, omega.re};
  const cx inv = cdiv(mk(1.0, 0.0), add(energy, iomega));
  g = mul(neg(delta), inv);
  gt = mul(conj_(delta), inv);
}

// riccati::computeStep, include/conga/riccati/RiccatiSolutions.h:65-94
inline cx riccati_step(cx delta, cx energy, cx g0, double h) {
  const cx q = cx{0.25 * 0.0, 0.25 * h};
  const cx step = cx{0.0, h};
  const cx a = mul(q, conj_(delta));
  const cx b = sub(add(mul(scl(a, 2.0), g0), mul(step, energy)), mk(1.0, 0.0));
  const cx c = add(mul(add(add(mul(a, g0), mul(step, energy)), mk(1.0, 0.0)), g0),
                   mul(delta, step));
  const cx disc = csqrt_(sub(mul(b, b), mul(scl(a, 4.0), c)));
  return cdiv(scl(c, 2.0), add(neg(b), disc));
}

// Greens, include/conga/green/LocalGreens.h:32-43
inline cx greens_g(cx g, cx gt) {
  const cx prod = mul(g, gt);
  const cx tmp = neg(cdiv(sub(mk(1.0, 0.0), prod), add(mk(1.0, 0.0), prod)));
  return cx{-tmp.im, tmp.re};
}
// Greens_Delta, include/conga/green/LocalGreens.h:54-70
inline cx greens_f(cx g, cx gt) {
  const cx tmp = cdiv(mk(2.0, 0.0), add(mk(1.0, 0.0), mul(g, gt)));
  const cx factor = cx{-tmp.im, tmp.re};
  const cx f = mul(neg(factor), g);
  const cx ftc = conj_(mul(factor, gt));
  return add(f, ftc);
}
// computeFreeEnergyKernelI, include/conga/compute/ComputeFreeEnergy.h:95-103
inline cx kernel_i(cx d, cx g, cx gt) {
  return sub(mul(conj_(d), g), mul(d, gt));
}

// ------------------------------------------------------------- utilities ----
// utils::wrapToRange, include/conga/utils.h:34-58
inline double wrap_range(double v, double lo, double hi) {
  if (lo <= v && v < hi) return v;
  const double range = hi - lo;
  const double s = (v - lo) / range;
  return (s - std::floor(s)) * range + lo;
}
inline float wrap_rangef(float v, float lo, float hi) {
  if (lo <= v && v < hi) return v;
  const float range = hi - lo;
  const float s = (v - lo) / range;
  return (s - std::floor(s)) * range + lo;
}
// utils::wrapToRange<int>, include/conga/utils.h:70-78
inline int wrap_int(int v, int lo, int hi) {
  const float f = wrap_rangef((float)v, (float)lo, (float)hi);
  return (int)std::round(f);
}
inline int sign_(double v) { return (0.0 < v) - (v < 0.0); }
inline void rotate(double ang, double x, double y, double &ox, double &oy) {
  const double c = std::cos(ang), s = std::sin(ang);
  ox = x * c - y * s;
  oy = x * s + y * c;
}

struct Grid {  // planar grid, row-major y*N+x
  int n = 0;
  std::vector<double> v;
};

enum { NORM_L1 = 0, NORM_L2 = 1, NORM_LINF = 2 };

// computeResidual(GridData), include/conga/compute/ComputeResidual.h:54-106
double residual_grid(const double *oldv, const double *newv, size_t n, int norm) {
  double numer = 0.0, denom = 0.0, eps = 1e-4;
  if (norm == NORM_L1) {
    for (size_t i = 0; i < n; ++i) {
      numer += std::fabs(oldv[i] - newv[i]);
      denom += std::fabs(oldv[i]);
    }
    eps *= (double)n;
  } else if (norm == NORM_L2) {
    for (size_t i = 0; i < n; ++i) {
      const double d = oldv[i] - newv[i];
      numer += d * d;
      denom += oldv[i] * oldv[i];
    }
    numer = std::sqrt(numer);
    denom = std::sqrt(denom);
    eps *= (double)n;
  } else {
    // LInfNorm, include/conga/grid/GridData.h:949-958 (min seeded with max(),
    // max seeded with the smallest positive normal).
    double mn = std::numeric_limits<double>::max();
    double mx = std::numeric_limits<double>::min();
    double mno = mn, mxo = mx;
    for (size_t i = 0; i < n; ++i) {
      const double d = oldv[i] - newv[i];
      mn = std::min(mn, d);
      mx = std::max(mx, d);
      mno = std::min(mno, oldv[i]);
      mxo = std::max(mxo, oldv[i]);
    }
    numer = std::max(std::fabs(mn), std::fabs(mx));
    denom = std::max(std::fabs(mno), std::fabs(mxo));
  }
  return numer / std::max(denom, eps);
}
double residual_scalar(double o, double n) {
  return std::fabs(o - n) / std::max(std::fabs(o), 1e-4);
}

}  // namespace

extern "C" {

struct orc_params {
  int n0, n1, n_angles, n_energies, n_comp;
  double h, grain_fraction, temperature, flux_quanta, penetration_depth;
  double convergence_criterion;
  int charge_sign, norm_type, gauge; /* gauge: 0 landau, 1 symmetric, 2 solenoid */
  double crystal_axes_rotation;
  int accelerator; /* 0 congacc, 1 picard, 2 polyak, 3 barzilai-borwein, 4 anderson */
  double acc_step_size, acc_step_size_factor, acc_cos_similarity_min;
  double acc_step_size_max, acc_step_size_min, acc_drag;
  int acc_rank;
  int n_filters;
  double vp_scale;
  /* Fermi surface: 0 circle (FermiSurfaceCircle.h), 1 square-lattice tight
   * binding (FermiSurfaceTightBinding.h) with next- and next-next-nearest
   * hopping and chemical potential (nearest hopping 1). */
  int fs_type;
  double tb_nnn, tb_nnnn, tb_mu;
};

}  // extern "C"

namespace {

struct GeomComp {
  int type;  // 0 disc, 1 polygon
  int add;
  double radius, cx_, cy_;  // disc (already scaled by the grain fraction)
  std::vector<double> vx, vy;  // polygon vertices (scaled by the grain fraction)
};

struct AngleGeom {
  std::vector<char> label;
  std::vector<double> nx, ny, dist;
};

struct Oracle {
  orc_params p;
  std::vector<double> e_im, res;  // Ozaki energies (imag part) and residues
  std::vector<double> e_re;       // real parts (zero on the Matsubara axis; LDOS energies)
  std::vector<int> sym;           // basis symmetry per component
  std::vector<double> tc;         // relative Tc per component
  std::vector<double> norm_factor, coupling;
  std::vector<GeomComp> geom;
  std::vector<char> domain_ref;
  int n_grain = 0;
  double area = 0.0;

  // Fermi surface tables.
  std::vector<double> polar, system_angle;
  // Tight-binding surface (p.fs_type == 1): per angle momentum, velocity
  // (normalised), integrand factor and speed; momentum origin.
  std::vector<double> tb_px, tb_py, tb_vx, tb_vy, tb_w, tb_speed;
  double tb_ox = 0.0, tb_oy = 0.0;

  // Per-angle geometry, precomputed (the reference rebuilds it each time, with
  // identical results).
  std::vector<AngleGeom> ag;

  // Boundary storage, include/conga/boundary/BoundaryStorage.h.
  std::vector<int> idx_in_g, idx_out_g, idx_in_gt, idx_out_gt;  // [a*N1+x]
  std::vector<int> nisect_g, nisect_gt;
  std::vector<int> coord_g, coord_gt;
  std::vector<int> xr0, xr1, yr0, yr1;
  int n_in_g = 0, n_out_g = 0, n_in_gt = 0, n_out_gt = 0;
  std::vector<cx> bin_g, bout_g, bin_gt, bout_gt;
  bool boundary_initialized = false;

  // Poisson filters.
  std::vector<std::vector<double>> filters;
  std::vector<int> filter_pos;

  // State: x (context order parameter and induced vector potential, the latter
  // scaled by lambda^2), and the compute-object results g(x).
  std::vector<cx> delta;      // [c][N0*N0]
  std::vector<double> avec;   // [2][N0*N0]
  std::vector<cx> delta_new;  // [c][N0*N0]
  std::vector<double> j_real; // [2][N0*N0]
  std::vector<double> a_new;  // [2][N0*N0]
  double fe = 0, fe_area = 0, fe_mag = 0, fe_mag_area = 0;
  double res_op = 0, res_j = 0, res_fe = 0, res_vp = 0, res_bc = 0;
  bool conv_op = false, conv_j = false, conv_fe = false;
  bool first_compute = true, first_j = true, first_fe = true;
  bool has_vp = false;
  int n_iterations = 0;

  // Accelerator state.
  bool acc_init = false;
  std::vector<double> acc_mean, acc_vel, acc_dprev;
  std::vector<double> acc_step, acc_inertia;
  double bb_step = 0;
  int acc_iter = 0;
  std::vector<std::vector<double>> and_x, and_d;
  std::vector<double> and_sq;
  std::vector<size_t> and_idx;

  // Scratch.
  std::vector<cx> gam, gamt;  // [e][N1*N1]

  int N0() const { return p.n0; }
  int N1() const { return p.n1; }

  // ------------------------------------------------------ Fermi surface ----
  // internal::getPolarAngle, include/conga/fermi_surface/FermiSurface.h:117-125
  double polar_angle(int k) const {
    const double v = M_PI * (double)(2 * k) / (double)p.n_angles + 0.5 * M_PI;
    return wrap_range(v, 0.0, 2.0 * M_PI);
  }
  // FermiSurfaceCircle::getSystemAngle, FermiSurfaceCircle.h:140-143
  double sys_angle(int k) const {
    return system_angle[wrap_int(k, 0, p.n_angles)];
  }
  // FermiSurface::getAngleWeight, FermiSurface.h:210-243
  double angle_weight(int k) const {
    const int n = p.n_angles, w = wrap_int(k, 0, n);
    if (n % 4 == 0) {
      if (w % 4 == 0) return 28.0 / 45.0;
      if (w % 2 == 0) return 24.0 / 45.0;
      return 64.0 / 45.0;
    } else if (n % 3 == 0) {
      return (w % 3 == 0) ? 6.0 / 8.0 : 9.0 / 8.0;
    } else if (n % 2 == 0) {
      return (w % 2 == 0) ? 2.0 / 3.0 : 4.0 / 3.0;
    }
    return 1.0;
  }
  // FermiSurfaceCircle::getIntegrandFactor, FermiSurfaceCircle.h:159-164
  // FermiSurfaceTightBinding::getIntegrandFactor, FermiSurfaceTightBinding.h:504-508
  double integrand(int k) const {
    if (p.fs_type == 1) return tb_w[wrap_int(k, 0, p.n_angles)];
    return angle_weight(k) / (double)p.n_angles;
  }
  void fermi_momentum(int k, double &px, double &py) const {
    if (p.fs_type == 1) {
      const int i = wrap_int(k, 0, p.n_angles);
      px = tb_px[i];
      py = tb_py[i];
      return;
    }
    const double phi = polar_angle(k);
    px = std::cos(phi);
    py = std::sin(phi);
  }
  // getFermiVelocity: the momentum on the circle (FermiSurfaceCircle.h:125-138)
  void fermi_velocity(int k, double &vx, double &vy) const {
    if (p.fs_type == 1) {
      const int i = wrap_int(k, 0, p.n_angles);
      vx = tb_vx[i];
      vy = tb_vy[i];
      return;
    }
    fermi_momentum(k, vx, vy);
  }
  // Riccati step h / |v_F|, RiccatiSolverConfined.h:525-527
  double step_size(int k) const {
    if (p.fs_type == 1) return p.h / tb_speed[wrap_int(k, 0, p.n_angles)];
    return p.h / 1.0;  // |v_F| = 1 on a circular Fermi surface
  }
  // BasisFunction::evaluate, OrderParameterBasis.h:145-219: polynomials of
  // the momentum on the circle, lattice harmonics otherwise.
  double basis_raw(int s, double px, double py) const {
    if (p.fs_type == 1) {
      switch (s) {
      case 0: return std::cos(px) + std::cos(py);
      case 1: return std::cos(px) - std::cos(py);
      case 2: return std::sin(px) * std::sin(py);
      case 3: return std::sin(px) * std::sin(py) * (std::cos(px) - std::cos(py));
      }
      return 0.0;
    }
    switch (s) {
    case 0: return 1.0;
    case 1: return px * px - py * py;
    case 2: return px * py;
    case 3: return px * py * (px * px - py * py);
    }
    return 0.0;
  }
  // OrderParameterComponent::computeMomentumDependence,
  // OrderParameterComponent.h:197-208 (basis is real for a circular surface)
  double basis(int c, double px, double py) const {
    double rx, ry;
    rotate(p.crystal_axes_rotation, px, py, rx, ry);
    return basis_raw(sym[c], rx, ry) * norm_factor[c];
  }

  // ------------------------------------------------------------ geometry ---
  // DiscGeometry::convertCoordinate, include/conga/geometry/DiscGeometry.h:62-70
  double convert_coord(double f, int nsim, int ngrid) const {
    const int diff = ngrid - nsim;
    const double half = 0.5 * (double)diff;
    return (double)(nsim - 1) * (f + 0.5) + half;
  }
  // internal::computeDomainLabel, DiscGeometry.h:75-150
  static char disc_label(int ix, int iy, double r, double ox, double oy) {
    const double r2 = r * r;
    bool nb[3];
    for (int j = 0; j < 3; ++j) {
      const double yy = (double)(iy - 1 + j) - oy;
      int rs = 0;
      for (int i = 0; i < 3; ++i) {
        const double xx = (double)(ix - 1 + i) - ox;
        rs += (xx * xx + yy * yy <= r2) ? 1 : 0;
      }
      nb[j] = rs > 1;
    }
    if (nb[0] && nb[1] && nb[2]) return 1;
    if (!nb[0] && nb[1] && nb[2]) return 2;
    if (nb[0] && nb[1] && !nb[2]) return 3;
    return 0;
  }
  // DiscGeometry::create + generateDisc_Kernel, DiscGeometry.h:152-198,262-283
  void disc_create(const GeomComp &g, double angle, AngleGeom &o) const {
    const int n = N1();
    double rcx, rcy;
    rotate(angle, g.cx_, g.cy_, rcx, rcy);
    const double ox = convert_coord(rcx, N0(), n);
    const double oy = convert_coord(rcy, N0(), n);
    const double r = g.radius * (double)(N0() - 1);
    o.label.assign((size_t)n * n, 0);
    o.nx.assign((size_t)n * n, 0.0);
    o.ny.assign((size_t)n * n, 0.0);
    o.dist.assign((size_t)n * n, 0.0);
    for (int ty = 0; ty < n; ++ty)
      for (int tx = 0; tx < n; ++tx) {
        const char lab = disc_label(tx, ty, r, ox, oy);
        const double x = (double)tx - ox, y = (double)ty - oy;
        double bd = 0.0, nxv = 0.0, nyv = 0.0;
        if (lab > 1) {
          bd = std::sqrt(r * r - x * x) - std::fabs(y);
          nxv = -x / r;
          nyv = (y <= 0.0) ? -(y - bd) / r : -(y + bd) / r;
        }
        const size_t i = (size_t)ty * n + tx;
        o.label[i] = lab;
        o.dist[i] = bd;
        o.nx[i] = nxv;
        o.ny[i] = nyv;
      }
  }
  // PolygonGeometry::create, generatePolygonGeometry_Kernel,
  // labelEntryExit_Kernel, maskNormals_Kernel:
  // include/conga/geometry/PolygonGeometry.h:100-190,234-252,355-381 and
  // include/conga/geometry/GeometryComponent.h:112-147
  void polygon_create(const GeomComp &g, double angle, AngleGeom &o) const {
    const int n = N1();
    const int nv = (int)g.vx.size();
    const double scale = (double)(N0() - 1);
    const double ca = std::cos(angle), sa = std::sin(angle);
    std::vector<double> px(nv), py(nv);
    for (int i = 0; i < nv; ++i) {
      px[i] = (ca * g.vx[i] - sa * g.vy[i]) * scale;
      py[i] = (sa * g.vx[i] + ca * g.vy[i]) * scale;
    }
    std::vector<char> raw((size_t)n * n);
    o.nx.assign((size_t)n * n, 0.0);
    o.ny.assign((size_t)n * n, 0.0);
    o.dist.assign((size_t)n * n, 0.0);
    for (int ty = 0; ty < n; ++ty)
      for (int tx = 0; tx < n; ++tx) {
        const double cxv = (double)tx - (double)(n - 1) * 0.5;
        const double cyv = (double)ty - (double)(n - 1) * 0.5;
        int sum_cross = 0;
        double bd = 100000.0, nxv = 0.0, nyv = 0.0;
        for (int i = 0; i < nv; ++i) {
          int ip = i + 1;
          if (ip == nv) ip = 0;
          const double lx = px[ip] - px[i], ly = py[ip] - py[i];
          const double cz = lx * (cyv - py[i]) - ly * (cxv - px[i]);
          if (cz >= 0.0) sum_cross++;
          double tnx = -ly, tny = lx;
          const double nt = 1.0 / std::sqrt(tnx * tnx + tny * tny);
          tnx *= nt;
          tny *= nt;
          double td;
          if (std::fabs(lx) > 0.00001) {
            const double k = ly / lx;
            const double m = py[i] - k * px[i];
            td = std::fabs(k * cxv + m - cyv);
          } else {
            td = 10000.0;
          }
          if (td < bd) {
            bd = td;
            nxv = tnx;
            nyv = tny;
          }
        }
        const size_t idx = (size_t)ty * n + tx;
        raw[idx] = (char)(int)(sum_cross == nv);
        o.dist[idx] = bd;
        o.nx[idx] = nxv;
        o.ny[idx] = nyv;
      }
    o.label.assign((size_t)n * n, 0);
    for (int ty = 0; ty < n; ++ty)
      for (int tx = 0; tx < n; ++tx) {
        char nl = 0;
        if (ty > 0 && ty < n - 1) {
          const char l0 = raw[(size_t)(ty - 1) * n + tx];
          const char l1 = raw[(size_t)ty * n + tx];
          const char l2 = raw[(size_t)(ty + 1) * n + tx];
          if (l1 == 1) {
            nl = 1;
            if (l0 == 0) nl = 2;
            else if (l2 == 0) nl = 3;
            if (l0 == 0 && l2 == 0) nl = 0;
          }
        }
        o.label[(size_t)ty * n + tx] = nl;
      }
    for (size_t i = 0; i < (size_t)n * n; ++i) {
      const double mult = (double)((int)o.label[i] > 1);
      o.dist[i] *= mult;
      o.nx[i] *= mult;
      o.ny[i] *= mult;
    }
  }
  static void normalize2(double &x, double &y) {
    const double nrm = 1.0 / std::sqrt(x * x + y * y);
    x *= nrm;
    y *= nrm;
  }
  // GeometryGroup::create + geomOp_kernel / geomOpRemove_kernel,
  // include/conga/geometry/GeometryGroup.h:216-334,499-522,590-628
  void group_create(double angle, AngleGeom &o) const {
    static const char op_add[16] = {0, 1, 2, 3, 1, 1, 1, 1, 2, 1, 2, 1, 3, 1, 1, 3};
    const int n = N1();
    const size_t nn = (size_t)n * n;
    o.label.assign(nn, 0);
    o.nx.assign(nn, 0.0);
    o.ny.assign(nn, 0.0);
    o.dist.assign(nn, 0.0);
    for (const GeomComp &g : geom) {
      AngleGeom c;
      if (g.type == 0) disc_create(g, angle, c);
      else polygon_create(g, angle, c);
      if (g.add) {
        for (size_t i = 0; i < nn; ++i) {
          const char d0 = o.label[i], d1 = c.label[i];
          const char nl = op_add[d0 * 4 + d1];
          double ax, ay;
          if (nl == 2 || nl == 3) {
            ax = o.nx[i] + c.nx[i];
            ay = o.ny[i] + c.ny[i];
            normalize2(ax, ay);
          } else {
            ax = 0.0;
            ay = 0.0;
          }
          o.nx[i] = ax;
          o.ny[i] = ay;
          o.label[i] = nl;
          o.dist[i] = std::max(o.dist[i], c.dist[i]);
        }
      } else {
        std::vector<char> tmp(nn, 0);
        for (int ty = 1; ty < n - 1; ++ty)
          for (int tx = 0; tx < n; ++tx) {
            const size_t im = (size_t)(ty - 1) * n + tx, i = (size_t)ty * n + tx,
                         ip = (size_t)(ty + 1) * n + tx;
            char d0 = o.label[i];
            const char d1m = c.label[im], d1 = c.label[i], d1p = c.label[ip];
            if (d1 > 0) {
              d0 = 0;
            } else if (d1p == 2) {
              if (d0 == 1) {
                d0 = 3;
                double ax = o.nx[i] - c.nx[ip], ay = o.ny[i] - c.ny[ip];
                normalize2(ax, ay);
                o.nx[i] = ax;
                o.ny[i] = ay;
                o.dist[i] = 1.0 - c.dist[ip];
              }
            } else if (d1m == 3) {
              if (d0 == 1) {
                d0 = 2;
                double ax = o.nx[i] - c.nx[im], ay = o.ny[i] - c.ny[im];
                normalize2(ax, ay);
                o.nx[i] = ax;
                o.ny[i] = ay;
                o.dist[i] = 1.0 - c.dist[im];
              }
            }
            tmp[i] = d0;
          }
        o.label = tmp;
      }
    }
  }
  // GeometryGroup::createDomain + component createDomain,
  // GeometryGroup.h:524-544; DiscGeometry.h:296-321; PolygonGeometry.h:200-232
  void create_domain_ref() {
    const int n = N0();
    const size_t nn = (size_t)n * n;
    domain_ref.assign(nn, 0);
    for (const GeomComp &g : geom) {
      std::vector<char> loc(nn, 0);
      if (g.type == 0) {
        const double ox = convert_coord(g.cx_, N0(), n);
        const double oy = convert_coord(g.cy_, N0(), n);
        const double r = g.radius * (double)(N0() - 1);
        for (int ty = 0; ty < n; ++ty)
          for (int tx = 0; tx < n; ++tx)
            loc[(size_t)ty * n + tx] = disc_label(tx, ty, r, ox, oy) > 0 ? 1 : 0;
      } else {
        const int nv = (int)g.vx.size();
        for (int ty = 0; ty < n; ++ty)
          for (int tx = 0; tx < n; ++tx) {
            const double cxv = (double)tx / (double)(n - 1) - 0.5;
            const double cyv = (double)ty / (double)(n - 1) - 0.5;
            int sc = 0;
            for (int i = 0; i < nv; ++i) {
              const int ip = (i == nv - 1) ? 0 : i + 1;
              const double lx = g.vx[ip] - g.vx[i], ly = g.vy[ip] - g.vy[i];
              const double cz = lx * (cyv - g.vy[i]) - ly * (cxv - g.vx[i]);
              if (cz >= 0.0) sc++;
            }
            loc[(size_t)ty * n + tx] = (char)(int)(sc == nv);
          }
      }
      for (size_t i = 0; i < nn; ++i) {
        if (g.add) {
          if (loc[i]) domain_ref[i] = 1;
        } else {
          const bool v0 = domain_ref[i] > 0, v1 = loc[i] > 0;
          domain_ref[i] = (!v0 || v1) ? 0 : 1;
        }
      }
    }
    n_grain = 0;
    for (size_t i = 0; i < nn; ++i)
      if (domain_ref[i] > 0) n_grain++;
    area = p.h * p.h * (double)n_grain;
  }

  // ---------------------------------------------------- boundary storage ---
  // BoundaryStorage::computeSparseIndices / computeIntersectingTrajectories and
  // the GeometryGroup counting helpers: BoundaryStorage.h:244-527,
  // GeometryGroup.h:750-894
  void init_boundary_storage() {
    const int n = N1(), na = p.n_angles;
    idx_in_g.assign((size_t)na * n, -1);
    idx_out_g.assign((size_t)na * n, -1);
    idx_in_gt.assign((size_t)na * n, -1);
    idx_out_gt.assign((size_t)na * n, -1);
    nisect_g.assign((size_t)na * n, 0);
    nisect_gt.assign((size_t)na * n, 0);
    coord_g.clear();
    coord_gt.clear();
    n_in_g = n_out_g = n_in_gt = n_out_gt = 0;
    for (int a = 0; a < na; ++a) {
      const std::vector<char> &lab = ag[a].label;
      for (int x = 0; x < n; ++x) {
        int c2 = 0, c3 = 0;
        for (int y = 0; y < n; ++y) {
          const char l = lab[(size_t)y * n + x];
          if (l == 2) c2++;
          if (l == 3) c3++;
        }
        nisect_g[(size_t)a * n + x] = c3;
        nisect_gt[(size_t)a * n + x] = c2;
      }
      for (int x = 0; x < n; ++x) {
        const int c3 = nisect_g[(size_t)a * n + x], c2 = nisect_gt[(size_t)a * n + x];
        idx_in_g[(size_t)a * n + x] = c2 ? n_in_g : -1;
        n_in_g += c2;
        idx_out_g[(size_t)a * n + x] = c3 ? n_out_g : -1;
        n_out_g += c3;
        idx_in_gt[(size_t)a * n + x] = c3 ? n_in_gt : -1;
        n_in_gt += c3;
        idx_out_gt[(size_t)a * n + x] = c2 ? n_out_gt : -1;
        n_out_gt += c2;
      }
    }
    for (int a = 0; a < na; ++a) {
      const std::vector<char> &lab = ag[a].label;
      for (int x = 0; x < n; ++x)
        for (int y = 0; y < n; ++y)
          if (lab[(size_t)y * n + x] == 3) coord_g.push_back(y);
      for (int x = 0; x < n; ++x)
        for (int y = n - 1; y >= 0; --y)
          if (lab[(size_t)y * n + x] == 2) coord_gt.push_back(y);
    }
    xr0.assign(na, 0);
    xr1.assign(na, 0);
    yr0.assign(na, 0);
    yr1.assign(na, 0);
    for (int a = 0; a < na; ++a) {
      int xs = 0;
      for (int i = 0; i < n; ++i)
        if (idx_in_g[(size_t)a * n + i] > -1) {
          xs = i;
          break;
        }
      int xe = xs;
      for (int i = n - 1; i >= xs; --i)
        if (idx_in_g[(size_t)a * n + i] > -1) {
          xe = i;
          break;
        }
      int ys = n - 1, ye = 0;
      const std::vector<char> &lab = ag[a].label;
      for (int i = xs; i <= xe; ++i) {
        for (int j = 0; j < n; ++j)
          if (lab[(size_t)j * n + i] > 0) {
            if (j < ys) ys = j;
            break;
          }
        for (int j = n - 1; j >= 0; --j)
          if (lab[(size_t)j * n + i] > 0) {
            if (j > ye) ye = j;
            break;
          }
      }
      xr0[a] = xs;
      xr1[a] = xe;
      yr0[a] = ys;
      yr1[a] = ye;
    }
    const int ne = p.n_energies;
    bin_g.assign((size_t)n_in_g * ne, mk(0, 0));
    bout_g.assign((size_t)n_out_g * ne, mk(0, 0));
    bin_gt.assign((size_t)n_in_gt * ne, mk(0, 0));
    bout_gt.assign((size_t)n_out_gt * ne, mk(0, 0));
  }

  // ------------------------------------------------------- grid helpers ---
  // extendValuesAtBoundary_kernel, include/conga/geometry/domain_ops.h:11-69
  static void extend(const std::vector<char> &lab, int n, double *v) {
    const int ext = 2;
    std::vector<double> src(v, v + (size_t)n * n);
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        if (lab[(size_t)y * n + x] != 0) continue;
        const int x0 = std::max(x - ext, 0), x1 = std::min(x + ext, n - 1);
        const int y0 = std::max(y - ext, 0), y1 = std::min(y + ext, n - 1);
        double val = 0.0;
        int np = 0, mind = 1000;
        for (int ky = y0; ky <= y1; ++ky)
          for (int kx = x0; kx <= x1; ++kx) {
            if (lab[(size_t)ky * n + kx] > 0) {
              const int dx = x - kx, dy = y - ky, d2 = dx * dx + dy * dy;
              const double s = src[(size_t)ky * n + kx];
              if (d2 < mind) {
                val = s;
                np = 1;
                mind = d2;
              } else if (d2 == mind) {
                val += s;
                np++;
              }
            }
          }
        if (np > 0) v[(size_t)y * n + x] = val / (double)np;
      }
  }
  // insertRotatedGrid(_Additive)_kernel, include/conga/grid/GridFunctions_GPU.h:436-546
  // out (size n x n) receives (or accumulates) the bilinear interpolation of
  // src (size m x m) rotated by phi (single-precision trigonometry).
  static void rotate_insert(double *out, int n, const double *src, int m, double phi,
                            bool additive) {
    const float pf = (float)phi;
    const double c = (double)std::cos(-pf), s = (double)std::sin(-pf);
    const double xt = (double)(m - n) / 2.0;
    const double sh = (double)(m - 1) / 2.0;
#pragma omp parallel for schedule(static)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const double X = x + xt - sh, Y = y + xt - sh;
        const double Xr = X * c - Y * s + sh;
        const double Yr = X * s + Y * c + sh;
        const int xi = (int)Xr, yi = (int)Yr;
        if (xi >= 0 && xi + 1 < m && yi >= 0 && yi + 1 < m) {
          const double xf = Xr - (double)xi, yf = Yr - (double)yi;
          const double x1 = (1.0 - xf) * src[(size_t)yi * m + xi] + xf * src[(size_t)yi * m + xi + 1];
          const double x2 = (1.0 - xf) * src[(size_t)(yi + 1) * m + xi] +
                            xf * src[(size_t)(yi + 1) * m + xi + 1];
          const double v = (1.0 - yf) * x1 + yf * x2;
          if (additive) out[(size_t)y * n + x] += v;
          else out[(size_t)y * n + x] = v;
        }
      }
  }

  // OrderParameter::getRotatedGrid(-a), include/conga/order_parameter/OrderParameter.h:233-258
  void rotated_delta(int a, std::vector<double> &re, std::vector<double> &im) const {
    const int n0 = N0(), n1 = N1();
    const size_t nn0 = (size_t)n0 * n0;
    double px, py;
    fermi_momentum(a, px, py);
    std::vector<double> sre(nn0, 0.0), sim(nn0, 0.0);
    for (int c = 0; c < p.n_comp; ++c) {
      const double b = basis(c, px, py);
      const cx bc = mk(b, 0.0);
      for (size_t i = 0; i < nn0; ++i) {
        const cx v = mul(delta[(size_t)c * nn0 + i], bc);
        sre[i] += v.re;
        sim[i] += v.im;
      }
    }
    extend(domain_ref, n0, sre.data());
    extend(domain_ref, n0, sim.data());
    const double phi = sys_angle(-a);
    re.assign((size_t)n1 * n1, 0.0);
    im.assign((size_t)n1 * n1, 0.0);
    rotate_insert(re.data(), n1, sre.data(), n0, phi, true);
    rotate_insert(im.data(), n1, sim.data(), n0, phi, true);
  }

  // Gauges, include/conga/riccati/energy_shift/Gauges.h:25-62
  void gauge_a(double b, double x, double y, double &ax, double &ay) const {
    if (p.gauge == 0) {
      ax = 0.0;
      ay = x * b;
    } else if (p.gauge == 1) {
      const double f = 0.5 * b;
      ax = -y * f;
      ay = x * f;
    } else {
      const double r2 = std::max(x * x + y * y, 1e-7);
      const double f = b * area / (2.0 * M_PI * r2);
      ax = -y * f;
      ay = x * f;
    }
  }
  // computeEnergyShift, include/conga/riccati/RiccatiSolver.h:127-176 and
  // VectorPotential_Kernel.h:21-99
  void energy_shift(int a, std::vector<double> &es) const {
    const int n0 = N0(), n1 = N1();
    const double b = M_PI * p.flux_quanta / area;
    const double theta = sys_angle(a);
    double vx, vy;
    fermi_velocity(a, vx, vy);
    es.assign((size_t)n1 * n1, 0.0);
    const double q = (double)p.charge_sign;
    const double off = -0.5 * (double)(n1 - 1);
    if (p.penetration_depth > 0.0) {
      std::vector<double> rx((size_t)n1 * n1, 0.0), ry((size_t)n1 * n1, 0.0);
      rotate_insert(rx.data(), n1, avec.data(), n0, -theta, false);
      rotate_insert(ry.data(), n1, avec.data() + (size_t)n0 * n0, n0, -theta, false);
      const double sc = 1.0 / (p.penetration_depth * p.penetration_depth);
      for (size_t i = 0; i < rx.size(); ++i) {
        rx[i] *= sc;
        ry[i] *= sc;
      }
      for (int yi = 0; yi < n1; ++yi)
        for (int xi = 0; xi < n1; ++xi) {
          double x = ((double)xi + off) * p.h, y = ((double)yi + off) * p.h;
          double xr, yr;
          rotate(theta, x, y, xr, yr);
          double ax, ay;
          gauge_a(b, xr, yr, ax, ay);
          const size_t i = (size_t)yi * n1 + xi;
          es[i] = q * (vx * (rx[i] + ax) + vy * (ry[i] + ay));
        }
    } else if (std::fabs(b) > 0.0) {
      for (int yi = 0; yi < n1; ++yi)
        for (int xi = 0; xi < n1; ++xi) {
          double x = ((double)xi + off) * p.h, y = ((double)yi + off) * p.h;
          double xr, yr;
          rotate(theta, x, y, xr, yr);
          double ax, ay;
          gauge_a(b, xr, yr, ax, ay);
          es[(size_t)yi * n1 + xi] = q * (vx * ax + vy * ay);
        }
    }
  }

  // --------------------------------------------------------- the sweeps ---
  // computeCoherenceFunction(BurnIn) + internal::computeStep,
  // include/conga/riccati/RiccatiSolverConfined.h:129-394,513-671
  void sweep(int a, const std::vector<double> &dre, const std::vector<double> &dim,
             const std::vector<double> &es, bool store) {
    const int n = N1(), ne = p.n_energies;
    const double step = step_size(a);
    const AngleGeom &G = ag[a];
    const int x0 = xr0[a], x1 = xr1[a], y0 = yr0[a], y1 = yr1[a];
    for (int dir = 0; dir < 2; ++dir) {
      const bool is_g = dir == 0;
      const char lab_entry = is_g ? 2 : 3, lab_exit = is_g ? 3 : 2;
      const int *sin_ = is_g ? idx_in_g.data() : idx_in_gt.data();
      const int *sout = is_g ? idx_out_g.data() : idx_out_gt.data();
      const cx *bin = is_g ? bin_g.data() : bin_gt.data();
      cx *bout = is_g ? bout_g.data() : bout_gt.data();
      std::vector<cx> &buf = is_g ? gam : gamt;
#pragma omp parallel for schedule(dynamic, 4) collapse(2)
      for (int x = x0; x <= x1; ++x)
        for (int e = 0; e < ne; ++e) {
          const cx e0 = mk(e_re[e], e_im[e]);
          int nin = 0, nout = 0;
          const int ystart = is_g ? y0 : y1;
          const int dy = is_g ? 1 : -1;
          cx eprev = mk(0, 0), dprev = mk(0, 0), coh = mk(0, 0);
          for (int i = 0; i <= y1 - y0; ++i) {
            const int y = ystart + dy * i;
            const size_t idx = (size_t)y * n + x;
            const cx en = add(e0, mk(es[idx], 0.0));
            const cx d = is_g ? mk(dre[idx], dim[idx]) : mk(-dre[idx], dim[idx]);
            const char lab = G.label[idx];
            if (lab == 1) {
              const cx em = scl(add(en, eprev), 0.5);
              const cx dm = scl(add(d, dprev), 0.5);
              coh = riccati_step(dm, em, coh, step);
            } else if (lab == lab_entry) {
              const int sp = (sin_[(size_t)a * n + x] + nin) * ne + e;
              const cx bc = bin[sp];
              const double dist = std::fabs(G.dist[idx]);
              coh = riccati_step(d, en, bc, dist * step);
              nin++;
            } else if (lab == lab_exit) {
              const cx em = scl(add(en, eprev), 0.5);
              const cx dm = scl(add(d, dprev), 0.5);
              coh = riccati_step(dm, em, coh, step);
              const double dist = std::fabs(G.dist[idx]);
              const cx bv = riccati_step(d, en, coh, dist * step);
              const int sp = (sout[(size_t)a * n + x] + nout) * ne + e;
              bout[sp] = bv;
              nout++;
            } else {
              coh = mk(0, 0);
            }
            if (store) buf[(size_t)e * n * n + idx] = coh;
            eprev = en;
            dprev = d;
          }
        }
    }
  }

  // computeGammaFunctionInitialBoundaryTemplate_kernel,
  // RiccatiSolverConfined.h:400-468 (all columns from x_min on).
  void initial_boundary(int a, const std::vector<double> &dre,
                        const std::vector<double> &dim, const std::vector<double> &es) {
    const int n = N1(), ne = p.n_energies;
    const AngleGeom &G = ag[a];
    for (int dir = 0; dir < 2; ++dir) {
      const bool is_g = dir == 0;
      const char lab_exit = is_g ? 3 : 2;
      const int *sout = is_g ? idx_out_g.data() : idx_out_gt.data();
      cx *bout = is_g ? bout_g.data() : bout_gt.data();
      for (int x = xr0[a]; x < n; ++x)
        for (int e = 0; e < ne; ++e) {
          const cx e0 = mk(e_re[e], e_im[e]);
          int nout = 0;
          const int ys = is_g ? 0 : n - 1, dy = is_g ? 1 : -1;
          for (int i = 0; i < n; ++i) {
            const int y = ys + dy * i;
            const size_t idx = (size_t)y * n + x;
            if (G.label[idx] == lab_exit) {
              const cx en = add(e0, mk(es[idx], 0.0));
              const cx d = mk(dre[idx], dim[idx]);
              const int sp = (sout[(size_t)a * n + x] + nout) * ne + e;
              cx g, gt;
              homogeneous(d, en, g, gt);
              bout[sp] = is_g ? g : gt;
              nout++;
            }
          }
        }
    }
  }

  // ----------------------------------------------- boundary condition -----
  // internal::interpolate, include/conga/boundary/BoundaryConditionSpecular.h:112-243
  void bc_interpolate(int xi, int yi, int ei, double sysang, double rpx, double rpy,
                      double coord_off, double bdist, int direction, const int *sout,
                      const int *nisect, const int *coords, const cx *bout, cx &acc,
                      double &wsum) const {
    const int nx = N1(), ne = p.n_energies, na = p.n_angles;
    double mx, my;
    rotate(sysang, rpx, rpy, mx, my);
    // FermiSurface::getFractionalAngleIndex, FermiSurface.h:151-172
    const double kx = wrap_range(mx, tb_ox - M_PI, tb_ox + M_PI);
    const double ky = wrap_range(my, tb_oy - M_PI, tb_oy + M_PI);
    const double phu = std::atan2(ky - tb_oy, kx - tb_ox) - 0.5 * M_PI;
    const double ph = wrap_range(phu, 0.0, 2.0 * M_PI);
    const double fai = (double)na * ph / (2.0 * M_PI);
    const int ia0 = wrap_int((int)fai, 0, na), ia1 = wrap_int((int)fai + 1, 0, na);
    const int iai[2] = {ia0, ia1};
    const double rot_ang[2] = {sysang - system_angle[ia0], sysang - system_angle[ia1]};
    const double frac = fai - std::floor(fai);
    const double aw[2] = {1.0 - frac, frac};
    const double bpx = (double)xi - coord_off;
    const double bpy = (double)yi - (double)sign_((double)direction) * bdist - coord_off;
    acc = mk(0, 0);
    wsum = 0.0;
    for (int r = 0; r < 2; ++r) {
      double rx, ry;
      rotate(rot_ang[r], bpx, bpy, rx, ry);
      rx += coord_off;
      ry += coord_off;
      const int pidx[2] = {(int)rx, (int)rx + 1};
      const double pf = rx - std::floor(rx);
      const double pw[2] = {1.0 - pf, pf};
      for (int pt = 0; pt < 2; ++pt) {
        const int some = iai[r] * nx + pidx[pt];
        const int nis = nisect[some];
        int isect = 0;
        double mind = 1e6;
        for (int i = 0; i < nis; ++i) {
          const int another = i + sout[some];
          const double dyv = std::fabs((double)coords[another] - ry);
          if (dyv < mind) {
            isect = i;
            mind = dyv;
          }
        }
        const int sp = (sout[some] + isect) * ne + ei;
        if (sp >= 0) {
          const double w = pw[pt] * aw[r];
          acc.re += bout[sp].re * w;
          acc.im += bout[sp].im * w;
          wsum += w;
        }
      }
    }
  }
  // BoundaryConditionSpecular::computeBoundaryCondition + kernel,
  // BoundaryConditionSpecular.h:245-358,361-486
  double compute_bc() {
    const std::vector<cx> prev_g = bin_g, prev_gt = bin_gt;
    const int n = N1(), ne = p.n_energies, na = p.n_angles;
    const double coff = (double)(n - 1) * 0.5;
    for (int a = 0; a < na; ++a) {
      const double sa = sys_angle(a);
      double px, py;
      fermi_momentum(a, px, py);
      rotate(-sa, px, py, px, py);
      const AngleGeom &G = ag[a];
      for (int dir = 0; dir < 2; ++dir) {
        const bool is_g = dir == 0;
        const char blab = is_g ? 2 : 3;
        const int direction = is_g ? 1 : -1;
        const int *sin_ = is_g ? idx_in_g.data() : idx_in_gt.data();
        const int *sout = is_g ? idx_out_g.data() : idx_out_gt.data();
        const int *nis = is_g ? nisect_g.data() : nisect_gt.data();
        const int *crd = is_g ? coord_g.data() : coord_gt.data();
        cx *bin = is_g ? bin_g.data() : bin_gt.data();
        const cx *bout = is_g ? bout_g.data() : bout_gt.data();
#pragma omp parallel for schedule(dynamic, 4) collapse(2)
        for (int x = xr0[a]; x <= xr1[a]; ++x)
          for (int e = 0; e < ne; ++e) {
            int nb = 0;
            const int ny = yr1[a] - yr0[a] + 1;
            for (int yy = 0; yy < ny; ++yy) {
              const int y = direction > 0 ? (yr0[a] + yy) : (yr1[a] - yy);
              const size_t idx = (size_t)y * n + x;
              if (G.label[idx] != blab) continue;
              const double bd = std::fabs(G.dist[idx]);
              const double nxv = G.nx[idx], nyv = G.ny[idx];
              const double td = 2.0 * (px * nxv + py * nyv);
              const double rpx = px - td * nxv, rpy = py - td * nyv;
              cx acc;
              double w;
              bc_interpolate(x, y, e, sa, rpx, rpy, coff, bd, direction, sout, nis, crd,
                             bout, acc, w);
              if (w < 1e-7) {
                bc_interpolate(x, y, e, sa, -px, -py, coff, bd, direction, sout, nis, crd,
                               bout, acc, w);
              }
              const int sp = (sin_[(size_t)a * n + x] + nb) * ne + e;
              if (w > 0.0) bin[sp] = mk(acc.re / w, acc.im / w);
              else bin[sp] = mk(0, 0);
              nb++;
            }
          }
      }
    }
    const double rg = residual_cx(prev_g, bin_g);
    const double rgt = residual_cx(prev_gt, bin_gt);
    return std::max(rg, rgt);
  }
  // Residual of a planar complex grid (real plane followed by the imaginary one).
  double residual_cx(const std::vector<cx> &o, const std::vector<cx> &nw) const {
    const size_t n = o.size();
    std::vector<double> a(2 * n), b(2 * n);
    for (size_t i = 0; i < n; ++i) {
      a[i] = o[i].re;
      a[n + i] = o[i].im;
      b[i] = nw[i].re;
      b[n + i] = nw[i].im;
    }
    return residual_grid(a.data(), b.data(), 2 * n, p.norm_type);
  }

  void set_boundary_initial() {
    // IntegrationIteratorOzaki::setBoundaryInitialCondition, IntegrationIteratorOzaki.h:244-300
    std::vector<double> dre, dim, es;
    for (int a = 0; a < p.n_angles; ++a) {
      rotated_delta(a, dre, dim);
      energy_shift(a, es);
      initial_boundary(a, dre, dim, es);
    }
    res_bc = compute_bc();
    boundary_initialized = true;
  }

  // Frame Green sums of one angle (before extension), as computed by
  // GreensFunctionStatic::computeGreensSumEnergy and computeFreeEnergy_Kernel:
  // include/conga/green/GreensFunctionStatic.h:125-157,
  // include/conga/compute/ComputeFreeEnergy.h:106-160.  Sites outside the
  // current angle's trajectory box hold gamma = gammaTilde = 0.
  void frame_greens(int a, const std::vector<double> &dre, const std::vector<double> &dim,
                    std::vector<double> &fre, std::vector<double> &fim,
                    std::vector<double> &gre, std::vector<double> &ire) {
    const int n = N1(), ne = p.n_energies;
    const size_t nn = (size_t)n * n;
    fre.assign(nn, 0.0);
    fim.assign(nn, 0.0);
    gre.assign(nn, 0.0);
    ire.assign(nn, 0.0);
#pragma omp parallel for schedule(static)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const size_t i = (size_t)y * n + x;
        cx sf = mk(0, 0), sg = mk(0, 0), si = mk(0, 0);
        const cx d = mk(dre[i], dim[i]);
        for (int e = 0; e < ne; ++e) {
          const cx g = gam[(size_t)e * nn + i], gt = gamt[(size_t)e * nn + i];
          const cx vf = greens_f(g, gt);
          const cx vg = greens_g(g, gt);
          const cx vi = kernel_i(d, g, gt);
          sf = add(sf, scl(vf, res[e]));
          sg = add(sg, scl(vg, res[e]));
          si = add(si, scl(vi, res[e]));
        }
        fre[i] = 0.0 + sf.re;
        fim[i] = 0.0 + sf.im;
        gre[i] = 0.0 + sg.re;
        ire[i] = 0.0 - si.im;
      }
  }

  // Clear the per-angle coherence buffers (the reference keeps values of other
  // angles outside the current trajectory box; they never reach a result).
  void clear_coherence() {
    std::fill(gam.begin(), gam.end(), mk(0, 0));
    std::fill(gamt.begin(), gamt.end(), mk(0, 0));
  }

  void angle_greens(int a, std::vector<double> &fre, std::vector<double> &fim,
                    std::vector<double> &gre, std::vector<double> &ire,
                    std::vector<double> *dre_out = nullptr) {
    std::vector<double> dre, dim, es;
    rotated_delta(a, dre, dim);
    energy_shift(a, es);
    clear_coherence();
    sweep(a, dre, dim, es, true);
    frame_greens(a, dre, dim, fre, fim, gre, ire);
    if (dre_out) *dre_out = dre;
  }

  // IntegrationIteratorOzaki::compute(false) plus the compute objects'
  // integrateGreensAngle / computePropertyFromGreens:
  // IntegrationIteratorOzaki.h:302-404; ComputeOrderParameter.h:174-262;
  // ComputeCurrent.h:142-222; ComputeFreeEnergy.h:260-414
  void integrate_all() {
    const int n0 = N0(), n1 = N1();
    const size_t nn0 = (size_t)n0 * n0;
    std::vector<cx> acc_d((size_t)p.n_comp * nn0, mk(0, 0));
    std::vector<double> cur_re(2 * nn0, 0.0), cur_im(2 * nn0, 0.0);
    std::vector<double> fe_re(nn0, 0.0);
    std::vector<double> fre, fim, gre, ire;
    std::vector<double> tre(nn0), tim(nn0), tmp1((size_t)n1 * n1);
    for (int a = 0; a < p.n_angles; ++a) {
      angle_greens(a, fre, fim, gre, ire);
      const AngleGeom &G = ag[a];
      const double sa = sys_angle(a);
      double px, py;
      fermi_momentum(a, px, py);
      const double w = integrand(a);
      // Order parameter.
      extend(G.label, n1, fre.data());
      extend(G.label, n1, fim.data());
      for (int c = 0; c < p.n_comp; ++c) {
        std::fill(tre.begin(), tre.end(), 0.0);
        std::fill(tim.begin(), tim.end(), 0.0);
        rotate_insert(tre.data(), n0, fre.data(), n1, sa, false);
        rotate_insert(tim.data(), n0, fim.data(), n1, sa, false);
        const cx bcj = conj_(mk(basis(c, px, py), 0.0));
        for (size_t i = 0; i < nn0; ++i) {
          const cx v = scl(mul(mk(tre[i], tim[i]), bcj), w);
          acc_d[(size_t)c * nn0 + i] = add(acc_d[(size_t)c * nn0 + i], v);
        }
      }
      // Current (real part only reaches the result), weighted by the Fermi
      // velocity (ComputeCurrent.h:155-160).
      extend(G.label, n1, gre.data());
      double vx, vy;
      fermi_velocity(a, vx, vy);
      for (int d = 0; d < 2; ++d) {
        const double f = (d == 0 ? vx : vy) * w;
        for (size_t i = 0; i < tmp1.size(); ++i) tmp1[i] = gre[i] * f;
        rotate_insert(cur_re.data() + d * nn0, n0, tmp1.data(), n1, sa, true);
      }
      // Free energy (real part only reaches the result).
      extend(G.label, n1, ire.data());
      for (size_t i = 0; i < ire.size(); ++i) ire[i] *= w;
      rotate_insert(fe_re.data(), n0, ire.data(), n1, sa, true);
    }
    // ComputeOrderParameter::computePropertyFromGreens
    delta_new.assign((size_t)p.n_comp * nn0, mk(0, 0));
    double r_op = 0.0;
    for (int c = 0; c < p.n_comp; ++c) {
      for (size_t i = 0; i < nn0; ++i) {
        cx v = scl(acc_d[(size_t)c * nn0 + i], coupling[c]);
        if (domain_ref[i] == 0) v = mk(0.0, 0.0);
        delta_new[(size_t)c * nn0 + i] = v;
      }
      std::vector<double> o(2 * nn0), nw(2 * nn0);
      for (size_t i = 0; i < nn0; ++i) {
        o[i] = delta[(size_t)c * nn0 + i].re;
        o[nn0 + i] = delta[(size_t)c * nn0 + i].im;
        nw[i] = delta_new[(size_t)c * nn0 + i].re;
        nw[nn0 + i] = delta_new[(size_t)c * nn0 + i].im;
      }
      r_op = std::max(r_op, residual_grid(o.data(), nw.data(), 2 * nn0, p.norm_type));
    }
    res_op = r_op;
    conv_op = r_op < p.convergence_criterion;
    // ComputeCurrent::computePropertyFromGreens
    {
      const std::vector<double> old = j_real;
      const double factor = (double)(2 * p.charge_sign) * p.temperature;
      for (int d = 0; d < 2; ++d)
        for (size_t i = 0; i < nn0; ++i) {
          double v = cur_re[d * nn0 + i] * factor;
          if (domain_ref[i] == 0) v = 0.0;
          j_real[d * nn0 + i] = v;
        }
      const double actual = residual_grid(old.data(), j_real.data(), 2 * nn0, p.norm_type);
      res_j = first_j ? p.convergence_criterion * 0.1 : actual;
      conv_j = res_j < p.convergence_criterion;
      first_j = false;
    }
    // ComputeFreeEnergy::computePropertyFromGreens
    {
      double sum_inv = 0.0;
      for (int e = 0; e < p.n_energies; ++e) sum_inv += res[e] / e_im[e];
      sum_inv *= p.temperature;
      double ksum = 0.0;
      for (size_t i = 0; i < nn0; ++i)
        if (domain_ref[i] != 0) ksum += fe_re[i];
      double nonmag = p.temperature * ksum;
      for (int c = 0; c < p.n_comp; ++c) {
        const double factor = std::log(p.temperature / tc[c]) + sum_inv;
        double s2 = 0.0;
        for (size_t i = 0; i < nn0; ++i) {
          if (domain_ref[i] == 0) continue;
          const cx v = delta[(size_t)c * nn0 + i];
          s2 += v.re * v.re + v.im * v.im;
        }
        nonmag += s2 * factor;
      }
      double mag = 0.0;
      if (p.penetration_depth > 0.0) {
        const std::vector<double> bz = curl(avec);
        const double mf = 0.5 / (p.penetration_depth * p.penetration_depth);
        double s = 0.0;
        for (double v : bz) s += v * v;
        mag += mf * s;
      }
      const double la = p.h * p.h;
      const double fe_mag_new = mag * la;
      const double fe_new = (nonmag + mag) * la;
      const double fe_mag_area_new = mag / (double)n_grain;
      const double fe_area_new = (nonmag + mag) / (double)n_grain;
      const double actual = residual_scalar(fe_area, fe_area_new);
      res_fe = first_fe ? p.convergence_criterion * 0.1 : actual;
      conv_fe = res_fe < p.convergence_criterion;
      fe = fe_new;
      fe_area = fe_area_new;
      fe_mag = fe_mag_new;
      fe_mag_area = fe_mag_area_new;
      first_fe = false;
    }
  }

  // curl_kernel, include/conga/grid/GridFunctions_GPU.h:326-352
  std::vector<double> curl(const std::vector<double> &A) const {
    const int n = N0();
    const size_t nn = (size_t)n * n;
    const double inv = 1.0 / p.h;
    std::vector<double> out(nn);
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const int xn = std::min(x + 1, n - 1), xp = std::max(x - 1, 0);
        const int yn = std::min(y + 1, n - 1), yp = std::max(y - 1, 0);
        const double dAydx = (A[nn + (size_t)y * n + xn] - A[nn + (size_t)y * n + xp]) / (double)(xn - xp);
        const double dAxdy = (A[(size_t)yn * n + x] - A[(size_t)yp * n + x]) / (double)(yn - yp);
        out[(size_t)y * n + x] = (dAydx - dAxdy) * inv;
      }
    return out;
  }

  // ----------------------------------------------------------- Poisson ----
  // cvp_internal::crossCorrelate1DTranspose, ComputeVectorPotential.h:437-499
  void xcorr_t(const double *src, const double *filt, double *dst) const {
    const int n = N0();
    const int rem = n % 2, nal = n - rem;
#pragma omp parallel for schedule(static)
    for (int d = 0; d < 2; ++d)
      for (int y = 0; y < n; ++y)
        for (int x = 0; x < n; ++x) {
          const int of = n - 1 - y;
          const int os = d * n * n + x;
          double s0 = 0.0, s1 = 0.0;
          for (int i = 0; i < nal; i += 2) {
            s0 += filt[i + of] * src[(size_t)i * n + os];
            s1 += filt[i + of + 1] * src[(size_t)(i + 1) * n + os];
          }
          double t = 0.0;
          for (int i = nal; i < n; ++i) t += src[(size_t)i * n + os] * filt[i + of];
          dst[(size_t)n * (d * n + x) + y] = t + s0 + s1;
        }
  }
  // ComputeVectorPotential::solve / solveInternal / subtractMean,
  // ComputeVectorPotential.h:575-745
  void poisson(const std::vector<double> &j) {
    const int n = N0();
    const size_t nn = (size_t)n * n;
    std::vector<double> s(2 * nn);
    for (int d = 0; d < 2; ++d) {
      double sum = 0.0;
      for (size_t i = 0; i < nn; ++i) sum += j[d * nn + i];
      const double mean = sum / (double)n_grain;
      for (size_t i = 0; i < nn; ++i) s[d * nn + i] = j[d * nn + i] - mean;
    }
    a_new.assign(2 * nn, 0.0);
    std::vector<double> t0(2 * nn), t1(2 * nn);
    for (size_t k = 0; k < filters.size(); ++k) {
      xcorr_t(s.data(), filters[k].data(), t0.data());
      xcorr_t(t0.data(), filters[k].data(), t1.data());
      if (filter_pos[k])
        for (size_t i = 0; i < 2 * nn; ++i) a_new[i] += t1[i];
      else
        for (size_t i = 0; i < 2 * nn; ++i) a_new[i] -= t1[i];
    }
    const double f = -1.0 * (p.h * p.h) * p.vp_scale;
    for (double &v : a_new) v *= f;
  }

  // ------------------------------------------------------- accelerators ---
  // concatenate / split, include/conga/accelerators/utils.h:42-186
  void concat(const std::vector<cx> &d, const std::vector<double> *a, std::vector<double> &X) const {
    const size_t nn = (size_t)N0() * N0();
    const int nf = 2 * p.n_comp + (a ? 2 : 0);
    X.assign((size_t)nf * nn, 0.0);
    for (int c = 0; c < p.n_comp; ++c)
      for (size_t i = 0; i < nn; ++i) {
        X[(size_t)(2 * c) * nn + i] = d[(size_t)c * nn + i].re;
        X[(size_t)(2 * c + 1) * nn + i] = d[(size_t)c * nn + i].im;
      }
    if (a)
      for (size_t i = 0; i < 2 * nn; ++i) X[(size_t)(2 * p.n_comp) * nn + i] = (*a)[i];
  }
  void split(const std::vector<double> &X, bool with_a) {
    const size_t nn = (size_t)N0() * N0();
    for (int c = 0; c < p.n_comp; ++c)
      for (size_t i = 0; i < nn; ++i)
        delta[(size_t)c * nn + i] = mk(X[(size_t)(2 * c) * nn + i], X[(size_t)(2 * c + 1) * nn + i]);
    if (with_a)
      for (size_t i = 0; i < 2 * nn; ++i) avec[i] = X[(size_t)(2 * p.n_comp) * nn + i];
  }
  // CongAcc::computeInertia, include/conga/accelerators/CongAcc.h:300-356
  static double congacc_inertia(double dn, double mn, double dot, double mincos) {
    double ea = dot / (dn * mn) - mincos, xa = 1.0;
    double eb = 1.0 - mincos, xb = 0.0;
    (void)eb;
    double x = 0.5 * (xa + xb);
    bool conv = false;
    while (!conv) {
      const double y = 1.0 - x;
      const double numer = x * dot + y * dn * dn;
      const double denom = dn * std::sqrt(x * x * mn * mn + 2.0 * x * y * dot + y * y * dn * dn);
      const double sim = numer / denom;
      const double err = sim - mincos;
      conv = std::fabs(err) < 0.01;
      if (sign_(err) == sign_(ea)) {
        ea = err;
        xa = x;
      } else {
        eb = err;
        xb = x;
      }
      if (sign_(ea) == sign_(eb)) break;
      x = 0.5 * (xa + xb);
    }
    return x;
  }
  void accelerate(std::vector<double> &X, const std::vector<double> &G, int nf) {
    const size_t nn = (size_t)N0() * N0();
    const size_t tot = (size_t)nf * nn;
    std::vector<double> diff(tot);
    for (size_t i = 0; i < tot; ++i) diff[i] = G[i] - X[i];
    if (p.accelerator == 0) {
      // CongAcc::computeInternal, CongAcc.h:361-419
      if (!acc_init) {
        acc_mean.assign(tot, 0.0);
        acc_step.assign(nf, p.acc_step_size);
        acc_inertia.assign(nf, 0.0);
        acc_init = true;
      }
      for (int f = 0; f < nf; ++f) {
        double d2 = 0, m2 = 0, dm = 0;
        for (size_t i = 0; i < nn; ++i) {
          const double dv = diff[(size_t)f * nn + i], mv = acc_mean[(size_t)f * nn + i];
          d2 += dv * dv;
          m2 += mv * mv;
          dm += dv * mv;
        }
        const double d = std::sqrt(d2), m = std::sqrt(m2), den = d * m;
        if (den > 0.0) {
          const double cs = dm / den;
          acc_step[f] *= std::pow(p.acc_step_size_factor, cs);
          if (cs < p.acc_cos_similarity_min)
            acc_inertia[f] = congacc_inertia(d, m, dm, p.acc_cos_similarity_min);
        }
        acc_step[f] = std::clamp(acc_step[f], p.acc_step_size_min, p.acc_step_size_max);
      }
      for (int f = 0; f < nf; ++f)
        for (size_t i = 0; i < nn; ++i) {
          const size_t k = (size_t)f * nn + i;
          const double mean = acc_mean[k] * acc_inertia[f] + diff[k] * (1.0 - acc_inertia[f]);
          acc_mean[k] = mean;
          X[k] += acc_step[f] * mean;
        }
    } else if (p.accelerator == 1) {
      // Picard::computeInternal, Picard.h:133-138
      for (size_t i = 0; i < tot; ++i) X[i] += diff[i] * p.acc_step_size;
    } else if (p.accelerator == 2) {
      // Polyak::computeInternal, Polyak.h:214-266
      if (!acc_init) {
        acc_vel.assign(tot, 0.0);
        acc_init = true;
      }
      for (size_t i = 0; i < tot; ++i) {
        const double v = acc_vel[i] * (1.0 - p.acc_drag) + diff[i] * p.acc_step_size;
        acc_vel[i] = v;
        X[i] += v;
      }
    } else if (p.accelerator == 3) {
      // BarzilaiBorwein::computeInternal, BarzilaiBorwein.h:208-241
      if (!acc_init) {
        bb_step = p.acc_step_size;
        acc_iter = 0;
        acc_init = true;
      }
      if (acc_iter > 0) {
        double dot = 0.0, ss = 0.0, sp = 0.0;
        for (int f = 0; f < nf; ++f) {
          double fs = 0.0;
          for (size_t i = 0; i < nn; ++i) {
            const size_t k = (size_t)f * nn + i;
            fs += acc_dprev[k] * (diff[k] - acc_dprev[k]);
          }
          dot += fs;
        }
        dot = std::fabs(dot);
        for (size_t k = 0; k < tot; ++k) {
          const double dd = diff[k] - acc_dprev[k];
          ss += dd * dd;
          sp += acc_dprev[k] * acc_dprev[k];
        }
        const double scale = (acc_iter % 2 == 0) ? dot / ss : sp / dot;
        bb_step *= scale;
      }
      bb_step = std::clamp(bb_step, p.acc_step_size_min, p.acc_step_size_max);
      acc_dprev = diff;
      for (size_t i = 0; i < tot; ++i) X[i] += diff[i] * bb_step;
      acc_iter++;
    } else {
      // Anderson::set / solve / computeInternal, Anderson.h:270-355
      if (!acc_init) {
        acc_iter = 0;
        acc_init = true;
      }
      double sq = 0.0;
      for (size_t k = 0; k < tot; ++k) sq += diff[k] * diff[k];
      if ((int)and_d.size() == p.acc_rank) {
        size_t best = 0;
        for (size_t i = 1; i < and_idx.size(); ++i)
          if (and_idx[i] < and_idx[best]) best = i;
        and_x[best] = X;
        and_d[best] = diff;
        and_sq[best] = sq;
        and_idx[best] = (size_t)acc_iter;
      } else {
        and_x.push_back(X);
        and_d.push_back(diff);
        and_sq.push_back(sq);
        and_idx.push_back((size_t)acc_iter);
      }
      const int m = (int)and_d.size(), mt = m + 1;
      std::vector<double> A((size_t)mt * mt, 1.0), b(mt, 0.0);
      double sr = 0.0;
      for (double v : and_sq) sr += v;
      const double scale = 1.0 / (sr / (double)m);
      for (int i = 0; i < m; ++i) {
        A[(size_t)i * mt + i] = and_sq[i] * scale;
        for (int jj = i + 1; jj < m; ++jj) {
          double v = 0.0;
          for (int f = 0; f < nf; ++f) {
            double fs = 0.0;
            for (size_t q = 0; q < nn; ++q)
              fs += and_d[i][(size_t)f * nn + q] * and_d[jj][(size_t)f * nn + q];
            v += fs;
          }
          v *= scale;
          A[(size_t)i * mt + jj] = v;
          A[(size_t)jj * mt + i] = v;
        }
      }
      A[(size_t)(mt - 1) * mt + (mt - 1)] = 0.0;
      b[mt - 1] = 1.0;
      // Gaussian elimination with partial pivoting.
      std::vector<double> M = A, rhs = b;
      for (int col = 0; col < mt; ++col) {
        int piv = col;
        for (int r = col + 1; r < mt; ++r)
          if (std::fabs(M[(size_t)r * mt + col]) > std::fabs(M[(size_t)piv * mt + col])) piv = r;
        if (piv != col) {
          for (int cc = 0; cc < mt; ++cc) std::swap(M[(size_t)col * mt + cc], M[(size_t)piv * mt + cc]);
          std::swap(rhs[col], rhs[piv]);
        }
        const double dg = M[(size_t)col * mt + col];
        for (int r = col + 1; r < mt; ++r) {
          const double f = M[(size_t)r * mt + col] / dg;
          for (int cc = col; cc < mt; ++cc) M[(size_t)r * mt + cc] -= f * M[(size_t)col * mt + cc];
          rhs[r] -= f * rhs[col];
        }
      }
      std::vector<double> wts(mt, 0.0);
      for (int r = mt - 1; r >= 0; --r) {
        double s = rhs[r];
        for (int cc = r + 1; cc < mt; ++cc) s -= M[(size_t)r * mt + cc] * wts[cc];
        wts[r] = s / M[(size_t)r * mt + r];
      }
      std::fill(X.begin(), X.end(), 0.0);
      for (int i = 0; i < m; ++i)
        for (size_t k = 0; k < tot; ++k)
          X[k] += (and_x[i][k] + and_d[i][k] * p.acc_step_size) * wts[i];
      acc_iter++;
    }
  }

  // ------------------------------------------------------------ context ---
  // Context::compute, include/conga/Context.h:391-447
  void compute() {
    const bool do_vp = has_vp && p.penetration_depth > 0.0;
    if (!first_compute) {
      std::vector<double> X, G;
      if (do_vp) {
        concat(delta, &avec, X);
        concat(delta_new, &a_new, G);
        accelerate(X, G, 2 * p.n_comp + 2);
        split(X, true);
      } else {
        concat(delta, nullptr, X);
        concat(delta_new, nullptr, G);
        accelerate(X, G, 2 * p.n_comp);
        split(X, false);
      }
    }
    if (!boundary_initialized) set_boundary_initial();
    integrate_all();
    res_bc = compute_bc();
    if (do_vp) {
      poisson(j_real);
      const size_t nn = (size_t)N0() * N0();
      res_vp = residual_grid(avec.data(), a_new.data(), 2 * nn, p.norm_type);
    }
    n_iterations++;
    first_compute = false;
  }
  // Context::burnIn + IntegrationIteratorOzaki::compute(true)
  void burn_in() {
    if (!boundary_initialized) set_boundary_initial();
    std::vector<double> dre, dim, es;
    for (int a = 0; a < p.n_angles; ++a) {
      rotated_delta(a, dre, dim);
      energy_shift(a, es);
      sweep(a, dre, dim, es, false);
    }
    res_bc = compute_bc();
    n_iterations++;
  }
  // IntegrationIteratorKeldysh::compute(false) with ComputeLDOS as the only
  // compute object (IntegrationIteratorKeldysh.h:300-389, ComputeLDOS.h:123-193):
  // per angle Im g of every energy, extended, weighted and rotated back; then
  // the boundary condition; LDOS = -sum, zero outside the grain, residual
  // against the previous iteration of this energy block.
  std::vector<double> ldos_prev;
  double res_ldos = 0.0;
  void ldos_iteration(int n_fields) {
    if (!boundary_initialized) set_boundary_initial();
    const int n0 = N0(), n1 = N1(), ne = p.n_energies;
    const size_t nn0 = (size_t)n0 * n0, nn1 = (size_t)n1 * n1;
    std::vector<double> acc((size_t)ne * nn0, 0.0), gim(nn1);
    std::vector<double> dre, dim, es;
    for (int a = 0; a < p.n_angles; ++a) {
      rotated_delta(a, dre, dim);
      energy_shift(a, es);
      clear_coherence();
      sweep(a, dre, dim, es, true);
      const double w = integrand(a), sa = sys_angle(a);
      for (int e = 0; e < ne; ++e) {
        for (size_t i = 0; i < nn1; ++i)
          gim[i] = greens_g(gam[(size_t)e * nn1 + i], gamt[(size_t)e * nn1 + i]).im;
        extend(ag[a].label, n1, gim.data());
        for (size_t i = 0; i < nn1; ++i) gim[i] *= w;
        rotate_insert(acc.data() + (size_t)e * nn0, n0, gim.data(), n1, sa, true);
      }
    }
    res_bc = compute_bc();
    const size_t n = (size_t)n_fields * nn0;
    std::vector<double> nw(n);
    for (size_t i = 0; i < n; ++i) nw[i] = domain_ref[i % nn0] ? -acc[i] : 0.0;
    if (ldos_prev.size() != n) ldos_prev.assign(n, 0.0);
    res_ldos = residual_grid(ldos_prev.data(), nw.data(), n, p.norm_type);
    ldos_prev = nw;
    n_iterations++;
  }

  // Context::getResidual, Context.h:462-483
  double total_residual() const {
    double r = 0.0;
    if (has_vp) r = res_vp;
    r = std::max(res_bc, r);
    r = std::max(r, res_op);
    r = std::max(r, res_j);
    r = std::max(r, res_fe);
    return r;
  }
};

// ------------------------------------------------ tight-binding surface ----
// DispersionTightBinding<T>::evaluate / derivative,
// include/conga/fermi_surface/DispersionTightBinding.h:62-125.
double tb_dispersion(double t1, double t2, double mu, double kx, double ky) {
  const double term_nn = (-2.0 * 1.0) * (std::cos(kx) + std::cos(ky));
  const double term_nnn = (-4.0 * t1) * std::cos(kx) * std::cos(ky);
  const double term_nnnn = (-2.0 * t2) * (std::cos(2.0 * kx) + std::cos(2.0 * ky));
  return term_nn + term_nnn + term_nnnn - mu;
}
void tb_velocity(double t1, double t2, double kx, double ky, double &vx, double &vy) {
  vx = (2.0 * 1.0) * std::sin(kx) + (4.0 * t1) * std::sin(kx) * std::cos(ky) + (4.0 * t2) * std::sin(2.0 * kx);
  vy = (2.0 * 1.0) * std::sin(ky) + (4.0 * t1) * std::cos(kx) * std::sin(ky) + (4.0 * t2) * std::sin(2.0 * ky);
}

// FermiSurfaceTightBinding<T>::initialize, FermiSurfaceTightBinding.h:384-470,
// with tightbinding_internal::computeMomentumOffset (:129-151),
// computeFermiMomentum (:167-290) and computeIntegrandFactor (:305-326).
// table [8][n]: polar angle, system angle, momentum x, y, velocity x, y
// (divided by the mean speed), integrand factor (normalised to sum 1), speed;
// info: mean |p|, mean |v|, origin x, y.
void tight_binding_tables(double t1, double t2, double mu, int n, double *table, double *info) {
  // Origin: (0,0) if the band has the same sign at (0,pi) and (pi,pi).
  const double e0pi = tb_dispersion(t1, t2, mu, 0.0, M_PI);
  const double epipi = tb_dispersion(t1, t2, mu, M_PI, M_PI);
  const double org = (sign_(e0pi) == sign_(epipi)) ? 0.0 : M_PI;
  const double crit = 1e2 * std::numeric_limits<double>::epsilon();
  double *phi = table, *sys = table + n, *px = table + 2 * n, *py = table + 3 * n;
  double *vx = table + 4 * n, *vy = table + 5 * n, *w = table + 6 * n, *sp = table + 7 * n;
  double fsum = 0.0, msum = 0.0, ssum = 0.0;
  for (int k = 0; k < n; ++k) {
    const double ph = wrap_range(M_PI * (double)(2 * k) / (double)n + 0.5 * M_PI, 0.0, 2.0 * M_PI);
    const double c = std::cos(ph), s = std::sin(ph);
    // Root of the band along the ray org + kappa (c, s).
    double lo = 0.0, e_lo = tb_dispersion(t1, t2, mu, lo * c + org, lo * s + org);
    double hi = M_PI / std::max(std::fabs(c), std::fabs(s));
    double e_hi = tb_dispersion(t1, t2, mu, hi * c + org, hi * s + org);
    double kappa = 0.5 * (lo + hi);
    bool newton = false;
    for (int it = 0; it < 100; ++it) {
      const double mx = kappa * c + org, my = kappa * s + org;
      const double e = tb_dispersion(t1, t2, mu, mx, my);
      if (!newton && std::fabs(e) > std::sqrt(crit)) {
        if (sign_(e) == sign_(e_lo)) {
          e_lo = e;
          lo = kappa;
        } else {
          e_hi = e;
          hi = kappa;
        }
        if (sign_(e_lo) == sign_(e_hi)) break;
        kappa = 0.5 * (lo + hi);
        continue;
      }
      if (!(std::fabs(e) > crit)) break;
      newton = true;
      double gx, gy;
      tb_velocity(t1, t2, mx, my, gx, gy);
      const double d = gx * c + gy * s;
      if (!(std::fabs(d) > 0.0)) break;
      kappa -= e / d;
    }
    const double pkx = wrap_range(kappa * c + org, -M_PI, M_PI);
    const double pky = wrap_range(kappa * s + org, -M_PI, M_PI);
    double gx, gy;
    tb_velocity(t1, t2, pkx, pky, gx, gy);
    // Buchholtz et al.'s Jacobian |k.k / k.v| with k the momentum from the origin.
    const double kx = wrap_range(pkx, org - M_PI, org + M_PI) - org;
    const double ky = wrap_range(pky, org - M_PI, org + M_PI) - org;
    const double f = std::fabs((kx * kx + ky * ky) / (kx * gx + ky * gy)) * [&] {
      if (n % 4 == 0) return (k % 4 == 0) ? 28.0 / 45.0 : (k % 2 == 0) ? 24.0 / 45.0 : 64.0 / 45.0;
      if (n % 3 == 0) return (k % 3 == 0) ? 6.0 / 8.0 : 9.0 / 8.0;
      if (n % 2 == 0) return (k % 2 == 0) ? 2.0 / 3.0 : 4.0 / 3.0;
      return 1.0;
    }();
    phi[k] = ph;
    sys[k] = std::atan2(gy, gx) - 0.5 * M_PI;
    px[k] = pkx;
    py[k] = pky;
    vx[k] = gx;
    vy[k] = gy;
    w[k] = f;
    fsum += f;
    msum += std::hypot(pkx, pky) * f;
    ssum += std::hypot(gx, gy) * f;
  }
  const double avg_p = msum / fsum, avg_v = ssum / fsum;
  for (int k = 0; k < n; ++k) {
    vx[k] /= avg_v;
    vy[k] /= avg_v;
    w[k] /= fsum;
    sp[k] = std::hypot(vx[k], vy[k]);
  }
  info[0] = avg_p;
  info[1] = avg_v;
  info[2] = org;
  info[3] = org;
}

}  // namespace

extern "C" {

/* The tight-binding Fermi-surface tables alone (see tight_binding_tables). */
void orc_tight_binding(double t1, double t2, double mu, int n, double *table, double *info) {
  tight_binding_tables(t1, t2, mu, n, table, info);
}

void *orc_create(const orc_params *p, const double *energies_im, const double *residues,
                 const int *comp_symmetry, const double *comp_tc, int n_geom,
                 const int *geom_type, const int *geom_add, const int *geom_nvert,
                 const double *geom_data, const double *filters, const int *filter_pos) {
  Oracle *o = new Oracle();
  o->p = *p;
  o->e_im.assign(energies_im, energies_im + p->n_energies);
  o->e_re.assign(p->n_energies, 0.0);
  o->res.assign(residues, residues + p->n_energies);
  o->sym.assign(comp_symmetry, comp_symmetry + p->n_comp);
  o->tc.assign(comp_tc, comp_tc + p->n_comp);
  size_t off = 0;
  for (int g = 0; g < n_geom; ++g) {
    GeomComp c;
    c.type = geom_type[g];
    c.add = geom_add[g];
    if (c.type == 0) {
      c.radius = geom_data[off];
      c.cx_ = geom_data[off + 1];
      c.cy_ = geom_data[off + 2];
      off += 3;
    } else {
      const int nv = geom_nvert[g];
      c.vx.assign(geom_data + off, geom_data + off + nv);
      c.vy.assign(geom_data + off + nv, geom_data + off + 2 * nv);
      off += 2 * (size_t)nv;
    }
    o->geom.push_back(c);
  }
  // Fermi surface, FermiSurfaceCircle::initialize (FermiSurfaceCircle.h:84-104)
  // or FermiSurfaceTightBinding::initialize (FermiSurfaceTightBinding.h:384-470).
  if (p->fs_type == 1) {
    const int na = p->n_angles;
    std::vector<double> t((size_t)8 * na);
    double info[4];
    tight_binding_tables(p->tb_nnn, p->tb_nnnn, p->tb_mu, na, t.data(), info);
    o->polar.assign(t.begin(), t.begin() + na);
    o->system_angle.assign(t.begin() + na, t.begin() + 2 * na);
    o->tb_px.assign(t.begin() + 2 * na, t.begin() + 3 * na);
    o->tb_py.assign(t.begin() + 3 * na, t.begin() + 4 * na);
    o->tb_vx.assign(t.begin() + 4 * na, t.begin() + 5 * na);
    o->tb_vy.assign(t.begin() + 5 * na, t.begin() + 6 * na);
    o->tb_w.assign(t.begin() + 6 * na, t.begin() + 7 * na);
    o->tb_speed.assign(t.begin() + 7 * na, t.end());
    o->tb_ox = info[2];
    o->tb_oy = info[3];
  } else {
    for (int k = 0; k < p->n_angles; ++k) {
      const double phi = o->polar_angle(k);
      o->polar.push_back(phi);
      o->system_angle.push_back(phi - 0.5 * M_PI);
    }
  }
  // BasisFunction::normalize, OrderParameterBasis.h:188-212.
  for (int c = 0; c < p->n_comp; ++c) {
    double avg = 0.0;
    for (int k = 0; k < p->n_angles; ++k) {
      double px, py;
      o->fermi_momentum(k, px, py);
      const double b = o->basis_raw(comp_symmetry[c], px, py);
      avg += (b * b + 0.0 * 0.0) * o->integrand(k);
    }
    o->norm_factor.push_back(1.0 / std::sqrt(avg));
  }
  // OrderParameterComponent::initCouplingConstant, OrderParameterComponent.h:156-181.
  for (int c = 0; c < p->n_comp; ++c) {
    double es = 0.0;
    for (int e = 0; e < p->n_energies; ++e) es += residues[e] / energies_im[e];
    es *= p->temperature;
    o->coupling.push_back(0.5 * p->temperature / (std::log(p->temperature / comp_tc[c]) + es));
  }
  o->create_domain_ref();
  o->ag.resize(p->n_angles);
  for (int a = 0; a < p->n_angles; ++a) o->group_create(-o->system_angle[a], o->ag[a]);
  o->init_boundary_storage();
  const size_t nn0 = (size_t)p->n0 * p->n0, nn1 = (size_t)p->n1 * p->n1;
  o->delta.assign((size_t)p->n_comp * nn0, mk(0, 0));
  o->delta_new = o->delta;
  o->avec.assign(2 * nn0, 0.0);
  o->a_new.assign(2 * nn0, 0.0);
  o->j_real.assign(2 * nn0, 0.0);
  o->gam.assign((size_t)p->n_energies * nn1, mk(0, 0));
  o->gamt.assign((size_t)p->n_energies * nn1, mk(0, 0));
  o->has_vp = p->penetration_depth > 0.0;
  for (int k = 0; k < p->n_filters; ++k) {
    o->filters.emplace_back(filters + (size_t)k * (2 * p->n0 - 1),
                            filters + (size_t)(k + 1) * (2 * p->n0 - 1));
    o->filter_pos.push_back(filter_pos[k]);
  }
  return o;
}

void orc_destroy(void *h) { delete (Oracle *)h; }

// Sets x: order-parameter components ([c][re/im][N0*N0]) and the induced vector
// potential in internal units (already multiplied by lambda^2), [2][N0*N0].  The
// order parameter is zeroed outside the grain as OrderParameter::initialize does
// (OrderParameter.h:180-199).
void orc_set_state(void *h, const double *delta, const double *a_internal) {
  Oracle *o = (Oracle *)h;
  const size_t nn = (size_t)o->p.n0 * o->p.n0;
  for (int c = 0; c < o->p.n_comp; ++c)
    for (size_t i = 0; i < nn; ++i) {
      const double re = delta[(size_t)(2 * c) * nn + i], im = delta[(size_t)(2 * c + 1) * nn + i];
      o->delta[(size_t)c * nn + i] = o->domain_ref[i] ? mk(re, im) : mk(0.0, 0.0);
    }
  if (a_internal) std::memcpy(o->avec.data(), a_internal, 2 * nn * sizeof(double));
}

void orc_compute(void *h) { ((Oracle *)h)->compute(); }
void orc_burn_in(void *h) { ((Oracle *)h)->burn_in(); }

void orc_get_state(void *h, double *delta, double *a_internal) {
  Oracle *o = (Oracle *)h;
  const size_t nn = (size_t)o->p.n0 * o->p.n0;
  for (int c = 0; c < o->p.n_comp; ++c)
    for (size_t i = 0; i < nn; ++i) {
      delta[(size_t)(2 * c) * nn + i] = o->delta[(size_t)c * nn + i].re;
      delta[(size_t)(2 * c + 1) * nn + i] = o->delta[(size_t)c * nn + i].im;
    }
  std::memcpy(a_internal, o->avec.data(), 2 * nn * sizeof(double));
}

// g(x) of the last iteration: new order parameter, current density, new vector
// potential (internal units).
void orc_get_results(void *h, double *delta_new, double *j, double *a_new) {
  Oracle *o = (Oracle *)h;
  const size_t nn = (size_t)o->p.n0 * o->p.n0;
  for (int c = 0; c < o->p.n_comp; ++c)
    for (size_t i = 0; i < nn; ++i) {
      delta_new[(size_t)(2 * c) * nn + i] = o->delta_new[(size_t)c * nn + i].re;
      delta_new[(size_t)(2 * c + 1) * nn + i] = o->delta_new[(size_t)c * nn + i].im;
    }
  std::memcpy(j, o->j_real.data(), 2 * nn * sizeof(double));
  std::memcpy(a_new, o->a_new.data(), 2 * nn * sizeof(double));
}

// out[0..10]: free energy, per area, magnetic, magnetic per area, residuals
// (order parameter, current, free energy, vector potential, boundary), total
// residual, number of grain lattice sites.
void orc_get_scalars(void *h, double *out) {
  Oracle *o = (Oracle *)h;
  out[0] = o->fe;
  out[1] = o->fe_area;
  out[2] = o->fe_mag;
  out[3] = o->fe_mag_area;
  out[4] = o->res_op;
  out[5] = o->res_j;
  out[6] = o->res_fe;
  out[7] = o->res_vp;
  out[8] = o->res_bc;
  out[9] = o->total_residual();
  out[10] = (double)o->n_grain;
}

int orc_is_converged(void *h) {
  Oracle *o = (Oracle *)h;
  const bool ok = o->total_residual() < o->p.convergence_criterion;
  return (ok && o->conv_op && o->conv_j && o->conv_fe) ? 1 : 0;
}

// Geometry of one angle in its trajectory frame (labels, |distance|, normals),
// plus the reference-frame domain.
void orc_get_geometry(void *h, int a, char *labels, double *dist, double *nx, double *ny) {
  Oracle *o = (Oracle *)h;
  const size_t nn = (size_t)o->p.n1 * o->p.n1;
  std::memcpy(labels, o->ag[a].label.data(), nn);
  std::memcpy(dist, o->ag[a].dist.data(), nn * sizeof(double));
  std::memcpy(nx, o->ag[a].nx.data(), nn * sizeof(double));
  std::memcpy(ny, o->ag[a].ny.data(), nn * sizeof(double));
}
void orc_get_domain(void *h, char *dom) {
  Oracle *o = (Oracle *)h;
  std::memcpy(dom, o->domain_ref.data(), o->domain_ref.size());
}
// Sizes of the sparse boundary storage: in/out for gamma and gammaTilde.
void orc_boundary_sizes(void *h, int *out) {
  Oracle *o = (Oracle *)h;
  out[0] = o->n_in_g;
  out[1] = o->n_out_g;
  out[2] = o->n_in_gt;
  out[3] = o->n_out_gt;
}
// which: 0 in-gamma, 1 out-gamma, 2 in-gammaTilde, 3 out-gammaTilde; written as
// interleaved (re, im) pairs of length count*n_energies.
void orc_get_boundary(void *h, int which, double *out) {
  Oracle *o = (Oracle *)h;
  const std::vector<cx> *v = which == 0 ? &o->bin_g : which == 1 ? &o->bout_g
                           : which == 2 ? &o->bin_gt : &o->bout_gt;
  for (size_t i = 0; i < v->size(); ++i) {
    out[2 * i] = (*v)[i].re;
    out[2 * i + 1] = (*v)[i].im;
  }
}
void orc_set_boundary(void *h, int which, const double *in) {
  Oracle *o = (Oracle *)h;
  std::vector<cx> *v = which == 0 ? &o->bin_g : which == 1 ? &o->bout_g
                     : which == 2 ? &o->bin_gt : &o->bout_gt;
  for (size_t i = 0; i < v->size(); ++i) (*v)[i] = mk(in[2 * i], in[2 * i + 1]);
  o->boundary_initialized = true;
}
// Per-angle tables: x range, y range.
void orc_get_ranges(void *h, int *x0, int *x1, int *y0, int *y1) {
  Oracle *o = (Oracle *)h;
  for (int a = 0; a < o->p.n_angles; ++a) {
    x0[a] = o->xr0[a];
    x1[a] = o->xr1[a];
    y0[a] = o->yr0[a];
    y1[a] = o->yr1[a];
  }
}
// Frame Green sums of angle a for the current state and boundary values (the
// boundary out-values are updated as a side effect, as the sweep does):
// F (re, im), Re G, Re I, and the rotated order parameter (re, im).
void orc_angle_greens(void *h, int a, double *fre, double *fim, double *gre, double *ire,
                      double *dre, double *dim) {
  Oracle *o = (Oracle *)h;
  std::vector<double> vfre, vfim, vgre, vire, vdre, vdim, es;
  o->rotated_delta(a, vdre, vdim);
  o->energy_shift(a, es);
  o->clear_coherence();
  o->sweep(a, vdre, vdim, es, true);
  o->frame_greens(a, vdre, vdim, vfre, vfim, vgre, vire);
  const size_t nn = vfre.size();
  std::memcpy(fre, vfre.data(), nn * 8);
  std::memcpy(fim, vfim.data(), nn * 8);
  std::memcpy(gre, vgre.data(), nn * 8);
  std::memcpy(ire, vire.data(), nn * 8);
  std::memcpy(dre, vdre.data(), nn * 8);
  std::memcpy(dim, vdim.data(), nn * 8);
}
// One frozen-boundary evaluation (the sweeps and compute objects of one
// Context::compute without the accelerator step and the boundary update):
// g(x), j and the free energy of the current state.
void orc_evaluate(void *h) {
  Oracle *o = (Oracle *)h;
  if (!o->boundary_initialized) o->set_boundary_initial();
  o->integrate_all();
}

// extendValuesAtBoundary on a grid of side n (domain_ops.h:11-69), in place.
void orc_extend_grid(int n, const signed char *labels, double *values) {
  std::vector<char> lab(labels, labels + (size_t)n * n);
  Oracle::extend(lab, n, values);
}

// External flux quanta (the field enters the energy shift through the gauge).
void orc_set_flux(void *h, double flux_quanta) { ((Oracle *)h)->p.flux_quanta = flux_quanta; }

// Real parts of the sweep energies (LDOS energies E_k; the imaginary parts,
// the broadening, are those given to orc_create).  Starts a new energy block:
// fresh boundary values and LDOS history.
void orc_set_energies_re(void *h, const double *e_re) {
  Oracle *o = (Oracle *)h;
  o->e_re.assign(e_re, e_re + o->p.n_energies);
  o->boundary_initialized = false;
  o->ldos_prev.clear();
}

// One LDOS iteration; ldos_out [n_fields][N0][N0] (may be NULL), residuals out.
void orc_ldos_iterate(void *h, int n_fields, double *ldos_out, double *res_ldos, double *res_bc) {
  Oracle *o = (Oracle *)h;
  o->ldos_iteration(n_fields);
  if (ldos_out) std::copy(o->ldos_prev.begin(), o->ldos_prev.end(), ldos_out);
  if (res_ldos) *res_ldos = o->res_ldos;
  if (res_bc) *res_bc = o->res_bc;
}

void orc_energy_shift(void *h, int a, double *es) {
  Oracle *o = (Oracle *)h;
  std::vector<double> v;
  o->energy_shift(a, v);
  std::memcpy(es, v.data(), v.size() * 8);
}
void orc_set_boundary_initial(void *h) { ((Oracle *)h)->set_boundary_initial(); }
double orc_compute_bc(void *h) { return ((Oracle *)h)->compute_bc(); }
void orc_poisson(void *h, const double *j, double *a_out) {
  Oracle *o = (Oracle *)h;
  const size_t nn = (size_t)o->p.n0 * o->p.n0;
  std::vector<double> jv(j, j + 2 * nn);
  o->poisson(jv);
  std::memcpy(a_out, o->a_new.data(), 2 * nn * 8);
}
// Riccati algebra probes for the known-answer tests.
void orc_riccati_step(const double *delta, const double *energy, const double *g0, double h,
                      double *out) {
  const cx r = riccati_step(mk(delta[0], delta[1]), mk(energy[0], energy[1]), mk(g0[0], g0[1]), h);
  out[0] = r.re;
  out[1] = r.im;
}
void orc_homogeneous(const double *delta, const double *energy, double *out) {
  cx g, gt;
  homogeneous(mk(delta[0], delta[1]), mk(energy[0], energy[1]), g, gt);
  out[0] = g.re;
  out[1] = g.im;
  out[2] = gt.re;
  out[3] = gt.im;
}
void orc_greens(const double *g, const double *gt, double *out) {
  const cx vg = greens_g(mk(g[0], g[1]), mk(gt[0], gt[1]));
  const cx vf = greens_f(mk(g[0], g[1]), mk(gt[0], gt[1]));
  out[0] = vg.re;
  out[1] = vg.im;
  out[2] = vf.re;
  out[3] = vf.im;
}
int orc_num_iterations(void *h) { return ((Oracle *)h)->n_iterations; }

}  // extern "C"

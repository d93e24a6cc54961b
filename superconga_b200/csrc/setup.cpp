// Host-side setup for the B200 self-consistency path.  See setup.hpp.
#include "setup.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>

#include "json.hpp"

#ifdef _OPENMP
#include <omp.h>
#endif

namespace scb {
namespace {

constexpr int GRAIN_SIZE_MARGIN = 3;       // defines.h:25
constexpr double MAXIMUM_COORDINATE = 0.5;  // defines.h:31
const double EULER_GAMMA = 0.57721566490153286060651209008240243;

// Largest Ozaki pole per pole count, Parameters.h:191-258 (first 60 entries).
const double MAX_OZAKI_POLE[] = {
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
    8346.608627256021, 8640.726968470750, 8939.938267543248, 9244.242524494641};

double wrap_range(double v, double lo, double hi) {
  if (lo <= v && v < hi) return v;
  const double r = hi - lo, s = (v - lo) / r;
  return (s - std::floor(s)) * r + lo;
}
float wrap_rangef(float v, float lo, float hi) {
  if (lo <= v && v < hi) return v;
  const float r = hi - lo, s = (v - lo) / r;
  return (s - std::floor(s)) * r + lo;
}
// utils::wrapToRange<int> goes through single precision (utils.h:70-78).
int wrap_int(int v, int lo, int hi) {
  return (int)std::round(wrap_rangef((float)v, (float)lo, (float)hi));
}
int sgn(double v) { return (0.0 < v) - (v < 0.0); }
void rotate(double ang, double x, double y, double &ox, double &oy) {
  const double c = std::cos(ang), s = std::sin(ang);
  ox = x * c - y * s;
  oy = x * s + y * c;
}
double wrap_range(double v, double lo, double hi);
int wrap_int(int v, int lo, int hi);
// FermiSurface::getAngleWeight (FermiSurface.h:210-243): Boole, Simpson 3/8,
// Simpson 1/3 or trapezoid weights by the divisibility of the angle count.
double angle_weight(int k, int na) {
  const int w = wrap_int(k, 0, na);
  if (na % 4 == 0) return (w % 4 == 0) ? 28.0 / 45.0 : (w % 2 == 0) ? 24.0 / 45.0 : 64.0 / 45.0;
  if (na % 3 == 0) return (w % 3 == 0) ? 6.0 / 8.0 : 9.0 / 8.0;
  if (na % 2 == 0) return (w % 2 == 0) ? 2.0 / 3.0 : 4.0 / 3.0;
  return 1.0;
}

// Square-lattice tight-binding band (DispersionTightBinding.h:62-125): hopping
// 1 to nearest neighbours, t1 to next-nearest, t2 to next-next-nearest,
// measured from the chemical potential mu; grad is the band velocity.
struct TbBand {
  double t1, t2, mu;
  double energy(double kx, double ky) const {
    const double nn = -2.0 * 1.0 * (std::cos(kx) + std::cos(ky));
    const double nnn = -4.0 * t1 * std::cos(kx) * std::cos(ky);
    const double nnnn = -2.0 * t2 * (std::cos(2.0 * kx) + std::cos(2.0 * ky));
    return nn + nnn + nnnn - mu;
  }
  void grad(double kx, double ky, double &gx, double &gy) const {
    const double a = 2.0 * 1.0, b = 4.0 * t1, c = 4.0 * t2;
    gx = a * std::sin(kx) + b * std::sin(kx) * std::cos(ky) + c * std::sin(2.0 * kx);
    gy = a * std::sin(ky) + b * std::cos(kx) * std::sin(ky) + c * std::sin(2.0 * ky);
  }
};

// The Fermi momentum along the ray offset + k (cos phi, sin phi): bisection
// between the origin and the zone edge until |e| < sqrt(tol), then Newton
// steps along the ray until |e| < tol, at most 100 evaluations; the result is
// wrapped into the first zone (tightbinding_internal::computeFermiMomentum,
// FermiSurfaceTightBinding.h:167-290).
void tb_fermi_momentum(const TbBand &band, double phi, double ox, double oy, double &px, double &py) {
  const double tol = 1e2 * std::numeric_limits<double>::epsilon();
  const double ux = std::cos(phi), uy = std::sin(phi);
  double ka = 0.0;
  double ea = band.energy(ka * ux + ox, ka * uy + oy);
  const double umax = std::max(std::fabs(ux), std::fabs(uy));
  double kb = M_PI / umax;
  double eb = band.energy(kb * ux + ox, kb * uy + oy);
  double k = 0.5 * (ka + kb);
  bool bisect = true;
  for (int it = 0; it < 100; ++it) {
    const double mx = k * ux + ox, my = k * uy + oy;
    const double e = band.energy(mx, my);
    const double err = std::fabs(e);
    if (err > std::sqrt(tol) && bisect) {
      if (sgn(e) == sgn(ea)) {
        ea = e;
        ka = k;
      } else {
        eb = e;
        kb = k;
      }
      if (sgn(ea) == sgn(eb)) break;
      k = 0.5 * (ka + kb);
    } else if (err > tol) {
      bisect = false;
      double gx, gy;
      band.grad(mx, my, gx, gy);
      const double slope = gx * ux + gy * uy;
      if (std::fabs(slope) > 0.0) k -= e / slope;
      else break;
    } else {
      break;
    }
  }
  px = wrap_range(k * ux + ox, -M_PI, M_PI);
  py = wrap_range(k * uy + oy, -M_PI, M_PI);
}

}  // namespace

// FermiSurfaceTightBinding::initialize (FermiSurfaceTightBinding.h:384-470):
// origin (0,0) or (pi,pi) by the band signs at (0,pi) and (pi,pi); per angle
// the Fermi momentum on the uniform polar grid, the band velocity, the system
// angle atan2(v) - pi/2 and the integrand factor |k.k / k.v| (momentum k
// measured from the origin) times the angle weight; the velocities are then
// divided by the weighted mean speed and the factors by their sum.
void tight_binding_surface(HostSetup &S) {
  const TbBand band{S.tb_hopping_nnn, S.tb_hopping_nnnn, S.tb_chemical_potential};
  const int na = S.n_angles;
  const double e_a = band.energy(0.0, M_PI), e_b = band.energy(M_PI, M_PI);
  S.p_off_x = S.p_off_y = (sgn(e_a) == sgn(e_b)) ? 0.0 : M_PI;
  S.phi.clear(), S.theta.clear(), S.px.clear(), S.py.clear();
  S.vx.clear(), S.vy.clear(), S.speed.clear(), S.weight.clear();
  double wsum = 0.0, psum = 0.0, vsum = 0.0;
  for (int k = 0; k < na; ++k) {
    const double ph = wrap_range(M_PI * (double)(2 * k) / (double)na + 0.5 * M_PI, 0.0, 2.0 * M_PI);
    double px, py, vx, vy;
    tb_fermi_momentum(band, ph, S.p_off_x, S.p_off_y, px, py);
    band.grad(px, py, vx, vy);
    const double kx = wrap_range(px, S.p_off_x - M_PI, S.p_off_x + M_PI) - S.p_off_x;
    const double ky = wrap_range(py, S.p_off_y - M_PI, S.p_off_y + M_PI) - S.p_off_y;
    const double jac = std::fabs((kx * kx + ky * ky) / (kx * vx + ky * vy));
    const double w = jac * angle_weight(k, na);
    S.phi.push_back(ph);
    S.theta.push_back(std::atan2(vy, vx) - 0.5 * M_PI);
    S.px.push_back(px);
    S.py.push_back(py);
    S.vx.push_back(vx);
    S.vy.push_back(vy);
    S.weight.push_back(w);
    wsum += w;
    psum += std::hypot(px, py) * w;
    vsum += std::hypot(vx, vy) * w;
  }
  S.avg_fermi_momentum = psum / wsum;
  S.avg_fermi_speed = vsum / wsum;
  for (int k = 0; k < na; ++k) {
    S.vx[k] /= S.avg_fermi_speed;
    S.vy[k] /= S.avg_fermi_speed;
    S.weight[k] /= wsum;
    S.speed.push_back(std::hypot(S.vx[k], S.vy[k]));  // FermiSurfaceTightBinding::getFermiSpeed
  }
}

double lattice_basis(int sym, double px, double py) {
  switch (sym) {
  case 0: return std::cos(px) + std::cos(py);
  case 1: return std::cos(px) - std::cos(py);
  case 2: return std::sin(px) * std::sin(py);
  default: return std::sin(px) * std::sin(py) * (std::cos(px) - std::cos(py));
  }
}

namespace {

// ------------------------------------------------------- eigen solvers ----
// Implicit QL iteration on a symmetric tridiagonal matrix (diagonal d,
// sub-diagonal e[1..n-1]); eigenvector rows z[i*n + k] are rotated alongside.
void tridiagonal_ql(int n, std::vector<double> &d, std::vector<double> &e,
                    std::vector<double> &z) {
  for (int i = 1; i < n; ++i) e[i - 1] = e[i];
  e[n - 1] = 0.0;
  for (int l = 0; l < n; ++l) {
    int iter = 0, m;
    do {
      for (m = l; m < n - 1; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) + dd == dd) break;
      }
      if (m != l) {
        if (++iter > 60) throw std::runtime_error("eigen: QL iteration did not converge");
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
        double s = 1.0, c = 1.0, p = 0.0;
        int i;
        for (i = m - 1; i >= l; --i) {
          double f = s * e[i];
          const double b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= p;
            e[m] = 0.0;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - p;
          r = (d[i] - g) * s + 2.0 * c * b;
          p = s * r;
          d[i + 1] = g + p;
          g = c * r - b;
          double *zi = &z[(size_t)i * n];
          double *zi1 = &z[(size_t)(i + 1) * n];
          for (int k = 0; k < n; ++k) {
            f = zi1[k];
            zi1[k] = s * zi[k] + c * f;
            zi[k] = c * zi[k] - s * f;
          }
        }
        if (r == 0.0 && i >= l) continue;
        d[l] -= p;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
}

// Householder reduction of a dense symmetric matrix (row-major, overwritten by
// the orthogonal transform) to tridiagonal form.
void householder_tridiagonal(int n, std::vector<double> &a, std::vector<double> &d,
                             std::vector<double> &e) {
  auto A = [&](int i, int j) -> double & { return a[(size_t)i * n + j]; };
  for (int i = n - 1; i > 0; --i) {
    const int l = i - 1;
    double hh = 0.0, scale = 0.0;
    if (l > 0) {
      for (int k = 0; k <= l; ++k) scale += std::fabs(A(i, k));
      if (scale == 0.0) {
        e[i] = A(i, l);
      } else {
        for (int k = 0; k <= l; ++k) {
          A(i, k) /= scale;
          hh += A(i, k) * A(i, k);
        }
        double f = A(i, l);
        double g = (f >= 0.0) ? -std::sqrt(hh) : std::sqrt(hh);
        e[i] = scale * g;
        hh -= f * g;
        A(i, l) = f - g;
        f = 0.0;
        for (int j = 0; j <= l; ++j) {
          A(j, i) = A(i, j) / hh;
          g = 0.0;
          for (int k = 0; k <= j; ++k) g += A(j, k) * A(i, k);
          for (int k = j + 1; k <= l; ++k) g += A(k, j) * A(i, k);
          e[j] = g / hh;
          f += e[j] * A(i, j);
        }
        const double hk = f / (hh + hh);
        for (int j = 0; j <= l; ++j) {
          f = A(i, j);
          g = e[j] - hk * f;
          e[j] = g;
          for (int k = 0; k <= j; ++k) A(j, k) -= (f * e[k] + g * A(i, k));
        }
      }
    } else {
      e[i] = A(i, l);
    }
    d[i] = hh;
  }
  d[0] = 0.0;
  e[0] = 0.0;
  for (int i = 0; i < n; ++i) {
    const int l = i - 1;
    if (d[i] != 0.0) {
      for (int j = 0; j <= l; ++j) {
        double g = 0.0;
        for (int k = 0; k <= l; ++k) g += A(i, k) * A(k, j);
        for (int k = 0; k <= l; ++k) A(k, j) -= g * A(k, i);
      }
    }
    d[i] = A(i, i);
    A(i, i) = 1.0;
    for (int j = 0; j <= l; ++j) {
      A(j, i) = 0.0;
      A(i, j) = 0.0;
    }
  }
}

}  // namespace

// Symmetric eigendecomposition: on return w holds the eigenvalues in ascending
// order and a holds the matching unit eigenvectors as rows.
void symmetric_eigen(int n, std::vector<double> &a, std::vector<double> &w) {
  std::vector<double> d(n), e(n);
  householder_tridiagonal(n, a, d, e);
  // Columns of a are the transform's vectors; QL rotates rows, so transpose.
  std::vector<double> z((size_t)n * n);
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < n; ++k) z[(size_t)i * n + k] = a[(size_t)k * n + i];
  tridiagonal_ql(n, d, e, z);
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    w[i] = d[order[i]];
    std::memcpy(&a[(size_t)i * n], &z[(size_t)order[i] * n], sizeof(double) * n);
  }
}

// Parameters::computeNumOzakiEnergies, Parameters.h:380-420.
int num_ozaki_poles(double temperature, double cutoff) {
  const double val = 2.0 * M_PI * (cutoff / temperature);
  const int n = (int)(sizeof(MAX_OZAKI_POLE) / sizeof(double));
  for (int i = 0; i < n; ++i)
    if (MAX_OZAKI_POLE[i] > val) return i + 1;
  int i = n - 1;
  while (true) {
    ++i;
    const double x = (double)i;
    if (x * (2.5465 * x + 1.2744) + 0.4651 >= val) return i;
  }
}

// IntegrationIteratorOzaki::computeOzakiPoles, IntegrationIteratorOzaki.h:108-163.
// The generalised problem A z = w B z with B = diag(2i+1) is brought to the
// symmetric tridiagonal B^-1/2 A B^-1/2 (zero diagonal); eigenvectors z are
// B-normalised as LAPACK dsygv returns them.
void ozaki_poles(int n, double *poles, double *residues) {
  const int N = 2 * n;
  std::vector<double> d(N, 0.0), e(N, 0.0), z((size_t)N * N, 0.0);
  for (int i = 1; i < N; ++i)
    e[i] = -0.5 / std::sqrt((2.0 * (i - 1) + 1.0) * (2.0 * i + 1.0));
  for (int i = 0; i < N; ++i) z[(size_t)i * N + i] = 1.0;
  tridiagonal_ql(N, d, e, z);
  std::vector<int> order(N);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
  for (int i = 0; i < n; ++i) {
    const int k = order[i];
    const double pole = -1.0 / d[k];
    const double z0 = z[(size_t)k * N + 0] / std::sqrt(1.0);
    const double rs = 0.5 * z0 * pole;
    poles[i] = pole;
    residues[i] = rs * rs;
  }
}

// computeOrderParameterBulkSWave, OrderParameterBulk.h:88-221: secant
// iteration on the bulk gap equation with the Matsubara sum cut at
// energy_cutoff, starting from S_WAVE_BULK sqrt(1 - t^3) and its square root.
double bulk_s_wave(double t, double crit, int max_it, double energy_cutoff) {
  const double eps = std::numeric_limits<double>::epsilon();
  if (t >= 1.0) return 0.0;
  const double s_bulk = 0.5 * std::exp(-EULER_GAMMA);
  if (t < eps) return s_bulk;
  const int ne = (int)(energy_cutoff / t - 0.5) + 1;
  double es = 0.0;
  for (int n = ne - 1; n >= 0; --n) es += 1.0 / (t * ((double)n + 0.5));
  const double coupling = 1.0 / (std::log(t) / t + es);
  auto resid = [&](double op) {
    double integ = 0.0;
    for (int n = ne - 1; n >= 0; --n) integ += 1.0 / std::hypot(op, t * ((double)n + 0.5));
    return op * (integ * coupling - 1.0);
  };
  double op = s_bulk * std::sqrt(1.0 - t * t * t);
  double ops[2] = {op, std::sqrt(op)}, rs[2] = {resid(ops[0]), resid(ops[1])};
  for (int it = 0; it < max_it; ++it) {
    const double w = 1.0 / (1.0 - (ops[0] / ops[1]) / (rs[0] / rs[1]));
    op = (1.0 - w) * ops[0] + w * ops[1];
    const double r = resid(op);
    const bool small = op < 10.0 * eps;
    const double rel = small ? r : std::fabs(r / op);
    if (rel < crit) break;
    const int k = std::fabs(rs[0]) > std::fabs(rs[1]) ? 0 : 1;
    ops[k] = op;
    rs[k] = r;
  }
  return op;
}

// computeFreeEnergyBulkSWave, OrderParameterBulk.h:224-246: the bulk free
// energy density Delta^2 (ln t + t sum_n [1/e_n - 2/(e_n + Omega_n)]).
double bulk_free_energy_s_wave(double t, double op, double energy_cutoff) {
  const int ne = (int)(energy_cutoff / t - 0.5) + 1;
  double esum = 0.0;
  for (int n = ne - 1; n >= 0; --n) {
    const double e = t * ((double)n + 0.5);
    esum += 1.0 / e - 2.0 / (e + std::hypot(op, e));
  }
  return op * op * (std::log(t) + t * esum);
}

// computeYoshidaBulkSWave, OrderParameterBulk.h:256-277: the Yoshida function
// Y = t Delta^2 sum_n 1/Omega_n^3 (1 at zero temperature).
double bulk_yoshida_s_wave(double t, double op, double energy_cutoff) {
  if (t < std::numeric_limits<double>::epsilon()) return 1.0;
  const int ne = (int)(energy_cutoff / t - 0.5) + 1;
  double esum = 0.0;
  for (int n = ne - 1; n >= 0; --n) {
    const double om = std::hypot(op, t * ((double)n + 0.5));
    esum += 1.0 / (om * om * om);
  }
  return t * op * op * esum;
}

long long HostSetup::site_updates_per_iteration() const {
  long long inside = 0;
  const size_t nn = (size_t)n1 * n1;
  for (int a = 0; a < n_angles; ++a)
    for (size_t i = 0; i < nn; ++i)
      if (labels[(size_t)a * nn + i] > 0) inside++;
  return 2LL * ne * inside;
}

namespace {

// ----------------------------------------------------------- geometry -----
struct FrameGeom {
  std::vector<uint8_t> label;
  std::vector<double> nx, ny, dist;
};

double convert_coord(double f, int nsim, int ngrid) {
  return (double)(nsim - 1) * (f + MAXIMUM_COORDINATE) + 0.5 * (double)(ngrid - nsim);
}

// Row-majority 3x3 disc labelling, DiscGeometry.h:75-150.
uint8_t disc_label(int ix, int iy, double r, double ox, double oy) {
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

// DiscGeometry::create / generateDisc_Kernel, DiscGeometry.h:152-198,262-283.
void disc_frame(const GeomComp &g, double angle, int n0, int n, FrameGeom &o) {
  double rcx, rcy;
  rotate(angle, g.cx, g.cy, rcx, rcy);
  const double ox = convert_coord(rcx, n0, n), oy = convert_coord(rcy, n0, n);
  const double r = g.radius * (double)(n0 - 1);
  const size_t nn = (size_t)n * n;
  o.label.assign(nn, 0);
  o.nx.assign(nn, 0.0);
  o.ny.assign(nn, 0.0);
  o.dist.assign(nn, 0.0);
  for (int ty = 0; ty < n; ++ty)
    for (int tx = 0; tx < n; ++tx) {
      const uint8_t lab = disc_label(tx, ty, r, ox, oy);
      const size_t i = (size_t)ty * n + tx;
      o.label[i] = lab;
      if (lab > 1) {
        const double x = (double)tx - ox, y = (double)ty - oy;
        const double bd = std::sqrt(r * r - x * x) - std::fabs(y);
        o.dist[i] = bd;
        o.nx[i] = -x / r;
        o.ny[i] = (y <= 0.0) ? -(y - bd) / r : -(y + bd) / r;
      }
    }
}

// PolygonGeometry::create with labelBoundaryNodes and maskNormals,
// PolygonGeometry.h:100-190,234-252,355-381; GeometryComponent.h:112-147.
void polygon_frame(const GeomComp &g, double angle, int n0, int n, FrameGeom &o) {
  const int nv = (int)g.vx.size();
  const double scale = (double)(n0 - 1);
  const double ca = std::cos(angle), sa = std::sin(angle);
  std::vector<double> px(nv), py(nv), enx(nv), eny(nv);
  for (int i = 0; i < nv; ++i) {
    px[i] = (ca * g.vx[i] - sa * g.vy[i]) * scale;
    py[i] = (sa * g.vx[i] + ca * g.vy[i]) * scale;
  }
  const size_t nn = (size_t)n * n;
  std::vector<uint8_t> raw(nn);
  o.nx.assign(nn, 0.0);
  o.ny.assign(nn, 0.0);
  o.dist.assign(nn, 0.0);
  for (int ty = 0; ty < n; ++ty)
    for (int tx = 0; tx < n; ++tx) {
      const double cx = (double)tx - (double)(n - 1) * 0.5;
      const double cy = (double)ty - (double)(n - 1) * 0.5;
      int crossings = 0;
      double bd = 100000.0, bnx = 0.0, bny = 0.0;
      for (int i = 0; i < nv; ++i) {
        const int ip = (i + 1 == nv) ? 0 : i + 1;
        const double lx = px[ip] - px[i], ly = py[ip] - py[i];
        if (lx * (cy - py[i]) - ly * (cx - px[i]) >= 0.0) crossings++;
        double tnx = -ly, tny = lx;
        const double inv = 1.0 / std::sqrt(tnx * tnx + tny * tny);
        tnx *= inv;
        tny *= inv;
        double td = 10000.0;
        if (std::fabs(lx) > 0.00001) {
          const double k = ly / lx, m = py[i] - k * px[i];
          td = std::fabs(k * cx + m - cy);
        }
        if (td < bd) {
          bd = td;
          bnx = tnx;
          bny = tny;
        }
      }
      const size_t idx = (size_t)ty * n + tx;
      raw[idx] = crossings == nv ? 1 : 0;
      o.dist[idx] = bd;
      o.nx[idx] = bnx;
      o.ny[idx] = bny;
    }
  o.label.assign(nn, 0);
  for (int ty = 1; ty < n - 1; ++ty)
    for (int tx = 0; tx < n; ++tx) {
      const uint8_t l0 = raw[(size_t)(ty - 1) * n + tx], l1 = raw[(size_t)ty * n + tx],
                    l2 = raw[(size_t)(ty + 1) * n + tx];
      uint8_t nl = 0;
      if (l1 == 1) {
        nl = 1;
        if (l0 == 0) nl = 2;
        else if (l2 == 0) nl = 3;
        if (l0 == 0 && l2 == 0) nl = 0;
      }
      o.label[(size_t)ty * n + tx] = nl;
    }
  for (size_t i = 0; i < nn; ++i) {
    const double m = (double)(o.label[i] > 1);
    o.dist[i] *= m;
    o.nx[i] *= m;
    o.ny[i] *= m;
  }
}

void normalize2(double &x, double &y) {
  const double inv = 1.0 / std::sqrt(x * x + y * y);
  x *= inv;
  y *= inv;
}

// GeometryGroup::create with the add/remove operators,
// GeometryGroup.h:216-334,499-522,590-628.
void group_frame(const std::vector<GeomComp> &geom, double angle, int n0, int n,
                 FrameGeom &o) {
  static const uint8_t op_add[16] = {0, 1, 2, 3, 1, 1, 1, 1, 2, 1, 2, 1, 3, 1, 1, 3};
  const size_t nn = (size_t)n * n;
  o.label.assign(nn, 0);
  o.nx.assign(nn, 0.0);
  o.ny.assign(nn, 0.0);
  o.dist.assign(nn, 0.0);
  FrameGeom c;
  for (const GeomComp &g : geom) {
    if (g.type == 0) disc_frame(g, angle, n0, n, c);
    else polygon_frame(g, angle, n0, n, c);
    if (g.add) {
      for (size_t i = 0; i < nn; ++i) {
        const uint8_t nl = op_add[o.label[i] * 4 + c.label[i]];
        double ax = 0.0, ay = 0.0;
        if (nl == 2 || nl == 3) {
          ax = o.nx[i] + c.nx[i];
          ay = o.ny[i] + c.ny[i];
          normalize2(ax, ay);
        }
        o.nx[i] = ax;
        o.ny[i] = ay;
        o.label[i] = nl;
        o.dist[i] = std::max(o.dist[i], c.dist[i]);
      }
    } else {
      std::vector<uint8_t> tmp(nn, 0);
      for (int ty = 1; ty < n - 1; ++ty)
        for (int tx = 0; tx < n; ++tx) {
          const size_t im = (size_t)(ty - 1) * n + tx, i = (size_t)ty * n + tx,
                       ip = (size_t)(ty + 1) * n + tx;
          uint8_t d0 = o.label[i];
          if (c.label[i] > 0) {
            d0 = 0;
          } else if (c.label[ip] == 2) {
            if (d0 == 1) {
              d0 = 3;
              double ax = o.nx[i] - c.nx[ip], ay = o.ny[i] - c.ny[ip];
              normalize2(ax, ay);
              o.nx[i] = ax;
              o.ny[i] = ay;
              o.dist[i] = 1.0 - c.dist[ip];
            }
          } else if (c.label[im] == 3) {
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
      o.label.swap(tmp);
    }
  }
}

// GeometryGroup::createDomain, GeometryGroup.h:524-544 (reference frame).
void domain_reference(const std::vector<GeomComp> &geom, int n0, std::vector<uint8_t> &dom) {
  const int n = n0;
  const size_t nn = (size_t)n * n;
  dom.assign(nn, 0);
  std::vector<uint8_t> loc(nn);
  for (const GeomComp &g : geom) {
    if (g.type == 0) {
      const double ox = convert_coord(g.cx, n0, n), oy = convert_coord(g.cy, n0, n);
      const double r = g.radius * (double)(n0 - 1);
      for (int ty = 0; ty < n; ++ty)
        for (int tx = 0; tx < n; ++tx)
          loc[(size_t)ty * n + tx] = disc_label(tx, ty, r, ox, oy) > 0 ? 1 : 0;
    } else {
      const int nv = (int)g.vx.size();
      for (int ty = 0; ty < n; ++ty)
        for (int tx = 0; tx < n; ++tx) {
          const double cx = (double)tx / (double)(n - 1) - 0.5;
          const double cy = (double)ty / (double)(n - 1) - 0.5;
          int crossings = 0;
          for (int i = 0; i < nv; ++i) {
            const int ip = (i == nv - 1) ? 0 : i + 1;
            const double lx = g.vx[ip] - g.vx[i], ly = g.vy[ip] - g.vy[i];
            if (lx * (cy - g.vy[i]) - ly * (cx - g.vx[i]) >= 0.0) crossings++;
          }
          loc[(size_t)ty * n + tx] = crossings == nv ? 1 : 0;
        }
    }
    for (size_t i = 0; i < nn; ++i) {
      if (g.add) {
        if (loc[i]) dom[i] = 1;
      } else {
        dom[i] = (dom[i] == 0 || loc[i] > 0) ? 0 : 1;
      }
    }
  }
}

// Extension sources of every label-0 site next to the grain (domain_ops.h:11-69).
void extension_table(const uint8_t *lab, int n, std::vector<int> &site, std::vector<int> &off,
                     std::vector<int> &src) {
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x) {
      if (lab[(size_t)y * n + x] != 0) continue;
      const int x0 = std::max(x - 2, 0), x1 = std::min(x + 2, n - 1);
      const int y0 = std::max(y - 2, 0), y1 = std::min(y + 2, n - 1);
      int best = 1000;
      for (int ky = y0; ky <= y1; ++ky)
        for (int kx = x0; kx <= x1; ++kx)
          if (lab[(size_t)ky * n + kx] > 0) {
            const int d2 = (x - kx) * (x - kx) + (y - ky) * (y - ky);
            best = std::min(best, d2);
          }
      if (best == 1000) continue;
      site.push_back(y * n + x);
      for (int ky = y0; ky <= y1; ++ky)
        for (int kx = x0; kx <= x1; ++kx)
          if (lab[(size_t)ky * n + kx] > 0) {
            const int d2 = (x - kx) * (x - kx) + (y - ky) * (y - ky);
            if (d2 == best) src.push_back(ky * n + kx);
          }
      off.push_back((int)src.size());
    }
}

struct BoundaryNode {
  int x, y;
  double nx, ny, dist;
};

}  // namespace

std::string build_setup(const std::string &json, HostSetup &S, const SetupOverrides *ov) {
  JsonValue cfg;
  try {
    cfg = JsonValue::parse(json);
  } catch (const std::exception &ex) {
    return std::string("config: ") + ex.what();
  }
  const JsonValue &phys = cfg["physics"], &num = cfg["numerics"], &misc = cfg["misc"];
  if (!phys.is_object() || !num.is_object() || !cfg["geometry"].is_array())
    return "config: 'physics', 'numerics' and 'geometry' are required";

  // src/simulation.cu:101-155.
  S.temperature = phys["temperature"].as_double();
  const double ppxi = num["points_per_coherence_length"].as_double();
  const double cutoff = num["energy_cutoff"].as_double();
  S.n_angles = num["num_fermi_momenta"].as_int();
  S.conv_crit = num["convergence_criterion"].as_double(1e-6);
  S.lambda = phys["penetration_depth"].as_double(-1.0);
  S.flux_quanta = phys["external_flux_quanta"].as_double();
  S.charge_sign = sgn((double)phys["charge_sign"].as_int(-1));
  const std::string norm = num["norm"].as_string("l2");
  if (norm == "l1") S.norm = NORM_L1;
  else if (norm == "l2") S.norm = NORM_L2;
  else if (norm == "linf") S.norm = NORM_LINF;
  else return "config: norm type '" + norm + "' not understood";
  S.vp_max_error = num["vector_potential_error"].as_double(1e-6);
  S.burnin = num["num_iterations_burnin"].as_int(0);
  S.it_min = num["num_iterations_min"].as_int(0);
  S.it_max = num["num_iterations_max"].as_int(-1);
  if (ov) {
    if (ov->n_angles > 0) S.n_angles = ov->n_angles;
    if (ov->conv_crit > 0.0) S.conv_crit = ov->conv_crit;
    if (ov->norm >= 0) S.norm = ov->norm;
  }
  if (!(S.temperature > 0.0) || !(ppxi > 0.0) || !(cutoff > 0.0) || S.n_angles < 1)
    return "config: temperature, points_per_coherence_length, energy_cutoff and "
           "num_fermi_momenta must be positive";
  (void)misc;

  // geometry_utils::computeGeometryScaling, geometry_utils.h:41-172.
  const JsonValue &gl = cfg["geometry"];
  double xmax = std::numeric_limits<double>::min(), xmin = std::numeric_limits<double>::max();
  double ymax = xmax, ymin = xmin;
  for (size_t i = 0; i < gl.size(); ++i) {
    const std::vector<std::string> names = gl[i].keys();
    if (names.empty()) return "config: empty geometry component";
    const std::string nm = names[0];
    const JsonValue &g = gl[i][nm];
    if (!g["add"].as_bool()) continue;
    if (nm == "disc") {
      const double r = g["radius"].as_double(), cx = g["center_x"].as_double(),
                   cy = g["center_y"].as_double();
      xmax = std::max(xmax, cx + r);
      xmin = std::min(xmin, cx - r);
      ymax = std::max(ymax, cy + r);
      ymin = std::min(ymin, cy - r);
    } else if (nm == "polygon") {
      const JsonValue &vx = g["vertices_x"], &vy = g["vertices_y"];
      if (vx.size() != vy.size()) return "config: polygon vertex arrays differ in length";
      for (size_t k = 0; k < vx.size(); ++k) {
        xmax = std::max(xmax, vx[k].as_double());
        xmin = std::min(xmin, vx[k].as_double());
        ymax = std::max(ymax, vy[k].as_double());
        ymin = std::min(ymin, vy[k].as_double());
      }
    } else if (nm == "regular_polygon") {
      const double side = g["side_length"].as_double(), cx = g["center_x"].as_double(),
                   cy = g["center_y"].as_double();
      const double rot = 2.0 * M_PI * g["rotation"].as_double();
      const double ne = (double)g["num_edges"].as_int();
      const double step = 2.0 * M_PI / ne;
      const double radius = side / std::hypot(std::cos(step) - 1.0, std::sin(step));
      const double off = 0.5 * step + rot;
      for (int k = 0; k < (int)ne; ++k) {
        const double ang = off + step * (double)k;
        const double x = cx + radius * std::cos(ang), y = cy + radius * std::sin(ang);
        xmax = std::max(xmax, x);
        xmin = std::min(xmin, x);
        ymax = std::max(ymax, y);
        ymin = std::min(ymin, y);
      }
    } else {
      return "config: unknown geometry type '" + nm + "'";
    }
  }
  const double xe = xmax - xmin, ye = ymax - ymin;
  const double xo = xmin + 0.5 * xe, yo = ymin + 0.5 * ye;
  const double scaling = std::max(xe, ye);
  if (!(scaling > 0.0)) return "config: the geometry has no added component";

  // Parameters::setLatticeResolution, Parameters.h:422-458.
  S.grain_width = scaling;
  S.h = 1.0 / ppxi;
  const double frac = scaling * ppxi;
  S.n0 = (int)std::ceil(frac) + 2 * GRAIN_SIZE_MARGIN;
  S.grain_fraction = frac / (double)S.n0;
  S.n1 = S.n0 + 2 * (int)std::ceil(0.5 * (std::sqrt(2.0) - 1.0) * (double)S.n0);
  const double gf = S.grain_fraction;

  // geometry_utils::addGeometryComponents, geometry_utils.h:189-325.
  for (size_t i = 0; i < gl.size(); ++i) {
    const std::string nm = gl[i].keys()[0];
    const JsonValue &g = gl[i][nm];
    GeomComp c;
    c.add = g["add"].as_bool();
    if (nm == "disc") {
      c.type = 0;
      const double cx = (g["center_x"].as_double() - xo) / scaling;
      const double cy = (g["center_y"].as_double() - yo) / scaling;
      const double r = g["radius"].as_double() / scaling;
      c.radius = r * gf;
      c.cx = cx * gf;
      c.cy = cy * gf;
    } else if (nm == "polygon") {
      c.type = 1;
      const JsonValue &vx = g["vertices_x"], &vy = g["vertices_y"];
      for (size_t k = 0; k < vx.size(); ++k) {
        c.vx.push_back((vx[k].as_double() - xo) / scaling * gf);
        c.vy.push_back((vy[k].as_double() - yo) / scaling * gf);
      }
      if (c.vx.size() < 3) return "config: a polygon needs at least 3 vertices";
    } else {
      c.type = 1;
      const double cx = (g["center_x"].as_double() - xo) / scaling;
      const double cy = (g["center_y"].as_double() - yo) / scaling;
      const double side = g["side_length"].as_double() / scaling;
      const int nedge = g["num_edges"].as_int();
      if (nedge < 3 || nedge > 256) return "config: num_edges must be in [3, 256]";
      const double rot = 2.0 * M_PI * g["rotation"].as_double();
      const double step = 2.0 * M_PI / (double)nedge;
      const double rfs = side / std::hypot(std::cos(step) - 1.0, std::sin(step));
      const double radius = side < 0.0 ? MAXIMUM_COORDINATE : rfs;
      const double rp = radius * gf, cpx = cx * gf, cpy = cy * gf;
      const double off = step * 0.5 + rot;
      for (int k = 0; k < nedge; ++k) {
        const double ang = step * (double)k + off;
        c.vx.push_back(rp * std::cos(ang) + cpx);
        c.vy.push_back(rp * std::sin(ang) + cpy);
      }
    }
    S.geom.push_back(c);
  }

  // Integration iterator (IntegrationIteratorOzaki.h:165-200).
  S.ne = num_ozaki_poles(S.temperature, cutoff);
  std::vector<double> poles(S.ne);
  S.residues.resize(S.ne);
  ozaki_poles(S.ne, poles.data(), S.residues.data());
  S.e_im.resize(S.ne);
  for (int i = 0; i < S.ne; ++i) S.e_im[i] = poles[i] * S.temperature / (2.0 * M_PI);
  S.e_re.assign(S.ne, 0.0);

  // Order parameter (src/simulation.cu:199-295).
  const JsonValue &ops = phys["order_parameter"];
  const char *order[4] = {"dx2-y2", "dxy", "g", "s"};
  const int ids[4] = {1, 2, 3, 0};
  for (int k = 0; k < 4; ++k)
    if (ops.has(order[k])) {
      S.sym.push_back(ids[k]);
      S.sym_name.push_back(order[k]);
      S.tc.push_back(ops[order[k]]["critical_temperature"].as_double(1.0));
    }
  S.nc = (int)S.sym.size();
  if (S.nc == 0) return "config: no order-parameter component set";
  S.crystal_rot = 2.0 * M_PI * phys["crystal_axes_rotation"].as_double();

  // Fermi surface model.  The reference selects it in code, through
  // Context::set(std::unique_ptr<FermiSurface<T>>) (Context.h:49-51; the
  // drivers keep the default circle, Context.h:189); here the JSON key
  // physics.fermi_surface = {"type": "tight_binding", "hopping_nnn",
  // "hopping_nnnn", "chemical_potential"} selects the tight-binding surface,
  // with the defaults of its constructor (FermiSurfaceTightBinding.h:374-381).
  {
    const JsonValue &fs = phys["fermi_surface"];
    const std::string fs_type = fs["type"].as_string("circle");
    if (fs_type == "tight_binding") {
      S.fs_tight_binding = 1;
      S.tb_hopping_nnn = fs["hopping_nnn"].as_double(0.0);
      S.tb_hopping_nnnn = fs["hopping_nnnn"].as_double(0.0);
      S.tb_chemical_potential = fs["chemical_potential"].as_double(1.0);
    } else if (fs_type != "circle") {
      return "config: fermi_surface type '" + fs_type + "' not understood";
    }
  }

  const std::string gauge = phys["gauge"].as_string("symmetric");
  if (gauge == "landau") S.gauge = GAUGE_LANDAU;
  else if (gauge == "symmetric") S.gauge = GAUGE_SYMMETRIC;
  else if (gauge == "solenoid") S.gauge = GAUGE_SOLENOID;
  else return "config: gauge '" + gauge + "' not understood";

  // Accelerator (src/simulation.cu:383-415; defaults from accelerators/*.h).
  const JsonValue &acc = cfg["accelerator"];
  const std::string an = acc["name"].as_string("congacc");
  if (an == "congacc") { S.acc.kind = ACC_CONGACC; S.acc.step_size = 0.5; }
  else if (an == "picard") { S.acc.kind = ACC_PICARD; S.acc.step_size = 1.0; }
  else if (an == "polyak") { S.acc.kind = ACC_POLYAK; S.acc.step_size = 2.0; }
  else if (an == "barzilai-borwein" || an == "bb") { S.acc.kind = ACC_BB; S.acc.step_size = 1.0; }
  else if (an == "anderson") { S.acc.kind = ACC_ANDERSON; S.acc.step_size = 1.0; }
  else return "config: accelerator '" + an + "' not understood";
  S.acc.step_size = acc["step_size"].as_double(S.acc.step_size);
  S.acc.step_size_factor = acc["step_size_factor"].as_double(1.234);
  S.acc.cos_similarity_min = acc["cos_similarity_min"].as_double(0.7);
  S.acc.step_size_max = acc["step_size_max"].as_double(100.0);
  S.acc.step_size_min = acc["step_size_min"].as_double(0.001);
  S.acc.drag = acc["drag"].as_double(0.5);
  S.acc.rank = acc["rank"].as_int(4);

  // Fermi surface (FermiSurface.h:104-250, FermiSurfaceCircle.h:84-164, or
  // FermiSurfaceTightBinding.h:384-470).
  const int na = S.n_angles;
  if (S.fs_tight_binding) {
    tight_binding_surface(S);
  } else {
    for (int k = 0; k < na; ++k) {
      const double ph = wrap_range(M_PI * (double)(2 * k) / (double)na + 0.5 * M_PI, 0.0, 2.0 * M_PI);
      S.phi.push_back(ph);
      S.theta.push_back(ph - 0.5 * M_PI);
      S.vx.push_back(std::cos(ph));
      S.vy.push_back(std::sin(ph));
      S.weight.push_back(angle_weight(k, na) / (double)na);
      S.speed.push_back(1.0);  // a circle: constant speed (FermiSurfaceCircle.h:51-52)
    }
    S.px = S.vx;  // momentum and velocity coincide on the circle
    S.py = S.vy;
  }
  for (int k = 0; k < na; ++k) S.step.push_back(S.fs_tight_binding ? S.h / S.speed[k] : S.h);
  auto basis_raw = [&](int s, double px, double py) {
    if (S.fs_tight_binding) return lattice_basis(s, px, py);
    switch (s) {
    case 0: return 1.0;
    case 1: return px * px - py * py;
    case 2: return px * py;
    default: return px * py * (px * px - py * py);
    }
  };
  // BasisFunction::normalize, OrderParameterBasis.h:222-248 (the momentum is
  // not rotated by the crystal axes here).
  for (int c = 0; c < S.nc; ++c) {
    double avg = 0.0;
    for (int k = 0; k < na; ++k) {
      const double b = basis_raw(S.sym[c], S.px[k], S.py[k]);
      avg += (b * b + 0.0 * 0.0) * S.weight[k];
    }
    S.norm_factor.push_back(1.0 / std::sqrt(avg));
  }
  // computeMomentumDependence, OrderParameterComponent.h:197-208.
  S.eta.resize((size_t)na * S.nc);
  for (int k = 0; k < na; ++k)
    for (int c = 0; c < S.nc; ++c) {
      double rx, ry;
      rotate(S.crystal_rot, S.px[k], S.py[k], rx, ry);
      S.eta[(size_t)k * S.nc + c] = basis_raw(S.sym[c], rx, ry) * S.norm_factor[c];
    }
  // OrderParameterComponent::initCouplingConstant, OrderParameterComponent.h:156-181.
  for (int c = 0; c < S.nc; ++c) {
    double es = 0.0;
    for (int e = 0; e < S.ne; ++e) es += S.residues[e] / S.e_im[e];
    es *= S.temperature;
    S.coupling.push_back(0.5 * S.temperature / (std::log(S.temperature / S.tc[c]) + es));
  }
  // Rotation coefficients (float trigonometry as insertRotatedGrid's kernels).
  for (int k = 0; k < na; ++k) {
    auto fc = [](double phi_d, double &c, double &s) {
      const float pf = (float)phi_d;
      c = (double)std::cos(-pf);
      s = (double)std::sin(-pf);
    };
    double c, s;
    fc(S.theta[wrap_int(-k, 0, na)], c, s);  // OrderParameter::getRotatedGrid(-k)
    S.cD.push_back(c);
    S.sD.push_back(s);
    fc(-S.theta[k], c, s);  // computeEnergyShift: insertRotatedGrid(A, -theta)
    S.cA.push_back(c);
    S.sA.push_back(s);
    fc(S.theta[k], c, s);  // integrateGreensAngle: insertRotatedGrid(G, theta)
    S.cB.push_back(c);
    S.sB.push_back(s);
    S.cE.push_back(std::cos(S.theta[k]));
    S.sE.push_back(std::sin(S.theta[k]));
  }

  // Geometry in the reference frame.
  const int n0 = S.n0, n1 = S.n1;
  domain_reference(S.geom, n0, S.domain_ref);
  S.n_grain = 0;
  for (uint8_t v : S.domain_ref) S.n_grain += v > 0 ? 1 : 0;
  S.area = S.h * S.h * (double)S.n_grain;
  if (S.n_grain == 0) return "config: the grain covers no lattice site";
  extension_table(S.domain_ref.data(), n0, S.rext_site, S.rext_src_off, S.rext_src);
  S.rext_src_off.insert(S.rext_src_off.begin(), 0);

  // Geometry in every trajectory frame (GeometryGroup::create(-theta)).
  const size_t nn1 = (size_t)n1 * n1;
  S.labels.assign((size_t)na * nn1, 0);
  std::vector<std::vector<BoundaryNode>> lab2(na), lab3(na);  // per angle, column-major y order
  std::vector<std::vector<int>> cnt2(na), cnt3(na);
  std::vector<std::vector<int>> h_site(na), h_off(na), h_src(na);
  S.col_lo.assign((size_t)na * n1, -1);
  S.col_hi.assign((size_t)na * n1, -1);
  std::string err;
#pragma omp parallel for schedule(dynamic, 1)
  for (int a = 0; a < na; ++a) {
    FrameGeom fg;
    group_frame(S.geom, -S.theta[a], n0, n1, fg);
    std::memcpy(&S.labels[(size_t)a * nn1], fg.label.data(), nn1);
    cnt2[a].assign(n1, 0);
    cnt3[a].assign(n1, 0);
    for (int x = 0; x < n1; ++x)
      for (int y = 0; y < n1; ++y) {
        const size_t i = (size_t)y * n1 + x;
        const uint8_t l = fg.label[i];
        if (l > 0) {
          if (S.col_lo[(size_t)a * n1 + x] < 0) S.col_lo[(size_t)a * n1 + x] = y;
          S.col_hi[(size_t)a * n1 + x] = y;
        }
        if (l == 2) {
          lab2[a].push_back({x, y, fg.nx[i], fg.ny[i], std::fabs(fg.dist[i])});
          cnt2[a][x]++;
        } else if (l == 3) {
          lab3[a].push_back({x, y, fg.nx[i], fg.ny[i], std::fabs(fg.dist[i])});
          cnt3[a][x]++;
        }
      }
    extension_table(fg.label.data(), n1, h_site[a], h_off[a], h_src[a]);
  }
  if (!err.empty()) return err;

  // Sparse boundary storage, BoundaryStorage.h:244-527 with GeometryGroup.h:750-894.
  S.idx_in_g.assign((size_t)na * n1, -1);
  S.idx_out_g = S.idx_in_g;
  S.idx_in_gt = S.idx_in_g;
  S.idx_out_gt = S.idx_in_g;
  S.nisect_g.assign((size_t)na * n1, 0);
  S.nisect_gt.assign((size_t)na * n1, 0);
  for (int a = 0; a < na; ++a)
    for (int x = 0; x < n1; ++x) {
      const size_t ax = (size_t)a * n1 + x;
      const int c2 = cnt2[a][x], c3 = cnt3[a][x];
      S.nisect_g[ax] = c3;
      S.nisect_gt[ax] = c2;
      S.idx_in_g[ax] = c2 ? S.n_in_g : -1;
      S.n_in_g += c2;
      S.idx_out_g[ax] = c3 ? S.n_out_g : -1;
      S.n_out_g += c3;
      S.idx_in_gt[ax] = c3 ? S.n_in_gt : -1;
      S.n_in_gt += c3;
      S.idx_out_gt[ax] = c2 ? S.n_out_gt : -1;
      S.n_out_gt += c2;
    }
  // Distances and crossing coordinates in sparse order.  lab2/lab3 are sorted by
  // column then ascending y; gammaTilde walks each column downward.
  S.dist_in_g.resize(S.n_in_g);
  S.dist_out_g.resize(S.n_out_g);
  S.dist_in_gt.resize(S.n_in_gt);
  S.dist_out_gt.resize(S.n_out_gt);
  S.coord_g.resize(S.n_out_g);
  S.coord_gt.resize(S.n_out_gt);
  std::vector<std::vector<int>> first2(na), first3(na);
  for (int a = 0; a < na; ++a) {
    first2[a].assign(n1 + 1, 0);
    first3[a].assign(n1 + 1, 0);
    for (int x = 0; x < n1; ++x) {
      first2[a][x + 1] = first2[a][x] + cnt2[a][x];
      first3[a][x + 1] = first3[a][x] + cnt3[a][x];
    }
    for (int x = 0; x < n1; ++x) {
      const size_t ax = (size_t)a * n1 + x;
      for (int k = 0; k < cnt2[a][x]; ++k) {
        const BoundaryNode &bn = lab2[a][first2[a][x] + k];
        S.dist_in_g[S.idx_in_g[ax] + k] = bn.dist;
        const BoundaryNode &bd = lab2[a][first2[a][x] + cnt2[a][x] - 1 - k];
        S.dist_out_gt[S.idx_out_gt[ax] + k] = bd.dist;
        S.coord_gt[S.idx_out_gt[ax] + k] = bd.y;
      }
      for (int k = 0; k < cnt3[a][x]; ++k) {
        const BoundaryNode &bn = lab3[a][first3[a][x] + k];
        S.dist_out_g[S.idx_out_g[ax] + k] = bn.dist;
        S.coord_g[S.idx_out_g[ax] + k] = bn.y;
        const BoundaryNode &bd = lab3[a][first3[a][x] + cnt3[a][x] - 1 - k];
        S.dist_in_gt[S.idx_in_gt[ax] + k] = bd.dist;
      }
    }
  }
  // Trajectory boxes, BoundaryStorage.h:265-350.
  S.x0.assign(na, 0);
  S.x1.assign(na, 0);
  S.y0.assign(na, 0);
  S.y1.assign(na, 0);
  for (int a = 0; a < na; ++a) {
    int xs = 0;
    for (int i = 0; i < n1; ++i)
      if (S.idx_in_g[(size_t)a * n1 + i] > -1) {
        xs = i;
        break;
      }
    int xe = xs;
    for (int i = n1 - 1; i >= xs; --i)
      if (S.idx_in_g[(size_t)a * n1 + i] > -1) {
        xe = i;
        break;
      }
    int ys = n1 - 1, ye = 0;
    for (int i = xs; i <= xe; ++i) {
      const int lo = S.col_lo[(size_t)a * n1 + i], hi = S.col_hi[(size_t)a * n1 + i];
      if (lo >= 0) {
        ys = std::min(ys, lo);
        ye = std::max(ye, hi);
      }
    }
    S.x0[a] = xs;
    S.x1[a] = xe;
    S.y0[a] = ys;
    S.y1[a] = ye;
  }

  // Specular boundary condition gather tables,
  // BoundaryConditionSpecular.h:112-243,245-358,361-486.
  const double coff = (double)(n1 - 1) * 0.5;
  auto interpolate = [&](int xi, int yi, double sysang, double rpx, double rpy, double bdist,
                         int direction, const std::vector<int> &sout,
                         const std::vector<int> &nis, const std::vector<int> &crd, int *src,
                         double *wt, double &wsum) {
    double mx, my;
    rotate(sysang, rpx, rpy, mx, my);
    // FermiSurface::getFractionalAngleIndex (FermiSurface.h:160-184).
    const double ox = S.p_off_x, oy = S.p_off_y;
    const double kx = wrap_range(mx, ox - M_PI, ox + M_PI);
    const double ky = wrap_range(my, oy - M_PI, oy + M_PI);
    const double ph = wrap_range(std::atan2(ky - oy, kx - ox) - 0.5 * M_PI, 0.0, 2.0 * M_PI);
    const double fai = (double)na * ph / (2.0 * M_PI);
    const int ia[2] = {wrap_int((int)fai, 0, na), wrap_int((int)fai + 1, 0, na)};
    const double rot_ang[2] = {sysang - S.theta[ia[0]], sysang - S.theta[ia[1]]};
    const double frac = fai - std::floor(fai);
    const double aw[2] = {1.0 - frac, frac};
    const double bpx = (double)xi - coff;
    const double bpy = (double)yi - (double)sgn((double)direction) * bdist - coff;
    wsum = 0.0;
    for (int r = 0; r < 2; ++r) {
      double rx, ry;
      rotate(rot_ang[r], bpx, bpy, rx, ry);
      rx += coff;
      ry += coff;
      const int pidx[2] = {(int)rx, (int)rx + 1};
      const double pf = rx - std::floor(rx);
      const double pw[2] = {1.0 - pf, pf};
      for (int pt = 0; pt < 2; ++pt) {
        const int slot = r * 2 + pt;
        src[slot] = -1;
        wt[slot] = 0.0;
        if (pidx[pt] < 0 || pidx[pt] >= n1) continue;  // outside the frame grid
        const size_t some = (size_t)ia[r] * n1 + pidx[pt];
        int isect = 0;
        double mind = 1e6;
        for (int i = 0; i < nis[some]; ++i) {
          const double dy = std::fabs((double)crd[i + sout[some]] - ry);
          if (dy < mind) {
            isect = i;
            mind = dy;
          }
        }
        const int base = sout[some] + isect;
        if (base >= 0) {
          src[slot] = base;
          wt[slot] = pw[pt] * aw[r];
          wsum += wt[slot];
        }
      }
    }
  };
  for (int dir = 0; dir < 2; ++dir) {
    const bool is_g = dir == 0;
    BcTable &T = is_g ? S.bc_g : S.bc_gt;
    const int nin = is_g ? S.n_in_g : S.n_in_gt;
    T.src.assign((size_t)4 * nin, -1);
    T.w.assign((size_t)4 * nin, 0.0);
    T.wsum.assign(nin, 0.0);
    const std::vector<int> &sin_ = is_g ? S.idx_in_g : S.idx_in_gt;
    const std::vector<int> &sout = is_g ? S.idx_out_g : S.idx_out_gt;
    const std::vector<int> &nis = is_g ? S.nisect_g : S.nisect_gt;
    const std::vector<int> &crd = is_g ? S.coord_g : S.coord_gt;
    const int direction = is_g ? 1 : -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int a = 0; a < na; ++a) {
      const double sa = S.theta[a];
      double px, py;
      rotate(-sa, S.px[a], S.py[a], px, py);  // Fermi momentum in the frame
      const std::vector<BoundaryNode> &nodes = is_g ? lab2[a] : lab3[a];
      const std::vector<int> &first = is_g ? first2[a] : first3[a];
      const std::vector<int> &cnt = is_g ? cnt2[a] : cnt3[a];
      for (int x = 0; x < n1; ++x) {
        for (int k = 0; k < cnt[x]; ++k) {
          // gamma walks up (k-th entry is the k-th node in ascending y);
          // gammaTilde walks down.
          const BoundaryNode &bn = is_g ? nodes[first[x] + k] : nodes[first[x] + cnt[x] - 1 - k];
          const int kin = sin_[(size_t)a * n1 + x] + k;
          const double td = 2.0 * (px * bn.nx + py * bn.ny);
          const double rpx = px - td * bn.nx, rpy = py - td * bn.ny;
          int src[4];
          double wt[4], ws;
          interpolate(bn.x, bn.y, sa, rpx, rpy, bn.dist, direction, sout, nis, crd, src, wt, ws);
          if (ws < 1e-7)
            interpolate(bn.x, bn.y, sa, -px, -py, bn.dist, direction, sout, nis, crd, src, wt, ws);
          for (int s = 0; s < 4; ++s) {
            T.src[(size_t)4 * kin + s] = src[s];
            T.w[(size_t)4 * kin + s] = wt[s];
          }
          T.wsum[kin] = ws;
        }
      }
    }
  }

  // Frame extension (halo) tables, concatenated over angles.
  S.halo_angle_off.assign(na + 1, 0);
  S.halo_src_off.assign(1, 0);
  for (int a = 0; a < na; ++a) {
    const int base = (int)S.halo_src.size();
    for (size_t k = 0; k < h_site[a].size(); ++k) {
      S.halo_site.push_back(h_site[a][k]);
      S.halo_src_off.push_back(base + h_off[a][k]);
    }
    S.halo_src.insert(S.halo_src.end(), h_src[a].begin(), h_src[a].end());
    S.halo_angle_off[a + 1] = (int)S.halo_site.size();
  }

  // Poisson filters, ComputeVectorPotential.h:212-416 (analytical elements).
  if (S.lambda > 0.0) {
    const int n = n0;
    std::vector<double> Q((size_t)n * n);
    auto alpha = [](int a, int b) {
      const double dist = std::hypot((double)a, (double)b);
      return (double)(a * b) * (2.0 * std::log(dist) - std::log(2.0));
    };
    auto beta = [](int a, int b) {
      const double f = 0.5 * (double)((2 - a + b) * (a + b) - 2);
      return f * std::atan((double)a / (double)b);
    };
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        const int iv[2] = {-i, i}, jv[2] = {-j, j};
        double sum = 0.0;
        for (int jj : jv) {
          const int b = 1 + 2 * jj;
          for (int ii : iv) {
            const int a = 1 + 2 * ii;
            sum += alpha(a, b) + beta(a, b) + beta(b, a);
          }
        }
        Q[(size_t)i * n + j] = sum * 0.25;
      }
    std::vector<double> Qs((size_t)n * n);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j)
        Qs[(size_t)i * n + j] = 0.5 * (Q[(size_t)i * n + j] + Q[(size_t)j * n + i]);
    const double sc = 1.0 / (4.0 * M_PI);
    double meanQ = 0.0;
    for (double &v : Qs) {
      v *= sc;
      meanQ += v;
    }
    meanQ /= (double)((size_t)n * n);
    double C = (2.0 * std::log(S.h) - std::log(2.0) - 3.0) * sc;
    for (double &v : Qs) v -= meanQ;
    C += meanQ;
    std::vector<double> w;
    symmetric_eigen(n, Qs, w);
    double maxabs = 0.0;
    for (double v : w) maxabs = std::max(maxabs, std::fabs(v));
    S.vp_scale = 0.5 * (maxabs + std::fabs(C));
    auto add_filter = [&](const double *vec, double val, bool ones) {
      const double sq = std::sqrt(std::fabs(val) / S.vp_scale);
      for (int i = -n + 1; i < n; ++i) S.filters.push_back((ones ? 1.0 : vec[std::abs(i)]) * sq);
      S.filter_pos.push_back(val > 0.0 ? 1 : 0);
      S.n_filters++;
    };
    if (std::fabs(C) > 0.0) add_filter(nullptr, C, true);
    std::vector<int> ord(n);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(),
                     [&](int x, int y) { return std::fabs(w[x]) > std::fabs(w[y]); });
    double norm2 = 0.0;
    for (double v : w) norm2 += v * v;
    double partial = 0.0;
    for (int k : ord) {
      add_filter(&Qs[(size_t)k * n], w[k], false);
      partial += w[k] * w[k];
      const double e2 = 1.0 - partial / norm2;
      if (std::sqrt(std::max(e2, 0.0)) < S.vp_max_error) break;
    }
  }
  return std::string();
}

std::string build_ldos_setup(const std::string &simulation_json, const std::string &postprocess_json,
                             HostSetup &S) {
  JsonValue pp;
  try {
    pp = JsonValue::parse(postprocess_json);
  } catch (const std::exception &ex) {
    return std::string("postprocess config: ") + ex.what();
  }
  const JsonValue &sp = pp["spectroscopy"], &num = pp["numerics"];
  if (!sp.is_object() || !num.is_object())
    return "postprocess config: 'spectroscopy' and 'numerics' are required";
  // src/postprocess.cu:152-186: angles, criterion and norm come from the
  // postprocess configuration, everything else from the loaded simulation.
  SetupOverrides ov;
  ov.n_angles = num["num_fermi_momenta"].as_int(-1);
  ov.conv_crit = num["convergence_criterion"].as_double(-1.0);
  const std::string norm = num["norm"].as_string("l2");
  if (norm == "l1") ov.norm = NORM_L1;
  else if (norm == "l2") ov.norm = NORM_L2;
  else if (norm == "linf") ov.norm = NORM_LINF;
  else return "postprocess config: norm type '" + norm + "' not understood";
  if (ov.n_angles < 1) return "postprocess config: num_fermi_momenta must be positive";
  const std::string e = build_setup(simulation_json, S, &ov);
  if (!e.empty()) return e;
  S.burnin = num["num_iterations_burnin"].as_int(0);
  S.it_min = num["num_iterations_min"].as_int(0);
  S.it_max = num["num_iterations_max"].as_int(-1);
  // IntegrationIteratorKeldysh::initEnergies / initIterators
  // (IntegrationIteratorKeldysh.h:91-160).
  const double emin = sp["energy_min"].as_double(), emax = sp["energy_max"].as_double();
  const int ne = sp["num_energies"].as_int(0);
  const double delta = sp["energy_broadening"].as_double();
  if (ne < 1) return "postprocess config: num_energies must be positive";
  if (!(delta > 0.0)) return "postprocess config: energy_broadening must be positive";
  const double step = ne > 1 ? (emax - emin) / (double)(ne - 1) : 0.0;
  S.ldos_energies.resize(ne);
  for (int i = 0; i < ne; ++i) S.ldos_energies[i] = emin + step * (double)i;
  S.ldos_broadening = delta;
  const int per = num["num_energies_per_block"].as_int(0);
  S.ldos_block = per < 1 ? ne : std::min(per, ne);
  S.ldos_n_blocks = (ne + S.ldos_block - 1) / S.ldos_block;
  S.keldysh = 1;
  S.ne = S.ldos_block;
  S.e_im.assign(S.ne, delta);
  S.residues.assign(S.ne, 0.0);
  ldos_block_energies(S, 0, S.e_re);
  return std::string();
}

void ldos_block_energies(const HostSetup &S, int b, std::vector<double> &e_re) {
  const int n = (int)S.ldos_energies.size();
  e_re.resize(S.ldos_block);
  for (int i = 0; i < S.ldos_block; ++i)
    e_re[i] = S.ldos_energies[std::min(b * S.ldos_block + i, n - 1)];
}

}  // namespace scb

// ------------------------------------------------------ host-only probes --
// These run build_setup alone (no CUDA) so the static tables can be checked on
// a machine without a GPU.  See include/scb200.h.
#include "../../include/scb200.h"

struct sc_setup {
  scb::HostSetup S;
};

namespace {
thread_local std::string g_setup_error;
}

extern "C" {

int sc_setup_create(const char *config_json, sc_setup **out) {
  if (!config_json || !out) return SC_ERR_ARG;
  *out = nullptr;
  sc_setup *s = new sc_setup();
  std::string e;
  try {
    e = scb::build_setup(config_json, s->S);
  } catch (const std::exception &ex) {
    e = ex.what();
  }
  if (!e.empty()) {
    g_setup_error = e;
    delete s;
    return SC_ERR_ARG;
  }
  *out = s;
  return SC_OK;
}

const char *sc_setup_last_error(void) { return g_setup_error.c_str(); }

int sc_setup_destroy(sc_setup *s) {
  delete s;
  return SC_OK;
}

int sc_setup_dims(const sc_setup *s, int *n0, int *n1, int *n_angles, int *n_energies, int *n_comp) {
  if (!s) return SC_ERR_ARG;
  if (n0) *n0 = s->S.n0;
  if (n1) *n1 = s->S.n1;
  if (n_angles) *n_angles = s->S.n_angles;
  if (n_energies) *n_energies = s->S.ne;
  if (n_comp) *n_comp = s->S.nc;
  return SC_OK;
}

int sc_setup_energies(const sc_setup *s, double *e_im, double *residues) {
  if (!s) return SC_ERR_ARG;
  for (int i = 0; i < s->S.ne; ++i) {
    if (e_im) e_im[i] = s->S.e_im[i];
    if (residues) residues[i] = s->S.residues[i];
  }
  return SC_OK;
}

int sc_setup_fermi_surface(const sc_setup *s, double *table, double *info) {
  if (!s) return SC_ERR_ARG;
  const scb::HostSetup &S = s->S;
  const int na = S.n_angles;
  if (table) {
    const std::vector<double> *cols[8] = {&S.phi, &S.theta, &S.px, &S.py, &S.vx, &S.vy, &S.weight, &S.step};
    for (int r = 0; r < 8; ++r)
      for (int k = 0; k < na; ++k) table[(size_t)r * na + k] = (*cols[r])[k];
  }
  if (info) {
    info[0] = S.avg_fermi_momentum;
    info[1] = S.avg_fermi_speed;
    info[2] = S.p_off_x;
    info[3] = S.p_off_y;
  }
  return SC_OK;
}

int sc_setup_frame(const sc_setup *s, int angle, signed char *labels, int *box) {
  if (!s || angle < 0 || angle >= s->S.n_angles) return SC_ERR_ARG;
  const size_t nn1 = (size_t)s->S.n1 * s->S.n1;
  if (labels) std::memcpy(labels, &s->S.labels[(size_t)angle * nn1], nn1);
  if (box) {
    box[0] = s->S.x0[angle];
    box[1] = s->S.x1[angle];
    box[2] = s->S.y0[angle];
    box[3] = s->S.y1[angle];
  }
  return SC_OK;
}

int sc_setup_domain(const sc_setup *s, signed char *domain) {
  if (!s || !domain) return SC_ERR_ARG;
  std::memcpy(domain, s->S.domain_ref.data(), s->S.domain_ref.size());
  return SC_OK;
}

int sc_setup_boundary_sizes(const sc_setup *s, int *sizes) {
  if (!s || !sizes) return SC_ERR_ARG;
  sizes[0] = s->S.n_in_g;
  sizes[1] = s->S.n_out_g;
  sizes[2] = s->S.n_in_gt;
  sizes[3] = s->S.n_out_gt;
  return SC_OK;
}

int sc_setup_filters(const sc_setup *s, int *n_filters, double *filters, int *positive,
                     double *scale) {
  if (!s) return SC_ERR_ARG;
  if (n_filters) *n_filters = s->S.n_filters;
  if (filters && !s->S.filters.empty())
    std::memcpy(filters, s->S.filters.data(), s->S.filters.size() * sizeof(double));
  if (positive)
    for (int k = 0; k < s->S.n_filters; ++k) positive[k] = s->S.filter_pos[k];
  if (scale) *scale = s->S.vp_scale;
  return SC_OK;
}

int sc_setup_site_updates(const sc_setup *s, long long *per_iteration) {
  if (!s || !per_iteration) return SC_ERR_ARG;
  *per_iteration = s->S.site_updates_per_iteration();
  return SC_OK;
}

int sc_bulk_order_parameter_s_wave(double temperature, double convergence_criterion,
                                   int max_iterations, double energy_cutoff, double *out) {
  if (!out || !(temperature >= 0.0) || !(energy_cutoff > 0.0) || max_iterations < 0 ||
      !(convergence_criterion > 0.0))
    return SC_ERR_ARG;
  *out = scb::bulk_s_wave(temperature, convergence_criterion, max_iterations, energy_cutoff);
  return SC_OK;
}

int sc_bulk_free_energy_s_wave(double temperature, double order_parameter, double energy_cutoff,
                               double *out) {
  if (!out || !(temperature > 0.0) || !(energy_cutoff > 0.0)) return SC_ERR_ARG;
  *out = scb::bulk_free_energy_s_wave(temperature, order_parameter, energy_cutoff);
  return SC_OK;
}

int sc_bulk_yoshida_s_wave(double temperature, double order_parameter, double energy_cutoff,
                           double *out) {
  if (!out || !(temperature >= 0.0) || !(energy_cutoff > 0.0)) return SC_ERR_ARG;
  *out = scb::bulk_yoshida_s_wave(temperature, order_parameter, energy_cutoff);
  return SC_OK;
}

int sc_grid_extend(int n, const signed char *domain, int n_fields, double *values) {
  if (n < 1 || !domain || n_fields < 1 || !values) return SC_ERR_ARG;
  // extendValuesAtBoundary_kernel (domain_ops.h:11-69): a site outside the
  // grain with grain sites in its 5x5 window takes the mean of the nearest
  // of them (squared distance, ties averaged); all reads from the input.
  const size_t nn = (size_t)n * n;
  std::vector<double> src(values, values + nn * n_fields);
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x) {
      if (domain[(size_t)y * n + x] > 0) continue;
      int best = 1000, cnt = 0;
      std::vector<size_t> near;
      for (int ky = std::max(y - 2, 0); ky <= std::min(y + 2, n - 1); ++ky)
        for (int kx = std::max(x - 2, 0); kx <= std::min(x + 2, n - 1); ++kx) {
          if (domain[(size_t)ky * n + kx] <= 0) continue;
          const int d2 = (x - kx) * (x - kx) + (y - ky) * (y - ky);
          if (d2 < best) {
            best = d2;
            near.clear();
            cnt = 0;
          }
          if (d2 == best) {
            near.push_back((size_t)ky * n + kx);
            ++cnt;
          }
        }
      if (!cnt) continue;
      for (int f = 0; f < n_fields; ++f) {
        double v = 0.0;
        for (size_t k : near) v += src[f * nn + k];
        values[f * nn + (size_t)y * n + x] = v / (double)cnt;
      }
    }
  return SC_OK;
}

int sc_grid_resample(int n_old, int n_new, int n_fields, const double *src, double *dst) {
  const int margin = 3;  // constants::GRAIN_SIZE_MARGIN (defines.h:25)
  if (n_old <= 2 * margin + 1 || n_new <= 2 * margin + 1 || n_fields < 1 || !src || !dst) return SC_ERR_ARG;
  // resample_kernel (GridFunctions_GPU.h:547-600): bilinear interpolation
  // with the safety margin mapped onto itself.  Sites whose interpolation
  // would reach past the old lattice (only in the margin when shrinking) read
  // the nearest edge value instead.
  const double sx = (double)(n_old - 1 - 2 * margin) / (double)(n_new - 1 - 2 * margin);
  auto clampi = [&](int i) { return std::min(std::max(i, 0), n_old - 1); };
  for (int z = 0; z < n_fields; ++z)
    for (int y = 0; y < n_new; ++y)
      for (int x = 0; x < n_new; ++x) {
        const double xo = sx * (double)(x - margin) + margin, yo = sx * (double)(y - margin) + margin;
        const int xf = (int)xo, yf = (int)yo;
        const double fx = xo - (double)xf, fy = yo - (double)yf;
        const int xn = x < n_new - 1 ? 1 : 0, yn = y < n_new - 1 ? 1 : 0;
        const double *p = src + (size_t)z * n_old * n_old;
        auto at = [&](int yy, int xx) { return p[(size_t)clampi(yy) * n_old + clampi(xx)]; };
        const double x1 = (1.0 - fx) * at(yf, xf) + fx * at(yf, xf + xn);
        const double x2 = (1.0 - fx) * at(yf + yn, xf) + fx * at(yf + yn, xf + xn);
        dst[((size_t)z * n_new + y) * n_new + x] = (1.0 - fy) * x1 + fy * x2;
      }
  return SC_OK;
}

}  // extern "C"

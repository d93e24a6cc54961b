// Checker-side harness around the reference's own header code (test
// infrastructure only; nothing in the product links or loads it).
//
// The reference library is header-only C++.  The parts of its hot path that
// need no third-party library -- the Riccati step algebra
// (riccati/RiccatiSolutions.h), the local Green functions (green/LocalGreens.h),
// the bulk s-wave thermodynamics (order_parameter/OrderParameterBulk.h), the
// circular Fermi surface's angles and weights (fermi_surface/FermiSurface.h)
// and the lattice sizing and Ozaki pole count (Parameters.h) -- compile with
// g++ on the reference's CPU backend (Thrust on OpenMP, as the reference's
// CMakeLists.txt:192-214 configures it).  This file instantiates them and
// exports plain C entry points, so the tests can hold the oracle's
// restatement of those functions against the reference's own code.
// Everything else on the path (geometry, boundary condition, compute objects,
// Poisson solve, accelerators) includes Armadillo, jsoncpp or LAPACK, which
// the reference does not vendor; it is not built here.
//
// Built by oracle.build_ref() into oracle/_ref/ from the headers where they lie.
#include "conga/Parameters.h"
#include "conga/fermi_surface/FermiSurfaceCircle.h"
#include "conga/green/LocalGreens.h"
#include "conga/order_parameter/OrderParameterBulk.h"
#include "conga/riccati/RiccatiSolutions.h"

#include <thrust/complex.h>

#include <cstring>
#include <new>

namespace {
using C = thrust::complex<double>;

// Parameters<double> over zeroed storage: its default constructor leaves the
// members unset, and each setter recomputes from the others (an unset energy
// cutoff or temperature could send the pole count's fallback loop far out).
struct ZeroedParameters {
  alignas(conga::Parameters<double>) unsigned char buf[sizeof(conga::Parameters<double>)];
  conga::Parameters<double> *p;
  ZeroedParameters() {
    std::memset(buf, 0, sizeof(buf));
    p = new (buf) conga::Parameters<double>();
  }
  ~ZeroedParameters() { p->~Parameters<double>(); }
};
}  // namespace

extern "C" {

// riccati::computeStep for n sites: delta, energy, g0 as (re, im) pairs, h[n].
void ref_riccati_step(int n, const double *delta, const double *energy, const double *g0,
                      const double *h, double *out) {
  for (int i = 0; i < n; ++i) {
    const C r = conga::riccati::computeStep<double>(C(delta[2 * i], delta[2 * i + 1]),
                                                    C(energy[2 * i], energy[2 * i + 1]),
                                                    C(g0[2 * i], g0[2 * i + 1]), h[i]);
    out[2 * i] = r.real();
    out[2 * i + 1] = r.imag();
  }
}

// riccati::computeHomogeneous: out[4 i ..] = gamma, gammaTilde.
void ref_homogeneous(int n, const double *delta, const double *energy, double *out) {
  for (int i = 0; i < n; ++i) {
    C g, gt;
    conga::riccati::computeHomogeneous<double>(C(delta[2 * i], delta[2 * i + 1]),
                                               C(energy[2 * i], energy[2 * i + 1]), g, gt);
    out[4 * i] = g.real();
    out[4 * i + 1] = g.imag();
    out[4 * i + 2] = gt.real();
    out[4 * i + 3] = gt.imag();
  }
}

// Greens::compute (g) and Greens_Delta::compute (f + f~*): out[4 i ..] = g, f + f~*.
void ref_greens(int n, const double *gamma, const double *gamma_tilde, double *out) {
  for (int i = 0; i < n; ++i) {
    const C g(gamma[2 * i], gamma[2 * i + 1]), gt(gamma_tilde[2 * i], gamma_tilde[2 * i + 1]);
    const C gg = conga::Greens<double>::compute(g, gt);
    const C fd = conga::Greens_Delta<double>::compute(g, gt);
    out[4 * i] = gg.real();
    out[4 * i + 1] = gg.imag();
    out[4 * i + 2] = fd.real();
    out[4 * i + 3] = fd.imag();
  }
}

double ref_bulk_gap(double temperature, double criterion, int max_iterations, double cutoff) {
  return conga::computeOrderParameterBulkSWave<double>(temperature, criterion, max_iterations, cutoff);
}

double ref_bulk_free_energy(double temperature, double order_parameter, double cutoff) {
  return conga::computeFreeEnergyBulkSWave<double>(temperature, order_parameter, cutoff);
}

double ref_bulk_yoshida(double temperature, double order_parameter, double cutoff) {
  return conga::computeYoshidaBulkSWave<double>(temperature, order_parameter, cutoff);
}

// FermiSurfaceCircle<double> with n angles: polar angle phi, system angle,
// Fermi velocity (x, y) and integrand factor (angle weight / n) of every angle.
void ref_fermi_circle(int n, double *phi, double *system_angle, double *vx, double *vy,
                      double *integrand_factor) {
  conga::FermiSurfaceCircle<double> fs;
  fs.initialize(n);
  for (int k = 0; k < n; ++k) {
    phi[k] = fs.getPolarAngle(k);
    system_angle[k] = fs.getSystemAngle(k);
    fs.getFermiVelocity(k, vx[k], vy[k]);
    integrand_factor[k] = fs.getIntegrandFactor(k);
  }
}

// Parameters<double>: lattice sizes of a grain of the given width and
// resolution, and the number of Ozaki poles at (temperature, cutoff).
void ref_lattice(double grain_width, double points_per_xi, int *n0, int *n1, double *grain_fraction) {
  ZeroedParameters z;
  z.p->setPointsPerCoherenceLength(points_per_xi);
  z.p->setGrainWidth(grain_width);
  *n0 = z.p->getGridResolutionBase();
  *n1 = z.p->getGridResolutionCoherence();
  *grain_fraction = z.p->getGrainFraction();
}

int ref_num_ozaki(double temperature, double cutoff) {
  ZeroedParameters z;
  z.p->setTemperature(temperature);
  z.p->setEnergyCutoff(cutoff);
  return z.p->getNumOzakiEnergies();
}

}  // extern "C"

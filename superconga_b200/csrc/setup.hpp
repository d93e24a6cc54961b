// Host-side setup of a SuperConga self-consistency context for the B200 path.
//
// Everything here runs once per context and is static during the iteration:
// lattice sizes, Ozaki poles, Fermi-surface tables, the grain rasterised into
// every trajectory frame, the sparse boundary-storage indexing, the specular
// boundary-condition gather tables, the frame extension (halo) tables and the
// separable Poisson filters.  The reference recomputes the per-angle geometry
// inside every iteration (IntegrationIteratorOzaki.h:355-388); here it is
// built once and kept in HBM.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace scb {

enum Norm { NORM_L1 = 0, NORM_L2 = 1, NORM_LINF = 2 };
enum Gauge { GAUGE_LANDAU = 0, GAUGE_SYMMETRIC = 1, GAUGE_SOLENOID = 2 };
enum Accel { ACC_CONGACC = 0, ACC_PICARD = 1, ACC_POLYAK = 2, ACC_BB = 3, ACC_ANDERSON = 4 };

struct GeomComp {
  int type = 0;  // 0 disc, 1 polygon
  bool add = true;
  double radius = 0, cx = 0, cy = 0;  // disc, already scaled by the grain fraction
  std::vector<double> vx, vy;         // polygon, already scaled by the grain fraction
};

struct AccelParams {
  int kind = ACC_CONGACC;
  double step_size = 0.5, step_size_factor = 1.234, cos_similarity_min = 0.7;
  double step_size_max = 100.0, step_size_min = 0.001, drag = 0.5;
  int rank = 4;
};

// Gather table of the specular boundary condition: incoming boundary value k
// (energy-independent base index) is sum_s w[4k+s] * out[src[4k+s]] / wsum[k].
struct BcTable {
  std::vector<int> src;      // 4 per incoming node, -1 = unused slot
  std::vector<double> w;     // 4 per incoming node
  std::vector<double> wsum;  // 1 per incoming node
};

struct HostSetup {
  // Parameters (Parameters.h:422-458, 380-420).
  int n0 = 0, n1 = 0, n_angles = 0, ne = 0, nc = 0;
  double h = 0, grain_fraction = 0, grain_width = 0, temperature = 0;
  double flux_quanta = 0, lambda = -1, conv_crit = 1e-6, vp_max_error = 1e-6;
  int charge_sign = -1, norm = NORM_L2, gauge = GAUGE_SYMMETRIC;
  double crystal_rot = 0;
  int burnin = 0, it_min = 0, it_max = -1;
  AccelParams acc;
  std::vector<GeomComp> geom;

  // Energies of the sweep, e = e_re + i e_im, and their residues.  The
  // self-consistency path sums Ozaki poles (e_re = 0); the LDOS path takes one
  // block of real energies with a common broadening (e_im = delta, residues 0).
  std::vector<double> e_re, e_im, residues;

  // LDOS postprocess (src/postprocess.cu:140-160,218-224;
  // IntegrationIteratorKeldysh.h:91-170): all real energies and the block size.
  int keldysh = 0;
  std::vector<double> ldos_energies;
  double ldos_broadening = 0.0;
  int ldos_block = 0, ldos_n_blocks = 0;

  // Order-parameter components (ordered as the reference: dx2-y2, dxy, g, s).
  std::vector<int> sym;                    // 0 s, 1 dx2-y2, 2 dxy, 3 g
  std::vector<std::string> sym_name;
  std::vector<double> tc, norm_factor, coupling;

  // Fermi surface model: the circle of FermiSurfaceCircle.h (default) or the
  // square-lattice tight-binding surface of FermiSurfaceTightBinding.h with
  // the dispersion of DispersionTightBinding.h (nearest-neighbour hopping 1).
  int fs_tight_binding = 0;
  double tb_hopping_nnn = 0.0, tb_hopping_nnnn = 0.0, tb_chemical_potential = 1.0;
  double p_off_x = 0.0, p_off_y = 0.0;                 // momentum origin (0,0) or (pi,pi)
  double avg_fermi_speed = 1.0, avg_fermi_momentum = 1.0;  // tight binding only

  // Fermi surface, per angle.  phi: polar angle of the momentum; theta: system
  // angle (velocity angle - pi/2); px, py: Fermi momentum; vx, vy: Fermi
  // velocity (normalised by its Fermi-surface average); speed = |v|;
  // step = h / speed, the Riccati step (RiccatiSolverConfined.h:525-527).
  std::vector<double> theta, phi, vx, vy, weight;  // weight = integrand factor
  std::vector<double> px, py, speed, step;
  std::vector<double> eta;                         // [a * nc + c]
  // Rotation coefficients (single-precision trigonometry promoted to double,
  // GridFunctions_GPU.h:436-489): cD/sD order parameter into the frame, cA/sA
  // vector potential into the frame, cB/sB frame back to the reference grid.
  // cE/sE: double-precision rotation of the external potential coordinates.
  std::vector<double> cD, sD, cA, sA, cB, sB, cE, sE;

  // Geometry.
  std::vector<uint8_t> domain_ref;  // n0 * n0
  int n_grain = 0;
  double area = 0;
  std::vector<uint8_t> labels;      // n_angles * n1 * n1, frame labels 0..3
  std::vector<int> x0, x1, y0, y1;  // per-angle trajectory box
  std::vector<int> col_lo, col_hi;  // per (a, x): first / last row with label > 0, -1 if none

  // Sparse boundary storage (BoundaryStorage.h:157-169): base index per (a, x).
  std::vector<int> idx_in_g, idx_out_g, idx_in_gt, idx_out_gt;
  int n_in_g = 0, n_out_g = 0, n_in_gt = 0, n_out_gt = 0;
  // |boundary distance| of every entry / exit node, in sparse order.
  std::vector<double> dist_in_g, dist_out_g, dist_in_gt, dist_out_gt;
  // Crossing bookkeeping used by the boundary condition.
  std::vector<int> nisect_g, nisect_gt, coord_g, coord_gt;
  BcTable bc_g, bc_gt;

  // Frame extension tables (domain_ops.h:11-69): for every label-0 site with a
  // grain site in its 5x5 window, the sources of the nearest-neighbour average.
  std::vector<int> halo_site;    // frame site index y*n1+x
  std::vector<int> halo_src_off; // offset into halo_src (size n_halo + 1)
  std::vector<int> halo_src;     // frame site indices
  std::vector<int> halo_angle_off;  // per angle: first halo entry (size n_angles + 1)
  // Reference-grid extension table (same rule, reference domain).
  std::vector<int> rext_site, rext_src_off, rext_src;

  // Poisson filters (ComputeVectorPotential.h:212-416).
  int n_filters = 0;
  std::vector<double> filters;  // n_filters * (2*n0 - 1)
  std::vector<int> filter_pos;
  double vp_scale = 1.0;

  long long site_updates_per_iteration() const;  // 2 * ne * sum_a #{label > 0}
};

// Settings a postprocess configuration takes over from the simulation
// configuration it loads (src/postprocess.cu:152-186).
struct SetupOverrides {
  int n_angles = -1;
  double conv_crit = -1.0;
  int norm = -1;
};

// Parses a reference JSON configuration and builds all static tables.
// Returns an empty string on success, otherwise an error message.
std::string build_setup(const std::string &json, HostSetup &out,
                        const SetupOverrides *ov = nullptr);

// Setup of an LDOS postprocess: the simulation configuration of the loaded run
// plus the postprocess configuration (spectroscopy and numerics sections).
// The sweep energies are those of block 0.
std::string build_ldos_setup(const std::string &simulation_json,
                             const std::string &postprocess_json, HostSetup &out);
// Energies of LDOS block b (a short last block repeats its final energy).
void ldos_block_energies(const HostSetup &S, int b, std::vector<double> &e_re);

// Individual pieces, exposed for tests.
int num_ozaki_poles(double temperature, double cutoff);
void ozaki_poles(int n, double *poles, double *residues);
void symmetric_eigen(int n, std::vector<double> &a, std::vector<double> &w);
double bulk_s_wave(double temperature, double criterion, int max_iterations, double energy_cutoff);
double bulk_free_energy_s_wave(double temperature, double order_parameter, double energy_cutoff);
double bulk_yoshida_s_wave(double temperature, double order_parameter, double energy_cutoff);
// Tight-binding Fermi surface (FermiSurfaceTightBinding.h): fills phi, theta,
// px, py, vx, vy, speed and weight of S for S.n_angles angles.
void tight_binding_surface(HostSetup &S);
// Square-lattice basis functions of a non-circular surface
// (OrderParameterBasis.h:187-213): sym 0 s, 1 dx2-y2, 2 dxy, 3 g.
double lattice_basis(int sym, double px, double py);

}  // namespace scb

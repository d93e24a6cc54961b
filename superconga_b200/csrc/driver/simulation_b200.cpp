// simulation_b200 -- drop-in replacement of the reference's simulation driver
// (src/simulation.cu) on the B200 engine.
//
//   simulation_b200 <config.json>
//
// Reads the reference's JSON configuration, builds one engine context through
// the C ABI, sets the initial order parameter (from misc.load_path or the
// reference's initial-guess rule with a fixed seed), runs the burn-in and the
// self-consistency iterations (run_simulation.h:124-187) and writes the
// reference's output files into misc.save_path:
//   domain.csv, order_parameter.csv, current_density.csv, vector_potential.csv,
//   magnetic_flux_density.csv (CSVGridWriter.h layout, 8 significant digits),
//   simulation_config.json, simulation_results.json, internal_parameters.json
//   (SimulationWriter.h:57-246) and simulation_convergence.csv
//   (CSVSimulationIterationWriter.h:42-101).
// The optional key b200.precision selects "fp64" (default) or "mixed".
// Exit status EXIT_SUCCESS / EXIT_FAILURE as the reference driver.
#include <random>

#include "common.hpp"
#include "scb200.h"

using namespace drv;

int main(int argc, char *argv[]) {
  if (argc < 2) return fail("Please provide a config file.");
  std::ifstream cfg_in(argv[1]);
  if (!cfg_in.good()) return fail(std::string("Could not find/open config file '") + argv[1] + "'.");
  std::stringstream buf;
  buf << cfg_in.rdbuf();
  const std::string text = buf.str();
  scb::JsonValue cfg;
  try {
    cfg = scb::JsonValue::parse(text);
  } catch (const std::exception &e) {
    return fail(std::string("config: ") + e.what());
  }
  const bool verbose = cfg["misc"]["verbose"].as_bool();
  const std::string prec = cfg["b200"]["precision"].as_string("fp64");
  const int mode = prec == "mixed" ? SC_MODE_MIXED : SC_MODE_FP64;

  sc_ctx *ctx = nullptr;
  if (sc_create(text.c_str(), mode, &ctx) != SC_OK) return fail(sc_last_error(nullptr));
  int n0, n1, na, ne, nc;
  sc_get_dims(ctx, &n0, &n1, &na, &ne, &nc);
  const size_t nn = (size_t)n0 * n0;
  const double lambda = cfg["physics"]["penetration_depth"].as_double(-1.0);
  const double temperature = cfg["physics"]["temperature"].as_double();
  const double h = 1.0 / cfg["numerics"]["points_per_coherence_length"].as_double();
  std::vector<std::string> comps;
  for (const char *s : {"dx2-y2", "dxy", "g", "s"})
    if (cfg["physics"]["order_parameter"].has(s)) comps.push_back(s);

  // Initial state.
  std::vector<double> delta((size_t)nc * 2 * nn, 0.0), avec(2 * nn, 0.0);
  const std::string load = cfg["misc"]["load_path"].as_string();
  if (!load.empty()) {
    const std::string e = load_state(load, comps, n0, lambda, delta, avec);
    if (!e.empty()) return fail(e);
  } else {
    // Initial::perturbedPhaseWindings / Initial::random
    // (OrderParameterInitial.h:186-237, 420-427), with a fixed seed in place of
    // the clock seed.
    std::mt19937_64 rng((unsigned long long)cfg["misc"]["seed"].as_double(0.0));
    std::normal_distribution<double> nd(0.0, 1.0);
    // Vortex centres are mapped as src/simulation.cu:259-275 does:
    // (centre - offset) / (scaling / 2) with the geometry's bounding box.
    double xmin = 1e300, xmax = -1e300, ymin = 1e300, ymax = -1e300;
    const scb::JsonValue &gl = cfg["geometry"];
    for (size_t g = 0; g < gl.size(); ++g) {
      const std::string nm = gl[g].keys()[0];
      const scb::JsonValue &d = gl[g][nm];
      if (!d["add"].as_bool()) continue;
      if (nm == "disc") {
        const double r = d["radius"].as_double(), cx = d["center_x"].as_double(), cy = d["center_y"].as_double();
        xmin = std::min(xmin, cx - r); xmax = std::max(xmax, cx + r);
        ymin = std::min(ymin, cy - r); ymax = std::max(ymax, cy + r);
      } else if (nm == "polygon") {
        for (size_t k = 0; k < d["vertices_x"].size(); ++k) {
          xmin = std::min(xmin, d["vertices_x"][k].as_double()); xmax = std::max(xmax, d["vertices_x"][k].as_double());
          ymin = std::min(ymin, d["vertices_y"][k].as_double()); ymax = std::max(ymax, d["vertices_y"][k].as_double());
        }
      } else {
        const int ned = d["num_edges"].as_int();
        const double step = 2.0 * M_PI / ned, rot = 2.0 * M_PI * d["rotation"].as_double();
        const double rad = d["side_length"].as_double() / std::hypot(std::cos(step) - 1.0, std::sin(step));
        for (int k = 0; k < ned; ++k) {
          const double ang = 0.5 * step + rot + step * k;
          const double vx = d["center_x"].as_double() + rad * std::cos(ang), vy = d["center_y"].as_double() + rad * std::sin(ang);
          xmin = std::min(xmin, vx); xmax = std::max(xmax, vx);
          ymin = std::min(ymin, vy); ymax = std::max(ymax, vy);
        }
      }
    }
    const double scaling = std::max(xmax - xmin, ymax - ymin);
    const double xoff = xmin + 0.5 * (xmax - xmin), yoff = ymin + 0.5 * (ymax - ymin);
    for (int c = 0; c < nc; ++c) {
      const scb::JsonValue &p = cfg["physics"]["order_parameter"][comps[c]];
      // OrderParameterComponent::deltaBulk uses the bare temperature
      // (OrderParameterComponent.h:210-235).
      const double sb = bulk_s_wave(temperature);
      const bool dwave = comps[c] != "s";
      const double db = dwave ? sb * (std::exp(-EULER_GAMMA - 0.5) / std::sqrt(2.0)) / (0.5 * std::exp(-EULER_GAMMA)) : sb;
      const double noise = p["initial_noise_stddev"].as_double(0.0);
      const double shift = 2.0 * M_PI * p["initial_phase_shift"].as_double(0.0);
      const scb::JsonValue &vort = p["vortices"];
      for (int j = 0; j < n0; ++j)
        for (int i = 0; i < n0; ++i) {
          double phase = shift;
          for (size_t v = 0; v < vort.size(); ++v) {
            const double vcx = (vort[v]["center_x"].as_double() - xoff) / (0.5 * scaling);
            const double vcy = (vort[v]["center_y"].as_double() - yoff) / (0.5 * scaling);
            const double x = (double)(2 * i) / (double)(n0 - 1) - 1.0 - vcx;
            const double y = (double)(2 * j) / (double)(n0 - 1) - 1.0 - vcy;
            const double ang = std::hypot(x, y) > 0.0 ? std::atan2(y, x) : 0.0;
            phase += ang * vort[v]["winding_number"].as_double();
          }
          const size_t k = (size_t)j * n0 + i;
          delta[(size_t)(2 * c) * nn + k] = db * std::cos(phase) + noise * nd(rng);
          delta[(size_t)(2 * c + 1) * nn + k] = db * std::sin(phase) + noise * nd(rng);
        }
    }
  }
  if (sc_set_state(ctx, delta.data(), avec.data()) != SC_OK) return fail(sc_last_error(ctx));

  const fs::path save = cfg["misc"]["save_path"].as_string();
  const int save_freq = cfg["misc"]["save_frequency"].as_int(-1);
  const bool save_data = !save.empty() && save_freq != 0;
  std::ofstream conv_csv;
  if (save_data) {
    fs::create_directories(save);
    std::ofstream cj(save / "simulation_config.json");
    dump_json(cj, cfg, 0);
    cj << "\n";
    conv_csv.open(save / "simulation_convergence.csv");
    conv_csv << "iteration,boundary_coherence_residual,order_parameter_residual,"
                "current_density_residual,vector_potential_residual,free_energy_residual,"
                "free_energy_per_unit_area\n";
  }
  const int burnin = cfg["numerics"]["num_iterations_burnin"].as_int(0);
  const int it_min = cfg["numerics"]["num_iterations_min"].as_int(0);
  const int it_max = cfg["numerics"]["num_iterations_max"].as_int(-1);
  int it_count = 0;
  double res = 0.0;
  int conv = 0;
  double sc[11];
  auto log_row = [&]() {
    sc_get_scalars(ctx, sc);
    if (conv_csv.is_open())
      conv_csv << std::scientific << std::setprecision(8) << it_count << "," << sc[8] << "," << sc[4]
               << "," << sc[5] << "," << sc[7] << "," << sc[6] << "," << sc[1] << "\n";
    if (verbose)
      std::cout << "-- iteration " << it_count << "  residual " << sc[9] << "  free energy/area "
                << sc[1] << std::endl;
  };
  for (int i = 0; i < burnin; ++i) {  // runBurnIn with min = max = burn-in count
    if (sc_burn_in(ctx, 1, &res, &conv) != SC_OK) return fail(sc_last_error(ctx));
    ++it_count;
    log_row();
  }
  bool converged = false;
  if (it_min != 0 || it_max != 0) {
    for (int i = 1;; ++i) {
      if (sc_compute(ctx, 1, &res, &conv) != SC_OK) return fail(sc_last_error(ctx));
      ++it_count;
      converged = conv != 0;
      log_row();
      if ((converged && i >= it_min) || (it_max >= 0 && i >= it_max)) break;
    }
  }
  if (verbose)
    std::cout << (converged ? "-- SUCCESS! Simulation converged." : "-- FAILURE! Simulation did not converge.")
              << std::endl;

  if (save_data) {
    // SimulationWriter::writeData / writeParameters (SimulationWriter.h:57-246).
    std::vector<double> dnew((size_t)nc * 2 * nn), j(2 * nn), anew(2 * nn), x(nc * 2 * nn), a(2 * nn);
    std::vector<signed char> dom(nn);
    sc_get_results(ctx, dnew.data(), j.data(), anew.data());
    sc_get_state(ctx, x.data(), a.data());
    sc_get_domain(ctx, dom.data());
    std::vector<double> domd(nn);
    for (size_t i = 0; i < nn; ++i) domd[i] = dom[i];
    const double vs = lambda > 0.0 ? 1.0 / (lambda * lambda) : 0.0;
    for (double &v : a) v *= vs;
    std::vector<double> bz(nn);
    for (int yy = 0; yy < n0; ++yy)
      for (int xx = 0; xx < n0; ++xx) {
        const int xn = std::min(xx + 1, n0 - 1), xp = std::max(xx - 1, 0);
        const int yn = std::min(yy + 1, n0 - 1), yp = std::max(yy - 1, 0);
        const double dAydx = (a[nn + (size_t)yy * n0 + xn] - a[nn + (size_t)yy * n0 + xp]) / (double)(xn - xp);
        const double dAxdy = (a[(size_t)yn * n0 + xx] - a[(size_t)yp * n0 + xx]) / (double)(yn - yp);
        bz[(size_t)yy * n0 + xx] = (dAydx - dAxdy) * (1.0 / h);
      }
    bool ok = write_grid(save / "domain.csv", n0, {"domain"}, false, {domd.data()}, true);
    std::vector<const double *> opl;
    for (int c = 0; c < nc; ++c) {
      opl.push_back(&dnew[(size_t)(2 * c) * nn]);
      opl.push_back(&dnew[(size_t)(2 * c + 1) * nn]);
    }
    ok = ok && write_grid(save / "order_parameter.csv", n0, comps, true, opl);
    ok = ok && write_grid(save / "current_density.csv", n0, {"j_x", "j_y"}, false, {j.data(), j.data() + nn});
    ok = ok && write_grid(save / "vector_potential.csv", n0, {"a_x", "a_y"}, false, {a.data(), a.data() + nn});
    ok = ok && write_grid(save / "magnetic_flux_density.csv", n0, {"b_z"}, false, {bz.data()});
    const int ng = (int)sc[10];
    double op_mag = 0.0, j_mag = 0.0, moment = 0.0, bsum = 0.0, a_mag = 0.0;
    for (size_t i = 0; i < nn; ++i) {
      for (int c = 0; c < nc; ++c)
        op_mag += std::hypot(dnew[(size_t)(2 * c) * nn + i], dnew[(size_t)(2 * c + 1) * nn + i]);
      j_mag += std::hypot(j[i], j[nn + i]);
      const int xi = (int)(i % n0), yi = (int)(i / n0);
      const double xc = (double)xi - 0.5 * (double)(n0 - 1), yc = (double)yi - 0.5 * (double)(n0 - 1);
      moment += xc * j[nn + i] - yc * j[i];
      if (dom[i]) {
        bsum += bz[i];
        a_mag += std::hypot(a[i], a[nn + i]);
      }
    }
    std::ofstream rj(save / "simulation_results.json");
    rj << "{\n"
       << "    \"current_density_average_magnitude\": " << json_number(j_mag / ng) << ",\n"
       << "    \"flux_density_average\": " << json_number(bsum / ng) << ",\n"
       << "    \"free_energy_per_unit_area\": " << json_number(sc[1]) << ",\n"
       << "    \"magnetic_free_energy_per_unit_area\": " << json_number(sc[3]) << ",\n"
       << "    \"magnetic_moment_per_unit_area\": "
       << json_number(0.5 * h * h * h * moment / (h * h * ng)) << ",\n"
       << "    \"order_parameter_average_magnitude\": " << json_number(op_mag / ng) << ",\n"
       << "    \"vector_potential_average_magnitude\": " << json_number(a_mag / ng) << "\n}\n";
    std::ofstream ij(save / "internal_parameters.json");
    ij << "{\n"
       << "    \"area_compute\": " << json_number(h * h * ng) << ",\n"
       << "    \"grain_margin\": 3,\n"
       << "    \"internal_lattice_points\": " << ng << ",\n"
       << "    \"num_lattice_points\": " << (long long)n0 * n0 << "\n}\n";
    if (!ok) {
      sc_destroy(ctx);
      return fail("could not write the results to " + save.string());
    }
  }
  sc_destroy(ctx);
  return EXIT_SUCCESS;
}

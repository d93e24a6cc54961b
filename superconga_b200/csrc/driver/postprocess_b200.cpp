// postprocess_b200 -- drop-in replacement of the reference's postprocess
// driver (src/postprocess.cu) on the B200 engine.
//
//   postprocess_b200 <postprocess_config.json>
//
// Reads the postprocess configuration, the simulation_config.json of the run
// in misc.load_path and its order_parameter.csv / vector_potential.csv
// (postprocess.cu:86-360), runs the LDOS postprocess energy block by energy
// block (runPostprocess, run_simulation.h:44-104) and writes into
// misc.save_path: postprocess_config.json, ldos.csv (CSVGridWriter.h with the
// energies as a third index: x_idx,y_idx,e_idx,ldos) and
// postprocess_convergence.csv (CSVPostprocessIterationWriter.h:40-70).
// The optional key b200.precision selects "fp64" (default) or "mixed".
#include "common.hpp"
#include "scb200.h"

using namespace drv;

int main(int argc, char *argv[]) {
  if (argc < 2) return fail("Please provide a config file.");
  std::string pp_text;
  if (!read_text(argv[1], pp_text)) return fail(std::string("Could not find/open config file '") + argv[1] + "'.");
  scb::JsonValue pp;
  try {
    pp = scb::JsonValue::parse(pp_text);
  } catch (const std::exception &e) {
    return fail(std::string("config: ") + e.what());
  }
  const fs::path load = pp["misc"]["load_path"].as_string();
  std::string sim_text;
  if (!read_text(load / "simulation_config.json", sim_text))
    return fail("Could not find/open config file '" + (load / "simulation_config.json").string() + "'.");
  scb::JsonValue sim;
  try {
    sim = scb::JsonValue::parse(sim_text);
  } catch (const std::exception &e) {
    return fail(std::string("simulation config: ") + e.what());
  }
  const bool verbose = pp["misc"]["verbose"].as_bool();
  const int mode = pp["b200"]["precision"].as_string("fp64") == "mixed" ? SC_MODE_MIXED : SC_MODE_FP64;

  sc_ctx *ctx = nullptr;
  if (sc_ldos_create(sim_text.c_str(), pp_text.c_str(), mode, &ctx) != SC_OK) return fail(sc_last_error(nullptr));
  int n0, n1, na, ne, nc;
  sc_get_dims(ctx, &n0, &n1, &na, &ne, &nc);
  int n_energies, per_block, n_blocks;
  sc_ldos_dims(ctx, &n_energies, &per_block, &n_blocks);
  const size_t nn = (size_t)n0 * n0;
  std::vector<std::string> comps;
  for (const char *s : {"dx2-y2", "dxy", "g", "s"})
    if (sim["physics"]["order_parameter"].has(s)) comps.push_back(s);

  // Order parameter and vector potential of the loaded run (postprocess.cu:286-364).
  std::vector<double> delta, avec;
  const double lambda = sim["physics"]["penetration_depth"].as_double(-1.0);
  {
    const std::string e = load_state(load, comps, n0, lambda, delta, avec);
    if (!e.empty()) return fail(e);
  }
  if (sc_set_state(ctx, delta.data(), avec.data()) != SC_OK) return fail(sc_last_error(ctx));

  const fs::path save = pp["misc"]["save_path"].as_string();
  const bool save_data = !save.empty();
  std::ofstream conv_csv;
  if (save_data) {
    fs::create_directories(save);
    conv_csv.open(save / "postprocess_convergence.csv");
    conv_csv << "iteration,boundary_coherence_residual,ldos_residual\n";
  }
  const int burnin = pp["numerics"]["num_iterations_burnin"].as_int(0);
  const int it_min = pp["numerics"]["num_iterations_min"].as_int(0);
  const int it_max = pp["numerics"]["num_iterations_max"].as_int(-1);
  const double crit = pp["numerics"]["convergence_criterion"].as_double();
  int it_count = 0;
  double sc[11];
  auto log_row = [&]() {
    sc_get_scalars(ctx, sc);
    if (conv_csv.is_open())
      conv_csv << std::scientific << std::setprecision(8) << it_count << "," << sc[8] << "," << sc[7] << "\n";
    if (verbose) std::cout << "-- iteration " << it_count << "  residual " << sc[9] << std::endl;
  };
  const int cap = 100000;  // bound of the "until converged" loops
  bool all = true;
  for (int b = 0; b < n_blocks && all; ++b) {
    if (verbose)
      std::printf("-- Energy block %.2f%% --> %.2f%%.\n", 100.0 * b * per_block / n_energies,
                  100.0 * std::min(n_energies, (b + 1) * per_block) / n_energies);
    if (sc_ldos_begin_block(ctx, b) != SC_OK) return fail(sc_last_error(ctx));
    double res = 0.0;
    int conv = 0;
    if (burnin != 0)
      for (int i = 1; i <= cap; ++i) {
        if (sc_burn_in(ctx, 1, &res, &conv) != SC_OK) return fail(sc_last_error(ctx));
        ++it_count;
        log_row();
        if ((res < crit && i >= burnin) || (burnin >= 0 && i >= burnin)) break;
      }
    bool block_conv = false;
    if (it_min != 0 || it_max != 0)
      for (int i = 1; i <= cap; ++i) {
        if (sc_ldos_iterate(ctx, 1, &res, &conv) != SC_OK) return fail(sc_last_error(ctx));
        ++it_count;
        block_conv = conv != 0;
        log_row();
        if ((block_conv && i >= it_min) || (it_max >= 0 && i >= it_max)) break;
      }
    if (verbose) std::cout << (block_conv ? "-- Energy block converged." : "-- Energy block did not converge.") << std::endl;
    all = block_conv;
  }
  if (verbose)
    std::cout << (all ? "-- SUCCESS! Postprocess converged." : "-- FAILURE! Postprocess did not converge.") << std::endl;

  if (save_data) {
    std::ofstream cj(save / "postprocess_config.json");
    dump_json(cj, pp, 0);
    cj << "\n";
    std::vector<double> ldos((size_t)n_energies * nn);
    if (sc_ldos_get(ctx, ldos.data()) != SC_OK) return fail(sc_last_error(ctx));
    std::ofstream out(save / "ldos.csv");
    out << "x_idx,y_idx,e_idx,ldos\n";
    std::ostringstream oss;
    for (int e = 0; e < n_energies; ++e)
      for (int y = 0; y < n0; ++y)
        for (int x = 0; x < n0; ++x) {
          oss.str("");
          oss << std::scientific << std::setprecision(8) << x << "," << y << "," << e << ","
              << ldos[(size_t)e * nn + (size_t)y * n0 + x];
          out << oss.str() << "\n";
        }
    if (!out.good()) {
      sc_destroy(ctx);
      return fail("could not write the LDOS to " + save.string());
    }
  }
  sc_destroy(ctx);
  return EXIT_SUCCESS;
}

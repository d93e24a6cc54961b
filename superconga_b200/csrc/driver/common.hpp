// Shared pieces of the drop-in drivers simulation_b200 and postprocess_b200:
// CSV grid reading (CSVReader.h) and writing (CSVGridWriter.h layout, 8
// significant digits), JSON echo, bulk gap and error exit.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "../json.hpp"
#include "scb200.h"

namespace fs = std::filesystem;

namespace drv {

constexpr double EULER_GAMMA = 0.57721566490153286060651209008240243;

// computeOrderParameterBulkSWave (OrderParameterBulk.h:88-221) with the
// reference's defaults, from the library.
inline double bulk_s_wave(double t) {
  double op = 0.0;
  sc_bulk_order_parameter_s_wave(t, 10.0 * 2.220446049250313e-16, 10, 100.0, &op);
  return op;
}

// One CSV file as column name -> values (CSVReader.h).
inline bool read_csv(const fs::path &p, std::map<std::string, std::vector<double>> &cols) {
  std::ifstream in(p);
  if (!in.good()) return false;
  std::string line;
  if (!std::getline(in, line)) return false;
  std::vector<std::string> names;
  {
    std::stringstream ss(line);
    std::string cell;
    while (std::getline(ss, cell, ',')) names.push_back(cell);
  }
  while (std::getline(in, line)) {
    if (line.empty()) continue;
    std::stringstream ss(line);
    std::string cell;
    size_t k = 0;
    while (std::getline(ss, cell, ',') && k < names.size()) cols[names[k++]].push_back(std::atof(cell.c_str()));
  }
  return true;
}

// CSVGridWriter::saveInternal layout: x_idx,y_idx,<fields...>, row-major y then x.
inline bool write_grid(const fs::path &p, int n, const std::vector<std::string> &titles, bool is_complex,
                const std::vector<const double *> &planes, bool integral = false) {
  std::ofstream out(p);
  if (!out.good()) return false;
  out << "x_idx,y_idx,";
  for (size_t k = 0; k < titles.size(); ++k) {
    out << titles[k];
    if (is_complex) out << "_re," << titles[k] << "_im";
    if (k + 1 < titles.size()) out << ",";
  }
  out << "\n";
  std::ostringstream oss;
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x) {
      oss.str("");
      oss << std::scientific << std::setprecision(8) << x << "," << y << ",";
      const size_t i = (size_t)y * n + x;
      for (size_t k = 0; k < planes.size(); ++k) {
        if (integral) oss << (int)planes[k][i];
        else oss << planes[k][i];
        if (k + 1 < planes.size()) oss << ",";
      }
      out << oss.str() << "\n";
    }
  return out.good();
}

inline std::string json_number(double v) {
  std::ostringstream o;
  o << std::setprecision(17) << v;
  return o.str();
}

// Serialises the parsed configuration back (simulation_config.json).
inline void dump_json(std::ostream &o, const scb::JsonValue &v, int ind) {
  const std::string pad(ind, ' ');
  switch (v.kind()) {
  case scb::JsonValue::Null: o << "null"; break;
  case scb::JsonValue::Bool: o << (v.as_bool() ? "true" : "false"); break;
  case scb::JsonValue::Number: o << json_number(v.as_double()); break;
  case scb::JsonValue::String: o << "\"" << v.as_string() << "\""; break;
  case scb::JsonValue::Array: {
    o << "[";
    for (size_t i = 0; i < v.size(); ++i) {
      if (i) o << ", ";
      dump_json(o, v[i], ind);
    }
    o << "]";
    break;
  }
  case scb::JsonValue::Object: {
    o << "{\n";
    const auto keys = v.keys();
    for (size_t i = 0; i < keys.size(); ++i) {
      o << pad << "    \"" << keys[i] << "\": ";
      dump_json(o, v[keys[i]], ind + 4);
      o << (i + 1 < keys.size() ? ",\n" : "\n");
    }
    o << pad << "}";
    break;
  }
  }
}

inline int fail(const std::string &m) {
  std::cerr << "-- ERROR! " << m << std::endl;
  return EXIT_FAILURE;
}


// Text of a file, false when it cannot be read.
inline bool read_text(const fs::path &p, std::string &out) {
  std::ifstream in(p);
  if (!in.good()) return false;
  std::stringstream buf;
  buf << in.rdbuf();
  out = buf.str();
  return true;
}

// Order parameter [Nc][2][n0][n0] and vector potential [2][n0][n0] (internal
// units, times lambda^2) of a saved run (src/simulation.cu:300-377,
// src/postprocess.cu:286-364).  Files written on another lattice are read as
// the reference's CSV reader does (csv.h:180-205, 297-395): the order
// parameter is extended past its grain with the saved domain.csv, then both
// fields are resampled onto n0.  Returns an error message, empty on success.
inline std::string load_state(const fs::path &load, const std::vector<std::string> &comps, int n0, double lambda,
                              std::vector<double> &delta, std::vector<double> &avec) {
  std::map<std::string, std::vector<double>> op, vp;
  if (!read_csv(load / "order_parameter.csv", op)) return "Could not find order parameter in " + load.string();
  if (!read_csv(load / "vector_potential.csv", vp)) return "Could not find vector potential in " + load.string();
  const size_t nn = (size_t)n0 * n0, nc = comps.size();
  delta.assign(nc * 2 * nn, 0.0);
  avec.assign(2 * nn, 0.0);
  std::vector<signed char> dom;
  int n_dom = 0;
  auto side = [](size_t count) {
    const int n = (int)std::lround(std::sqrt((double)count));
    return (size_t)n * n == count ? n : -1;
  };
  for (size_t c = 0; c < nc; ++c) {
    const auto &re = op[comps[c] + "_re"], &im = op[comps[c] + "_im"];
    if (re.empty() || re.size() != im.size())
      return "The file does not contain the columns, '" + comps[c] + "_re' and '" + comps[c] + "_im'.";
    double *dst = &delta[c * 2 * nn];
    if (re.size() == nn) {
      std::copy(re.begin(), re.end(), dst);
      std::copy(im.begin(), im.end(), dst + nn);
      continue;
    }
    const int n = side(re.size());
    if (n < 0) return "The data is not square.";
    if (dom.empty()) {
      std::map<std::string, std::vector<double>> dm;
      if (!read_csv(load / "domain.csv", dm) || side(dm["domain"].size()) != n)
        return "Could not read the domain of the saved lattice in " + load.string();
      n_dom = n;
      for (double v : dm["domain"]) dom.push_back((signed char)v);
    }
    if (n != n_dom) return "order-parameter and domain lattices differ";
    std::vector<double> planes(2 * (size_t)n * n);
    std::copy(re.begin(), re.end(), planes.begin());
    std::copy(im.begin(), im.end(), planes.begin() + (size_t)n * n);
    if (sc_grid_extend(n, dom.data(), 2, planes.data()) != SC_OK ||
        sc_grid_resample(n, n0, 2, planes.data(), dst) != SC_OK)
      return "could not resample the order parameter";
  }
  const auto &ax = vp["a_x"], &ay = vp["a_y"];
  if (ax.empty() || ax.size() != ay.size()) return "The file does not contain the columns, 'a_x' and 'a_y'.";
  if (ax.size() == nn) {
    std::copy(ax.begin(), ax.end(), avec.begin());
    std::copy(ay.begin(), ay.end(), avec.begin() + nn);
  } else {
    const int n = side(ax.size());
    if (n < 0) return "The data is not square.";
    std::vector<double> planes(2 * (size_t)n * n);
    std::copy(ax.begin(), ax.end(), planes.begin());
    std::copy(ay.begin(), ay.end(), planes.begin() + (size_t)n * n);
    if (sc_grid_resample(n, n0, 2, planes.data(), avec.data()) != SC_OK) return "could not resample the vector potential";
  }
  const double s = lambda > 0.0 ? lambda * lambda : 0.0;
  for (double &v : avec) v *= s;
  return std::string();
}

}  // namespace drv

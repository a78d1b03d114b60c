// Reader for the reference's setup.txt (host code).
//
// Grammar as in Parameter::read_one_file / read_struct (reference
// src/Parameter.cpp:38-184): "type name = value" lines for int, real, bool and
// string; "array type name = { ... }" spanning lines; "struct name { ... }"
// blocks of typed entries closed by a lone "}".  Defaults follow
// Parameter::setup_default_settings (reference src/Parameter.cpp:342-523) and
// the derived quantities deduce_known_info (reference src/Parameter.cpp:186-340)
// and the reference-state scaling of weno_eps_scale (reference
// src/BoundCond.cpp:159-283, src/DParameter.cu:25-28).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <variant>
#include <vector>

#include "corefl_b200.h"

namespace {

using Value = std::variant<std::string, int, double>;
using Struct = std::map<std::string, Value>;

struct Setup {
  std::map<std::string, int> ints;
  std::map<std::string, double> reals;
  std::map<std::string, bool> bools;
  std::map<std::string, std::string> strings;
  std::map<std::string, std::vector<std::string>> arrays;  // all arrays kept as tokens
  std::map<std::string, Struct> structs;
};

bool starts_with(const std::string &s, const char *p) { return s.rfind(p, 0) == 0; }

// Reads array tokens until "}"; returns false if the array continues on the next line.
bool read_array_tokens(std::istringstream &line, std::vector<std::string> &out) {
  std::string t;
  while (line >> t) {
    if (t == "}") return true;
    if (t == "//") return false;
    out.push_back(t);
  }
  return false;
}

bool next_line(std::ifstream &f, std::string &input, std::istringstream &line) {
  while (std::getline(f, input)) {
    if (input.empty() || starts_with(input, "//") || starts_with(input, "!")) continue;
    line.clear();
    line.str(input);
    return true;
  }
  return false;
}

bool parse(const char *path, Setup &s, std::string &err) {
  std::ifstream f(path);
  if (!f) { err = std::string("cannot open ") + path; return false; }
  std::string input;
  std::istringstream line;
  while (std::getline(f, input)) {
    if (input.empty() || starts_with(input, "//") || starts_with(input, "!")) continue;
    line.clear();
    line.str(input);
    std::string type, key, temp;
    line >> type >> key >> temp;
    if (type == "int") { int v = 0; line >> v; s.ints[key] = v; }
    else if (type == "real") { double v = 0; line >> v; s.reals[key] = v; }
    else if (type == "bool") { int v = 0; line >> v; s.bools[key] = v != 0; }
    else if (type == "string") { std::string v; line >> v; s.strings[key] = v; }
    else if (type == "array" || type == "range") {
      const std::string name = temp;
      line >> temp >> temp;  // "=" "{"
      std::vector<std::string> toks;
      while (!read_array_tokens(line, toks)) {
        if (!next_line(f, input, line)) { err = "unterminated array " + name; return false; }
      }
      s.arrays[name] = toks;
    } else if (type == "struct") {
      Struct st;
      while (next_line(f, input, line)) {
        std::string k;
        line >> k;
        if (k == "}") break;
        std::string n, eq;
        if (k == "string") { std::string v; line >> n >> eq >> v; st.emplace(n, v); }
        else if (k == "int") { int v = 0; line >> n >> eq >> v; st.emplace(n, v); }
        else if (k == "real") { double v = 0; line >> n >> eq >> v; st.emplace(n, v); }
      }
      s.structs[key] = st;
    }
  }
  return true;
}

template <class M, class V>
V get(const M &m, const std::string &k, V dflt) {
  auto it = m.find(k);
  return it == m.end() ? dflt : static_cast<V>(it->second);
}

double struct_real(const Struct &st, const char *k, double dflt) {
  auto it = st.find(k);
  if (it == st.end()) return dflt;
  if (auto p = std::get_if<double>(&it->second)) return *p;
  if (auto p = std::get_if<int>(&it->second)) return *p;
  return dflt;
}

std::string struct_string(const Struct &st, const char *k) {
  auto it = st.find(k);
  if (it == st.end()) return std::string();
  if (auto p = std::get_if<std::string>(&it->second)) return *p;
  return std::string();
}

int struct_int(const Struct &st, const char *k, int dflt) {
  auto it = st.find(k);
  if (it == st.end()) return dflt;
  if (auto p = std::get_if<int>(&it->second)) return *p;
  return dflt;
}

// The wall condition of the boundary_conditions list (reference
// src/BoundCond.cpp:480-528, Wall::Wall): thermal_type isothermal (default,
// also for an unknown name, as there), adiabatic or equilibrium_radiation
// (kept as 2, which cfk_create rejects); temperature defaults to 300 K.
// Returns false when more than one wall struct is listed, or when the wall
// asks for blowing/suction fluctuations or shock blowing (problem set-ups
// outside this path).
bool read_wall(const Setup &s, cfk_wall &w, std::string &err) {
  w.thermal_type = 0;
  w.catalytic_type = 0;
  w.temperature = 300.0;
  auto list = s.arrays.find("boundary_conditions");
  if (list == s.arrays.end()) return true;
  int n_wall = 0;
  for (const std::string &name : list->second) {
    auto it = s.structs.find(name);
    if (it == s.structs.end() || struct_string(it->second, "type") != "wall") continue;
    if (++n_wall > 1) {
      err = "more than one wall condition in boundary_conditions; cfk_param carries one";
      return false;
    }
    if (struct_int(it->second, "fluctuation_type", 0) != 0 || struct_int(it->second, "if_blow_shock_wave", 0) != 0) {
      err = "wall " + name + ": wall fluctuations and shock blowing are not supported";
      return false;
    }
    const std::string t = struct_string(it->second, "thermal_type");
    w.thermal_type = t == "adiabatic" ? 1 : t == "equilibrium_radiation" ? 2 : 0;
    w.temperature = struct_real(it->second, "temperature", 300.0);
  }
  return true;
}


// The two streams of an air mixing layer (problem_type 1), as
// get_mixing_layer_info computes them for air (reference
// src/MixingLayer.cu:9-119): each stream's density and sound speed from its
// temperature and pressure; with velocity_ratio r > 0, u_slow = Ma_c (c_upper
// + c_lower) / (r - 1) and u_fast = r u_slow (r > 1; else u_fast = Ma_c (c_upper
// + c_lower) / (1 - r), u_slow = r u_fast), the faster stream above when
// upper_faster; with r <= 0 the streams' own Mach numbers (one of them may be
// derived from Ma_c).
bool mixing_layer_streams(const Setup &s, cfk_inflow &q, std::string &err) {
  const double R_u = 8314.462618, mw = 28.9647, gamma = 1.4;
  auto up_it = s.structs.find("upper_stream"), lo_it = s.structs.find("lower_stream");
  if (up_it == s.structs.end() || lo_it == s.structs.end()) {
    err = "problem_type 1 needs the upper_stream and lower_stream structs";
    return false;
  }
  const Struct &up = up_it->second, &lo = lo_it->second;
  const double ma_c = get(s.reals, "ma_c", 0.0), vel_ratio = get(s.reals, "velocity_ratio", 0.0);
  const bool upper_faster = get(s.bools, "upper_faster", false);
  double ma_upper = struct_real(up, "mach", -1), ma_lower = struct_real(lo, "mach", -1);
  const double T_upper = struct_real(up, "temperature", -1), T_lower = struct_real(lo, "temperature", -1);
  const double p_upper = struct_real(up, "pressure", -1), p_lower = struct_real(lo, "pressure", -1);
  if (!(T_upper > 0) || !(T_lower > 0) || !(p_upper > 0) || !(p_lower > 0)) {
    err = "mixing-layer streams need temperature and pressure > 0";
    return false;
  }
  const double c_upper = std::sqrt(gamma * R_u / mw * T_upper), c_lower = std::sqrt(gamma * R_u / mw * T_lower);
  if (vel_ratio > 0) {
    double u_slow, u_fast;
    if (vel_ratio > 1) {
      u_slow = ma_c * (c_upper + c_lower) / (vel_ratio - 1);
      u_fast = vel_ratio * u_slow;
    } else {
      u_fast = ma_c * (c_upper + c_lower) / (1 - vel_ratio);
      u_slow = u_fast * vel_ratio;
    }
    ma_upper = (upper_faster ? u_fast : u_slow) / c_upper;
    ma_lower = (upper_faster ? u_slow : u_fast) / c_lower;
  } else if (ma_upper < 0 && ma_lower < 0) {
    err = "at least one of the streams' Mach numbers and the convective Mach number must be given";
    return false;
  } else if (ma_upper > 0 && ma_lower > 0) {
    // both given: the streams win over ma_c, as in the reference
  } else if (ma_upper > 0) {
    ma_lower = upper_faster ? (ma_upper - ma_c) * c_upper / c_lower - ma_c
                            : (ma_c + ma_upper) * c_upper / c_lower + ma_c;
  } else {
    ma_upper = upper_faster ? (ma_c + ma_lower) * c_lower / c_upper + ma_c
                            : (ma_lower - ma_c) * c_lower / c_upper - ma_c;
  }
  q.inflow_type = 2;
  q.density = p_upper * mw / (R_u * T_upper);
  q.u = ma_upper * c_upper;
  q.v = q.w = 0;
  q.pressure = p_upper;
  q.temperature = T_upper;
  q.mw = mw;
  q.density_lower = p_lower * mw / (R_u * T_lower);
  q.u_lower = ma_lower * c_lower;
  q.v_lower = q.w_lower = 0;
  q.p_lower = p_lower;
  q.t_lower = T_lower;
  q.delta_omega = get(s.reals, "delta_omega", 0.0);
  if (!(q.delta_omega > 0)) {
    err = "problem_type 1 needs delta_omega > 0";
    return false;
  }
  return true;
}

// The inflow condition of the boundary_conditions list, air (reference
// src/BoundCond.cpp:9-260, Inflow::Inflow): a constant inflow, the state
// from one of (mach, pressure, temperature), (density, velocity, pressure)
// or (mach, temperature, reynolds), the velocity along aoa (degrees) or along
// (u, v, w); with problem_type 1 the mixing-layer inflow of
// mixing_layer_streams.  fluctuation_type 1 (white noise) takes
// fluctuation_intensity; the deviates are seeded by the int random_seed
// (default 0) where the reference seeds curand from the clock.  Profile
// inflows and the other fluctuation forms are reported; so is a second
// inflow struct.
bool read_inflow(const Setup &s, cfk_inflow &q, std::string &err) {
  std::memset(&q, 0, sizeof(q));
  auto list = s.arrays.find("boundary_conditions");
  if (list == s.arrays.end()) return true;
  int n_inflow = 0;
  for (const std::string &name : list->second) {
    auto it = s.structs.find(name);
    if (it == s.structs.end() || struct_string(it->second, "type") != "inflow") continue;
    const Struct &st = it->second;
    if (++n_inflow > 1) { err = "more than one inflow condition; cfk_param carries one"; return false; }
    const int problem_type = get(s.ints, "problem_type", 0);
    int inflow_type = struct_int(st, "inflow_type", 0);
    if (problem_type == 1) inflow_type = 2;                      // src/BoundCond.cpp:12-16
    if (problem_type == 0 && inflow_type == 2) inflow_type = 0;
    const int fluctuation_type = struct_int(st, "fluctuation_type", 0);
    if (inflow_type != 0 && inflow_type != 2) {
      err = "inflow " + name + ": profile inflows are not supported";
      return false;
    }
    if (fluctuation_type != 0 && fluctuation_type != 1) {
      err = "inflow " + name + ": only the white-noise fluctuation (fluctuation_type 1) is supported";
      return false;
    }
    q.fluctuation_type = fluctuation_type;
    q.fluctuation_intensity = fluctuation_type == 1 ? struct_real(st, "fluctuation_intensity", 0.0) : 0.0;
    q.seed = (unsigned long long)get(s.ints, "random_seed", 0);
    q.subsonic = struct_int(st, "inflow_sub", 0);
    if (inflow_type == 2) {
      if (!mixing_layer_streams(s, q, err)) return false;
      continue;
    }
    const double R_u = 8314.462618, mw = 28.9647, gamma = 1.4, pi = 3.141592653589793;
    double mach = struct_real(st, "mach", -1), pressure = struct_real(st, "pressure", -1);
    double temperature = struct_real(st, "temperature", -1), velocity = struct_real(st, "velocity", 0);
    double density = struct_real(st, "density", -1), aoa = struct_real(st, "aoa", -1000);
    double u = struct_real(st, "u", 1), v = struct_real(st, "v", 0), w = struct_real(st, "w", 0);
    const double reynolds = struct_real(st, "reynolds", -1);
    if (temperature < 0) temperature = pressure * mw / (density * R_u);
    const double viscosity = 1.7894e-5 * std::pow(temperature / 288.16, 1.5) * (288.16 + 110) / (temperature + 110);
    const double c = std::sqrt(gamma * R_u / mw * temperature);
    if (mach < 0) mach = velocity / c;
    else velocity = mach * c;
    if (aoa > -1000) {
      u = std::cos(aoa * pi / 180) * velocity;
      v = std::sin(aoa * pi / 180) * velocity;
      w = 0;
    } else {
      u *= velocity;
      v *= velocity;
      w *= velocity;
    }
    if (density < 0) {
      if (pressure < 0) {
        if (reynolds < 0) { err = "inflow " + name + ": give pressure, density or reynolds"; return false; }
        density = viscosity * reynolds / velocity;
        pressure = density * temperature * R_u / mw;
      } else {
        density = pressure * mw / (R_u * temperature);
      }
    }
    q.subsonic = struct_int(st, "inflow_sub", 0);
    q.density = density;
    q.u = u;
    q.v = v;
    q.w = w;
    q.pressure = pressure;
    q.temperature = temperature;
    q.mw = mw;
  }
  return true;
}

// The outflow condition of the boundary_conditions list (reference
// src/BoundCond.cpp:597-618, Outflow::Outflow): if_backPressure and
// backPressure.  A non-reflecting outflow is not part of this path and is
// reported; so are two outflow structs with different back pressures.
bool read_outflow(const Setup &s, cfk_outflow &o, std::string &err) {
  o.back_pressure_on = 0;
  o.back_pressure = 0;
  auto list = s.arrays.find("boundary_conditions");
  if (list == s.arrays.end()) return true;
  int n_outflow = 0;
  for (const std::string &name : list->second) {
    auto it = s.structs.find(name);
    if (it == s.structs.end() || struct_string(it->second, "type") != "outflow") continue;
    const Struct &st = it->second;
    if (struct_int(st, "nonReflecting", 0) > 0) {
      err = "outflow " + name + ": non-reflecting outflow is not supported";
      return false;
    }
    const int on = struct_int(st, "if_backPressure", 0);
    const double pb = on == 1 ? struct_real(st, "backPressure", -1) : 0;
    if (n_outflow++ > 0 && (on != o.back_pressure_on || pb != o.back_pressure)) {
      err = "outflow conditions differ; cfk_param carries one";
      return false;
    }
    o.back_pressure_on = on;
    o.back_pressure = pb;
  }
  return true;
}

}  // namespace

extern "C" int cfk_param_from_setup(const char *setup_path, cfk_param *out, char *errbuf, size_t err_len) {
  auto report = [&](const std::string &m) {
    if (errbuf && err_len) {
      std::snprintf(errbuf, err_len, "%s", m.c_str());
    }
    return CFK_ERR_IO;
  };
  if (!setup_path || !out) return CFK_ERR_ARG;
  Setup s;
  std::string err;
  if (!parse(setup_path, s, err)) return report(err);
  cfk_param p;
  std::memset(&p, 0, sizeof(p));
  p.dim = get(s.ints, "dimension", 3);
  p.inviscid_scheme = get(s.ints, "inviscid_scheme", 3);
  p.reconstruction = get(s.ints, "reconstruction", 2);
  p.limiter = get(s.ints, "limiter", 0);
  p.viscous_order = get(s.ints, "viscous_order", 2);
  p.positive_preserving = get(s.bools, "positive_preserving", false);
  p.gradPInDiffusionFlux = get(s.bools, "gradPInDiffusionFlux", false);
  p.fixed_dt = get(s.bools, "fixed_time_step", false);
  p.chem_advance_method = get(s.ints, "chem_advance_method", 0);
  p.entropy_fix_factor = get(s.reals, "entropy_fix_factor", 0.125);
  p.Pr = get(s.reals, "prandtl_number", 0.72);
  p.Sc = get(s.reals, "schmidt_number", 0.5);
  p.cfl = get(s.reals, "cfl", 0.8);
  p.dt = get(s.reals, "dt", 1e-8);
  p.sensor_threshold = get(s.reals, "shockSensor_threshold", 0.0);
  p.shock_sensor = get(s.ints, "shock_sensor", 0);
  p.sensor_eps = get(s.reals, "shockSensor_epsilon", -1.0);
  const int species = get(s.ints, "species", 0);
  // hardCodedMech > 0 selects the reference's hard-coded H2/air kinetics
  // (src/FiniteRateChem.cu:19-358, src/StrangSplitting.cu:423-473, 479-484),
  // whose arithmetic order differs from the table-driven kinetics this
  // library implements: rejected rather than silently replaced
  if (const int hc = get(s.ints, "hardCodedMech", 0); hc != 0)
    return report("hardCodedMech = " + std::to_string(hc) +
                  ": the hard-coded kinetics are not implemented; use the mechanism tables (hardCodedMech = 0)");
  if (species != 0) return report("species != 0 needs a mechanism; pass n_spec/n_scalar explicitly");
  p.n_spec = 0;
  p.n_scalar = 0;
  p.n_var = 5;
  p.n_reac = 0;
  // reference state -> rho_ref, v_ref (air)
  const std::string ref = get(s.strings, "reference_state", std::string());
  p.rho_ref = 1.0;
  p.v_ref = 1.0;
  double p_inf = 1.0;
  auto it = s.structs.find(ref);
  if (it != s.structs.end()) {
    const Struct &st = it->second;
    const double R_u = 8314.462618, mw = 28.9647, gamma = 1.4;
    double mach = struct_real(st, "mach", -1), pressure = struct_real(st, "pressure", -1);
    double temperature = struct_real(st, "temperature", -1), velocity = struct_real(st, "velocity", -1);
    double density = struct_real(st, "density", -1);
    if (temperature < 0) temperature = pressure * mw / (density * R_u);
    const double c = std::sqrt(gamma * R_u / mw * temperature);
    if (mach < 0) mach = velocity / c;
    else velocity = mach * c;
    if (density < 0) density = pressure * mw / (R_u * temperature);
    if (pressure < 0) pressure = density * temperature * R_u / mw;
    p.rho_ref = density;
    p.v_ref = std::fabs(velocity) < 1 ? c : velocity;
    p_inf = pressure;
  }
  p.weno_eps_scale = p.rho_ref * p.v_ref * p.rho_ref * p.v_ref;
  // limit_flow and its bounds from the reference state: rho_inf, v_inf (the
  // speed of sound below 1 m/s) and p_inf (reference src/DParameter.cu:333-349,
  // src/BoundCond.cpp:276-290)
  p.limit_flow = get(s.bools, "limit_flow", false);
  p.limit_ll[0] = 1e-6 * p.rho_ref;
  p.limit_ul[0] = 1e+3 * p.rho_ref;
  for (int l = 1; l < 4; ++l) {
    p.limit_ll[l] = -1000 * p.v_ref;
    p.limit_ul[l] = 1000 * p.v_ref;
  }
  p.limit_ll[4] = 1e-6 * p_inf;
  p.limit_ul[4] = 1e+3 * p_inf;
  if (!read_wall(s, p.wall, err)) return report(err);
  if (!read_inflow(s, p.inflow, err)) return report(err);
  if (!read_outflow(s, p.outflow, err)) return report(err);
  p.n_face = 0;
  *out = p;
  return CFK_OK;
}

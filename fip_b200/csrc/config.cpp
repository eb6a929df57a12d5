#include "config.h"

#include <algorithm>
#include <cmath>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <map>
#include <sstream>
#include <stdexcept>

#include "yaml_lite.h"

namespace fip {

float TimeSeries::interp(float time) const {
  // std::map::lower_bound: first key not less than `time`
  const size_t n = t.size();
  size_t lo = std::lower_bound(t.begin(), t.end(), time) - t.begin();
  if (lo == 0) return v[0];
  if (lo == n) return v[n - 1];
  float dt = t[lo] - t[lo - 1];
  float f = (time - t[lo - 1]) / dt;
  return f * v[lo] + (1.f - f) * v[lo - 1];
}

TimeSeries TimeSeries::from_csv(const std::string& path, int time_col, int data_col, float time_scale,
                                bool skip_header) {
  std::ifstream f(path);
  if (!f.is_open()) throw std::invalid_argument("Could not open file " + path);
  auto is_float = [](const std::string& s) {
    std::istringstream iss(s);
    float x;
    iss >> std::noskipws >> x;
    return iss.eof() && !iss.fail();
  };
  std::map<float, float> series;
  std::string line;
  time_t first = -1;
  if (skip_header) std::getline(f, line);
  while (std::getline(f, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty()) continue;
    std::stringstream ss(line);
    std::string val;
    float time = 0.f, data = 0.f;
    bool got_t = false, got_d = false;
    int col = 0;
    while (std::getline(ss, val, ';')) {
      if (col == time_col) {
        if (is_float(val)) {
          time = std::stof(val) * time_scale;
        } else {
          std::tm tm = {};
          std::istringstream ts(val);
          ts >> std::get_time(&tm, "%d.%m.%Y %H:%M:%S");
          if (ts.fail())
            throw std::invalid_argument("Wrong date format in timeseries " + path +
                                        ". Expected %d.%m.%Y %H:%M:%S");
          time_t stamp = std::mktime(&tm);
          if (first == -1) first = stamp;
          time = static_cast<float>(stamp - first);
        }
        got_t = true;
      }
      if (col == data_col) {
        data = std::stof(val);
        got_d = true;
      }
      ++col;
    }
    if (!got_t || !got_d) throw std::invalid_argument("timeseries " + path + ": missing column in line \"" + line + "\"");
    series.emplace(time, data);
  }
  if (series.empty()) throw std::invalid_argument("timeseries " + path + " has no data rows");
  TimeSeries r;
  for (const auto& kv : series) {
    r.t.push_back(kv.first);
    r.v.push_back(kv.second);
  }
  return r;
}

double solve_simple_math(const std::string& expr) {
  if (expr.find_first_not_of("0123456789.* ") != std::string::npos)
    throw std::invalid_argument("Unsupported math expression " + expr);
  double result = 1.0;
  std::stringstream ss(expr);
  std::string item;
  while (std::getline(ss, item, '*')) result *= std::stof(item);
  return result;
}

static size_t boundary_index(const Config& c, BcSide side, int n) {
  switch (side) {  // getIdxForNthBoundaryCell (src/boundary_condition.cpp:20-40), unpitched
    case BcSide::left: return (size_t)n * c.W;
    case BcSide::right: return (size_t)n * c.W + (c.W - 1);
    case BcSide::top: return (size_t)n + (c.H - 1) * c.W;
    default: return (size_t)n;
  }
}

float Config::sum_water_depths(const BoundaryCondition& bc, float z_soll) const {
  float sum = 0.f;
  const float G = 9.81f;
  for (int n = bc.from; n < bc.to; ++n) {
    float ah = z_soll - terrain[boundary_index(*this, bc.side, n)];
    if (ah < 0.01f) ah = 0.f;
    sum += std::sqrt(G * ah) * ah;
  }
  sum *= dx;
  return sum;
}

float Config::const_q(const BoundaryCondition& bc) const {
  if (bc.type != BcType::q) return bc.q;
  return bc.q / sum_water_depths(bc, bc.z);
}

namespace {

template <typename E>
E enum_of(const std::string& s, std::initializer_list<const char*> names) {
  int i = 0;
  for (const char* n : names) {
    if (s == n) return static_cast<E>(i);
    ++i;
  }
  throw std::invalid_argument("Invalid enum value: " + s);  // stringToEnum (src/enumhelper.h:15-23)
}
BcType bc_type(const std::string& s) { return enum_of<BcType>(s, {"z", "q", "close", "open"}); }
BcSide bc_side(const std::string& s) { return enum_of<BcSide>(s, {"left", "right", "top", "bottom"}); }
SampleType sample_type(const std::string& s) { return enum_of<SampleType>(s, {"z", "h", "qx", "qy"}); }
Solver solver_of(const std::string& s) { return enum_of<Solver>(s, {"rmg", "cn"}); }

// validateSimDataConfig (src/simdata.cpp:152-236), same messages; `quiet` drops the warnings
// (never the errors)
bool validate(const YNode& config, bool quiet) {
  bool ok = true;
  auto error = [&ok](const YNode& node, const std::string& msg) {
    ok = false;
    std::cerr << "Config error at line " << node.line() + 1 << ": " << msg << std::endl;
  };
  auto in_config = [&](const YNode& node, const std::string& a) {
    if (!node[a].defined()) error(node, "\"" + a + "\" missing");
  };
  auto xor_in_config = [&](const YNode& node, const std::string& a, const std::string& b) {
    if (node[a].defined() && node[b].defined()) error(node[a], "Both \"" + a + "\" and \"" + b + "\" defined");
  };
  auto good_path = [&](const YNode& node, const std::string& a) {
    if (node[a].defined() && (!node[a].is_sequence() || node[a].size() != 2))
      error(node[a], "file path \"" + a + "\" needs format [path, byte_offset]");
  };
  auto good_series = [&](const YNode& node, const std::string& a) {
    if (node[a].defined() && (!node[a].is_sequence() || node[a].size() != 3))
      error(node[a], "timeseries \"" + a + "\" needs format [csv_filename, int_time_column, int_data_column]");
  };
  for (const char* k : {"name", "terrain", "W", "H", "dt", "dx", "duration"}) in_config(config, k);
  xor_in_config(config, "kSt_var", "kSt");
  for (const char* k : {"terrain", "z", "qx", "qy", "kSt_var"}) good_path(config, k);
  if (!quiet && !config["kSt_var"].defined() && !config["kSt"].defined())
    std::cerr << "Warning: both \"kSt_var\" and \"kSt\" missing, using default kSt " << 30.f << std::endl;
  for (const YNode& bc : config["boundary_conditions"].seq()) {
    in_config(bc, "side");
    in_config(bc, "type");
    if (!bc["type"].defined()) continue;
    BcType type = bc_type(bc["type"].as_string());
    if (type == BcType::z) in_config(bc, "z");
    if (type == BcType::q) {
      in_config(bc, "z");
      in_config(bc, "q");
    }
    if (bc["z"].defined() && bc["z"].is_sequence()) good_series(bc, "z");
    if (bc["q"].defined() && bc["q"].is_sequence()) good_series(bc, "q");
  }
  if (config["sampling_interval"].defined()) {
    if (!config["sampling"].defined() || !config["sampling"].is_sequence()) {
      ok = false;
      std::cerr << "Configuration error: sampling interval specified but no sampling points given" << std::endl;
    }
    for (const YNode& sp : config["sampling"].seq())
      for (const char* k : {"x", "y", "label", "type"}) in_config(sp, k);
  }
  if (!quiet && !config["save_state"].defined()) std::cerr << "Warning: no save_state times given" << std::endl;
  return ok;
}

struct IoError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

// loadSimDataFileWithOffset + utils::loadFileIntoArray (src/simdata.cpp:143-150, utils.h:45-54)
std::vector<float> load_grid(const YNode& node, size_t W, size_t H) {
  const std::string path = node[0].as_string();
  const long long offset = node[1].as_int64();
  std::ifstream f(path, std::ios::binary);
  if (!f) throw IoError("Failed to open file " + path);
  std::vector<float> a(W * H);
  f.seekg(offset);
  f.read(reinterpret_cast<char*>(a.data()), (std::streamsize)(a.size() * sizeof(float)));
  if ((size_t)f.gcount() != a.size() * sizeof(float))
    throw IoError("File " + path + " is too short: expected " + std::to_string(a.size() * sizeof(float)) +
                  " bytes at offset " + std::to_string(offset) + ", read " + std::to_string(f.gcount()));
  return a;
}

}  // namespace

int load_config(const std::string& path, Config* out, std::string* err, bool quiet) {
  Config c;
  c.yaml_path = path;
  try {
    YNode config = YNode::load_file(path);
    if (!validate(config, quiet)) throw std::invalid_argument("one or more configuration errors found");
    c.name = config["name"].as_string();
    c.target_duration = solve_simple_math(config["duration"].as_string());
    long long W = config["W"].as_int64(), H = config["H"].as_int64();
    if (W < 4 || H < 4) throw std::invalid_argument("grid must be at least 4 x 4 cells");
    c.W = (size_t)W;
    c.H = (size_t)H;
    c.dt = config["dt"].as_float();
    c.dx = config["dx"].as_float();
    c.variable_dt = config["variable_dt"].as_bool(true);
    c.solver = config["solver"].defined() ? solver_of(config["solver"].as_string()) : Solver::rmg;
    c.kst_fixed = config["kSt"].as_float(30.f);

    const size_t n = c.W * c.H;
    c.terrain = load_grid(config["terrain"], c.W, c.H);
    if (config["no_data"].defined()) c.no_data = config["no_data"].as_float();
    c.h0.assign(n, 0.f);
    if (config["z"].defined()) {
      std::vector<float> z = load_grid(config["z"], c.W, c.H);
      for (size_t i = 0; i < n; ++i) c.h0[i] = z[i] - c.terrain[i];
    }
    c.qx0 = config["qx"].defined() ? load_grid(config["qx"], c.W, c.H) : std::vector<float>(n, 0.f);
    c.qy0 = config["qy"].defined() ? load_grid(config["qy"], c.W, c.H) : std::vector<float>(n, 0.f);
    // zeros as +0 (the step writes +0 for every zero discharge and depth it computes, so a dry
    // tile skipped by the active-tile plan then holds exactly what computing it would give)
    for (std::vector<float>* g : {&c.h0, &c.qx0, &c.qy0})
      for (float& v : *g)
        if (v == 0.f) v = 0.f;
    if (config["kSt_var"].defined()) {
      c.has_kst_var = true;
      c.kst = load_grid(config["kSt_var"], c.W, c.H);
    }

    // createBoundaryCondition (src/simdata.cpp:98-131)
    for (const YNode& b : config["boundary_conditions"].seq()) {
      BoundaryCondition bc;
      bc.type = bc_type(b["type"].as_string());
      bc.side = bc_side(b["side"].as_string());
      const bool lr = bc.side == BcSide::left || bc.side == BcSide::right;
      bc.from = b["from"].as_int(0);
      bc.to = b["to"].as_int(lr ? (int)c.H - 1 : (int)c.W - 1);
      const int len = lr ? (int)c.H : (int)c.W;
      if (bc.from < 0 || bc.to >= len || bc.from > bc.to + 1)
        throw std::invalid_argument("boundary condition cells " + std::to_string(bc.from) + ".." +
                                    std::to_string(bc.to) + " outside the " + b["side"].as_string() +
                                    " side (0.." + std::to_string(len - 1) + ")");
      bc.is_series = (b["q"].defined() && b["q"].is_sequence()) || (b["z"].defined() && b["z"].is_sequence());
      if (bc.is_series) {
        auto series = [&](const char* key, bool* has) {
          const YNode& node = b[key];
          if (!node.defined()) return TimeSeries();
          if (!node.is_sequence()) throw std::invalid_argument(std::string("\"") + key + "\" must be a timeseries "
                                                               "when the other value of the condition is one");
          *has = true;
          return TimeSeries::from_csv(node[0].as_string(), node[1].as_int(), node[2].as_int());
        };
        bc.q_series = series("q", &bc.has_q_series);
        bc.z_series = series("z", &bc.has_z_series);
        if (bc.type == BcType::z && !bc.has_z_series)
          throw std::invalid_argument("BoundaryCondition error: type z but no z timeseries given");
        if (bc.type == BcType::q && (!bc.has_z_series || !bc.has_q_series))
          throw std::invalid_argument("BoundaryCondition error: type q requires both z and q timeseries");
      } else {
        bc.q = b["q"].as_float(0.f);
        bc.z = b["z"].as_float(0.f);
      }
      c.bcs.push_back(std::move(bc));
    }

    if (config["sampling_interval"].defined()) {
      c.sampling_interval = config["sampling_interval"].as_int();
      for (const YNode& sp : config["sampling"].seq()) {
        SamplePoint p;
        p.x = sp["x"].as_int();
        p.y = sp["y"].as_int();
        p.label = sp["label"].as_string();
        p.type = sample_type(sp["type"].as_string());
        if (p.x < 0 || p.y < 0 || (size_t)p.x >= c.W || (size_t)p.y >= c.H)
          throw std::invalid_argument("sampling point " + p.label + " outside the grid");
        c.points.push_back(p);
      }
    }
    if (config["save_state"].defined()) {
      for (const YNode& s : config["save_state"].seq()) c.save_times.push_back(solve_simple_math(s.as_string()));
      std::sort(c.save_times.begin(), c.save_times.end());
    }
  } catch (const IoError& e) {
    *err = e.what();
    return 2;
  } catch (const std::exception& e) {
    *err = e.what();
    return 1;
  }
  *out = std::move(c);
  return 0;
}

}  // namespace fip

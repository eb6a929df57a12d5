// Simulation configuration: the reference's SimData globals (src/simdata.h:333-373) as one
// value type, filled from the YAML parameter file and the raw float32 input grids.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

namespace fip {

enum class BcSide { left = 0, right = 1, top = 2, bottom = 3 };   // RandSide
enum class BcType { z = 0, q = 1, close = 2, open = 3 };          // RandType
enum class SampleType { z = 0, h = 1, qx = 2, qy = 3 };           // SampleType
enum class Solver { rmg = 0, cn = 1 };                             // Solver

// TimeSeries (src/timeseries.{h,cpp}): sorted unique times, first value wins on duplicates.
struct TimeSeries {
  std::vector<float> t, v;
  // clamped linear interpolation in float, same operation order as TimeSeries::interp
  float interp(float time) const;
  // `;` separated CSV; header line skipped; time in float seconds or %d.%m.%Y %H:%M:%S
  // (local time, counted from the first row). Throws std::invalid_argument like fromCsv.
  static TimeSeries from_csv(const std::string& path, int time_col, int data_col, float time_scale = 1.f,
                             bool skip_header = true);
};

struct BoundaryCondition {
  BcType type;
  BcSide side;
  int from, to;       // inclusive cell range on the side (the kernel's `tid > to` test)
  bool is_series;     // BoundaryConditionTimeseries
  float z = 0.f, q = 0.f;
  bool has_z_series = false, has_q_series = false;
  TimeSeries z_series, q_series;
};

struct SamplePoint {
  int x, y;
  std::string label;
  SampleType type;
};

struct Config {
  std::string yaml_path;
  std::string name;
  size_t W = 0, H = 0;
  float dx = 0.f, dt = 0.f;
  bool variable_dt = true;
  Solver solver = Solver::rmg;
  double target_duration = 0.0;
  float kst_fixed = 30.f;
  float no_data = -9999.f;
  bool has_kst_var = false;
  std::vector<float> terrain;   // h_sohle
  std::vector<float> h0;        // initial depth: z - terrain, or 0
  std::vector<float> qx0, qy0;  // initial discharges, or 0
  std::vector<float> kst;       // kSt_var grid when has_kst_var
  std::vector<BoundaryCondition> bcs;
  int sampling_interval = 0;
  std::vector<SamplePoint> points;
  std::vector<double> save_times;  // sorted

  bool staggered() const { return solver == Solver::rmg; }
  // BoundaryCondition::sumWaterDepths (src/boundary_condition.cpp:6-18), host float
  float sum_water_depths(const BoundaryCondition& bc, float z_soll) const;
  // BoundaryCondition::getZ / getQ for a condition without time series
  float const_z(const BoundaryCondition& bc) const { return bc.z; }
  float const_q(const BoundaryCondition& bc) const;
};

// utils::solveSimpleMathExpression (src/utils.h:29-43): products of floats only.
double solve_simple_math(const std::string& expr);

// Loads and validates a parameter file (SimData::loadSimData, src/simdata.cpp:238-310).
// Validation messages and warnings go to stderr with the reference's wording; on failure the
// return value is nonzero and *err holds the message the reference's main() prints after
// "Config error: ". Returns 2 for I/O errors on the input files. With `quiet` the warnings (no
// save_state times, default kSt) are not printed; errors always are.
int load_config(const std::string& path, Config* out, std::string* err, bool quiet = false);

}  // namespace fip

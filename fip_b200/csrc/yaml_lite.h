// Minimal YAML reader for fip parameter files (the schema of the reference's README.md:46-64).
// Supports block mappings and sequences, flow sequences [a, b] and flow mappings {k: v},
// plain / single- / double-quoted scalars and # comments. Every node keeps the 0-based line it
// starts on, for "Config error at line N" messages (src/simdata.cpp:156-159).
// Conversions mirror the yaml-cpp ones the reference relies on: as<T>() throws on a bad scalar,
// as<T>(fallback) returns the fallback when the node is missing or does not convert.
#pragma once
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace fip {

struct YamlError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

class YNode {
 public:
  enum Kind { Undefined, Null, Scalar, Sequence, Map };

  YNode() = default;
  Kind kind() const { return kind_; }
  bool defined() const { return kind_ != Undefined; }
  bool is_scalar() const { return kind_ == Scalar; }
  bool is_sequence() const { return kind_ == Sequence; }
  bool is_map() const { return kind_ == Map; }
  int line() const { return line_; }
  size_t size() const;

  // map lookup (Undefined node when absent or not a map); sequence index
  const YNode& operator[](const std::string& key) const;
  const YNode& operator[](size_t i) const;
  const std::vector<std::pair<std::string, YNode>>& items() const { return map_; }
  const std::vector<YNode>& seq() const { return seq_; }

  std::string as_string() const;  // throws if not a scalar
  int as_int() const;
  long long as_int64() const;
  float as_float() const;
  bool as_bool() const;
  bool try_int(int* out) const;
  bool try_float(float* out) const;
  bool try_bool(bool* out) const;
  int as_int(int fallback) const;
  float as_float(float fallback) const;
  bool as_bool(bool fallback) const;

  static YNode parse(const std::string& text);  // throws YamlError
  static YNode load_file(const std::string& path);

  // builders (used by the parser)
  static YNode make_scalar(const std::string& s, int line, bool quoted);
  static YNode make_null(int line);
  static YNode make_seq(int line);
  static YNode make_map(int line);
  void push(YNode n) { seq_.push_back(std::move(n)); }
  void set(const std::string& k, YNode n);

 private:
  Kind kind_ = Undefined;
  int line_ = -1;
  bool quoted_ = false;
  std::string scalar_;
  std::vector<YNode> seq_;
  std::vector<std::pair<std::string, YNode>> map_;
};

}  // namespace fip

#include "yaml_lite.h"

#include <cctype>
#include <cmath>
#include <cerrno>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>

namespace fip {

namespace {

const YNode& undefined_node() {
  static const YNode u;
  return u;
}

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

struct Line {
  int indent;
  std::string text;  // without indentation and comment
  int no;            // 0-based line number
};

// Removes a # comment that is not inside quotes and starts the line or follows whitespace.
std::string strip_comment(const std::string& s) {
  char q = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    char c = s[i];
    if (q) {
      if (c == q) {
        if (q == '\'' && i + 1 < s.size() && s[i + 1] == '\'') {
          ++i;
          continue;
        }
        q = 0;
      } else if (q == '"' && c == '\\') {
        ++i;
      }
      continue;
    }
    if (c == '"' || c == '\'') {
      // a quote only opens a quoted scalar at the start of a token
      if (i == 0 || std::isspace((unsigned char)s[i - 1]) || s[i - 1] == '[' || s[i - 1] == '{' || s[i - 1] == ',' ||
          s[i - 1] == ':' || s[i - 1] == '-')
        q = c;
      continue;
    }
    if (c == '#' && (i == 0 || std::isspace((unsigned char)s[i - 1]))) return s.substr(0, i);
  }
  return s;
}

// position of the ": " (or trailing ':') that separates a mapping key, outside quotes/brackets
size_t find_key_colon(const std::string& s) {
  char q = 0;
  int depth = 0;
  for (size_t i = 0; i < s.size(); ++i) {
    char c = s[i];
    if (q) {
      if (c == q) q = 0;
      continue;
    }
    if ((c == '"' || c == '\'') && (i == 0)) {
      q = c;
      continue;
    }
    if (c == '[' || c == '{') ++depth;
    if (c == ']' || c == '}') --depth;
    if (c == ':' && depth == 0 && (i + 1 == s.size() || s[i + 1] == ' ' || s[i + 1] == '\t')) return i;
  }
  return std::string::npos;
}

std::string unquote(const std::string& s, bool* quoted) {
  *quoted = false;
  if (s.size() >= 2 && s.front() == '\'' && s.back() == '\'') {
    *quoted = true;
    std::string r;
    for (size_t i = 1; i + 1 < s.size(); ++i) {
      if (s[i] == '\'' && i + 2 < s.size() && s[i + 1] == '\'') ++i;
      r += s[i];
    }
    return r;
  }
  if (s.size() >= 2 && s.front() == '"' && s.back() == '"') {
    *quoted = true;
    std::string r;
    for (size_t i = 1; i + 1 < s.size(); ++i) {
      if (s[i] == '\\' && i + 2 < s.size()) {
        char e = s[++i];
        switch (e) {
          case 'n': r += '\n'; break;
          case 't': r += '\t'; break;
          case '\\': r += '\\'; break;
          case '"': r += '"'; break;
          default: r += '\\'; r += e; break;
        }
      } else {
        r += s[i];
      }
    }
    return r;
  }
  return s;
}

YNode scalar_node(const std::string& raw, int line) {
  std::string t = trim(raw);
  if (t.empty() || t == "~" || t == "null" || t == "Null" || t == "NULL") return YNode::make_null(line);
  bool quoted;
  std::string v = unquote(t, &quoted);
  return YNode::make_scalar(v, line, quoted);
}

// ---- flow collections -------------------------------------------------------------------
struct FlowParser {
  const std::string& s;
  size_t i;
  int line;
  void ws() {
    while (i < s.size() && std::isspace((unsigned char)s[i])) ++i;
  }
  [[noreturn]] void fail(const std::string& m) {
    throw YamlError("yaml: line " + std::to_string(line + 1) + ": " + m);
  }
  std::string token() {  // scalar up to , ] } or ': ' (mapping separator)
    ws();
    if (i < s.size() && (s[i] == '"' || s[i] == '\'')) {
      char q = s[i];
      size_t j = i + 1;
      while (j < s.size()) {
        if (s[j] == q) {
          if (q == '\'' && j + 1 < s.size() && s[j + 1] == '\'') {
            j += 2;
            continue;
          }
          break;
        }
        if (q == '"' && s[j] == '\\') ++j;
        ++j;
      }
      if (j >= s.size()) fail("unterminated quoted scalar");
      std::string r = s.substr(i, j + 1 - i);
      i = j + 1;
      return r;
    }
    size_t j = i;
    while (j < s.size() && s[j] != ',' && s[j] != ']' && s[j] != '}' &&
           !(s[j] == ':' && (j + 1 == s.size() || s[j + 1] == ' ' || s[j + 1] == ',' || s[j + 1] == '}')))
      ++j;
    std::string r = trim(s.substr(i, j - i));
    i = j;
    return r;
  }
  YNode value() {
    ws();
    if (i >= s.size()) fail("unexpected end of flow collection");
    if (s[i] == '[') {
      ++i;
      YNode n = YNode::make_seq(line);
      ws();
      if (i < s.size() && s[i] == ']') {
        ++i;
        return n;
      }
      for (;;) {
        n.push(value());
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == ']') {
          ++i;
          return n;
        }
        fail("expected ',' or ']'");
      }
    }
    if (s[i] == '{') {
      ++i;
      YNode n = YNode::make_map(line);
      ws();
      if (i < s.size() && s[i] == '}') {
        ++i;
        return n;
      }
      for (;;) {
        std::string k = token();
        bool q;
        k = unquote(k, &q);
        ws();
        if (i < s.size() && s[i] == ':') {
          ++i;
          n.set(k, value());
        } else {
          n.set(k, YNode::make_null(line));
        }
        ws();
        if (i < s.size() && s[i] == ',') {
          ++i;
          continue;
        }
        if (i < s.size() && s[i] == '}') {
          ++i;
          return n;
        }
        fail("expected ',' or '}'");
      }
    }
    return scalar_node(token(), line);
  }
};

// ---- block structure ---------------------------------------------------------------------
struct BlockParser {
  std::vector<Line> L;
  size_t p = 0;

  [[noreturn]] void fail(int line, const std::string& m) {
    throw YamlError("yaml: line " + std::to_string(line + 1) + ": " + m);
  }

  YNode flow_or_scalar(const std::string& text, int line) {
    std::string t = trim(text);
    if (!t.empty() && (t[0] == '[' || t[0] == '{')) {
      // a flow collection may continue on the following lines until its brackets close
      std::string acc = t;
      auto balanced = [](const std::string& s) {
        int d = 0;
        char q = 0;
        for (char c : s) {
          if (q) {
            if (c == q) q = 0;
            continue;
          }
          if (c == '"' || c == '\'') q = c;
          if (c == '[' || c == '{') ++d;
          if (c == ']' || c == '}') --d;
        }
        return d <= 0;
      };
      while (!balanced(acc) && p < L.size()) acc += " " + L[p++].text;
      FlowParser fp{acc, 0, line};
      YNode n = fp.value();
      fp.ws();
      if (fp.i != acc.size()) fail(line, "trailing characters after flow collection");
      return n;
    }
    return scalar_node(t, line);
  }

  // value of "key:" with nothing after the colon: a nested block, or null
  YNode nested(int parent_indent, int line, bool allow_same_indent_seq) {
    if (p < L.size()) {
      const Line& n = L[p];
      bool is_seq = n.text.size() >= 1 && n.text[0] == '-' && (n.text.size() == 1 || n.text[1] == ' ');
      if (n.indent > parent_indent || (allow_same_indent_seq && n.indent == parent_indent && is_seq))
        return block(n.indent);
    }
    return YNode::make_null(line);
  }

  YNode block(int indent) {
    const Line& first = L[p];
    bool is_seq = first.text[0] == '-' && (first.text.size() == 1 || first.text[1] == ' ');
    if (is_seq) {
      YNode seq = YNode::make_seq(first.no);
      while (p < L.size() && L[p].indent == indent && L[p].text[0] == '-' &&
             (L[p].text.size() == 1 || L[p].text[1] == ' ')) {
        Line cur = L[p++];
        std::string rest = cur.text.size() > 1 ? cur.text.substr(1) : "";
        size_t off = 1;
        while (off < cur.text.size() && cur.text[off] == ' ') ++off;
        rest = trim(rest);
        if (rest.empty()) {
          seq.push(nested(indent, cur.no, false));
        } else if (find_key_colon(rest) != std::string::npos && rest[0] != '[' && rest[0] != '{') {
          // "- key: value": a mapping whose indentation is the column of its first key
          --p;
          L[p].indent = indent + (int)off;
          L[p].text = rest;
          seq.push(block(L[p].indent));
        } else {
          seq.push(flow_or_scalar(rest, cur.no));
        }
      }
      return seq;
    }
    if (find_key_colon(first.text) == std::string::npos) {
      // a lone scalar line
      Line cur = L[p++];
      return flow_or_scalar(cur.text, cur.no);
    }
    YNode map = YNode::make_map(first.no);
    while (p < L.size() && L[p].indent == indent) {
      Line cur = L[p++];
      size_t k = find_key_colon(cur.text);
      if (k == std::string::npos) fail(cur.no, "expected 'key: value'");
      bool q;
      std::string key = unquote(trim(cur.text.substr(0, k)), &q);
      std::string rest = trim(cur.text.substr(k + 1));
      if (rest.empty())
        map.set(key, nested(indent, cur.no, true));
      else
        map.set(key, flow_or_scalar(rest, cur.no));
    }
    if (p < L.size() && L[p].indent > indent) fail(L[p].no, "bad indentation");
    return map;
  }
};

bool parse_int64(const std::string& s0, long long* out) {
  std::string s = trim(s0);
  if (s.empty()) return false;
  const char* b = s.c_str();
  char* e = nullptr;
  errno = 0;
  long long v = std::strtoll(b, &e, 0);
  if (e == b || errno) return false;
  while (*e && std::isspace((unsigned char)*e)) ++e;
  if (*e) return false;
  *out = v;
  return true;
}

}  // namespace

size_t YNode::size() const {
  if (kind_ == Sequence) return seq_.size();
  if (kind_ == Map) return map_.size();
  return 0;
}

const YNode& YNode::operator[](const std::string& key) const {
  if (kind_ != Map) return undefined_node();
  for (const auto& kv : map_)
    if (kv.first == key) return kv.second;
  return undefined_node();
}

const YNode& YNode::operator[](size_t i) const {
  if (kind_ != Sequence || i >= seq_.size()) return undefined_node();
  return seq_[i];
}

std::string YNode::as_string() const {
  if (kind_ == Scalar) return scalar_;
  if (kind_ == Null) return "null";
  throw YamlError("bad conversion" + (line_ >= 0 ? " at line " + std::to_string(line_ + 1) : std::string()));
}

bool YNode::try_int(int* out) const {
  long long v;
  if (kind_ != Scalar || !parse_int64(scalar_, &v)) return false;
  if (v < std::numeric_limits<int>::min() || v > std::numeric_limits<int>::max()) return false;
  *out = (int)v;
  return true;
}

bool YNode::try_float(float* out) const {
  if (kind_ != Scalar) return false;
  std::string s = trim(scalar_);
  if (s == ".inf" || s == ".Inf" || s == ".INF" || s == "+.inf" || s == "+.Inf" || s == "+.INF") {
    *out = std::numeric_limits<float>::infinity();
    return true;
  }
  if (s == "-.inf" || s == "-.Inf" || s == "-.INF") {
    *out = -std::numeric_limits<float>::infinity();
    return true;
  }
  if (s == ".nan" || s == ".NaN" || s == ".NAN") {
    *out = std::numeric_limits<float>::quiet_NaN();
    return true;
  }
  std::istringstream is(s);
  float v;
  is >> v;
  if (is.fail()) return false;
  is >> std::ws;
  if (!is.eof()) return false;
  *out = v;
  return true;
}

bool YNode::try_bool(bool* out) const {
  if (kind_ != Scalar) return false;
  static const char* t[] = {"y", "Y", "yes", "Yes", "YES", "true", "True", "TRUE", "on", "On", "ON"};
  static const char* f[] = {"n", "N", "no", "No", "NO", "false", "False", "FALSE", "off", "Off", "OFF"};
  for (const char* x : t)
    if (scalar_ == x) {
      *out = true;
      return true;
    }
  for (const char* x : f)
    if (scalar_ == x) {
      *out = false;
      return true;
    }
  return false;
}

static YamlError bad_conv(const YNode& n) {
  return YamlError("bad conversion" + (n.line() >= 0 ? " at line " + std::to_string(n.line() + 1) : std::string()));
}

int YNode::as_int() const {
  int v;
  if (!try_int(&v)) throw bad_conv(*this);
  return v;
}
long long YNode::as_int64() const {
  long long v;
  if (kind_ != Scalar || !parse_int64(scalar_, &v)) throw bad_conv(*this);
  return v;
}
float YNode::as_float() const {
  float v;
  if (!try_float(&v)) throw bad_conv(*this);
  return v;
}
bool YNode::as_bool() const {
  bool v;
  if (!try_bool(&v)) throw bad_conv(*this);
  return v;
}
int YNode::as_int(int fb) const {
  int v;
  return try_int(&v) ? v : fb;
}
float YNode::as_float(float fb) const {
  float v;
  return try_float(&v) ? v : fb;
}
bool YNode::as_bool(bool fb) const {
  bool v;
  return try_bool(&v) ? v : fb;
}

YNode YNode::make_scalar(const std::string& s, int line, bool quoted) {
  YNode n;
  n.kind_ = Scalar;
  n.scalar_ = s;
  n.line_ = line;
  n.quoted_ = quoted;
  return n;
}
YNode YNode::make_null(int line) {
  YNode n;
  n.kind_ = Null;
  n.line_ = line;
  return n;
}
YNode YNode::make_seq(int line) {
  YNode n;
  n.kind_ = Sequence;
  n.line_ = line;
  return n;
}
YNode YNode::make_map(int line) {
  YNode n;
  n.kind_ = Map;
  n.line_ = line;
  return n;
}
void YNode::set(const std::string& k, YNode n) {
  for (auto& kv : map_)
    if (kv.first == k) return;  // first definition wins
  map_.emplace_back(k, std::move(n));
}

YNode YNode::parse(const std::string& text) {
  BlockParser bp;
  std::istringstream is(text);
  std::string raw;
  int no = 0;
  while (std::getline(is, raw)) {
    if (!raw.empty() && raw.back() == '\r') raw.pop_back();
    std::string s = strip_comment(raw);
    int ind = 0;
    while (ind < (int)s.size() && s[ind] == ' ') ++ind;
    if (ind < (int)s.size() && s[ind] == '\t') throw YamlError("yaml: line " + std::to_string(no + 1) + ": tab indentation");
    std::string t = trim(s);
    if (!t.empty() && t != "---" && t != "...") bp.L.push_back(Line{ind, t, no});
    ++no;
  }
  if (bp.L.empty()) return make_null(0);
  YNode root = bp.block(bp.L[0].indent);
  if (bp.p != bp.L.size()) throw YamlError("yaml: line " + std::to_string(bp.L[bp.p].no + 1) + ": unexpected content");
  return root;
}

YNode YNode::load_file(const std::string& path) {
  std::ifstream f(path, std::ios::binary);
  if (!f) throw YamlError("bad file: " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  return parse(ss.str());
}

}  // namespace fip

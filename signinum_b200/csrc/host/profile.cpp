// Environment-gated profiling rows (see profile.h).
#include "profile.h"

#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>

namespace sgn {
namespace prof {

namespace {

bool ieq(const std::string& a, const char* b) {
  if (a.size() != std::strlen(b)) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::tolower((unsigned char)a[i]) != std::tolower((unsigned char)b[i])) return false;
  return true;
}

std::string trim(const char* v) {
  std::string s(v);
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

bool timing_field(const std::string& k) {
  auto ends = [&](const char* suf) {
    const size_t n = std::strlen(suf);
    return k.size() >= n && k.compare(k.size() - n, n, suf) == 0;
  };
  return ends("_us") || ends("_ms") || ends("_ns");
}

bool parse_u64(const std::string& v, unsigned long long& out) {
  if (v.empty()) return false;
  for (char c : v)
    if (c < '0' || c > '9') return false;
  out = std::strtoull(v.c_str(), nullptr, 10);
  return true;
}

struct Key {
  std::string codec, op, path;
  std::vector<std::pair<std::string, std::string>> labels;
  bool operator<(const Key& o) const {
    if (codec != o.codec) return codec < o.codec;
    if (op != o.op) return op < o.op;
    if (path != o.path) return path < o.path;
    return labels < o.labels;
  }
};

struct Row {
  unsigned long long count = 0;
  std::map<std::string, unsigned long long> sums;
};

// One thread's aggregated events; printed when the thread ends (the main
// thread's at process exit), as ProfileSummary's Drop does.
struct Summary {
  std::map<Key, Row> rows;
  ~Summary() {
    for (const auto& kv : rows) {
      std::string line = "signinum_profile_summary codec=" + kv.first.codec + " op=" + kv.first.op +
                         " path=" + kv.first.path;
      for (const auto& l : kv.first.labels) line += " " + l.first + "=" + l.second;
      line += " count=" + std::to_string(kv.second.count);
      for (const auto& s : kv.second.sums) {
        line += " " + s.first + "_sum=" + std::to_string(s.second);
        if (timing_field(s.first)) line += " " + s.first + "_avg=" + std::to_string(s.second / kv.second.count);
      }
      std::fprintf(stderr, "%s\n", line.c_str());
    }
  }
};

thread_local Summary t_stage_summary;
thread_local Summary t_route_summary;

const char* const kRouteLabels[][2] = {{"op", "route_op"}, {"request", "request"}, {"fmt", "fmt"},
                                       {"decision", "decision"}, {"reason", "reason"},
                                       {"has_fast_packet", "has_fast_packet"},
                                       {"supports_output_format", "supports_output_format"},
                                       {"hardware_decode", "hardware_decode"}};

}  // namespace

Mode mode_from_value(const char* value) {
  if (!value) return Mode::Disabled;
  const std::string v = trim(value);
  if (ieq(v, "summary") || ieq(v, "summaries") || ieq(v, "aggregate") || ieq(v, "aggregates")) return Mode::Summary;
  for (const char* t : {"1", "true", "t", "yes", "y", "on", "enable", "enabled"})
    if (ieq(v, t)) return Mode::Rows;
  return Mode::Disabled;
}

Mode stage_mode() {
  static const Mode m = mode_from_value(std::getenv("SIGNINUM_J2K_PROFILE_STAGES"));
  return m;
}

Mode route_mode() {
  static const Mode m = mode_from_value(std::getenv("SIGNINUM_GPU_ROUTE_PROFILE"));
  return m;
}

std::string format_row(const char* codec, const char* op, const char* path, const Fields& fields) {
  std::string row = std::string("signinum_profile codec=") + codec + " op=" + op + " path=" + path;
  for (const auto& f : fields) row += " " + f.first + "=" + f.second;
  return row;
}

void emit_stages(const char* codec, const char* op, const char* path, const Fields& fields) {
  const Mode m = stage_mode();
  if (m == Mode::Rows) {
    std::fprintf(stderr, "%s\n", format_row(codec, op, path, fields).c_str());
  } else if (m == Mode::Summary) {
    Row& r = t_stage_summary.rows[Key{codec, op, path, {}}];
    ++r.count;
    for (const auto& f : fields) {
      unsigned long long v;
      if (parse_u64(f.second, v)) r.sums[f.first] += v;
    }
  }
}

void emit_route(const char* codec, const char* path, const Fields& fields) {
  const Mode m = route_mode();
  if (m == Mode::Rows) {
    std::fprintf(stderr, "%s\n", format_row(codec, "gpu_route", path, fields).c_str());
  } else if (m == Mode::Summary) {
    Key k{codec, "gpu_route", path, {}};
    for (const auto& lab : kRouteLabels)
      for (const auto& f : fields)
        if (f.first == lab[0]) {
          k.labels.emplace_back(lab[1], f.second);
          break;
        }
    ++t_route_summary.rows[k].count;
  }
}

}  // namespace prof
}  // namespace sgn

// JSON -> Config, mirroring draugr_amg_config_from_json
// (src/cfunction_interface.jl:34-221 of Draugr.jl): all keys optional and
// case-sensitive, string values case-insensitive, numbers may arrive as
// strings, unknown keys ignored, unknown names are an error that lists the
// valid names.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <sstream>

#include "dr_host.h"

namespace dr {

void fail(const std::string& msg) { throw Error(msg); }

namespace {

// ----------------------------------------------------------------- JSON value
struct JVal {
  enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
  bool b = false;
  double num = 0.0;
  bool is_int = false;
  std::string s;
  std::vector<std::shared_ptr<JVal>> arr;
  std::map<std::string, std::shared_ptr<JVal>> obj;
};
using JPtr = std::shared_ptr<JVal>;

struct Parser {
  const char* begin;
  const char* p;
  const char* end;
  explicit Parser(const char* s) : begin(s), p(s), end(s + std::strlen(s)) {}
  void ws() {
    while (p < end && std::isspace((unsigned char)*p)) ++p;
  }
  [[noreturn]] void bad(const char* what) {
    std::ostringstream o;
    o << "JSON parse error: " << what << " at offset " << (long)(p - begin);
    fail(o.str());
  }
  JPtr value() {
    ws();
    if (p >= end) bad("unexpected end of input");
    auto v = std::make_shared<JVal>();
    char c = *p;
    if (c == '{') {
      v->kind = JVal::Obj;
      ++p;
      ws();
      if (p < end && *p == '}') { ++p; return v; }
      for (;;) {
        ws();
        if (p >= end || *p != '"') bad("expected string key");
        std::string k = string();
        ws();
        if (p >= end || *p != ':') bad("expected ':'");
        ++p;
        v->obj[k] = value();
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == '}') { ++p; break; }
        bad("expected ',' or '}'");
      }
    } else if (c == '[') {
      v->kind = JVal::Arr;
      ++p;
      ws();
      if (p < end && *p == ']') { ++p; return v; }
      for (;;) {
        v->arr.push_back(value());
        ws();
        if (p < end && *p == ',') { ++p; continue; }
        if (p < end && *p == ']') { ++p; break; }
        bad("expected ',' or ']'");
      }
    } else if (c == '"') {
      v->kind = JVal::Str;
      v->s = string();
    } else if (!std::strncmp(p, "true", 4)) {
      v->kind = JVal::Bool; v->b = true; p += 4;
    } else if (!std::strncmp(p, "false", 5)) {
      v->kind = JVal::Bool; v->b = false; p += 5;
    } else if (!std::strncmp(p, "null", 4)) {
      v->kind = JVal::Null; p += 4;
    } else if (c == '-' || (c >= '0' && c <= '9')) {
      const char* s = p;
      if (*p == '-') ++p;
      bool frac = false;
      while (p < end && (std::isdigit((unsigned char)*p) || *p == '.' || *p == 'e' ||
                         *p == 'E' || *p == '+' || *p == '-')) {
        if (*p == '.' || *p == 'e' || *p == 'E') frac = true;
        ++p;
      }
      std::string tok(s, p);
      char* e2 = nullptr;
      v->num = std::strtod(tok.c_str(), &e2);
      if (!e2 || *e2) bad("bad number");
      v->kind = JVal::Num;
      v->is_int = !frac;
      v->s = tok;
    } else {
      bad("unexpected character");
    }
    return v;
  }
  std::string string() {
    ++p;  // opening quote
    std::string out;
    while (p < end && *p != '"') {
      if (*p == '\\') {
        ++p;
        if (p >= end) bad("bad escape");
        switch (*p) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (end - p < 5) bad("bad \\u escape");
            unsigned cp = (unsigned)std::strtoul(std::string(p + 1, p + 5).c_str(), nullptr, 16);
            if (cp < 0x80) out += (char)cp;
            else if (cp < 0x800) { out += (char)(0xC0 | (cp >> 6)); out += (char)(0x80 | (cp & 0x3F)); }
            else { out += (char)(0xE0 | (cp >> 12)); out += (char)(0x80 | ((cp >> 6) & 0x3F)); out += (char)(0x80 | (cp & 0x3F)); }
            p += 4;
            break;
          }
          default: bad("bad escape");
        }
        ++p;
      } else {
        out += *p++;
      }
    }
    if (p >= end) bad("unterminated string");
    ++p;
    return out;
  }
};

std::string lower(std::string s) {
  for (auto& c : s) c = (char)std::tolower((unsigned char)c);
  return s;
}

// string(v) in Julia for the scalar kinds used here.
std::string jstr(const JPtr& v) {
  switch (v->kind) {
    case JVal::Str: return v->s;
    case JVal::Bool: return v->b ? "true" : "false";
    case JVal::Num: return v->s;
    case JVal::Null: return "nothing";
    case JVal::Arr: return "array";
    case JVal::Obj: return "object";
  }
  return "";
}

// _to_float / _to_int / _to_bool / _to_string (cfunction_interface.jl:34-43).
double to_float(const JPtr& v) {
  if (v->kind == JVal::Num) return v->num;
  if (v->kind == JVal::Bool) return v->b ? 1.0 : 0.0;
  std::string s = jstr(v);
  char* e = nullptr;
  double d = std::strtod(s.c_str(), &e);
  if (s.empty() || !e || *e) fail("ArgumentError: cannot parse \"" + s + "\" as Float64");
  return d;
}
long to_int(const JPtr& v) {
  if (v->kind == JVal::Num) return (long)std::nearbyint(v->num);  // round-half-even
  if (v->kind == JVal::Bool) return v->b ? 1 : 0;
  std::string s = jstr(v);
  char* e = nullptr;
  long d = std::strtol(s.c_str(), &e, 10);
  if (s.empty() || !e || *e) fail("ArgumentError: invalid base 10 digit in \"" + s + "\"");
  return d;
}
bool to_bool(const JPtr& v) {
  if (v->kind == JVal::Bool) return v->b;
  std::string s = lower(jstr(v));
  return s == "true" || s == "1";
}
std::string to_string(const JPtr& v) { return lower(jstr(v)); }

template <class T>
T lookup(const std::map<std::string, T>& table, const std::string& name, const char* label) {
  auto it = table.find(name);
  if (it != table.end()) return it->second;
  std::string valid;
  for (auto& kv : table) {  // std::map iterates in sorted key order
    if (!valid.empty()) valid += ", ";
    valid += kv.first;
  }
  fail(std::string("Unknown ") + label + ": \"" + name + "\". Valid: " + valid);
}

JPtr get(const JPtr& d, const char* key) {
  if (!d || d->kind != JVal::Obj) return nullptr;
  auto it = d->obj.find(key);
  if (it == d->obj.end()) return nullptr;
  return it->second;
}

const std::map<std::string, SmootherKind>& smoother_table() {
  static const std::map<std::string, SmootherKind> t = {
      {"jacobi", SmootherKind::Jacobi},           {"colored_gs", SmootherKind::ColoredGS},
      {"serial_gs", SmootherKind::SerialGS},      {"spai0", SmootherKind::SPAI0},
      {"spai1", SmootherKind::SPAI1},             {"l1_jacobi", SmootherKind::L1Jacobi},
      {"l1_colored_gs", SmootherKind::L1ColoredGS}, {"l1_serial_gs", SmootherKind::L1SerialGS},
      {"chebyshev", SmootherKind::Chebyshev},     {"ilu0", SmootherKind::ILU0},
      {"serial_ilu0", SmootherKind::SerialILU0},
  };
  return t;
}

Interp parse_interp_named(const std::string& name, const JPtr& d) {
  static const std::map<std::string, InterpKind> t = {
      {"direct", InterpKind::Direct},
      {"standard", InterpKind::Standard},
      {"extended_i", InterpKind::ExtendedI},
  };
  Interp ip;
  ip.kind = lookup(t, name, "interpolation");
  if (JPtr v = get(d, "trunc_factor")) ip.trunc_factor = to_float(v);
  if (ip.kind == InterpKind::ExtendedI) {
    if (JPtr v = get(d, "max_elements")) ip.max_elements = (int)to_int(v);
    if (JPtr v = get(d, "norm_p")) ip.norm_p = (int)to_int(v);
    if (JPtr v = get(d, "rescale")) ip.rescale = to_bool(v);
  }
  return ip;
}

Interp parse_interpolation(const JPtr& v) {
  if (!v) return parse_interp_named("extended_i", nullptr);
  if (v->kind == JVal::Str) return parse_interp_named(lower(v->s), nullptr);
  if (v->kind == JVal::Obj) {
    JPtr t = get(v, "type");
    std::string name = t ? to_string(t) : std::string("extended_i");
    return parse_interp_named(name, v);
  }
  fail("\"interpolation\" must be a string or object, got: " + jstr(v));
}

Coarsening parse_coarsening(const JPtr& v, double theta, const Interp& ip) {
  static const std::map<std::string, CoarsenKind> t = {
      {"aggregation", CoarsenKind::Aggregation},
      {"pmis", CoarsenKind::PMIS},
      {"hmis", CoarsenKind::HMIS},
      {"rs", CoarsenKind::RS},
      {"aggressive_pmis", CoarsenKind::AggressivePMIS},
      {"aggressive_hmis", CoarsenKind::AggressiveHMIS},
      {"smoothed_aggregation", CoarsenKind::SmoothedAggregation},
  };
  std::string name = v ? to_string(v) : std::string("hmis");
  Coarsening c;
  c.kind = lookup(t, name, "coarsening");
  c.theta = theta;
  c.interp = ip;
  if (c.kind == CoarsenKind::Aggregation || c.kind == CoarsenKind::SmoothedAggregation) {
    c.interp = Interp();  // aggregation ignores the interpolation argument
  }
  return c;
}

}  // namespace

Config default_config() {
  Config c;
  c.coarsening.kind = CoarsenKind::HMIS;
  c.coarsening.theta = 0.5;
  c.coarsening.interp = Interp();
  c.initial_coarsening = c.coarsening;
  return c;
}

Config hypre_default_config(double agg_trunc_factor) {
  // src/types.jl:569-584
  Config c = default_config();
  Interp ip;
  ip.kind = InterpKind::ExtendedI;
  ip.trunc_factor = agg_trunc_factor;
  c.coarsening.kind = CoarsenKind::HMIS;
  c.coarsening.theta = 0.5;
  c.coarsening.interp = ip;
  c.initial_coarsening.kind = CoarsenKind::AggressiveHMIS;
  c.initial_coarsening.theta = 0.5;
  c.initial_coarsening.interp = ip;
  c.initial_coarsening_levels = 1;
  return c;
}

Config config_from_json(const char* json) {
  const char* src = json ? json : "{}";
  Parser ps(src);
  JPtr d = ps.value();
  ps.ws();
  if (ps.p != ps.end) fail("JSON parse error: trailing characters");
  if (d->kind != JVal::Obj) fail("JSON config must be an object");

  Config c = default_config();
  Interp ip = parse_interpolation(get(d, "interpolation"));
  double theta = 0.5;
  if (JPtr v = get(d, "theta")) theta = to_float(v);
  c.coarsening = parse_coarsening(get(d, "coarsening"), theta, ip);
  JPtr ic = get(d, "initial_coarsening");
  // Extensions: "initial_theta" / "initial_interpolation" give the initial
  // coarsening its own θ and interpolation (the reference's JSON shares
  // one θ and one interpolation between both).
  double itheta = theta;
  if (JPtr v = get(d, "initial_theta")) itheta = to_float(v);
  Interp iip = ip;
  if (JPtr v = get(d, "initial_interpolation")) iip = parse_interpolation(v);
  if (ic && ic->kind != JVal::Null)
    c.initial_coarsening = parse_coarsening(ic, itheta, iip);
  else
    c.initial_coarsening = c.coarsening;
  // Extensions for aggregation-type coarsening options that the reference
  // only exposes through its Julia constructors.
  for (Coarsening* cc : {&c.coarsening, &c.initial_coarsening}) {
    if (JPtr v = get(d, "aggregation_filtering")) cc->filtering = to_bool(v);
    if (JPtr v = get(d, "filter_tol")) cc->filter_tol = to_float(v);
    if (JPtr v = get(d, "sa_omega")) cc->sa_omega = to_float(v);
  }

  double omega_override = NAN;
  bool has_override = false;
  JPtr sm = get(d, "smoother");
  if (!sm) {
    c.smoother = SmootherKind::L1ColoredGS;
  } else if (sm->kind == JVal::Str) {
    c.smoother = lookup(smoother_table(), lower(sm->s), "smoother");
  } else if (sm->kind == JVal::Obj) {
    JPtr t = get(sm, "type");
    std::string name = t ? to_string(t) : std::string("l1_colored_gs");
    c.smoother = lookup(smoother_table(), name, "smoother");
    if (JPtr o = get(sm, "omega")) { omega_override = to_float(o); has_override = true; }
  } else {
    fail("\"smoother\" must be a string or object, got: " + jstr(sm));
  }
  if (has_override) c.jacobi_omega = omega_override;
  else if (JPtr v = get(d, "jacobi_omega")) c.jacobi_omega = to_float(v);

  if (JPtr v = get(d, "strength")) {
    static const std::map<std::string, StrengthKind> t = {{"absolute", StrengthKind::Absolute},
                                                          {"signed", StrengthKind::Signed}};
    c.strength = lookup(t, to_string(v), "strength");
  }
  if (JPtr v = get(d, "cycle")) {
    static const std::map<std::string, bool> t = {{"v", false}, {"w", true}};
    c.cycle_w = lookup(t, to_string(v), "cycle");
  }
  if (JPtr v = get(d, "max_levels")) c.max_levels = (int)to_int(v);
  if (JPtr v = get(d, "max_coarse_size")) c.max_coarse_size = (int)to_int(v);
  if (JPtr v = get(d, "pre_smoothing_steps")) c.pre_smoothing_steps = (int)to_int(v);
  if (JPtr v = get(d, "post_smoothing_steps")) c.post_smoothing_steps = (int)to_int(v);
  if (JPtr v = get(d, "verbose")) c.verbose = (int)to_int(v);
  if (JPtr v = get(d, "initial_coarsening_levels")) c.initial_coarsening_levels = (int)to_int(v);
  if (JPtr v = get(d, "max_row_sum")) c.max_row_sum = to_float(v);
  if (JPtr v = get(d, "coarse_solve_on_cpu")) c.coarse_solve_on_cpu = to_bool(v);
  // Extension: seed of the random PMIS/HMIS measures (the reference draws
  // them from an unseeded global generator).  Unknown to the reference, so
  // a reference caller never sets it.
  if (JPtr v = get(d, "seed")) c.seed = (uint64_t)to_int(v);
  return c;
}

std::string smoother_name(SmootherKind k) {
  for (auto& kv : smoother_table())
    if (kv.second == k) return kv.first;
  return "?";
}

std::string coarsening_name(const Coarsening& c) {
  std::ostringstream o;
  const char* in = c.interp.kind == InterpKind::Direct     ? "DirectInterpolation"
                   : c.interp.kind == InterpKind::Standard ? "StandardInterpolation"
                                                           : "ExtendedIInterpolation";
  switch (c.kind) {
    case CoarsenKind::Aggregation: o << "Aggregation(θ=" << c.theta << (c.filtering ? ", filtered)" : ")"); break;
    case CoarsenKind::PMIS: o << "PMIS(θ=" << c.theta << ", " << in << ")"; break;
    case CoarsenKind::HMIS: o << "HMIS(θ=" << c.theta << ", " << in << ")"; break;
    case CoarsenKind::RS: o << "RS(θ=" << c.theta << ", " << in << ")"; break;
    case CoarsenKind::AggressivePMIS: o << "Aggressive(θ=" << c.theta << ", base=pmis, " << in << ")"; break;
    case CoarsenKind::AggressiveHMIS: o << "Aggressive(θ=" << c.theta << ", base=hmis, " << in << ")"; break;
    case CoarsenKind::SmoothedAggregation: o << "SmoothedAgg(θ=" << c.theta << ", ω=" << c.sa_omega << ")"; break;
  }
  return o.str();
}

namespace {
const char* coarsen_key(CoarsenKind k) {
  switch (k) {
    case CoarsenKind::Aggregation: return "aggregation";
    case CoarsenKind::PMIS: return "pmis";
    case CoarsenKind::HMIS: return "hmis";
    case CoarsenKind::RS: return "rs";
    case CoarsenKind::AggressivePMIS: return "aggressive_pmis";
    case CoarsenKind::AggressiveHMIS: return "aggressive_hmis";
    case CoarsenKind::SmoothedAggregation: return "smoothed_aggregation";
  }
  return "?";
}

const char* interp_key(InterpKind k) {
  return k == InterpKind::Direct ? "direct" : k == InterpKind::Standard ? "standard" : "extended_i";
}

void coarsening_json(std::ostringstream& o, const Coarsening& c) {
  o << "{\"type\": \"" << coarsen_key(c.kind) << "\", \"theta\": " << c.theta
    << ", \"interpolation\": {\"type\": \"" << interp_key(c.interp.kind)
    << "\", \"trunc_factor\": " << c.interp.trunc_factor << ", \"max_elements\": " << c.interp.max_elements
    << ", \"norm_p\": " << c.interp.norm_p << ", \"rescale\": " << (c.interp.rescale ? "true" : "false")
    << "}, \"filtering\": " << (c.filtering ? "true" : "false") << ", \"filter_tol\": " << c.filter_tol
    << ", \"omega\": " << c.sa_omega << "}";
}
}  // namespace

std::string config_to_json(const Config& c) {
  std::ostringstream o;
  o.precision(17);
  o << "{\"coarsening\": ";
  coarsening_json(o, c.coarsening);
  o << ", \"initial_coarsening\": ";
  coarsening_json(o, c.initial_coarsening);
  o << ", \"initial_coarsening_levels\": " << c.initial_coarsening_levels << ", \"smoother\": \""
    << smoother_name(c.smoother) << "\", \"jacobi_omega\": " << c.jacobi_omega
    << ", \"max_levels\": " << c.max_levels << ", \"max_coarse_size\": " << c.max_coarse_size
    << ", \"pre_smoothing_steps\": " << c.pre_smoothing_steps
    << ", \"post_smoothing_steps\": " << c.post_smoothing_steps << ", \"verbose\": " << c.verbose
    << ", \"max_row_sum\": " << c.max_row_sum << ", \"cycle\": \"" << (c.cycle_w ? "w" : "v")
    << "\", \"strength\": \"" << (c.strength == StrengthKind::Signed ? "signed" : "absolute")
    << "\", \"coarse_solve_on_cpu\": " << (c.coarse_solve_on_cpu ? "true" : "false")
    << ", \"seed\": " << c.seed << "}";
  return o.str();
}

}  // namespace dr

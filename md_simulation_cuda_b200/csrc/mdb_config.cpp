// MDConfig <-> JSON, overrides. Semantics of MDConfigManager
// (include/md_config.hpp:14-111, src/md_config.cpp): missing keys keep the
// struct defaults; output is a JSON object with keys in sorted order, numbers
// in shortest round-trip form with a ".0" for integral doubles, pretty form
// indented by `indent` spaces (the reference writes dump(4) + '\n').
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <climits>
#include <map>
#include <string>
#include <vector>

#include "mdb200.h"
#include "mdb_util.h"

namespace mdb {
namespace {

enum FieldKind { F_INT, F_DBL, F_STR };
struct Field {
  const char* name;
  FieldKind kind;
  size_t off;
  size_t cap;  // strings
};

#define FI(n) {#n, F_INT, offsetof(mdb_config_t, n), 0}
#define FD(n) {#n, F_DBL, offsetof(mdb_config_t, n), 0}
#define FS(n) {#n, F_STR, offsetof(mdb_config_t, n), sizeof(((mdb_config_t*)0)->n)}

// Every key of load_from_json_object / store_to_json_object
// (src/md_config.cpp:43-195).
const Field kFields[] = {
    FI(n_particles_global), FI(n_particles_type0), FD(box_w_global), FD(box_h_global),
    FD(T_init), FD(T_target), FD(SIGMA_AA), FD(SIGMA_BB), FD(SIGMA_AB), FD(EPSILON_AA),
    FD(EPSILON_BB), FD(EPSILON_AB), FD(MASS_A), FD(MASS_B), FD(devide_p), FD(dt), FD(Q),
    FD(save_dt_interval), FD(cutoff), FS(run_name), FS(load_name), FI(THREADS_PER_BLOCK),
    FI(rank_size), FD(mu), FD(v0), FD(D_r), FD(D_theta), FD(barostat_mass), FD(k_piston),
    FD(barostat_area_rate_init), FD(barostat_height_min_ratio), FD(barostat_height_max_ratio),
    FS(pressure_target_mode), FD(P_target), FI(pressure_target_auto_steps),
    FI(pressure_eval_interval_steps), FI(pressure_window_samples), FD(pressure_tolerance_rel),
    FI(pressure_stable_required_windows), FI(nph_warmup_min_steps), FI(nph_warmup_max_steps),
    FI(nph_steps), FI(rank_idx), FI(n_local), FI(n_halo_left), FI(n_halo_right), FI(n_cap),
    FI(halo_left_cap), FI(halo_right_cap), FI(left_rank), FI(right_rank), FD(x_min),
    FD(x_max),
};
#undef FI
#undef FD
#undef FS

const Field* find_field(const std::string& k) {
  for (const Field& f : kFields)
    if (k == f.name) return &f;
  return nullptr;
}

// ---- a small JSON reader (objects, arrays, strings, numbers, literals) ----
struct JVal {
  enum T { NUL, BOOL, NUM, STR, ARR, OBJ } t = NUL;
  bool b = false;
  double num = 0.0;
  bool is_int = false;
  long long inum = 0;
  std::string s;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
};

struct JParser {
  const char* p;
  const char* e;
  std::string err;
  void ws() {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r')) ++p;
  }
  bool fail(const char* m) {
    if (err.empty()) err = m;
    return false;
  }
  bool parse_string(std::string& out) {
    if (p >= e || *p != '"') return fail("expected string");
    ++p;
    out.clear();
    while (p < e && *p != '"') {
      char c = *p++;
      if (c == '\\') {
        if (p >= e) return fail("bad escape");
        char q = *p++;
        switch (q) {
          case '"': out += '"'; break;
          case '\\': out += '\\'; break;
          case '/': out += '/'; break;
          case 'b': out += '\b'; break;
          case 'f': out += '\f'; break;
          case 'n': out += '\n'; break;
          case 'r': out += '\r'; break;
          case 't': out += '\t'; break;
          case 'u': {
            if (e - p < 4) return fail("bad unicode escape");
            unsigned cp = 0;
            for (int k = 0; k < 4; ++k) {
              char h = *p++;
              cp <<= 4;
              if (h >= '0' && h <= '9') cp |= (unsigned)(h - '0');
              else if (h >= 'a' && h <= 'f') cp |= (unsigned)(h - 'a' + 10);
              else if (h >= 'A' && h <= 'F') cp |= (unsigned)(h - 'A' + 10);
              else return fail("bad unicode escape");
            }
            if (cp < 0x80) {
              out += (char)cp;
            } else if (cp < 0x800) {
              out += (char)(0xC0 | (cp >> 6));
              out += (char)(0x80 | (cp & 0x3F));
            } else {
              out += (char)(0xE0 | (cp >> 12));
              out += (char)(0x80 | ((cp >> 6) & 0x3F));
              out += (char)(0x80 | (cp & 0x3F));
            }
            break;
          }
          default: return fail("bad escape");
        }
      } else {
        out += c;
      }
    }
    if (p >= e) return fail("unterminated string");
    ++p;
    return true;
  }
  bool parse(JVal& v) {
    ws();
    if (p >= e) return fail("unexpected end");
    char c = *p;
    if (c == '{') {
      ++p;
      v.t = JVal::OBJ;
      ws();
      if (p < e && *p == '}') {
        ++p;
        return true;
      }
      for (;;) {
        ws();
        std::string k;
        if (!parse_string(k)) return false;
        ws();
        if (p >= e || *p != ':') return fail("expected ':'");
        ++p;
        JVal x;
        if (!parse(x)) return false;
        v.obj.emplace_back(k, std::move(x));
        ws();
        if (p < e && *p == ',') {
          ++p;
          continue;
        }
        if (p < e && *p == '}') {
          ++p;
          return true;
        }
        return fail("expected ',' or '}'");
      }
    }
    if (c == '[') {
      ++p;
      v.t = JVal::ARR;
      ws();
      if (p < e && *p == ']') {
        ++p;
        return true;
      }
      for (;;) {
        JVal x;
        if (!parse(x)) return false;
        v.arr.push_back(std::move(x));
        ws();
        if (p < e && *p == ',') {
          ++p;
          continue;
        }
        if (p < e && *p == ']') {
          ++p;
          return true;
        }
        return fail("expected ',' or ']'");
      }
    }
    if (c == '"') {
      v.t = JVal::STR;
      return parse_string(v.s);
    }
    if (e - p >= 4 && strncmp(p, "true", 4) == 0) {
      p += 4;
      v.t = JVal::BOOL;
      v.b = true;
      return true;
    }
    if (e - p >= 5 && strncmp(p, "false", 5) == 0) {
      p += 5;
      v.t = JVal::BOOL;
      v.b = false;
      return true;
    }
    if (e - p >= 4 && strncmp(p, "null", 4) == 0) {
      p += 4;
      v.t = JVal::NUL;
      return true;
    }
    // number
    const char* s0 = p;
    if (p < e && *p == '-') ++p;
    bool frac = false;
    while (p < e && (isdigit((unsigned char)*p) || *p == '.' || *p == 'e' || *p == 'E' ||
                     *p == '+' || *p == '-')) {
      if (*p == '.' || *p == 'e' || *p == 'E') frac = true;
      ++p;
    }
    if (p == s0) return fail("unexpected character");
    std::string num(s0, p);
    char* end = nullptr;
    v.t = JVal::NUM;
    v.num = strtod(num.c_str(), &end);
    if (end == num.c_str() || *end != '\0') return fail("bad number");
    if (!frac) {
      errno = 0;
      long long q = strtoll(num.c_str(), &end, 10);
      if (errno == 0 && *end == '\0') {
        v.is_int = true;
        v.inum = q;
      }
    }
    return true;
  }
};

// Shortest decimal digits that round-trip a finite double, and its exponent:
// value = 0.d1d2...dn * 10^(exp10).
void shortest_digits(double v, std::string& digits, int& dec_exp) {
  char buf[64];
  for (int prec = 1; prec <= 17; ++prec) {
    snprintf(buf, sizeof(buf), "%.*e", prec - 1, v);
    if (strtod(buf, nullptr) == v) break;
  }
  // buf = d.ddde[+-]XX
  std::string s(buf);
  size_t epos = s.find('e');
  std::string mant = s.substr(0, epos);
  int ex = atoi(s.c_str() + epos + 1);
  digits.clear();
  for (char c : mant)
    if (isdigit((unsigned char)c)) digits += c;
  while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
  dec_exp = ex + 1;
}

// Number formatting of the reference's JSON writer: shortest round-trip
// digits; fixed notation for decimal exponents in (-4, 15], scientific
// otherwise; integral values keep a trailing ".0".
std::string format_double(double v) {
  if (!std::isfinite(v)) return "null";
  if (v == 0.0) return std::signbit(v) ? "-0.0" : "0.0";
  std::string out;
  if (v < 0) {
    out += '-';
    v = -v;
  }
  std::string d;
  int n;
  shortest_digits(v, d, n);
  const int k = (int)d.size();
  if (k <= n && n <= 15) {
    out += d;
    out.append((size_t)(n - k), '0');
    out += ".0";
  } else if (0 < n && n <= 15) {
    out += d.substr(0, (size_t)n);
    out += '.';
    out += d.substr((size_t)n);
  } else if (-4 < n && n <= 0) {
    out += "0.";
    out.append((size_t)(-n), '0');
    out += d;
  } else {
    out += d[0];
    if (k > 1) {
      out += '.';
      out += d.substr(1);
    }
    out += 'e';
    int ex = n - 1;
    out += ex < 0 ? '-' : '+';
    ex = ex < 0 ? -ex : ex;
    char b[16];
    snprintf(b, sizeof(b), "%02d", ex);
    out += b;
  }
  return out;
}

std::string escape_string(const char* s) {
  std::string o = "\"";
  for (const unsigned char* q = (const unsigned char*)s; *q; ++q) {
    unsigned char c = *q;
    switch (c) {
      case '"': o += "\\\""; break;
      case '\\': o += "\\\\"; break;
      case '\b': o += "\\b"; break;
      case '\f': o += "\\f"; break;
      case '\n': o += "\\n"; break;
      case '\r': o += "\\r"; break;
      case '\t': o += "\\t"; break;
      default:
        if (c < 0x20) {
          char b[8];
          snprintf(b, sizeof(b), "\\u%04x", c);
          o += b;
        } else {
          o += (char)c;
        }
    }
  }
  o += '"';
  return o;
}

// Text parse of an override value (parse_scalar, src/md_config.cpp:10-20):
// the whole string (surrounding whitespace allowed) must be one value.
bool parse_int_text(const char* s, int32_t& out) {
  while (isspace((unsigned char)*s)) ++s;
  if (!*s) return false;
  const char* q = s;
  if (*q == '+' || *q == '-') ++q;
  if (!isdigit((unsigned char)*q)) return false;
  errno = 0;
  char* end = nullptr;
  long long v = strtoll(s, &end, 10);
  if (errno != 0 || v < INT32_MIN || v > INT32_MAX) return false;
  while (isspace((unsigned char)*end)) ++end;
  if (*end) return false;
  out = (int32_t)v;
  return true;
}

bool parse_double_text(const char* s, double& out) {
  while (isspace((unsigned char)*s)) ++s;
  if (!*s) return false;
  const char* q = s;
  if (*q == '+' || *q == '-') ++q;
  if (!(isdigit((unsigned char)*q) || (*q == '.' && isdigit((unsigned char)q[1])))) return false;
  for (const char* r = q; *r; ++r)
    if (*r == 'x' || *r == 'X') return false;
  errno = 0;
  char* end = nullptr;
  double v = strtod(s, &end);
  if (errno == ERANGE && (v == HUGE_VAL || v == -HUGE_VAL)) return false;
  while (isspace((unsigned char)*end)) ++end;
  if (*end) return false;
  out = v;
  return true;
}

bool set_string(char* dst, size_t cap, const std::string& v) {
  if (v.size() + 1 > cap) return false;
  memcpy(dst, v.c_str(), v.size() + 1);
  return true;
}

}  // namespace

int config_from_json_text(const char* text, mdb_config_t* out) {
  mdb_config_t cfg;
  mdb_config_default(&cfg);
  JParser P{text, text + strlen(text), {}};
  JVal root;
  if (!P.parse(root)) return set_error(MDB_ERR_CONFIG, "config JSON parse error: " + P.err);
  P.ws();
  if (P.p != P.e) return set_error(MDB_ERR_CONFIG, "config JSON: trailing characters");
  if (root.t != JVal::OBJ) return set_error(MDB_ERR_CONFIG, "config JSON: top level is not an object");
  for (auto& kv : root.obj) {
    const Field* f = find_field(kv.first);
    if (!f) continue;  // unknown keys are ignored, as j.value() ignores them
    char* base = reinterpret_cast<char*>(&cfg) + f->off;
    const JVal& v = kv.second;
    if (f->kind == F_STR) {
      if (v.t != JVal::STR)
        return set_error(MDB_ERR_CONFIG, "config key " + kv.first + " must be a string");
      if (!set_string(base, f->cap, v.s))
        return set_error(MDB_ERR_CONFIG, "config key " + kv.first + " is too long");
    } else if (f->kind == F_INT) {
      if (v.t != JVal::NUM)
        return set_error(MDB_ERR_CONFIG, "config key " + kv.first + " must be a number");
      double d = v.is_int ? (double)v.inum : v.num;
      if (!(d >= (double)INT32_MIN && d <= (double)INT32_MAX))
        return set_error(MDB_ERR_CONFIG, "config key " + kv.first + " is out of range");
      *reinterpret_cast<int32_t*>(base) = v.is_int ? (int32_t)v.inum : (int32_t)v.num;
    } else {
      if (v.t != JVal::NUM)
        return set_error(MDB_ERR_CONFIG, "config key " + kv.first + " must be a number");
      *reinterpret_cast<double*>(base) = v.is_int ? (double)v.inum : v.num;
    }
  }
  *out = cfg;
  return MDB_OK;
}

std::string config_to_json_text(const mdb_config_t* cfg, int indent) {
  std::map<std::string, std::string> kv;  // sorted keys
  for (const Field& f : kFields) {
    const char* base = reinterpret_cast<const char*>(cfg) + f.off;
    std::string val;
    if (f.kind == F_INT) {
      val = std::to_string(*reinterpret_cast<const int32_t*>(base));
    } else if (f.kind == F_DBL) {
      val = format_double(*reinterpret_cast<const double*>(base));
    } else {
      std::string tmp(base, strnlen(base, f.cap));
      val = escape_string(tmp.c_str());
    }
    kv[f.name] = val;
  }
  std::string o;
  if (indent < 0) {
    o = "{";
    bool first = true;
    for (auto& p : kv) {
      if (!first) o += ",";
      first = false;
      o += escape_string(p.first.c_str()) + ":" + p.second;
    }
    o += "}";
  } else {
    std::string pad((size_t)indent, ' ');
    o = "{\n";
    bool first = true;
    for (auto& p : kv) {
      if (!first) o += ",\n";
      first = false;
      o += pad + escape_string(p.first.c_str()) + ": " + p.second;
    }
    o += "\n}";
  }
  return o;
}

int config_apply_override(mdb_config_t* cfg, const char* key, const char* value) {
  const Field* f = find_field(key);
  if (!f) return set_error(MDB_ERR_CONFIG, std::string("unknown config key '") + key + "'");
  char* base = reinterpret_cast<char*>(cfg) + f->off;
  if (f->kind == F_STR) {
    if (!set_string(base, f->cap, value))
      return set_error(MDB_ERR_CONFIG, std::string("value too long for ") + key);
    return MDB_OK;
  }
  if (f->kind == F_INT) {
    int32_t v;
    if (!parse_int_text(value, v))
      return set_error(MDB_ERR_CONFIG,
                       std::string("Invalid override '") + key + "=" + value + "'");
    *reinterpret_cast<int32_t*>(base) = v;
    return MDB_OK;
  }
  double d;
  if (!parse_double_text(value, d))
    return set_error(MDB_ERR_CONFIG, std::string("Invalid override '") + key + "=" + value + "'");
  *reinterpret_cast<double*>(base) = d;
  return MDB_OK;
}

}  // namespace mdb

extern "C" {

int mdb_config_default(mdb_config_t* out) {
  if (!out) return mdb::set_error(MDB_ERR_ARG, "null config");
  memset(out, 0, sizeof(*out));
  // in-class defaults of MDConfig (include/md_config.hpp:21-65)
  out->SIGMA_AA = 1.0;
  out->SIGMA_BB = 1.0;
  out->SIGMA_AB = 1.0;
  out->EPSILON_AA = 1.0;
  out->EPSILON_BB = 1.0;
  out->EPSILON_AB = 0.25;
  out->MASS_A = 1.0;
  out->MASS_B = 1.0;
  out->devide_p = 0.5;
  out->dt = 1e-3;
  out->Q = 100.0;
  out->save_dt_interval = 0.1;
  out->cutoff = 2.5;
  strcpy(out->run_name, "test");
  out->load_name[0] = '\0';
  out->THREADS_PER_BLOCK = 256;
  out->rank_size = 8;
  out->mu = 1.0;
  out->v0 = 0.0;
  out->D_r = 0.0;
  out->D_theta = 0.0;
  out->barostat_mass = 1.0e4;
  out->k_piston = 100.0;
  out->barostat_area_rate_init = 0.0;
  out->barostat_height_min_ratio = 0.6;
  out->barostat_height_max_ratio = 1.4;
  strcpy(out->pressure_target_mode, "auto_initial");
  out->P_target = 0.0;
  out->pressure_target_auto_steps = 5000;
  out->pressure_eval_interval_steps = 100;
  out->pressure_window_samples = 50;
  out->pressure_tolerance_rel = 0.05;
  out->pressure_stable_required_windows = 3;
  out->nph_warmup_min_steps = 20000;
  out->nph_warmup_max_steps = 200000;
  out->nph_steps = 300000;
  out->rank_idx = 0;
  return MDB_OK;
}

int mdb_config_from_json(const char* json_text, mdb_config_t* out) {
  if (!json_text || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  return mdb::config_from_json_text(json_text, out);
}

int mdb_config_from_json_file(const char* path, mdb_config_t* out) {
  if (!path || !out) return mdb::set_error(MDB_ERR_ARG, "null argument");
  FILE* f = fopen(path, "rb");
  if (!f) return mdb::set_error(MDB_ERR_IO, std::string("Failed to open config file: ") + path);
  std::string text;
  char buf[65536];
  size_t k;
  while ((k = fread(buf, 1, sizeof(buf), f)) > 0) text.append(buf, k);
  fclose(f);
  return mdb::config_from_json_text(text.c_str(), out);
}

int mdb_config_to_json(const mdb_config_t* cfg, int32_t indent, char* buf, size_t cap,
                       size_t* needed) {
  if (!cfg) return mdb::set_error(MDB_ERR_ARG, "null config");
  std::string s = mdb::config_to_json_text(cfg, indent);
  if (needed) *needed = s.size();
  if (!buf) return MDB_OK;
  if (cap < s.size() + 1) return mdb::set_error(MDB_ERR_CAPACITY, "JSON buffer too small");
  memcpy(buf, s.c_str(), s.size() + 1);
  return MDB_OK;
}

int mdb_config_apply_override(mdb_config_t* cfg, const char* key, const char* value) {
  if (!cfg || !key || !value) return mdb::set_error(MDB_ERR_ARG, "null argument");
  return mdb::config_apply_override(cfg, key, value);
}

int mdb_parse_override_argument(const char* arg, char* key, size_t key_cap, char* value,
                                size_t value_cap) {
  if (!arg || !key || !value) return mdb::set_error(MDB_ERR_ARG, "null argument");
  std::string token(arg);
  if (token.empty()) return mdb::set_error(MDB_ERR_ARG, "empty override");
  if (token.rfind("--", 0) == 0) token.erase(0, 2);
  if (token.rfind('D', 0) == 0) token.erase(0, 1);
  size_t eq = token.find('=');
  if (eq == std::string::npos) return mdb::set_error(MDB_ERR_ARG, "override has no '='");
  std::string k = token.substr(0, eq), v = token.substr(eq + 1);
  if (k.empty()) return mdb::set_error(MDB_ERR_ARG, "override has an empty key");
  if (k.size() + 1 > key_cap || v.size() + 1 > value_cap)
    return mdb::set_error(MDB_ERR_CAPACITY, "override buffers too small");
  memcpy(key, k.c_str(), k.size() + 1);
  memcpy(value, v.c_str(), v.size() + 1);
  return MDB_OK;
}

void mdb_options_default(mdb_options_t* out) {
  if (!out) return;
  memset(out, 0, sizeof(*out));
  out->device = 0;
  out->skin = 0.0;
  out->use_graphs = 1;
  out->max_neighbors = 48;
}

}  // extern "C"

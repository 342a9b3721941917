// Simulation parameters: the sim_params defaults (reference
// src/sim_params.h:15-124) and a reader for the TOML keys of parse_config
// (src/sim_params.cpp:7-146).  The reader accepts the TOML subset COFFEE's
// configs use: `key = value` lines, booleans, integers, floats, one-line
// arrays, `#` comments; any key it does not know is ignored, and any key
// missing from the text keeps its default, as parse_config's value_or does.
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "coffee_b200.h"
#include "coffee_internal.h"

extern "C" void coffee_params_default(coffee_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->dt = 0.01;
  p->max_steps = 10000;
  p->data_interval = 100;
  p->snapshot_interval = 1000;
  p->downsample = 1;
  p->slice_interval = 100;
  p->downsample_2d = 1;
  p->N[0] = 1;
  p->size[0] = 1.0;
  p->nodes[0] = 1;
  p->kn[0] = 1;
  p->kn[1] = 1;
  p->a = 0.99;
  p->calc_current = 1;
  p->clean_ep = 1;
  p->check_egb = 1;
  for (int i = 0; i < 3; ++i) p->pml[i] = 60;
  p->pmllen = 10;
  p->sigpml = 0.1;
  p->divB_clean = 1;
  p->ch2 = 1.0;
  p->tau = 2.0;
  p->KOeps = 0.5;
  p->KO_geometry = 1;
  p->use_edotb_damping = 1;
  p->damp_gamma = 0.2;
  p->radius = 10.0;
  p->omega = 0.001;
  p->b0 = 1e3;
  p->p3 = 1.0;
  p->tp_end = 0.5;
  p->rpert1 = 5.0;
  p->rpert2 = 10.0;
  p->thp1 = 0.3;
  p->thp2 = 0.4;
  p->nT = 1.0;
  p->ph1 = 3.0 / 16.0;
  p->ph2 = 5.0 / 16.0;
  p->dph = 1.0 / 64.0;
  p->theta0 = 0.2;
  p->drpert = 0.1;
  p->tp_start1 = 1.0;
  p->tp_end1 = 1.5;
  p->rpert11 = 5.0;
  p->rpert21 = 10.0;
  p->thp11 = 0.3;
  p->thp21 = 0.4;
  p->nT1 = 1.0;
  p->ph11 = 3.0 * M_PI / 16.0;
  p->ph21 = 5.0 * M_PI / 16.0;
  p->dph1 = M_PI / 64.0;
  p->skymap_Nth = 256;
  p->skymap_Nph = 512;
}

namespace {

struct TomlValue {
  enum Kind { NONE, BOOL, INT, FLOAT, ARRAY } kind = NONE;
  bool b = false;
  long long i = 0;
  double f = 0;
  std::vector<TomlValue> arr;
};

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

bool parse_scalar(const std::string& t, TomlValue* v) {
  if (t == "true" || t == "false") {
    v->kind = TomlValue::BOOL;
    v->b = (t == "true");
    return true;
  }
  std::string s;
  for (char ch : t)
    if (ch != '_') s += ch;  // TOML digit separators
  if (s.empty()) return false;
  char* end = nullptr;
  const bool looks_float = s.find_first_of(".eE") != std::string::npos ||
                           s == "inf" || s == "+inf" || s == "-inf" || s == "nan";
  if (!looks_float) {
    long long x = std::strtoll(s.c_str(), &end, 10);
    if (*end == '\0') {
      v->kind = TomlValue::INT;
      v->i = x;
      return true;
    }
  }
  double d = std::strtod(s.c_str(), &end);
  if (*end == '\0') {
    v->kind = TomlValue::FLOAT;
    v->f = d;
    return true;
  }
  return false;
}

bool parse_value(const std::string& t, TomlValue* v) {
  if (!t.empty() && t.front() == '[') {
    if (t.back() != ']') return false;
    v->kind = TomlValue::ARRAY;
    std::string inner = t.substr(1, t.size() - 2);
    size_t start = 0;
    while (start <= inner.size()) {
      size_t comma = inner.find(',', start);
      std::string item = trim(inner.substr(start, comma == std::string::npos ? std::string::npos
                                                                               : comma - start));
      if (!item.empty()) {
        TomlValue e;
        if (!parse_scalar(item, &e)) return false;
        v->arr.push_back(e);
      }
      if (comma == std::string::npos) break;
      start = comma + 1;
    }
    return true;
  }
  return parse_scalar(t, v);
}

// cpptoml's get_as<double> accepts integers; get_as<int> and get_as<bool>
// accept only their own kind (anything else falls back to the default).
bool as_double(const TomlValue& v, double* out) {
  if (v.kind == TomlValue::FLOAT) { *out = v.f; return true; }
  if (v.kind == TomlValue::INT) { *out = (double)v.i; return true; }
  return false;
}
bool as_int(const TomlValue& v, int* out) {
  if (v.kind == TomlValue::INT) { *out = (int)v.i; return true; }
  return false;
}
bool as_bool(const TomlValue& v, int* out) {
  if (v.kind == TomlValue::BOOL) { *out = v.b ? 1 : 0; return true; }
  return false;
}

}  // namespace

extern "C" int coffee_params_parse_toml(const char* text, coffee_params* p) {
  if (!text || !p) return coffee::fail(COFFEE_E_INVALID, "coffee_params_parse_toml: null argument");
  coffee_params_default(p);
  const char* cur = text;
  int lineno = 0;
  while (*cur) {
    const char* nl = std::strchr(cur, '\n');
    std::string line = nl ? std::string(cur, nl - cur) : std::string(cur);
    cur = nl ? nl + 1 : cur + line.size();
    ++lineno;
    size_t hash = line.find('#');
    if (hash != std::string::npos) line = line.substr(0, hash);
    line = trim(line);
    if (line.empty() || line.front() == '[') continue;  // blank / table header
    size_t eq = line.find('=');
    if (eq == std::string::npos)
      return coffee::fail(COFFEE_E_CONFIG, "config line %d: expected key = value", lineno);
    std::string key = trim(line.substr(0, eq));
    std::string val = trim(line.substr(eq + 1));
    TomlValue v;
    if (!parse_value(val, &v))
      return coffee::fail(COFFEE_E_CONFIG, "config line %d: cannot parse value of %s", lineno,
                          key.c_str());
    auto d = [&](double* dst) { as_double(v, dst); };
    auto i = [&](int* dst) { as_int(v, dst); };
    auto b = [&](int* dst) { as_bool(v, dst); };
    auto arr3 = [&](auto setter) {
      if (v.kind != TomlValue::ARRAY || v.arr.size() < 3) return;
      for (int a = 0; a < 3; ++a) setter(a, v.arr[a]);
    };
#define DKEY(name) else if (key == #name) d(&p->name)
#define IKEY(name) else if (key == #name) i(&p->name)
#define BKEY(name) else if (key == #name) b(&p->name)
    if (key == "max_steps") {
      if (v.kind == TomlValue::INT) p->max_steps = (uint64_t)v.i;
    }
    DKEY(dt); IKEY(data_interval); IKEY(snapshot_interval); IKEY(downsample);
    BKEY(slice_x); BKEY(slice_y); BKEY(slice_z); BKEY(slice_xy);
    DKEY(slice_x_pos); DKEY(slice_y_pos); DKEY(slice_z_pos);
    IKEY(slice_interval); IKEY(downsample_2d);
    else if (key == "periodic_boundary") arr3([&](int a, const TomlValue& e) { as_bool(e, &p->periodic_boundary[a]); });
    else if (key == "guard") arr3([&](int a, const TomlValue& e) { as_int(e, &p->guard[a]); });
    else if (key == "N") arr3([&](int a, const TomlValue& e) { as_int(e, &p->N[a]); });
    else if (key == "lower") arr3([&](int a, const TomlValue& e) { as_double(e, &p->lower[a]); });
    else if (key == "size") arr3([&](int a, const TomlValue& e) { as_double(e, &p->size[a]); });
    else if (key == "nodes") arr3([&](int a, const TomlValue& e) { double x; if (as_double(e, &x)) p->nodes[a] = (int)x; });
    else if (key == "pml") arr3([&](int a, const TomlValue& e) { as_int(e, &p->pml[a]); });
    IKEY(shift_ghost); DKEY(a);
    BKEY(calc_current); BKEY(clean_ep); BKEY(check_egb);
    IKEY(pmllen); DKEY(sigpml); DKEY(damp_gamma); BKEY(use_edotb_damping);
    BKEY(divB_clean); DKEY(ch2); DKEY(tau); DKEY(KOeps); BKEY(KO_geometry);
    IKEY(problem); DKEY(radius); DKEY(omega); DKEY(b0);
    DKEY(p1); DKEY(p2); DKEY(p3); DKEY(q11); DKEY(q12); DKEY(q13); DKEY(q22); DKEY(q23);
    DKEY(q_offset_x); DKEY(q_offset_y); DKEY(q_offset_z);
    DKEY(tp_start); DKEY(tp_end); DKEY(rpert1); DKEY(rpert2); DKEY(thp1); DKEY(thp2);
    DKEY(dw0); DKEY(nT); DKEY(shear); DKEY(ph1); DKEY(ph2); DKEY(dph); DKEY(theta0);
    DKEY(drpert);
    DKEY(tp_start1); DKEY(tp_end1); DKEY(rpert11); DKEY(rpert21); DKEY(thp11); DKEY(thp21);
    DKEY(dw1); DKEY(nT1); DKEY(shear1); DKEY(ph11); DKEY(ph21); DKEY(dph1);
    IKEY(pert_type);
#undef DKEY
#undef IKEY
#undef BKEY
  }
  return COFFEE_OK;
}

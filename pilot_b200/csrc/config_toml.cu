// config_toml.cu — the stage TOML reader (host code only).
//
// The reference reads `<base-dir>/stage.toml` with toml++ (pilot/staging/Stage.cxx:25-49,
// pilot/TomlUtils.h:33-107): a [dataset_providers.<name>] table per provider with
// `type` and `cell_dims` (SubdividedSpheresDescriptor.cxx:22-44). toml++ is not
// available here, so this is a reader for the subset of TOML such a file uses:
//   [table] and [a.b] headers, [[array-of-tables]] headers, key = value with
//   basic / literal strings, integers (with _), floats (exponents, inf, nan),
//   booleans and arrays of those (across lines, trailing comma allowed), and
//   # comments. Inline tables, dates and multi-line strings are rejected.
// The schema walker then fills a beams_scene_desc; unknown tables or keys and
// wrong types are errors with the line number.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/beams_b200.h"

namespace beams {
namespace {

struct Value {
  enum Kind { STR, INT, FLT, BOOL, ARR } kind = INT;
  std::string s;
  long long i = 0;
  double f = 0.0;
  bool b = false;
  std::vector<Value> arr;
  bool is_num() const { return kind == INT || kind == FLT; }
  double num() const { return kind == INT ? (double)i : f; }
};

struct Entry {
  std::string table;  // "render", "dataset_providers.spheres", "light#0", ...
  std::string key;
  Value v;
  int line;
};

struct ParseError {
  int line;
  std::string msg;
};

class Reader {
 public:
  explicit Reader(const std::string& text) : t_(text) {}

  std::vector<Entry> parse() {
    std::vector<Entry> out;
    std::string table;
    std::vector<std::pair<std::string, int>> aot;  // array-of-table name -> count
    while (p_ < t_.size()) {
      skip_ws();
      if (p_ >= t_.size()) break;
      const char c = t_[p_];
      if (c == '#' ) {
        skip_comment();
        continue;
      }
      if (c == '\n') {
        ++line_;
        ++p_;
        continue;
      }
      if (c == '\r') {
        ++p_;
        continue;
      }
      if (c == '[') {
        const bool arr = p_ + 1 < t_.size() && t_[p_ + 1] == '[';
        p_ += arr ? 2 : 1;
        std::string name = dotted_key();
        skip_ws();
        if (!consume(']') || (arr && !consume(']'))) fail("malformed table header");
        if (arr) {
          int idx = 0;
          bool found = false;
          for (auto& a : aot)
            if (a.first == name) {
              idx = ++a.second;
              found = true;
            }
          if (!found) aot.push_back({name, 0});
          table = name + "#" + std::to_string(idx);
        } else {
          table = name;
        }
        end_of_line();
        continue;
      }
      Entry e;
      e.line = line_;
      e.table = table;
      e.key = dotted_key();
      skip_ws();
      if (!consume('=')) fail("expected '=' after key '" + e.key + "'");
      skip_ws();
      e.v = value();
      end_of_line();
      for (const auto& o : out)
        if (o.table == e.table && o.key == e.key) fail("duplicate key '" + e.key + "'");
      out.push_back(e);
    }
    return out;
  }

 private:
  const std::string& t_;
  size_t p_ = 0;
  int line_ = 1;

  [[noreturn]] void fail(const std::string& m) { throw ParseError{line_, m}; }
  void skip_ws() {
    while (p_ < t_.size() && (t_[p_] == ' ' || t_[p_] == '\t')) ++p_;
  }
  void skip_comment() {
    while (p_ < t_.size() && t_[p_] != '\n') ++p_;
  }
  bool consume(char c) {
    if (p_ < t_.size() && t_[p_] == c) {
      ++p_;
      return true;
    }
    return false;
  }
  void end_of_line() {
    skip_ws();
    if (p_ < t_.size() && t_[p_] == '#') skip_comment();
    if (p_ < t_.size() && t_[p_] == '\r') ++p_;
    if (p_ < t_.size() && t_[p_] != '\n') fail("unexpected text after value");
  }
  std::string bare_or_quoted() {
    skip_ws();
    if (p_ < t_.size() && (t_[p_] == '"' || t_[p_] == '\'')) return string_lit();
    size_t b = p_;
    while (p_ < t_.size() && (std::isalnum((unsigned char)t_[p_]) || t_[p_] == '_' || t_[p_] == '-')) ++p_;
    if (p_ == b) fail("expected a key");
    return t_.substr(b, p_ - b);
  }
  std::string dotted_key() {
    std::string k = bare_or_quoted();
    skip_ws();
    while (consume('.')) {
      k += ".";
      k += bare_or_quoted();
      skip_ws();
    }
    return k;
  }
  std::string string_lit() {
    const char q = t_[p_++];
    if (p_ + 1 < t_.size() && t_[p_] == q && t_[p_ + 1] == q) fail("multi-line strings are not supported");
    std::string s;
    while (p_ < t_.size() && t_[p_] != q) {
      char c = t_[p_++];
      if (c == '\n') fail("unterminated string");
      if (q == '"' && c == '\\') {
        if (p_ >= t_.size()) fail("unterminated string");
        const char e = t_[p_++];
        switch (e) {
          case 'n': c = '\n'; break;
          case 't': c = '\t'; break;
          case '\\': c = '\\'; break;
          case '"': c = '"'; break;
          default: fail(std::string("unsupported escape \\") + e);
        }
      }
      s += c;
    }
    if (!consume(q)) fail("unterminated string");
    return s;
  }
  void skip_blank_lines() {
    for (;;) {
      skip_ws();
      if (p_ < t_.size() && t_[p_] == '#') {
        skip_comment();
        continue;
      }
      if (p_ < t_.size() && (t_[p_] == '\n' || t_[p_] == '\r')) {
        if (t_[p_] == '\n') ++line_;
        ++p_;
        continue;
      }
      return;
    }
  }
  Value value() {
    Value v;
    if (p_ >= t_.size()) fail("missing value");
    const char c = t_[p_];
    if (c == '"' || c == '\'') {
      v.kind = Value::STR;
      v.s = string_lit();
      return v;
    }
    if (c == '[') {
      ++p_;
      v.kind = Value::ARR;
      skip_blank_lines();
      while (!consume(']')) {
        v.arr.push_back(value());
        skip_blank_lines();
        if (consume(',')) {
          skip_blank_lines();
          continue;
        }
        skip_blank_lines();
        if (!consume(']')) fail("expected ',' or ']' in array");
        break;
      }
      return v;
    }
    if (c == '{') fail("inline tables are not supported");
    size_t b = p_;
    while (p_ < t_.size() && !std::strchr(" \t\r\n,]#", t_[p_])) ++p_;
    std::string tok = t_.substr(b, p_ - b);
    if (tok == "true" || tok == "false") {
      v.kind = Value::BOOL;
      v.b = tok == "true";
      return v;
    }
    std::string clean;
    for (char ch : tok)
      if (ch != '_') clean += ch;
    if (clean.empty()) fail("missing value");
    const bool is_float = clean.find_first_of(".eE") != std::string::npos || clean.find("inf") != std::string::npos ||
                          clean.find("nan") != std::string::npos;
    char* end = nullptr;
    errno = 0;
    if (is_float) {
      v.kind = Value::FLT;
      v.f = std::strtod(clean.c_str(), &end);
    } else {
      v.kind = Value::INT;
      v.i = std::strtoll(clean.c_str(), &end, 10);
    }
    if (!end || *end != '\0' || errno == ERANGE) fail("invalid value '" + tok + "'");
    return v;
  }
};

// ---- schema -------------------------------------------------------------------
void defaults(beams_scene_desc& d) {
  std::memset(&d, 0, sizeof(d));
  std::snprintf(d.provider_name, sizeof(d.provider_name), "%s", "default");
  std::snprintf(d.provider_type, sizeof(d.provider_type), "%s", "subdivided_spheres");
  d.cell_dims[0] = d.cell_dims[1] = d.cell_dims[2] = 64;
  d.seed = 1;
  d.octaves = 4;
  d.base_freq = 4.f;
  d.width = d.height = 512;
  d.sample_distance = -1.f;
  d.termination_alpha = 1.f;
  d.form = BEAMS_FORM_EXACT;
  d.field_dtype = BEAMS_BF16;
  d.background[0] = d.background[1] = d.background[2] = d.background[3] = 1.f;
  d.shadow_enabled = 1;
  d.light_steps = 128.f;
  d.fov_y_deg = 30.f;
  d.up[1] = 1.0;
  std::snprintf(d.tf_preset, sizeof(d.tf_preset), "%s", "cool to warm");
  // the alpha points of the reference's sphere scenes (SubdividedSpheresScene.cxx)
  const double xs[] = {0.0, 0.1, 0.2, 0.3, 0.4, 0.5, 0.6, 0.7, 0.8, 0.9, 1.0};
  const float as[] = {0.f, 0.008f, 0.2f, 1.f, 0.1f, 1.f, 0.6f, 0.7f, 1.f, 0.7f, 1.f};
  d.tf_points = 11;
  for (int i = 0; i < 11; ++i) {
    d.tf_x[i] = xs[i];
    d.tf_alpha[i] = as[i];
  }
  d.tf_range[0] = 0.f;
  d.tf_range[1] = 1.f;
  d.tf_size = 256;
  d.mlp_knot = 4;
  d.mlp_probe_fraction = 0.01f;
  d.mlp_fallback_tol = 0.01f;
  d.mlp_samples_log2 = 24;
  d.mlp_lights = 32;
}

struct Schema {
  beams_scene_desc& d;
  const Entry* e = nullptr;
  [[noreturn]] void bad(const std::string& m) { throw ParseError{e->line, m}; }
  double num() {
    if (!e->v.is_num()) bad("'" + e->key + "' must be a number");
    return e->v.num();
  }
  long long integer() {
    if (e->v.kind != Value::INT) bad("'" + e->key + "' must be an integer");
    return e->v.i;
  }
  bool boolean() {
    if (e->v.kind != Value::BOOL) bad("'" + e->key + "' must be true or false");
    return e->v.b;
  }
  std::string str() {
    if (e->v.kind != Value::STR) bad("'" + e->key + "' must be a string");
    return e->v.s;
  }
  std::vector<double> nums(size_t n_min, size_t n_max) {
    if (e->v.kind != Value::ARR) bad("'" + e->key + "' must be an array");
    if (e->v.arr.size() < n_min || e->v.arr.size() > n_max)
      bad("'" + e->key + "' must have " + std::to_string(n_min) +
          (n_max != n_min ? ".." + std::to_string(n_max) : std::string()) + " elements");
    std::vector<double> out;
    for (const auto& x : e->v.arr) {
      if (!x.is_num()) bad("'" + e->key + "' must hold numbers");
      out.push_back(x.num());
    }
    return out;
  }
  void int3(int v[3], long long lo, long long hi) {
    if (e->v.kind == Value::INT) {
      v[0] = v[1] = v[2] = (int)e->v.i;
    } else {
      if (e->v.kind != Value::ARR || e->v.arr.size() != 3) bad("'" + e->key + "' must be an integer or [x, y, z]");
      for (int k = 0; k < 3; ++k) {
        if (e->v.arr[k].kind != Value::INT) bad("'" + e->key + "' must hold integers");
        v[k] = (int)e->v.arr[k].i;
      }
    }
    for (int k = 0; k < 3; ++k)
      if (v[k] < lo || v[k] > hi) bad("'" + e->key + "' out of range");
  }

  void apply(const std::vector<Entry>& es) {
    std::string provider;
    for (const auto& x : es) {
      e = &x;
      const std::string& t = x.table;
      const std::string& k = x.key;
      if (t.rfind("dataset_providers.", 0) == 0) {
        const std::string name = t.substr(std::strlen("dataset_providers."));
        if (provider.empty()) provider = name;
        if (name != provider) continue;  // the first provider is the scene's dataset
        std::snprintf(d.provider_name, sizeof(d.provider_name), "%s", name.c_str());
        if (k == "type") {
          const std::string v = str();
          if (v != "subdivided_spheres" && v != "spheres" && v != "blobs" && v != "noise" && v != "vtk_file")
            bad("unknown dataset provider type '" + v + "'");
          std::snprintf(d.provider_type, sizeof(d.provider_type), "%s", v.c_str());
        } else if (k == "cell_dims") {
          int3(d.cell_dims, 1, 4095);
        } else if (k == "file_name") {
          const std::string v = str();
          if (v.empty() || v.size() >= sizeof(d.file_name)) bad("'file_name' must be 1..255 characters");
          std::snprintf(d.file_name, sizeof(d.file_name), "%s", v.c_str());
        } else if (k == "seed") {
          d.seed = (unsigned)integer();
        } else if (k == "octaves") {
          d.octaves = (int)integer();
          if (d.octaves < 1 || d.octaves > 12) bad("'octaves' out of range");
        } else if (k == "base_freq") {
          d.base_freq = (float)num();
        } else {
          bad("unknown key '" + k + "' in [" + t + "]");
        }
      } else if (t == "render") {
        if (k == "width" || k == "height") {
          const long long v = integer();
          if (v < 1 || v > 16384) bad("'" + k + "' out of range");
          (k == "width" ? d.width : d.height) = (int)v;
        } else if (k == "sample_distance") {
          d.sample_distance = (float)num();
        } else if (k == "termination_alpha") {
          d.termination_alpha = (float)num();
          if (!(d.termination_alpha > 0.f && d.termination_alpha <= 1.f)) bad("'termination_alpha' must be in (0, 1]");
        } else if (k == "form") {
          const std::string v = str();
          if (v == "exact") d.form = BEAMS_FORM_EXACT;
          else if (v == "precision") d.form = BEAMS_FORM_PRECISION;
          else if (v == "mlp") d.form = BEAMS_FORM_MLP;
          else bad("unknown form '" + v + "'");
        } else if (k == "field_dtype") {
          const std::string v = str();
          if (v == "bf16") d.field_dtype = BEAMS_BF16;
          else if (v == "f16") d.field_dtype = BEAMS_F16;
          else bad("field_dtype must be \"bf16\" or \"f16\"");
        } else if (k == "composite_background") {
          d.composite_background = boolean() ? 1 : 0;
        } else if (k == "background") {
          const auto v = nums(4, 4);
          for (int i = 0; i < 4; ++i) d.background[i] = (float)v[i];
        } else {
          bad("unknown key '" + k + "' in [render]");
        }
      } else if (t == "shadow_map") {
        if (k == "enabled") d.shadow_enabled = boolean() ? 1 : 0;
        else if (k == "size") int3(d.shadow_size, 1, 1024);
        else if (k == "size_ratio") {
          d.shadow_size_ratio = (float)num();
          if (!(d.shadow_size_ratio > 0.f)) bad("'size_ratio' must be positive");
        } else if (k == "num_steps") {
          const long long v = integer();
          if (v < 1 || v > 65536) bad("'num_steps' out of range");
          d.light_steps = (float)v;
        } else {
          bad("unknown key '" + k + "' in [shadow_map]");
        }
      } else if (t == "camera") {
        if (k == "azimuth") d.azimuth = (float)num();
        else if (k == "elevation") d.elevation = (float)num();
        else if (k == "fov_y") {
          d.fov_y_deg = (float)num();
          if (!(d.fov_y_deg > 0.f && d.fov_y_deg < 180.f)) bad("'fov_y' must be in (0, 180)");
        } else if (k == "type") {
          const std::string v = str();
          if (v != "orbit" && v != "explicit") bad("camera type must be \"orbit\" or \"explicit\"");
          d.camera_explicit = v == "explicit";
        } else if (k == "position" || k == "look_at" || k == "up") {
          const auto v = nums(3, 3);
          double* dst = k == "position" ? d.position : (k == "look_at" ? d.look_at : d.up);
          for (int i = 0; i < 3; ++i) dst[i] = v[i];
          d.camera_explicit = 1;
        } else {
          bad("unknown key '" + k + "' in [camera]");
        }
      } else if (t.rfind("light#", 0) == 0) {
        const int idx = std::atoi(t.c_str() + 6);
        if (idx >= BEAMS_MAX_CONFIG_LIGHTS) bad("too many [[light]] tables");
        if (idx + 1 > d.n_lights) {
          d.n_lights = idx + 1;
          beams_config_light& L = d.lights[idx];
          L.kind = 0;
          L.color[0] = L.color[1] = L.color[2] = 1.f;
          L.intensity = 1.f;
        }
        beams_config_light& L = d.lights[idx];
        if (k == "type") {
          const std::string v = str();
          if (v == "point") L.kind = 0;
          else if (v == "directional") L.kind = 1;
          else bad("light type must be \"point\" or \"directional\"");
        } else if (k == "position" || k == "direction") {
          const auto v = nums(3, 3);
          for (int i = 0; i < 3; ++i) L.position[i] = v[i];
        } else if (k == "color") {
          const auto v = nums(3, 3);
          for (int i = 0; i < 3; ++i) L.color[i] = (float)v[i];
        } else if (k == "intensity") {
          L.intensity = (float)num();
        } else {
          bad("unknown key '" + k + "' in [[light]]");
        }
      } else if (t == "transfer_function") {
        if (k == "preset") {
          const std::string v = str();
          if (v != "cool to warm" && v != "ramp") bad("transfer_function preset must be \"cool to warm\" or \"ramp\"");
          std::snprintf(d.tf_preset, sizeof(d.tf_preset), "%s", v.c_str());
        } else if (k == "points") {
          const auto v = nums(1, BEAMS_MAX_TF_POINTS);
          d.tf_points = (int)v.size();
          for (size_t i = 0; i < v.size(); ++i) d.tf_x[i] = v[i];
        } else if (k == "alphas") {
          const auto v = nums(1, BEAMS_MAX_TF_POINTS);
          for (size_t i = 0; i < v.size(); ++i) d.tf_alpha[i] = (float)v[i];
          alphas_n = (int)v.size();
          alphas_line = x.line;
        } else if (k == "range") {
          const auto v = nums(2, 2);
          d.tf_range[0] = (float)v[0];
          d.tf_range[1] = (float)v[1];
        } else if (k == "size") {
          const long long v = integer();
          if (v < 2 || v > 1024) bad("'size' must be in [2, 1024]");
          d.tf_size = (int)v;
        } else {
          bad("unknown key '" + k + "' in [transfer_function]");
        }
      } else if (t == "form") {
        if (k == "knot") {
          d.mlp_knot = (int)integer();
          if (d.mlp_knot < 1 || d.mlp_knot > 64) bad("'knot' must be in [1, 64]");
        } else if (k == "probe_fraction") {
          d.mlp_probe_fraction = (float)num();
        } else if (k == "fallback_tol") {
          d.mlp_fallback_tol = (float)num();
        } else if (k == "samples_log2") {
          d.mlp_samples_log2 = (int)integer();
        } else if (k == "lights") {
          d.mlp_lights = (int)integer();
        } else {
          bad("unknown key '" + k + "' in [form]");
        }
      } else if (t.empty()) {
        bad("key '" + k + "' outside any table");
      } else {
        bad("unknown table [" + t + "]");
      }
    }
    if (alphas_n >= 0 && alphas_n != d.tf_points)
      throw ParseError{alphas_line, "transfer_function: points and alphas differ in length"};
    for (int i = 0; i < d.n_lights; ++i)
      if (d.lights[i].kind == 1 && d.lights[i].position[0] == 0 && d.lights[i].position[1] == 0 &&
          d.lights[i].position[2] == 0)
        throw ParseError{0, "a directional light needs a non-zero direction"};
  }
  int alphas_n = -1, alphas_line = 0;
};

}  // namespace
}  // namespace beams

using namespace beams;

extern "C" {

beams_status beams_parse_config_toml(const char* text, beams_scene_desc* out, char* err, int errlen) {
  if (err && errlen > 0) err[0] = '\0';
  if (!text || !out) return BEAMS_ERR_INVALID_ARG;
  beams_scene_desc d;
  defaults(d);
  try {
    std::string t(text);
    Reader rd(t);
    const std::vector<Entry> es = rd.parse();
    Schema sc{d};
    sc.apply(es);
  } catch (const ParseError& pe) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "line %d: %s", pe.line, pe.msg.c_str());
    return BEAMS_ERR_CONFIG;
  } catch (...) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "configuration: internal error");
    return BEAMS_ERR_INTERNAL;
  }
  *out = d;
  return BEAMS_OK;
}

beams_status beams_load_config_toml(const char* path, beams_scene_desc* out, char* err, int errlen) {
  if (err && errlen > 0) err[0] = '\0';
  if (!path || !out) return BEAMS_ERR_INVALID_ARG;
  std::ifstream f(path, std::ios::binary);
  if (!f) {
    if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "cannot open %s", path);
    return BEAMS_ERR_CONFIG;
  }
  std::stringstream ss;
  ss << f.rdbuf();
  beams_status st = beams_parse_config_toml(ss.str().c_str(), out, err, errlen);
  if (st == BEAMS_OK && out->file_name[0] && out->file_name[0] != '/') {
    // a relative dataset file is relative to the stage file's directory
    const std::string p(path);
    const size_t slash = p.find_last_of('/');
    if (slash != std::string::npos) {
      const std::string full = p.substr(0, slash + 1) + out->file_name;
      if (full.size() >= sizeof(out->file_name)) {
        if (err && errlen > 0) std::snprintf(err, (size_t)errlen, "dataset file path too long");
        return BEAMS_ERR_CONFIG;
      }
      std::snprintf(out->file_name, sizeof(out->file_name), "%s", full.c_str());
    }
  }
  return st;
}

}  // extern "C"

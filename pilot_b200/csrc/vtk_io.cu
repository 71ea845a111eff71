// vtk_io.cu — legacy VTK reader for the volumes the reference's file scenes use.
//
// The reference reads its file datasets through VTK-m's legacy VTK reader
// (pilot/io/DataSetUtils.cxx:13-42, vtkm::io::VTKDataSetReader). This is a
// reader of the same file format (the published "VTK legacy" format), for the
// two dataset kinds a volume renderer of structured grids consumes:
//   DATASET STRUCTURED_POINTS  DIMENSIONS, ORIGIN, SPACING (or ASPECT_RATIO)
//   DATASET RECTILINEAR_GRID   DIMENSIONS, X/Y/Z_COORDINATES n type + values
// followed by POINT_DATA n or CELL_DATA n and one SCALARS name type [1]
// (LOOKUP_TABLE line) array, in ASCII or BINARY (big-endian) encoding. Scalar
// types: bit is not supported; char ... double are widened or narrowed to
// float32. Host code only; the result feeds beams_set_volume (and, for a
// rectilinear grid, beams_set_volume_coordinates).
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/beams_b200.h"
#include "renderer.h"

using beams::fail;

namespace {

struct VtkReader {
  std::vector<unsigned char> buf;
  size_t pos = 0;
  bool binary = false;
  std::string err;

  bool eof() const { return pos >= buf.size(); }
  void skip_space() {
    while (!eof() && std::isspace(buf[pos])) ++pos;
  }
  std::string line() {  // the rest of the current line, without the newline
    std::string s;
    while (!eof() && buf[pos] != '\n') s.push_back((char)buf[pos++]);
    if (!eof()) ++pos;
    if (!s.empty() && s.back() == '\r') s.pop_back();
    return s;
  }
  std::string token() {
    skip_space();
    std::string s;
    while (!eof() && !std::isspace(buf[pos])) s.push_back((char)buf[pos++]);
    return s;
  }
  bool number(double& v) {
    const std::string t = token();
    if (t.empty()) return false;
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    return end && *end == '\0';
  }
  bool integer(long long& v) {
    double d;
    if (!number(d) || d != std::floor(d)) return false;
    v = (long long)d;
    return true;
  }
  static int type_size(const std::string& t) {
    if (t == "char" || t == "unsigned_char") return 1;
    if (t == "short" || t == "unsigned_short") return 2;
    if (t == "int" || t == "unsigned_int" || t == "float") return 4;
    if (t == "long" || t == "unsigned_long" || t == "double" || t == "vtkIdType") return 8;
    return 0;
  }
  // n values of VTK type t, as float32
  bool values(const std::string& t, size_t n, float* out) {
    const int sz = type_size(t);
    if (!sz) {
      err = "unsupported data type '" + t + "'";
      return false;
    }
    if (!binary) {
      for (size_t i = 0; i < n; ++i) {
        double v;
        if (!number(v)) {
          err = "expected " + std::to_string(n) + " ASCII values";
          return false;
        }
        out[i] = (float)v;
      }
      return true;
    }
    // binary: the values start after the end of the keyword line
    if (buf.size() - pos < n * (size_t)sz) {
      err = "binary data shorter than its header says";
      return false;
    }
    for (size_t i = 0; i < n; ++i) {
      unsigned char b[8];
      for (int k = 0; k < sz; ++k) b[k] = buf[pos + i * sz + (sz - 1 - k)];  // big-endian -> host order
      double v;
      if (t == "char") v = (double)(int8_t)b[0];
      else if (t == "unsigned_char") v = (double)b[0];
      else if (t == "short") { int16_t x; std::memcpy(&x, b, 2); v = x; }
      else if (t == "unsigned_short") { uint16_t x; std::memcpy(&x, b, 2); v = x; }
      else if (t == "int") { int32_t x; std::memcpy(&x, b, 4); v = x; }
      else if (t == "unsigned_int") { uint32_t x; std::memcpy(&x, b, 4); v = x; }
      else if (t == "float") { float x; std::memcpy(&x, b, 4); out[i] = x; continue; }
      else if (t == "double") { double x; std::memcpy(&x, b, 8); v = x; }
      else if (t == "unsigned_long") { uint64_t x; std::memcpy(&x, b, 8); v = (double)x; }
      else { int64_t x; std::memcpy(&x, b, 8); v = (double)x; }
      out[i] = (float)v;
    }
    pos += n * (size_t)sz;
    return true;
  }
};

bool upper_eq(const std::string& a, const char* b) {
  if (a.size() != std::strlen(b)) return false;
  for (size_t i = 0; i < a.size(); ++i)
    if (std::toupper((unsigned char)a[i]) != b[i]) return false;
  return true;
}

}  // namespace

extern "C" beams_status beams_vtk_read(const char* path, beams_vtk_field* out) {
  if (!path || !out) return fail(nullptr, BEAMS_ERR_INVALID_ARG, "vtk_read: NULL argument");
  std::memset(out, 0, sizeof(*out));
  FILE* f = std::fopen(path, "rb");
  if (!f) return fail(nullptr, BEAMS_ERR_INVALID_ARG, std::string("vtk_read: cannot open ") + path);
  VtkReader R;
  {
    unsigned char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0) R.buf.insert(R.buf.end(), chunk, chunk + n);
    std::fclose(f);
  }
  auto bad = [&](const std::string& m) {
    return fail(nullptr, BEAMS_ERR_CONFIG, std::string("vtk_read: ") + path + ": " + m);
  };
  const std::string l0 = R.line();
  if (l0.rfind("# vtk DataFile", 0) != 0) return bad("not a legacy VTK file (first line)");
  R.line();  // title
  const std::string enc = R.token();
  if (upper_eq(enc, "BINARY")) R.binary = true;
  else if (!upper_eq(enc, "ASCII")) return bad("encoding must be ASCII or BINARY");
  if (!upper_eq(R.token(), "DATASET")) return bad("expected DATASET");
  const std::string kind = R.token();
  const bool rect = upper_eq(kind, "RECTILINEAR_GRID");
  if (!rect && !upper_eq(kind, "STRUCTURED_POINTS")) return bad("dataset must be STRUCTURED_POINTS or RECTILINEAR_GRID");
  long long dims[3] = {0, 0, 0};
  double origin[3] = {0, 0, 0}, spacing[3] = {1, 1, 1};
  std::vector<float> coords[3];
  bool have_dims = false;
  std::string assoc;
  long long count = 0;
  for (;;) {
    const std::string kw = R.token();
    if (kw.empty()) return bad("no POINT_DATA or CELL_DATA section");
    if (upper_eq(kw, "DIMENSIONS")) {
      for (auto& d : dims)
        if (!R.integer(d) || d < 1 || d > 8192) return bad("bad DIMENSIONS");
      have_dims = true;
    } else if (upper_eq(kw, "ORIGIN")) {
      for (auto& o : origin)
        if (!R.number(o)) return bad("bad ORIGIN");
    } else if (upper_eq(kw, "SPACING") || upper_eq(kw, "ASPECT_RATIO")) {
      for (auto& h : spacing)
        if (!R.number(h) || !(h > 0)) return bad("bad SPACING");
    } else if (rect && (upper_eq(kw, "X_COORDINATES") || upper_eq(kw, "Y_COORDINATES") ||
                        upper_eq(kw, "Z_COORDINATES"))) {
      const int ax = std::toupper((unsigned char)kw[0]) - 'X';
      long long n;
      if (!R.integer(n) || !have_dims || n != dims[ax]) return bad("coordinate count differs from DIMENSIONS");
      const std::string t = R.token();
      R.line();
      coords[ax].resize((size_t)n);
      if (!R.values(t, (size_t)n, coords[ax].data())) return bad(R.err);
    } else if (upper_eq(kw, "POINT_DATA") || upper_eq(kw, "CELL_DATA")) {
      assoc = kw;
      if (!R.integer(count)) return bad("bad data count");
      break;
    } else if (upper_eq(kw, "FIELD")) {
      return bad("FIELD data before the scalars is not supported");
    } else {
      return bad("unexpected keyword '" + kw + "'");
    }
  }
  if (!have_dims) return bad("no DIMENSIONS");
  const bool cells = upper_eq(assoc, "CELL_DATA");
  for (int d = 0; d < 3; ++d) {
    if (cells && dims[d] < 2) return bad("cell data needs at least 2 points per axis");
    if (!cells && dims[d] < 2) return bad("a volume needs at least 2 points per axis");
    if (rect && coords[d].empty()) return bad("missing X/Y/Z_COORDINATES");
    for (size_t i = 1; i < coords[d].size(); ++i)
      if (!(coords[d][i] > coords[d][i - 1])) return bad("coordinates must be strictly increasing");
  }
  const long long want = cells ? (dims[0] - 1) * (dims[1] - 1) * (dims[2] - 1) : dims[0] * dims[1] * dims[2];
  if (count != want) return bad("data count differs from the grid");
  // the first SCALARS array
  for (;;) {
    const std::string kw = R.token();
    if (kw.empty()) return bad("no SCALARS array");
    if (upper_eq(kw, "SCALARS")) break;
    return bad("expected SCALARS, found '" + kw + "'");
  }
  const std::string name = R.token();
  const std::string t = R.token();
  std::string rest = R.line();  // optional component count
  if (!rest.empty() && std::atoi(rest.c_str()) > 1) return bad("only one-component scalars are supported");
  const size_t save = R.pos;
  if (upper_eq(R.token(), "LOOKUP_TABLE")) {
    R.line();
  } else {
    R.pos = save;
  }
  float* data = (float*)std::malloc((size_t)want * sizeof(float));
  if (!data) return fail(nullptr, BEAMS_ERR_OOM, "vtk_read: out of host memory");
  if (!R.values(t, (size_t)want, data)) {
    std::free(data);
    return bad(R.err);
  }
  double lo = INFINITY, hi = -INFINITY;
  for (long long i = 0; i < want; ++i) {
    if (data[i] < lo) lo = data[i];
    if (data[i] > hi) hi = data[i];
  }
  for (int d = 0; d < 3; ++d) {
    out->dims[d] = (int)dims[d];
    out->origin[d] = rect ? coords[d][0] : origin[d];
    out->spacing[d] = rect ? (coords[d].back() - coords[d][0]) / (double)(dims[d] - 1) : spacing[d];
    if (rect) {
      out->coords[d] = (float*)std::malloc(coords[d].size() * sizeof(float));
      if (!out->coords[d]) {
        beams_vtk_free(out);
        std::free(data);
        return fail(nullptr, BEAMS_ERR_OOM, "vtk_read: out of host memory");
      }
      std::memcpy(out->coords[d], coords[d].data(), coords[d].size() * sizeof(float));
    }
  }
  out->assoc = cells ? BEAMS_ASSOC_CELLS : BEAMS_ASSOC_POINTS;
  out->data = data;
  out->range[0] = lo;
  out->range[1] = hi;
  std::snprintf(out->name, sizeof(out->name), "%s", name.c_str());
  return BEAMS_OK;
}

extern "C" void beams_vtk_free(beams_vtk_field* f) {
  if (!f) return;
  std::free(f->data);
  for (auto& c : f->coords) std::free(c);
  std::memset(f, 0, sizeof(*f));
}

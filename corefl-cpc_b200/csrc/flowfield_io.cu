// Tecplot V112 binary flowfield files (host code): the writer of the
// reference's FieldIO (reference src/FieldIO.h:83-420: header, then per block
// the zone record, min/max pairs and double-precision node data) and the
// same-mesh branch of its restart reader (reference src/Initialize.cu:97-345,
// variable labels src/Initialize.cu:346-400).  The byte layout has to be the
// reference's so that files written here open in Tecplot and restart the
// reference, and files from the reference restart this library.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "corefl_b200.h"

namespace {

struct Writer {
  std::vector<unsigned char> buf;
  template <class T> void put(T v) {
    const size_t n = buf.size();
    buf.resize(n + sizeof(T));
    std::memcpy(buf.data() + n, &v, sizeof(T));
  }
  // Tecplot string: one int32 per character, then a zero int32.
  void str(const std::string &s) {
    for (unsigned char ch : s) put<int32_t>(static_cast<int32_t>(static_cast<char>(ch)));
    put<int32_t>(0);
  }
};

int report(char *err, size_t len, const std::string &msg, int code) {
  if (err && len) std::snprintf(err, len, "%s", msg.c_str());
  return code;
}

// Index of node (i, j, k) in a padded array of ghost width g.
inline int64_t pidx(int mx, int my, int g, int i, int j, int k) {
  return ((int64_t)(k + g) * (my + 2 * g) + (j + g)) * (mx + 2 * g) + (i + g);
}

int64_t plane_size(int mx, int my, int mz, int g) { return (int64_t)(mx + 2 * g) * (my + 2 * g) * (mz + 2 * g); }

}  // namespace

extern "C" int cfk_write_flowfield(const char *path, const cfk_plt_block *blocks, int n_block, int ngg_output,
                                   const char *const *var_names, int n_scalar, int n_other, double solution_time,
                                   char *err, size_t err_len) {
  if (!path || !blocks || n_block < 1 || !var_names || n_scalar < 0 || n_other < 0 || ngg_output < 0)
    return report(err, err_len, "bad argument", CFK_ERR_ARG);
  const int n_var = 9 + n_scalar + n_other;
  for (int l = 0; l < n_var; ++l)
    if (!var_names[l]) return report(err, err_len, "a variable name is NULL", CFK_ERR_ARG);
  for (int b = 0; b < n_block; ++b) {
    const cfk_plt_block &B = blocks[b];
    if (B.mx < 1 || B.my < 1 || B.mz < 1 || B.ngg < ngg_output)
      return report(err, err_len, "block " + std::to_string(b) + ": sizes, or ngg below ngg_output", CFK_ERR_ARG);
    if (!B.x || !B.y || !B.z || !B.bv || (n_scalar && !B.sv) || (n_other && !B.ov))
      return report(err, err_len, "block " + std::to_string(b) + ": missing array", CFK_ERR_ARG);
  }
  Writer w;
  // I. header: magic number, byte order, file type 0 (full), title, variables
  for (const char *m = "#!TDV112"; *m; ++m) w.put<char>(*m);
  w.put<int32_t>(1);
  w.put<int32_t>(0);
  w.str("Solution file");
  w.put<int32_t>(n_var);
  for (int l = 0; l < n_var; ++l) w.str(var_names[l]);
  const int g = ngg_output;
  for (int b = 0; b < n_block; ++b) {
    w.put<float>(299.0f);                    // zone marker
    w.str("zone " + std::to_string(b));
    w.put<int32_t>(-1);                      // parent zone
    w.put<int32_t>(-2);                      // strand id: assigned by Tecplot
    w.put<double>(solution_time);
    w.put<int32_t>(-1);                      // zone colour
    w.put<int32_t>(0);                       // ordered zone
    w.put<int32_t>(0);                       // data at the nodes
    w.put<int32_t>(0);                       // no raw face neighbours
    w.put<int32_t>(0);                       // no user face connections
    w.put<int32_t>(blocks[b].mx + 2 * g);
    w.put<int32_t>(blocks[b].my + 2 * g);
    w.put<int32_t>(blocks[b].mz + 2 * g);
    w.put<int32_t>(0);                       // no auxiliary data
  }
  w.put<float>(357.0f);                      // end of header
  // II. data: per block the zone record, min/max of every variable, then the
  // variables over the nodes widened by ngg_output, i fastest.
  for (int b = 0; b < n_block; ++b) {
    const cfk_plt_block &B = blocks[b];
    const int64_t P = plane_size(B.mx, B.my, B.mz, B.ngg);
    std::vector<const double *> vars = {B.x, B.y, B.z};
    for (int l = 0; l < 6; ++l) vars.push_back(B.bv + l * P);
    for (int l = 0; l < n_scalar; ++l) vars.push_back(B.sv + l * P);
    for (int l = 0; l < n_other; ++l) vars.push_back(B.ov + l * P);
    w.put<float>(299.0f);
    for (int l = 0; l < n_var; ++l) w.put<int32_t>(2);  // double precision
    w.put<int32_t>(0);                                  // no passive variables
    w.put<int32_t>(0);                                  // no variable sharing
    w.put<int32_t>(-1);                                 // no connectivity sharing
    for (const double *v : vars) {
      double lo = v[pidx(B.mx, B.my, B.ngg, -g, -g, -g)], hi = lo;
      for (int k = -g; k < B.mz + g; ++k)
        for (int j = -g; j < B.my + g; ++j)
          for (int i = -g; i < B.mx + g; ++i) {
            const double x = v[pidx(B.mx, B.my, B.ngg, i, j, k)];
            lo = std::min(lo, x);
            hi = std::max(hi, x);
          }
      w.put<double>(lo);
      w.put<double>(hi);
    }
    for (const double *v : vars)
      for (int k = -g; k < B.mz + g; ++k)
        for (int j = -g; j < B.my + g; ++j)
          for (int i = -g; i < B.mx + g; ++i) w.put<double>(v[pidx(B.mx, B.my, B.ngg, i, j, k)]);
  }
  FILE *f = std::fopen(path, "wb");
  if (!f) return report(err, err_len, std::string("cannot open ") + path + " for writing", CFK_ERR_IO);
  const size_t n = std::fwrite(w.buf.data(), 1, w.buf.size(), f);
  const bool ok = n == w.buf.size() && std::fclose(f) == 0;
  if (!ok) return report(err, err_len, std::string("short write to ") + path, CFK_ERR_IO);
  return CFK_OK;
}

namespace {

struct Reader {
  const std::vector<unsigned char> &buf;
  size_t at = 0;
  bool ok = true;
  template <class T> T get() {
    T v{};
    if (at + sizeof(T) > buf.size()) { ok = false; return v; }
    std::memcpy(&v, buf.data() + at, sizeof(T));
    at += sizeof(T);
    return v;
  }
  std::string str() {
    std::string s;
    for (;;) {
      const int32_t c = get<int32_t>();
      if (!ok || static_cast<char>(c) == '\0') break;
      s += static_cast<char>(c);
    }
    return s;
  }
  void skip(size_t n) {
    if (at + n > buf.size()) ok = false;
    else at += n;
  }
};

std::string upper(std::string s) {
  for (char &c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
  return s;
}

// Variable label of a name, as the reference's identify_variable_labels:
// 0..5 the basic variables, 6 + l species l, -1 anything else.
int label_of(const std::string &name, const char *const *species, int n_spec) {
  const std::string n = upper(name);
  if (n == "DENSITY" || n == "ROE" || n == "RHO") return 0;
  if (n == "U") return 1;
  if (n == "V") return 2;
  if (n == "W") return 3;
  if (n == "P" || n == "PRESSURE") return 4;
  if (n == "T" || n == "TEMPERATURE") return 5;
  for (int l = 0; l < n_spec; ++l)
    if (species && species[l] && n == upper(species[l])) return 6 + l;
  return -1;
}

}  // namespace

extern "C" int cfk_read_flowfield(const char *path, const cfk_plt_target *blocks, int n_block,
                                  const char *const *species_names, int n_spec, double *solution_time, char *err,
                                  size_t err_len) {
  if (!path || !blocks || n_block < 1 || n_spec < 0) return report(err, err_len, "bad argument", CFK_ERR_ARG);
  FILE *f = std::fopen(path, "rb");
  if (!f) return report(err, err_len, std::string("cannot open ") + path, CFK_ERR_IO);
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  for (size_t n; (n = std::fread(chunk, 1, sizeof chunk, f)) > 0;) buf.insert(buf.end(), chunk, chunk + n);
  std::fclose(f);
  Reader r{buf};
  if (buf.size() < 16 || std::memcmp(buf.data(), "#!TDV1", 6) != 0)
    return report(err, err_len, "not a Tecplot binary file", CFK_ERR_IO);
  r.skip(16);  // magic number, byte order, file type
  r.str();     // title
  const int32_t n_var = r.get<int32_t>();
  if (!r.ok || n_var < 3 || n_var > 4096) return report(err, err_len, "bad variable count", CFK_ERR_IO);
  std::vector<int> label(n_var);
  for (int l = 0; l < n_var; ++l) label[l] = label_of(r.str(), species_names, n_spec);
  for (int l = 0; l < 3; ++l) label[l] = -1;  // x, y, z
  std::vector<int> dims;
  double t = 0;
  for (float marker = r.get<float>(); r.ok && std::fabs(marker - 299.0f) < 1e-3f; marker = r.get<float>()) {
    r.str();      // zone name
    r.skip(8);    // parent zone, strand id
    t = r.get<double>();
    r.skip(20);   // colour, zone type, location, face neighbours, user connections
    for (int a = 0; a < 3; ++a) dims.push_back(r.get<int32_t>());
    r.skip(4);    // auxiliary data flag
  }
  if (!r.ok) return report(err, err_len, "truncated header", CFK_ERR_IO);
  const int n_zone = static_cast<int>(dims.size() / 3);
  if (n_zone != n_block)
    return report(err, err_len, "file has " + std::to_string(n_zone) + " zones, " + std::to_string(n_block) +
                                    " blocks given", CFK_ERR_ARG);
  std::vector<int> g_file(n_block);
  for (int b = 0; b < n_block; ++b) {
    const cfk_plt_target &B = blocks[b];
    const int m[3] = {B.mx, B.my, B.mz};
    const int d0 = dims[3 * b] - m[0];
    bool fits = d0 >= 0 && d0 % 2 == 0 && d0 / 2 <= B.ngg;
    for (int a = 1; a < 3; ++a) fits = fits && dims[3 * b + a] - m[a] == d0;
    if (!fits)
      return report(err, err_len, "zone " + std::to_string(b) + " does not match block " + std::to_string(b) +
                                      " (same mesh, same block order, at most ngg ghost layers)", CFK_ERR_ARG);
    g_file[b] = d0 / 2;
    for (int l = 0; l < n_var; ++l)
      if ((label[l] >= 0 && label[l] < 6 && !B.bv) || (label[l] >= 6 && !B.sv))
        return report(err, err_len, "block " + std::to_string(b) + ": bv/sv array missing", CFK_ERR_ARG);
  }
  for (int b = 0; b < n_block; ++b) {
    const cfk_plt_target &B = blocks[b];
    const int g = g_file[b];
    const int64_t P = plane_size(B.mx, B.my, B.mz, B.ngg);
    const int64_t N = (int64_t)dims[3 * b] * dims[3 * b + 1] * dims[3 * b + 2];
    r.skip(4 + 4 * (size_t)n_var + 12 + 16 * (size_t)n_var);  // zone record, formats, flags, min/max pairs
    for (int l = 0; l < n_var; ++l) {
      if (label[l] < 0) { r.skip((size_t)N * 8); continue; }
      double *dst = label[l] < 6 ? B.bv + label[l] * P : B.sv + (label[l] - 6) * P;
      for (int k = -g; k < B.mz + g; ++k)
        for (int j = -g; j < B.my + g; ++j)
          for (int i = -g; i < B.mx + g; ++i) dst[pidx(B.mx, B.my, B.ngg, i, j, k)] = r.get<double>();
    }
    if (!r.ok) return report(err, err_len, "truncated data of zone " + std::to_string(b), CFK_ERR_IO);
  }
  if (solution_time) *solution_time = t;
  return CFK_OK;
}

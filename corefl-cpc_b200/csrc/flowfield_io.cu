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

// Appends one variable's node window (nodes widened by g, i fastest) to f,
// one contiguous i-row per fwrite.
bool write_window(FILE *f, const double *v, const cfk_plt_block &B, int g) {
  const size_t row = (size_t)(B.mx + 2 * g);
  for (int k = -g; k < B.mz + g; ++k)
    for (int j = -g; j < B.my + g; ++j)
      if (std::fwrite(v + pidx(B.mx, B.my, B.ngg, -g, j, k), sizeof(double), row, f) != row) return false;
  return true;
}

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
  FILE *f = std::fopen(path, "wb");
  if (!f) return report(err, err_len, std::string("cannot open ") + path + " for writing", CFK_ERR_IO);
  bool ok = std::fwrite(w.buf.data(), 1, w.buf.size(), f) == w.buf.size();
  // II. data: per block the zone record, min/max of every variable, then the
  // variables over the nodes widened by ngg_output, i fastest — streamed
  // row by row, so no copy of the field is held in memory.
  for (int b = 0; ok && b < n_block; ++b) {
    const cfk_plt_block &B = blocks[b];
    const int64_t P = plane_size(B.mx, B.my, B.mz, B.ngg);
    std::vector<const double *> vars = {B.x, B.y, B.z};
    for (int l = 0; l < 6; ++l) vars.push_back(B.bv + l * P);
    for (int l = 0; l < n_scalar; ++l) vars.push_back(B.sv + l * P);
    for (int l = 0; l < n_other; ++l) vars.push_back(B.ov + l * P);
    Writer z;
    z.put<float>(299.0f);
    for (int l = 0; l < n_var; ++l) z.put<int32_t>(2);  // double precision
    z.put<int32_t>(0);                                  // no passive variables
    z.put<int32_t>(0);                                  // no variable sharing
    z.put<int32_t>(-1);                                 // no connectivity sharing
    for (const double *v : vars) {
      double lo = v[pidx(B.mx, B.my, B.ngg, -g, -g, -g)], hi = lo;
      for (int k = -g; k < B.mz + g; ++k)
        for (int j = -g; j < B.my + g; ++j)
          for (int i = -g; i < B.mx + g; ++i) {
            const double x = v[pidx(B.mx, B.my, B.ngg, i, j, k)];
            lo = std::min(lo, x);
            hi = std::max(hi, x);
          }
      z.put<double>(lo);
      z.put<double>(hi);
    }
    ok = std::fwrite(z.buf.data(), 1, z.buf.size(), f) == z.buf.size();
    for (size_t l = 0; ok && l < vars.size(); ++l) ok = write_window(f, vars[l], B, g);
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return report(err, err_len, std::string("short write to ") + path, CFK_ERR_IO);
  return CFK_OK;
}

namespace {

// Sequential reads from a FILE*; any short read clears ok.
struct Reader {
  FILE *f;
  bool ok = true;
  template <class T> T get() {
    T v{};
    if (std::fread(&v, sizeof(T), 1, f) != 1) ok = false;
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
  void skip(int64_t n) {
    if (ok && std::fseek(f, (long)n, SEEK_CUR) != 0) ok = false;
  }
  void read(double *dst, size_t n) {
    if (ok && std::fread(dst, sizeof(double), n, f) != n) ok = false;
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
  struct Closer { FILE *f; ~Closer() { std::fclose(f); } } closer{f};
  Reader r{f};
  char magic[8] = {0};
  if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "#!TDV1", 6) != 0)
    return report(err, err_len, "not a Tecplot binary file", CFK_ERR_IO);
  r.skip(8);   // byte order, file type
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
    r.skip(4 + 4 * (int64_t)n_var + 12 + 16 * (int64_t)n_var);  // zone record, formats, flags, min/max pairs
    const size_t row = (size_t)(B.mx + 2 * g);
    for (int l = 0; r.ok && l < n_var; ++l) {
      if (label[l] < 0) { r.skip(N * 8); continue; }
      double *dst = label[l] < 6 ? B.bv + label[l] * P : B.sv + (label[l] - 6) * P;
      for (int k = -g; k < B.mz + g; ++k)
        for (int j = -g; j < B.my + g; ++j) r.read(dst + pidx(B.mx, B.my, B.ngg, -g, j, k), row);
    }
    if (!r.ok) return report(err, err_len, "truncated data of zone " + std::to_string(b), CFK_ERR_IO);
  }
  // fseek past the end of the file succeeds, so a file cut inside the
  // skipped variables of the last zone shows only here
  const long end_of_data = std::ftell(f);
  if (end_of_data < 0 || std::fseek(f, 0, SEEK_END) != 0 || std::ftell(f) < end_of_data)
    return report(err, err_len, "truncated data of zone " + std::to_string(n_block - 1), CFK_ERR_IO);
  if (solution_time) *solution_time = t;
  return CFK_OK;
}

// Inner-face registration (host code): the 0-based loop description of a face
// shared by two blocks, built from the 1-based, sign-coded node ranges of the
// mesh's inner-interface records as InnerFace::register_boundary does
// (reference src/Mesh.cpp:39-172).  The steps have to give the reference's
// numbers exactly, since the communication kernel walks them.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "corefl_b200.h"

namespace {

int sign_of(int a) { return (a > 0) - (a < 0); }

// One side of the record: start/end per axis, its normal axis and side.
struct Side {
  int s[3], e[3];
  int normal = -1, side = 1;
};

// Finds the normal axis (equal ends; the value 1 marks the min side) and
// makes it 0-based.
bool take_normal(int dim, const int r[6], Side &x) {
  for (int a = 0; a < 3; ++a) { x.s[a] = r[2 * a]; x.e[a] = r[2 * a + 1]; }
  for (int a = 0; a < dim; ++a) {
    if (x.s[a] != x.e[a]) continue;
    x.normal = a;
    x.side = x.s[a] == 1 ? -1 : 1;
    --x.s[a];
    --x.e[a];
    return true;
  }
  return false;
}

// 3-D: the first axis with negated values is the first tangential axis.
int take_marked(int dim, Side &x) {
  for (int a = 0; a < dim; ++a) {
    if (x.s[a] >= 0) continue;
    x.s[a] = -x.s[a] - 1;
    x.e[a] = -x.e[a] - 1;
    return a;
  }
  return -1;
}

}  // namespace

extern "C" int cfk_register_inner_face(int dim, int ngg, const int src[6], const int tar[6], int target_block,
                                       cfk_inner_face *out) {
  if (!src || !tar || !out || (dim != 2 && dim != 3) || ngg < 0) return CFK_ERR_ARG;
  Side me, it;
  if (!take_normal(dim, src, me) || !take_normal(dim, tar, it)) return CFK_ERR_ARG;
  int map[3] = {0, 0, 0};  // signed, 1-based source axis of each target axis
  map[it.normal] = -(me.side * it.side) * (me.normal + 1);
  // pairs one tangential axis of this block with one of the target block
  auto pair = [&](int a, int ta) {
    map[ta] = sign_of((it.e[ta] - it.s[ta]) * (me.e[a] - me.s[a])) * (a + 1);
  };
  if (dim == 2) {
    const int a = 1 - me.normal, ta = 1 - it.normal;
    me.s[a] = std::abs(me.s[a]) - 1;
    me.e[a] = std::abs(me.e[a]) - 1;
    it.s[ta] = std::abs(it.s[ta]) - 1;
    it.e[ta] = std::abs(it.e[ta]) - 1;
    pair(a, ta);
    map[2] = 3;
    me.s[2] = me.e[2] = it.s[2] = it.e[2] = 0;
  } else {
    int a = take_marked(dim, me), ta = take_marked(dim, it);
    if (a < 0 || ta < 0) return CFK_ERR_ARG;
    pair(a, ta);
    a = 3 - me.normal - a;
    ta = 3 - it.normal - ta;
    --me.s[a];
    --me.e[a];
    --it.s[ta];
    --it.e[ta];
    pair(a, ta);
  }
  // Along the normal the loop covers the face node and the ngg ghost layers
  // behind it; the target's start is the node that pairs with the loop's
  // first one.
  const int f = me.normal, tf = it.normal;
  const int face_end = me.e[f];
  me.s[f] = me.side < 0 ? -ngg : face_end;
  me.e[f] = me.side < 0 ? 0 : face_end + ngg;
  const bool same_sense = sign_of(map[tf]) > 0;
  if (it.side > 0) it.s[tf] = same_sense ? it.e[tf] - ngg : it.e[tf];
  else it.s[tf] = same_sense ? 0 : ngg;

  cfk_inner_face r{};
  for (int a = 0; a < 3; ++a) {
    r.range_start[a] = me.s[a];
    r.range_end[a] = me.e[a];
    r.target_start[a] = it.s[a];
    r.target_end[a] = it.e[a];
    r.loop_dir[a] = me.s[a] <= me.e[a] ? 1 : -1;
    r.target_loop_dir[a] = sign_of(map[a]);
    r.src_tar[a] = std::abs(map[a]) - 1;
    r.n_point[a] = std::abs(me.s[a] - me.e[a]) + 1;
  }
  r.face = f;
  r.direction = me.side;
  r.target_face = tf;
  r.target_direction = it.side;
  r.target_block = target_block - 1;
  *out = r;
  return CFK_OK;
}

// The mesh's inner-interface file (reference src/Mesh.cpp:927-958,
// Mesh::read_inner_interface): a title line; the number of inner faces of
// each block; a second title line; then per block, per face, two lines of
// seven integers — this block's range and the target's range followed by the
// target block's 1-based number (the first line's seventh integer is not
// used).  Faces are registered in file order.
extern "C" int cfk_read_inner_interface(const char *path, int dim, int ngg, int n_block, cfk_inner_face *faces,
                                        int max_faces, int *n_per_block, char *err, size_t err_len) {
  auto fail = [&](const std::string &m, int code) {
    if (err && err_len) std::snprintf(err, err_len, "%s", m.c_str());
    return code;
  };
  if (!path || n_block < 1 || !n_per_block || (max_faces > 0 && !faces)) return fail("bad argument", CFK_ERR_ARG);
  std::ifstream in(path);
  if (!in) return fail(std::string("cannot open ") + path, CFK_ERR_IO);
  std::string line;
  std::getline(in, line);
  std::vector<int> count(n_block);
  for (int b = 0; b < n_block; ++b)
    if (!(in >> count[b]) || count[b] < 0) return fail("bad face count of block " + std::to_string(b), CFK_ERR_IO);
  std::getline(in, line);  // rest of the counts line
  std::getline(in, line);  // second title line
  int n = 0;
  for (int b = 0; b < n_block; ++b) {
    for (int l = 0; l < count[b]; ++l) {
      int a[7], t[7];
      for (int *rec : {a, t}) {
        if (!std::getline(in, line)) return fail("file ends inside block " + std::to_string(b), CFK_ERR_IO);
        std::istringstream ls(line);
        for (int q = 0; q < 7; ++q)
          if (!(ls >> rec[q])) return fail("short record in block " + std::to_string(b), CFK_ERR_IO);
      }
      if (n >= max_faces) return fail("more than max_faces inner faces", CFK_ERR_ARG);
      if (cfk_register_inner_face(dim, ngg, a, t, t[6], &faces[n]) != CFK_OK)
        return fail("block " + std::to_string(b) + " face " + std::to_string(l) + ": record cannot be decoded",
                    CFK_ERR_IO);
      ++n;
    }
    n_per_block[b] = count[b];
  }
  return CFK_OK;
}
